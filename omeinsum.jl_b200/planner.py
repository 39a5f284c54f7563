"""Contraction-order planning on the host: a greedy order, a greedy slicer and
the complexity measures the reference re-exports from OMEinsumContractionOrders
(src/contractionorder.jl:30-51).

OMEinsumContractionOrders (compat 1.1, not vendored with the reference) is an
external package; this module restates the published greedy method
(repeatedly contract the pair of tensors that share a label and minimise
size(result) - alpha * (size(a) + size(b)), ties broken at random from a seeded
generator, best of `nrepeat` runs by time complexity) and a greedy slicer
(repeatedly slice the label that most reduces the largest intermediate until
it fits 2^sc_target elements).  Orders are not expected to equal the Julia
package's; values are order-independent up to rounding.
"""
from __future__ import annotations

import json
import math
from dataclasses import dataclass
from typing import Any, Dict, List, Sequence, Tuple

import numpy as np

from ._lib import ArgumentError
from .core import AbstractEinsum, EinCode, NestedEinsum, SlicedEinsum


@dataclass
class GreedyMethod:
    """Greedy pairwise contraction order (α = 0: minimise the result size)."""

    alpha: float = 0.0
    temperature: float = 0.0
    nrepeat: int = 10
    seed: int = 0


@dataclass
class GreedySlicer:
    """Greedy slicer: slice labels until the largest intermediate has at most
    2^sc_target elements (stand-in for TreeSASlicer(score=ScoreFunction(sc_target)))."""

    sc_target: float = 27.0


def _log2sz(labels, log2sd) -> float:
    return float(sum(log2sd[l] for l in labels))


def _greedy_once(ixs: List[List[Any]], iy: List[Any], log2sd: Dict[Any, float], rng, alpha, temperature):
    """One greedy pass; returns a list of (i, j) merges over tensor slots."""
    n = len(ixs)
    tensors: Dict[int, Tuple[Any, ...]] = {i: tuple(dict.fromkeys(ix)) for i, ix in enumerate(ixs)}
    where: Dict[Any, set] = {}
    for i, ix in tensors.items():
        for l in ix:
            where.setdefault(l, set()).add(i)
    out = set(iy)
    nodes: Dict[int, Any] = {i: i for i in range(n)}  # slot -> tree (leaf index or tuple)
    labels_of: Dict[int, Tuple[Any, ...]] = dict(tensors)
    next_id = n

    def result_labels(a, b):
        la, lb = labels_of[a], labels_of[b]
        res = []
        for l in la + tuple(x for x in lb if x not in la):
            others = where[l] - {a, b}
            if l in out or others:
                res.append(l)
        return tuple(res)

    def cost(a, b):
        r = result_labels(a, b)
        sr = 2.0 ** _log2sz(r, log2sd)
        sa = 2.0 ** _log2sz(labels_of[a], log2sd)
        sb = 2.0 ** _log2sz(labels_of[b], log2sd)
        return sr - alpha * (sa + sb)

    while len(labels_of) > 1:
        cand = set()
        for l, ts in where.items():
            ts = sorted(ts)
            for x in range(len(ts)):
                for y in range(x + 1, len(ts)):
                    cand.add((ts[x], ts[y]))
        if not cand:
            ks = sorted(labels_of, key=lambda k: _log2sz(labels_of[k], log2sd))
            cand = {(min(ks[0], ks[1]), max(ks[0], ks[1]))}
        cand = sorted(cand)
        costs = np.array([cost(a, b) for a, b in cand])
        if temperature > 0:
            w = np.exp(-(costs - costs.min()) / (temperature * max(abs(costs.min()), 1.0)))
            k = rng.choice(len(cand), p=w / w.sum())
        else:
            best = np.flatnonzero(costs == costs.min())
            k = int(rng.choice(best))
        a, b = cand[k]
        r = result_labels(a, b)
        nid = next_id
        next_id += 1
        nodes[nid] = (nodes.pop(a), nodes.pop(b), labels_of[a], labels_of[b], r)
        for l in labels_of[a]:
            where[l].discard(a)
        for l in labels_of[b]:
            where[l].discard(b)
        del labels_of[a]
        del labels_of[b]
        labels_of[nid] = r
        for l in r:
            where.setdefault(l, set()).add(nid)
        for l in list(where):
            if not where[l]:
                del where[l]
    (root_slot,) = labels_of.keys()
    return nodes[root_slot], labels_of[root_slot]


def _to_nested(t, iy) -> NestedEinsum:
    """Build a NestedEinsum from the greedy merge tree; the root contracts to iy."""
    if isinstance(t, int):
        raise ValueError("single leaf")

    def rec(t, out):
        a, b, la, lb, _ = t
        args, ixs = [], []
        for sub, lab in ((a, la), (b, lb)):
            if isinstance(sub, int):
                args.append(NestedEinsum(sub))
            else:
                args.append(rec(sub, lab))
            ixs.append(tuple(lab))
        return NestedEinsum(args, EinCode(ixs, tuple(out)))

    return rec(t, iy)


def tree_complexity(ne: NestedEinsum, size_dict) -> Tuple[float, float, float]:
    """(tc, sc, rwc) in log2 (OMEinsumContractionOrders ``contraction_complexity``)."""
    tc = sc = rw = 0.0
    lg = lambda ls: float(np.prod([size_dict[l] for l in ls], dtype=np.float64)) if ls else 1.0

    def rec(n: NestedEinsum):
        nonlocal tc, sc, rw
        for a in n.args:
            if not a.isleaf:
                rec(a)
        labs = list(dict.fromkeys([l for ix in n.eins.ixs for l in ix] + list(n.eins.iy)))
        tc += lg(labs)
        sc = max(sc, lg(n.eins.iy))
        rw += lg(n.eins.iy) + sum(lg(ix) for ix in n.eins.ixs)

    rec(ne)
    return math.log2(tc), math.log2(sc) if sc > 0 else 0.0, math.log2(rw)


@dataclass
class Complexity:
    tc: float
    sc: float
    rwc: float

    def __iter__(self):
        return iter((self.tc, self.sc, self.rwc))


def contraction_complexity(code: AbstractEinsum, size_dict) -> Complexity:
    """Time, space and read-write complexity (log2) of a code; for a flat
    EinCode the single n-ary contraction."""
    if isinstance(code, SlicedEinsum):
        sd = dict(size_dict)
        nsl = 1
        for l in code.slicing:
            nsl *= sd[l]
            sd[l] = 1
        tc, sc, rw = contraction_complexity(code.eins, sd)
        return Complexity(tc + math.log2(nsl), sc, rw + math.log2(nsl))
    if isinstance(code, NestedEinsum):
        return Complexity(*tree_complexity(code, size_dict))
    labs = code.uniquelabels()
    tc = sum(math.log2(size_dict[l]) for l in labs)
    sc = sum(math.log2(size_dict[l]) for l in code.iy)
    rw = math.log2(sum(float(np.prod([size_dict[l] for l in ix])) if ix else 1.0
                       for ix in list(code.ixs) + [code.iy]))
    return Complexity(tc, sc, rw)


def flop(code: AbstractEinsum, size_dict) -> int:
    """Sum over nodes of the product of all label extents of the node."""
    if isinstance(code, EinCode):
        return int(np.prod([size_dict[l] for l in code.uniquelabels()], dtype=np.float64))
    if isinstance(code, SlicedEinsum):
        sd = dict(size_dict)
        nsl = 1
        for l in code.slicing:
            nsl *= sd[l]
            sd[l] = 1
        return nsl * flop(code.eins, sd)
    total = 0

    def rec(n):
        nonlocal total
        for a in n.args:
            if not a.isleaf:
                rec(a)
        labs = list(dict.fromkeys([l for ix in n.eins.ixs for l in ix] + list(n.eins.iy)))
        total += int(np.prod([size_dict[l] for l in labs], dtype=np.float64))

    rec(code)
    return total


def peak_memory(code: AbstractEinsum, size_dict) -> int:
    """Peak elements held while evaluating the tree (inputs of the node being
    evaluated, the live intermediates and its output)."""
    if isinstance(code, SlicedEinsum):
        sd = dict(size_dict)
        for l in code.slicing:
            sd[l] = 1
        return peak_memory(code.eins, sd)
    sz = lambda ix: int(np.prod([size_dict[l] for l in ix], dtype=np.int64)) if len(ix) else 1

    def rec(n):
        cur = peak = 0
        for ix, a in zip(n.eins.ixs, n.args):
            if a.isleaf:
                cur += sz(ix)
                peak = max(peak, cur)
            else:
                p, o = rec(a)
                peak = max(peak, cur + p)
                cur += o
        peak = max(peak, cur + sz(n.eins.iy))
        return peak, sz(n.eins.iy)

    if isinstance(code, EinCode):
        return sum(sz(ix) for ix in code.ixs) + sz(code.iy)
    return rec(code)[0]


def label_elimination_order(code: AbstractEinsum) -> List[Any]:
    """Labels in the order the tree's nodes sum them out (post-order)."""
    ne = code.eins if isinstance(code, SlicedEinsum) else code
    order: List[Any] = []

    def rec(n):
        for a in n.args:
            if not a.isleaf:
                rec(a)
        for ix in n.eins.ixs:
            for l in ix:
                if l not in n.eins.iy and l not in order:
                    order.append(l)

    rec(ne)
    return order


def optimize_code(code: AbstractEinsum, size_dict: Dict[Any, int], optimizer: GreedyMethod | None = None,
                  slicer: GreedySlicer | None = None):
    """``optimize_code`` (src/contractionorder.jl:30-32): a NestedEinsum (or a
    SlicedEinsum when a slicer is given) for the flattened code."""
    optimizer = optimizer or GreedyMethod()
    flat = code if isinstance(code, EinCode) else code.flatten()
    ixs = [list(ix) for ix in flat.ixs]
    iy = list(flat.iy)
    if len(ixs) == 1:
        ne = NestedEinsum([NestedEinsum(0)], EinCode([tuple(ixs[0])], tuple(iy)))
    else:
        log2sd = {l: math.log2(max(size_dict[l], 1)) for l in flat.uniquelabels()}
        rng = np.random.default_rng(optimizer.seed)
        best = None
        for _ in range(max(1, optimizer.nrepeat)):
            t, _ = _greedy_once(ixs, iy, log2sd, rng, optimizer.alpha, optimizer.temperature)
            ne = _to_nested(t, iy)
            tc = tree_complexity(ne, size_dict)
            key = (tc[0], tc[1])
            if best is None or key < best[0]:
                best = (key, ne)
        ne = best[1]
    if slicer is not None:
        return slice_code(ne, size_dict, slicer)
    return ne


def slice_code(code: NestedEinsum, size_dict: Dict[Any, int], slicer: GreedySlicer | None = None) -> SlicedEinsum:
    """``slice_code`` (src/contractionorder.jl:33-35) with the greedy slicer."""
    slicer = slicer or GreedySlicer()
    sd = dict(size_dict)
    sliced: List[Any] = []
    labels = code.uniquelabels() if not isinstance(code, NestedEinsum) else \
        list(dict.fromkeys([l for ix in code.getixsv() for l in ix] + code.getiyv()))
    inner = []

    def collect(n):
        for a in n.args:
            if not a.isleaf:
                collect(a)
        for l in n.eins.iy:
            if l not in inner:
                inner.append(l)
        for ix in n.eins.ixs:
            for l in ix:
                if l not in inner:
                    inner.append(l)

    collect(code)
    while True:
        tc, sc, _ = tree_complexity(code, sd)
        if sc <= slicer.sc_target + 1e-9:
            break
        best = None
        for l in inner:
            if l in sliced or sd[l] <= 1:
                continue
            sd2 = dict(sd)
            sd2[l] = 1
            tc2, sc2, _ = tree_complexity(code, sd2)
            key = (sc2, tc2 + math.log2(sd[l]))
            if best is None or key < best[0]:
                best = (key, l)
        if best is None:
            break
        sliced.append(best[1])
        sd[best[1]] = 1
    return SlicedEinsum(sliced, code)


# ----------------------------------------------------------------------------
# tree files
# ----------------------------------------------------------------------------


# Contraction-tree JSON in the layout of OMEinsumContractionOrders'
# writejson/readjson, which OMEinsum re-exports (src/contractionorder.jl:48-51;
# dependency compat "1.1" in the reference's Project.toml): a top-level object
# with "label-type" ("Char" for one-character string labels, "Int64" for
# integers), "inputs" (every leaf's labels), "output", "tree" and, for a
# SlicedEinsum, "slices".  A tree node is {"isleaf": true, "tensorindex": i}
# with Julia's 1-based index, or {"isleaf": false, "args": [...], "eins":
# {"ixs": [...], "iy": [...]}}.  Files written by a Julia installation load
# here and the other way round.


def _label_type(labels) -> str:
    labels = list(labels)
    if all(isinstance(l, str) and len(l) == 1 for l in labels):
        return "Char"
    if all(isinstance(l, int) and not isinstance(l, bool) for l in labels):
        return "Int64"
    raise ArgumentError("JSON trees take one-character string labels or integer labels")


def _tree_to_obj(ne: NestedEinsum):
    if ne.isleaf:
        return {"isleaf": True, "tensorindex": ne.tensorindex + 1}
    return {"isleaf": False, "args": [_tree_to_obj(a) for a in ne.args],
            "eins": {"ixs": [list(ix) for ix in ne.eins.ixs], "iy": list(ne.eins.iy)}}


def _obj_to_tree(o, conv, base):
    if o["isleaf"]:
        return NestedEinsum(int(o["tensorindex"]) - base)
    return NestedEinsum([_obj_to_tree(a, conv, base) for a in o["args"]],
                        EinCode([tuple(conv(l) for l in ix) for ix in o["eins"]["ixs"]],
                                tuple(conv(l) for l in o["eins"]["iy"])))


def writejson(filename: str, code) -> None:
    """``writejson`` (src/contractionorder.jl:48-50): save a NestedEinsum or
    SlicedEinsum in OMEinsumContractionOrders' JSON layout."""
    ne = code.eins if isinstance(code, SlicedEinsum) else code
    ixs, iy = ne.getixsv(), list(ne.getiyv())
    labels = [l for ix in ixs for l in ix] + iy + (list(code.slicing) if isinstance(code, SlicedEinsum) else [])
    obj = {"label-type": _label_type(labels), "inputs": [list(ix) for ix in ixs], "output": iy,
           "tree": _tree_to_obj(ne)}
    if isinstance(code, SlicedEinsum):
        obj["slices"] = list(code.slicing)
    with open(filename, "w") as f:
        json.dump(obj, f)


def readjson(filename: str):
    """``readjson`` (src/contractionorder.jl:51): load a tree written by
    ``writejson`` here or by OMEinsumContractionOrders in Julia."""
    with open(filename) as f:
        obj = json.load(f)
    lt = obj.get("label-type")
    if lt is None:  # this package's earlier layout: 0-based leaves, labels as stored
        t = _obj_to_tree(obj["tree"], lambda l: l, 0)
        return t if obj.get("slices") is None else SlicedEinsum(obj["slices"], t)
    if lt == "Char":
        conv = lambda l: str(l)[0]
    elif lt.startswith("Int") or lt.startswith("UInt"):
        conv = int
    else:
        raise ArgumentError(f"label type {lt} is not supported")
    t = _obj_to_tree(obj["tree"], conv, 1)
    return t if "slices" not in obj else SlicedEinsum([conv(l) for l in obj["slices"]], t)
