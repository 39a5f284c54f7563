"""Contraction-order planning on the host: greedy and simulated-annealing
orders (native searches, ``ome_greedy`` / ``ome_treesa``), slicers and the
complexity measures the reference re-exports from OMEinsumContractionOrders
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
from dataclasses import dataclass, field
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


@dataclass
class ScoreFunction:
    """Score of a contraction order, OMEinsumContractionOrders' ScoreFunction:
    time (2^tc) plus rw_weight * read-write (2^rw), with every contraction's
    space complexity above sc_target penalised by sc_weight per unit of log2."""

    tc_weight: float = 1.0
    sc_weight: float = 1.0
    rw_weight: float = 0.0
    sc_target: float = 20.0


@dataclass
class TreeSA:
    """Simulated annealing over binary contraction trees (OMEinsumContractionOrders'
    TreeSA; the search runs natively, ``ome_treesa``).  ``betas`` = (start,
    step, stop) of the inverse temperature (Julia's 0.01:0.05:15), ``niters``
    sweeps per temperature, ``ntrials`` independent trials from the
    ``initializer`` tree ("greedy" or "random").  Space complexity above
    min(score.sc_target, the initial tree's) is penalised, so the search does
    not trade a larger peak intermediate for time."""

    betas: Tuple[float, float, float] = (0.01, 0.05, 15.0)
    ntrials: int = 10
    niters: int = 50
    initializer: str = "greedy"
    score: ScoreFunction = field(default_factory=ScoreFunction)
    seed: int = 0


@dataclass
class TreeSASlicer:
    """Slicer in the manner of OMEinsumContractionOrders' TreeSASlicer: slice
    one label at a time (the one that most reduces the space complexity) and
    re-anneal the tree on the sliced sizes, until the largest intermediate fits
    2^score.sc_target elements."""

    score: ScoreFunction = field(default_factory=lambda: ScoreFunction(sc_target=20.0))
    betas: Tuple[float, float, float] = (14.0, 0.05, 15.0)
    ntrials: int = 2
    niters: int = 10
    seed: int = 0


@dataclass
class MergeVectors:
    """Simplifier: every rank-1 tensor is first multiplied into a tensor that
    shares its label (OMEinsumContractionOrders' MergeVectors), so the order
    search sees fewer, larger tensors; the merges become the first nodes of
    the returned tree."""


def _log2sz(labels, log2sd) -> float:
    return float(sum(log2sd[l] for l in labels))


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


def _post_order_pairs(ne: NestedEinsum) -> List[Tuple[int, int]]:
    """Binary tree -> post-order child-ref pairs (r >= 0 internal, r < 0 leaf -r-1)."""
    pairs: List[Tuple[int, int]] = []

    def rec(n) -> int:
        if n.isleaf:
            return -n.tensorindex - 1
        if len(n.args) != 2:
            raise ArgumentError("TreeSA works on binary trees")
        a, b = rec(n.args[0]), rec(n.args[1])
        pairs.append((a, b))
        return len(pairs) - 1

    rec(ne)
    return pairs


def _from_pairs(pairs, ixs, iy) -> NestedEinsum:
    """Post-order pairs -> NestedEinsum; a node's output labels are the labels
    of its leaves that occur outside its subtree or in the output."""
    n = len(ixs)
    count: Dict[Any, int] = {}
    for ix in ixs:
        for l in dict.fromkeys(ix):
            count[l] = count.get(l, 0) + 1
    out = set(iy)
    built: List[Tuple[NestedEinsum, Tuple[Any, ...], Dict[Any, int]]] = []

    def get(r):
        if r < 0:
            t = -r - 1
            c = {}
            for l in dict.fromkeys(ixs[t]):
                c[l] = 1
            return NestedEinsum(t), tuple(ixs[t]), c
        return built[r]

    for k, (a, b) in enumerate(pairs):
        na, la, ca = get(a)
        nb, lb, cb = get(b)
        c = dict(ca)
        for l, v in cb.items():
            c[l] = c.get(l, 0) + v
        if k == len(pairs) - 1:
            lab = tuple(iy)
        else:
            lab = tuple(l for l in dict.fromkeys(la + lb) if l in out or c[l] < count[l])
        built.append((NestedEinsum([na, nb], EinCode([la, lb], lab)), lab, c))
    return built[-1][0]


def _merge_vectors(ixs: List[List[Any]]):
    """MergeVectors: groups (absorbing tensor, vectors merged into it, in order)
    and the merged network's tensors."""
    n = len(ixs)
    absorbed = [False] * n
    groups: Dict[int, List[int]] = {}
    for v in range(n):
        if len(ixs[v]) != 1:
            continue
        (l,) = ixs[v]
        host = next((u for u in range(n) if u != v and not absorbed[u] and len(ixs[u]) > 1 and l in ixs[u]), None)
        if host is None:
            continue
        absorbed[v] = True
        groups.setdefault(host, []).append(v)
    keep = [t for t in range(n) if not absorbed[t]]
    return keep, groups


def _expand_merged(ne: NestedEinsum, keep: List[int], groups: Dict[int, List[int]], ixs) -> NestedEinsum:
    def leaf(t):
        node = NestedEinsum(t)
        for v in groups.get(t, []):
            node = NestedEinsum([node, NestedEinsum(v)], EinCode([tuple(ixs[t]), tuple(ixs[v])], tuple(ixs[t])))
        return node

    def rec(x):
        if x.isleaf:
            return leaf(keep[x.tensorindex])
        return NestedEinsum([rec(a) for a in x.args], x.eins)

    return rec(ne)


def _net(ixs: List[List[Any]], iy: List[Any], size_dict):
    """The network as the native planners take it: label ids, per-tensor label
    counts and ids, output ids, log2 extents."""
    import ctypes as C
    labels = list(dict.fromkeys([l for ix in ixs for l in ix] + list(iy)))
    lid = {l: i for i, l in enumerate(labels)}
    arr = lambda T, v: (T * max(len(v), 1))(*v)
    return (arr(C.c_int32, [len(ix) for ix in ixs]), arr(C.c_int32, [lid[l] for ix in ixs for l in ix]),
            len([l for l in iy if l in lid]), arr(C.c_int32, [lid[l] for l in iy if l in lid]), len(labels),
            arr(C.c_double, [math.log2(max(size_dict[l], 1)) for l in labels]))


def _greedy(ixs: List[List[Any]], iy: List[Any], size_dict, opt: GreedyMethod) -> NestedEinsum:
    """GreedyMethod through the native search (``ome_greedy``)."""
    import ctypes as C

    from . import _lib
    n = len(ixs)
    nl, fl, no, ol, nids, l2 = _net(ixs, iy, size_dict)
    out = (C.c_int32 * (2 * (n - 1)))()
    rc = _lib.load().ome_greedy(n, nl, fl, no, ol, nids, l2, float(opt.alpha), float(opt.temperature),
                                int(opt.nrepeat), int(opt.seed) & 0xFFFFFFFFFFFFFFFF, out, None)
    if rc != 0:
        raise ArgumentError(f"ome_greedy failed with status {rc}")
    return _from_pairs([(out[2 * k], out[2 * k + 1]) for k in range(n - 1)], [tuple(ix) for ix in ixs], tuple(iy))


def _treesa(ixs: List[List[Any]], iy: List[Any], size_dict, opt: TreeSA, init: NestedEinsum | None = None):
    """Run ome_treesa on the network and return the best tree as a NestedEinsum."""
    import ctypes as C

    from . import _lib
    n = len(ixs)
    if init is None:
        if opt.initializer == "random":
            rng = np.random.default_rng(opt.seed)
            slots = [-(t + 1) for t in range(n)]
            pairs = []
            while len(slots) > 1:
                i, j = rng.choice(len(slots), 2, replace=False)
                a, b = slots[i], slots[j]
                pairs.append((a, b))
                slots = [x for k, x in enumerate(slots) if k not in (i, j)] + [len(pairs) - 1]
        else:
            pairs = _post_order_pairs(_greedy(ixs, iy, size_dict, GreedyMethod(nrepeat=1, seed=opt.seed)))
    else:
        pairs = _post_order_pairs(init)
    # never accept a larger peak intermediate than the starting tree's: the
    # effective target is min(score.sc_target, sc of the initial tree)
    start_sc = tree_complexity(_from_pairs(pairs, [tuple(ix) for ix in ixs], tuple(iy)), size_dict)[1]
    nl, fl, no, ol, nids, l2 = _net(ixs, iy, size_dict)
    init_arr = (C.c_int32 * (2 * (n - 1)))(*[x for p in pairs for x in p])
    out = (C.c_int32 * (2 * (n - 1)))()
    cx = (C.c_double * 3)()
    sc = opt.score
    b0, db, b1 = opt.betas
    rc = _lib.load().ome_treesa(n, nl, fl, no, ol, nids, l2, init_arr, float(min(sc.sc_target, start_sc)),
                                float(sc.sc_weight), float(sc.rw_weight) / max(float(sc.tc_weight), 1e-300),
                                float(b0), float(db), float(b1), int(opt.niters), int(opt.ntrials),
                                int(opt.seed) & 0xFFFFFFFFFFFFFFFF, out, cx)
    if rc != 0:
        raise ArgumentError(f"ome_treesa failed with status {rc}")
    res = [(out[2 * k], out[2 * k + 1]) for k in range(n - 1)]
    return _from_pairs(res, [tuple(ix) for ix in ixs], tuple(iy))


def optimize_code(code: AbstractEinsum, size_dict: Dict[Any, int], optimizer=None, simplifier=None,
                  slicer=None):
    """``optimize_code`` (src/contractionorder.jl:30-32): a NestedEinsum (or a
    SlicedEinsum when a slicer is given) for the flattened code; optimizer
    GreedyMethod (default) or TreeSA, simplifier None or MergeVectors()."""
    optimizer = optimizer or GreedyMethod()
    flat = code if isinstance(code, EinCode) else code.flatten()
    ixs = [list(ix) for ix in flat.ixs]
    iy = list(flat.iy)
    if isinstance(simplifier, MergeVectors) and len(ixs) > 2:
        keep, groups = _merge_vectors(ixs)
        if groups and len(keep) >= 2:
            merged = EinCode([tuple(ixs[t]) for t in keep], tuple(iy))
            inner = optimize_code(merged, size_dict, optimizer)
            ne = _expand_merged(inner, keep, groups, ixs)
            return slice_code(ne, size_dict, slicer) if slicer is not None else ne
    if len(ixs) == 1:
        ne = NestedEinsum([NestedEinsum(0)], EinCode([tuple(ixs[0])], tuple(iy)))
    elif isinstance(optimizer, TreeSA):
        ne = _treesa(ixs, iy, size_dict, optimizer)
    else:
        ne = _greedy(ixs, iy, size_dict, optimizer)
    if slicer is not None:
        return slice_code(ne, size_dict, slicer)
    return ne


def _native_slice(code: NestedEinsum, size_dict, sc_target: float, max_slices: int, forbid=()):
    """Labels to slice, chosen by ``ome_slice_greedy``; None when the tree is
    not one the native search describes exactly (a node with other than two
    children, or intermediates that keep more labels than their leaves need)."""
    import ctypes as C

    from . import _lib
    try:
        pairs = _post_order_pairs(code)
    except ArgumentError:
        return None
    flat = code.flatten()
    ixs = [list(ix) for ix in flat.ixs]
    iy = list(flat.iy)
    if len(ixs) < 2:
        return []
    canon = _from_pairs(pairs, [tuple(ix) for ix in ixs], tuple(iy))

    def same(a, b):
        if a.isleaf or b.isleaf:
            return a.isleaf and b.isleaf
        return set(a.eins.iy) == set(b.eins.iy) and all(same(x, y) for x, y in zip(a.args, b.args))

    if not same(code, canon):
        return None
    labels = list(dict.fromkeys([l for ix in ixs for l in ix] + iy))
    nl, fl, no, ol, nids, l2 = _net(ixs, iy, size_dict)
    tree = (C.c_int32 * (2 * len(pairs)))(*[x for p in pairs for x in p])
    fb = (C.c_int32 * nids)(*[1 if l in forbid else 0 for l in labels])
    out = (C.c_int32 * nids)()
    cnt = C.c_int32()
    rc = _lib.load().ome_slice_greedy(len(ixs), nl, fl, no, ol, nids, l2, tree, float(sc_target), int(max_slices),
                                      fb, out, C.byref(cnt))
    if rc != 0:
        raise ArgumentError(f"ome_slice_greedy failed with status {rc}")
    return [labels[out[k]] for k in range(cnt.value)]


def _treesa_slice(code: NestedEinsum, size_dict, slicer: TreeSASlicer) -> SlicedEinsum:
    sd = dict(size_dict)
    sliced: List[Any] = []
    ne = code
    flat = code.flatten()
    ixs = [list(ix) for ix in flat.ixs]
    iy = list(flat.iy)
    target = slicer.score.sc_target
    for _ in range(len(sd)):
        tc, sc, _ = tree_complexity(ne, sd)
        if sc <= target + 1e-9:
            break
        pick = _native_slice(ne, sd, target, 1, forbid=set(iy))
        if pick is None:   # a tree the native search does not describe
            best = None
            for l in flat.uniquelabels():
                if l in sliced or sd[l] <= 1 or l in iy:
                    continue
                sd2 = dict(sd)
                sd2[l] = 1
                tc2, sc2, _ = tree_complexity(ne, sd2)
                key = (sc2, tc2 + math.log2(sd[l]))
                if best is None or key < best[0]:
                    best = (key, l)
            pick = [] if best is None else [best[1]]
        if not pick:
            break
        sliced.append(pick[0])
        sd[pick[0]] = 1
        if len(ixs) > 2:
            ne = _treesa(ixs, iy, sd, TreeSA(betas=slicer.betas, ntrials=slicer.ntrials, niters=slicer.niters,
                                             score=slicer.score, seed=slicer.seed + len(sliced)), init=ne)
    return SlicedEinsum(sliced, ne)


def slice_code(code: NestedEinsum, size_dict: Dict[Any, int], slicer=None) -> SlicedEinsum:
    """``slice_code`` (src/contractionorder.jl:33-35): GreedySlicer (default) or
    TreeSASlicer."""
    slicer = slicer or GreedySlicer()
    if isinstance(slicer, TreeSASlicer):
        return _treesa_slice(code, size_dict, slicer)
    picked = _native_slice(code, size_dict, slicer.sc_target, len(size_dict))
    if picked is not None:
        return SlicedEinsum(picked, code)
    # a tree with n-ary nodes or wider intermediates: the same search on the tree itself
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
