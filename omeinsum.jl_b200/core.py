"""Contraction codes: EinCode, NestedEinsum, SlicedEinsum and the ein"..." parser.

Python mirror of OMEinsum.jl's code types (src/Core.jl:10-114,
src/einsequence.jl:155-376, src/slicing.jl:10-17, src/interfaces.jl:21-114).
Differences that follow from the host language: labels are any hashable
(single characters from ``ein``), leaf tensor indices are 0-based, and
StaticEinCode/DynamicEinCode are one class (Python has no compile-time
specialisation to choose between them).
"""
from __future__ import annotations

import re
from typing import Any, Dict, Iterable, List, Sequence

from ._lib import ArgumentError, DimensionMismatch


class AbstractEinsum:
    """``AbstractEinsum`` (src/Core.jl:10): anything with getixsv/getiyv."""

    def getixsv(self) -> List[List[Any]]:
        raise NotImplementedError

    def getiyv(self) -> List[Any]:
        raise NotImplementedError

    def uniquelabels(self) -> List[Any]:
        """``uniquelabels`` (src/Core.jl:11)."""
        out: List[Any] = []
        for ix in self.getixsv() + [self.getiyv()]:
            for l in ix:
                if l not in out:
                    out.append(l)
        return out

    def labeltype(self):
        labs = self.uniquelabels()
        return type(labs[0]) if labs else type(None)


class EinCode(AbstractEinsum):
    """``EinCode(ixs, iy)`` (src/Core.jl:13-114): input label tuples and output labels."""

    def __init__(self, ixs: Sequence[Iterable[Any]], iy: Iterable[Any]):
        ixs = [tuple(ix) for ix in ixs]
        if len(ixs) == 0:
            raise RuntimeError("number of input tensors must be greater than 0")
        self.ixs = ixs
        self.iy = tuple(iy)

    def getixs(self):
        return self.ixs

    def getiy(self):
        return self.iy

    def getixsv(self):
        return [list(ix) for ix in self.ixs]

    def getiyv(self):
        return list(self.iy)

    def __eq__(self, other):
        return isinstance(other, EinCode) and self.getixsv() == other.getixsv() and self.getiyv() == other.getiyv()

    def __hash__(self):
        return hash((tuple(self.ixs), self.iy))

    def __repr__(self):
        j = lambda ix: "".join(map(str, ix)) if all(isinstance(l, str) and len(l) == 1 for l in ix) \
            else "∘".join(map(str, ix))
        return ", ".join(j(ix) for ix in self.ixs) + " -> " + j(self.iy)

    def replace(self, *pairs):
        m = dict(pairs)
        return EinCode([[m.get(l, l) for l in ix] for ix in self.ixs], [m.get(l, l) for l in self.iy])

    def __call__(self, *xs, size_info=None):
        from .engine import einsum
        sd = get_size_dict(self.ixs, xs, size_info)
        return einsum(self, xs, sd)


DynamicEinCode = EinCode
StaticEinCode = EinCode


class NestedEinsum(AbstractEinsum):
    """Contraction tree (``DynamicNestedEinsum``, src/einsequence.jl:172-189).

    ``NestedEinsum(tensorindex)`` is a leaf (0-based input index);
    ``NestedEinsum(args, eins)`` contracts the children ``args`` with ``eins``.
    """

    def __init__(self, args, eins: EinCode | None = None):
        if isinstance(args, int):
            self.tensorindex = args
            self.args: List[NestedEinsum] = []
            self.eins = None
        else:
            args = list(args)
            assert eins is not None and len(args) == len(eins.ixs)
            self.tensorindex = -1
            self.args = args
            self.eins = eins

    @property
    def isleaf(self) -> bool:
        return self.tensorindex >= 0

    def siblings(self):
        return self.args

    def rootcode(self):
        return self.eins

    def _collect(self, d: Dict[int, List[Any]]):
        for i, a in enumerate(self.args):
            if a.isleaf:
                d[a.tensorindex] = list(self.eins.ixs[i])
            else:
                a._collect(d)
        return d

    def getixsv(self):
        """``getixsv`` (src/einsequence.jl:340-347)."""
        if self.isleaf:
            raise RuntimeError("Can not call `getixsv` on leaf nodes!")
        d = self._collect({})
        return [d[i] for i in sorted(d)]

    def getiyv(self):
        if self.isleaf:
            raise RuntimeError("Can not call `getiyv` on leaf nodes!")
        return list(self.eins.iy)

    def flatten(self) -> EinCode:
        """``flatten`` (src/einsequence.jl:319-337)."""
        return EinCode(self.getixsv(), self.getiyv())

    def __eq__(self, other):
        if not isinstance(other, NestedEinsum) or self.isleaf != other.isleaf:
            return False
        if self.isleaf:
            return self.tensorindex == other.tensorindex
        return self.eins == other.eins and len(self.args) == len(other.args) and \
            all(a == b for a, b in zip(self.args, other.args))

    def __hash__(self):
        return hash(self.tensorindex) if self.isleaf else hash((self.eins, tuple(self.args)))

    def __repr__(self):
        if self.isleaf:
            return str(self.tensorindex)
        return f"({', '.join(map(repr, self.args))} | {self.eins})"

    def replace(self, *pairs):
        if self.isleaf:
            return NestedEinsum(self.tensorindex)
        return NestedEinsum([a.replace(*pairs) for a in self.args], self.eins.replace(*pairs))

    def __call__(self, *xs, size_info=None):
        from .engine import einsum
        sd = get_size_dict(self.getixsv(), xs, size_info)
        return einsum(self, xs, sd)


DynamicNestedEinsum = NestedEinsum
StaticNestedEinsum = NestedEinsum


class SlicedEinsum(AbstractEinsum):
    """``SlicedEinsum(slicing, eins)`` (src/slicing.jl:10-13)."""

    def __init__(self, slicing: Sequence[Any], eins):
        self.slicing = list(slicing)
        self.eins = eins

    def getixsv(self):
        return self.eins.getixsv()

    def getiyv(self):
        return self.eins.getiyv()

    def flatten(self):
        return self.eins.flatten() if isinstance(self.eins, NestedEinsum) else self.eins

    def __eq__(self, other):
        return isinstance(other, SlicedEinsum) and self.slicing == other.slicing and self.eins == other.eins

    def __hash__(self):
        return hash((tuple(self.slicing), self.eins))

    def replace(self, *pairs):
        m = dict(pairs)
        return SlicedEinsum([m.get(l, l) for l in self.slicing], self.eins.replace(*pairs))

    def __call__(self, *xs, size_info=None):
        from .engine import einsum
        sd = get_size_dict(self.getixsv(), xs, size_info)
        return einsum(self, xs, sd)


def slice_iterator(slicing, size_dict):
    """``SliceIterator`` order (src/slicing.jl:37-71): column-major over the
    sliced labels, first label fastest; yields 0-based slice maps."""
    import itertools

    sizes = [size_dict[l] for l in slicing]
    for ci in itertools.product(*[range(s) for s in reversed(sizes)]):
        yield dict(zip(slicing, reversed(ci)))


# ----------------------------------------------------------------------------
# ein"..." string parsing (src/interfaces.jl:35-47, src/einsequence.jl:9-86)
# ----------------------------------------------------------------------------

_EIN_RE = re.compile(r"^([\(\),\w]*)->(\w*)$", re.UNICODE)


def ein(s: str):
    """Parse an einsum string; parentheses give a NestedEinsum."""
    s = s.replace("\n", "").replace(" ", "")
    m = _EIN_RE.match(s)
    if m is None or any(c.isdigit() or c == "_" for c in s):
        raise ArgumentError(f"invalid einsum specification {s}")
    sixs, siy = m.group(1), m.group(2)
    if "(" in sixs:
        return parse_nested(sixs, list(siy))
    return EinCode([tuple(ix) for ix in sixs.split(",")], tuple(siy))


def parse_nested(s: str, iy: List[Any]):
    """``parse_nested`` + ``filliys!`` (src/einsequence.jl:9-86): an intermediate
    keeps the labels it shares with its parent's output or with a sibling."""
    if s.count("(") != s.count(")"):
        raise ArgumentError(f"Parentheses don't pair up in {s}")
    counter = [0]

    def parse(i):
        args, inds, cur = [], [], []

        def flush():
            if cur:
                args.append({"leaf": counter[0], "inds": list(cur)})
                counter[0] += 1
                for l in cur:
                    if l not in inds:
                        inds.append(l)
                cur.clear()

        while i < len(s):
            c = s[i]
            if c == "(":
                i, sub = parse(i + 1)
                args.append(sub)
                for l in sub["inds"]:
                    if l not in inds:
                        inds.append(l)
                continue
            if c in "),":
                flush()
                i += 1
                if c == ")":
                    return i, {"args": args, "inds": inds, "iy": []}
                continue
            if not c.isalpha():
                raise ArgumentError(f"parsing {s} failed, {c} is not a valid entry")
            cur.append(c)
            i += 1
        flush()
        return i, {"args": args, "inds": inds, "iy": []}

    _, out = parse(0)
    out["iy"] = list(iy)

    def fill(n):
        for i, a in enumerate(n["args"]):
            if "leaf" in a:
                continue
            for l in a["inds"]:
                if l in n["iy"] and l not in a["iy"]:
                    a["iy"].append(l)
            for j, b in enumerate(n["args"]):
                if i != j:
                    for l in a["inds"]:
                        if l in b["inds"] and l not in a["iy"]:
                            a["iy"].append(l)
            fill(a)

    fill(out)

    def build(n):
        args, ixs = [], []
        for a in n["args"]:
            if "leaf" in a:
                args.append(NestedEinsum(a["leaf"]))
                ixs.append(tuple(a["inds"]))
            else:
                args.append(build(a))
                ixs.append(tuple(a["iy"]))
        return NestedEinsum(args, EinCode(ixs, n["iy"]))

    return build(out)


# ----------------------------------------------------------------------------
# size dictionaries (src/interfaces.jl:67-114)
# ----------------------------------------------------------------------------


def _shape(x):
    return tuple(int(s) for s in x.shape)


def get_size_dict(ixs, xs, size_info=None) -> Dict[Any, int]:
    """``get_size_dict!``: label -> extent with the reference's error contract:
    ArgumentError on a tensor-count or rank mismatch, DimensionMismatch on
    conflicting extents."""
    d = dict(size_info) if size_info else {}
    if len(xs) < 1:
        raise RuntimeError("empty input tensors")
    if len(ixs) != len(xs):
        raise ArgumentError(f"{len(xs)} tensors labelled by {len(ixs)} indices")
    for ix, x in zip(ixs, xs):
        s = _shape(x)
        if len(ix) != len(s):
            raise ArgumentError(f"indices {tuple(ix)} invalid for tensor with ndims = {len(s)}")
        for l, e in zip(ix, s):
            if l in d:
                if d[l] != e:
                    raise DimensionMismatch(f"{l} = {d[l]} or {e})?")
            else:
                d[l] = e
    return d


def uniformsize(code: AbstractEinsum, size: int) -> Dict[Any, int]:
    """``uniformsize`` (src/contractionorder.jl:41)."""
    return {l: size for l in code.uniquelabels()}


def getixsv(code):
    return code.getixsv()


def getiyv(code):
    return code.getiyv()


def flatten(code):
    return code if isinstance(code, EinCode) else code.flatten()


def drop_slicedim(ne: NestedEinsum, slicing) -> NestedEinsum:
    """``drop_slicedim`` (src/slicing.jl:139-145)."""
    if ne.isleaf:
        return ne
    e = ne.eins
    return NestedEinsum([drop_slicedim(a, slicing) for a in ne.args],
                        EinCode([[l for l in ix if l not in slicing] for ix in e.ixs],
                                [l for l in e.iy if l not in slicing]))
