"""CPU oracle: a NumPy restatement of OMEinsum.jl's DefaultBackend einsum path.

TEST INFRASTRUCTURE ONLY.  Only ``tests/``, ``__graft_entry__.smoke()`` and the
``cpu_baseline`` / ``--impl reference`` legs of ``bench.py`` may import this
module, and only as the checker or as the timed CPU baseline.  The product
(the ``omeinsum.jl_b200`` package and its CUDA library) never calls it.

Conventions follow the reference (Julia):

* arrays are column-major: a NumPy array here has axes in Julia's dimension
  order and every reshape uses ``order="F"``;
* ``sx, sy`` mean ``y <- sy*y + sx*f(xs)`` with the four ``@addmul!`` branches
  of ``src/utils.jl:8-37``;
* three algebras: ordinary numbers (float32/64, complex64/128, int64 with
  wrap-around), Bool as OR-AND, and tropical max-plus (TropicalNumbers.jl:
  ``a (+) b = max(a, b)``, ``a (*) b = a + b``, zero = -Inf, one = 0).

Each function names the reference ``file:line`` it restates.  Parity pins:
the reference's own known-answer tests (analyze_binary, the 36-rule sweep,
EinArray indexing, the C60 tropical count 66, 3-colouring counts, scalar
``ein",->"``) are asserted in ``tests/test_oracle.py``.
"""
from __future__ import annotations

import itertools
import math
from dataclasses import dataclass, field
from typing import Any, Dict, List, Sequence, Tuple

import numpy as np

# ----------------------------------------------------------------------------
# algebras
# ----------------------------------------------------------------------------


class Algebra:
    """Ordinary (+, *) numbers: float, complex, int64 (wraps like Julia Int64)."""

    name = "real"

    def zero(self, dtype):
        return np.zeros((), dtype=dtype)[()]

    def one(self, dtype):
        return np.ones((), dtype=dtype)[()]

    def iszero(self, s):
        return s == 0

    def isone(self, s):
        return s == 1

    def add(self, a, b):
        return a + b

    def mul(self, a, b):
        return a * b

    def conj(self, a):
        return np.conj(a) if np.iscomplexobj(a) else a

    def sum(self, x, axes):
        if len(axes) == 0:
            return np.array(x)
        with np.errstate(over="ignore"):
            return np.sum(x, axis=tuple(axes), dtype=x.dtype)

    def matmul(self, a, b):
        """Batched (..., m, k) @ (..., k, n) in the working dtype (BLAS for floats).

        Int64 (Julia's generic ``mul!``, ``src/binaryrules.jl:129-131``):
        when max|a| * max|b| * k < 2^53 every partial sum is an integer that
        FP64 holds exactly and no Int64 wrap-around can occur, so the product
        is formed by FP64 BLAS and converted back -- the same integers as the
        Int64 loop, in a fraction of the time.  Otherwise NumPy's Int64
        matmul (wrapping, like Julia's Int64)."""
        if a.dtype == np.int64 and b.dtype == np.int64 and a.size and b.size:
            bound = float(np.max(np.abs(a))) * float(np.max(np.abs(b))) * a.shape[-1]
            if bound < 2.0 ** 53:
                return np.matmul(a.astype(np.float64), b.astype(np.float64)).astype(np.int64)
        with np.errstate(over="ignore"):
            return np.matmul(a, b)


class BoolAlgebra(Algebra):
    """Bool contraction as OR-AND (0/1 semantics of Julia's Bool sum-product)."""

    name = "bool"

    def iszero(self, s):
        return not bool(s)

    def isone(self, s):
        return bool(s)

    def add(self, a, b):
        return np.logical_or(a, b)

    def mul(self, a, b):
        return np.logical_and(a, b)

    def conj(self, a):
        return a

    def sum(self, x, axes):
        if len(axes) == 0:
            return np.array(x)
        return np.any(x, axis=tuple(axes))

    def matmul(self, a, b):
        return np.matmul(a.astype(np.int64), b.astype(np.int64)) != 0


class TropicalAlgebra(Algebra):
    """Max-plus semiring (TropicalNumbers.jl Tropical{T}); values stored as floats."""

    name = "tropical"

    def zero(self, dtype):
        return np.array(-np.inf, dtype=dtype)[()]

    def one(self, dtype):
        return np.zeros((), dtype=dtype)[()]

    def iszero(self, s):
        return s == -np.inf

    def isone(self, s):
        return s == 0

    def add(self, a, b):
        return np.maximum(a, b)

    def mul(self, a, b):
        return a + b

    def conj(self, a):
        return a

    def sum(self, x, axes):
        if len(axes) == 0:
            return np.array(x)
        if x.size == 0:
            shape = [s for i, s in enumerate(x.shape) if i not in axes]
            return np.full(shape, -np.inf, dtype=x.dtype)
        return np.max(x, axis=tuple(axes))

    def matmul(self, a, b):
        # max_k (a[..., m, k] + b[..., k, n]) chunked over k to bound memory
        out_shape = np.broadcast_shapes(a.shape[:-2], b.shape[:-2]) + (a.shape[-2], b.shape[-1])
        out = np.full(out_shape, -np.inf, dtype=np.result_type(a, b))
        for k in range(a.shape[-1]):
            np.maximum(out, a[..., :, k:k + 1] + b[..., k:k + 1, :], out=out)
        return out


REAL = Algebra()
BOOL = BoolAlgebra()
TROPICAL = TropicalAlgebra()


def algebra_for(x, alg=None):
    if alg is not None:
        return alg
    return BOOL if np.asarray(x).dtype == np.bool_ else REAL


# ----------------------------------------------------------------------------
# eltype promotion (Julia promote_type over the supported eltypes)
# ----------------------------------------------------------------------------

_RANK = {np.dtype(np.bool_): 0, np.dtype(np.int64): 1, np.dtype(np.float32): 2, np.dtype(np.float64): 3}


def promote_type(*dtypes):
    """Julia ``promote_type`` for Bool/Int64/Float32/Float64 and their complexes.

    Differs from NumPy: Julia promotes (Int64, Float32) to Float32.
    Reference: ``get_output_array`` ``src/loop_einsum.jl:48-61``.
    """
    dtypes = [np.dtype(d) for d in dtypes]
    cplx = any(d.kind == "c" for d in dtypes)
    real = [np.dtype(np.float32) if d == np.complex64 else np.dtype(np.float64) if d == np.complex128 else d
            for d in dtypes]
    r = max(real, key=lambda d: _RANK[d])
    if cplx:
        return np.dtype(np.complex64) if r in (np.dtype(np.float32), np.dtype(np.int64), np.dtype(np.bool_)) \
            else np.dtype(np.complex128)
    return r


# ----------------------------------------------------------------------------
# helpers
# ----------------------------------------------------------------------------


def reshape_f(x, shape):
    return np.reshape(x, tuple(shape), order="F")


def _unique(ix):
    """``_unique`` (``src/utils.jl:105-106``): order-preserving unique."""
    out = []
    for l in ix:
        if l not in out:
            out.append(l)
    return out


def addmul_(sy, y, sx, terms, alg=REAL, flatten=False):
    """``@addmul!`` / ``@flatten_addmul!`` (``src/utils.jl:8-37``), in place on ``y``.

    ``added = Ref(sx) .* x1 .* x2 ...`` (left to right); then the branch on
    (iszero(sx), iszero(sy), isone(sy)).
    """
    added = sx
    for x in terms:
        x = np.asarray(x)
        if flatten:
            x = reshape_f(x, y.shape)
        added = alg.mul(added, x)
    with np.errstate(over="ignore", invalid="ignore"):
        if alg.iszero(sx):
            y[...] = alg.mul(sy, y)
        elif alg.iszero(sy):
            y[...] = added
        elif alg.isone(sy):
            y[...] = alg.add(y, added)
        else:
            y[...] = alg.add(alg.mul(sy, y), added)
    return y


def _axpby_(y, f, sx, sy, alg):
    """``mul!(y, A, B, sx, sy)`` / ``_batched_gemm!`` result assembly: y = sx*f + sy*y
    (y is not read when sy is zero), ``src/binaryrules.jl:46-61,129-139``."""
    with np.errstate(over="ignore", invalid="ignore"):
        if alg.iszero(sy):
            y[...] = alg.mul(sx, f)
        else:
            y[...] = alg.add(alg.mul(sx, f), alg.mul(sy, y))
    return y


# ----------------------------------------------------------------------------
# size dict / output allocation
# ----------------------------------------------------------------------------


class DimensionMismatch(Exception):
    """Julia ``DimensionMismatch``."""


def get_size_dict(ixs, xs, size_info=None):
    """``get_size_dict!`` (``src/interfaces.jl:67-106``).

    Raises ``ValueError`` (Julia ``ArgumentError``) on tensor-count or rank
    mismatch and ``DimensionMismatch`` on conflicting extents.
    """
    d = dict(size_info) if size_info else {}
    if len(xs) < 1:
        raise RuntimeError("empty input tensors")
    if len(ixs) != len(xs):
        raise ValueError(f"{len(xs)} tensors labelled by {len(ixs)} indices")
    for ix, x in zip(ixs, xs):
        s = np.shape(x)
        if len(ix) != len(s):
            raise ValueError(f"indices {ix} invalid for tensor with ndims = {len(s)}")
        for l, e in zip(ix, s):
            if l in d:
                if d[l] != e:
                    raise DimensionMismatch(f"{l} = {d[l]} or {e})?")
            else:
                d[l] = e
    return d


def get_output_array(xs, shape, fillzero, alg=None):
    """``get_output_array`` (``src/loop_einsum.jl:48-61``)."""
    dt = promote_type(*[np.asarray(x).dtype for x in xs])
    if fillzero:
        a = alg if alg is not None else algebra_for(np.zeros((), dt))
        return np.full(tuple(shape), a.zero(dt), dtype=dt, order="F")
    return np.zeros(tuple(shape), dtype=dt, order="F")


# ----------------------------------------------------------------------------
# unary rules (src/unaryrules.jl) and tensorpermute! (src/utils.jl:122-156)
# ----------------------------------------------------------------------------


def tensorpermute_(C, A, perm, sx, sy, alg=REAL):
    """``tensorpermute!`` (``src/utils.jl:122-156``): group adjacent permuted
    dims, then ``permutedims!``; the grouping changes no value."""
    N = A.ndim
    assert N == len(perm)
    if N == 0:
        return addmul_(sy, C, sx, [A], alg, flatten=True)
    # grouping (utils.jl:126-146)
    newshape_slots = [-1] * N
    permk = perm[0]
    newperm = [permk]
    newshape_slots[permk] = A.shape[permk]
    dk = 1
    for i in range(1, N):
        p = perm[i]
        if p == permk + dk:
            newshape_slots[permk] *= A.shape[p]
            dk += 1
        else:
            permk = p
            newshape_slots[permk] = A.shape[p]
            newperm.append(permk)
            dk = 1
    newshape = [s for s in newshape_slots if s != -1]
    order = sorted(range(len(newperm)), key=lambda i: newperm[i])
    newperm = sorted(range(len(order)), key=lambda i: order[i])  # sortperm(sortperm(newperm))
    A_ = reshape_f(A, newshape)
    P = np.transpose(A_, newperm)
    if alg.iszero(sy):
        Cv = reshape_f(C, P.shape) if C.flags.f_contiguous else None
        res = np.array(P, order="F")
        if not alg.isone(sx):
            res = alg.mul(sx, res)
        C[...] = reshape_f(res, C.shape)
        return C
    return addmul_(sy, C, sx, [P], alg, flatten=True)


def unary_tr_(ix, iy, x, y, sx, sy, alg=REAL):
    """``Tr`` (``src/unaryrules.jl:22-26``): y .= sy .* y .+ sx * tr(x)."""
    t = alg.sum(np.diagonal(x), [0])
    y[...] = alg.add(alg.mul(sy, y), alg.mul(sx, t))
    return y


def unary_sum_(ix, iy, x, y, sx, sy, alg=REAL):
    """``Sum`` (``src/unaryrules.jl:30-40``): sum the dims not in iy, then permute."""
    dims = [i for i, l in enumerate(ix) if l not in iy]
    res = alg.sum(x, dims)
    ix1f = [l for l in ix if l in iy]
    if list(ix1f) != list(iy):
        return unary_permutedims_(ix1f, iy, res, y, sx, sy, alg)
    return addmul_(sy, y, sx, [res], alg, flatten=True)


def unary_repeat_(ix, iy, x, y, sx, sy, alg=REAL):
    """``Repeat`` (``src/unaryrules.jl:44-58``): broadcast over labels absent from ix."""
    ix1f = [l for l in iy if l in ix]
    shape1 = [s for l, s in zip(iy, y.shape) if l in ix]
    shape2 = [s if l in ix else 1 for l, s in zip(iy, y.shape)]
    if list(ix1f) != list(ix):
        y1 = np.zeros(shape1, dtype=x.dtype, order="F")
        unary_permutedims_(ix, ix1f, x, y1, alg.one(x.dtype), alg.zero(x.dtype), alg)
    else:
        y1 = x
    rep = np.broadcast_to(reshape_f(y1, shape2), y.shape)
    return addmul_(sy, y, sx, [rep], alg, flatten=True)


def unary_diag_(ix, iy, x, y, sx, sy, alg=REAL):
    """``Diag`` / ``compactify!`` (``src/unaryrules.jl:62-91``): y[ci] = x[ci[locs]]."""
    locs = [iy.index(l) for l in ix]
    assert tuple(x.shape) == tuple(y.shape[l] for l in locs)
    idx = []
    for loc in locs:
        sh = [1] * y.ndim
        sh[loc] = y.shape[loc]
        idx.append(np.arange(y.shape[loc]).reshape(sh))
    g = x[tuple(idx)] if idx else np.asarray(x)
    g = np.broadcast_to(g, y.shape)
    with np.errstate(over="ignore", invalid="ignore"):
        if alg.iszero(sy):
            y[...] = g if alg.isone(sx) else alg.mul(sx, g)
        else:
            y[...] = alg.add(alg.mul(sy, y), alg.mul(sx, g))
    return y


def unary_duplicate_(ix, iy, x, y, sx, sy, alg=REAL):
    """``Duplicate`` / ``duplicate!`` (``src/unaryrules.jl:93-121``): scatter x onto
    the diagonal positions of y; off-diagonal entries become 0 (sy zero) or sy*y."""
    locs = [ix.index(l) for l in iy]
    idx = []
    for loc in locs:
        sh = [1] * x.ndim
        sh[loc] = x.shape[loc]
        idx.append(np.arange(x.shape[loc]).reshape(sh))
    with np.errstate(over="ignore", invalid="ignore"):
        if alg.iszero(sy):
            y[...] = alg.zero(y.dtype)
            y[tuple(idx)] = alg.mul(sx, x)
        else:
            y[...] = alg.mul(sy, y)
            cur = y[tuple(idx)]
            y[tuple(idx)] = alg.add(alg.mul(sx, x), cur)
    return y


def unary_permutedims_(ix, iy, x, y, sx, sy, alg=REAL):
    """``Permutedims`` (``src/unaryrules.jl:125-129``)."""
    perm = [list(ix).index(l) for l in iy]
    return tensorpermute_(y, x, perm, sx, sy, alg)


def unary_identity_(ix, iy, x, y, sx, sy, alg=REAL):
    """``Identity`` (``src/unaryrules.jl:133-136``)."""
    return addmul_(sy, y, sx, [x], alg, flatten=True)


_UNARY_RULES = {
    "Diag": unary_diag_, "Sum": unary_sum_, "Permutedims": unary_permutedims_,
    "Repeat": unary_repeat_, "Duplicate": unary_duplicate_, "Tr": unary_tr_,
    "Identity": unary_identity_,
}


def unary_pipeline(ix, iy):
    """``unary_pipeline`` (``src/einsum.jl:60-82``): Diag -> Sum|Permutedims -> Repeat -> Duplicate."""
    ix_unique = _unique(ix)
    iy_unique = _unique(iy)
    iy_a = [i for i in iy_unique if i in ix]
    ops = []
    if len(ix_unique) != len(ix):
        ops.append(("Diag", list(ix), ix_unique))
    if len(ix_unique) != len(iy_a):
        ops.append(("Sum", ix_unique, iy_a))
    elif ix_unique != iy_a:
        ops.append(("Permutedims", ix_unique, iy_a))
    if len(iy_a) != len(iy_unique):
        ops.append(("Repeat", iy_a, iy_unique))
    if len(iy_unique) != len(iy):
        ops.append(("Duplicate", iy_unique, list(iy)))
    return ops


def einsum_unary_(ix, iy, x, y, sx, sy, size_dict, alg=REAL):
    """Unary ``einsum!`` (``src/einsum.jl:84-101``): one temporary per pipeline stage."""
    ops = unary_pipeline(list(ix), list(iy))
    last = np.asarray(x)
    for k, (rule, oix, oiy) in enumerate(ops):
        if k == len(ops) - 1:
            _UNARY_RULES[rule](oix, oiy, last, y, sx, sy, alg)
        else:
            cache = np.zeros([size_dict[l] for l in oiy], dtype=y.dtype, order="F")
            _UNARY_RULES[rule](oix, oiy, last, cache, alg.one(y.dtype), alg.zero(y.dtype), alg)
            last = cache
    if len(ops) == 0:
        addmul_(sy, y, sx, [last], alg, flatten=True)
    return y


# ----------------------------------------------------------------------------
# binary path (src/einsum.jl:104-211, src/binaryrules.jl, src/utils.jl:162-177)
# ----------------------------------------------------------------------------


def _analyze_binary_input(ix1, ix2, iy):
    """``_analyze_binary_input`` (``src/einsum.jl:187-211``)."""
    batch, inner, outer = [], [], []
    for l1 in ix1:
        if l1 in ix2:
            if l1 in iy:
                if l1 not in batch:
                    batch.append(l1)
            elif l1 not in inner:
                inner.append(l1)
        elif l1 in iy:
            if l1 not in outer:
                outer.append(l1)
    outer2 = []
    for l2 in ix2:
        if l2 not in ix1 and l2 in iy and l2 not in outer2:
            outer2.append(l2)
    return inner, outer, outer2, batch


def analyze_binary(ix1, ix2, iy, size_dict):
    """``analyze_binary`` (``src/einsum.jl:139-185``).

    Returns ``c1, c2, cy, s1, s2, s3, i1, i2, iyb``.
    """
    inner, o1, o2, batch = _analyze_binary_input(list(ix1), list(ix2), list(iy))
    c1 = o1 + inner + batch
    c2 = inner + o2 + batch
    cy = o1 + o2 + batch
    prod = lambda ls: int(np.prod([size_dict[l] for l in ls], dtype=np.int64)) if ls else 1
    si, sj, sk, sl = prod(o1), prod(inner), prod(o2), prod(batch)
    i1, i2, iyb, s1, s2, s3 = [], [], [], [], [], []
    if o1:
        i1.append("i"); iyb.append("i"); s1.append(si); s3.append(si)
    if inner:
        i1.append("j"); i2.append("j"); s1.append(sj); s2.append(sj)
    if o2:
        i2.append("k"); iyb.append("k"); s2.append(sk); s3.append(sk)
    if batch:
        i1.append("l"); i2.append("l"); iyb.append("l"); s1.append(sl); s2.append(sl); s3.append(sl)
    return c1, c2, cy, s1, s2, s3, i1, i2, iyb


def simplifyto(ix1, c1, x1, size_dict, alg=REAL):
    """``simplifyto`` (``src/einsum.jl:127-134``): unary einsum into canonical order."""
    if list(c1) != list(ix1):
        xs1 = np.zeros([size_dict[l] for l in c1], dtype=np.asarray(x1).dtype, order="F")
        dt = xs1.dtype
        return einsum_unary_(list(ix1), list(c1), x1, xs1, alg.one(dt), alg.zero(dt), size_dict, alg)
    return np.asarray(x1)


def binary_einsum_(rule, x1, x2, y, sx, sy, alg=REAL):
    """``binary_einsum!(::SimpleBinaryRule, ...)`` (``src/binaryrules.jl:18-141``).

    All 36 rules are sum-products over the letters i (outer1), j (inner),
    k (outer2), l (batch); contractions (rules with ``j``) go through BLAS
    matmul in the working dtype (``mul!`` / ``_batched_gemm!``), the others are
    ``@addmul!`` broadcasts.  ``rule = (i1, i2, iyb)`` letter tuples.
    """
    i1, i2, iyb = rule
    x1 = np.asarray(x1)
    x2 = np.asarray(x2)
    has_j = "j" in i1
    if not has_j:
        # broadcast product: @addmul! sy*y + sx*x1*x2 over the output letters
        letters = list(iyb)
        def expand(x, ix):
            sh = [x.shape[ix.index(c)] if c in ix else 1 for c in letters]
            perm = [ix.index(c) for c in letters if c in ix]
            return np.transpose(x, perm).reshape(sh) if x.ndim else x
        a = expand(x1, list(i1))
        b = expand(x2, list(i2))
        return addmul_(sy, y, sx, [a, b], alg)
    # contraction: canonical (l, i, j) @ (l, j, k) -> (l, i, k)
    def canon(x, ix, first, second):
        want = ["l", first, second]
        shape = [x.shape[ix.index(c)] if c in ix else 1 for c in want]
        perm = [ix.index(c) for c in want if c in ix]
        return np.transpose(x, perm).reshape(shape)
    A = canon(x1, list(i1), "i", "j")
    B = canon(x2, list(i2), "j", "k")
    f = alg.matmul(A, B)  # (l, i, k)
    present = [c for c in ["l", "i", "k"] if c in iyb]
    f = f.reshape([f.shape[["l", "i", "k"].index(c)] for c in present]) if f.ndim else f
    f = np.transpose(f, [present.index(c) for c in iyb])
    return _axpby_(y, f, sx, sy, alg)


def einsum_binary_(ix1, ix2, iy, x1, x2, y, sx, sy, size_dict, alg=REAL):
    """Binary ``einsum!`` (``src/einsum.jl:104-124``)."""
    c1, c2, cy, s1, s2, s3, i1, i2, iyb = analyze_binary(ix1, ix2, iy, size_dict)
    xs1 = simplifyto(ix1, c1, x1, size_dict, alg)
    xs2 = simplifyto(ix2, c2, x2, size_dict, alg)
    x1_ = reshape_f(xs1, s1)
    x2_ = reshape_f(xs2, s2)
    rule = (tuple(i1), tuple(i2), tuple(iyb))
    if list(cy) != list(iy):
        y_ = np.zeros(s3, dtype=y.dtype, order="F")
        binary_einsum_(rule, x1_, x2_, y_, alg.one(y.dtype), alg.zero(y.dtype), alg)
        y_ = reshape_f(y_, [size_dict[l] for l in cy])
        return einsum_unary_(cy, list(iy), y_, y, sx, sy, size_dict, alg)
    yv = reshape_f(y, s3)
    binary_einsum_(rule, x1_, x2_, yv, sx, sy, alg)
    y[...] = reshape_f(yv, y.shape)
    return y


def batched_gemm_(c1, c2, alpha, A, B, beta, C, alg=REAL):
    """``_batched_gemm!`` (``src/utils.jl:162-177``): per-batch (N|T)x(N|T) GEMM."""
    for l in range(A.shape[2]):
        a = A[:, :, l].T if c1 == "T" else A[:, :, l]
        b = B[:, :, l].T if c2 == "T" else B[:, :, l]
        f = alg.matmul(a, b)
        cv = C[:, :, l]
        _axpby_(cv, f, alpha, beta, alg)
        C[:, :, l] = cv
    return C


# ----------------------------------------------------------------------------
# loop_einsum (src/loop_einsum.jl:21-45, src/Core.jl:201-268)
# ----------------------------------------------------------------------------


def indices_and_locs(ixs, iy):
    """``indices_and_locs`` (``src/Core.jl:256-268``): inner labels first, then outer."""
    outer = _unique(iy)
    allx = [l for ix in ixs for l in ix]
    inner = []
    for l in allx:
        if l not in outer and l not in inner:
            inner.append(l)
    indices = inner + outer
    locs_xs = [[indices.index(l) for l in ix] for ix in ixs]
    locs_y = [outer.index(l) for l in iy]
    return inner, outer, locs_xs, locs_y


def einarray_value(ixs, iy, xs, size_dict, ind, alg=REAL):
    """``getindex(::EinArray, ind)`` = ``map_prod`` (``src/Core.jl:231-243``) with a
    0-based ``ind`` over (inner..., outer...)."""
    _, _, locs_xs, _ = indices_and_locs(ixs, iy)
    v = None
    for x, locs in zip(xs, locs_xs):
        e = np.asarray(x)[tuple(ind[l] for l in locs)]
        v = e if v is None else alg.mul(v, e)
    return v


def loop_einsum_(ixs, iy, xs, y, sx, sy, size_dict, alg=REAL):
    """``loop_einsum!`` (``src/loop_einsum.jl:21-45``): y <- sy*y, then for every
    outer index ``y[iy] += sx * sum_inner prod_i x_i``; products left to right."""
    inner, outer, locs_xs, locs_y = indices_and_locs([list(ix) for ix in ixs], list(iy))
    allsz = [size_dict[l] for l in inner + outer]
    nd = len(allsz)
    prod = None
    for x, locs in zip(xs, locs_xs):
        x = np.asarray(x)
        # take diagonals for repeated labels and broadcast into the full label space
        idx = []
        for loc in locs:
            sh = [1] * nd
            sh[loc] = allsz[loc]
            idx.append(np.arange(allsz[loc]).reshape(sh))
        v = x[tuple(idx)] if idx else np.broadcast_to(x, [1] * nd)
        prod = v if prod is None else alg.mul(prod, v)
    prod = np.broadcast_to(prod, allsz)
    dt = y.dtype
    acc = alg.sum(prod.astype(dt, copy=False), list(range(len(inner))))  # over outer labels
    with np.errstate(over="ignore", invalid="ignore"):
        if alg.iszero(sy):
            y[...] = alg.zero(dt)
        elif not alg.isone(sy):
            y[...] = alg.mul(sy, y)
        # y indexer: y dim d takes the outer index at locs_y[d]
        osz = [size_dict[l] for l in outer]
        idx = []
        for loc in locs_y:
            sh = [1] * len(osz)
            sh[loc] = osz[loc]
            idx.append(np.arange(osz[loc]).reshape(sh))
        if idx:
            cur = y[tuple(idx)]
            y[tuple(idx)] = alg.add(cur, alg.mul(sx, acc))
        else:
            y[...] = alg.add(y, alg.mul(sx, acc))
    return y


def loop_einsum(ixs, iy, xs, size_dict, alg=None):
    alg = algebra_for(xs[0], alg)
    y = get_output_array(xs, [size_dict[l] for l in iy], False)
    dt = y.dtype
    return loop_einsum_(ixs, iy, xs, y, alg.one(dt), alg.zero(dt), size_dict, alg)


# ----------------------------------------------------------------------------
# dispatch: einsum / einsum! (src/einsum.jl:24-50)
# ----------------------------------------------------------------------------


def einsum_(ixs, iy, xs, y, sx, sy, size_dict, alg=None):
    """``einsum!(ixs, iy, xs, y, sx, sy, size_dict)`` dispatch on the input count."""
    alg = algebra_for(y, alg)
    xs = [np.asarray(x) for x in xs]
    if len(xs) == 1:
        return einsum_unary_(list(ixs[0]), list(iy), xs[0], y, sx, sy, size_dict, alg)
    if len(xs) == 2:
        T = y.dtype
        x1, x2 = (x if x.dtype == T else x.astype(T) for x in xs)
        return einsum_binary_(list(ixs[0]), list(ixs[1]), list(iy), x1, x2, y, sx, sy, size_dict, alg)
    return loop_einsum_(ixs, iy, xs, y, sx, sy, size_dict, alg)


def einsum(ixs, iy, xs, size_dict=None, alg=None):
    """``einsum(code, xs, size_dict)`` (``src/einsum.jl:24-27``)."""
    xs = [np.asarray(x) for x in xs]
    if size_dict is None:
        size_dict = get_size_dict(ixs, xs)
    y = get_output_array(xs, [size_dict[l] for l in iy], False)
    a = algebra_for(y, alg)
    dt = y.dtype
    return einsum_(ixs, iy, xs, y, a.one(dt), a.zero(dt), size_dict, a)


# ----------------------------------------------------------------------------
# rule matcher (src/matchrule.jl), used only for the reference's 36-rule KAT
# ----------------------------------------------------------------------------


def _isunique(ix):
    """``_isunique`` (``src/matchrule.jl:84-97``), restated as written."""
    if len(ix) <= 1:
        return True
    if len(ix) == 2:
        return ix[0] != ix[1]
    if len(ix) == 3:
        a, b, c = ix
        return a != c and a != c and a != b
    return False


def _match_simple2(ix1, ix2, iy, n1, n2, ny):
    """``_match_simple2`` (``src/matchrule.jl:99-148``)."""
    R = lambda a, b, c: (tuple(a), tuple(b), tuple(c))
    if n1 == 0:
        if ny == n2 == 0:
            return R((), (), ())
        if ny == n2 == 1 and ix2[0] == iy[0]:
            return R((), "k", "k")
    elif n1 == 1:
        if n2 == 0 and ny == 1 and iy[0] == ix1[0]:
            return R("i", (), "i")
        if n2 == 1 and ny == 0 and ix1[0] == ix2[0]:
            return R("j", "j", ())
        if n2 == 1 and ny == 2:
            if iy[0] == ix1[0] and iy[1] == ix2[0]:
                return R("i", "k", "ik")
            if iy[0] == ix2[0] and iy[1] == ix1[0]:
                return R("i", "k", "ki")
        elif n2 == 2 and ny == 1:
            if ix2[0] == ix1[0] and ix2[1] == iy[0]:
                return R("j", "jk", "k")
            if ix2[0] == iy[0] and ix2[1] == ix1[0]:
                return R("j", "kj", "k")
    elif n1 == 2:
        if n2 == 1 and ny == 1:
            if ix1[0] == ix2[0] and ix1[1] == iy[0]:
                return R("ji", "j", "i")
            if ix1[0] == iy[0] and ix1[1] == ix2[0]:
                return R("ij", "j", "i")
        elif n2 == 2 and ny == 2:
            a, b = ix1[0], ix1[1]
            c, d = ix2[0], ix2[1]
            e, f = iy[0], iy[1]
            table = [
                (a == c and b == e and d == f, ("ji", "jk", "ik")),
                (a == d and b == e and c == f, ("ji", "kj", "ik")),
                (a == c and b == f and d == e, ("ji", "jk", "ki")),
                (a == d and b == f and c == e, ("ji", "kj", "ki")),
                (b == c and a == e and d == f, ("ij", "jk", "ik")),
                (b == d and a == e and c == f, ("ij", "kj", "ik")),
                (b == c and a == f and d == e, ("ij", "jk", "ki")),
                (b == d and a == f and c == e, ("ij", "kj", "ki")),
            ]
            for cond, r in table:
                if cond:
                    return R(*r)
    return None


def match_rule_binary(ix1, ix2, iy):
    """``match_rule_binary`` (``src/matchrule.jl:69-82``); None = DefaultRule."""
    n1, n2, ny = len(ix1), len(ix2), len(iy)
    if not _isunique(ix1) or not _isunique(ix2) or not _isunique(iy):
        return None
    if (n1 + n2 + ny) % 2 == 0:
        return _match_simple2(ix1, ix2, iy, n1, n2, ny)
    if n1 > 0 and n2 > 0 and ny > 0 and ix1[-1] == ix2[-1] == iy[-1]:
        r = _match_simple2(ix1, ix2, iy, n1 - 1, n2 - 1, ny - 1)
        if r is None:
            return None
        return (r[0] + ("l",), r[1] + ("l",), r[2] + ("l",))
    return None


# ----------------------------------------------------------------------------
# nested and sliced execution (src/einsequence.jl, src/slicing.jl)
# ----------------------------------------------------------------------------


@dataclass
class Node:
    """A contraction-tree node: a leaf (``tensorindex >= 0``) or an einsum over children.

    Mirrors ``DynamicNestedEinsum`` (``src/einsequence.jl:172-189``); tensor
    indices are 0-based here.
    """

    tensorindex: int = -1
    args: List["Node"] = field(default_factory=list)
    ixs: List[List[Any]] = field(default_factory=list)
    iy: List[Any] = field(default_factory=list)

    @property
    def isleaf(self):
        return self.tensorindex >= 0


def leaf(i):
    return Node(tensorindex=i)


def collect_ixs(ne, d=None):
    """``collect_ixs!`` (``src/einsequence.jl:348-359``)."""
    d = {} if d is None else d
    for i, a in enumerate(ne.args):
        if a.isleaf:
            d[a.tensorindex] = list(ne.ixs[i])
        else:
            collect_ixs(a, d)
    return d


def getixsv(ne):
    d = collect_ixs(ne)
    return [d[i] for i in sorted(d)]


def nested_einsum(ne, xs, size_dict, alg=None):
    """``einsum(::NestedEinsum, xs, size_dict)`` (``src/einsequence.jl:279-287``): post-order."""
    mxs = [xs[a.tensorindex] if a.isleaf else nested_einsum(a, xs, size_dict, alg) for a in ne.args]
    return einsum(ne.ixs, ne.iy, mxs, size_dict, alg)


def nested_einsum_(ne, xs, y, sx, sy, size_dict, alg=None):
    """``einsum!(::NestedEinsum, ...)`` (``src/einsequence.jl:270-278``)."""
    mxs = [xs[a.tensorindex] if a.isleaf else nested_einsum(a, xs, size_dict, alg) for a in ne.args]
    return einsum_(ne.ixs, ne.iy, mxs, y, sx, sy, size_dict, alg)


def parse_nested(s):
    """``ein"..."`` with parentheses -> Node tree (``src/einsequence.jl:9-86``,
    ``src/interfaces.jl:35-47``): the intermediate output of a child keeps the
    labels it shares with the parent output or with any sibling (``filliys!``)."""
    s = s.replace(" ", "").replace("\n", "")
    lhs, rhs = s.split("->")
    counter = [0]

    def parse(i):
        args, inds = [], []
        cur = []
        while i < len(lhs):
            c = lhs[i]
            if c == "(":
                i, sub = parse(i + 1)
                args.append(sub)
                for l in sub["inds"]:
                    if l not in inds:
                        inds.append(l)
                continue
            if c in "),":
                if cur:
                    args.append({"leaf": counter[0], "inds": cur})
                    counter[0] += 1
                    for l in cur:
                        if l not in inds:
                            inds.append(l)
                cur = []
                i += 1
                if c == ")":
                    return i, {"args": args, "inds": inds, "iy": []}
                continue
            if not c.isalpha():
                raise ValueError(f"parsing {s} failed, {c} is not a valid entry")
            cur.append(c)
            i += 1
        if cur:
            args.append({"leaf": counter[0], "inds": cur})
            counter[0] += 1
            for l in cur:
                if l not in inds:
                    inds.append(l)
        return i, {"args": args, "inds": inds, "iy": []}

    if lhs.count("(") != lhs.count(")"):
        raise ValueError(f"Parentheses don't pair up in {lhs}")
    _, out = parse(0)
    out["iy"] = list(rhs)

    def fill(n):
        for i, a in enumerate(n["args"]):
            if "leaf" in a:
                continue
            for l in a["inds"]:
                if l in n["iy"] and l not in a["iy"]:
                    a["iy"].append(l)
            for j, b in enumerate(n["args"]):
                if i == j:
                    continue
                for l in a["inds"]:
                    if l in b["inds"] and l not in a["iy"]:
                        a["iy"].append(l)
            fill(a)

    fill(out)

    def build(n):
        args, ixs = [], []
        for a in n["args"]:
            if "leaf" in a:
                args.append(leaf(a["leaf"]))
                ixs.append(list(a["inds"]))
            else:
                args.append(build(a))
                ixs.append(list(a["iy"]))
        return Node(args=args, ixs=ixs, iy=list(n["iy"]))

    return build(out)


def drop_slicedim(ne, slicing):
    """``drop_slicedim`` (``src/slicing.jl:139-145``)."""
    if ne.isleaf:
        return ne
    return Node(args=[drop_slicedim(a, slicing) for a in ne.args],
                ixs=[[l for l in ix if l not in slicing] for ix in ne.ixs],
                iy=[l for l in ne.iy if l not in slicing])


def slice_iterator(slicing, size_dict):
    """``SliceIterator`` (``src/slicing.jl:37-71``): CartesianIndices order, first
    sliced label fastest; yields 0-based slicemaps."""
    sizes = [size_dict[l] for l in slicing]
    for ci in itertools.product(*[range(s) for s in reversed(sizes)]):
        yield dict(zip(slicing, reversed(ci)))


def take_slice(x, ix, slicemap):
    """``take_slice`` (``src/slicing.jl:78-85``): copy of the slice."""
    sl = tuple(slicemap[l] if l in slicemap else slice(None) for l in ix)
    return np.array(np.asarray(x)[sl], order="F")


def sliced_einsum(slicing, ne, xs, size_dict, alg=None, acc_dtype=None):
    """``einsum(::SlicedEinsum, xs, size_dict)`` (``src/slicing.jl:123-137``).

    ``acc_dtype`` (e.g. float64) optionally accumulates the slices in a wider
    type; the reference accumulates in the output eltype.
    """
    if not slicing:
        return nested_einsum(ne, xs, size_dict, alg)
    ixsv = getixsv(ne)
    iyv = list(ne.iy)
    res = get_output_array(xs, [size_dict[l] for l in iyv], True, alg)
    if acc_dtype is not None:
        res = res.astype(acc_dtype)
    sd = dict(size_dict)
    for l in slicing:
        sd[l] = 1
    eins = drop_slicedim(ne, slicing)
    a = algebra_for(res, alg)
    for sm in slice_iterator(slicing, size_dict):
        xsi = [take_slice(x, ix, sm) for x, ix in zip(xs, ixsv)]
        resi = nested_einsum(eins, xsi, sd, alg)
        sl = tuple(sm[l] if l in sm else slice(None) for l in iyv)
        res[sl] = a.add(res[sl], resi.astype(res.dtype))
    return res


def sliced_partial(slicing, ne, xs, size_dict, begin, end, alg=None, acc_dtype=None):
    """The body of ``einsum(::SlicedEinsum)`` (``src/slicing.jl:123-137``) over
    the slices ``begin..end-1`` of the ``SliceIterator`` order only: the
    algebra's zero everywhere, then every slice's tree value added at its
    sliced output positions.  Partials of disjoint ranges combine with the
    algebra's addition (sum; max for max-plus; or for Bool) into the full
    cross-slice result."""
    ixsv = getixsv(ne)
    iyv = list(ne.iy)
    res = get_output_array(xs, [size_dict[l] for l in iyv], True, alg)
    if acc_dtype is not None:
        res = res.astype(acc_dtype)
    sd = dict(size_dict)
    for l in slicing:
        sd[l] = 1
    eins = drop_slicedim(ne, slicing)
    a = algebra_for(res, alg)
    for k, sm in enumerate(slice_iterator(slicing, size_dict)):
        if k < begin or k >= end:
            continue
        xsi = [take_slice(x, ix, sm) for x, ix in zip(xs, ixsv)]
        resi = nested_einsum(eins, xsi, sd, alg)
        sl = tuple(sm[l] if l in sm else slice(None) for l in iyv)
        res[sl] = a.add(res[sl], resi.astype(res.dtype))
    return res


# ----------------------------------------------------------------------------
# autodiff (src/autodiff.jl:24-33, src/bp.jl:24-160)
# ----------------------------------------------------------------------------


def einsum_grad(ixs, xs, iy, size_dict, dy, i, alg=None):
    """``einsum_grad`` (``src/autodiff.jl:24-30``): contract conj(dy) in place of
    input ``i`` to ``ixs[i]``, conjugate, project to the input's eltype."""
    nixs = [list(ix) for ix in ixs]
    nixs[i] = list(iy)
    nxs = list(xs)
    nxs[i] = np.conj(dy) if np.iscomplexobj(dy) else dy
    y = einsum(nixs, list(ixs[i]), nxs, size_dict, alg)
    y = np.conj(y) if np.iscomplexobj(y) else y
    if not np.iscomplexobj(xs[i]) and np.iscomplexobj(y):
        y = y.real
    return y.astype(np.asarray(xs[i]).dtype, copy=False)


def cached_einsum(ne, xs, size_dict, alg=None):
    """``cached_einsum`` (``src/bp.jl:33-48``): returns (content, children caches)."""
    if ne.isleaf:
        return (np.asarray(xs[ne.tensorindex]), [])
    caches = [cached_einsum(a, xs, size_dict, alg) for a in ne.args]
    y = einsum(ne.ixs, ne.iy, [c[0] for c in caches], size_dict, alg)
    return (y, caches)


def back_propagate(ne, cache, dy, size_dict, alg=None):
    """``back_propagate`` (``src/bp.jl:79-96``) with ``einsum_backward_rule``."""
    if ne.isleaf:
        return (dy, [])
    xs = [c[0] for c in cache[1]]
    dxs = [einsum_grad(ne.ixs, xs, ne.iy, size_dict, dy, i, alg) for i in range(len(xs))]
    return (dy, [back_propagate(a, c, dx, size_dict, alg) for a, c, dx in zip(ne.args, cache[1], dxs)])


def cost_and_gradient(ne, xs, dy=None, alg=None):
    """``cost_and_gradient`` (``src/bp.jl:122-130``): forward with all
    intermediates cached, then the reverse sweep; gradients on the leaves."""
    size_dict = get_size_dict(getixsv(ne), xs)
    if dy is None:
        y_shape = [size_dict[l] for l in ne.iy]
        dt = promote_type(*[np.asarray(x).dtype for x in xs])
        dy = np.ones(y_shape, dtype=dt, order="F")
        assert dy.ndim == 0, "The output must be a scalar!"
    cache = cached_einsum(ne, xs, size_dict, alg)
    tree = back_propagate(ne, cache, dy, size_dict, alg)
    grads = [None] * len(xs)

    def extract(n, t):
        if n.isleaf:
            grads[n.tensorindex] = t[0]
        else:
            for a, c in zip(n.args, t[1]):
                extract(a, c)

    extract(ne, tree)
    return np.array(cache[0]), grads


# ----------------------------------------------------------------------------
# contraction complexity (OMEinsumContractionOrders: flop/peak_memory) for KATs
# ----------------------------------------------------------------------------


def node_flop(ixs, iy, size_dict):
    labels = _unique([l for ix in ixs for l in ix] + list(iy))
    return int(np.prod([size_dict[l] for l in labels], dtype=np.float64))


def contraction_complexity(ne, size_dict):
    """(tc, sc, rwc) in log2 (OMEinsumContractionOrders ``contraction_complexity``,
    pinned by ``test/einsequence.jl:198-206``)."""
    tc, sc, rw = 0.0, 0.0, 0.0

    def rec(n):
        nonlocal tc, sc, rw
        for a in n.args:
            if not a.isleaf:
                rec(a)
        tc += node_flop(n.ixs, n.iy, size_dict)
        outsz = float(np.prod([size_dict[l] for l in n.iy])) if n.iy else 1.0
        sc = max(sc, outsz)
        rw += outsz + sum(float(np.prod([size_dict[l] for l in ix])) if ix else 1.0 for ix in n.ixs)

    rec(ne)
    return math.log2(tc), math.log2(sc), math.log2(rw)


def peak_memory(ne, size_dict):
    """``peak_memory`` (OMEinsumContractionOrders; pinned by
    ``test/einsequence.jl:205``): inputs plus live intermediates, in elements."""
    sz = lambda ix: int(np.prod([size_dict[l] for l in ix], dtype=np.int64)) if ix else 1

    def rec(n):
        # returns (peak during evaluation of n, size of n's output)
        cur = 0
        peak = 0
        for ix, a in zip(n.ixs, n.args):
            if a.isleaf:
                cur += sz(ix)
                peak = max(peak, cur)
            else:
                p, o = rec(a)
                peak = max(peak, cur + p)
                cur += o
        peak = max(peak, cur + sz(n.iy))
        return peak, sz(n.iy)

    return rec(ne)[0]
