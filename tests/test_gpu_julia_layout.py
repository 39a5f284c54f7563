"""The contraction-tree entry points driven with arrays laid out exactly as the
Julia extension builds them (omeinsum.jl_b200/julia/ext/B200Ext.jl,
flatten_tree): input labels in getixsv order first, node references in
post-order with a leaf of 1-based tensorindex t written as -t, Char labels
mapped to ids in first-seen order, column-major device buffers, a non-NULL
context passed to ome_plan_create.  Results against the oracle's restatement
of src/einsequence.jl, src/slicing.jl and src/bp.jl.

A CPU test checks that every library symbol the Julia files call is declared
in include/ome_b200.h.
"""
import ctypes as C
import glob
import os
import re

import numpy as np
import pytest
import torch

import ome_oracle as O
import omeinsum_b200 as ome
from omeinsum_b200 import _lib
from helpers import gen, relerr

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
JULIA = os.path.join(ROOT, "omeinsum.jl_b200", "julia")


def julia_flatten(ne, slicing, size_dict):
    """B200Ext.flatten_tree, line for line (0-based node numbers, leaves -t)."""
    ids = {}

    def lm(l):
        return ids.setdefault(l, len(ids))

    ixsv = ne.getixsv()
    input_nlabels = [len(ix) for ix in ixsv]
    input_labels = [lm(l) for ix in ixsv for l in ix]
    node_nargs, node_args, node_niy, node_iy = [], [], [], []

    def rec(n):
        refs = [-(a.tensorindex + 1) if a.isleaf else rec(a) for a in n.args]
        iy = n.eins.iy
        node_nargs.append(len(refs))
        node_args.extend(refs)
        node_niy.append(len(iy))
        node_iy.extend(lm(l) for l in iy)
        return len(node_nargs) - 1

    rec(ne)
    sliced = [lm(l) for l in slicing]
    labels = list(ids)
    return dict(nin=len(ixsv), input_nlabels=input_nlabels, input_labels=input_labels, node_nargs=node_nargs,
                node_args=node_args, node_niy=node_niy, node_iy=node_iy, label_ids=[ids[l] for l in labels],
                label_extents=[size_dict[l] for l in labels], sliced=sliced)


def arr(T, v):
    return (T * max(len(v), 1))(*v)


def oracle_tree(ne):
    if ne.isleaf:
        return O.leaf(ne.tensorindex)
    return O.Node(args=[oracle_tree(a) for a in ne.args], ixs=[list(ix) for ix in ne.eins.ixs], iy=list(ne.eins.iy))


def colmajor(x):
    return torch.from_numpy(np.array(x, order="F")).cuda()


def plan_and_run(ne, slicing, sd, xs, dtype, grad=False, dy=None):
    lib = _lib.load()
    f = julia_flatten(ne, slicing, sd)
    ctx = C.c_void_p()
    _lib.check(lib.ome_ctx_create(torch.cuda.current_device(), 64 << 20, C.byref(ctx)))
    plan = C.c_void_p()
    try:
        _lib.check(lib.ome_plan_create(
            ctx, dtype, f["nin"], arr(C.c_int32, f["input_nlabels"]), arr(C.c_int32, f["input_labels"]),
            len(f["node_nargs"]), arr(C.c_int32, f["node_nargs"]), arr(C.c_int32, f["node_args"]),
            arr(C.c_int32, f["node_niy"]), arr(C.c_int32, f["node_iy"]), len(f["label_ids"]),
            arr(C.c_int32, f["label_ids"]), arr(C.c_int64, f["label_extents"]), len(f["sliced"]),
            arr(C.c_int32, f["sliced"]), 0, C.byref(plan)))
        fb, gb = C.c_size_t(), C.c_size_t()
        _lib.check(lib.ome_plan_peak_bytes(plan, C.byref(fb), C.byref(gb)))
        need = (gb if grad else fb).value
        if need > (64 << 20):   # grow the context as the Julia side does (ctx(min_bytes))
            lib.ome_ctx_destroy(ctx)
            ctx = C.c_void_p()
            _lib.check(lib.ome_ctx_create(torch.cuda.current_device(), need, C.byref(ctx)))
        dxs = [colmajor(x) for x in xs]
        ptrs = (C.c_void_p * len(dxs))(*[t.data_ptr() for t in dxs])
        shape = [sd[l] for l in ne.getiyv()]
        y = colmajor(np.zeros(shape, dtype=xs[0].dtype))
        stream = C.c_void_p(torch.cuda.current_stream().cuda_stream)
        if not grad:
            one = (C.c_ubyte * 16)()
            zero = (C.c_ubyte * 16)()
            C.memmove(one, np.array([1], dtype=xs[0].dtype).tobytes(), xs[0].itemsize)
            _lib.check(lib.ome_plan_execute(ctx, plan, stream, ptrs, C.c_void_p(y.data_ptr()), one, zero))
            torch.cuda.synchronize()
            return y.cpu().numpy(), None
        gs = [torch.empty_like(t) for t in dxs]
        gp = (C.c_void_p * len(gs))(*[g.data_ptr() for g in gs])
        dyp = None if dy is None else colmajor(dy)
        _lib.check(lib.ome_plan_gradient(ctx, plan, stream, ptrs, None if dyp is None else C.c_void_p(dyp.data_ptr()),
                                         C.c_void_p(y.data_ptr()), gp))
        torch.cuda.synchronize()
        return y.cpu().numpy(), [g.cpu().numpy() for g in gs]
    finally:
        if plan:
            lib.ome_plan_destroy(plan)
        lib.ome_ctx_destroy(ctx)


@pytest.mark.gpu
@pytest.mark.parametrize("dt", ["f64", "f32", "i64"])
def test_nested_tree_julia_layout(dt):
    rng = np.random.default_rng(8)
    ne = ome.ein("((ij,jk),(kl,lm)),mi->")
    sd = {l: 3 + (ord(l) % 5) for l in "ijklm"}
    xs = [gen(rng, [sd[a], sd[b]], dt) for a, b in ["ij", "jk", "kl", "lm", "mi"]]
    got, _ = plan_and_run(ne, [], sd, xs, {"f64": _lib.F64, "f32": _lib.F32, "i64": _lib.I64}[dt])
    want = O.nested_einsum(oracle_tree(ne), xs, sd)
    if dt == "i64":
        assert np.array_equal(got, want)
    else:
        assert relerr(got, want) <= (1e-12 if dt == "f64" else 1e-5)


@pytest.mark.gpu
def test_sliced_tree_julia_layout():
    rng = np.random.default_rng(9)
    ne = ome.ein("(ij,jk),(kl,lm)->im")
    sd = {"i": 5, "j": 6, "k": 4, "l": 7, "m": 3}
    xs = [gen(rng, [sd[a], sd[b]], "f64") for a, b in ["ij", "jk", "kl", "lm"]]
    got, _ = plan_and_run(ne, ["k", "j"], sd, xs, _lib.F64)
    want = O.sliced_einsum(["k", "j"], oracle_tree(ne), xs, sd)
    assert relerr(got, want) <= 1e-12


@pytest.mark.gpu
def test_cost_and_gradient_julia_layout():
    rng = np.random.default_rng(10)
    ne = ome.ein("(ij,jk),ki->")
    sd = {"i": 4, "j": 5, "k": 6}
    xs = [gen(rng, [sd[a], sd[b]], "f64") for a, b in ["ij", "jk", "ki"]]
    cost, grads = plan_and_run(ne, [], sd, xs, _lib.F64, grad=True)
    c0, g0 = O.cost_and_gradient(oracle_tree(ne), xs)
    assert relerr(cost, c0) <= 1e-12
    for g, w in zip(grads, g0):
        assert relerr(g, w) <= 1e-12


def test_julia_files_call_only_declared_symbols():
    """Every `sym(:ome_...)` the Julia extension resolves is declared in the header."""
    header = open(os.path.join(ROOT, "include", "ome_b200.h")).read()
    declared = set(re.findall(r"OME_API\s+[\w\s\*]+?\b(ome_\w+)\s*\(", header))
    called = set()
    for f in glob.glob(os.path.join(JULIA, "**", "*.jl"), recursive=True):
        called |= set(re.findall(r"sym\(:(ome_\w+)\)", open(f).read()))
    assert called, "no library calls found in the Julia files"
    assert called <= declared, sorted(called - declared)
    lib = _lib.load()
    for n in called:
        assert hasattr(lib, n), n
