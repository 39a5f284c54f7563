"""Contraction-tree execution (NestedEinsum, SlicedEinsum, cost_and_gradient)
through the library's plan API (ome_plan_* in include/ome_b200.h).

A tree is flattened once into post-order arrays, planned once per (tree,
sizes, slicing, dtype, precision) and cached; evaluation is one library call
that runs every node from the device workspace.
"""
from __future__ import annotations

import ctypes as C
from typing import Any, Dict, List, Sequence, Tuple

import torch

from . import _lib
from ._lib import ArgumentError, check
from .backends import get_einsum_backend
from .core import NestedEinsum, SlicedEinsum, get_size_dict
from .engine import (TropicalTensor, _alloc, _f_contig, _LabelMap, _Prepared, _require_b200, _scalar_buf,
                     _stream)


class Plan:
    """A planned contraction tree in the library (owns an ome_plan*)."""

    def __init__(self, ne: NestedEinsum, slicing: Sequence[Any], size_dict: Dict[Any, int], ome_dtype: int,
                 prec: int):
        lm = _LabelMap()
        nodes: List[Tuple[List[int], List[int]]] = []
        inputs: Dict[int, List[int]] = {}

        def rec(n: NestedEinsum) -> int:
            refs = []
            for ix, a in zip(n.eins.ixs, n.args):
                if a.isleaf:
                    inputs[a.tensorindex] = [lm(l) for l in ix]
                    refs.append(-a.tensorindex - 1)
                else:
                    refs.append(rec(a))
            nodes.append((refs, [lm(l) for l in n.eins.iy]))
            return len(nodes) - 1

        rec(ne)
        self.ninputs = len(inputs)
        if sorted(inputs) != list(range(self.ninputs)):
            raise ArgumentError("leaf tensor indices must be 0..n-1, each used once")
        for l in slicing:
            lm(l)
        self.labels = lm.ids
        self.out_labels = list(ne.eins.iy)
        in_n = [len(inputs[t]) for t in range(self.ninputs)]
        in_l = [x for t in range(self.ninputs) for x in inputs[t]]
        nn = [len(r) for r, _ in nodes]
        na = [x for r, _ in nodes for x in r]
        ny = [len(y) for _, y in nodes]
        nyl = [x for _, y in nodes for x in y]
        lab_ids = list(range(len(lm.ids)))
        inv = {v: k for k, v in lm.ids.items()}
        for i in lab_ids:
            if inv[i] not in size_dict:
                raise ArgumentError(f"label {inv[i]} has no size")
        exts = [int(size_dict[inv[i]]) for i in lab_ids]
        sl = [lm.ids[l] for l in slicing]
        arr = lambda T, v: (T * max(len(v), 1))(*v)
        h = C.c_void_p()
        check(_lib.load().ome_plan_create(
            None, ome_dtype, self.ninputs, arr(C.c_int32, in_n), arr(C.c_int32, in_l), len(nodes),
            arr(C.c_int32, nn), arr(C.c_int32, na), arr(C.c_int32, ny), arr(C.c_int32, nyl), len(lab_ids),
            arr(C.c_int32, lab_ids), arr(C.c_int64, exts), len(sl), arr(C.c_int32, sl), prec, C.byref(h)))
        self.handle = h
        fb, gb = C.c_size_t(), C.c_size_t()
        check(_lib.load().ome_plan_peak_bytes(h, C.byref(fb), C.byref(gb)))
        self.forward_bytes = fb.value
        self.grad_bytes = gb.value
        self.ome_dtype = ome_dtype

    def __del__(self):
        try:
            if self.handle:
                _lib.load().ome_plan_destroy(self.handle)
        except Exception:
            pass


_CACHE: Dict[Any, Plan] = {}


def _tree_key(ne: NestedEinsum):
    if ne.isleaf:
        return ne.tensorindex
    return (tuple(_tree_key(a) for a in ne.args), tuple(map(tuple, ne.eins.ixs)), tuple(ne.eins.iy))


def get_plan(code, size_dict, ome_dtype, prec) -> Plan:
    if isinstance(code, SlicedEinsum):
        ne, slicing = code.eins, list(code.slicing)
    else:
        ne, slicing = code, []
    labels = set(l for ix in ne.getixsv() for l in ix) | set(ne.getiyv())
    key = (_tree_key(ne), tuple(slicing), tuple(sorted((repr(l), size_dict[l]) for l in labels if l in size_dict)),
           ome_dtype, prec)
    p = _CACHE.get(key)
    if p is None:
        p = Plan(ne, slicing, size_dict, ome_dtype, prec)
        _CACHE[key] = p
    return p


def _ptrs(ts: Sequence[torch.Tensor]):
    return (C.c_void_p * len(ts))(*[t.data_ptr() for t in ts])


def run_tree(code, xs, size_dict=None, y=None, sx=True, sy=False):
    """einsum / einsum! for NestedEinsum and SlicedEinsum."""
    be = _require_b200()
    ne = code.eins if isinstance(code, SlicedEinsum) else code
    if size_dict is None:
        size_dict = get_size_dict(code.getixsv(), xs)
    if ne.isleaf:
        raise ArgumentError("a bare leaf is not a contraction")
    out_dtype = None
    if y is not None:
        out_dtype = (y.data if isinstance(y, TropicalTensor) else y).dtype
    p = _Prepared(xs, out_dtype=out_dtype)
    plan = get_plan(code, size_dict, p.ome, be.prec)
    dev = p.device
    ctx = _lib.context(dev.index, plan.forward_bytes)
    ins = [_f_contig(t) for t in p.tensors]
    shape = [size_dict[l] for l in ne.eins.iy]
    if y is None:
        yt = _alloc(shape, p.dtype, dev)
    else:
        yt = y.data if isinstance(y, TropicalTensor) else y
        if tuple(yt.shape) != tuple(shape):
            raise _lib.DimensionMismatch(f"output shape {tuple(yt.shape)} != {tuple(shape)}")
    work = yt if (y is None or tuple(yt.stride()) == tuple(_f_contig(yt).stride())) else _f_contig(yt)
    with torch.cuda.device(dev):
        check(_lib.load().ome_plan_execute(ctx.handle, plan.handle, _stream(dev), _ptrs(ins), work.data_ptr(),
                                           _scalar_buf(p.ome, sx), _scalar_buf(p.ome, sy)))
    if work is not yt:
        yt.copy_(work)
    if y is not None:
        return y
    return p.wrap(yt)


def tree_gradient(code, xs, dy=None):
    """cost_and_gradient on the device: forward with cached intermediates, then
    einsum_grad per node (src/bp.jl:99-130)."""
    be = _require_b200()
    ne = code.eins if isinstance(code, SlicedEinsum) else code
    if isinstance(code, NestedEinsum) or isinstance(code, SlicedEinsum):
        pass
    else:
        # a flat EinCode: a one-node tree
        ne = NestedEinsum([NestedEinsum(i) for i in range(len(code.ixs))], code)
    size_dict = get_size_dict(ne.getixsv(), xs)
    p = _Prepared(xs)
    plan = get_plan(ne, size_dict, p.ome, be.prec)
    dev = p.device
    ctx = _lib.context(dev.index, plan.grad_bytes)
    ins = [_f_contig(t) for t in p.tensors]
    shape = [size_dict[l] for l in ne.eins.iy]
    yt = _alloc(shape, p.dtype, dev)
    dxs = [_alloc(t.shape, p.dtype, dev) for t in ins]
    dyp = None
    if dy is not None:
        dyt = dy.data if isinstance(dy, TropicalTensor) else torch.as_tensor(dy)
        dyt = _f_contig(dyt.to(device=dev, dtype=p.dtype))
        if tuple(dyt.shape) != tuple(shape):
            raise _lib.DimensionMismatch("dy has the wrong shape")
        dyp = dyt
    elif len(shape) != 0:
        raise ArgumentError(f"The output must be a scalar! Or you need to feed the gradient manually. Got: {len(shape)}!")
    with torch.cuda.device(dev):
        check(_lib.load().ome_plan_gradient(ctx.handle, plan.handle, _stream(dev), _ptrs(ins),
                                            dyp.data_ptr() if dyp is not None else None, yt.data_ptr(),
                                            _ptrs(dxs)))
    return p.wrap(yt), [p.wrap(d) for d in dxs]
