"""Batched contractions of uneven shapes: one persistent grouped launch.

``BatchedEinsum(code, xs_list)`` binds a list of input pairs (each contracted
by the same binary ``code``, with its own extents) and their outputs to one
library batch (``ome_batch_*`` in include/ome_b200.h).  ``run()`` issues a
single grouped kernel for all of them; ``graph()`` captures that launch in a
CUDA graph.  This replaces a loop of ``einsum`` calls, one launch each, e.g.
the 8192 transfer contractions of an MPS sweep.  Inputs are used in
column-major (Julia) layout; tensors in another layout are copied once at
construction.
"""
from __future__ import annotations

import ctypes as C
from typing import Any, List, Sequence

import torch

from . import _lib
from ._lib import ArgumentError, check
from .core import EinCode, get_size_dict
from .engine import _alloc, _f_contig, _LabelMap, _Prepared, _require_b200, _scalar_buf, _stream, _tensor_struct


class BatchedEinsum:
    def __init__(self, code: EinCode, xs_list: Sequence[Sequence[Any]], ys: Sequence[torch.Tensor] | None = None,
                 tile_config: int = -1):
        _require_b200()
        if len(code.ixs) != 2:
            raise ArgumentError("BatchedEinsum takes a binary code")
        if len(xs_list) == 0:
            raise ArgumentError("empty batch")
        self.code = code
        self.inputs: List[List[torch.Tensor]] = []
        self.outputs: List[torch.Tensor] = []
        dtype = None
        for i, xs in enumerate(xs_list):
            p = _Prepared(xs, out_dtype=dtype)
            dtype = p.dtype
            if p.host:
                raise ArgumentError("BatchedEinsum needs device tensors")
            self.ome = p.ome
            self.device = p.device
            ts = [_f_contig(t) for t in p.tensors]  # column-major (Julia layout): a one-time copy otherwise
            sd = get_size_dict(code.ixs, ts)
            self.inputs.append(ts)
            if ys is None:
                self.outputs.append(_alloc([sd[l] for l in code.iy], p.dtype, p.device))
            else:
                self.outputs.append(ys[i])
        self.tropical = p.tropical
        lm = _LabelMap()
        keep: list = []
        n = len(xs_list)
        t1, t2, ty = (_lib.Tensor * n)(), (_lib.Tensor * n)(), (_lib.Tensor * n)()
        l1 = [lm(l) for l in code.ixs[0]]
        l2 = [lm(l) for l in code.ixs[1]]
        lyy = [lm(l) for l in code.iy]
        for i in range(n):
            t1[i] = _tensor_struct(self.inputs[i][0], l1, keep)
            t2[i] = _tensor_struct(self.inputs[i][1], l2, keep)
            ty[i] = _tensor_struct(self.outputs[i], lyy, keep)
        self.ctx = _lib.context(self.device.index)
        h = C.c_void_p()
        with torch.cuda.device(self.device):
            check(_lib.load().ome_batch_create(self.ctx.handle, _stream(self.device), self.ome, n, t1, t2, ty,
                                               int(tile_config), C.byref(h)))
        self.handle = h
        cfg = C.c_int32()
        us = (C.c_float * 4)()
        check(_lib.load().ome_batch_info(h, C.byref(cfg), us))
        self.tile_config = cfg.value
        self.tuned_us = list(us)

    def run(self, sx=True, sy=False) -> List[torch.Tensor]:
        with torch.cuda.device(self.device):
            check(_lib.load().ome_batch_run(self.ctx.handle, self.handle, _stream(self.device),
                                            _scalar_buf(self.ome, sx), _scalar_buf(self.ome, sy)))
        return self.outputs

    def __del__(self):
        try:
            if self.handle:
                _lib.load().ome_batch_destroy(self.handle)
        except Exception:
            pass


def capture_graph(fn) -> "torch.cuda.CUDAGraph":
    """Capture ``fn()`` (e.g. a sequence of BatchedEinsum.run calls) in a CUDA graph."""
    fn()  # warm-up outside the capture
    torch.cuda.synchronize()
    g = torch.cuda.CUDAGraph()
    with torch.cuda.graph(g):
        fn()
    return g


class BatchGraph:
    """A CUDA graph of grouped launches built by the library
    (``ome_batch_graph_create``): ``BatchGraph([b1, b2])`` captures b1.run()
    then b2.run() once; ``launch()`` replays them with one call.  The same
    capture that ``capture_graph`` makes through torch, available to a C or
    Julia caller of the ABI.  sxs / sys: per batch scalars (default 1, 0)."""

    def __init__(self, batches: Sequence[BatchedEinsum], sxs=None, sys=None):
        if len(batches) == 0:
            raise ArgumentError("empty graph")
        self.batches = list(batches)   # the graph reads their tables and tensors
        dev = self.batches[0].device
        self.device = dev
        n = len(self.batches)
        hs = (C.c_void_p * n)(*[b.handle.value for b in self.batches])
        keep = []

        def scal(vals):
            if vals is None:
                return None
            bufs = [_scalar_buf(b.ome, v) for b, v in zip(self.batches, vals)]
            keep.extend(bufs)
            return (C.c_void_p * n)(*[C.cast(x, C.c_void_p) for x in bufs])

        g = C.c_void_p()
        with torch.cuda.device(dev):
            check(_lib.load().ome_batch_graph_create(self.batches[0].ctx.handle, _stream(dev), n, hs, scal(sxs),
                                                     scal(sys), C.byref(g)))
        self.handle = g

    def launch(self):
        with torch.cuda.device(self.device):
            check(_lib.load().ome_graph_launch(self.handle, _stream(self.device)))
        return [b.outputs for b in self.batches]

    def __del__(self):
        try:
            if self.handle:
                _lib.load().ome_graph_destroy(self.handle)
        except Exception:
            pass
