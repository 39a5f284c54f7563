"""Slice sharding of a SlicedEinsum across GPUs (one process per GPU).

The reference evaluates the slices of a ``SlicedEinsum`` one after another
(``src/slicing.jl:118-137``); its only multi-device code copies slices through
the host (``examples/slicing_multigpu.jl:54-75``).  Here the slice index
space 0..nslices-1 (``SliceIterator`` order, first sliced label fastest,
``src/slicing.jl:37-50``) is cut into one contiguous range per rank.  Each
rank contracts its range on its own GPU into a partial of the full output
(``ome_plan_execute_slices``: FP64 for FP32/FP64 networks, complex128 for
complex64 ones, so the cross-slice sum keeps the single-GPU accumulation
type), the partials meet in ONE all-reduce (NCCL over NVLink on GPUs;
``gloo`` works the same for host tensors), and every rank applies
``y <- sy*y + sx*partial`` (``ome_plan_finish``).  There is no other exchange:
inputs are replicated, intermediates never leave their GPU.

Partials combine with the algebra's addition: a sum for real, complex and
Int64 networks, a max for Tropical (max-plus) and Bool (or-and) ones
(``ome_plan_partial_info``).  NaN in a max-plus partial follows the
collective library's max, not Julia's NaN-propagating ``max``.
"""
from __future__ import annotations

import ctypes as C
from typing import Any, Optional, Tuple

import torch
import torch.distributed as dist

from . import _lib
from ._lib import ArgumentError, check
from .core import SlicedEinsum, get_size_dict
from .engine import TropicalTensor, _alloc, _f_contig, _Prepared, _require_b200, _scalar_buf, _stream, _to_host
from .plan import _ptrs, get_plan

SUM, MAX = 0, 1

_PARTIAL_TORCH = {
    _lib.F32: torch.float32, _lib.F64: torch.float64, _lib.C32: torch.complex64, _lib.C64: torch.complex128,
    _lib.I64: torch.int64, _lib.BOOL: torch.bool, _lib.TROP_F32: torch.float32, _lib.TROP_F64: torch.float64,
}


def slice_range(nslices: int, rank: int, world: int) -> Tuple[int, int]:
    """Contiguous slice range [begin, end) of ``rank``: the first
    ``nslices % world`` ranks take one slice more than the others."""
    if world < 1 or not 0 <= rank < world:
        raise ArgumentError(f"rank {rank} outside a world of {world}")
    q, r = divmod(int(nslices), world)
    b = rank * q + min(rank, r)
    return b, b + q + (1 if rank < r else 0)


def _group_rank_world(group) -> Tuple[int, int]:
    if not dist.is_available() or not dist.is_initialized():
        return 0, 1
    return dist.get_rank(group), dist.get_world_size(group)


def _flat(t: torch.Tensor) -> torch.Tensor:
    """1-D view of a dense tensor's storage, row- or column-major
    (collectives want C-contiguous tensors; the partials are Julia-layout)."""
    if t.dim() <= 1 or t.is_contiguous():
        return t.view(-1)
    return t.permute(*range(t.dim() - 1, -1, -1)).reshape(-1)


def allreduce_partial(partial: torch.Tensor, op: int, group=None) -> torch.Tensor:
    """Combine the ranks' partials in place: elementwise sum (op 0) or max
    (op 1).  Complex partials reduce as (re, im) pairs; Bool ones as bytes.
    Without an initialised process group there is nothing to combine."""
    if not dist.is_available() or not dist.is_initialized():
        return partial
    rop = dist.ReduceOp.SUM if op == SUM else dist.ReduceOp.MAX
    flat = _flat(partial)
    if flat.data_ptr() != partial.data_ptr() and partial.numel() > 0:
        raise ArgumentError("partial must be a dense row- or column-major tensor")
    if partial.dtype == torch.bool:
        t = flat.to(torch.uint8)
        dist.all_reduce(t, op=rop, group=group)
        flat.copy_(t.to(torch.bool))
    elif partial.is_complex():
        if op != SUM:
            raise ArgumentError("complex partials only combine by sum")
        dist.all_reduce(torch.view_as_real(flat), op=rop, group=group)
    else:
        dist.all_reduce(flat, op=rop, group=group)
    return partial


class ShardedSlices:
    """A SlicedEinsum planned for slice sharding on this rank's GPU.

    ``partial(xs)`` runs this rank's slice range into a fresh partial buffer,
    ``reduce`` all-reduces it over ``group`` and ``finish`` writes
    ``y <- sy*y + sx*partial``; ``__call__`` does the three in order.  Every
    rank of the group must call the same steps in the same order."""

    def __init__(self, code: SlicedEinsum, xs, size_dict=None, group=None, prec: Optional[int] = None):
        be = _require_b200()
        if not isinstance(code, SlicedEinsum):
            raise ArgumentError("slice sharding takes a SlicedEinsum")
        self.code = code
        self.group = group
        self.rank, self.world = _group_rank_world(group)
        self.size_dict = size_dict if size_dict is not None else get_size_dict(code.getixsv(), xs)
        p = _Prepared(xs)
        self.ome = p.ome
        self.dtype = p.dtype
        self.device = p.device
        self.host = p.host
        self.plan = get_plan(code, self.size_dict, p.ome, be.prec if prec is None else prec)
        lib = _lib.load()
        n = C.c_int64()
        check(lib.ome_plan_slice_count(self.plan.handle, C.byref(n)))
        self.nslices = n.value
        pd, pb, op = C.c_int(), C.c_size_t(), C.c_int()
        check(lib.ome_plan_partial_info(self.plan.handle, C.byref(pd), C.byref(pb), C.byref(op)))
        self.partial_dtype = _PARTIAL_TORCH[pd.value]
        self.partial_bytes = pb.value
        self.reduce_op = op.value
        self.range = slice_range(self.nslices, self.rank, self.world)
        self.out_shape = [self.size_dict[l] for l in code.eins.eins.iy]

    def partial(self, xs) -> torch.Tensor:
        p = _Prepared(xs)
        if p.ome != self.ome:
            raise ArgumentError("inputs changed element type since planning")
        ins = [_f_contig(t) for t in p.tensors]
        part = _alloc(self.out_shape, self.partial_dtype, self.device)
        ctx = _lib.context(self.device.index, self.plan.forward_bytes)
        b, e = self.range
        with torch.cuda.device(self.device):
            check(_lib.load().ome_plan_execute_slices(ctx.handle, self.plan.handle, _stream(self.device), _ptrs(ins),
                                                      b, e, part.data_ptr()))
        self._keep = ins
        return part

    def reduce(self, part: torch.Tensor) -> torch.Tensor:
        return allreduce_partial(part, self.reduce_op, self.group)

    def finish(self, part: torch.Tensor, y: Optional[torch.Tensor] = None, sx=True, sy=False) -> torch.Tensor:
        yt = _alloc(self.out_shape, self.dtype, self.device) if y is None else y
        if tuple(yt.shape) != tuple(self.out_shape) or tuple(yt.stride()) != tuple(_f_contig(yt).stride()):
            raise ArgumentError("y must be a column-major array of the output shape")
        ctx = _lib.context(self.device.index, self.plan.forward_bytes)
        with torch.cuda.device(self.device):
            check(_lib.load().ome_plan_finish(ctx.handle, self.plan.handle, _stream(self.device), part.data_ptr(),
                                              yt.data_ptr(), _scalar_buf(self.ome, sx), _scalar_buf(self.ome, sy)))
        return yt

    def __call__(self, xs, y=None, sx=True, sy=False):
        part = self.reduce(self.partial(xs))
        yt = self.finish(part, None if y is None else (y.data if isinstance(y, TropicalTensor) else y), sx, sy)
        if y is not None:
            return y
        if self.host:
            yt = _to_host(yt)
        return TropicalTensor(yt) if self.ome in (_lib.TROP_F32, _lib.TROP_F64) else yt


def sharded_einsum(code: SlicedEinsum, xs, group=None, size_dict=None, y=None, sx: Any = True, sy: Any = False):
    """``einsum(code, xs)`` for a SlicedEinsum with its slices spread over the
    ranks of ``group`` (default: the whole process group; a single process
    without one runs every slice).  Returns the full result on every rank."""
    return ShardedSlices(code, xs, size_dict, group)(xs, y, sx, sy)
