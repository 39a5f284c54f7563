"""einsum / einsum! / loop_einsum / einsum_grad / cost_and_gradient on the B200 backend.

Host side of the backend: turns codes and torch tensors into C-ABI calls of
libomeb200 (include/ome_b200.h).  Mirrors the reference's entry points:
``einsum`` and ``einsum!`` (src/einsum.jl:24-50), ``loop_einsum`` /
``loop_einsum!`` (src/loop_einsum.jl:8-32), NestedEinsum/SlicedEinsum
evaluation (src/einsequence.jl:257-287, src/slicing.jl:104-137),
``einsum_grad`` (src/autodiff.jl:24-30) and ``cost_and_gradient``
(src/bp.jl:122-130).  Tensors are torch tensors; CUDA tensors stay on their
device, host (CPU / NumPy) inputs are copied to the current device and the
result copied back.
"""
from __future__ import annotations

import contextlib
import ctypes as C
import threading
from typing import Any, Dict, List, Sequence, Tuple

import numpy as np
import torch

from . import _lib
from ._lib import ArgumentError, check
from .backends import B200Backend, get_einsum_backend
from .core import (AbstractEinsum, EinCode, NestedEinsum, SlicedEinsum, get_size_dict)

# ----------------------------------------------------------------------------
# element types
# ----------------------------------------------------------------------------


class TropicalTensor:
    """A tensor of TropicalNumbers.jl ``Tropical{T}`` values (max-plus algebra)
    stored as a float32/float64 torch tensor of their contents."""

    def __init__(self, data):
        if not isinstance(data, torch.Tensor):
            data = torch.as_tensor(np.asarray(data))
        if data.dtype not in (torch.float32, torch.float64):
            data = data.to(torch.float64)
        self.data = data

    @property
    def shape(self):
        return self.data.shape

    @property
    def dtype(self):
        return self.data.dtype

    @property
    def device(self):
        return self.data.device

    def cpu(self):
        return TropicalTensor(self.data.cpu())

    def __repr__(self):
        return f"TropicalTensor({self.data!r})"


_TORCH_TO_OME = {
    torch.float32: _lib.F32, torch.float64: _lib.F64, torch.complex64: _lib.C32,
    torch.complex128: _lib.C64, torch.int64: _lib.I64, torch.bool: _lib.BOOL,
}
_RANK = {torch.bool: 0, torch.int64: 1, torch.float32: 2, torch.float64: 3}


def promote_dtype(dts: Sequence[torch.dtype]) -> torch.dtype:
    """Julia ``promote_type`` over Bool/Int64/Float32/Float64 and complexes
    (Int64 with Float32 gives Float32, unlike NumPy)."""
    cplx = any(d.is_complex for d in dts)
    real = [torch.float32 if d == torch.complex64 else torch.float64 if d == torch.complex128 else d for d in dts]
    for d in real:
        if d not in _RANK:
            raise _lib.OMEError(f"unsupported element type {d}")
    r = max(real, key=lambda d: _RANK[d])
    if cplx:
        return torch.complex128 if r == torch.float64 else torch.complex64
    return r


def _as_tensor(x):
    if isinstance(x, (torch.Tensor, TropicalTensor)):
        return x
    return torch.as_tensor(np.asarray(x))


def _colmajor_strides(shape) -> Tuple[int, ...]:
    s, out = 1, []
    for e in shape:
        out.append(s)
        s *= int(e)
    return tuple(out)


def _alloc(shape, dtype, device) -> torch.Tensor:
    """Column-major (Julia-layout) output array."""
    return torch.empty_strided(tuple(shape), _colmajor_strides(shape), dtype=dtype, device=device)


def _f_contig(x: torch.Tensor) -> torch.Tensor:
    if x.dim() == 0 or tuple(x.stride()) == _colmajor_strides(x.shape) or x.numel() <= 1:
        return x
    y = _alloc(x.shape, x.dtype, x.device)
    y.copy_(x)
    return y


def _to_host(y: torch.Tensor) -> torch.Tensor:
    """Device result -> host tensor for callers that passed host inputs: the
    copy lands in page-locked memory (torch's caching host allocator, reused
    across calls), which moves at link speed; a pageable copy runs several
    times slower.  Returns once the data is on the host."""
    out = torch.empty_strided(tuple(y.shape), tuple(y.stride()), dtype=y.dtype, pin_memory=True)
    out.copy_(y, non_blocking=True)
    torch.cuda.current_stream(y.device).synchronize()
    return out


class _Prepared:
    """Inputs moved to one CUDA device with one element type."""

    def __init__(self, xs: Sequence[Any], out_dtype=None):
        xs = [_as_tensor(x) for x in xs]
        self.tropical = any(isinstance(x, TropicalTensor) for x in xs)
        if self.tropical and not all(isinstance(x, TropicalTensor) for x in xs):
            raise ArgumentError("cannot mix tropical and ordinary tensors")
        raw = [x.data if isinstance(x, TropicalTensor) else x for x in xs]
        self.host = all(not t.is_cuda for t in raw)
        if self.host:
            dev = torch.device("cuda", torch.cuda.current_device())
        else:
            dev = next(t.device for t in raw if t.is_cuda)
        self.device = dev
        self.dtype = out_dtype or promote_dtype([t.dtype for t in raw])
        ts = []
        for t in raw:
            if t.is_conj():
                t = t.resolve_conj()
            if t.dtype != self.dtype:
                t = t.to(device=dev, dtype=self.dtype, non_blocking=True)
            elif t.device != dev:
                t = t.to(dev, non_blocking=True)
            ts.append(t)
        self.tensors = ts
        if self.tropical:
            self.ome = _lib.TROP_F32 if self.dtype == torch.float32 else _lib.TROP_F64
        else:
            self.ome = _TORCH_TO_OME[self.dtype]

    def wrap(self, y: torch.Tensor):
        if self.host:
            y = _to_host(y)
        return TropicalTensor(y) if self.tropical else y


def _scalar_buf(ome: int, v) -> C.Array:
    """One value of the call's dtype; Python bools are the algebra's one/zero
    (Julia converts true/false to one(T)/zero(T))."""
    b = (C.c_ubyte * 16)()
    if ome in (_lib.TROP_F32, _lib.TROP_F64):
        val = (0.0 if v else -np.inf) if isinstance(v, (bool, np.bool_)) else float(v)
        arr = np.array([val], dtype=np.float32 if ome == _lib.TROP_F32 else np.float64)
    elif ome == _lib.BOOL:
        arr = np.array([bool(v)], dtype=np.uint8)
    elif ome == _lib.I64:
        arr = np.array([int(v)], dtype=np.int64)
    elif ome == _lib.F32:
        arr = np.array([float(v)], dtype=np.float32)
    elif ome == _lib.F64:
        arr = np.array([float(v)], dtype=np.float64)
    elif ome == _lib.C32:
        arr = np.array([complex(v)], dtype=np.complex64)
    else:
        arr = np.array([complex(v)], dtype=np.complex128)
    raw = arr.tobytes()
    C.memmove(b, raw, len(raw))
    return b


class _LabelMap:
    def __init__(self):
        self.ids: Dict[Any, int] = {}

    def __call__(self, l) -> int:
        if l not in self.ids:
            self.ids[l] = len(self.ids)
        return self.ids[l]


def _tensor_struct(t: torch.Tensor, labels: Sequence[int], keep: list) -> _lib.Tensor:
    nd = t.dim()
    dims = (C.c_int64 * max(nd, 1))(*[int(s) for s in t.shape])
    strides = (C.c_int64 * max(nd, 1))(*[int(s) for s in t.stride()])
    labs = (C.c_int32 * max(nd, 1))(*labels)
    keep.extend([dims, strides, labs])
    return _lib.Tensor(t.data_ptr(), nd, dims, strides, labs)


# torch's raw queries (what torch.cuda.current_stream / current_device wrap;
# the wrappers cost several microseconds per call)
_RAW_STREAM = getattr(torch._C, "_cuda_getCurrentRawStream", None)
_GET_DEVICE = getattr(torch._C, "_cuda_getDevice", None)


def _raw_stream(index: int) -> int:
    if _RAW_STREAM is not None:
        return _RAW_STREAM(index)
    return torch.cuda.current_stream(index).cuda_stream


def _current_device() -> int:
    return _GET_DEVICE() if _GET_DEVICE is not None else torch.cuda.current_device()


def _stream(device) -> C.c_void_p:
    return C.c_void_p(torch.cuda.current_stream(device).cuda_stream)


def _require_b200():
    be = get_einsum_backend()
    if not isinstance(be, B200Backend):
        raise _lib.OMEError(f"backend {type(be).__name__} is not provided by this package; "
                            "select B200Backend() with set_einsum_backend")
    return be


# Call descriptors (ctypes tensor structs) by layout, per host thread: a
# repeated call with the same codes, shapes, strides and dtype only rewrites
# the data pointers.
_TLS = threading.local()
_CALLS_MAX = 4096
_SCALARS: Dict[Any, C.Array] = {}


def _scalar_cached(ome: int, v) -> C.Array:
    try:
        key = (ome, type(v), v)
        b = _SCALARS.get(key)
    except TypeError:  # unhashable scalar (e.g. a 0-d array)
        return _scalar_buf(ome, v)
    if b is None:
        b = _scalar_buf(ome, v)
        if len(_SCALARS) < 1024:
            _SCALARS[key] = b
    return b


def _run_eincode(ixs, iy, p: _Prepared, y: torch.Tensor, sx, sy, loop_only=False, prec=None):
    be = _require_b200()
    prec = be.prec if prec is None else prec
    ts = p.tensors
    try:
        key = (tuple(map(tuple, ixs)), tuple(iy), p.ome, loop_only, prec,
               tuple((tuple(t.shape), t.stride()) for t in ts), tuple(y.shape), y.stride())
        hash(key)
    except TypeError:  # unhashable labels
        key = None
    calls = getattr(_TLS, "calls", None)
    if calls is None:
        calls = _TLS.calls = {}
    hit = calls.get(key) if key is not None else None
    if hit is None:
        lm = _LabelMap()
        keep: list = []
        xs = (_lib.Tensor * len(ixs))()
        for i, (ix, t) in enumerate(zip(ixs, ts)):
            if len(ix) != t.dim():
                raise ArgumentError(f"indices {tuple(ix)} invalid for tensor with ndims = {t.dim()}")
            xs[i] = _tensor_struct(t, [lm(l) for l in ix], keep)
        yt = _tensor_struct(y, [lm(l) for l in iy], keep)
        hit = (xs, yt, keep)
        if key is not None:
            if len(calls) >= _CALLS_MAX:
                calls.pop(next(iter(calls)))
            calls[key] = hit
    else:
        xs, yt, _ = hit
        for i, t in enumerate(ts):
            xs[i].data = t.data_ptr()
        yt.data = y.data_ptr()
    sxb, syb = _scalar_cached(p.ome, sx), _scalar_cached(p.ome, sy)
    cur = _current_device()
    dev = y.device.index if y.device.index is not None else cur
    ctx = _lib.context(dev)
    lib = _lib.load()
    with contextlib.nullcontext() if dev == cur else torch.cuda.device(dev):
        st = C.c_void_p(_raw_stream(dev))
        if loop_only:
            rc = lib.ome_loop_einsum(ctx.handle, st, p.ome, len(ixs), xs, C.byref(yt), sxb, syb)
        else:
            rc = lib.ome_einsum(ctx.handle, st, p.ome, len(ixs), xs, C.byref(yt), sxb, syb, prec)
    check(rc)
    return y


# ----------------------------------------------------------------------------
# public API
# ----------------------------------------------------------------------------


def get_output_array(xs, shape, fillzero=False):
    """``get_output_array`` (src/loop_einsum.jl:48-61; ext/CUDAExt.jl:34-47)."""
    p = _Prepared(xs)
    y = _alloc(shape, p.dtype, p.device)
    if fillzero:
        y.fill_(-np.inf if p.tropical else 0)
    return p.wrap(y)


def einsum(code: AbstractEinsum, xs: Sequence[Any], size_dict: Dict[Any, int] | None = None, **kw):
    """``einsum(code, xs, size_dict)``: a new output array (src/einsum.jl:24-27)."""
    _require_b200()
    if isinstance(code, (NestedEinsum, SlicedEinsum)):
        from .plan import run_tree
        return run_tree(code, xs, size_dict)
    if size_dict is None:
        size_dict = get_size_dict(code.getixs(), xs)
    p = _Prepared(xs)
    for l in code.iy:
        if l not in size_dict:
            raise ArgumentError(f"output label {l} has no size; pass size_info")
    y = _alloc([size_dict[l] for l in code.iy], p.dtype, p.device)
    _run_eincode(code.ixs, code.iy, p, y, True, False, **kw)
    return p.wrap(y)


def einsum_(code: AbstractEinsum, xs: Sequence[Any], y, sx=True, sy=False, size_dict=None, **kw):
    """``einsum!(code, xs, y, sx, sy, size_dict)``: y <- sy*y + sx*code(xs), in place
    (src/einsum.jl:28-50).  ``y`` must be a CUDA tensor (or TropicalTensor)."""
    _require_b200()
    yt = y.data if isinstance(y, TropicalTensor) else y
    if not yt.is_cuda:
        raise ArgumentError("einsum_ needs a CUDA output tensor")
    if isinstance(code, (NestedEinsum, SlicedEinsum)):
        from .plan import run_tree
        return run_tree(code, xs, size_dict, y=y, sx=sx, sy=sy)
    if size_dict is None:
        size_dict = get_size_dict(code.getixs(), xs)
    p = _Prepared(xs, out_dtype=yt.dtype)
    _run_eincode(code.ixs, code.iy, p, yt, sx, sy, **kw)
    return y


_COPY_STREAMS: Dict[int, Tuple[torch.cuda.Stream, torch.cuda.Stream]] = {}


def einsum_many(jobs: Sequence[Tuple[AbstractEinsum, Sequence[Any], Dict[Any, int] | None]], window: int = 2):
    """``[einsum(code, xs, size_dict) for code, xs, size_dict in jobs]`` for
    independent contractions whose inputs live on the host, with the host link
    kept busy in both directions: job i's inputs go up on one copy stream,
    it runs on the current stream, and its result comes down on a second
    copy stream while job i+1's inputs go up.  At most ``window`` jobs hold
    device memory at once.  Results are page-locked host tensors (TropicalTensor
    for tropical jobs), in job order; the call returns once all are on the
    host.  Jobs whose inputs are already on the device run as ``einsum`` and
    return device tensors."""
    _require_b200()
    jobs = list(jobs)
    if window < 1:
        raise ArgumentError("window must be at least 1")
    dev = torch.device("cuda", torch.cuda.current_device())
    if dev.index not in _COPY_STREAMS:
        _COPY_STREAMS[dev.index] = (torch.cuda.Stream(dev), torch.cuda.Stream(dev))
    up, down = _COPY_STREAMS[dev.index]
    comp = torch.cuda.current_stream(dev)
    outs: List[Any] = []
    landed: List[Any] = [None] * len(jobs)
    for i, (code, xs, size_dict) in enumerate(jobs):
        xs = [_as_tensor(x) for x in xs]
        raw = [x.data if isinstance(x, TropicalTensor) else x for x in xs]
        if any(t.is_cuda for t in raw):
            outs.append(einsum(code, xs, size_dict))
            continue
        if i >= window and landed[i - window] is not None:
            landed[i - window].synchronize()
        with torch.cuda.stream(up):
            dx = [t.to(dev, non_blocking=True) for t in raw]
        for t in dx:
            t.record_stream(comp)
        comp.wait_stream(up)
        y = einsum(code, [TropicalTensor(t) if isinstance(x, TropicalTensor) else t for t, x in zip(dx, xs)],
                   size_dict)
        yt = y.data if isinstance(y, TropicalTensor) else y
        down.wait_stream(comp)
        with torch.cuda.stream(down):
            h = torch.empty_strided(tuple(yt.shape), tuple(yt.stride()), dtype=yt.dtype, pin_memory=True)
            h.copy_(yt, non_blocking=True)
        yt.record_stream(down)
        landed[i] = torch.cuda.Event()
        landed[i].record(down)
        outs.append(TropicalTensor(h) if isinstance(y, TropicalTensor) else h)
    down.synchronize()
    return outs


def loop_einsum(code: EinCode, xs, size_dict=None):
    """``loop_einsum`` (src/loop_einsum.jl:8-12): the generic index kernel."""
    _require_b200()
    if size_dict is None:
        size_dict = get_size_dict(code.getixs(), xs)
    p = _Prepared(xs)
    y = _alloc([size_dict[l] for l in code.iy], p.dtype, p.device)
    _run_eincode(code.ixs, code.iy, p, y, True, False, loop_only=True)
    return p.wrap(y)


def loop_einsum_(ixs, iy, xs, y, sx, sy, size_dict=None):
    """``loop_einsum!`` (src/loop_einsum.jl:21-32)."""
    yt = y.data if isinstance(y, TropicalTensor) else y
    p = _Prepared(xs, out_dtype=yt.dtype)
    _run_eincode([tuple(ix) for ix in ixs], tuple(iy), p, yt, sx, sy, loop_only=True)
    return y


def einsum_grad(ixs, xs, iy, size_dict, dy, i):
    """``einsum_grad`` (src/autodiff.jl:24-30): the gradient of ``einsum`` w.r.t.
    input ``i`` (0-based): contract conj(dy) in place of input i into ixs[i],
    then conjugate -- one ``ome_einsum_grad`` call (the conjugations run in
    the library).  A real input of a complex contraction gets the real part
    (``ProjectTo(xs[i])``)."""
    be = _require_b200()
    ixs = [tuple(ix) for ix in ixs]
    nxs = [_as_tensor(x) for x in xs]
    nxs[i] = _as_tensor(dy)
    p = _Prepared(nxs)
    ts = p.tensors
    lm = _LabelMap()
    keep: list = []
    structs = (_lib.Tensor * len(ixs))()
    for k, (ix, t) in enumerate(zip(ixs, ts)):
        if k == i:
            continue
        if len(ix) != t.dim():
            raise ArgumentError(f"indices {ix} invalid for tensor with ndims = {t.dim()}")
        structs[k] = _tensor_struct(t, [lm(l) for l in ix], keep)
    if len(tuple(iy)) != ts[i].dim():
        raise ArgumentError(f"indices {tuple(iy)} invalid for the cotangent with ndims = {ts[i].dim()}")
    dyt = _tensor_struct(ts[i], [lm(l) for l in iy], keep)
    if size_dict is None:
        size_dict = get_size_dict([ix for k, ix in enumerate(ixs) if k != i] + [tuple(iy)],
                                  [t for k, t in enumerate(ts) if k != i] + [ts[i]])
    shape = [size_dict[l] for l in ixs[i]]
    out = _alloc(shape, p.dtype, p.device)
    dxt = _tensor_struct(out, [lm(l) for l in ixs[i]], keep)
    nd = len(shape)
    dims = (C.c_int64 * max(nd, 1))(*shape)
    labs = (C.c_int32 * max(nd, 1))(*[lm(l) for l in ixs[i]])
    keep.extend([dims, labs])
    structs[i] = _lib.Tensor(None, nd, dims, None, labs)
    dev = out.device.index
    ctx = _lib.context(dev)
    with torch.cuda.device(dev):
        check(_lib.load().ome_einsum_grad(ctx.handle, _stream(dev), p.ome, len(ixs), structs, C.byref(dyt), i,
                                          C.byref(dxt), be.prec))
    xi = _as_tensor(xs[i])
    xi = xi.data if isinstance(xi, TropicalTensor) else xi
    if out.is_complex() and not xi.is_complex():
        out = out.real.contiguous()
    return p.wrap(out)


def cost_and_gradient(code, xs, dy=None):
    """``cost_and_gradient`` (src/bp.jl:122-130) on the device: returns
    (cost, [gradient of each input])."""
    from .plan import tree_gradient
    return tree_gradient(code, xs, dy)
