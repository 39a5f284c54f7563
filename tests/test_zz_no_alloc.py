"""ome_reduce_noalloc: the allocation-free reduction entry point, called
through the C ABI and checked against the context-based ome_einsum on the
same inputs, two calls in a row (the fixed scratch array keeps the previous
call's partial sums, which must not leak into the next result).

It exists for callers that cannot let the library allocate device memory
(their memory belongs to their own pool or fixed arena).  This file is named
so that pytest collects it last.
"""
import ctypes as C

import numpy as np
import pytest
import torch

import omeinsum_b200 as ome
from omeinsum_b200 import _lib

pytestmark = pytest.mark.gpu

RTOL = {torch.float32: 1e-5, torch.float64: 1e-12}


def _tensor(t, labels, keep):
    nd = t.dim()
    dims = (C.c_int64 * max(nd, 1))(*t.shape)
    strides = (C.c_int64 * max(nd, 1))(*t.stride())
    labs = (C.c_int32 * max(nd, 1))(*labels)
    keep += [dims, strides, labs]
    return _lib.Tensor(t.data_ptr(), nd, dims, strides, labs)


def _scalar(v, dtype):
    a = np.array([v], dtype={torch.float32: np.float32, torch.float64: np.float64, torch.int64: np.int64}[dtype])
    b = (C.c_ubyte * 16)()
    C.memmove(b, a.tobytes(), a.nbytes)
    return b


def noalloc(x, xl, y, yl, sx, sy):
    keep = []
    xt, yt = _tensor(x, xl, keep), _tensor(y, yl, keep)
    dt = {torch.float32: _lib.F32, torch.float64: _lib.F64, torch.int64: _lib.I64}[x.dtype]
    stream = C.c_void_p(torch.cuda.current_stream().cuda_stream)
    return _lib.load().ome_reduce_noalloc(stream, dt, C.byref(xt), C.byref(yt), _scalar(sx, x.dtype),
                                          _scalar(sy, x.dtype))


def reference(x, xl, y0, yl, sx, sy):
    """The existing entry point (ome_einsum through the package) on a copy of y."""
    y = y0.clone()
    ome.einsum_(ome.EinCode([tuple(xl)], tuple(yl)), [x], y, sx, sy)
    return y


def check(got, want):
    if got.dtype in RTOL:
        err = (got.double() - want.double()).norm() / max(want.double().norm(), 1e-300)
        assert err <= RTOL[got.dtype], float(err)
    else:
        assert torch.equal(got, want)


CASES = [
    # labels of x, labels of y, shape of x, dtype
    ((1, 1), (), (4096, 4096), torch.float32),             # Tr
    ((1, 2, 3), (2,), (256, 128, 64), torch.float64),      # Sum over a leading and a trailing mode
    ((1, 2, 3), (3, 1), (64, 300, 5), torch.float32),      # Sum with a permuted output
    ((1, 2), (), (1000, 999), torch.int64),                # full Sum, exact
    ((1, 2, 2), (1,), (70, 33, 33), torch.int64),          # partial trace, exact
]


@pytest.mark.parametrize("xl,yl,shape,dtype", CASES)
def test_noalloc_matches_context_entry_point_twice(xl, yl, shape, dtype):
    g = torch.Generator(device="cuda").manual_seed(7)
    if dtype == torch.int64:
        x = torch.randint(-8, 9, shape, device="cuda", generator=g)
    else:
        x = torch.randn(shape, device="cuda", dtype=dtype, generator=g)
    size = dict(zip(xl, shape))
    yshape = [size[l] for l in yl]
    for sx, sy in [(1, 0), (3, 2)]:
        y0 = (torch.randint(-8, 9, yshape, device="cuda", generator=g) if dtype == torch.int64
              else torch.randn(yshape, device="cuda", dtype=dtype, generator=g))
        want = reference(x, xl, y0, yl, sx, sy)
        for _ in range(2):  # two calls in a row: the second must not see the first's partial sums
            y = y0.clone()
            _lib.check(noalloc(x, xl, y, yl, sx, sy))
            torch.cuda.synchronize()
            check(y, want)
        # a different input right after: stale partials would show up here
        x2 = x.flip(0).contiguous()
        want2 = reference(x2, xl, y0, yl, sx, sy)
        y = y0.clone()
        _lib.check(noalloc(x2, xl, y, yl, sx, sy))
        torch.cuda.synchronize()
        check(y, want2)


def test_noalloc_rejects_outputs_beyond_its_scratch():
    cap = 4 << 20
    n = cap // (2 * 4) + 1                      # one float32 output more than the scratch allows
    x = torch.zeros((n, 2), device="cuda")
    y = torch.zeros((n,), device="cuda")
    rc = noalloc(x, (1, 2), y, (1,), 1, 0)
    assert rc == _lib.UNSUPPORTED
    assert b"scratch" in _lib.load().ome_last_error()
