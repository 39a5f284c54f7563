"""ome_reduce_noalloc: the allocation-free reduction entry point, called
through the C ABI and checked against the context-based ome_einsum on the
same inputs, two calls in a row (the fixed scratch array keeps the previous
call's partial sums, which must not leak into the next result), and against
the oracle (the CPU restatement of the reference's unary Sum/Tr rules).

It exists for callers that cannot let the library allocate device memory
(their memory belongs to their own pool or fixed arena).  This file is named
so that pytest collects it last.
"""
import ctypes as C

import numpy as np
import pytest
import torch

import ome_oracle as O
import omeinsum_b200 as ome
from omeinsum_b200 import _lib
from omeinsum_b200.engine import _scalar_buf

pytestmark = pytest.mark.gpu

RTOL = {torch.float32: 1e-5, torch.float64: 1e-12}


def _tensor(t, labels, keep):
    nd = t.dim()
    dims = (C.c_int64 * max(nd, 1))(*t.shape)
    strides = (C.c_int64 * max(nd, 1))(*t.stride())
    labs = (C.c_int32 * max(nd, 1))(*labels)
    keep += [dims, strides, labs]
    return _lib.Tensor(t.data_ptr(), nd, dims, strides, labs)


def _dt(x, trop):
    if trop:
        return _lib.TROP_F32 if x.dtype == torch.float32 else _lib.TROP_F64
    return {torch.float32: _lib.F32, torch.float64: _lib.F64, torch.int64: _lib.I64, torch.bool: _lib.BOOL}[x.dtype]


def noalloc(x, xl, y, yl, sx, sy, trop=False):
    keep = []
    xt, yt = _tensor(x, xl, keep), _tensor(y, yl, keep)
    dt = _dt(x, trop)
    stream = C.c_void_p(torch.cuda.current_stream().cuda_stream)
    return _lib.load().ome_reduce_noalloc(stream, dt, C.byref(xt), C.byref(yt), _scalar_buf(dt, sx),
                                          _scalar_buf(dt, sy))


def reference(x, xl, y0, yl, sx, sy, trop=False):
    """The existing entry point (ome_einsum through the package) on a copy of y."""
    y = y0.clone()
    if trop:
        ome.einsum_(ome.EinCode([tuple(xl)], tuple(yl)), [ome.TropicalTensor(x)], ome.TropicalTensor(y), sx, sy)
    else:
        ome.einsum_(ome.EinCode([tuple(xl)], tuple(yl)), [x], y, sx, sy)
    return y


def oracle(x, xl, y0, yl, sx, sy, trop=False):
    """The oracle's einsum!(ixs, iy, xs, y, sx, sy) on host copies."""
    xn = x.cpu().numpy()
    y = np.array(y0.cpu().numpy(), order="F")
    sd = dict(zip(xl, x.shape))
    alg = O.TROPICAL if trop else None
    if trop:
        sx = 0.0 if sx is True else float(sx)
        sy = -np.inf if sy is False else float(sy)
    O.einsum_([tuple(xl)], tuple(yl), [xn], y, sx, sy, sd, alg)
    return torch.from_numpy(y)


def check(got, want):
    got, want = got.cpu(), want.cpu()
    assert tuple(got.shape) == tuple(want.shape)
    if got.dtype in RTOL:
        err = (got.double() - want.double()).norm() / max(want.double().norm(), 1e-300)
        assert err <= RTOL[got.dtype], float(err)
    else:
        assert torch.equal(got, want.to(got.dtype))


CASES = [
    # labels of x, labels of y, shape of x, dtype, tropical
    ((1, 1), (), (4096, 4096), torch.float32, False),             # Tr
    ((1, 2, 3), (2,), (256, 128, 64), torch.float64, False),      # Sum over a leading and a trailing mode
    ((1, 2, 3), (3, 1), (64, 300, 5), torch.float32, False),      # Sum with a permuted output
    ((1, 2), (), (1000, 999), torch.int64, False),                # full Sum, exact
    ((1, 2, 2), (1,), (70, 33, 33), torch.int64, False),          # partial trace, exact
    ((1, 2, 3), (3,), (40, 50, 7), torch.bool, False),            # Bool sum (OR of ANDs), exact
    ((1, 2, 3), (2, 1), (30, 9, 200), torch.float64, True),       # tropical (max-plus) sum, exact
    ((1, 2, 3), (1, 3), (300, 41, 1), torch.float32, False),      # an output mode of extent 1
    ((1, 2), (), (0, 5), torch.float32, False),                   # an empty summed mode first
    ((1, 2, 3), (2,), (6, 4, 0), torch.int64, False),             # an empty summed mode last
]


def _rand(shape, dtype, g, trop=False):
    if dtype == torch.int64:
        return torch.randint(-8, 9, shape, device="cuda", generator=g)
    if dtype == torch.bool:
        return torch.randint(0, 2, shape, device="cuda", generator=g) > 0
    if trop:  # integers plus a quarter-integer part: max-plus results are exact
        return (torch.randint(-32, 33, shape, device="cuda", generator=g).to(dtype) / 4)
    return torch.randn(shape, device="cuda", dtype=dtype, generator=g)


def _scalars(dtype, trop):
    if dtype == torch.bool:
        return [(True, False), (True, True)]
    if trop:
        return [(True, False), (1.5, -2.0)]
    return [(1, 0), (3, 2)]


@pytest.mark.parametrize("xl,yl,shape,dtype,trop", CASES)
def test_noalloc_matches_context_entry_point_twice(xl, yl, shape, dtype, trop):
    g = torch.Generator(device="cuda").manual_seed(7)
    x = _rand(shape, dtype, g, trop)
    size = dict(zip(xl, shape))
    yshape = [size[l] for l in yl]
    for sx, sy in _scalars(dtype, trop):
        y0 = _rand(yshape, dtype, g, trop)
        want = reference(x, xl, y0, yl, sx, sy, trop)
        check(want, oracle(x, xl, y0, yl, sx, sy, trop))
        for _ in range(2):  # two calls in a row: the second must not see the first's partial sums
            y = y0.clone()
            _lib.check(noalloc(x, xl, y, yl, sx, sy, trop))
            torch.cuda.synchronize()
            check(y, want)
        # a different input right after: stale partials would show up here
        x2 = x.flip(0).contiguous()
        want2 = reference(x2, xl, y0, yl, sx, sy, trop)
        check(want2, oracle(x2, xl, y0, yl, sx, sy, trop))
        y = y0.clone()
        _lib.check(noalloc(x2, xl, y, yl, sx, sy, trop))
        torch.cuda.synchronize()
        check(y, want2)


def test_noalloc_dimension_mismatch_message():
    x = torch.zeros((5, 6), device="cuda")
    y = torch.zeros((7,), device="cuda")
    rc = noalloc(x, (1, 2), y, (2,), 1, 0)
    assert rc == _lib.DIMENSION_MISMATCH
    assert _lib.load().ome_last_error() == b"label 2: input extent 6, output extent 7"


def test_noalloc_rejects_outputs_beyond_its_scratch():
    cap = 4 << 20
    n = cap // (2 * 4) + 1                      # one float32 output more than the scratch allows
    x = torch.zeros((n, 2), device="cuda")
    y = torch.zeros((n,), device="cuda")
    rc = noalloc(x, (1, 2), y, (1,), 1, 0)
    assert rc == _lib.UNSUPPORTED
    assert b"scratch" in _lib.load().ome_last_error()
