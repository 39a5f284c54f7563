"""Shared helpers for the parity tests: seeded inputs per element type, the
oracle call for a code, and the comparison rule per element type.

Tolerances (norm-wise relative error, like Julia's isapprox on arrays):
FP64/ComplexF64 1e-12; FP32/ComplexF32 1e-5 (the reference's own GPU backend
agreement tolerance, test/cueinsum.jl:299).  Int64, Bool and tropical results
must be bit-exact.
"""
import numpy as np
import torch

import ome_oracle as O
import omeinsum_b200 as ome

DTYPES = ["f64", "f32", "c128", "c64", "i64", "bool", "trop"]
RTOL = {"f64": 1e-12, "c128": 1e-12, "f32": 1e-5, "c64": 1e-5}


def gen(rng, shape, dt):
    shape = tuple(shape)
    if dt in ("f64", "f32"):
        a = rng.standard_normal(shape)
        return a.astype(np.float32 if dt == "f32" else np.float64)
    if dt in ("c128", "c64"):
        a = rng.standard_normal(shape) + 1j * rng.standard_normal(shape)
        return a.astype(np.complex64 if dt == "c64" else np.complex128)
    if dt == "i64":
        return rng.integers(-8, 9, shape).astype(np.int64)
    if dt == "bool":
        return rng.integers(0, 2, shape).astype(bool)
    if dt == "trop":
        return rng.integers(-8, 9, shape).astype(np.float64) + rng.standard_normal(shape) * 0.25
    raise ValueError(dt)


def alg_of(dt):
    return O.TROPICAL if dt == "trop" else O.BOOL if dt == "bool" else O.REAL


def to_dev(a, dt):
    t = torch.from_numpy(np.array(a, order="F")).cuda()
    return ome.TropicalTensor(t) if dt == "trop" else t


def to_np(t):
    if isinstance(t, ome.TropicalTensor):
        t = t.data
    return t.detach().cpu().numpy()


def oracle(ixs, iy, xs, sd, dt, wide=False):
    """The oracle's result for the code; wide=True evaluates floats in FP64/C128."""
    if wide and dt in ("f32", "c64"):
        xs = [x.astype(np.float64 if dt == "f32" else np.complex128) for x in xs]
    return O.einsum([tuple(ix) for ix in ixs], tuple(iy), xs, sd, alg_of(dt))


def relerr(got, want):
    got = np.asarray(got, dtype=np.complex128 if np.iscomplexobj(got) or np.iscomplexobj(want) else np.float64)
    want = np.asarray(want, dtype=got.dtype)
    d = np.linalg.norm((got - want).ravel())
    n = max(np.linalg.norm(got.ravel()), np.linalg.norm(want.ravel()))
    return 0.0 if n == 0 and d == 0 else d / max(n, 1e-300)


def assert_match(got, want, dt, rtol=None):
    got = np.asarray(got)
    want = np.asarray(want)
    assert got.shape == want.shape, (got.shape, want.shape)
    if dt in ("i64", "bool", "trop"):
        assert got.dtype == want.dtype, (got.dtype, want.dtype)
        assert np.array_equal(got, want), f"not bit-exact: max diff {np.max(np.abs(got.astype(float) - want.astype(float)))}"
    else:
        e = relerr(got, want)
        assert e <= (rtol or RTOL[dt]), f"relative error {e:.3e} > {rtol or RTOL[dt]}"


def parse(s):
    lhs, iy = s.replace(" ", "").split("->")
    ixs = [tuple(ix) for ix in lhs.split(",")] if lhs else [()]
    return ixs, tuple(iy)
