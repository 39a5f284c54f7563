"""GPU parity at the rule-suite benchmark's exact shapes and inputs.

The six contractions the benchmark times (binary and unary rules at full
size), each run through the package exactly as the benchmark runs it, in
FP32 and in Int64:

* FP32 against the oracle evaluated in FP64 on the same inputs, at the
  reference's own GPU agreement tolerance rtol = 1e-5 (test/cueinsum.jl:
  296-299), and against the oracle's FP32 DefaultBackend result at the same
  tolerance; permutations are copies and must be bit-exact;
* Int64 (uniform integers in [-8, 8]) bit-exact against the oracle;
* in both, the kernel the benchmark's roofline names must be the one that
  ran (the library's kernel-event record, ome_kernel_times).
"""
import ctypes as C
import os
import sys

import numpy as np
import pytest
import torch

import ome_oracle as O
import omeinsum_b200 as ome
from omeinsum_b200 import _lib
from helpers import relerr

sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
import bench  # noqa: E402  (the benchmark's case list and input generator)

pytestmark = pytest.mark.gpu

# main kernel per suite case: FP32, Int64
MAIN_KERNEL = {
    "abcd,cdef->abef": ("k_gemm_tma2", "k_gemm_simt"),
    "ijk,jkl->il": ("k_gemm_tma2", "k_gemm_simt"),
    "bij,bjk->bik": ("k_gemm_bdiag", "k_gemm_bstage"),
    "abcde->ecadb": ("k_transpose_v4", "k_transpose32"),
    "ii->": ("k_loop_block", "k_loop_block"),
    "ijk->j": ("k_reduce_contig", "k_reduce_contig"),
}
CASES = [(name, code, ext, seed) for name, code, ext, seed in bench.CASES]


def run_recording_kernels(fn):
    """Run fn() with the library's kernel-event record on; return (result, kernel names)."""
    lib = _lib.load()
    lib.ome_kernel_timing(64)
    try:
        out = fn()
        torch.cuda.synchronize()
        ome.device_status()
        ms = (C.c_float * 64)()
        names = (C.c_char_p * 64)()
        cnt = C.c_int32()
        _lib.check(lib.ome_kernel_times(64, ms, names, C.byref(cnt)))
    finally:
        lib.ome_kernel_timing(0)
    return out, [names[i].decode() for i in range(cnt.value)]


def run_suite_case(code, ext, xs):
    """The benchmark's call: einsum!(code, xs, y, true, false, size_dict) on resident inputs."""
    ixs, iy = bench.parse_code(code)
    c = ome.EinCode(ixs, iy)
    d = [torch.from_numpy(x).cuda() for x in xs]
    y = ome.get_output_array(d, [ext[l] for l in iy])
    ome.einsum_(c, d, y, True, False, ext)
    return y


@pytest.mark.parametrize("name,code,ext,seed", CASES, ids=[c[0] for c in CASES])
def test_suite_case_fp32_vs_fp64_oracle(name, code, ext, seed):
    xs = bench.make_inputs(code, ext, seed, "f32")
    y, names = run_recording_kernels(lambda: run_suite_case(code, ext, xs))
    assert MAIN_KERNEL[name][0] in names, names
    got = y.cpu().numpy()
    ixs, iy = bench.parse_code(code)
    if len(ixs) == 1 and len(iy) == len(ixs[0]):
        # Permutedims is a copy: bit-exact
        want = O.einsum(ixs, iy, xs, ext)
        assert got.dtype == want.dtype and np.array_equal(got, want)
        return
    want64 = O.einsum(ixs, iy, [x.astype(np.float64) for x in xs], ext)
    e64 = relerr(got, want64)
    assert e64 <= 1e-5, f"{name}: relative error {e64:.3e} against the FP64 oracle"
    want32 = O.einsum(ixs, iy, xs, ext)
    e32 = relerr(got, want32)
    assert e32 <= 1e-5, f"{name}: relative error {e32:.3e} against the FP32 DefaultBackend restatement"


@pytest.mark.parametrize("name,code,ext,seed", CASES, ids=[c[0] for c in CASES])
def test_suite_case_int64_bit_exact(name, code, ext, seed):
    xs = bench.make_inputs(code, ext, seed, "i64")
    y, names = run_recording_kernels(lambda: run_suite_case(code, ext, xs))
    assert MAIN_KERNEL[name][1] in names, names
    got = y.cpu().numpy()
    ixs, iy = bench.parse_code(code)
    want = O.einsum(ixs, iy, xs, ext)
    assert got.dtype == np.int64 and want.dtype == np.int64
    assert got.shape == want.shape
    assert np.array_equal(got, want), f"{name}: {int(np.sum(got != want))} entries differ"


@pytest.mark.parametrize("dt", ["f32", "i64"])
def test_permute_robustness_shape(dt):
    """abcde->ecadb on the odd extents (47, 43, 41, 37, 40), where the
    16-byte transpose does not apply: bit-exact."""
    ext = dict(a=47, b=43, c=41, d=37, e=40)
    xs = bench.make_inputs("abcde->ecadb", ext, 4, dt)
    got = run_suite_case("abcde->ecadb", ext, xs).cpu().numpy()
    assert np.array_equal(got, np.transpose(xs[0], (4, 2, 0, 3, 1)))


@pytest.mark.parametrize("dt", ["f32", "i64"])
def test_suite_case_alpha_beta(dt):
    """y <- 3y + 2f at the full sizes of the three HBM-bound unary cases."""
    for name, code, ext, seed in CASES[3:]:
        xs = bench.make_inputs(code, ext, seed, dt)
        ixs, iy = bench.parse_code(code)
        rng = np.random.default_rng(seed + 100)
        shape = [ext[l] for l in iy]
        y0 = (rng.integers(-8, 9, shape, dtype=np.int64) if dt == "i64"
              else rng.standard_normal(shape).astype(np.float32))
        y0 = np.array(y0, order="F")
        yd = torch.from_numpy(y0.copy(order="F")).cuda()   # keeps the column-major strides
        ome.einsum_(ome.EinCode(ixs, iy), [torch.from_numpy(x).cuda() for x in xs], yd, 2, 3, ext)
        got = yd.cpu().numpy()
        want = np.array(y0, order="F")
        O.einsum_(ixs, iy, xs, want, want.dtype.type(2), want.dtype.type(3), ext)
        if dt == "i64":
            assert np.array_equal(got, want), name
        else:
            assert relerr(got, want) <= 1e-5, name
