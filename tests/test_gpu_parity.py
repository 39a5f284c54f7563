"""GPU parity: libomeb200 (through the C ABI via the package) against the oracle
on seeded inputs.  Case lists follow the reference's own tests
(test/cueinsum.jl, test/einsum.jl, test/binaryrules.jl, test/unaryrules.jl).
"""
import itertools
import zlib

import numpy as np
import pytest
import torch

import ome_oracle as O
import omeinsum_b200 as ome
from helpers import DTYPES, assert_match, gen, oracle, parse, to_dev, to_np

pytestmark = pytest.mark.gpu

UNARY = ["ij->", "ij->j", "ii->", "ii->i", "ijk->kij", "a->aaaa", "ac->acc", "->ii", "i->ik", "->ik",
         "illljkk->kijjcc", "ijkl->ijkl", "ijk->ki", "ijk->", "iijj->", "ij->ji", "ijk->jik"]
BINARY = [",->", "i,->i", "j,j->", ",k->k", "j,jk->k", "j,kj->k", "ij,j->i", "ji,j->i", "i,k->ik", "i,k->ki"]
for X1, X2, X3 in itertools.product(["ij", "ji"], ["jk", "kj"], ["ik", "ki"]):
    BINARY.append(f"{X1},{X2}->{X3}")
BINARY += [c.replace(",", "l,").replace("->", "l->") + "l" for c in list(BINARY)]
COMPOSITE = ["abb,bc->ac", "ab,bc->acc", "ab,bce->ac", "ab,bc->ace", "bal,bcl->lcae", "bal,bcl->ca",
             "bal,bc->lca", "ddebal,bcf->lcac", "c,c->cc", "c,cc->c", "cc,c->cc", "cc,cc->cc", "cc,cb->bc",
             "cb,bc->cc", "ac,cc->ac", "ijk,jkl->il", "ij,ik,il->jkl", "ij,jk,kl->il", "ij,ij,ij->ij"]


def run_case(code, dt, D=2, seed=0, sx=True, sy=False, size_info=None):
    rng = np.random.default_rng(seed)
    ixs, iy = parse(code)
    sd = {l: D for l in "abcdefghijklmnopqrstuvwxyz"}
    if size_info:
        sd.update(size_info)
    xs = [gen(rng, [sd[l] for l in ix], dt) for ix in ixs]
    want = oracle(ixs, iy, xs, sd, dt)
    got = ome.einsum(ome.EinCode(ixs, iy), [to_dev(x, dt) for x in xs], sd)
    assert_match(to_np(got), want, dt)
    if dt in ("f32", "c64"):
        assert_match(to_np(got), oracle(ixs, iy, xs, sd, dt, wide=True), dt)


@pytest.mark.parametrize("dt", DTYPES)
@pytest.mark.parametrize("code", UNARY)
def test_unary_rules(code, dt):
    run_case(code, dt, D=3, seed=zlib.crc32(code.encode()) % 1000)


@pytest.mark.parametrize("dt", DTYPES)
@pytest.mark.parametrize("code", BINARY)
def test_binary_rules(code, dt):
    run_case(code, dt, D=3, seed=zlib.crc32(code.encode()) % 1000)


@pytest.mark.parametrize("dt", DTYPES)
@pytest.mark.parametrize("code", COMPOSITE)
def test_composite_rules(code, dt):
    run_case(code, dt, D=3, seed=zlib.crc32(code.encode()) % 1000)


@pytest.mark.parametrize("dt", ["f64", "c128", "i64", "trop"])
def test_nary_reference_cases(dt):
    # test/cueinsum.jl:45-49, 62-78 (D = 2 networks)
    run_case("npu,por,dom,lmn->urdl", dt, D=2)
    run_case("abewcd,bfixgh,ajeycd,jfizgh->wxyz", dt, D=2)


@pytest.mark.parametrize("dt", DTYPES)
@pytest.mark.parametrize("sxy", [(5, 3), (5, 1), (2, 0), (0, 3)])
def test_alpha_beta(dt, sxy):
    # test/einsum.jl:55-66 and test/cueinsum.jl:15-28: y <- sy*y + sx*f(xs)
    if dt == "bool":
        sxy = (bool(sxy[0]), bool(sxy[1]))
    if dt == "trop":
        sxy = (float(sxy[0]), float(sxy[1]) if sxy[1] else -np.inf)
    sx, sy = sxy
    rng = np.random.default_rng(7)
    for code in ["ij,jk->ik", "ijl,jkl->ikl", "abb,bc->acc", "ij->ji", "ij->", "ij,ik,il->jkl", "i->ii"]:
        ixs, iy = parse(code)
        sd = {l: 3 for l in "abcijkl"}
        xs = [gen(rng, [sd[l] for l in ix], dt) for ix in ixs]
        y0 = gen(rng, [sd[l] for l in iy], dt)
        yd = to_dev(y0, dt)
        ome.einsum_(ome.EinCode(ixs, iy), [to_dev(x, dt) for x in xs], yd, sx, sy, sd)
        want = np.array(y0, order="F")
        O.einsum_(ixs, iy, xs, want, sx, sy, sd, O.TROPICAL if dt == "trop" else None)
        assert_match(to_np(yd), want, dt)


def test_size_info_broadcast_identity():
    # test/einsum.jl:191-194: ein"->ii"(1; size_info = i=>5) == I(5)
    got = ome.ein("->ii")(torch.ones((), dtype=torch.int64, device="cuda"), size_info={"i": 5})
    assert torch.equal(got.cpu(), torch.eye(5, dtype=torch.int64))
    r = ome.ein(",->")(torch.tensor(3, device="cuda"), torch.tensor(4, device="cuda"))
    assert r.dtype == torch.int64 and int(r) == 12


def test_high_rank_permute():
    # test/cueinsum.jl:164-167: rank-18 permutedims
    rng = np.random.default_rng(3)
    shape = [4] + [int(v) for v in rng.integers(1, 4, 17)]
    x = rng.standard_normal(shape)
    labels = [chr(ord("a") + i) for i in range(18)]
    code = ome.EinCode([labels], labels[::-1])
    got = to_np(ome.einsum(code, [to_dev(x, "f64")]))
    assert np.array_equal(got, np.transpose(x, list(range(17, -1, -1))))


@pytest.mark.parametrize("dt", ["f32", "f64", "c64", "i64", "trop", "bool"])
@pytest.mark.parametrize("code,sizes", [
    ("ij,jk->ik", dict(i=200, j=300, k=250)),
    ("ji,jk->ki", dict(i=130, j=70, k=90)),
    ("ij,kj->ik", dict(i=64, j=200, k=96)),
    ("bij,bjk->bik", dict(b=40, i=33, j=65, k=40)),
    ("abcd,cdef->abef", dict(a=12, b=12, c=12, d=12, e=12, f=12)),
    ("ijk,jkl->il", dict(i=40, j=40, k=40, l=40)),
    ("ijl,jkl->kil", dict(i=48, j=64, k=80, l=3)),
])
def test_gemm_shapes(code, sizes, dt):
    """GEMM-shaped contractions (strided GEMM / BF16x3 tensor-core path)."""
    rng = np.random.default_rng(11)
    ixs, iy = parse(code)
    xs = [gen(rng, [sizes[l] for l in ix], dt) for ix in ixs]
    got = to_np(ome.einsum(ome.EinCode(ixs, iy), [to_dev(x, dt) for x in xs], sizes))
    ome.device_status()
    want = oracle(ixs, iy, xs, sizes, dt)
    assert_match(got, want, dt)
    if dt in ("f32", "c64"):
        assert_match(got, oracle(ixs, iy, xs, sizes, dt, wide=True), dt)


@pytest.mark.parametrize("prec,rtol", [(1, 1e-6), (2, 1e-5), (3, 1e-6)])
def test_precision_modes(prec, rtol):
    """FP32 (CUDA cores), BF16x3 and BF16x6 (tensor cores) against FP64."""
    rng = np.random.default_rng(5)
    a, b = rng.standard_normal((200, 3000)).astype(np.float32), rng.standard_normal((3000, 300)).astype(np.float32)
    ome.set_einsum_backend(ome.B200Backend(prec=prec))
    try:
        got = to_np(ome.ein("ij,jk->ik")(to_dev(a, "f32"), to_dev(b, "f32")))
        ome.device_status()
    finally:
        ome.set_einsum_backend(ome.B200Backend())
    assert_match(got, a.astype(np.float64) @ b.astype(np.float64), "f32", rtol)


def test_loop_einsum_entry():
    # test/cueinsum.jl:15-28: loop_einsum! with sx, sy and a duplicated output label
    rng = np.random.default_rng(2)
    a = rng.standard_normal((3, 3))
    ad = to_dev(a, "f64")
    y = torch.ones((3, 3, 3), dtype=torch.float64, device="cuda")
    ome.loop_einsum_([(1, 2), (2, 3)], (1, 3, 3), [ad, ad], y, 4.0, 2.0)
    out = 2 * np.ones((3, 3, 3))
    res = 4.0 * a @ a
    for k in range(3):
        out[:, k, k] += res[:, k]
    assert np.allclose(to_np(y), out)
    assert np.allclose(to_np(ome.loop_einsum(ome.ein("ij,jk->ik"), [ad, ad])), a @ a)


def test_errors_from_library():
    a = torch.zeros(3, 3, device="cuda")
    b = torch.zeros(4, 4, device="cuda")
    with pytest.raises(ome.DimensionMismatch):
        ome.einsum(ome.EinCode([(1, 2), (2, 3)], (1, 3)), [a, b], {1: 3, 2: 3, 3: 3})
    with pytest.raises(ome.ArgumentError):
        ome.einsum(ome.EinCode([(1, 2, 3), (2, 3)], (1, 3)), [a, a], {1: 3, 2: 3, 3: 3})


def test_host_buffers_round_trip():
    rng = np.random.default_rng(4)
    a, b = rng.standard_normal((20, 30)), rng.standard_normal((30, 10))
    got = ome.ein("ij,jk->ik")(torch.from_numpy(a), torch.from_numpy(b))
    assert not got.is_cuda and np.allclose(got.numpy(), a @ b)


def test_empty_extents():
    # test/einsum.jl:306-309 (issue 136)
    got = ome.EinCode([(1, 2, 3), (2,)], (1, 3))(torch.ones(2, 2, 1, device="cuda"), torch.ones(2, device="cuda"))
    assert torch.equal(got.cpu(), torch.tensor([[2.0], [2.0]]))
    got = ome.EinCode([(1, 2, 3), (2,)], (1, 3))(torch.ones(2, 2, 0, device="cuda"), torch.ones(2, device="cuda"))
    assert tuple(got.shape) == (2, 0)
    got = ome.ein("ij,jk->ik")(torch.ones(3, 0, device="cuda"), torch.ones(0, 4, device="cuda"))
    assert torch.equal(got.cpu(), torch.zeros(3, 4))


@pytest.mark.parametrize("code,sizes", [
    ("ij,jk->ik", dict(i=512, j=2048, k=512)),            # 8 tiles of 128x256, every tile split along K
    ("ij,jk->ik", dict(i=2304, j=512, k=2304)),           # a whole wave of tiles + a split remainder wave
    ("ij,kj->ki", dict(i=1000, j=1536, k=700)),           # ragged tiles (last 256-wide tile 188 columns)
    ("bij,bjk->bik", dict(b=4, i=512, j=512, k=512)),     # batched
    ("abcd,cdef->abef", dict(a=24, b=20, c=32, d=40, e=18, f=30)),   # multi-mode groups
])
def test_large_gemm_packed(code, sizes):
    """GEMMs large enough for the pre-split (packed-operand) tensor-core kernel
    (M, N >= 256, K >= 512, >= 1 GFLOP), FP32 against FP64 at the BF16x6
    tolerance."""
    rng = np.random.default_rng(12)
    ixs, iy = parse(code)
    xs = [gen(rng, [sizes[l] for l in ix], "f32") for ix in ixs]
    got = to_np(ome.einsum(ome.EinCode(ixs, iy), [to_dev(x, "f32") for x in xs], sizes))
    ome.device_status()
    assert_match(got, oracle(ixs, iy, xs, sizes, "f32", wide=True), "f32", 1e-6)


def kernel_names(fn):
    """Run fn() with the library's kernel-event record on; (result, main kernel names)."""
    import ctypes as C
    from omeinsum_b200 import _lib
    lib = _lib.load()
    lib.ome_kernel_timing(16)
    try:
        out = fn()
        torch.cuda.synchronize()
        ome.device_status()
        ms = (C.c_float * 16)()
        names = (C.c_char_p * 16)()
        cnt = C.c_int32()
        lib.ome_kernel_times(16, ms, names, C.byref(cnt))
    finally:
        lib.ome_kernel_timing(0)
    return out, [names[i].decode() for i in range(cnt.value)]


@pytest.mark.parametrize("prec,rtol", [(3, 1e-6), (2, 1e-5)])
@pytest.mark.parametrize("code,sizes", [
    ("ij,jk->ik", dict(i=300, j=520, k=700)),          # A row-major (M contiguous), B K-major; ragged M, N, K
    ("ji,jk->ik", dict(i=260, j=1000, k=390)),         # both K-major
    ("ij,kj->ik", dict(i=512, j=776, k=640)),          # A row-major, B row-major (N contiguous)
    ("ji,kj->ik", dict(i=384, j=1000, k=300)),         # A K-major, B row-major
    ("ijl,jkl->ikl", dict(i=256, j=1024, k=256, l=3)),  # batched: 3-D tensor maps
    ("ij,jk->ik", dict(i=2560, j=320, k=2560)),        # a whole wave of cluster tiles + a split remainder
    ("ij,jk->ik", dict(i=256, j=16384, k=256)),        # one tile split along K over every cluster
])
def test_gemm_tma2(code, sizes, prec, rtol):
    """The 2-SM tensor-core GEMM fed by tensor maps over the FP32 operands
    (BF16 terms formed in shared memory) against FP64, in every operand
    orientation, with y <- 2y + 3f on a second call."""
    rng = np.random.default_rng(31)
    ixs, iy = parse(code)
    xs = [gen(rng, [sizes[l] for l in ix], "f32") for ix in ixs]
    c = ome.EinCode(ixs, iy)
    dxs = [to_dev(x, "f32") for x in xs]
    want = oracle(ixs, iy, xs, sizes, "f32", wide=True)
    ome.set_einsum_backend(ome.B200Backend(prec=prec))
    try:
        got, names = kernel_names(lambda: ome.einsum(c, dxs, sizes))
        assert names == ["k_gemm_tma2"], names
        assert_match(to_np(got), want, "f32", rtol)
        y0 = gen(rng, [sizes[l] for l in iy], "f32")
        yd = to_dev(y0, "f32")
        ome.einsum_(c, dxs, yd, 3, 2, sizes)
        ome.device_status()
        assert_match(to_np(yd), 3 * want + 2 * y0.astype(np.float64), "f32", rtol)
    finally:
        ome.set_einsum_backend(ome.B200Backend())


def test_packed_gemm_overflow_scratch():
    """A GEMM whose BF16 operand terms (804 MB for M = 1023, N = 1024,
    K = 65536) exceed the 256 MiB default workspace still runs on the packed
    kernel (a K stride of 1023 elements is not a whole number of 16-byte
    units, which the tensor-map kernel needs), through the context's overflow
    scratch, and matches FP64."""
    import ctypes as C
    from omeinsum_b200 import _lib
    _lib.release_workspaces()
    torch.manual_seed(3)
    a = torch.randn(1023, 65536, dtype=torch.float32, device="cuda")
    b = torch.randn(65536, 1024, dtype=torch.float32, device="cuda")
    A, B = a.t().contiguous().t(), b.t().contiguous().t()   # column-major
    lib = _lib.load()
    lib.ome_kernel_timing(8)
    try:
        y = ome.einsum(ome.EinCode([("i", "j"), ("j", "k")], ("i", "k")), [A, B])
        torch.cuda.synchronize()
        ome.device_status()
        ms = (C.c_float * 8)()
        names = (C.c_char_p * 8)()
        cnt = C.c_int32()
        lib.ome_kernel_times(8, ms, names, C.byref(cnt))
    finally:
        lib.ome_kernel_timing(0)
    assert [names[i].decode() for i in range(cnt.value)] == ["k_gemm_packed"]
    ref = A.double() @ B.double()
    err = ((y.double() - ref).norm() / ref.norm()).item()
    assert err < 1e-6, err


@pytest.mark.parametrize("dt", ["f32", "f64", "c64", "i64", "trop", "bool"])
@pytest.mark.parametrize("code,sizes", [
    ("ji,j->i", dict(i=12000, j=64)),              # GEMV with the summed mode contiguous: a warp per output
    ("i,i->", dict(i=65536)),                      # dot: one long run cut into rows, split over blocks
    ("ij,ij->j", dict(i=96, j=500)),               # batched dot, few outputs
    ("ijk,ik->k", dict(i=64, j=30, k=20)),         # second input constant along the row mode j
    ("ij,i,i->j", dict(i=33, j=40)),               # three inputs, rows not a multiple of the vector
])
def test_multi_input_contiguous_sums(code, sizes, dt):
    """Sum-products whose first summed mode is contiguous (or constant) in
    every input (dot products, GEMV with a contiguous row), and y <- 3y + 2f
    for Int64."""
    rng = np.random.default_rng(17)
    ixs, iy = parse(code)
    xs = [gen(rng, [sizes[l] for l in ix], dt) for ix in ixs]
    c = ome.EinCode(ixs, iy)
    got = to_np(ome.einsum(c, [to_dev(x, dt) for x in xs], sizes))
    ome.device_status()
    assert_match(got, oracle(ixs, iy, xs, sizes, dt), dt)
    if dt == "i64":
        y0 = gen(rng, [sizes[l] for l in iy], dt)
        yd = to_dev(y0, dt)
        ome.einsum_(c, [to_dev(x, dt) for x in xs], yd, 2, 3, sizes)
        assert_match(to_np(yd), 2 * oracle(ixs, iy, xs, sizes, dt) + 3 * y0, dt)


@pytest.mark.parametrize("dt", ["f32", "f64", "c64", "i64", "trop", "bool"])
@pytest.mark.parametrize("code,sizes", [
    ("ij,j->i", dict(i=300, j=200)),               # GEMV: summed mode strided, outputs contiguous
    ("ijk->ik", dict(i=40, j=300, k=10)),          # middle sum
    ("ij,j,j->i", dict(i=260, j=70)),              # three inputs
    ("ijk,jk->i", dict(i=512, j=9, k=11)),         # two summed modes (odometer carries)
])
def test_strided_sums(code, sizes, dt):
    """Sum-products whose summed modes are strided while the outputs are
    contiguous (a thread per output, summed space split), and y <- 3y + 2f
    for Int64."""
    rng = np.random.default_rng(16)
    ixs, iy = parse(code)
    xs = [gen(rng, [sizes[l] for l in ix], dt) for ix in ixs]
    c = ome.EinCode(ixs, iy)
    got = to_np(ome.einsum(c, [to_dev(x, dt) for x in xs], sizes))
    ome.device_status()
    assert_match(got, oracle(ixs, iy, xs, sizes, dt), dt)
    if dt == "i64":
        y0 = gen(rng, [sizes[l] for l in iy], dt)
        yd = to_dev(y0, dt)
        ome.einsum_(c, [to_dev(x, dt) for x in xs], yd, 2, 3, sizes)
        assert_match(to_np(yd), 2 * oracle(ixs, iy, xs, sizes, dt) + 3 * y0, dt)


@pytest.mark.parametrize("dt", ["f32", "f64", "c64", "i64", "trop", "bool"])
@pytest.mark.parametrize("code,sizes", [
    ("ijk->k", dict(i=64, j=512, k=8)),            # i, j merge into one run of 32768: cut into rows
    ("ij->j", dict(i=100000, j=3)),                # run of 100000 = 25 rows of 4000
    ("ij->j", dict(i=16411, j=5)),                 # prime run: no row length divides it
])
def test_sum_few_outputs_long_runs(code, sizes, dt):
    """Sum of one long contiguous run per output with few outputs (the run
    is viewed as rows so that the split reduction can spread it), and
    y <- 3y + 2f for Int64."""
    rng = np.random.default_rng(15)
    ixs, iy = parse(code)
    xs = [gen(rng, [sizes[l] for l in ix], dt) for ix in ixs]
    c = ome.EinCode(ixs, iy)
    got = to_np(ome.einsum(c, [to_dev(x, dt) for x in xs], sizes))
    ome.device_status()
    assert_match(got, oracle(ixs, iy, xs, sizes, dt), dt)
    if dt == "i64":
        y0 = gen(rng, [sizes[l] for l in iy], dt)
        yd = to_dev(y0, dt)
        ome.einsum_(c, [to_dev(x, dt) for x in xs], yd, 2, 3, sizes)
        assert_match(to_np(yd), 2 * oracle(ixs, iy, xs, sizes, dt) + 3 * y0, dt)


@pytest.mark.parametrize("dt", ["f32", "f64", "c64", "i64", "trop", "bool"])
@pytest.mark.parametrize("code,sizes", [
    ("ijk->jk", dict(i=64, j=96, k=160)),          # 15360 outputs of 64 contiguous elements: 16-byte loads
    ("ijk->jk", dict(i=37, j=100, k=100)),         # rows of 37: element loads
    ("ijkl->jl", dict(i=40, j=50, k=6, l=200)),    # a second summed mode (strided rows)
])
def test_sum_many_outputs(code, sizes, dt):
    """Sum over a contiguous leading mode with many outputs (one warp per
    output), and y <- 3y + 2f for Int64."""
    rng = np.random.default_rng(14)
    ixs, iy = parse(code)
    xs = [gen(rng, [sizes[l] for l in ix], dt) for ix in ixs]
    c = ome.EinCode(ixs, iy)
    got = to_np(ome.einsum(c, [to_dev(x, dt) for x in xs], sizes))
    ome.device_status()
    assert_match(got, oracle(ixs, iy, xs, sizes, dt), dt)
    if dt == "i64":
        y0 = gen(rng, [sizes[l] for l in iy], dt)
        yd = to_dev(y0, dt)
        ome.einsum_(c, [to_dev(x, dt) for x in xs], yd, 2, 3, sizes)
        assert_match(to_np(yd), 2 * oracle(ixs, iy, xs, sizes, dt) + 3 * y0, dt)


@pytest.mark.parametrize("dt", ["f32", "f64", "c64", "i64", "trop", "bool"])
@pytest.mark.parametrize("code,sizes", [
    ("bij,bjk->bik", dict(b=100, i=37, j=50, k=23)),     # ragged batch warp, partial 16x16 tiles
    ("bij,bkj->bki", dict(b=64, i=64, j=9, k=64)),        # transposed operands, full tiles
    ("bcij,bcjk->bcik", dict(b=40, c=3, i=5, j=7, k=6)),  # two batch modes, b innermost
    ("bij,bjk->bik", dict(b=101, i=64, j=200, k=40)),    # ragged batch group, 13 K chunks, partial second N slab
    ("bij,bjk->bik", dict(b=64, i=64, j=32, k=64)),      # no bounds tests (M = 64, N, K, L whole)
])
def test_batch_innermost_gemm(code, sizes, dt):
    """Batches of small GEMMs whose batch mode is contiguous in every tensor
    (column-major bij,bjk->bik), with y <- 2y + 3f for Int64."""
    rng = np.random.default_rng(13)
    ixs, iy = parse(code)
    xs = [gen(rng, [sizes[l] for l in ix], dt) for ix in ixs]
    c = ome.EinCode(ixs, iy)
    got = to_np(ome.einsum(c, [to_dev(x, dt) for x in xs], sizes))
    ome.device_status()
    assert_match(got, oracle(ixs, iy, xs, sizes, dt), dt)
    if dt == "i64":
        y0 = gen(rng, [sizes[l] for l in iy], dt)
        yd = to_dev(y0, dt)
        ome.einsum_(c, [to_dev(x, dt) for x in xs], yd, 3, 2, sizes)
        assert_match(to_np(yd), 3 * oracle(ixs, iy, xs, sizes, dt) + 2 * y0, dt)


@pytest.mark.parametrize("dts,want_dtype", [
    (("i64", "f32"), torch.float32),       # Julia: promote_type(Int64, Float32) == Float32 (NumPy would give float64)
    (("bool", "i64"), torch.int64),
    (("f32", "f64"), torch.float64),
    (("i64", "c64"), torch.complex64),
    (("f32", "c128"), torch.complex128),
])
@pytest.mark.parametrize("code", ["ij,jk->ik", "ij,jk,kl->il", "ijk,jkl->il"])
def test_mixed_eltype_inputs(code, dts, want_dtype):
    """Mixed-eltype inputs: the output eltype is Julia's promote_type of the
    inputs' (src/loop_einsum.jl:55-61, ext/CUDAExt.jl:34-47) and the inputs are
    converted to it before contracting (ext/CUDAExt.jl:116)."""
    rng = np.random.default_rng(21)
    ixs, iy = parse(code)
    sd = {l: 5 + (ord(l) % 4) for l in "ijkl"}
    kinds = [dts[k % 2] for k in range(len(ixs))]
    xs = [gen(rng, [sd[l] for l in ix], dt) for ix, dt in zip(ixs, kinds)]
    got = ome.einsum(ome.EinCode(ixs, iy), [to_dev(x, dt) for x, dt in zip(xs, kinds)], sd)
    assert got.dtype == want_dtype
    want = O.einsum(ixs, iy, xs, sd)
    assert str(want.dtype) == str(want_dtype).replace("torch.", "")
    tgt = {torch.float32: "f32", torch.float64: "f64", torch.int64: "i64", torch.complex64: "c64",
           torch.complex128: "c128"}[want_dtype]
    assert_match(to_np(got), want, tgt)


@pytest.mark.parametrize("dt", ["f64", "c64", "i64", "trop", "bool", "f32"])
@pytest.mark.parametrize("code,sizes", [
    ("ij,jk->ik", dict(i=100, j=20000, k=90)),          # a 2 x 2 grid of tiles: K split over blocks
    ("ijl,jkl->ikl", dict(i=70, j=5000, k=60, l=2)),    # batched
    ("ji,kj->ik", dict(i=130, j=3000, k=33)),           # transposed operands, ragged tiles
])
def test_cuda_core_gemm_split_k(code, sizes, dt):
    """CUDA-core GEMMs with a long K and few output tiles split K over blocks
    (partials summed in split order): FP64, complex, Int64, max-plus, Bool and
    plain FP32, with y <- 3y + 2f."""
    rng = np.random.default_rng(41)
    ixs, iy = parse(code)
    xs = [gen(rng, [sizes[l] for l in ix], dt) for ix in ixs]
    c = ome.EinCode(ixs, iy)
    if dt == "f32":
        ome.set_einsum_backend(ome.B200Backend(prec=1))
    try:
        got, names = kernel_names(lambda: ome.einsum(c, [to_dev(x, dt) for x in xs], sizes))
        assert names == ["k_gemm_simt"], names
        assert_match(to_np(got), oracle(ixs, iy, xs, sizes, dt), dt)
        if dt == "i64":
            y0 = gen(rng, [sizes[l] for l in iy], dt)
            yd = to_dev(y0, dt)
            ome.einsum_(c, [to_dev(x, dt) for x in xs], yd, 2, 3, sizes)
            assert_match(to_np(yd), 2 * oracle(ixs, iy, xs, sizes, dt) + 3 * y0, dt)
    finally:
        ome.set_einsum_backend(ome.B200Backend())


@pytest.mark.parametrize("prec,rtol", [(3, 1e-6), (2, 1e-5)])
@pytest.mark.parametrize("code,sizes", [
    ("bij,bjk->bik", dict(b=512, i=64, j=64, k=64)),    # the benchmark's shape: whole boxes
    ("bij,bjk->bik", dict(b=100, i=37, j=50, k=23)),    # ragged rows, columns and k, a last group of 4
    ("bij,bkj->bki", dict(b=64, i=64, j=200, k=48)),    # B and C with transposed modes, 7 k stages
    ("bij,bjk->bik", dict(b=8, i=16, j=8, k=64)),       # one k stage, mostly padding
])
def test_batch_innermost_tensor_core_gemm(code, sizes, prec, rtol):
    """Batches of small FP32 GEMMs with the batch mode contiguous everywhere
    (column-major bij,bjk->bik) on the tensor cores, two batches per
    block-diagonal MMA, against FP64, with y <- 2y + 3f on a second call."""
    rng = np.random.default_rng(43)
    ixs, iy = parse(code)
    xs = [gen(rng, [sizes[l] for l in ix], "f32") for ix in ixs]
    c = ome.EinCode(ixs, iy)
    dxs = [to_dev(x, "f32") for x in xs]
    want = oracle(ixs, iy, xs, sizes, "f32", wide=True)
    ome.set_einsum_backend(ome.B200Backend(prec=prec))
    try:
        got, names = kernel_names(lambda: ome.einsum(c, dxs, sizes))
        assert names == ["k_gemm_bdiag"], names
        assert_match(to_np(got), want, "f32", rtol)
        y0 = gen(rng, [sizes[l] for l in iy], "f32")
        yd = to_dev(y0, "f32")
        ome.einsum_(c, dxs, yd, 3, 2, sizes)
        ome.device_status()
        assert_match(to_np(yd), 3 * want + 2 * y0.astype(np.float64), "f32", rtol)
    finally:
        ome.set_einsum_backend(ome.B200Backend())


@pytest.mark.parametrize("dt", ["f32", "trop"])
@pytest.mark.parametrize("code,sizes", [
    ("abcd->dcab", dict(a=8, b=9, c=12, d=64)),      # x's contiguous mode of 8 merged with b: 72-wide rows
    ("abcd->dcab", dict(a=16, b=5, c=7, d=36)),
    ("abcd->dcab", dict(a=16, b=3, c=7, d=36)),      # 48 < 64: not merged
    ("abcd->dcab", dict(a=32, b=6, c=2, d=128)),
    ("abcde->ecadb", dict(a=32, b=32, c=4, d=4, e=128)),   # the rule-suite permutation, smaller
])
def test_transpose_merged_x_rows(dt, code, sizes):
    """k_transpose_v4 (Float32) with x's short contiguous mode and the next x
    mode tiled together (256-byte x rows): exact against the oracle, with and
    without alpha-beta; the same permutations of tropical numbers."""
    rng = np.random.default_rng(zlib.crc32(code.encode()) + sizes["a"])
    ixs, iy = parse(code)
    x = gen(rng, [sizes[l] for l in ixs[0]], dt)
    y0 = gen(rng, [sizes[l] for l in iy], dt)
    for sx, sy in [(True, False)] + ([(2.0, 0.5)] if dt == "f32" else []):
        yd = to_dev(y0, dt)
        ynp = to_np(yd).copy()
        out, names = kernel_names(lambda: ome.einsum_(ome.ein(code), [to_dev(x, dt)], yd, sx, sy, sizes))
        want = oracle(ixs, iy, [x], sizes, dt)
        if not (sx is True and sy is False):
            want = sx * want + sy * ynp
        if dt == "f32":   # (tropical numbers here are 8 bytes: k_transpose32)
            assert "k_transpose_v4" in names, names
        assert_match(to_np(yd), want, dt)
