"""Batched contractions of uneven shapes (one grouped launch) against the
oracle: MPS transfer contractions (ab,bcd)->acd, (acd,de)->ace in ComplexF32
with random bond dimensions, plus exact Int64 and tropical batches.  Tile
config 3 is the tensor-core grouped kernel (BF16x6 split products; ComplexF32
through its real 2 x 2 embedding), held to the same 1e-5 as the CUDA-core
tiles."""
import numpy as np
import pytest
import torch

import ome_oracle as O
import omeinsum_b200 as ome
from helpers import assert_match, gen, relerr, to_dev, to_np

pytestmark = pytest.mark.gpu


def mps_jobs(n, seed):
    rng = np.random.default_rng(seed)
    jobs = []
    for _ in range(n):
        a, b, d, e = (int(8 * rng.integers(1, 17)) for _ in range(4))
        c = int(rng.choice([2, 4]))
        jobs.append(dict(a=a, b=b, c=c, d=d, e=e))
    return jobs


@pytest.mark.parametrize("tile_config", [-1, 0, 2, 3])
def test_mps_transfer_batch_complex64(tile_config):
    rng = np.random.default_rng(9)
    jobs = mps_jobs(40, 9)
    X = []
    for s in jobs:
        X.append([gen(rng, (s["a"], s["b"]), "c64"), gen(rng, (s["b"], s["c"], s["d"]), "c64"),
                  gen(rng, (s["d"], s["e"]), "c64")])
    dev = [[to_dev(x, "c64") for x in xs] for xs in X]
    b1 = ome.BatchedEinsum(ome.ein("ab,bcd->acd"), [(x[0], x[1]) for x in dev], tile_config=tile_config)
    b2 = ome.BatchedEinsum(ome.ein("acd,de->ace"), [(t, x[2]) for t, x in zip(b1.outputs, dev)],
                           tile_config=tile_config)
    g = ome.capture_graph(lambda: (b1.run(), b2.run()))
    for _ in range(2):
        g.replay()
        torch.cuda.synchronize()
        for s, xs, y in zip(jobs, X, b2.outputs):
            ne = O.parse_nested("(ab,bcd),de->ace")
            want = O.nested_einsum(ne, [x.astype(np.complex128) for x in xs], s)
            assert relerr(to_np(y), want) < 1e-5
    if tile_config >= 0:
        assert b1.tile_config == tile_config


@pytest.mark.parametrize("dt", ["i64", "trop", "f64"])
def test_uneven_batch_exact(dt):
    rng = np.random.default_rng(3)
    xs_list, wants = [], []
    for i in range(17):
        m, k, n = (int(v) for v in rng.integers(1, 70, 3))
        a, b = gen(rng, (m, k), dt), gen(rng, (k, n), dt)
        xs_list.append((to_dev(a, dt), to_dev(b, dt)))
        wants.append(O.einsum([("i", "j"), ("j", "k")], ("k", "i"), [a, b], {"i": m, "j": k, "k": n},
                              O.TROPICAL if dt == "trop" else None))
    bt = ome.BatchedEinsum(ome.ein("ij,jk->ki"), xs_list)
    bt.run()
    torch.cuda.synchronize()
    for y, w in zip(bt.outputs, wants):
        assert_match(to_np(y), w, dt)


def test_batch_rejects_unmergeable_groups():
    x = torch.zeros(4, 4, 4, device="cuda")
    with pytest.raises(ome.OMEError):
        # output (k, i, j) of x1's (i, j): i and j are not adjacent in the output -> two M modes
        ome.BatchedEinsum(ome.ein("ijl,lk->ikj"), [(x, torch.zeros(4, 4, device="cuda"))])


def _tc_kernel_ran(fn):
    from test_gpu_parity import kernel_names
    _, names = kernel_names(fn)
    return "k_group_tc" in names


@pytest.mark.parametrize("dt", ["f32", "c64"])
def test_tensor_core_group_uneven_alpha_beta(dt):
    """Uneven problems (ragged M, N, K around the 128 x 128 x 32 tiles, K = 1,
    a batch mode, transposed operands) with y = 2.5 x1 x2 - 0.75 y (complex:
    (1.5 - 0.5i) x1 x2 + (0.25 + 1i) y)."""
    rng = np.random.default_rng(21)
    shapes = [(1, 1, 1, 1), (127, 33, 129, 1), (128, 32, 128, 1), (129, 31, 257, 2), (300, 1, 64, 1),
              (17, 513, 200, 3), (64, 64, 64, 5), (250, 100, 3, 1), (2, 700, 2, 1)]
    cplx = dt == "c64"
    sx = complex(1.5, -0.5) if cplx else 2.5
    sy = complex(0.25, 1.0) if cplx else -0.75
    xs_list, ys, wants = [], [], []
    for (m, k, n, l) in shapes:
        a, b = gen(rng, (k, m, l), dt), gen(rng, (k, n, l), dt)   # x1 K-major (k first)
        y0 = gen(rng, (m, n, l), dt)
        xs_list.append((to_dev(a, dt), to_dev(b, dt)))
        ys.append(to_dev(y0, dt))
        wide = np.complex128 if cplx else np.float64
        ab = O.einsum([("k", "i", "l"), ("k", "j", "l")], ("i", "j", "l"), [a.astype(wide), b.astype(wide)],
                      {"i": m, "j": n, "k": k, "l": l})
        wants.append(sx * ab + sy * y0.astype(ab.dtype))
    bt = ome.BatchedEinsum(ome.ein("kil,kjl->ijl"), xs_list, ys=ys, tile_config=3)
    assert bt.tile_config == 3
    assert _tc_kernel_ran(lambda: bt.run(sx, sy))
    for y, w in zip(bt.outputs, wants):
        assert relerr(to_np(y), w) < 1e-5


def test_tensor_core_group_rejects_other_dtypes():
    x = torch.zeros(8, 8, dtype=torch.int64, device="cuda")
    with pytest.raises(ome.OMEError):
        ome.BatchedEinsum(ome.ein("ij,jk->ik"), [(x, x)], tile_config=3)
    bt = ome.BatchedEinsum(ome.ein("ij,jk->ik"), [(x, x)])   # autotune skips the tensor-core kernel
    assert bt.tuned_us[3] == -1 and bt.tile_config != 3
