"""Batched contractions of uneven shapes (one grouped launch) against the
oracle: MPS transfer contractions (ab,bcd)->acd, (acd,de)->ace in ComplexF32
with random bond dimensions, plus exact Int64 and tropical batches."""
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


@pytest.mark.parametrize("tile_config", [-1, 0, 2])
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
