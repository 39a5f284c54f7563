"""einsum_many: independent contractions of host tensors with uploads,
contractions and downloads on three streams.  Every result must equal the
same contraction through einsum (bit for bit: the same kernels run) and the
oracle."""
import numpy as np
import pytest
import torch

import omeinsum_b200 as ome
from helpers import assert_match, gen, oracle, parse, to_np

pytestmark = pytest.mark.gpu

JOBS = [
    ("ij,jk->ik", dict(i=300, j=700, k=500), "f32"),
    ("abcde->ecadb", dict(a=17, b=9, c=33, d=5, e=12), "f32"),
    ("ijk,jkl->il", dict(i=40, j=30, k=20, l=50), "i64"),
    ("ij,jk->ik", dict(i=64, j=48, k=32), "trop"),
    ("ii->", dict(i=513), "f64"),
    ("bij,bjk->bik", dict(b=64, i=16, j=24, k=8), "c64"),
    ("ij,jk,kl->il", dict(i=30, j=20, k=40, l=10), "f32"),
]


def _host(a, dt):
    t = torch.from_numpy(np.array(a, order="F")).pin_memory()
    return ome.TropicalTensor(t) if dt == "trop" else t


@pytest.mark.parametrize("window", [1, 3])
def test_many_matches_einsum(window):
    rng = np.random.default_rng(21)
    jobs, raw = [], []
    for code, sd, dt in JOBS:
        ixs, iy = parse(code)
        xs = [gen(rng, [sd[l] for l in ix], dt) for ix in ixs]
        raw.append((ixs, iy, xs, sd, dt))
        c = ome.ein("(ij,jk),kl->il") if len(ixs) == 3 else ome.EinCode(ixs, iy)
        jobs.append((c, [_host(x, dt) for x in xs], sd))
    # one job with device inputs runs as plain einsum
    dev_x = [torch.from_numpy(np.array(x, order="F")).cuda() for x in raw[0][2]]
    jobs.append((ome.EinCode(raw[0][0], raw[0][1]), dev_x, raw[0][3]))
    got = ome.einsum_many(jobs, window=window)
    ome.device_status()
    assert len(got) == len(jobs)
    for (c, xs, sd), g in zip(jobs, got[:-1]):
        ref = ome.einsum(c, xs, sd)
        assert not (g.data if isinstance(g, ome.TropicalTensor) else g).is_cuda
        assert np.array_equal(to_np(g), to_np(ref))
    for (ixs, iy, xs, sd, dt), g in zip(raw, got[:-1]):
        assert_match(to_np(g), oracle(ixs, iy, xs, sd, dt), dt)
    assert got[-1].is_cuda
    assert np.array_equal(to_np(got[-1]), to_np(got[0]))


def test_many_empty_and_window():
    assert ome.einsum_many([]) == []
    with pytest.raises(ome.ArgumentError):
        ome.einsum_many([], window=0)
