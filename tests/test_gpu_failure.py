"""Failure detection of the bounded device-side waits, exercised without a
GPU fault: a one-block kernel waits on an mbarrier that nothing arrives on,
gives up after a short limit and records the timeout flag; the host then
reads OME_TIMEOUT through ome_device_status, once, and the context keeps
working."""
import numpy as np
import pytest
import torch

import omeinsum_b200 as ome
from helpers import assert_match, gen, oracle, parse, to_dev, to_np

pytestmark = pytest.mark.gpu


def test_expired_wait_reports_timeout_once():
    lib = ome.load_library()
    torch.cuda.synchronize()
    ome.device_status()                                   # start from a clear flag
    assert lib.ome_selftest_wait_timeout(None, 20_000_000) == 0   # 20 ms limit
    with pytest.raises(ome.OMEError, match="bounded wait"):
        ome.device_status()
    ome.device_status()                                   # reported once, then clear


def test_context_usable_after_timeout():
    lib = ome.load_library()
    assert lib.ome_selftest_wait_timeout(None, 1_000_000) == 0
    with pytest.raises(ome.OMEError):
        ome.device_status()
    rng = np.random.default_rng(21)
    ixs, iy = parse("ij,jk->ik")
    sizes = dict(i=300, j=400, k=200)
    xs = [gen(rng, [sizes[l] for l in ix], "f32") for ix in ixs]
    got = to_np(ome.einsum(ome.EinCode(ixs, iy), [to_dev(x, "f32") for x in xs], sizes))
    ome.device_status()
    assert_match(got, oracle(ixs, iy, xs, sizes, "f32", wide=True), "f32", 1e-6)
