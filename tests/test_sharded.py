"""Slice sharding (multi-GPU row) on the host: the slice-range partition and
the all-reduce of partials, run as world_size-2 ``gloo`` ranks on the CPU.
Each rank's partial comes from the oracle; the combined result must equal the
oracle's full cross-slice result (bit-exact for Int64, Bool and max-plus;
FP64 partials to 1e-12, as they only re-associate the slice sum)."""
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp

import omeinsum_b200 as ome
import sharded_worker as W


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


@pytest.mark.parametrize("n,world", [(0, 1), (1, 2), (5, 2), (6, 2), (7, 3), (100, 8), (3, 8)])
def test_slice_range_partition(n, world):
    ranges = [ome.slice_range(n, r, world) for r in range(world)]
    assert ranges[0][0] == 0 and ranges[-1][1] == n
    for (b0, e0), (b1, _) in zip(ranges, ranges[1:]):
        assert e0 == b1
    sizes = [e - b for b, e in ranges]
    assert max(sizes) - min(sizes) <= 1 and min(sizes) >= 0


def test_slice_range_rejects_bad_rank():
    with pytest.raises(ome.ArgumentError):
        ome.slice_range(4, 2, 2)


@pytest.mark.parametrize("name", sorted(W.CASES))
def test_gloo_two_ranks(name, tmp_path):
    out = str(tmp_path / "r.npy")
    mp.start_processes(W.worker, args=(2, _free_port(), name, out), nprocs=2, join=True, start_method="spawn")
    got = np.load(out)
    O, ne, slicing, sd, xs, alg, acc, op = W.make_case(name)
    want = np.asarray(O.sliced_partial(slicing, ne, xs, sd, 0, 1 << 62, alg, acc))
    assert got.shape == want.shape and got.dtype == want.dtype
    if want.dtype in (np.float64, np.complex128) and alg is None:
        assert np.linalg.norm(got - want) <= 1e-12 * max(np.linalg.norm(want), 1e-300)
        # and the combined partial is the unsliced contraction: slices are
        # evaluated in FP32/ComplexF32, so to the FP32 tolerance of FP64 values
        wide = [x.astype(np.float64 if x.dtype == np.float32 else np.complex128) for x in xs]
        ref = O.nested_einsum(ne, wide, sd)
        assert np.linalg.norm(got - ref) <= 1e-5 * max(np.linalg.norm(ref), 1e-300)
    else:
        assert np.array_equal(got, want)
        assert np.array_equal(got, np.asarray(O.nested_einsum(ne, xs, sd, alg)))
