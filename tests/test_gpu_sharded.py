"""GPU parity of slice sharding (ome_plan_execute_slices / ome_plan_finish):
the full slice range equals ome_plan_execute bit for bit, ranges computed
separately and combined with the algebra's addition equal the oracle, and a
one-rank NCCL group runs the whole sharded path.  Ranks on several GPUs are
emulated as separate ranges on one GPU, combined by torch (no two NCCL ranks
share a GPU)."""
import datetime
import socket

import numpy as np
import pytest
import torch
import torch.distributed as dist

import ome_oracle as O
import omeinsum_b200 as ome
from helpers import assert_match, gen, to_dev, to_np

pytestmark = pytest.mark.gpu

CODE = "(ij,jk),(kl,lm)->im"
SD = {"i": 6, "j": 5, "k": 4, "l": 3, "m": 7}


def _tree(ne):
    if ne.isleaf:
        return O.leaf(ne.tensorindex)
    return O.Node(args=[_tree(a) for a in ne.args], ixs=[list(ix) for ix in ne.eins.ixs], iy=list(ne.eins.iy))


def _inputs(dt, seed):
    rng = np.random.default_rng(seed)
    return [gen(rng, (SD[a], SD[b]), dt) for a, b in ["ij", "jk", "kl", "lm"]]


@pytest.mark.parametrize("slicing", [["j", "k"], ["i", "l"], ["m"]])
@pytest.mark.parametrize("dt", ["f32", "f64", "c64", "i64", "trop", "bool"])
def test_full_range_equals_execute(dt, slicing):
    se = ome.SlicedEinsum(slicing, ome.ein(CODE))
    xs = _inputs(dt, 3)
    dxs = [to_dev(x, dt) for x in xs]
    want = to_np(se(*dxs))
    sh = ome.ShardedSlices(se, dxs)
    assert sh.range == (0, int(np.prod([SD[l] for l in slicing])))
    got = to_np(sh(dxs))
    assert got.dtype == want.dtype and np.array_equal(got, want)


@pytest.mark.parametrize("world", [2, 3, 5])
@pytest.mark.parametrize("dt", ["f32", "c64", "i64", "trop", "bool"])
def test_emulated_ranks(dt, world):
    se = ome.SlicedEinsum(["j", "k"], ome.ein(CODE))
    xs = _inputs(dt, 4)
    dxs = [to_dev(x, dt) for x in xs]
    sh = ome.ShardedSlices(se, dxs)
    parts = []
    for r in range(world):
        sh.range = ome.slice_range(sh.nslices, r, world)
        parts.append(sh.partial(dxs))
    if sh.reduce_op == 0:
        total = sum(parts[1:], parts[0].clone())
    else:
        total = parts[0].clone()
        for q in parts[1:]:
            total = torch.maximum(total, q) if total.dtype != torch.bool else (total | q)
    y = to_np(sh.finish(total))
    want = O.nested_einsum(_tree(se.eins), xs, SD, O.TROPICAL if dt == "trop" else None)
    assert_match(y, want, dt)
    if dt in ("f32", "c64"):
        assert parts[0].dtype == (torch.float64 if dt == "f32" else torch.complex128)


def test_finish_alpha_beta():
    se = ome.SlicedEinsum(["k"], ome.ein(CODE))
    xs = _inputs("f64", 5)
    dxs = [to_dev(x, "f64") for x in xs]
    sh = ome.ShardedSlices(se, dxs)
    y0 = np.random.default_rng(6).standard_normal((SD["i"], SD["m"]))
    yd = to_dev(y0, "f64")
    sh(dxs, y=yd, sx=2.0, sy=-0.5)
    want = 2.0 * O.nested_einsum(_tree(se.eins), xs, SD) - 0.5 * y0
    assert_match(to_np(yd), want, "f64")


def test_range_errors():
    se = ome.SlicedEinsum(["j"], ome.ein(CODE))
    dxs = [to_dev(x, "f32") for x in _inputs("f32", 7)]
    sh = ome.ShardedSlices(se, dxs)
    for bad in [(-1, 2), (3, 2), (0, SD["j"] + 1)]:
        sh.range = bad
        with pytest.raises(ome.ArgumentError):
            sh.partial(dxs)


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def test_one_rank_nccl_group():
    se = ome.SlicedEinsum(["j", "l"], ome.ein(CODE))
    xs = _inputs("f32", 8)
    dxs = [to_dev(x, "f32") for x in xs]
    want = to_np(se(*dxs))
    dist.init_process_group("nccl", init_method=f"tcp://127.0.0.1:{_free_port()}", rank=0, world_size=1,
                            timeout=datetime.timedelta(seconds=60))
    try:
        got = to_np(ome.sharded_einsum(se, dxs))
        # the all-reduce of a column-major partial over the one-rank group
        # leaves it unchanged
        sh = ome.ShardedSlices(se, dxs)
        part = sh.partial(dxs)
        before = part.clone()
        ome.allreduce_partial(part, sh.reduce_op)
        torch.cuda.synchronize()
        assert torch.equal(part, before)
    finally:
        dist.destroy_process_group()
    assert np.array_equal(got, want)
