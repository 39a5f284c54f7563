"""Rank body for the world_size-2 slice-sharding tests (spawned processes).

Each rank evaluates its contiguous slice range with the oracle (the CPU
stand-in for ome_plan_execute_slices on its GPU), combines the partials with
the package's all-reduce over a ``gloo`` group, and rank 0 saves the result.
"""
import datetime
import os

import numpy as np
import torch
import torch.distributed as dist

from conftest import load_oracle, load_package

# name -> (tree, slicing, extents, dtype); extents keep each oracle run tiny
CASES = {
    "f32_internal": ("(ij,jk),(kl,lm)->im", ["j", "k"], dict(i=3, j=4, k=3, l=2, m=3), "f32"),
    "f32_output": ("(ij,jk),(kl,lm)->im", ["i", "l"], dict(i=3, j=2, k=4, l=3, m=2), "f32"),
    "c64": ("(ij,jk),(kl,lm)->im", ["j"], dict(i=2, j=5, k=3, l=2, m=3), "c64"),
    "i64": ("(ijk,jkl),klm->im", ["k", "l"], dict(i=2, j=3, k=3, l=2, m=2), "i64"),
    "trop": ("(ij,jk),(kl,lm)->", ["j", "l"], dict(i=3, j=3, k=2, l=3, m=2), "trop"),
    "bool": ("(ij,jk),(kl,lm)->im", ["k"], dict(i=2, j=2, k=3, l=2, m=2), "bool"),
    "one_slice": ("(ij,jk),(kl,lm)->im", ["j"], dict(i=2, j=1, k=3, l=2, m=3), "f32"),
}


def make_case(name):
    O = load_oracle()
    code, slicing, sd, dt = CASES[name]
    ne = O.parse_nested(code)
    rng = np.random.default_rng(sum(map(ord, name)))
    xs = []
    for ix in O.getixsv(ne):
        shape = tuple(sd[l] for l in ix)
        if dt == "f32":
            xs.append(rng.standard_normal(shape).astype(np.float32))
        elif dt == "c64":
            xs.append((rng.standard_normal(shape) + 1j * rng.standard_normal(shape)).astype(np.complex64))
        elif dt == "i64":
            xs.append(rng.integers(-8, 9, shape).astype(np.int64))
        elif dt == "bool":
            xs.append(rng.integers(0, 2, shape).astype(bool))
        else:
            xs.append(rng.integers(-8, 9, shape).astype(np.float64) + 0.25 * rng.standard_normal(shape))
    alg = O.TROPICAL if dt == "trop" else None
    acc = np.float64 if dt == "f32" else np.complex128 if dt == "c64" else None
    op = 1 if dt in ("trop", "bool") else 0
    return O, ne, slicing, sd, xs, alg, acc, op


def worker(rank, world, port, name, out_path):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        ome = load_package()
        O, ne, slicing, sd, xs, alg, acc, op = make_case(name)
        ns = int(np.prod([sd[l] for l in slicing]))
        b, e = ome.slice_range(ns, rank, world)
        part = O.sliced_partial(slicing, ne, xs, sd, b, e, alg, acc)
        t = torch.from_numpy(np.array(part, order="F"))  # Julia layout, as on the device
        ome.allreduce_partial(t, op)
        if rank == 0:
            np.save(out_path, t.numpy())
    finally:
        dist.destroy_process_group()
