"""GPU parity of contraction trees: NestedEinsum, SlicedEinsum (FP64 cross-slice
sum), cost_and_gradient, against the oracle's restatement of
src/einsequence.jl, src/slicing.jl and src/bp.jl."""
import numpy as np
import pytest
import torch

import ome_oracle as O
import omeinsum_b200 as ome
from helpers import assert_match, gen, relerr, to_dev, to_np

pytestmark = pytest.mark.gpu


def oracle_tree(ne):
    if ne.isleaf:
        return O.leaf(ne.tensorindex)
    return O.Node(args=[oracle_tree(a) for a in ne.args], ixs=[list(ix) for ix in ne.eins.ixs], iy=list(ne.eins.iy))


@pytest.mark.parametrize("dt", ["f32", "f64", "c64", "i64", "trop"])
def test_nested_config1(dt):
    # ein"(ijk,jkl),klm->im" with every extent 64, uniform[0,1) Float32 (seed 0)
    rng = np.random.default_rng(0)
    ne = ome.ein("(ijk,jkl),klm->im")
    sd = {l: 64 for l in "ijklm"}
    if dt == "f32":
        xs = [rng.random((64, 64, 64)).astype(np.float32) for _ in range(3)]
    else:
        xs = [gen(rng, (64, 64, 64), dt) for _ in range(3)]
    alg = O.TROPICAL if dt == "trop" else None
    want = O.nested_einsum(oracle_tree(ne), xs, sd, alg)
    got = to_np(ne(*[to_dev(x, dt) for x in xs]))
    assert_match(got, want, dt)
    if dt == "f32":
        want64 = O.nested_einsum(oracle_tree(ne), [x.astype(np.float64) for x in xs], sd)
        assert relerr(got, want64) <= 1e-5


@pytest.mark.parametrize("dt", ["f32", "f64", "c64", "i64", "trop", "bool"])
def test_sliced_matches_unsliced(dt):
    # test/slicing.jl:13-32
    rng = np.random.default_rng(1)
    se = ome.SlicedEinsum(["i", "l"], ome.ein("(ij,jk),(kl,lm)->im"))
    sd = {"i": 2, "j": 3, "k": 4, "l": 5, "m": 6}
    alg = O.TROPICAL if dt == "trop" else None
    for _ in range(3):
        xs = [gen(rng, s, dt) for s in [(2, 3), (3, 4), (4, 5), (5, 6)]]
        want = O.nested_einsum(oracle_tree(se.eins), xs, sd, alg)
        got = to_np(se(*[to_dev(x, dt) for x in xs]))
        assert_match(got, want, dt)
        # einsum! into a preallocated output with sx, sy
        if dt in ("f64", "i64"):
            y0 = gen(rng, (2, 6), dt)
            yd = to_dev(y0, dt)
            ome.einsum_(se, [to_dev(x, dt) for x in xs], yd, 2, 3)
            assert_match(to_np(yd), 2 * want + 3 * y0, dt)


def test_sliced_internal_labels_fp64_accumulation():
    rng = np.random.default_rng(2)
    ne = ome.ein("(ij,jk),(kl,lm)->im")
    se = ome.SlicedEinsum(["j", "k"], ne)
    sd = {"i": 8, "j": 16, "k": 16, "l": 8, "m": 8}
    xs = [rng.standard_normal(s).astype(np.float32) for s in [(8, 16), (16, 16), (16, 8), (8, 8)]]
    want = O.nested_einsum(oracle_tree(ne), [x.astype(np.float64) for x in xs], sd)
    got = to_np(se(*[to_dev(x, "f32") for x in xs]))
    assert relerr(got, want) <= 1e-6


@pytest.mark.parametrize("dt", ["f64", "c128", "f32"])
def test_cost_and_gradient(dt):
    # test/bp.jl:3-17 (Zygote replaced by the oracle's restatement of bp.jl)
    rng = np.random.default_rng(3)
    ne = ome.ein("(ij, jk), ki->")
    xs = [gen(rng, s, dt) for s in [(2, 3), (3, 4), (4, 2)]]
    cost, grads = ome.cost_and_gradient(ne, [to_dev(x, dt) for x in xs])
    c0, g0 = O.cost_and_gradient(oracle_tree(ne), xs)
    rt = 1e-5 if dt == "f32" else 1e-12
    assert_match(to_np(cost), c0, dt, rt)
    for g, w in zip(grads, g0):
        assert_match(to_np(g), w, dt, rt)


def test_gradient_with_cotangent_and_optimized_tree():
    rng = np.random.default_rng(4)
    code = ome.ein("ij,jk,kl->il")
    opt = ome.optimize_code(code, ome.uniformsize(code, 5), ome.GreedyMethod())
    xs = [rng.standard_normal((5, 5)) for _ in range(3)]
    dy = rng.standard_normal((5, 5))
    cost, grads = ome.cost_and_gradient(opt, [to_dev(x, "f64") for x in xs], to_dev(dy, "f64"))
    c0, g0 = O.cost_and_gradient(oracle_tree(opt), xs, dy)
    assert relerr(to_np(cost), c0) < 1e-12
    for g, w in zip(grads, g0):
        assert relerr(to_np(g), w) < 1e-12


def test_fullerene_tropical_66_on_gpu():
    from test_oracle import c60_code
    edges, verts = c60_code()
    code = ome.EinCode(edges + verts, ())
    sd = {i: 2 for i in range(1, 61)}
    opt = ome.optimize_code(code, sd, ome.GreedyMethod(nrepeat=3, seed=2))
    xs = [torch.tensor([[-1.0, 1.0], [1.0, -1.0]], dtype=torch.float64)] * 90 + \
         [torch.tensor([0.0, 0.0], dtype=torch.float64)] * 60
    xs = [ome.TropicalTensor(x.cuda()) for x in xs]
    assert float(opt(*xs).data.cpu()) == 66
    sc = ome.slice_code(opt, sd, ome.GreedySlicer(sc_target=8))
    assert float(sc(*xs).data.cpu()) == 66


def test_three_colouring_petersen_int64():
    s = np.zeros((3, 3, 3), dtype=np.int64)
    for i in range(3):
        for j in range(3):
            for k in range(3):
                s[i, j, k] = int(len({i, j, k}) == 3)
    sd = torch.from_numpy(s).cuda()
    assert int(ome.ein("ijk,ijk->")(sd, sd)) == 6
    code = ome.ein("afl,bhn,cjf,dlh,enj,ago,big,cki,dmk,eom->")
    opt = ome.optimize_code(code, ome.uniformsize(code, 3), ome.GreedyMethod())
    assert int(opt(*([sd] * 10))) == 0


@pytest.mark.parametrize("dt", ["f64", "f32", "i64"])
def test_sliced_network_many_nodes(dt):
    """A 3-regular network (24 vertices, bond 2) sliced on three labels equals
    the unsliced tree; exercises the workspace plan with many live buffers."""
    rng = np.random.default_rng(12)
    n = 24
    while True:
        stubs = np.repeat(np.arange(n), 3)
        rng.shuffle(stubs)
        pairs = [tuple(sorted(p)) for p in stubs.reshape(-1, 2)]
        if all(a != b for a, b in pairs) and len(set(pairs)) == len(pairs):
            break
    inc = [[] for _ in range(n)]
    for i, (a, b) in enumerate(pairs):
        inc[a].append(i)
        inc[b].append(i)
    code = ome.EinCode([tuple(v) for v in inc], ())
    sd = {i: 2 for i in range(len(pairs))}
    opt = ome.optimize_code(code, sd, ome.GreedyMethod(nrepeat=2))
    inner = [l for l in ome.label_elimination_order(opt)][:3]
    se = ome.SlicedEinsum(inner, opt)
    xs = [gen(rng, (2, 2, 2), dt) for _ in range(n)]
    want = O.nested_einsum(oracle_tree(opt), xs, sd)
    got = to_np(se(*[to_dev(x, dt) for x in xs]))
    assert_match(got, want, dt, 1e-5 if dt == "f32" else None)
    got2 = to_np(opt(*[to_dev(x, dt) for x in xs]))
    assert_match(got2, want, dt, 1e-5 if dt == "f32" else None)


def test_config3_network_slices_against_oracle():
    """The precision benchmark's network (random 3-regular graph, n = 180,
    bond 2, FP32 normal(0,1)/sqrt(3), greedy order, sliced to 2^27 elements):
    the device's FP64 partial over the first and the last slice against the
    oracle's restatement of the slice loop (src/slicing.jl:118-137) on the
    same slices in FP64, and the BF16x6 FP32 partials against the same FP64
    oracle at 1e-5.  This anchors the benchmark's "error vs FP64" figures,
    which compare the device's own runs, to an independent evaluation."""
    import os
    import sys
    sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
    import bench
    code, sd, xs = bench.tn_network(ome, 180)
    opt = ome.optimize_code(code, sd, ome.GreedyMethod(nrepeat=10, seed=0))
    se = ome.slice_code(opt, sd, ome.GreedySlicer(sc_target=27))
    tree = oracle_tree(se.eins)
    x64 = [x.astype(np.float64) for x in xs]
    ome.set_einsum_backend(ome.B200Backend(prec=3))
    try:
        sh64 = ome.ShardedSlices(se, [torch.from_numpy(x).cuda() for x in x64])
        sh32 = ome.ShardedSlices(se, [torch.from_numpy(x).cuda() for x in xs])
        n = sh64.nslices
        assert n >= 2
        for b in (0, n - 1):
            want = O.sliced_partial(list(se.slicing), tree, x64, sd, b, b + 1)
            sh64.range = (b, b + 1)
            got64 = to_np(sh64.partial([torch.from_numpy(x).cuda() for x in x64]))
            ome.device_status()
            assert relerr(got64, want) <= 1e-12, (b, relerr(got64, want))
            sh32.range = (b, b + 1)
            got32 = to_np(sh32.partial([torch.from_numpy(x).cuda() for x in xs]))
            ome.device_status()
            assert relerr(got32, want) <= 1e-5, (b, relerr(got32, want))
    finally:
        ome.set_einsum_backend(ome.B200Backend())
