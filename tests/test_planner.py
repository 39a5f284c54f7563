"""Contraction-order search (host): TreeSA, TreeSASlicer and the MergeVectors
simplifier, against the reference's own expectations for them
(test/contractionorder.jl:31-70: on the C60 fullerene, TreeSA(ntrials=1) with
MergeVectors reaches space complexity 10, TreeSASlicer with sc_target=8
slices to 8, and both trees give the tropical ground state 66)."""
import math

import numpy as np
import pytest

import ome_oracle as O
import omeinsum_b200 as ome
from test_oracle import c60_code, to_oracle_tree


def _c60():
    edges, verts = c60_code()
    code = ome.EinCode(edges + verts, ())
    sd = {i: 2 for i in range(1, 61)}
    xs = [np.array([[-1.0, 1.0], [1.0, -1.0]])] * 90 + [np.array([0.0, 0.0])] * 60
    return code, sd, xs


def test_treesa_c60_space_complexity_10():
    code, sd, xs = _c60()
    opt = ome.optimize_code(code, sd, ome.TreeSA(ntrials=1, seed=1), simplifier=ome.MergeVectors())
    assert opt.flatten() == code
    assert ome.contraction_complexity(opt, sd).sc == 10
    assert O.nested_einsum(to_oracle_tree(opt), xs, sd, O.TROPICAL)[()] == 66


def test_treesa_slicer_c60_sc_8():
    code, sd, xs = _c60()
    opt = ome.optimize_code(code, sd, ome.TreeSA(ntrials=1, seed=1), simplifier=ome.MergeVectors())
    sc = ome.slice_code(opt, sd, ome.TreeSASlicer(score=ome.ScoreFunction(sc_target=8)))
    assert isinstance(sc, ome.SlicedEinsum)
    assert ome.contraction_complexity(sc, sd).sc == 8
    assert O.sliced_einsum(sc.slicing, to_oracle_tree(sc.eins), xs, sd, O.TROPICAL)[()] == 66


def _regular3(n, seed):
    rng = np.random.default_rng(seed)
    while True:
        stubs = rng.permutation(np.repeat(np.arange(n), 3))
        e = [tuple(sorted((int(a), int(b)))) for a, b in stubs.reshape(-1, 2)]
        if all(a != b for a, b in e) and len(set(e)) == len(e):
            return e


@pytest.mark.parametrize("n", [30, 60])
def test_treesa_not_worse_than_greedy(n):
    edges = _regular3(n, 5)
    inc = [[] for _ in range(n)]
    for k, (a, b) in enumerate(edges):
        inc[a].append(k)
        inc[b].append(k)
    code = ome.EinCode([tuple(v) for v in inc], ())
    sd = {k: 2 for k in range(len(edges))}
    g = ome.optimize_code(code, sd, ome.GreedyMethod(nrepeat=1, seed=0))
    t = ome.optimize_code(code, sd, ome.TreeSA(ntrials=2, niters=10, seed=3))
    assert t.flatten() == code
    cg, ct = ome.contraction_complexity(g, sd), ome.contraction_complexity(t, sd)
    assert ct.tc <= cg.tc + 1e-9 or ct.sc < cg.sc
    # values agree (a random real network, FP64 oracle on both trees)
    rng = np.random.default_rng(7)
    xs = [rng.standard_normal((2, 2, 2)) for _ in range(n)]
    a = O.nested_einsum(to_oracle_tree(g), xs, sd)[()]
    b = O.nested_einsum(to_oracle_tree(t), xs, sd)[()]
    assert abs(a - b) <= 1e-9 * max(abs(a), 1e-300)


def test_treesa_random_initializer_and_hyperedges():
    # a label shared by three tensors (hyperedge) and an open output label
    code = ome.EinCode([("a", "b"), ("b", "c", "x"), ("c", "d", "x"), ("d", "e", "x"), ("e", "a")], ("x",))
    sd = {l: 3 for l in "abcdex"}
    t = ome.optimize_code(code, sd, ome.TreeSA(ntrials=3, niters=5, initializer="random", seed=4))
    assert t.flatten() == code
    rng = np.random.default_rng(8)
    xs = [rng.standard_normal([sd[l] for l in ix]) for ix in code.ixs]
    want = O.einsum([list(ix) for ix in code.ixs], ["x"], xs, sd)
    got = O.nested_einsum(to_oracle_tree(t), xs, sd)
    assert np.allclose(got, want, rtol=1e-12)


def test_treesa_rejects_bad_tree():
    import ctypes as C
    lib = ome.load_library()
    arr = lambda T, v: (T * len(v))(*v)
    out = (C.c_int32 * 2)()
    # leaf 0 used twice
    rc = lib.ome_treesa(2, arr(C.c_int32, [1, 1]), arr(C.c_int32, [0, 0]), 0, arr(C.c_int32, [0]), 1,
                        arr(C.c_double, [1.0]), arr(C.c_int32, [-1, -1]), 20.0, 1.0, 0.0, 0.01, 0.05, 1.0, 1, 1, 0,
                        out, None)
    assert rc == 1
