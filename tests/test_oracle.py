"""The CPU oracle pinned against the reference's own known-answer tests.

Every expected value below is transcribed from OMEinsum.jl's test suite (the
file:line is given per test).  The oracle (oracle/ome_oracle.py) restates the
reference's DefaultBackend algorithm; these tests show it reproduces the
reference's answers before it is trusted as the GPU parity checker.
"""
import itertools
import math

import numpy as np
import pytest

import ome_oracle as O
import omeinsum_b200 as ome

rng = np.random.default_rng(1234)


def close(a, b, rtol=1e-9):
    a, b = np.asarray(a), np.asarray(b)
    assert a.shape == b.shape, (a.shape, b.shape)
    na = np.linalg.norm((a - b).ravel())
    return na <= rtol * max(np.linalg.norm(a.ravel()), np.linalg.norm(b.ravel()), 1e-300)


# --- test/binaryrules.jl ------------------------------------------------------


def test_analyze_binary_kat():
    # test/binaryrules.jl:5-16
    sd = {1: 1, 2: 2, 3: 3, 4: 4, 6: 6, 7: 7, 8: 8}
    c1, c2, cy, s1, s2, s3, i1, i2, iy = O.analyze_binary([1, 2, 3, 4, 8], [2, 6, 6, 8, 4, 2], [7, 2, 1, 2, 2, 6], sd)
    assert c1 == [1, 4, 8, 2] and c2 == [4, 8, 6, 2] and cy == [1, 6, 2]
    assert s1 == [1, 32, 2] and s2 == [32, 6, 2]
    assert i1 == ["i", "j", "l"] and i2 == ["j", "k", "l"] and iy == ["i", "k", "l"]


def test_binary_rule_sweep_36():
    # test/binaryrules.jl:18-45: 2x5x5x5 sweep, 36 SimpleBinaryRules match
    sd = {c: 5 for c in "ijkl"}
    nmatch = 0
    for hb in (True, False):
        for i1 in [(), ("i",), ("j",), ("i", "j"), ("j", "i")]:
            for i2 in [(), ("k",), ("j",), ("k", "j"), ("j", "k")]:
                for i3 in [(), ("i",), ("k",), ("i", "k"), ("k", "i")]:
                    b = ("l",) if hb else ()
                    a1, a2, a3 = i1 + b, i2 + b, i3 + b
                    x1 = rng.standard_normal([5] * len(a1))
                    x2 = rng.standard_normal([5] * len(a2))
                    ref = O.loop_einsum([a1, a2], a3, [x1, x2], sd)
                    r = O.match_rule_binary(a1, a2, a3)
                    if r is not None:
                        nmatch += 1
                        out = np.zeros([5] * len(a3), order="F")
                        got = O.binary_einsum_(r, x1, x2, out, 1.0, 0.0)
                    else:
                        got = O.einsum([a1, a2], a3, [x1, x2], sd)
                    assert close(got, ref)
    assert nmatch == 36


@pytest.mark.parametrize("code", ["->", ",->", "ijl,jl->il", "ab,bc->ac", "abb,bc->ac", "ab,bc->acc", "ab,bce->ac",
                                  "ab,bc->ace", "bal,bcl->lcae", "bal,bcl->ca", "bal,bc->lca", "ddebal,bcf->lcac"])
def test_binary_einsum_composite(code):
    # test/binaryrules.jl:57-75 (ComplexF64, extents 5)
    lhs, iy = code.split("->")
    ixs = lhs.split(",") if lhs else [""]
    if code == "->":
        return
    sd = {c: 5 for c in "abcdefijkl"}
    xs = [np.asarray(rng.standard_normal([5] * len(ix)) + 1j * rng.standard_normal([5] * len(ix))) for ix in ixs]
    assert close(O.einsum([tuple(ix) for ix in ixs], tuple(iy), xs, sd), O.loop_einsum(ixs, iy, xs, sd))


def test_binary_regression_rank8():
    # test/binaryrules.jl:77-81
    x, y = rng.standard_normal([2] * 8), rng.standard_normal([2] * 5)
    ixs = [(10, 5, 4, 2, 6, 6, 7, 9), (1, 9, 8, 2, 10)]
    iy = (4, 10, 9, 7, 10)
    sd = O.get_size_dict(ixs, [x, y])
    assert close(O.einsum(ixs, iy, [x, y], sd), O.loop_einsum(ixs, iy, [x, y], sd))


# --- test/Core.jl -------------------------------------------------------------


def test_einarray_index_kat():
    # test/Core.jl:59-70: arr[3,4,2] == x1[4,3]*x2[3,2] (1-based; inner labels first)
    x1, x2 = rng.standard_normal((8, 8)), rng.standard_normal((8, 8))
    v = O.einarray_value([(1, 2), (2, 3)], (1, 3), [x1, x2], {1: 8, 2: 8, 3: 8}, (2, 3, 1))
    assert v == x1[3, 2] * x2[2, 1]


# --- test/unaryrules.jl -------------------------------------------------------


def test_unary_rules():
    sd = {1: 3, 2: 3, 3: 3, 4: 5}
    # Duplicate :5-13
    x = rng.standard_normal((3, 3, 3))
    y = np.zeros((3, 3, 3, 3, 3), order="F")
    ref = O.loop_einsum([(1, 2, 3)], (3, 2, 1, 1, 2), [x], sd)
    assert close(O.unary_duplicate_([1, 2, 3], [3, 2, 1, 1, 2], x, y, 1.0, 0.0), ref)
    # Diag with alpha/beta :15-25
    x = rng.standard_normal((3, 3, 3, 3, 3))
    y0 = rng.standard_normal((3, 3, 3))
    ref = O.loop_einsum([(3, 2, 1, 1, 2)], (1, 2, 3), [x], sd)
    for sx, sy in [(1.0, 0.0), (2.0, 0.0), (1.0, 2.0), (2.0, 3.0)]:
        got = O.unary_diag_([3, 2, 1, 1, 2], [1, 2, 3], x, y0.copy(order="F"), sx, sy)
        assert close(got, sx * ref + sy * y0)
    # Repeat :27-34
    x = rng.standard_normal((3, 3, 3))
    y = np.zeros((3, 5, 3, 3), order="F")
    assert close(O.unary_repeat_([1, 2, 3], [3, 4, 2, 1], x, y, 1.0, 0.0),
                 O.loop_einsum([(1, 2, 3)], (3, 4, 2, 1), [x], sd))
    # Tr :36-41
    a = rng.random((5, 5))
    assert np.isclose(O.unary_tr_([1, 1], [], a, np.zeros(()), 1.0, 0.0)[()], np.trace(a))
    # Permutedims :43-46
    a = rng.random((5, 5, 3))
    assert np.array_equal(O.unary_permutedims_([1, 2, 3], [2, 3, 1], a, np.zeros((5, 3, 5), order="F"), 1.0, 0.0),
                          np.transpose(a, (1, 2, 0)))
    # Identity :48-51
    a = rng.random((5, 5, 3))
    assert close(O.unary_identity_([1, 2, 3], [1, 2, 3], a, np.ones((5, 5, 3), order="F"), 2.0, 3.0), 3 + 2 * a)
    # Sum :53-58 (exact integers)
    a = rng.integers(1, 100, (2, 2, 5))
    assert np.array_equal(O.unary_sum_([1, 2, 3], [1, 2], a, np.zeros((2, 2), dtype=np.int64), 1, 0), a.sum(axis=2))


# --- test/einsum.jl -----------------------------------------------------------


def test_einsum_unary_binary_nary_alpha_beta():
    # test/einsum.jl:27-77
    sd = {1: 3, 2: 3, 3: 3, 4: 4, 5: 5}
    x = rng.standard_normal((3, 3, 3, 3, 4))
    y = np.asarray(rng.standard_normal((3, 5, 3, 3, 3, 5)), order="F")
    ix, iy = (1, 2, 3, 3, 4), (3, 5, 1, 1, 2, 5)
    assert close(O.einsum_([ix], iy, [x], y.copy(order="F"), 1.0, 0.0, sd), O.loop_einsum([ix], iy, [x], sd))
    for ix2, iy2, shp in [((1, 2, 3, 4), (4, 3, 1, 2), (3, 3, 3, 4)), ((1, 2, 3, 4), (1, 2, 3, 4), (3, 3, 3, 4))]:
        xx = rng.standard_normal(shp)
        yy = np.zeros([sd[l] for l in iy2], order="F")
        assert close(O.einsum_([ix2], iy2, [xx], yy, 1.0, 0.0, sd), O.loop_einsum([ix2], iy2, [xx], sd))
    xx = rng.standard_normal((3, 3))
    assert np.isclose(O.einsum_([(1, 1)], (), [xx], np.ones(()), 1.0, 0.0, sd)[()], np.trace(xx))
    # binary with alpha beta (:55-66)
    iz = (1, 2, 3, 4, 5, 5)
    z = np.asarray(rng.standard_normal((3, 3, 3, 4, 5, 5)), order="F")
    for sx, sy in [(1.0, 0.0), (5.0, 3.0), (5.0, 1.0)]:
        a = O.einsum_([ix, iy], iz, [x, y], z.copy(order="F"), sx, sy, sd)
        b = O.loop_einsum_([ix, iy], iz, [x, y], z.copy(order="F"), sx, sy, sd)
        assert close(a, b)
    # n-ary (:68-77)
    y3 = rng.standard_normal((3, 5, 3))
    a = O.einsum_([ix, (3, 5, 1), iz], (), [x, y3, z], np.ones(()), 1.0, 0.0, sd)
    assert close(a, O.loop_einsum([ix, (3, 5, 1), iz], (), [x, y3, z], sd))


def test_einsum_assorted():
    # test/einsum.jl:103-212
    a, b, c = rng.standard_normal((2, 2)), rng.random((2, 2)), rng.random((2, 2))
    v = rng.random(2)
    t = rng.standard_normal((2, 2, 2, 2))
    e = lambda s, *xs, **kw: O.einsum(*_code(s), list(xs), kw.get("sd"))
    assert close(e("ijkl->ijkl", t), t)
    assert close(O.einsum([(1, 2), (2, 3), (3, 4)], (1, 4), [a, b, c]), a @ b @ c)
    assert close(O.einsum([(1, 2), (2, 3), (3, 4)], (4, 1), [a, b, c]), (a @ b @ c).T)
    assert close(O.einsum([(1, 2), (2,)], (1,), [a, v]), a @ v)
    for s, f in [("ij,jk->ik", a @ a), ("ij,jk->ki", (a @ a).T), ("ij,kj->ik", a @ a.T), ("ij,kj->ki", (a @ a.T).T),
                 ("ji,jk->ik", a.T @ a), ("ji,jk->ki", (a.T @ a).T), ("ji,kj->ik", a.T @ a.T),
                 ("ji,kj->ki", (a.T @ a.T).T)]:
        assert close(e(s, a, a), f)
    assert np.isclose(O.einsum([(1, 2), (1, 2)], (), [a, a])[()], np.sum(a * a))
    assert np.isclose(O.einsum([(1, 1)], (), [a])[()], np.trace(a))
    aa = rng.random((2, 4, 4, 2))
    assert np.isclose(O.einsum([(1, 2, 2, 1)], (), [aa])[()], sum(aa[i, j, j, i] for i in range(2) for j in range(4)))
    ptr = sum(aa[:, i, i, :] for i in range(4))
    assert close(O.einsum([(1, 2, 2, 3)], (1, 3), [aa]), ptr)
    assert close(O.einsum([(1, 2, 2, 3)], (3, 1), [aa]), ptr.T)
    assert close(O.einsum([(1, 2, 2, 3)], (1, 2, 3), [aa]), np.stack([aa[:, i, i, :] for i in range(4)], axis=1))
    assert close(O.einsum([(1, 2)], (2, 1), [a]), a.T)
    assert close(O.einsum([(1, 2, 3, 4)], (2, 3, 1, 4), [t]), np.transpose(t, (1, 2, 0, 3)))
    ta = np.einsum("ijkl,jk->il", t, a)
    assert close(O.einsum([(1, 2, 3, 4), (2, 3)], (1, 4), [t, a]), ta)
    ta = np.einsum("lkji,jk->il", t, a)
    assert close(O.einsum([(4, 3, 2, 1), (2, 3)], (1, 4), [t, a]), ta)
    assert close(O.einsum([(1, 2), (1, 3), (1, 4)], (2, 3, 4), [a, a, a]), np.einsum("ij,ik,il->jkl", a, a, a))
    assert close(O.einsum([(1, 2), (1, 2), (1, 3)], (3,), [a, a, a]), np.einsum("ij,ij,il->l", a, a, a))
    a3 = rng.random((2, 2, 5))
    assert close(O.einsum([(1, 2, 3)], (1, 2), [a3]), a3.sum(axis=2))
    assert close(e("ijk->ki", a3), a3.sum(axis=1).T)
    assert np.isclose(e("ijk->", a3)[()], a3.sum())
    h1, h2 = rng.random((2, 3)), rng.random((2, 3))
    assert close(O.einsum([(1, 2), (1, 2)], (1, 2), [h1, h2]), h1 * h2)
    assert close(O.einsum([(1, 2), (3, 4)], (1, 2, 3, 4), [h1, h2]), np.einsum("ij,kl->ijkl", h1, h2))
    # broadcasting / identity: ein"->ii"(asarray(1); size_info=Dict('i'=>5)) == I(5)
    got = O.einsum([()], ("i", "i"), [np.array(1)], {"i": 5})
    assert np.array_equal(got, np.eye(5, dtype=np.int64))
    # ein",->"(asarray(3), asarray(4))[] === 12
    r = O.einsum([(), ()], (), [np.array(3), np.array(4)])
    assert r.dtype == np.int64 and r[()] == 12
    # projecting to diag
    a = rng.random((2, 2))
    assert close(O.einsum([(1, 1)], (1, 1), [a]), np.diag(np.diag(a)))
    a4 = rng.random((2, 2, 2, 2))
    assert np.isclose(O.einsum([(1, 1, 2, 2)], (), [a4])[()], sum(a4[i, i, j, j] for i in range(2) for j in range(2)))
    assert close(O.einsum([(1, 2, 3, 4), (3, 4, 5, 6)], (1, 2, 5, 6), [a4, a4]),
                 (a4.reshape(4, 4, order="F") @ a4.reshape(4, 4, order="F")).reshape(2, 2, 2, 2, order="F"))


def _code(s):
    lhs, iy = s.replace(" ", "").split("->")
    return [tuple(ix) for ix in lhs.split(",")], tuple(iy)


def test_size_dict_errors():
    # test/einsum.jl:86-101, 231-235, 289-294
    a = rng.standard_normal((3, 3))
    with pytest.raises(ValueError):
        O.get_size_dict([(1, 2), (2, 3)], [a, a, a])
    with pytest.raises(ValueError):
        O.get_size_dict([(1, 2), (2, 3)], [rng.random((3, 3, 3))] * 2)
    b = rng.standard_normal((3, 2))
    sd = O.get_size_dict([(1, 2), (2, 3)], [b, b.T])
    assert (sd[1], sd[2], sd[3]) == (3, 2, 3)
    with pytest.raises(O.DimensionMismatch):
        O.get_size_dict([("i", "j"), ("j", "k")], [b, b])
    with pytest.raises(O.DimensionMismatch):
        O.get_size_dict([(1, 2), (2, 3)], [rng.random((3, 3)), rng.random((4, 4))])


def test_issue_136_and_cc_rules():
    # test/einsum.jl:306-319
    got = O.einsum([(1, 2, 3), (2,)], (1, 3), [np.ones((2, 2, 1)), np.ones(2)])
    assert np.array_equal(got, np.array([[2.0], [2.0]]))
    got = O.einsum([(1, 2, 3), (2,)], (1, 3), [np.ones((2, 2, 0)), np.ones(2)])
    assert got.shape == (2, 0)
    sd = {"a": 2, "b": 2, "c": 2}
    for s in ["c,c->cc", "c,cc->c", "cc,c->cc", "cc,cc->cc", "cc,cb->bc", "cb,bc->cc", "ac,cc->ac"]:
        ixs, iy = _code(s)
        xs = [rng.standard_normal([2] * len(ix)) for ix in ixs]
        assert close(O.einsum(ixs, iy, xs, sd), O.loop_einsum(ixs, iy, xs, sd))


def test_symbolic_duplicate_exact():
    # test/einsum.jl:343-345 (ij->ijij places x on the (i,j,i,j) diagonal)
    x = np.array([[1, 2], [3, 4]], dtype=np.int64)
    got = O.einsum([("i", "j")], ("i", "j", "i", "j"), [x])
    want = np.zeros((2, 2, 2, 2), dtype=np.int64)
    for i, j in itertools.product(range(2), range(2)):
        want[i, j, i, j] = x[i, j]
    assert np.array_equal(got, want)


# --- test/einsequence.jl, test/slicing.jl -------------------------------------


def test_nested_parse_and_eval():
    e1 = O.parse_nested("((i,ij),i),j->i")
    assert O.getixsv(e1) == [["i"], ["i", "j"], ["i"], ["j"]]
    assert e1.args[1].isleaf and e1.args[1].tensorindex == 3      # 4 in 1-based Julia
    a, b, c = rng.random((2, 2)), rng.random((2, 2)), rng.random((2, 2))
    ne = O.parse_nested("(ij,jk),km->im")
    sd = {l: 2 for l in "ijkm"}
    assert close(O.nested_einsum(ne, [a, b, c], sd), a @ b @ c)
    a, b, c, d = rng.standard_normal(2), rng.standard_normal((2, 2)), rng.standard_normal(2), rng.standard_normal(2)
    ne = O.parse_nested("((i,ij),i),j->ik")
    sd = {"i": 2, "j": 2, "k": 2}
    flat = O.einsum([("i",), ("i", "j"), ("i",), ("j",)], ("i", "k"), [a, b, c, d], sd)
    assert close(O.nested_einsum(ne, [a, b, c, d], sd), flat)


def test_complexity_kat():
    # test/einsequence.jl:198-206
    ne = O.parse_nested("(ij,jkc),klc->il")
    sd = {l: 10 for l in "ijklc"}
    tc, sc, rw = O.contraction_complexity(ne, sd)
    assert math.isclose(tc, math.log2(20000)) and math.isclose(sc, math.log2(1000))
    assert math.isclose(rw, math.log2(100 + 1000 + 1000 + 1000 + 1000 + 100))
    assert O.peak_memory(ne, sd) == 2100
    # the package's planner gives the same numbers
    pne = ome.ein("(ij,jkc),klc->il")
    c = ome.contraction_complexity(pne, sd)
    assert math.isclose(c.tc, math.log2(20000)) and math.isclose(c.sc, math.log2(1000))
    assert math.isclose(c.rwc, math.log2(4200))
    assert ome.peak_memory(pne, sd) == 2100


def test_sliced_equals_unsliced():
    # test/slicing.jl:1-33
    ne = O.parse_nested("(ij,jk),(kl,lm)->im")
    sd = {"i": 2, "j": 3, "k": 4, "l": 5, "m": 6}
    assert len(list(O.slice_iterator(["i", "l"], {l: 2 for l in "ijklm"}))) == 4
    for _ in range(5):
        xs = [rng.standard_normal((2, 3)), rng.standard_normal((3, 4)), rng.standard_normal((4, 5)),
              rng.standard_normal((5, 6))]
        assert close(O.sliced_einsum(["i", "l"], ne, xs, sd), O.nested_einsum(ne, xs, sd))
    se = ome.SlicedEinsum(["i", "l"], ome.ein("(ij,jk),(kl,lm)->im"))
    assert ome.label_elimination_order(se) == ["j", "l", "k"]


# --- test/contractionorder.jl, docs/src/applications.md ------------------------


def fullerene():
    # coordinates generated as in test/contractionorder.jl:32-46
    phi = (1 + math.sqrt(5)) / 2
    res = []
    for (x, y, z) in ((0.0, 1.0, 3 * phi), (1.0, 2 + phi, 2 * phi), (phi, 2.0, 2 * phi + 1.0)):
        for (al, be, ga) in ((x, y, z), (y, z, x), (z, x, y)):
            for loc in ((al, be, ga), (al, be, -ga), (al, -be, ga), (al, -be, -ga), (-al, be, ga), (-al, be, -ga),
                        (-al, -be, ga), (-al, -be, -ga)):
                if loc not in res:
                    res.append(loc)
    return res


def c60_code():
    xy = fullerene()
    edges = [(i + 1, j + 1) for j in range(60) for i in range(60)
             if i < j and sum((xy[i][k] - xy[j][k]) ** 2 for k in range(3)) < 5.0]
    return edges, [(i,) for i in range(1, 61)]


def to_oracle_tree(ne):
    if ne.isleaf:
        return O.leaf(ne.tensorindex)
    return O.Node(args=[to_oracle_tree(a) for a in ne.args], ixs=[list(ix) for ix in ne.eins.ixs],
                  iy=list(ne.eins.iy))


def test_fullerene_tropical_66():
    # test/contractionorder.jl:31-70: the C60 spin-glass ground state is 66,
    # unsliced and sliced with sc_target = 8
    edges, verts = c60_code()
    assert len(edges) == 90
    code = ome.EinCode(edges + verts, ())
    sd = {i: 2 for i in range(1, 61)}
    assert ome.contraction_complexity(code, sd).tc == 60
    opt = ome.optimize_code(code, sd, ome.GreedyMethod(nrepeat=3, seed=2))
    assert opt.flatten() == code
    xs = [np.array([[-1.0, 1.0], [1.0, -1.0]])] * 90 + [np.array([0.0, 0.0])] * 60
    r = O.nested_einsum(to_oracle_tree(opt), xs, sd, O.TROPICAL)
    assert r[()] == 66
    sc = ome.slice_code(opt, sd, ome.GreedySlicer(sc_target=8))
    assert ome.contraction_complexity(sc, sd).sc <= 8
    r2 = O.sliced_einsum(sc.slicing, to_oracle_tree(sc.eins), xs, sd, O.TROPICAL)
    assert r2[()] == 66


def colouring_tensor():
    s = np.zeros((3, 3, 3), dtype=np.int64)
    for i, j, k in itertools.product(range(3), repeat=3):
        s[i, j, k] = int(len({i, j, k}) == 3)
    return s


def test_three_colouring():
    # docs/src/applications.md:20-33: two vertices -> 6, Petersen graph -> 0
    s = colouring_tensor()
    assert O.einsum([tuple("ijk"), tuple("ijk")], (), [s, s])[()] == 6
    code = ome.ein("afl,bhn,cjf,dlh,enj,ago,big,cki,dmk,eom->")
    sd = ome.uniformsize(code, 3)
    opt = ome.optimize_code(code, sd, ome.GreedyMethod(nrepeat=2))
    assert O.nested_einsum(to_oracle_tree(opt), [s] * 10, sd)[()] == 0


# --- autodiff (test/bp.jl, test/autodiff.jl) ------------------------------------


def test_cost_and_gradient_finite_difference():
    A, B, Cm = rng.standard_normal((2, 3)), rng.standard_normal((3, 4)), rng.standard_normal((4, 2))
    ne = O.parse_nested("(ij,jk),ki->")
    cost, grads = O.cost_and_gradient(ne, [A, B, Cm])
    assert np.isclose(cost[()], np.einsum("ij,jk,ki->", A, B, Cm))
    eps = 1e-6
    for t, g in zip([A, B, Cm], grads):
        for idx in itertools.product(*[range(s) for s in t.shape]):
            old = t[idx]
            t[idx] = old + eps
            fp = np.einsum("ij,jk,ki->", A, B, Cm)
            t[idx] = old - eps
            fm = np.einsum("ij,jk,ki->", A, B, Cm)
            t[idx] = old
            assert abs((fp - fm) / (2 * eps) - g[idx]) < 1e-6


def test_bool_and_int_semantics():
    x = rng.integers(0, 2, (3, 4)).astype(bool)
    y = rng.integers(0, 2, (4, 5)).astype(bool)
    got = O.einsum([("i", "j"), ("j", "k")], ("i", "k"), [x, y])
    assert got.dtype == np.bool_ and np.array_equal(got, (x.astype(int) @ y.astype(int)) > 0)
    big = np.array([2 ** 62, 2 ** 62], dtype=np.int64)
    r = O.einsum([("i",), ("i",)], (), [big, np.array([2, 2], dtype=np.int64)])
    assert r[()] == np.int64(0)  # 2^64 wraps to 0 like Julia Int64


def test_int64_matmul_exact_path_equals_integer_loop():
    """The oracle's Int64 GEMM (FP64 BLAS when every partial sum is an integer
    below 2^53) gives the same integers as NumPy's Int64 matmul, and large
    values still wrap like Julia's Int64."""
    rng = np.random.default_rng(1)
    a = rng.integers(-8, 9, (3, 40, 70), dtype=np.int64)
    b = rng.integers(-8, 9, (3, 70, 30), dtype=np.int64)
    got = O.REAL.matmul(a, b)
    assert got.dtype == np.int64 and np.array_equal(got, np.matmul(a, b))
    big = np.full((2, 2), 2 ** 62, dtype=np.int64)
    with np.errstate(over="ignore"):
        assert np.array_equal(O.REAL.matmul(big, big), np.matmul(big, big))
