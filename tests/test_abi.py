"""The C-ABI library loads here (no GPU) and exports every entry point that
include/*.h declares; host-side logic of the package that needs no device."""
import glob
import os
import re

import pytest
import torch

import omeinsum_b200 as ome
from omeinsum_b200 import _lib

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_symbols():
    names = set()
    for h in glob.glob(os.path.join(ROOT, "include", "*.h")):
        src = open(h).read()
        names |= set(re.findall(r"OME_API\s+[\w\s\*]+?\b(ome_\w+)\s*\(", src))
    return sorted(names)


def test_library_exports_every_declared_symbol():
    names = declared_symbols()
    assert len(names) >= 12
    lib = _lib.load()
    for n in names:
        assert hasattr(lib, n), n
    assert set(_lib.EXPORTS) <= set(names)
    assert lib.ome_version() == 1


def test_no_device_is_an_error_not_a_crash():
    if torch.cuda.is_available():
        pytest.skip("a device is present")
    import ctypes as C
    h = C.c_void_p()
    rc = _lib.load().ome_ctx_create(0, 0, C.byref(h))
    assert rc == _lib.CUDA_ERROR
    assert _lib.load().ome_last_error()


def test_backend_registry():
    assert isinstance(ome.get_einsum_backend(), ome.B200Backend)
    ome.set_einsum_backend(ome.DefaultBackend())
    assert isinstance(ome.get_einsum_backend(), ome.DefaultBackend)
    with pytest.raises(ome.OMEError):
        ome.einsum(ome.ein("ij,jk->ik"), (torch.zeros(2, 2), torch.zeros(2, 2)))
    ome.set_einsum_backend(ome.B200Backend())


def test_codes_and_parsing():
    c = ome.ein("ij,jk->ik")
    assert c.getixsv() == [["i", "j"], ["j", "k"]] and c.getiyv() == ["i", "k"]
    assert c == ome.EinCode([("i", "j"), ("j", "k")], ("i", "k"))
    with pytest.raises(RuntimeError):
        ome.EinCode([], ())
    e1 = ome.ein("((i,ij),i),j->i")
    assert e1.getixsv() == [["i"], ["i", "j"], ["i"], ["j"]]
    assert e1.args[1].isleaf and e1.args[1].tensorindex == 3
    assert e1.rootcode() == ome.ein("ij,j->i")
    ne = ome.ein("(ij,j),k->")
    assert ne.flatten() == ome.ein("ij,j,k->")
    with pytest.raises(ome.ArgumentError):
        ome.parse_nested("((ij,jk),km", [])
    ne = ome.ein("(ij, jk), kl->il")
    assert ne.replace(("i", "a"), ("j", "b"), ("k", "c"), ("l", "d")) == ome.ein("(ab, bc), cd->ad")


def test_size_dict_contract():
    a = torch.zeros(3, 3)
    with pytest.raises(ome.ArgumentError):
        ome.get_size_dict([(1, 2), (2, 3)], (a, a, a))
    with pytest.raises(ome.ArgumentError):
        ome.get_size_dict([(1, 2), (2, 3)], (torch.zeros(3, 3, 3),) * 2)
    with pytest.raises(ome.DimensionMismatch):
        ome.get_size_dict([("i", "j"), ("j", "k")], (torch.zeros(3, 2), torch.zeros(3, 2)))


def test_promotion_follows_julia():
    assert ome.promote_dtype([torch.int64, torch.float32]) == torch.float32
    assert ome.promote_dtype([torch.float32, torch.complex64]) == torch.complex64
    assert ome.promote_dtype([torch.float64, torch.complex64]) == torch.complex128
    assert ome.promote_dtype([torch.bool, torch.int64]) == torch.int64


def test_planner_and_json(tmp_path):
    code = ome.EinCode([["a", "b"], ["b", "c"], ["c", "d"]], ["a", "d"])
    g = ome.optimize_code(code, ome.uniformsize(code, 2), ome.GreedyMethod())
    assert isinstance(g, ome.NestedEinsum) and g.flatten() == code
    s = ome.optimize_code(code, ome.uniformsize(code, 2), ome.GreedyMethod(), slicer=ome.GreedySlicer(sc_target=1))
    assert isinstance(s, ome.SlicedEinsum)
    for c in (g, s):
        f = str(tmp_path / "tree.json")
        ome.writejson(f, c)
        assert ome.readjson(f) == c
    # flop of a unary sum (test/contractionorder.jl:17)
    assert ome.flop(ome.ein("i->"), {"i": 4}) == 4


def test_greedy_bounds_kat():
    # test/contractionorder.jl:5-19: greedy tc within the reference bounds
    import math
    sd = {c: 1 << (i + 1) for i, c in enumerate("abcdef")}
    opt = ome.optimize_code(ome.ein("ab,acd,bcef,e,df->"), sd, ome.GreedyMethod())
    tc, sc, _ = ome.contraction_complexity(opt, sd)
    assert math.isclose(tc, math.log2(ome.flop(opt, sd)))
    assert 16 <= tc <= math.log2(2 ** 10 + 2 ** 16 + 2 ** 15 + 2 ** 9 + 1e-8)
    assert sc == 11


def test_json_layout_interchange(tmp_path):
    """writejson/readjson use OMEinsumContractionOrders' layout (1-based leaf
    indices, "label-type", "inputs", "output", "tree", "slices"), so trees
    written by a Julia installation load here and the other way round."""
    import json
    # a tree as OMEinsumContractionOrders writes it for ein"(ij,jk),kl->il" sliced over j
    julia_file = tmp_path / "julia.json"
    julia_file.write_text(json.dumps({
        "label-type": "Char", "inputs": [["i", "j"], ["j", "k"], ["k", "l"]], "output": ["i", "l"],
        "slices": ["j"],
        "tree": {"isleaf": False, "eins": {"ixs": [["i", "k"], ["k", "l"]], "iy": ["i", "l"]},
                 "args": [{"isleaf": False, "eins": {"ixs": [["i", "j"], ["j", "k"]], "iy": ["i", "k"]},
                           "args": [{"isleaf": True, "tensorindex": 1}, {"isleaf": True, "tensorindex": 2}]},
                          {"isleaf": True, "tensorindex": 3}]}}))
    se = ome.readjson(str(julia_file))
    assert isinstance(se, ome.SlicedEinsum) and list(se.slicing) == ["j"]
    assert se.eins == ome.ein("(ij,jk),kl->il")
    # written files carry the same layout: 1-based leaves and the top-level keys
    out = tmp_path / "out.json"
    ome.writejson(str(out), se)
    obj = json.loads(out.read_text())
    assert obj["label-type"] == "Char" and obj["slices"] == ["j"] and obj["output"] == ["i", "l"]
    assert obj["inputs"] == [["i", "j"], ["j", "k"], ["k", "l"]]
    assert obj["tree"]["args"][1] == {"isleaf": True, "tensorindex": 3}
    assert ome.readjson(str(out)) == se
    # integer labels
    code = ome.EinCode([[1, 2], [2, 3], [3, 4]], [1, 4])
    g = ome.slice_code(ome.optimize_code(code, ome.uniformsize(code, 4), ome.GreedyMethod()),
                       ome.uniformsize(code, 4), ome.GreedySlicer(sc_target=2))
    f = tmp_path / "int.json"
    ome.writejson(str(f), g)
    assert json.loads(f.read_text())["label-type"] == "Int64"
    assert ome.readjson(str(f)) == g
    with pytest.raises(ome.ArgumentError):
        ome.writejson(str(f), ome.ein("(ab,bc),cd->ad").__class__([ome.NestedEinsum(0), ome.NestedEinsum(1)],
                                                                    ome.EinCode([("xx", "y"), ("y", "z")], ("xx", "z"))))
