"""pytest configuration: the `gpu` marker and loaders for the package and the oracle.

The package directory ``omeinsum.jl_b200`` is not a valid Python identifier,
so it is registered as the module ``omeinsum_b200``.  The oracle
(``oracle/ome_oracle.py``) is test infrastructure and is imported only here
and by the tests.
"""
import importlib.util
import os
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def load_package():
    if "omeinsum_b200" in sys.modules:
        return sys.modules["omeinsum_b200"]
    pkg = os.path.join(ROOT, "omeinsum.jl_b200")
    spec = importlib.util.spec_from_file_location("omeinsum_b200", os.path.join(pkg, "__init__.py"),
                                                  submodule_search_locations=[pkg])
    mod = importlib.util.module_from_spec(spec)
    sys.modules["omeinsum_b200"] = mod
    spec.loader.exec_module(mod)
    return mod


def load_oracle():
    d = os.path.join(ROOT, "oracle")
    if d not in sys.path:
        sys.path.insert(0, d)
    import ome_oracle
    return ome_oracle


load_package()
load_oracle()


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200) and the built libomeb200.so")
