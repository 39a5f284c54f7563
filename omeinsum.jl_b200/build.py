"""Build libomeb200.so (sm_100a) in-tree with nvcc.

Usage: python omeinsum.jl_b200/build.py [--force] [-j N]

Each csrc/*.cu is compiled to an object under omeinsum.jl_b200/_build/ and
linked into omeinsum.jl_b200/libomeb200.so.  Objects are rebuilt when their
source or any header is newer.
"""
from __future__ import annotations

import argparse
import concurrent.futures as cf
import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
BUILD = os.path.join(HERE, "_build")
LIB = os.path.join(HERE, "libomeb200.so")
INCLUDE = os.path.join(ROOT, "include")

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = ARCH + [
    "-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC", "-Xcompiler", "-fvisibility=hidden",
    "--expt-relaxed-constexpr", "-I", INCLUDE, "-I", CSRC,
]


def nvcc() -> str:
    p = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    if not os.path.exists(p):
        raise RuntimeError("nvcc not found")
    return p


def _headers_mtime() -> float:
    t = os.path.getmtime(os.path.join(INCLUDE, "ome_b200.h"))
    for f in os.listdir(CSRC):
        if f.endswith((".h", ".cuh")):
            t = max(t, os.path.getmtime(os.path.join(CSRC, f)))
    return t


def _compile(src: str, obj: str, extra: list[str]) -> str:
    cmd = [nvcc(), "-c", src, "-o", obj] + NVCC_FLAGS + extra
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"nvcc failed for {os.path.basename(src)}:\n{r.stderr}")
    return r.stderr


def build(force: bool = False, jobs: int = 8, verbose: bool = False, ptxas_v: bool = False) -> str:
    os.makedirs(BUILD, exist_ok=True)
    srcs = sorted(f for f in os.listdir(CSRC) if f.endswith(".cu"))
    hdr = _headers_mtime()
    todo = []
    objs = []
    for f in srcs:
        src = os.path.join(CSRC, f)
        obj = os.path.join(BUILD, f[:-3] + ".o")
        objs.append(obj)
        if force or not os.path.exists(obj) or os.path.getmtime(obj) < max(os.path.getmtime(src), hdr):
            todo.append((src, obj))
    extra = ["-Xptxas", "-v"] if ptxas_v else []
    with cf.ThreadPoolExecutor(max_workers=max(1, jobs)) as ex:
        futs = {ex.submit(_compile, s, o, extra): s for s, o in todo}
        for fu in cf.as_completed(futs):
            err = fu.result()
            if verbose and err:
                print(err, file=sys.stderr)
    if todo or force or not os.path.exists(LIB):
        cmd = [nvcc(), "-shared", "-o", LIB, "-cudart", "static"] + ARCH + objs
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"link failed:\n{r.stderr}")
    return LIB


if __name__ == "__main__":
    ap = argparse.ArgumentParser()
    ap.add_argument("--force", action="store_true")
    ap.add_argument("-j", type=int, default=8)
    ap.add_argument("-v", action="store_true", help="print ptxas resource usage")
    a = ap.parse_args()
    print(build(force=a.force, jobs=a.j, verbose=a.v, ptxas_v=a.v))
