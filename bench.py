#!/usr/bin/env python
"""Benchmark: the binary + unary rule suite (FP32) on B200.

One step = the six contractions of the rule-suite workload, each on resident
inputs with the L2 flushed (a 256 MiB write) before it:

  abcd,cdef->abef  all extents 48            (GEMM 2304^3)
  ijk,jkl->il      all extents 256           (GEMM 256 x 65536 x 256)
  bij,bjk->bik     b=512, i=j=k=64           (batch-innermost batched GEMM)
  abcde->ecadb     (32,32,32,32,128), 2^27   (Permutedims)
  ii->             16384^2                   (Tr)
  ijk->j           1024 x 1024 x 64          (Sum)

Inputs: normal(0,1) FP32, seeds 1..6.  metric = contractions/s (whole job,
all ranks); e2e = the same through the public einsum API with pinned host
inputs (host->device copy and device->host read of every result inside the
timed region).  `--impl reference` times the CPU oracle (a NumPy restatement
of OMEinsum.jl's DefaultBackend) on the same workload.

Run: python bench.py [--gpus N] [--steps K] [--warmup W] [--impl b200|reference]
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

CASES = [
    # name, code, extents, seed
    ("abcd,cdef->abef", "abcd,cdef->abef", dict(a=48, b=48, c=48, d=48, e=48, f=48), 1),
    ("ijk,jkl->il", "ijk,jkl->il", dict(i=256, j=256, k=256, l=256), 2),
    ("bij,bjk->bik", "bij,bjk->bik", dict(b=512, i=64, j=64, k=64), 3),
    ("abcde->ecadb", "abcde->ecadb", dict(a=32, b=32, c=32, d=32, e=128), 4),
    ("ii->", "ii->", dict(i=16384), 5),
    ("ijk->j", "ijk->j", dict(i=1024, j=1024, k=64), 6),
]
WORKLOAD = ("binary+unary rule suite FP32: abcd,cdef->abef d=48; ijk,jkl->il d=256; "
            "bij,bjk->bik b=512 i=j=k=64; abcde->ecadb 2^27 (32,32,32,32,128); ii-> 16384^2; "
            "ijk->j 1024x1024x64")
METRIC = "rule-suite contractions/s (FP32)"


def parse_code(s):
    lhs, iy = s.split("->")
    return [tuple(ix) for ix in lhs.split(",")], tuple(iy)


def case_work(code, ext):
    """(algorithmic flops, algorithmic bytes) of one contraction (FP32)."""
    ixs, iy = parse_code(code)
    labels = sorted(set(l for ix in ixs for l in ix) | set(iy))
    nin = sum(int(np.prod([ext[l] for l in ix])) for ix in ixs)
    if code == "ii->":
        nin = ext["i"]  # only the diagonal is algorithmically needed
    nout = int(np.prod([ext[l] for l in iy])) if iy else 1
    flops = 2 * int(np.prod([ext[l] for l in labels], dtype=np.float64)) if len(ixs) == 2 else 0
    return flops, 4 * (nin + nout)


def make_inputs(code, ext, seed):
    rng = np.random.default_rng(seed)
    ixs, _ = parse_code(code)
    return [np.asfortranarray(rng.standard_normal([ext[l] for l in ix]).astype(np.float32)) for ix in ixs]


def load_peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        d = json.load(open(p))
        return d["hbm_gbs"], d["bf16_tflops"], "measured"
    return 6650.0, 1590.0, "fallback"


def load_traffic():
    """Per-launch DRAM bytes of each suite kernel from an ncu capture (profiles/)."""
    p = os.path.join(ROOT, "profiles", "suite_traffic.json")
    if os.path.exists(p):
        return json.load(open(p))
    return {}


class ClockSampler:
    """nvidia-smi clocks/throttle sampling during the timed region."""

    def __init__(self, index):
        self.index = index
        self.proc = None
        self.path = None

    def __enter__(self):
        try:
            fd, self.path = tempfile.mkstemp(suffix=".csv")
            os.close(fd)
            q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
                 "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
                 "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
            self.proc = subprocess.Popen(["nvidia-smi", f"--id={self.index}", f"--query-gpu={q}",
                                          "--format=csv,noheader,nounits", "-lms", "100"],
                                         stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None
        return self

    def __exit__(self, *a):
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()

    def summary(self):
        if not self.path or not os.path.exists(self.path):
            return None
        sm, mx, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in open(self.path):
            f = [x.strip() for x in line.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                mx.append(float(f[2]))
            except ValueError:
                continue
            for n, v in zip(names, f[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(n)
        if not sm:
            return None
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": max(mx), "reasons": sorted(reasons),
                "samples": len(sm)}


def cpu_suite(O, inputs, steps=1):
    """Oracle (NumPy DefaultBackend restatement) on the suite; returns seconds per pass."""
    t0 = time.perf_counter()
    for _ in range(steps):
        for (name, code, ext, seed), xs in zip(CASES, inputs):
            ixs, iy = parse_code(code)
            O.einsum(ixs, iy, xs, ext)
    return (time.perf_counter() - t0) / steps


def run_reference(args, rank):
    if rank != 0:
        return
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import ome_oracle as O
    inputs = [make_inputs(code, ext, seed) for _, code, ext, seed in CASES]
    for _ in range(args.warmup):
        cpu_suite(O, inputs)
    t = cpu_suite(O, inputs, args.steps)
    v = len(CASES) / t
    cores = os.cpu_count()
    line = {"metric": METRIC, "value": v, "unit": "contractions/s", "n_gpus": args.gpus, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": t * 1e3, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded normal(0,1))",
            "config": {"workload": WORKLOAD}, "impl": "reference",
            "cpu_baseline": {"value": v, "unit": "contractions/s", "cores": cores, "kind": "port",
                             "sample": f"the full suite, {args.steps} passes, NumPy/OpenBLAS DefaultBackend "
                                       f"restatement (OPENBLAS threads = {cores}; copies single-threaded)"},
            "e2e": {"value": v, "unit": "contractions/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--prec", type=int, default=0, help="0 AUTO (BF16x3), 1 plain FP32")
    ap.add_argument("--no-cpu", action="store_true", help="skip the cpu_baseline leg")
    args = ap.parse_args()

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if args.impl == "reference":
        return run_reference(args, rank)

    import torch
    import torch.distributed as dist
    from __graft_entry__ import load_package

    ome = load_package()
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    if world > 1:
        import datetime
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    ome.set_einsum_backend(ome.B200Backend(prec=args.prec))
    lib = ome.load_library()

    hosts, devs, outs, codes = [], [], [], []
    for name, code, ext, seed in CASES:
        xs = make_inputs(code, ext, seed)
        hosts.append([torch.from_numpy(x).pin_memory() for x in xs])
        devs.append([h.to(dev) for h in hosts[-1]])
        ixs, iy = parse_code(code)
        c = ome.EinCode(ixs, iy)
        codes.append((c, ext))
        outs.append(ome.get_output_array(devs[-1], [ext[l] for l in iy]))
    flush = torch.empty(256 << 20, dtype=torch.uint8, device=dev)
    ev = [[(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in CASES]
          for _ in range(args.steps)]

    def step(k=None):
        for i, (c, ext) in enumerate(codes):
            flush.fill_(i)
            if k is not None:
                ev[k][i][0].record()
            ome.einsum_(c, devs[i], outs[i], True, False, ext)
            if k is not None:
                ev[k][i][1].record()

    for _ in range(max(args.warmup, 3)):
        step()
    torch.cuda.synchronize()
    if world > 1:
        dist.barrier()
    n0 = lib.ome_launch_count()
    with ClockSampler(local) as cs:
        torch.cuda.synchronize()
        for k in range(args.steps):
            step(k)
        torch.cuda.synchronize()
    launches = lib.ome_launch_count() - n0
    if world > 1:
        dist.barrier()
    per_case = [sum(ev[k][i][0].elapsed_time(ev[k][i][1]) for k in range(args.steps)) / args.steps
                for i in range(len(CASES))]  # ms
    step_ms = sum(per_case)
    t = torch.tensor([step_ms], dtype=torch.float64, device=dev)
    if world > 1:
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
    step_ms_max = float(t.item())
    value = len(CASES) * world / (step_ms_max / 1e3)

    # end to end through the public API with pinned host inputs
    e2e_ev = []
    h2d = sum(h.numel() * h.element_size() for hs in hosts for h in hs)
    d2h = sum(o.numel() * o.element_size() for o in outs)
    for _ in range(2):
        for i, (c, ext) in enumerate(codes):
            ome.einsum(c, hosts[i], ext)
    torch.cuda.synchronize()
    s0, s1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    s0.record()
    for k in range(args.steps):
        for i, (c, ext) in enumerate(codes):
            r = ome.einsum(c, hosts[i], ext)  # H2D of inputs, contraction, D2H of the result
    s1.record()
    torch.cuda.synchronize()
    e2e_ms = s0.elapsed_time(s1) / args.steps
    te = torch.tensor([e2e_ms], dtype=torch.float64, device=dev)
    if world > 1:
        dist.all_reduce(te, op=dist.ReduceOp.MAX)
    e2e_value = len(CASES) * world / (float(te.item()) / 1e3)

    # roofline of the dominant contraction
    hbm, bf16, src = load_peaks()
    dom = int(np.argmax(per_case))
    name, code, ext, _ = CASES[dom]
    flops, nbytes = case_work(code, ext)
    dur_s = per_case[dom] / 1e3
    tc_peak = bf16 / 3.0  # BF16x3: three BF16 products per FP32 product
    t_flop = flops / (tc_peak * 1e12) if flops else 0.0
    t_mem = nbytes / (hbm * 1e9)
    traffic = load_traffic().get(name)
    if t_flop > t_mem:
        roof = {"bound": "tensor", "achieved": flops / dur_s / 1e12, "peak": tc_peak, "unit": "TFLOP/s",
                "frac": (flops / dur_s / 1e12) / tc_peak, "traffic": traffic,
                "kernel": name, "peak_source": f"{src} bf16_tflops / 3 (FP32-equivalent BF16x3)"}
    else:
        roof = {"bound": "hbm", "achieved": nbytes / dur_s / 1e9, "peak": hbm, "unit": "GB/s",
                "frac": (nbytes / dur_s / 1e9) / hbm, "traffic": traffic, "kernel": name,
                "peak_source": f"{src} hbm_gbs"}

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu:
        sys.path.insert(0, os.path.join(ROOT, "oracle"))
        import ome_oracle as O
        inputs = [[h.numpy() for h in hs] for hs in hosts]
        tc = cpu_suite(O, inputs, 1)
        cpu = {"value": len(CASES) / tc, "unit": "contractions/s", "cores": os.cpu_count(), "kind": "port",
               "sample": "the full suite once, NumPy/OpenBLAS DefaultBackend restatement "
                         f"(BLAS threads = {os.cpu_count()}; copies single-threaded)"}

    detail = {}
    for (nm, code, ext, _), ms in zip(CASES, per_case):
        f, b = case_work(code, ext)
        detail[nm] = {"us": ms * 1e3, "GB/s": b / (ms / 1e3) / 1e9}
        if f:
            detail[nm]["TFLOP/s"] = f / (ms / 1e3) / 1e12
    if rank == 0:
        line = {"metric": METRIC, "value": value, "unit": "contractions/s", "n_gpus": world, "steps": args.steps,
                "warmup": max(args.warmup, 3), "ms_per_step": step_ms_max, "higher_is_better": True,
                "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded normal(0,1))",
                "config": {"workload": WORKLOAD, "l2": "flushed by a 256 MiB write before every contraction",
                           "prec": "BF16x3 where GEMM-shaped" if args.prec == 0 else "plain FP32",
                           "parallelism": f"replicas x{world}", "per_case": detail},
                "e2e": {"value": e2e_value, "unit": "contractions/s", "h2d_bytes_per_step": h2d,
                        "d2h_bytes_per_step": d2h},
                "gpu_launches": int(launches), "roofline": roof, "cpu_baseline": cpu,
                "clocks": cs.summary()}
        print(json.dumps(line), flush=True)
    if world > 1:
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
