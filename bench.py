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
all ranks); e2e = the same through the public einsum_many API with pinned
host inputs (host->device copy and device->host read of every result inside
the timed region; each result's download overlaps the next upload), with
the one-blocking-einsum-call-per-contraction figure beside it.  `--impl reference` times the CPU oracle (a NumPy restatement
of OMEinsum.jl's DefaultBackend) on the same workload.

Run: python bench.py [--gpus N] [--steps K] [--warmup W] [--impl b200|reference]
"""
from __future__ import annotations

import argparse
import json
import math
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


def make_inputs(code, ext, seed, dtype="f32"):
    """Column-major inputs of a suite contraction: normal(0,1) FP32, or
    uniform integers in [-8, 8] for Int64."""
    rng = np.random.default_rng(seed)
    ixs, _ = parse_code(code)
    if dtype == "i64":
        return [np.asfortranarray(rng.integers(-8, 9, [ext[l] for l in ix], dtype=np.int64)) for ix in ixs]
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
                "samples": len(sm), "window": "from 1 s of warm-up load through the timed steps"}


L2_POLICY = ("GPU arm: L2 flushed before every contraction (outside its events) by a 256 MiB write followed by "
             "a 256 MiB read, so that no dirty lines remain in L2; CPU arm: inputs of 21 MB to 2 GB per "
             "contraction, beyond the host caches")


def cpu_suite(O, inputs, steps=1, results=None):
    """Oracle (NumPy DefaultBackend restatement) on the suite; returns seconds
    per pass (and the last pass's results in `results` when given)."""
    t0 = time.perf_counter()
    for _ in range(steps):
        for (name, code, ext, seed), xs in zip(CASES, inputs):
            ixs, iy = parse_code(code)
            r = O.einsum(ixs, iy, xs, ext)
            if results is not None:
                results[name] = r
    return (time.perf_counter() - t0) / steps


def relerr(got, want):
    wide = np.complex128 if np.iscomplexobj(got) or np.iscomplexobj(want) else np.float64
    got = np.asarray(got, dtype=wide)
    want = np.asarray(want, dtype=wide)
    n = max(np.linalg.norm(got.ravel()), np.linalg.norm(want.ravel()))
    d = np.linalg.norm((got - want).ravel())
    return 0.0 if d == 0 else float(d / max(n, 1e-300))


def suite_parity(O, fp32_inputs, fp32_gpu, fp32_oracle, i64_inputs, i64_gpu):
    """The GPU results of the timed suite against the oracle (the checker):
    FP32 against the oracle in FP64 and in FP32 (rtol 1e-5 is the reference's
    GPU agreement tolerance), Int64 entry for entry."""
    out = {}
    for (name, code, ext, _), xs in zip(CASES, fp32_inputs):
        ixs, iy = parse_code(code)
        w64 = O.einsum(ixs, iy, [x.astype(np.float64) for x in xs], ext)
        out[name] = {"fp32_rel_err_vs_fp64_oracle": relerr(fp32_gpu[name], w64),
                     "fp32_rel_err_vs_fp32_oracle": relerr(fp32_gpu[name], fp32_oracle[name])}
    if i64_gpu:
        for (name, code, ext, _), xs in zip(CASES, i64_inputs):
            ixs, iy = parse_code(code)
            w = O.einsum(ixs, iy, xs, ext)
            g = i64_gpu[name]
            out[name]["int64_bit_exact"] = bool(g.dtype == w.dtype and g.shape == w.shape and np.array_equal(g, w))
    out["all_within_1e-5_and_int64_exact"] = all(
        v["fp32_rel_err_vs_fp64_oracle"] <= 1e-5 and v.get("int64_bit_exact", True)
        for k, v in out.items() if isinstance(v, dict))
    return out


def int64_section(ome, dev, steps, flush_l2, lib):
    """The rule suite in Int64 (uniform integers in [-8, 8], the same seeds):
    per contraction the event-timed device time with the L2 flushed before it,
    and the main kernel; results are returned for the exactness check."""
    import ctypes as C
    import torch
    per, kern, inputs, results = {}, {}, [], {}
    for i, (name, code, ext, seed) in enumerate(CASES):
        xs = make_inputs(code, ext, seed, "i64")
        inputs.append(xs)
        d = [torch.from_numpy(x).to(dev) for x in xs]
        ixs, iy = parse_code(code)
        c = ome.EinCode(ixs, iy)
        y = ome.get_output_array(d, [ext[l] for l in iy])
        for _ in range(2):
            ome.einsum_(c, d, y, True, False, ext)
        torch.cuda.synchronize()
        lib.ome_kernel_timing(8)
        ome.einsum_(c, d, y, True, False, ext)
        torch.cuda.synchronize()
        fb, nb, cnt = (C.c_float * 8)(), (C.c_char_p * 8)(), C.c_int32()
        lib.ome_kernel_times(8, fb, nb, C.byref(cnt))
        lib.ome_kernel_timing(0)
        kern[name] = "+".join(nb[j].decode() for j in range(cnt.value))
        ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(steps)]
        for k in range(steps):
            flush_l2(k)
            ev[k][0].record()
            ome.einsum_(c, d, y, True, False, ext)
            ev[k][1].record()
        torch.cuda.synchronize()
        ome.device_status()
        per[name] = sum(a.elapsed_time(b) for a, b in ev) / steps
        results[name] = y.cpu().numpy()
        del d, y
    step_ms = sum(per.values())
    detail = {}
    for name, code, ext, _ in CASES:
        f, b = case_work(code, ext)
        detail[name] = {"us": per[name] * 1e3, "main_kernel": kern[name], "GB/s": 2 * b / (per[name] / 1e3) / 1e9}
        if f:
            detail[name]["Gop/s"] = f / (per[name] / 1e3) / 1e9
    return {"workload": WORKLOAD.replace("FP32", "Int64") + "; uniform integers in [-8, 8]",
            "contractions_per_s": len(CASES) / (step_ms / 1e3), "ms_per_step": step_ms, "steps": steps,
            "per_case": detail}, inputs, results


def run_case_only(ome, name, dev):
    """Run one suite contraction twice (warm-up + the launch a profiler captures)."""
    import torch
    for nm, code, ext, seed in CASES:
        if nm != name:
            continue
        xs = [torch.from_numpy(x).to(dev) for x in make_inputs(code, ext, seed)]
        ixs, iy = parse_code(code)
        c = ome.EinCode(ixs, iy)
        y = ome.get_output_array(xs, [ext[l] for l in iy])
        for _ in range(2):
            ome.einsum_(c, xs, y, True, False, ext)
        torch.cuda.synchronize()
        ome.device_status()
        return
    raise SystemExit(f"unknown case {name!r}; one of {[c[0] for c in CASES]}")


def random_regular3(n, seed):
    """Random 3-regular graph (pairing model, resampled until simple), numpy seed."""
    rng = np.random.default_rng(seed)
    while True:
        stubs = np.repeat(np.arange(n), 3)
        rng.shuffle(stubs)
        pairs = stubs.reshape(-1, 2)
        if np.any(pairs[:, 0] == pairs[:, 1]):
            continue
        e = set()
        ok = True
        for a, b in pairs:
            k = (int(min(a, b)), int(max(a, b)))
            if k in e:
                ok = False
                break
            e.add(k)
        if ok:
            return sorted(e)


def tn_network(ome, n, graph_seed=7, value_seed=8, scale=True):
    """3-regular tensor network: one rank-3 bond-2 tensor per vertex, labels =
    edges; FP32 normal(0,1)/sqrt(3) entries (unscaled if scale=False)."""
    import math
    edges = random_regular3(n, graph_seed)
    inc = [[] for _ in range(n)]
    for i, (a, b) in enumerate(edges):
        inc[a].append(i)
        inc[b].append(i)
    code = ome.EinCode([tuple(v) for v in inc], ())
    sd = {i: 2 for i in range(len(edges))}
    rng = np.random.default_rng(value_seed)
    f = 1 / math.sqrt(3) if scale else 1.0
    xs = [(rng.standard_normal((2, 2, 2)) * f).astype(np.float32) for _ in range(n)]
    return code, sd, xs


def tn_section(ome, dev, n=180, sc_target=27):
    """Precision and speed of a 3-regular n=180 network: plain FP32 (CUDA
    cores) vs BF16x6 / BF16x3 (tensor cores), each against FP64 on the same
    plan, FP64 cross-slice sums."""
    import torch
    code, sd, xs = tn_network(ome, n)
    opt = ome.optimize_code(code, sd, ome.GreedyMethod(nrepeat=10, seed=0))
    se = ome.slice_code(opt, sd, ome.GreedySlicer(sc_target=sc_target))
    cs = ome.contraction_complexity(se, sd)
    out = {"workload": f"random 3-regular graph n={n} (seed 7), bond 2, FP32 normal(0,1)/sqrt(3) (seed 8); "
                       f"greedy order (seed 0), sliced to 2^{sc_target} elements "
                       f"({len(se.slicing)} labels, {2 ** len(se.slicing)} slices), tc=2^{cs.tc:.2f}",
           "flops_per_contraction": 2 * 2 ** cs.tc}
    vals = {}
    for name, dt, prec in [("fp64", torch.float64, 0), ("fp32", torch.float32, 1), ("bf16x6", torch.float32, 3),
                           ("bf16x3", torch.float32, 2)]:
        ome.set_einsum_backend(ome.B200Backend(prec=prec))
        d = [torch.from_numpy(x.astype(np.float64 if dt == torch.float64 else np.float32)).to(dev) for x in xs]
        r = se(*d)
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        r = se(*d)
        e1.record()
        torch.cuda.synchronize()
        ome.device_status()
        vals[name] = float(r.double().cpu())
        out[name] = {"s": e0.elapsed_time(e1) / 1e3, "value": vals[name]}
    for k in ("fp32", "bf16x6", "bf16x3"):
        out[k]["rel_err_vs_fp64"] = abs(vals[k] - vals["fp64"]) / abs(vals["fp64"])
        out[k]["contractions_per_s"] = 1.0 / out[k]["s"]
    for k in ("fp64", "fp32", "bf16x6", "bf16x3"):
        out[k]["tflops"] = out["flops_per_contraction"] / out[k]["s"] / 1e12
    # each arm against its own peak: plain FP32 against the CUDA cores' FP32
    # FMA rate (148 SMs x 128 lanes x 2 flops at the 1965 MHz maximum clock),
    # the split products against measured bf16 / (number of BF16 MMAs)
    _, bf16, src = load_peaks()
    fp32_peak = 148 * 128 * 2 * 1.965e9 / 1e12
    out["fp32"]["frac_of_fp32_cuda_core_peak"] = out["fp32"]["tflops"] / fp32_peak
    out["fp32"]["peak"] = {"tflops": fp32_peak, "source": "nominal: 148 SMs x 128 FP32 lanes x 2 x 1965 MHz"}
    out["bf16x6"]["frac_of_bf16x6_peak"] = out["bf16x6"]["tflops"] / (bf16 / 6)
    out["bf16x3"]["frac_of_bf16x3_peak"] = out["bf16x3"]["tflops"] / (bf16 / 3)
    out["speedup_bf16x6_vs_fp32"] = out["fp32"]["s"] / out["bf16x6"]["s"]
    ome.set_einsum_backend(ome.B200Backend())
    out["_cpu_job"] = (se, sd, xs)   # for the CPU leg (popped before printing)
    return out


def _oracle_tree(O, ne):
    """The package's NestedEinsum as the oracle's tree."""
    if ne.isleaf:
        return O.leaf(ne.tensorindex)
    return O.Node(args=[_oracle_tree(O, a) for a in ne.args], ixs=[list(ix) for ix in ne.eins.ixs],
                  iy=list(ne.eins.iy))


def tn_cpu_baseline(O, job, nsample=1):
    """The oracle's sliced evaluation of the n = 180 network on the host cores,
    FP32 and FP64, over the first nsample slices; the whole contraction's time
    is that times nslices / nsample (slices have equal shapes)."""
    se, sd, xs = job
    tree = _oracle_tree(O, se.eins)
    nsl = 2 ** len(se.slicing)
    res = {}
    for name, dt in (("fp32", np.float32), ("fp64", np.float64)):
        xd = [np.asfortranarray(x.astype(dt)) for x in xs]
        t0 = time.perf_counter()
        O.sliced_partial(list(se.slicing), tree, xd, sd, 0, nsample)
        t = time.perf_counter() - t0
        res[name] = {"s_per_contraction": t * nsl / nsample, "contractions_per_s": nsample / (t * nsl)}
    res.update({"cores": os.cpu_count(), "kind": "port",
                "sample": f"{nsample} of {nsl} slices, oracle (NumPy/OpenBLAS) tree evaluation, scaled by "
                          f"{nsl}/{nsample}"})
    return res


def tn_sharded_section(ome, dev, world, n=180, sc_target=27):
    """The n=180 network's slices spread over the ranks (contiguous slice
    ranges, one NCCL all-reduce of the FP64 partial); device time of one whole
    contraction, max over ranks."""
    import torch
    import torch.distributed as dist
    code, sd, xs = tn_network(ome, n)
    opt = ome.optimize_code(code, sd, ome.GreedyMethod(nrepeat=10, seed=0))
    se = ome.slice_code(opt, sd, ome.GreedySlicer(sc_target=sc_target))
    d = [torch.from_numpy(x).to(dev) for x in xs]
    sh = ome.ShardedSlices(se, d)
    r = sh(d)  # warm-up: plan, workspace, NCCL communicator
    torch.cuda.synchronize()
    dist.barrier()
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    r = sh(d)
    e1.record()
    torch.cuda.synchronize()
    ome.device_status()
    t = torch.tensor([e0.elapsed_time(e1)], dtype=torch.float64, device=dev)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    s = float(t.item()) / 1e3
    return {"workload": f"random 3-regular graph n={n} (seeds 7/8), greedy order (seed 0), sliced to "
                        f"2^{sc_target} elements, BF16x6", "slices": sh.nslices, "ranks": world,
            "slices_per_rank": (sh.nslices + world - 1) // world, "s": s, "contractions_per_s": 1.0 / s,
            "value": float(r.double().cpu()),
            "parallelism": "contiguous slice ranges per rank, one NCCL all-reduce of the FP64 partial"}


def run_group_case(ome, dev, njobs, seed=9):
    """Profiling aid: the first contraction ab,bcd->acd of njobs MPS transfer
    jobs (the batching section's distribution) as one grouped launch on the
    tensor-core kernel (tile config 3): 3 warm-up launches, 5 timed."""
    import torch
    jobs = mps_jobs(njobs, seed)
    g = torch.Generator(device=dev).manual_seed(seed)

    def cx(*shape):
        r = torch.randn(*shape[::-1], generator=g, device=dev)
        i = torch.randn(*shape[::-1], generator=g, device=dev)
        return torch.complex(r, i).permute(*range(len(shape) - 1, -1, -1))

    X = [(cx(j["a"], j["b"]), cx(j["b"], j["c"], j["d"])) for j in jobs]
    b1 = ome.BatchedEinsum(ome.ein("ab,bcd->acd"), X, tile_config=3)
    for _ in range(3):
        b1.run()
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(5):
        b1.run()
    e1.record()
    torch.cuda.synchronize()
    ome.device_status()
    flops = sum(8 * j["a"] * j["b"] * j["c"] * j["d"] for j in jobs)
    ms = e0.elapsed_time(e1) / 5
    print(json.dumps({"group_case": f"{njobs} x ab,bcd->acd ComplexF32, tile config 3", "ms_per_launch": ms,
                      "complex_tflops": flops / (ms / 1e3) / 1e12}))


def mps_jobs(njobs, seed):
    rng = np.random.default_rng(seed)
    jobs = []
    for _ in range(njobs):
        a, b, d, e = (int(8 * rng.integers(1, 17)) for _ in range(4))
        jobs.append(dict(a=a, b=b, c=int(rng.choice([2, 4])), d=d, e=e))
    return jobs


def batch_section(ome, dev, njobs=8192, seed=9):
    """8192 MPS transfer contractions ein"(ab,bcd),de->ace" (ComplexF32, bond
    dims in {8,...,128}, c in {2,4}): two grouped launches in a CUDA graph vs
    one launch per contraction (host loop, and the same launches in a graph)."""
    import torch
    jobs = mps_jobs(njobs, seed)
    g = torch.Generator(device=dev).manual_seed(seed)
    def cx(*shape):  # column-major (Julia layout) ComplexF32 normal(0,1) re/im
        r = torch.randn(*shape[::-1], generator=g, device=dev)
        i = torch.randn(*shape[::-1], generator=g, device=dev)
        return torch.complex(r, i).permute(*range(len(shape) - 1, -1, -1))
    X = [(cx(j["a"], j["b"]), cx(j["b"], j["c"], j["d"]), cx(j["d"], j["e"])) for j in jobs]
    flops = sum(8 * (j["a"] * j["b"] * j["c"] * j["d"] + j["a"] * j["c"] * j["d"] * j["e"]) for j in jobs)
    code1, code2 = ome.ein("ab,bcd->acd"), ome.ein("acd,de->ace")
    b1 = ome.BatchedEinsum(code1, [(x[0], x[1]) for x in X])
    b2 = ome.BatchedEinsum(code2, [(t, x[2]) for t, x in zip(b1.outputs, X)])
    graph = ome.capture_graph(lambda: (b1.run(), b2.run()))

    def timed(fn, reps=3):
        fn()
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        for _ in range(reps):
            fn()
        e1.record()
        torch.cuda.synchronize()
        return e0.elapsed_time(e1) / reps

    t_group = timed(graph.replay)
    mids = [torch.empty_like(t) for t in b1.outputs]
    outs = [torch.empty_like(t) for t in b2.outputs]
    sd = [dict(j) for j in jobs]

    def per_contraction():
        for j, x, m, o in zip(sd, X, mids, outs):
            ome.einsum_(code1, [x[0], x[1]], m, True, False, j)
            ome.einsum_(code2, [m, x[2]], o, True, False, j)

    t_loop = timed(per_contraction, reps=1)
    graph2 = ome.capture_graph(per_contraction)
    t_loop_graph = timed(graph2.replay)
    err = max(float((a - b).abs().max() / b.abs().max()) for a, b in zip(outs[:64], b2.outputs[:64]))

    # each kernel family forced: CUDA-core 64x32 tiles (config 1) and the
    # tensor-core grouped kernel (config 3, BF16x6 splits of the real 2 x 2
    # embedding), errors against a ComplexF64 evaluation by the library
    nref = 256
    refs = []
    for j, x in zip(sd[:nref], X[:nref]):
        m = ome.einsum(code1, [x[0].to(torch.complex128), x[1].to(torch.complex128)], j)
        refs.append(ome.einsum(code2, [m, x[2].to(torch.complex128)], j))
    forced, sampled = {}, {}
    nsmp = 32   # jobs whose results the CPU leg checks against the oracle
    for cfg in (1, 3):
        f1 = ome.BatchedEinsum(code1, [(x[0], x[1]) for x in X], tile_config=cfg)
        f2 = ome.BatchedEinsum(code2, [(t, x[2]) for t, x in zip(f1.outputs, X)], tile_config=cfg)
        fg = ome.capture_graph(lambda: (f1.run(), f2.run()))
        ms = timed(fg.replay)
        e = [float(torch.linalg.vector_norm(y.to(torch.complex128) - r) / torch.linalg.vector_norm(r))
             for y, r in zip(f2.outputs[:nref], refs)]
        forced[cfg] = {"graph_ms": ms, "tflops": flops / (ms / 1e3) / 1e12,
                       "rel_err_vs_c128": {"jobs": nref, "max": max(e), "median": float(np.median(e))}}
        sampled[cfg] = [y.cpu().numpy() for y in f2.outputs[:nsmp]]
        del fg, f1, f2
    _, bf16, src = load_peaks()
    tc_peak = bf16 / 6   # 4 real products x 6 BF16 MMAs = 48 BF16 flops per complex multiply-add (8 flops)
    forced[3]["frac_of_bf16x6_peak"] = forced[3]["tflops"] / tc_peak
    forced[3]["peak"] = {"tflops": tc_peak, "source": f"{src} bf16_tflops / 6 (ComplexF32 flops, BF16x6 of "
                                                      "the real 2 x 2 embedding)"}
    return {"workload": f"{njobs} MPS transfer contractions (ab,bcd),de->ace, a,b,d,e uniform in "
                        "{8,16,...,128}, c in {2,4}, ComplexF32 normal(0,1) re/im (seed 9)",
            "contractions": 2 * njobs, "complex_flops": flops,
            "grouped_graph_ms": t_group, "per_contraction_loop_ms": t_loop,
            "per_contraction_graph_ms": t_loop_graph,
            "jobs_per_s_grouped": njobs / (t_group / 1e3), "jobs_per_s_loop": njobs / (t_loop / 1e3),
            "speedup_vs_loop": t_loop / t_group, "speedup_vs_graphed_loop": t_loop_graph / t_group,
            "tflops_grouped": flops / (t_group / 1e3) / 1e12,
            "tile_config": [b1.tile_config, b2.tile_config], "autotune_us": [b1.tuned_us, b2.tuned_us],
            "tile_configs": "0-2 CUDA-core 32x32, 64x32, 64x64 tiles; 3 tensor cores (k_group_tc)",
            "cuda_core_cfg1": forced[1], "tensor_core_cfg3": forced[3],
            "max_rel_diff_grouped_vs_loop": err,
            "_oracle_samples": [(j, [t.cpu().numpy() for t in x], sampled[1][i], sampled[3][i])
                                for i, (j, x) in enumerate(zip(sd[:nsmp], X[:nsmp]))]}


def serve_section(ome, dev, njobs=400, rate=2000.0, seed=10, nmin=40, nmax=200, grad_frac=0.1, cap_s=120.0,
                  ref_cap_s=25.0):
    """Serving: a Poisson stream (rate/s) of whole 3-regular networks, n
    uniform over even [nmin, nmax], bond 2, unscaled FP32 normal(0,1) entries
    (power-of-two rescaled, log2 scale in FP64), 10% cost_and_gradient jobs;
    admitted by planned peak workspace bytes; 16 slots share a 150 GB budget.
    The offered rate is far above what one GPU completes, so the stream
    measures continuous batching under overload: latency includes queueing.
    Each completed job's value is compared with an FP64 evaluation of the same
    tree by the library on the device (a sample, cheapest first, within
    ref_cap_s seconds); the device FP64 path is itself checked against the
    oracle by the test suite."""
    import torch
    rng = np.random.default_rng(seed)
    t = np.cumsum(rng.exponential(1.0 / rate, njobs))
    ns = rng.integers(nmin // 2, nmax // 2 + 1, njobs) * 2
    grads = rng.random(njobs) < grad_frac
    jobs, plan_s, raw = [], 0.0, []
    for i, (n, g) in enumerate(zip(ns, grads)):
        code, sd, xs = tn_network(ome, int(n), graph_seed=1000 + i, value_seed=2000 + i, scale=False)
        t0 = time.perf_counter()
        opt = ome.optimize_code(code, sd, ome.GreedyMethod(nrepeat=10, seed=i))
        cc = ome.contraction_complexity(opt, sd)
        if cc.sc > 27 and not g:
            opt = ome.slice_code(opt, sd, ome.GreedySlicer(sc_target=27))
        plan_s += time.perf_counter() - t0
        xs, exps = ome.pow2_rescale(xs)
        raw.append((opt, sd, xs, float(sum(exps)), cc.tc))
        jobs.append(ome.Job(opt, [torch.from_numpy(x).to(dev) for x in xs], grad=bool(g), arrival=float(t[i]),
                            log2_scale=float(sum(exps))))
    ome.release_workspaces()
    torch.cuda.empty_cache()
    # admission: planned peak workspace within the budget, and at most 2^45
    # multiply-adds per job (about 0.7 s of device time, the n = 180 network
    # of the precision section): the greedy orders of some large networks
    # need up to 2^54, minutes of device time each
    work_cap = 2.0 ** 45
    srv = ome.TNServer(n_slots=16, hbm_budget_bytes=150e9, max_job_flops=work_cap)
    # one untimed pass of the first 48 jobs (kernel loading, slot workspaces),
    # then the measured stream on the same server
    srv.run_trace([ome.Job(j.code, j.xs, grad=j.grad, arrival=j.arrival, log2_scale=j.log2_scale)
                   for j in jobs[:48]], timeout_s=cap_s)
    st = srv.run_trace(jobs, timeout_s=cap_s)
    srv.close()
    finished_ids = {id(j) for j in srv.finished}
    done = [j for j in jobs if j.done >= 0 and j.value is not None and id(j) in finished_ids]
    pos = {id(j): i for i, j in enumerate(jobs)}
    # relative error of the served values against FP64 on the same trees
    ome.release_workspaces()
    torch.cuda.empty_cache()
    errs, refs, t_ref = [], {}, time.perf_counter()
    order = sorted(done, key=lambda j: raw[pos[id(j)]][4])
    for j in order:
        if time.perf_counter() - t_ref > ref_cap_s:
            break
        opt, sd, xs, lg, _ = raw[pos[id(j)]]
        ref = ome.einsum(opt, [torch.from_numpy(x.astype(np.float64)).to(dev) for x in xs], sd)
        ref = float(ref.double().cpu()) * 2.0 ** lg
        if ref != 0 and math.isfinite(ref):
            errs.append(abs(j.scalar() - ref) / abs(ref))
            refs[pos[id(j)]] = ref
    # the same stream through the library's own serving loop (ome_server_*):
    # admission, slots and issue threads in C++, the same rules
    ome.release_workspaces()
    torch.cuda.empty_cache()
    nsrv = ome.NativeTNServer(n_slots=16, hbm_budget_bytes=150e9, max_job_flops=work_cap)
    nsrv.run_trace([ome.Job(j.code, j.xs, grad=j.grad, arrival=j.arrival, log2_scale=j.log2_scale)
                    for j in jobs[:48]], timeout_s=cap_s)
    njobs_native = [ome.Job(j.code, j.xs, grad=j.grad, arrival=j.arrival, log2_scale=j.log2_scale) for j in jobs]
    nsrv.finished, nsrv.rejected = [], []
    t_native = time.perf_counter()
    nsrv.run_trace(njobs_native, timeout_s=cap_s)
    nsrv.close()
    ndone = {id(j) for j in nsrv.finished}
    both = [(a, b) for a, b in zip(jobs, njobs_native) if id(a) in finished_ids and id(b) in ndone]
    same = sum(1 for a, b in both if torch.equal(a.value, b.value))
    # kernels may differ between the two runs where a GEMM's operand buffer
    # depends on free device memory, so values agree to rounding, not always bitwise
    vdiff = max((float((a.value.double() - b.value.double()).abs().max()
                       / max(a.value.double().abs().max(), b.value.double().abs().max()))
                 for a, b in both if float(b.value.double().abs().max()) > 0), default=0.0)
    nerrs = [abs(b.scalar() - refs[i]) / abs(refs[i]) for i, b in enumerate(njobs_native)
             if i in refs and id(b) in ndone]
    nlat = np.array([j.done - j.arrival for j in nsrv.finished]) if nsrv.finished else np.zeros(1)
    reasons = [j.reject_reason for j in nsrv.rejected]   # this stream only (the library counts both passes)
    native = {"completed": len(nsrv.finished), "rejected_over_work_cap": reasons.count("work"),
              "rejected_memory": reasons.count("memory"), "failed": reasons.count("failed"),
              "p50_ms": float(np.percentile(nlat, 50) * 1e3), "p90_ms": float(np.percentile(nlat, 90) * 1e3),
              "p99_ms": float(np.percentile(nlat, 99) * 1e3),
              "jobs_per_s": len(nsrv.finished) / max(max((j.done for j in nsrv.finished), default=0.0)
                                                     - min((j.arrival for j in nsrv.finished), default=0.0), 1e-9),
              "wall_s": time.perf_counter() - t_native,
              "queue_wait_p50_ms": float(np.percentile([j.admitted - j.arrival for j in nsrv.finished], 50) * 1e3)
              if nsrv.finished else 0.0,
              "service_p50_ms": float(np.percentile([j.done - j.admitted for j in nsrv.finished], 50) * 1e3)
              if nsrv.finished else 0.0,
              "values_identical_to_python_server": f"{same}/{len(both)}",
              "max_rel_diff_vs_python_server": vdiff,
              "rel_err_vs_fp64": {"jobs": len(nerrs), "max": max(nerrs) if nerrs else None,
                                  "median": float(np.median(nerrs)) if nerrs else None,
                                  "within_1e-5": sum(e <= 1e-5 for e in nerrs),
                                  "reference": "the same FP64 values as the Python server's check"},
              "api": "ome_server_create/submit/poll/stats (C ABI), driven by NativeTNServer"}
    lat = np.array([j.latency for j in done]) if done else np.zeros(1)
    st.update({"workload": f"{njobs} jobs, Poisson {rate:.0f}/s (seed {seed}), n uniform even [{nmin},{nmax}], "
                           "bond 2, unscaled FP32 normal(0,1), 10% gradient jobs, greedy order (best of 10) + greedy "
                           "slicing to 2^27 (client side), 16 slots sharing a 150 GB workspace budget, jobs above "
                           "2^45 multiply-adds rejected at admission; measured after one untimed pass of the first "
                           "48 jobs",
               "submitted": njobs, "offered_jobs_per_s": rate, "max_job_multiply_adds": work_cap,
               "incomplete": njobs - len(done) - int(st.get("rejected", 0)), "cap_s": cap_s,
               "p90_ms": float(np.percentile(lat, 90) * 1e3),
               "queue_wait_p50_ms": float(np.percentile([j.admitted - j.arrival for j in done], 50) * 1e3)
               if done else 0.0,
               "service_p50_ms": float(np.percentile([j.done - j.admitted for j in done], 50) * 1e3) if done else 0.0,
               "gradient_jobs_completed": sum(1 for j in done if j.grad),
               "rel_err_vs_fp64": {"jobs": len(errs), "max": max(errs) if errs else None,
                                   "median": float(np.median(errs)) if errs else None,
                                   "within_1e-5": sum(e <= 1e-5 for e in errs),
                                   "reference": "FP64 evaluation of the same tree by the library (cheapest jobs "
                                                f"first, {ref_cap_s:.0f} s cap)"},
               "client_planning_s": plan_s, "native_server": native})
    return st


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
            "config": {"workload": WORKLOAD, "l2": L2_POLICY}, "impl": "reference",
            "prec": "plain FP32 (OpenBLAS SGEMM on the host cores)", "parallelism": "rank 0 only",
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
    ap.add_argument("--prec", type=int, default=0, help="0 AUTO (BF16x6), 1 plain FP32, 2 BF16x3, 3 BF16x6")
    ap.add_argument("--no-cpu", action="store_true", help="skip the cpu_baseline leg")
    ap.add_argument("--no-tn", action="store_true", help="skip the tensor-network precision section")
    ap.add_argument("--no-batch", action="store_true", help="skip the batched MPS-transfer section")
    ap.add_argument("--no-serve", action="store_true", help="skip the serving section")
    ap.add_argument("--no-int64", action="store_true", help="skip the Int64 rule-suite section")
    ap.add_argument("--tn-sharded", action="store_true",
                    help="run the slice-sharded network section at N=1 too (a one-rank NCCL group)")
    ap.add_argument("--case", default=None,
                    help="profiling aid: run only this suite contraction (e.g. 'ijk->j') twice and exit")
    ap.add_argument("--group-case", type=int, default=0,
                    help="profiling aid: one grouped tensor-core launch over this many MPS jobs (ab,bcd->acd)")
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
    grouped = world > 1 or args.tn_sharded
    if grouped:
        import datetime
        if world == 1:
            os.environ.setdefault("MASTER_ADDR", "127.0.0.1")
            os.environ.setdefault("MASTER_PORT", "29517")
            os.environ.setdefault("RANK", "0")
            os.environ.setdefault("WORLD_SIZE", "1")
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    ome.set_einsum_backend(ome.B200Backend(prec=args.prec))
    lib = ome.load_library()
    if args.case is not None:
        return run_case_only(ome, args.case, dev)
    if args.group_case:
        return run_group_case(ome, dev, args.group_case)

    hosts, devs, outs, codes = [], [], [], []
    for name, code, ext, seed in CASES:
        xs = make_inputs(code, ext, seed)
        hosts.append([torch.from_numpy(x).pin_memory() for x in xs])
        devs.append([h.to(dev) for h in hosts[-1]])
        ixs, iy = parse_code(code)
        c = ome.EinCode(ixs, iy)
        codes.append((c, ext))
        outs.append(ome.get_output_array(devs[-1], [ext[l] for l in iy]))
    # L2 flush before every contraction, outside its events: a 256 MiB write
    # followed by a 256 MiB read, so the timed kernel starts with a cold L2
    # that holds no dirty lines (the write alone leaves up to 126 MB of dirty
    # lines whose write-back would land inside the next timed window)
    flush = torch.empty(256 << 20, dtype=torch.uint8, device=dev)
    clean = torch.ones(64 << 20, dtype=torch.float32, device=dev)
    sink = torch.empty((), dtype=torch.float32, device=dev)

    def flush_l2(i):
        flush.fill_(i)
        torch.sum(clean, dim=0, out=sink)

    ev = [[(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in CASES]
          for _ in range(args.steps)]

    def step(k=None):
        for i, (c, ext) in enumerate(codes):
            flush_l2(i)
            if k is not None:
                ev[k][i][0].record()
            ome.einsum_(c, devs[i], outs[i], True, False, ext)
            if k is not None:
                ev[k][i][1].record()

    cs = ClockSampler(local).__enter__()   # sampling starts under the warm-up load
    t_w = time.perf_counter()
    nw = 0
    while nw < max(args.warmup, 3) or time.perf_counter() - t_w < 1.0:
        step()
        nw += 1
        if nw % 8 == 0:
            torch.cuda.synchronize()
    torch.cuda.synchronize()
    # main kernels per contraction (the library brackets each dispatch's main
    # kernel with events on its stream when asked): one probe pass
    import ctypes as C
    kcount = []
    fbuf, nbuf, cnt = (C.c_float * 4096)(), (C.c_char_p * 4096)(), C.c_int32()
    for i, (c, ext) in enumerate(codes):
        lib.ome_kernel_timing(64)
        ome.einsum_(c, devs[i], outs[i], True, False, ext)
        torch.cuda.synchronize()
        lib.ome_kernel_times(4096, fbuf, nbuf, C.byref(cnt))
        kcount.append((cnt.value, [nbuf[j].decode() for j in range(cnt.value)]))
    lib.ome_kernel_timing(0)
    torch.cuda.synchronize()
    if world > 1:
        dist.barrier()
    n0 = lib.ome_launch_count()
    torch.cuda.synchronize()
    for k in range(args.steps):
        step(k)
    torch.cuda.synchronize()
    launches = lib.ome_launch_count() - n0
    # the same steps again with the main kernels bracketed by events (they
    # add a few microseconds per contraction, so the timed steps above run
    # without them); event pairs are created before this pass
    nt = args.steps * sum(c for c, _ in kcount)
    lib.ome_kernel_timing(max(nt, 1))
    for k in range(args.steps):
        step()
    torch.cuda.synchronize()
    kt = (C.c_float * max(nt, 1))()
    knames = (C.c_char_p * max(nt, 1))()
    lib.ome_kernel_times(nt, kt, knames, C.byref(cnt))
    lib.ome_kernel_timing(0)
    kernel_ms = [0.0] * len(CASES)   # per contraction: its main kernels' time, averaged over steps
    if cnt.value == nt:
        pos = 0
        for _ in range(args.steps):
            for i, (c, _) in enumerate(kcount):
                kernel_ms[i] += sum(kt[pos + j] for j in range(c)) / args.steps
                pos += c
    cs.__exit__()
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
    jobs = [(c, hosts[i], ext) for i, (c, ext) in enumerate(codes)]

    def e2e_leg(step):
        for _ in range(2):
            step()
        torch.cuda.synchronize()
        s0, s1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        s0.record()
        for k in range(args.steps):
            step()
        s1.record()
        torch.cuda.synchronize()
        te = torch.tensor([s0.elapsed_time(s1) / args.steps], dtype=torch.float64, device=dev)
        if world > 1:
            dist.all_reduce(te, op=dist.ReduceOp.MAX)
        return len(CASES) * world / (float(te.item()) / 1e3)

    # one step = the six contractions through einsum_many: each result's
    # device->host copy overlaps the next contraction's host->device copy
    e2e_value = e2e_leg(lambda: ome.einsum_many(jobs))
    # the same, one blocking einsum call per contraction
    e2e_serial = e2e_leg(lambda: [ome.einsum(c, xs, ext) for c, xs, ext in jobs])

    # roofline of the dominant contraction's main kernel: algorithmic work of
    # the contraction / that kernel's average event-timed duration in the
    # timed steps; case_frac is the same over the whole contraction (all its
    # launches, e.g. the operand packing of the tensor-core GEMM)
    hbm, bf16, src = load_peaks()
    dom = int(np.argmax(per_case))
    name, code, ext, _ = CASES[dom]
    flops, nbytes = case_work(code, ext)
    case_s = per_case[dom] / 1e3
    dur_s = kernel_ms[dom] / 1e3 if kernel_ms[dom] > 0 else case_s
    kname = "+".join(kcount[dom][1]) or "all launches"
    nmma = {0: 6, 3: 6, 2: 3}.get(args.prec, 6)   # BF16 MMAs per FP32 product (BF16x6 / BF16x3)
    tc_peak = bf16 / nmma
    t_flop = flops / (tc_peak * 1e12) if flops else 0.0
    t_mem = nbytes / (hbm * 1e9)
    traffic = load_traffic().get(name)
    if t_flop > t_mem:
        roof = {"bound": "tensor", "achieved": flops / dur_s / 1e12, "peak": tc_peak, "unit": "TFLOP/s",
                "frac": (flops / dur_s / 1e12) / tc_peak, "traffic": traffic,
                "kernel": f"{kname} ({name})", "kernel_us": dur_s * 1e6, "case_us": case_s * 1e6,
                "case_frac": (flops / case_s / 1e12) / tc_peak,
                "peak_source": f"{src} bf16_tflops / {nmma} (FP32-equivalent of BF16x{nmma})"}
    else:
        roof = {"bound": "hbm", "achieved": nbytes / dur_s / 1e9, "peak": hbm, "unit": "GB/s",
                "frac": (nbytes / dur_s / 1e9) / hbm, "traffic": traffic, "kernel": f"{kname} ({name})",
                "kernel_us": dur_s * 1e6, "case_us": case_s * 1e6, "case_frac": (nbytes / case_s / 1e9) / hbm,
                "peak_source": f"{src} hbm_gbs"}

    i64 = i64_inputs = i64_results = None
    if not args.no_int64:
        i64, i64_inputs, i64_results = int64_section(ome, dev, args.steps, flush_l2, lib)

    cpu = parity = None
    if rank == 0 and world == 1 and not args.no_cpu:
        sys.path.insert(0, os.path.join(ROOT, "oracle"))
        import ome_oracle as O
        inputs = [[h.numpy() for h in hs] for hs in hosts]
        oracle_out = {}
        tc = cpu_suite(O, inputs, 1, oracle_out)
        cpu = {"value": len(CASES) / tc, "unit": "contractions/s", "cores": os.cpu_count(), "kind": "port",
               "sample": "the full suite once, NumPy/OpenBLAS DefaultBackend restatement "
                         f"(BLAS threads = {os.cpu_count()}; copies single-threaded)"}
        gpu_out = {name: o.cpu().numpy() for (name, _, _, _), o in zip(CASES, outs)}
        parity = suite_parity(O, inputs, gpu_out, oracle_out, i64_inputs, i64_results)

    del devs, outs, flush, clean
    ome.release_workspaces()
    torch.cuda.empty_cache()
    tn = None if (args.no_tn or world > 1) else tn_section(ome, dev)
    if tn is not None:
        job = tn.pop("_cpu_job")
        if cpu is not None:   # the CPU leg ran: the oracle on a sample of the slices
            tn["cpu_baseline"] = tn_cpu_baseline(O, job)
    ome.release_workspaces()
    torch.cuda.empty_cache()
    sharded = tn_sharded_section(ome, dev, world) if (grouped and not args.no_tn) else None
    batch = None if (args.no_batch or world > 1) else batch_section(ome, dev)
    if batch is not None:
        smp = batch.pop("_oracle_samples")
        if cpu is not None:   # the CPU leg ran: check sampled jobs of both kernels against the oracle
            ne = O.parse_nested("(ab,bcd),de->ace")
            errs = {1: [], 3: []}
            for j, xs, y1, y3 in smp:
                want = O.nested_einsum(ne, [x.astype(np.complex128) for x in xs], j)
                errs[1].append(relerr(y1, want))
                errs[3].append(relerr(y3, want))
            for cfg, key in ((1, "cuda_core_cfg1"), (3, "tensor_core_cfg3")):
                batch[key]["rel_err_vs_oracle"] = {"jobs": len(smp), "max": max(errs[cfg]),
                                                   "median": float(np.median(errs[cfg])),
                                                   "reference": "oracle (ComplexF64 NumPy restatement)"}
            # CPU baseline: the sampled jobs as a NumPy ComplexF32 loop (tensordot = BLAS CGEMM)
            reps = 3
            t0 = time.perf_counter()
            for _ in range(reps):
                for j, xs, _, _ in smp:
                    t = np.tensordot(xs[0], xs[1], axes=(1, 0))      # (a, c, d)
                    np.tensordot(t, xs[2], axes=(2, 0))             # (a, c, e)
            tc = (time.perf_counter() - t0) / reps
            batch["cpu_baseline"] = {"jobs_per_s": len(smp) / tc, "unit": "jobs/s", "cores": os.cpu_count(),
                                     "kind": "port", "sample": f"{len(smp)} of the jobs, {reps} passes, NumPy "
                                                               "complex64 tensordot loop"}
    serve = None if (args.no_serve or world > 1) else serve_section(ome, dev)
    detail = {}
    for (nm, code, ext, _), ms in zip(CASES, per_case):
        f, b = case_work(code, ext)
        detail[nm] = {"us": ms * 1e3, "GB/s": b / (ms / 1e3) / 1e9}
        if kernel_ms[len(detail) - 1] > 0:
            detail[nm]["main_kernel_us"] = kernel_ms[len(detail) - 1] * 1e3
            detail[nm]["main_kernel"] = "+".join(kcount[len(detail) - 1][1])
        if f:
            detail[nm]["TFLOP/s"] = f / (ms / 1e3) / 1e12
    if rank == 0:
        line = {"metric": METRIC, "value": value, "unit": "contractions/s", "n_gpus": world, "steps": args.steps,
                "warmup": args.warmup, "warmup_steps_run": nw, "ms_per_step": step_ms_max, "higher_is_better": True,
                "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded normal(0,1))",
                "config": {"workload": WORKLOAD, "l2": L2_POLICY},
                "prec": {0: "BF16x6 tensor-core split products (FP32-faithful) where GEMM-shaped",
                         1: "plain FP32 (CUDA cores)", 2: "BF16x3 where GEMM-shaped",
                         3: "BF16x6 where GEMM-shaped"}[args.prec],
                "parallelism": f"replicas x{world}", "per_case": detail, "parity_vs_oracle": parity,
                "int64_suite": i64,
                "e2e": {"value": e2e_value, "unit": "contractions/s", "h2d_bytes_per_step": h2d,
                        "d2h_bytes_per_step": d2h, "api": "einsum_many", "serial_einsum_value": e2e_serial},
                "gpu_launches": int(launches), "roofline": roof, "cpu_baseline": cpu,
                "clocks": cs.summary(), "tn_precision": tn, "tn_sharded": sharded, "batching": batch,
                "serving": serve}
        print(json.dumps(line), flush=True)
    if grouped:
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
