"""The serving loop inside the library (ome_server_*, NativeTNServer) and the
library-built CUDA graph of grouped launches (ome_batch_graph_create,
BatchGraph): the same results as the Python server and as eager runs, the
same admission rules, and the FP64 oracle."""
import numpy as np
import pytest
import torch

import ome_oracle as O
import omeinsum_b200 as ome
from helpers import gen, relerr, to_dev, to_np
from test_gpu_serve import _tree, network

pytestmark = pytest.mark.gpu


def test_native_server_matches_python_server_and_oracle():
    specs = [(20 + 4 * i, 100 + i, i % 4 == 3) for i in range(10)]
    nets = [network(n, s) for n, s, _ in specs]
    py = ome.TNServer(n_slots=4, hbm_budget_bytes=8e9)
    ref = [ome.Job(o, xs, grad=g, arrival=0.001 * i) for i, ((o, sd, xs), (_, _, g)) in enumerate(zip(nets, specs))]
    py.run_trace(ref)
    py.close()
    srv = ome.NativeTNServer(n_slots=4, hbm_budget_bytes=8e9)
    jobs = [ome.Job(o, xs, grad=g, arrival=0.001 * i) for i, ((o, sd, xs), (_, _, g)) in enumerate(zip(nets, specs))]
    st = srv.run_trace(jobs)
    srv.close()
    assert st["submitted"] == st["completed"] == len(specs)
    assert st["failed"] == st["rejected_memory"] == st["rejected_work"] == 0
    assert st["p99_ms"] >= st["p50_ms"] > 0 and st["jobs_per_s"] > 0
    for a, m, (o, sd, xs) in zip(ref, jobs, nets):
        assert m.done >= m.admitted >= m.arrival >= 0
        assert torch.equal(a.value, m.value)
        if m.grad:
            for ga, gm in zip(a.grads, m.grads):
                assert torch.equal(ga, gm)
        want = O.nested_einsum(_tree(o), [x.double().cpu().numpy() for x in xs], sd)
        assert abs(m.scalar() - float(want)) <= 1e-5 * abs(float(want))


def test_native_server_runs_a_large_job_alone_and_rejects_by_budget_and_work():
    from omeinsum_b200 import _lib
    from omeinsum_b200.plan import get_plan
    big = network(48, 21)
    opt, sd, xs = big
    need = get_plan(opt, sd, _lib.F32, 0).grad_bytes
    smalls = [network(16, 30 + i) for i in range(3)]
    # slot share = need / 2: the big gradient job must run alone
    srv = ome.NativeTNServer(n_slots=4, hbm_budget_bytes=2 * need)
    jobs = [ome.Job(smalls[0][0], smalls[0][2], arrival=0.0),
            ome.Job(opt, xs, grad=True, arrival=0.001),
            ome.Job(smalls[1][0], smalls[1][2], arrival=0.002),
            ome.Job(smalls[2][0], smalls[2][2], grad=True, arrival=0.003)]
    st = srv.run_trace(jobs)
    srv.close()
    assert st["completed"] == 4 and st["rejected_memory"] == 0
    for job, (o, s, x) in zip(jobs, [smalls[0], big, smalls[1], smalls[2]]):
        xd = [t.double().cpu().numpy() for t in x]
        want = O.nested_einsum(_tree(o), xd, s)
        assert abs(job.scalar() - float(want)) <= 1e-5 * abs(float(want))
        if job.grad:
            _, g0 = O.cost_and_gradient(_tree(o), xd)
            for g, w in zip(job.grads, g0):
                w = np.asarray(w)
                assert np.linalg.norm(g.double().cpu().numpy() - w) <= 1e-5 * np.linalg.norm(w)
    # nothing fits a 1-byte budget; a work cap below the big job's work
    srv = ome.NativeTNServer(n_slots=2, hbm_budget_bytes=1)
    st = srv.run_trace([ome.Job(smalls[0][0], smalls[0][2])])
    srv.close()
    assert st["rejected_memory"] == 1 and st["completed"] == 0
    cap = 2.0 ** ome.contraction_complexity(smalls[0][0], smalls[0][1]).tc * 2
    srv = ome.NativeTNServer(n_slots=2, hbm_budget_bytes=8e9, max_job_flops=cap)
    jobs = [ome.Job(smalls[0][0], smalls[0][2]), ome.Job(opt, xs, arrival=0.001)]
    st = srv.run_trace(jobs)
    srv.close()
    assert st["completed"] == 1 and st["rejected_work"] == 1
    assert jobs[1].reject_reason == "work" and jobs[1].value is None


@pytest.mark.parametrize("tile_config", [1, 3])
def test_batch_graph_replays_the_grouped_launches(tile_config):
    """ome_batch_graph_create captures the two contractions of an MPS sweep
    step; each replay equals eager runs and the oracle (ComplexF64)."""
    rng = np.random.default_rng(5)
    jobs = []
    for _ in range(24):
        a, b, d, e = (int(8 * rng.integers(1, 9)) for _ in range(4))
        jobs.append(dict(a=a, b=b, c=int(rng.choice([2, 4])), d=d, e=e))
    X = [[gen(rng, (s["a"], s["b"]), "c64"), gen(rng, (s["b"], s["c"], s["d"]), "c64"),
          gen(rng, (s["d"], s["e"]), "c64")] for s in jobs]
    dev = [[to_dev(x, "c64") for x in xs] for xs in X]
    b1 = ome.BatchedEinsum(ome.ein("ab,bcd->acd"), [(x[0], x[1]) for x in dev], tile_config=tile_config)
    b2 = ome.BatchedEinsum(ome.ein("acd,de->ace"), [(t, x[2]) for t, x in zip(b1.outputs, dev)],
                           tile_config=tile_config)
    b1.run()
    b2.run()
    torch.cuda.synchronize()
    eager = [y.clone() for y in b2.outputs]
    for y in b2.outputs:
        y.zero_()
    g = ome.BatchGraph([b1, b2])
    ne = O.parse_nested("(ab,bcd),de->ace")
    for _ in range(2):
        g.launch()
        torch.cuda.synchronize()
        for s, xs, y, ye in zip(jobs, X, b2.outputs, eager):
            assert torch.equal(y, ye)
            want = O.nested_einsum(ne, [x.astype(np.complex128) for x in xs], s)
            assert relerr(to_np(y), want) < 1e-5
    # per-batch scalars: y2 <- 2 * (x1 x2) (the first launch as before)
    g2 = ome.BatchGraph([b1, b2], sxs=[1.0, 2.0], sys=[0.0, 0.0])
    g2.launch()
    torch.cuda.synchronize()
    for y, ye in zip(b2.outputs, eager):
        assert torch.allclose(y, 2 * ye, rtol=1e-6, atol=0)


def test_native_server_waits_for_the_submitting_stream():
    """Inputs written on the default stream just before submit (behind a long
    fill): the jobs' kernels on the slots' non-blocking streams must run after
    them.  Values against the oracle."""
    nets = [network(24 + 4 * i, 300 + i) for i in range(8)]
    big = torch.empty(1 << 28, device="cuda")   # 1 GiB: a fill of ~0.2 ms on the default stream
    srv = ome.NativeTNServer(n_slots=8, hbm_budget_bytes=8e9)
    jobs = []
    for i, (o, sd, xs) in enumerate(nets):
        big.fill_(float(i))
        ys = [x * 1.0 for x in xs]              # queued behind the fill
        jobs.append(ome.Job(o, ys))
        srv.submit(jobs[-1])
        srv.poll()
    while srv.poll() or srv._live:
        pass
    srv.close()
    assert len(srv.finished) == len(nets)
    for job, (o, sd, xs) in zip(jobs, nets):
        want = O.nested_einsum(_tree(o), [x.double().cpu().numpy() for x in xs], sd)
        assert abs(job.scalar() - float(want)) <= 1e-5 * abs(float(want))
