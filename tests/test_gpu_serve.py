"""Serving loop: jobs admitted as slots and memory free up, overlapping on the
device; every result must be the same alone and in the mix, and match FP64."""
import math

import numpy as np
import pytest
import torch

import ome_oracle as O
import omeinsum_b200 as ome

pytestmark = pytest.mark.gpu


def network(n, seed):
    rng = np.random.default_rng(seed)
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
    opt = ome.optimize_code(code, sd, ome.GreedyMethod(nrepeat=2, seed=seed))
    xs = [torch.from_numpy(rng.standard_normal((2, 2, 2)).astype(np.float32)).cuda() for _ in range(n)]
    return opt, sd, xs


def test_results_same_alone_and_in_the_mix():
    specs = [(20 + 4 * i, 100 + i, i % 4 == 3) for i in range(10)]
    nets = [network(n, s) for n, s, _ in specs]
    alone = []
    for (opt, sd, xs), (_, _, g) in zip(nets, specs):
        srv = ome.TNServer(n_slots=1, hbm_budget_bytes=4e9)
        job = ome.Job(opt, xs, grad=g)
        srv.run_trace([job])
        srv.close()
        alone.append(job)
    srv = ome.TNServer(n_slots=4, hbm_budget_bytes=8e9)
    mixed = [ome.Job(opt, xs, grad=g, arrival=0.001 * i) for i, ((opt, sd, xs), (_, _, g)) in enumerate(zip(nets, specs))]
    st = srv.run_trace(mixed)
    srv.close()
    assert st["completed"] == len(specs) and st["p99_ms"] >= st["p50_ms"] > 0
    for a, m, (opt, sd, xs), (n, _, g) in zip(alone, mixed, nets, specs):
        assert torch.equal(a.value, m.value) and a.log2_scale == m.log2_scale
        if g:
            for ga, gm in zip(a.grads, m.grads):
                assert torch.equal(ga, gm)
        # FP64 oracle on the same tree
        want = O.nested_einsum(_tree(opt), [x.double().cpu().numpy() for x in xs], sd)
        assert abs(m.scalar() - float(want)) <= 1e-5 * abs(float(want))


def _tree(ne):
    if ne.isleaf:
        return O.leaf(ne.tensorindex)
    return O.Node(args=[_tree(a) for a in ne.args], ixs=[list(ix) for ix in ne.eins.ixs], iy=list(ne.eins.iy))


def test_admission_respects_the_memory_budget():
    opt, sd, xs = network(40, 7)
    srv = ome.TNServer(n_slots=4, hbm_budget_bytes=1)  # nothing fits: rejected, not run
    st = srv.run_trace([ome.Job(opt, xs)])
    assert st["rejected"] == 1 and st["completed"] == 0


def test_large_job_runs_alone_in_its_own_workspace():
    """A gradient job whose planned workspace exceeds a slot's share (but not
    the budget) is not rejected: it waits until the device is idle and runs
    alone in a workspace of its own size; the jobs around it still run in
    their slots.  Every result against the FP64 oracle."""
    from omeinsum_b200 import _lib
    from omeinsum_b200.plan import get_plan
    big = network(48, 21)
    opt, sd, xs = big
    need = get_plan(opt, sd, _lib.F32, 0).grad_bytes
    smalls = [network(16, 30 + i) for i in range(3)]
    srv = ome.TNServer(n_slots=4, hbm_budget_bytes=2 * need)
    assert srv.slot_bytes < need <= srv.budget
    jobs = [ome.Job(smalls[0][0], smalls[0][2], arrival=0.0),
            ome.Job(opt, xs, grad=True, arrival=0.001),
            ome.Job(smalls[1][0], smalls[1][2], arrival=0.002),
            ome.Job(smalls[2][0], smalls[2][2], grad=True, arrival=0.003)]
    st = srv.run_trace(jobs)
    srv.close()
    assert st["completed"] == 4 and st["rejected"] == 0
    for job, (o, s, x) in zip(jobs, [smalls[0], big, smalls[1], smalls[2]]):
        xd = [t.double().cpu().numpy() for t in x]
        want = O.nested_einsum(_tree(o), xd, s)
        assert abs(job.scalar() - float(want)) <= 1e-5 * abs(float(want))
        if job.grad:
            _, g0 = O.cost_and_gradient(_tree(o), xd)
            for g, w in zip(job.grads, g0):
                w = np.asarray(w)
                assert np.linalg.norm(g.double().cpu().numpy() - w) <= 1e-5 * np.linalg.norm(w)


def test_work_cap_rejects_only_oversized_jobs():
    """Jobs above the server's per-job work cap are rejected at admission
    (reason "work"); the others complete and match the oracle."""
    small = network(20, 41)
    big = network(60, 42)
    cap = 2.0 ** ome.contraction_complexity(small[0], small[1]).tc * 2
    assert 2.0 ** ome.contraction_complexity(big[0], big[1]).tc > cap
    srv = ome.TNServer(n_slots=2, hbm_budget_bytes=4e9, max_job_flops=cap)
    jobs = [ome.Job(small[0], small[2]), ome.Job(big[0], big[2], arrival=0.001)]
    st = srv.run_trace(jobs)
    srv.close()
    assert st["completed"] == 1 and st["rejected"] == 1 and st["rejected_over_work_cap"] == 1
    assert jobs[1].reject_reason == "work" and jobs[1].value is None
    want = O.nested_einsum(_tree(small[0]), [t.double().cpu().numpy() for t in small[2]], small[1])
    assert abs(jobs[0].scalar() - float(want)) <= 1e-5 * abs(float(want))
