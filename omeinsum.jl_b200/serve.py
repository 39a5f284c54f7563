"""Serving loop for whole tensor-network contraction jobs (continuous batching).

A job is an optimised contraction code (NestedEinsum or SlicedEinsum, as a
client gets from ``optimize_code``/``slice_code``) plus its input tensors, and
asks either for the value or for ``cost_and_gradient``.  ``TNServer`` keeps a
fixed number of slots; each slot owns a CUDA stream, a host thread that
issues its job, and a library context whose device workspace (the slot's
share of the HBM budget) holds one job's intermediates.  Jobs are admitted in
arrival order when a slot is free and the job's planned peak workspace bytes
(``ome_plan_peak_bytes``) fit a slot's share; a job larger than a share but
within the whole budget (a gradient job keeps every intermediate) waits until
the device is idle and runs alone in a workspace of its own size; only jobs
beyond the budget are rejected.  Work of different jobs overlaps on the
device (one stream per slot, the slices of different jobs interleave); a
finished slot takes the next job at once.  Latency is
measured from arrival to the completion event of the job's last kernel.

Large networks: ``pow2_rescale`` scales every input by an exact power of two
so that its largest magnitude is in [1, 2) and returns the exponents; a job
carries their sum as ``log2_scale`` (FP64) and its result is reported as
(mantissa, log2 scale) -- a log-scale renormalisation that keeps unscaled
networks of 200 vertices inside the FP32 range without changing a rounding.
Rescaling happens when the job is built (on the host), so admission never
waits for the device.
"""
from __future__ import annotations

import ctypes as C
import math
import queue as _queue
import threading
import time
from collections import deque
from dataclasses import dataclass, field
from typing import Any, List, Optional, Sequence

import numpy as np
import torch

from . import _lib
from ._lib import check
from .core import NestedEinsum, SlicedEinsum, get_size_dict
from .engine import _alloc, _f_contig, _Prepared, _scalar_buf
from .plan import get_plan


def pow2_rescale(xs: Sequence[Any]):
    """Scale each floating array (NumPy or torch) by 2^-e, e = floor(log2 max|x|)
    (exact unless it underflows); returns (arrays, per-array exponents)."""
    out, exps = [], []
    for x in xs:
        e = 0
        floating = (x.dtype.kind in "fc") if isinstance(x, np.ndarray) else (x.is_floating_point() or x.is_complex())
        if floating and x.size if isinstance(x, np.ndarray) else floating and x.numel():
            m = float(np.abs(x).max()) if isinstance(x, np.ndarray) else float(x.abs().max())
            if m > 0 and math.isfinite(m):
                e = math.floor(math.log2(m))
        if e != 0:
            x = x * x.dtype.type(2.0 ** -e) if isinstance(x, np.ndarray) else x * (2.0 ** -e)
        out.append(x)
        exps.append(e)
    return out, exps


@dataclass(eq=False)   # jobs compare by identity (they hold tensors)
class Job:
    code: Any
    xs: List[torch.Tensor]
    grad: bool = False
    arrival: float = 0.0          # seconds on the server clock
    log2_scale: float = 0.0       # inputs were scaled by 2^-log2_scale in total (pow2_rescale)
    id: int = -1
    # results
    value: Optional[torch.Tensor] = None
    grads: Optional[List[torch.Tensor]] = None
    admitted: float = -1.0
    done: float = -1.0
    _event: Any = None
    _slot: int = -1
    _bytes: int = 0
    _work: Optional[float] = None
    reject_reason: str = ""       # "memory" (beyond the budget) or "work" (beyond max_job_flops)

    def scalar(self) -> float:
        """The contraction value as a Python float (mantissa * 2^log2_scale)."""
        return float(self.value.double().cpu()) * 2.0 ** self.log2_scale

    @property
    def latency(self) -> float:
        return self.done - self.arrival


def job_work(job: Job) -> float:
    """Multiply-adds of the job's tree (gradient jobs: three forward passes)."""
    if job._work is None:
        from .planner import contraction_complexity
        sd = get_size_dict(job.code.getixsv(), job.xs)
        job._work = 2.0 ** contraction_complexity(job.code, sd).tc * (3.0 if job.grad else 1.0)
    return job._work


class _Slot:
    """One admission slot: a stream, a context, and a host thread that issues
    the slot's job (a big job's kernel issue must not block the others)."""

    def __init__(self, device):
        self.device = device
        self.stream = torch.cuda.Stream(device=device)
        self.ctx: Optional[_lib.Context] = None
        self.exclusive = False   # the context is a one-job workspace beyond a slot's share
        self.job: Optional[Job] = None
        self.issued = threading.Event()
        self.error: Optional[BaseException] = None
        self.work: "_queue.Queue" = _queue.Queue()
        self.thread = threading.Thread(target=self._run, daemon=True)
        self.thread.start()

    def _run(self):
        torch.cuda.set_device(self.device)
        while True:
            fn = self.work.get()
            if fn is None:
                return
            try:
                fn()
            except BaseException as e:  # reported to the scheduler
                self.error = e
            self.issued.set()


class TNServer:
    """Each slot's workspace is allocated once, at budget / n_slots, on the
    slot's first job and kept until close(): freeing device memory
    synchronises the whole device, which would stall every running job."""

    def __init__(self, n_slots: int = 8, hbm_budget_bytes: float = 150e9, device: int = 0, prec: int = 0,
                 max_job_flops: Optional[float] = None):
        """``max_job_flops`` (optional): jobs whose contraction tree needs more
        multiply-adds than this (the planner's time complexity, gradient jobs
        counted as three forward passes) are rejected at admission, as a
        service would refuse work that holds the device for minutes; None
        admits everything that fits the memory budget."""
        self.device = torch.device("cuda", device)
        self.max_job_flops = max_job_flops
        self.slots = [_Slot(self.device) for _ in range(n_slots)]
        self.budget = int(hbm_budget_bytes)
        self.slot_bytes = int(hbm_budget_bytes) // n_slots
        self.prec = prec
        self.queue: deque = deque()
        self.finished: List[Job] = []
        self.next_id = 0
        self.t0 = time.perf_counter()
        self.rejected: List[Job] = []

    def clock(self) -> float:
        return time.perf_counter() - self.t0

    # ------------------------------------------------------------------
    def submit(self, job: Job) -> int:
        job.id = self.next_id
        self.next_id += 1
        if job.arrival <= 0:
            job.arrival = self.clock()
        self.queue.append(job)
        return job.id

    def _plan(self, job: Job):
        p = _Prepared(job.xs)
        ts = p.tensors
        sd = get_size_dict(job.code.getixsv(), ts)
        code = job.code
        if job.grad and isinstance(code, SlicedEinsum):
            code = code.eins  # gradients run unsliced, as the reference does (src/bp.jl:26-28)
        plan = get_plan(code, sd, p.ome, self.prec)
        need = plan.grad_bytes if job.grad else plan.forward_bytes
        return p, [_f_contig(t) for t in ts], sd, plan, need

    def _work(self, job: Job) -> float:
        return job_work(job)

    def _launch(self, slot: _Slot, job: Job, prepared):
        """Reserve the slot and hand the job's kernel issue to the slot's thread."""
        p, ins, sd, plan, need = prepared
        if slot.ctx is None:
            slot.ctx = _lib.Context(self.device.index, self.slot_bytes)  # MemoryError -> caller
        slot.stream.wait_stream(torch.cuda.current_stream(self.device))  # inputs prepared on this stream
        slot.job = job
        job.admitted = self.clock()
        job._event = None
        slot.issued.clear()
        slot.error = None
        slot.work.put(lambda: self._issue(slot, job, prepared))

    def _launch_exclusive(self, job: Job, prepared):
        """Run one job that exceeds a slot's share: all slot workspaces are
        released, slot 0 gets a context of the job's planned peak bytes, and
        the job runs alone; the context is released when the job retires."""
        need = prepared[4]
        torch.cuda.synchronize(self.device)
        for s in self.slots:
            if s.ctx is not None:
                s.ctx.close()
                s.ctx = None
        slot = self.slots[0]
        slot.ctx = _lib.Context(self.device.index, need)   # MemoryError -> caller
        slot.exclusive = True
        self._launch(slot, job, prepared)

    def _issue(self, slot: _Slot, job: Job, prepared):
        p, ins, sd, plan, need = prepared
        ne = job.code.eins if isinstance(job.code, SlicedEinsum) else job.code
        shape = [sd[l] for l in ne.eins.iy]
        y = _alloc(shape, p.dtype, self.device)
        ptrs = (C.c_void_p * len(ins))(*[t.data_ptr() for t in ins])
        job._keep = (ins, ptrs)
        y.record_stream(slot.stream)
        with torch.cuda.stream(slot.stream):
            if job.grad:
                dxs = [_alloc(t.shape, p.dtype, self.device) for t in ins]
                for d in dxs:
                    d.record_stream(slot.stream)
                dptr = (C.c_void_p * len(dxs))(*[t.data_ptr() for t in dxs])
                check(_lib.load().ome_plan_gradient(slot.ctx.handle, plan.handle,
                                                    C.c_void_p(slot.stream.cuda_stream), ptrs, None,
                                                    y.data_ptr(), dptr))
                job.grads = dxs
            else:
                check(_lib.load().ome_plan_execute(slot.ctx.handle, plan.handle, C.c_void_p(slot.stream.cuda_stream),
                                                   ptrs, y.data_ptr(), _scalar_buf(p.ome, True),
                                                   _scalar_buf(p.ome, False)))
            ev = torch.cuda.Event()
            ev.record(slot.stream)
        job.value = y
        job._bytes = slot.ctx.workspace_bytes
        job._event = ev

    def poll(self) -> int:
        """Retire finished jobs, admit queued ones; returns the number running."""
        now = None
        for s in self.slots:
            if s.job is None or not s.issued.is_set():
                continue
            if s.error is not None:
                err, s.error = s.error, None
                s.job.done = self.clock()
                self.rejected.append(s.job)
                s.job = None
                if s.exclusive:
                    s.stream.synchronize()
                    s.ctx.close()
                    s.ctx = None
                    s.exclusive = False
                if not isinstance(err, MemoryError):
                    raise err
                continue
            if s.job._event.query():
                now = now if now is not None else self.clock()
                s.job.done = now
                self.finished.append(s.job)
                s.job = None
                if s.exclusive:
                    s.ctx.close()   # the job has finished: the workspace is free
                    s.ctx = None
                    s.exclusive = False
        while self.queue:
            free = [s for s in self.slots if s.job is None]
            if not free:
                break
            job = self.queue[0]
            if self.max_job_flops is not None and self._work(job) > self.max_job_flops:
                self.queue.popleft()
                job.done = self.clock()
                job.reject_reason = "work"
                self.rejected.append(job)
                continue
            prepared = self._plan(job)
            need = prepared[4]
            if need > self.budget:
                self.queue.popleft()
                job.done = self.clock()
                job.reject_reason = "memory"
                self.rejected.append(job)
                continue
            running = any(s.job is not None for s in self.slots)
            if need > self.slot_bytes:
                # larger than a slot's share (typically a gradient job, which
                # keeps every intermediate): it waits, in arrival order, until
                # the device is idle, then runs alone in a workspace of its own
                # size taken from the whole budget; the slots' workspaces are
                # released first (freeing memory synchronises the device, which
                # costs nothing once it is idle)
                if running:
                    break
                self.queue.popleft()
                try:
                    self._launch_exclusive(job, prepared)
                except MemoryError:
                    job.done = self.clock()
                    self.rejected.append(job)
                continue
            slot = next((s for s in free if s.ctx is not None), free[0])
            if slot.ctx is None and self.slot_bytes + (256 << 20) > torch.cuda.mem_get_info(self.device)[0]:
                if running:
                    break  # wait for a slot with a workspace (arrival order is kept)
                self.queue.popleft()
                job.done = self.clock()
                self.rejected.append(job)
                continue
            self.queue.popleft()
            try:
                self._launch(slot, job, prepared)
            except MemoryError:
                if running:
                    self.queue.appendleft(job)
                    break
                job.done = self.clock()
                self.rejected.append(job)
        return sum(s.job is not None for s in self.slots)

    def run_trace(self, jobs: Sequence[Job], timeout_s: float = 600.0):
        """Feed jobs at their arrival times (seconds from now) and run until all
        finish; the returned stats() cover this trace only (slots, contexts and
        workspaces carry over from earlier traces)."""
        pending = deque(sorted(jobs, key=lambda j: j.arrival))
        self.finished, self.rejected = [], []
        self.t0 = time.perf_counter()
        while pending or self.queue or any(s.job is not None for s in self.slots):
            now = self.clock()
            while pending and pending[0].arrival <= now:
                self.submit(pending.popleft())
            self.poll()
            if now > timeout_s:
                break
            time.sleep(0.0002)
        return self.stats()

    def close(self):
        """Stop the slot threads and free every slot's workspace; a job error
        that no poll() has reported yet is raised here."""
        pending = None
        for s in self.slots:
            s.work.put(None)
            # no timeout: a slot thread may still be issuing a job's kernels,
            # and its workspace must not be freed under them
            s.thread.join()
            if s.error is not None and pending is None:
                pending = s.error
        for s in self.slots:
            s.stream.synchronize()
            if s.ctx is not None:
                s.ctx.close()
                s.ctx = None
        if pending is not None:
            raise pending

    def stats(self):
        lat = np.array([j.latency for j in self.finished]) if self.finished else np.zeros(1)
        span = max((j.done for j in self.finished), default=0.0) - min((j.arrival for j in self.finished), default=0.0)
        return {"completed": len(self.finished), "rejected": len(self.rejected),
                "rejected_over_work_cap": sum(1 for j in self.rejected if j.reject_reason == "work"),
                "p50_ms": float(np.percentile(lat, 50) * 1e3), "p99_ms": float(np.percentile(lat, 99) * 1e3),
                "jobs_per_s": len(self.finished) / span if span > 0 else 0.0, "makespan_s": span}


class NativeTNServer:
    """The same serving loop inside the library (``ome_server_*`` in
    include/ome_b200.h): slots, issue threads, admission by planned peak
    bytes, exclusive runs of jobs above a slot's share and the work cap are
    C++; Python only plans jobs, allocates their outputs and polls.  This is
    the interface a Julia service binds (no Python on its path); ``TNServer``
    above is the Python rendering of the same rules."""

    def __init__(self, n_slots: int = 8, hbm_budget_bytes: float = 150e9, device: int = 0, prec: int = 0,
                 max_job_flops: Optional[float] = None):
        self.device = torch.device("cuda", device)
        self.prec = prec
        self.max_job_flops = max_job_flops
        h = C.c_void_p()
        check(_lib.load().ome_server_create(device, n_slots, int(hbm_budget_bytes),
                                            float(max_job_flops or 0.0), C.byref(h)))
        self.handle = h
        self._live = {}            # job id -> (job, buffers the library reads or writes)
        self.finished: List[Job] = []
        self.rejected: List[Job] = []
        self._t0 = None            # server clock at the start of run_trace (None: report the library's times)

    def submit(self, job: Job) -> int:
        """Plan the job, allocate its outputs and queue it; the job's kernels
        run after the work queued on the current stream (the legacy default
        stream too: its handle 0 is passed as NULL, which the library reads as
        that stream)."""
        p = _Prepared(job.xs)
        ts = [_f_contig(t) for t in p.tensors]
        sd = get_size_dict(job.code.getixsv(), ts)
        code = job.code
        if job.grad and isinstance(code, SlicedEinsum):
            code = code.eins   # gradients run unsliced, as the reference does (src/bp.jl:26-28)
        plan = get_plan(code, sd, p.ome, self.prec)
        ne = code.eins if isinstance(code, SlicedEinsum) else code
        y = _alloc([sd[l] for l in ne.eins.iy], p.dtype, self.device)
        ptrs = (C.c_void_p * len(ts))(*[t.data_ptr() for t in ts])
        dxs = dptr = None
        if job.grad:
            dxs = [_alloc(t.shape, p.dtype, self.device) for t in ts]
            dptr = (C.c_void_p * len(dxs))(*[d.data_ptr() for d in dxs])
        work = job_work(job) if self.max_job_flops is not None else 0.0
        jid = C.c_int64()
        check(_lib.load().ome_server_submit(self.handle, plan.handle, len(ts), ptrs, y.data_ptr(), dptr, work,
                                            C.c_void_p(torch.cuda.current_stream(self.device).cuda_stream),
                                            C.byref(jid)))
        job.id = jid.value
        job.value, job.grads = y, dxs
        self._live[job.id] = (job, (plan, ts, ptrs, y, dxs, dptr))
        return job.id

    def poll(self) -> int:
        """Retire finished jobs and admit queued ones; returns the number running."""
        recs = (_lib.ServerJob * 64)()
        n, running = C.c_int32(), C.c_int32()
        while True:
            check(_lib.load().ome_server_poll(self.handle, 64, recs, C.byref(n), C.byref(running)))
            for r in recs[:n.value]:
                job, _ = self._live.pop(r.id)
                if self._t0 is None:
                    job.arrival, job.admitted, job.done = r.arrival_s, r.admitted_s, r.done_s
                else:   # trace time: latency from the job's nominal arrival, as TNServer reports it
                    job.admitted, job.done = r.admitted_s - self._t0, r.done_s - self._t0
                if r.outcome == _lib.JOB_COMPLETED:
                    self.finished.append(job)
                else:
                    job.reject_reason = {_lib.JOB_REJECTED_MEMORY: "memory", _lib.JOB_REJECTED_WORK: "work"}.get(
                        r.outcome, "failed")
                    job.value = job.grads = None
                    self.rejected.append(job)
            if n.value < 64:
                return running.value

    def run_trace(self, jobs: Sequence[Job], timeout_s: float = 600.0):
        """Submit jobs at their arrival times (seconds from now) and poll until
        all have finished; job times are then seconds from the trace start,
        and latency runs from each job's nominal arrival.  Returns the
        library's counters (which also cover earlier traces)."""
        pending = deque(sorted(jobs, key=lambda j: j.arrival))
        c = C.c_double()
        check(_lib.load().ome_server_clock(self.handle, C.byref(c)))
        self._t0 = c.value
        t0 = time.perf_counter()
        try:
            while pending or self._live:
                now = time.perf_counter() - t0
                while pending and pending[0].arrival <= now:
                    self.submit(pending.popleft())
                    self.poll()   # admission keeps up while a burst of arrivals is planned
                self.poll()
                if now > timeout_s:
                    break
                time.sleep(0.0002)
        finally:
            self._t0 = None
        return self.stats()

    def stats(self):
        st = _lib.ServingStats()
        check(_lib.load().ome_server_stats(self.handle, C.byref(st)))
        return {k: getattr(st, k) for k, _ in _lib.ServingStats._fields_}

    def close(self):
        """Wait for every issued job and free the slots (queued jobs are dropped)."""
        if self.handle:
            _lib.load().ome_server_destroy(self.handle)
            self.handle = None
        self._live.clear()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
