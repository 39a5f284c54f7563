// Native serving loop for whole contraction-tree jobs (continuous batching),
// behind the C ABI: ome_server_create / submit / poll / stats / destroy.
//
// The reference serves nothing itself; a Julia service would call
// einsum(::NestedEinsum) or cost_and_gradient (src/einsequence.jl:270-287,
// src/bp.jl:122-130) once per request.  This server keeps a fixed number of
// slots on one device.  A slot owns a CUDA stream, a host issue thread and a
// library context whose workspace is the slot's share of the HBM budget,
// allocated on the slot's first job and kept (freeing device memory
// synchronises the whole device).  Jobs are admitted in arrival order when a
// slot is free and the plan's peak workspace bytes (ome_plan_peak_bytes) fit a
// share; a job above a share but within the whole budget waits until every
// slot is idle and then runs alone in a workspace of its own size (the slots'
// workspaces are released first); jobs above the budget, or above the optional
// work cap, are rejected at admission.  A slot's thread issues the job's
// kernels (ome_plan_execute, or ome_plan_gradient for gradient jobs, which run
// unsliced as src/bp.jl:26-28 does) so that a large job's host-side issue never
// blocks admission; completion is the job's event on the slot's stream,
// observed by ome_server_poll.  All of a job's buffers belong to the caller and
// must stay valid until poll reports the job.
#include <string.h>

#include <algorithm>
#include <atomic>
#include <chrono>
#include <condition_variable>
#include <deque>
#include <mutex>
#include <string>
#include <thread>
#include <vector>

#include "dispatch.h"

using namespace ome;

namespace {

struct SrvJob {
  int64_t id = 0;
  ome_plan* plan = nullptr;
  std::vector<const void*> inputs;
  void* y = nullptr;
  std::vector<void*> dxs;        // empty: a value job
  double work = 0;               // multiply-adds (for the work cap)
  cudaEvent_t ready = nullptr;   // the caller's stream at submit (inputs and outputs ready)
  cudaEvent_t done_ev = nullptr;
  double arrival = 0, admitted = -1, done = -1;
  int status = OME_OK;
  int outcome = 0;               // ome_job_outcome
  std::string msg;
};

struct SrvSlot {
  cudaStream_t stream = nullptr;
  ome_ctx* ctx = nullptr;
  bool exclusive = false;        // the context is a one-job workspace beyond a slot's share
  SrvJob* job = nullptr;         // the job the slot runs (owned by the poll side)
  std::thread thr;
  std::mutex m;
  std::condition_variable cv;
  SrvJob* pending = nullptr;     // handed to the issue thread
  bool stop = false;
  std::atomic<int> issued{0};    // the issue thread has issued (or failed to issue) `job`
};

// Restores the calling thread's current device on scope exit.
struct DeviceScope {
  int old = -1;
  explicit DeviceScope(int dev) {
    cudaGetDevice(&old);
    if (old != dev) cudaSetDevice(dev);
  }
  ~DeviceScope() {
    int cur = -1;
    cudaGetDevice(&cur);
    if (old >= 0 && cur != old) cudaSetDevice(old);
  }
};

}  // namespace

struct ome_server {
  int device = 0;
  size_t budget = 0, slot_bytes = 0;
  double max_work = 0;           // <= 0: no work cap
  std::vector<SrvSlot*> slots;
  std::deque<SrvJob*> queue;
  std::deque<SrvJob*> retired;   // finished, failed or rejected; not yet returned by poll
  std::vector<double> lat;       // latencies (s) of completed jobs
  double first_arrival = 1e300, last_done = 0;
  int64_t next_id = 0, submitted = 0, completed = 0, failed = 0, rej_memory = 0, rej_work = 0;
  std::mutex mu;
  std::chrono::steady_clock::time_point t0;
  double clock() const {
    return std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
  }
};

namespace {

void free_job(SrvJob* j) {
  if (j->ready) cudaEventDestroy(j->ready);
  if (j->done_ev) cudaEventDestroy(j->done_ev);
  delete j;
}

// Issue thread of one slot: waits for a job, issues its kernels on the slot's
// stream and records its completion event.
void slot_main(ome_server* srv, SrvSlot* sl) {
  cudaSetDevice(srv->device);
  for (;;) {
    SrvJob* j = nullptr;
    {
      std::unique_lock<std::mutex> lk(sl->m);
      sl->cv.wait(lk, [&] { return sl->stop || sl->pending != nullptr; });
      if (!sl->pending) return;   // stop requested and nothing left to issue
      j = sl->pending;
      sl->pending = nullptr;
    }
    int rc = OME_OK;
    if (j->ready) {
      const cudaError_t e = cudaStreamWaitEvent(sl->stream, j->ready, 0);
      if (e != cudaSuccess) rc = cuda_err(e, "waiting for the job's inputs");
    }
    if (rc == OME_OK) {
      if (j->dxs.empty()) {
        const ome_dtype dt = plan_dtype(j->plan);
        const Scalar one = scalar_one(dt), zero = scalar_zero(dt);
        rc = ome_plan_execute(sl->ctx, j->plan, sl->stream, j->inputs.data(), j->y, one.b, zero.b);
      } else {
        rc = ome_plan_gradient(sl->ctx, j->plan, sl->stream, j->inputs.data(), nullptr, j->y, j->dxs.data());
      }
    }
    if (rc == OME_OK) {
      const cudaError_t e = cudaEventRecord(j->done_ev, sl->stream);
      if (e != cudaSuccess) rc = cuda_err(e, "recording the job's completion");
    }
    if (rc != OME_OK) {
      j->status = rc;
      j->msg = ome_last_error();
    }
    sl->issued.store(1, std::memory_order_release);
  }
}

void release_slot_ctx(SrvSlot* sl) {
  if (sl->ctx) {
    cudaStreamSynchronize(sl->stream);
    ome_ctx_destroy(sl->ctx);
    sl->ctx = nullptr;
  }
  sl->exclusive = false;
}

void retire_one(ome_server* s, SrvJob* j) {
  s->retired.push_back(j);
  if (j->outcome == OME_JOB_COMPLETED) {
    ++s->completed;
    s->lat.push_back(j->done - j->arrival);
    s->first_arrival = std::min(s->first_arrival, j->arrival);
    s->last_done = std::max(s->last_done, j->done);
  } else if (j->outcome == OME_JOB_FAILED) {
    ++s->failed;
  } else if (j->outcome == OME_JOB_REJECTED_MEMORY) {
    ++s->rej_memory;
  } else {
    ++s->rej_work;
  }
}

void reject(ome_server* s, SrvJob* j, int outcome) {
  j->outcome = outcome;
  j->status = OME_OUT_OF_MEMORY;
  j->done = s->clock();
  retire_one(s, j);
}

// Finished (or failed) jobs leave their slots.
void retire(ome_server* s) {
  for (SrvSlot* sl : s->slots) {
    SrvJob* j = sl->job;
    if (!j || !sl->issued.load(std::memory_order_acquire)) continue;
    if (j->status == OME_OK) {
      const cudaError_t e = cudaEventQuery(j->done_ev);
      if (e == cudaErrorNotReady) continue;
      if (e != cudaSuccess) {
        j->status = OME_CUDA_ERROR;
        j->msg = cudaGetErrorString(e);
      }
    }
    // a job whose issue failed part-way may still have kernels queued: they
    // finish before the caller hears of the job (and may free its buffers)
    if (j->status != OME_OK) cudaStreamSynchronize(sl->stream);
    j->done = s->clock();
    j->outcome = j->status == OME_OK ? OME_JOB_COMPLETED : OME_JOB_FAILED;
    sl->job = nullptr;
    if (sl->exclusive) release_slot_ctx(sl);   // the one-job workspace is free again
    retire_one(s, j);
  }
}

void launch(SrvSlot* sl, SrvJob* j, double now) {
  sl->job = j;
  j->admitted = now;
  sl->issued.store(0, std::memory_order_relaxed);
  {
    std::lock_guard<std::mutex> lk(sl->m);
    sl->pending = j;
  }
  sl->cv.notify_one();
}

// Admit queued jobs in arrival order while slots are free.
void admit(ome_server* s) {
  while (!s->queue.empty()) {
    std::vector<SrvSlot*> free;
    bool running = false;
    for (SrvSlot* sl : s->slots) {
      if (sl->job) running = true;
      else free.push_back(sl);
    }
    if (free.empty()) return;
    SrvJob* j = s->queue.front();
    if (s->max_work > 0 && j->work > s->max_work) {
      s->queue.pop_front();
      reject(s, j, OME_JOB_REJECTED_WORK);
      continue;
    }
    size_t fwd = 0, grad = 0;
    ome_plan_peak_bytes(j->plan, &fwd, &grad);
    const size_t need = j->dxs.empty() ? fwd : grad;
    if (need > s->budget) {
      s->queue.pop_front();
      reject(s, j, OME_JOB_REJECTED_MEMORY);
      continue;
    }
    if (need > s->slot_bytes) {
      // above a slot's share: wait (keeping arrival order) until the device
      // is idle, then run alone in a workspace of the job's own size
      if (running) return;
      s->queue.pop_front();
      for (SrvSlot* sl : s->slots) release_slot_ctx(sl);
      SrvSlot* sl = s->slots[0];
      if (ome_ctx_create(s->device, need, &sl->ctx) != OME_OK) {
        sl->ctx = nullptr;
        reject(s, j, OME_JOB_REJECTED_MEMORY);
        continue;
      }
      sl->exclusive = true;
      launch(sl, j, s->clock());
      continue;
    }
    SrvSlot* sl = free[0];
    for (SrvSlot* f : free)
      if (f->ctx) {
        sl = f;
        break;
      }
    if (!sl->ctx) {
      size_t fr = 0, tot = 0;
      cudaMemGetInfo(&fr, &tot);
      if (s->slot_bytes + (256u << 20) > fr || ome_ctx_create(s->device, s->slot_bytes, &sl->ctx) != OME_OK) {
        sl->ctx = nullptr;
        if (running) return;   // wait for a slot that has a workspace
        s->queue.pop_front();
        reject(s, j, OME_JOB_REJECTED_MEMORY);
        continue;
      }
    }
    s->queue.pop_front();
    launch(sl, j, s->clock());
  }
}

double percentile(std::vector<double> v, double q) {
  if (v.empty()) return 0.0;
  std::sort(v.begin(), v.end());
  const double pos = q / 100.0 * (double)(v.size() - 1);
  const size_t i = (size_t)pos;
  const double f = pos - (double)i;
  return i + 1 < v.size() ? v[i] * (1.0 - f) + v[i + 1] * f : v[i];
}

}  // namespace

extern "C" {

int ome_server_create(int device, int32_t n_slots, size_t hbm_budget_bytes, double max_job_work, ome_server** out) {
  if (!out || n_slots < 1 || n_slots > 256 || hbm_budget_bytes == 0)
    return set_err(OME_INVALID_ARGUMENT, "bad server arguments");
  *out = nullptr;
  DeviceScope ds(device);
  auto s = new ome_server();
  s->device = device;
  s->budget = hbm_budget_bytes;
  s->slot_bytes = hbm_budget_bytes / (size_t)n_slots;
  s->max_work = max_job_work;
  s->t0 = std::chrono::steady_clock::now();
  for (int i = 0; i < n_slots; ++i) {
    auto sl = new SrvSlot();
    const cudaError_t e = cudaStreamCreateWithFlags(&sl->stream, cudaStreamNonBlocking);
    if (e != cudaSuccess) {
      delete sl;
      ome_server_destroy(s);
      return cuda_err(e, "server stream");
    }
    s->slots.push_back(sl);
    sl->thr = std::thread(slot_main, s, sl);
  }
  *out = s;
  return OME_OK;
}

int ome_server_submit(ome_server* s, ome_plan* plan, int32_t ninputs, const void* const* inputs, void* y,
                      void* const* dxs, double work, void* input_stream, int64_t* job_id) {
  if (!s || !plan || !inputs || !y || !job_id) return set_err(OME_INVALID_ARGUMENT, "NULL argument");
  if (ninputs != plan_ninputs(plan))
    return set_err(OME_INVALID_ARGUMENT, "the plan has %d inputs, %d given", plan_ninputs(plan), ninputs);
  DeviceScope ds(s->device);
  auto j = new SrvJob();
  j->plan = plan;
  j->inputs.assign(inputs, inputs + ninputs);
  j->y = y;
  if (dxs) j->dxs.assign(dxs, dxs + ninputs);
  j->work = work;
  cudaError_t e = cudaEventCreateWithFlags(&j->done_ev, cudaEventDisableTiming);
  // the job's kernels run after the work already queued on input_stream (NULL
  // is the legacy default stream, as everywhere in CUDA): the slots' streams
  // are non-blocking, so without this event they would not wait for it
  if (e == cudaSuccess) e = cudaEventCreateWithFlags(&j->ready, cudaEventDisableTiming);
  if (e == cudaSuccess) e = cudaEventRecord(j->ready, static_cast<cudaStream_t>(input_stream));
  if (e != cudaSuccess) {
    free_job(j);
    return cuda_err(e, "job events");
  }
  std::lock_guard<std::mutex> lk(s->mu);
  j->id = s->next_id++;
  j->arrival = s->clock();
  s->queue.push_back(j);
  ++s->submitted;
  *job_id = j->id;
  return OME_OK;
}

int ome_server_poll(ome_server* s, int32_t max_jobs, ome_server_job* jobs, int32_t* n_jobs, int32_t* running) {
  if (!s) return set_err(OME_INVALID_ARGUMENT, "NULL server");
  DeviceScope ds(s->device);
  std::lock_guard<std::mutex> lk(s->mu);
  retire(s);
  admit(s);
  int32_t n = 0;
  bool reported = false;
  while (jobs && n < max_jobs && !s->retired.empty()) {
    SrvJob* j = s->retired.front();
    s->retired.pop_front();
    ome_server_job& r = jobs[n++];
    r.id = j->id;
    r.outcome = j->outcome;
    r.status = j->status;
    r.arrival_s = j->arrival;
    r.admitted_s = j->admitted;
    r.done_s = j->done;
    if (j->outcome == OME_JOB_FAILED && !reported) {   // the first failure's message, for ome_last_error
      set_err(j->status, "job %lld: %s", (long long)j->id, j->msg.c_str());
      reported = true;
    }
    free_job(j);
  }
  if (n_jobs) *n_jobs = n;
  if (running) {
    int32_t r = 0;
    for (SrvSlot* sl : s->slots) r += sl->job != nullptr;
    *running = r;
  }
  return OME_OK;
}

int ome_server_stats(ome_server* s, ome_serving_stats* st) {
  if (!s || !st) return set_err(OME_INVALID_ARGUMENT, "NULL argument");
  std::lock_guard<std::mutex> lk(s->mu);
  memset(st, 0, sizeof(*st));
  st->submitted = s->submitted;
  st->completed = s->completed;
  st->failed = s->failed;
  st->rejected_memory = s->rej_memory;
  st->rejected_work = s->rej_work;
  st->queued = (int64_t)s->queue.size();
  for (SrvSlot* sl : s->slots) st->running += sl->job != nullptr;
  st->p50_ms = percentile(s->lat, 50) * 1e3;
  st->p90_ms = percentile(s->lat, 90) * 1e3;
  st->p99_ms = percentile(s->lat, 99) * 1e3;
  const double span = s->completed ? s->last_done - s->first_arrival : 0.0;
  st->makespan_s = span;
  st->jobs_per_s = span > 0 ? (double)s->completed / span : 0.0;
  return OME_OK;
}

int ome_server_clock(const ome_server* s, double* seconds) {
  if (!s || !seconds) return set_err(OME_INVALID_ARGUMENT, "NULL argument");
  *seconds = s->clock();
  return OME_OK;
}

int ome_server_destroy(ome_server* s) {
  if (!s) return OME_OK;
  DeviceScope ds(s->device);
  for (SrvSlot* sl : s->slots) {
    {
      std::lock_guard<std::mutex> lk(sl->m);
      sl->stop = true;
    }
    sl->cv.notify_one();
  }
  // no time limit: a slot thread may still be issuing kernels into its
  // workspace, which must not be freed under them
  for (SrvSlot* sl : s->slots)
    if (sl->thr.joinable()) sl->thr.join();
  for (SrvSlot* sl : s->slots) {
    if (sl->stream) cudaStreamSynchronize(sl->stream);
    if (sl->ctx) ome_ctx_destroy(sl->ctx);
    if (sl->stream) cudaStreamDestroy(sl->stream);
    if (sl->job) free_job(sl->job);
    delete sl;
  }
  for (SrvJob* j : s->queue) free_job(j);
  for (SrvJob* j : s->retired) free_job(j);
  delete s;
  return OME_OK;
}

}  // extern "C"
