/*
 * ome_b200.h -- C ABI of libomeb200.so, a B200 (sm_100a) einsum engine that
 * plugs in behind OMEinsum.jl's backend registry.
 *
 * Plain C: pointers, sizes and int status codes.  No exceptions cross this
 * boundary and the library never aborts the process.  Every compute entry
 * point takes an explicit CUDA stream (passed as void*, i.e. a cudaStream_t)
 * and is asynchronous on it.
 *
 * Conventions (those of OMEinsum.jl):
 *   - tensors are strided views; dims[d] is the extent of dimension d and
 *     strides[d] its step in ELEMENTS (NULL strides = column-major contiguous,
 *     Julia's layout: dimension 1 fastest);
 *   - labels are int32 (Julia Char code points or Int labels);
 *   - y <- sy*y + sx*f(xs); sx, sy point to one value of the call's dtype;
 *     sy equal to the algebra's zero means "overwrite" (y is not read), as in
 *     the iszero(sy) branch of @addmul! (src/utils.jl:25-35);
 *   - all inputs and the output share one dtype (the caller converts mixed
 *     eltypes first, like CUDAExt.jl:116 / align_eltypes, src/utils.jl:108-115);
 *   - the output must not alias an input.
 */
#ifndef OME_B200_H
#define OME_B200_H

#include <stddef.h>
#include <stdint.h>

#if defined(__GNUC__)
#define OME_API __attribute__((visibility("default")))
#else
#define OME_API
#endif

#ifdef __cplusplus
extern "C" {
#endif

/* Status codes.  Mapping to Julia exceptions on the Julia side:
 * INVALID_ARGUMENT -> ArgumentError, DIMENSION_MISMATCH -> DimensionMismatch
 * (src/interfaces.jl:78-88,100), everything else -> ErrorException. */
typedef enum {
  OME_OK = 0,
  OME_INVALID_ARGUMENT = 1,
  OME_DIMENSION_MISMATCH = 2,
  OME_UNSUPPORTED = 3,
  OME_OUT_OF_MEMORY = 4,
  OME_TIMEOUT = 5,      /* a bounded device-side wait gave up */
  OME_CUDA_ERROR = 6
} ome_status;

/* Element types.  BOOL is one byte per element, contracted as OR-AND.
 * TROP_F32/TROP_F64 are TropicalNumbers.jl Tropical{Float32/Float64}:
 * (+) = max, (*) = +, zero = -Inf, one = 0.  Complex types are interleaved
 * (re, im) pairs, Julia's ComplexF32/ComplexF64. */
typedef enum {
  OME_F32 = 0,
  OME_F64 = 1,
  OME_C32 = 2,
  OME_C64 = 3,
  OME_I64 = 4,
  OME_BOOL = 5,
  OME_TROP_F32 = 6,
  OME_TROP_F64 = 7
} ome_dtype;

/* Precision mode for F32 contractions (other dtypes ignore it).
 * GEMM-shaped F32 contractions run on the tensor cores as split BF16
 * products accumulated in FP32: each value x = t0 + t1 (+ t2) in bf16.
 * OME_PREC_AUTO   : BF16x6 (3 terms, 6 MMAs per K step; products exact to
 *                   about 2^-24, i.e. FP32-faithful).
 * OME_PREC_FP32   : CUDA-core FP32 FMA everywhere (the plain GPU path).
 * OME_PREC_BF16X3 : 2 terms, 3 MMAs (hi*hi + hi*lo + lo*hi); products exact
 *                   to about 2^-16 -- twice as fast, not FP32-accurate.
 * OME_PREC_BF16X6 : same as AUTO. */
typedef enum { OME_PREC_AUTO = 0, OME_PREC_FP32 = 1, OME_PREC_BF16X3 = 2, OME_PREC_BF16X6 = 3 } ome_prec;

typedef struct {
  void* data;
  int32_t ndim;
  const int64_t* dims;
  const int64_t* strides; /* elements; NULL = column-major contiguous */
  const int32_t* labels;  /* ndim labels */
} ome_tensor;

typedef struct ome_ctx ome_ctx;
typedef struct ome_plan ome_plan;

/* Library / context ------------------------------------------------------- */

/* ABI version of this header. */
OME_API int ome_version(void);

/* Number of kernels this library has launched since it was loaded (all
 * threads); lets a caller count device launches in a timed region. */
OME_API unsigned long long ome_launch_count(void);

/* Synchronise `stream` (a cudaStream_t, NULL = legacy default stream), then
 * report whether any kernel of this library gave up a bounded device-side
 * wait since the last call: OME_TIMEOUT if so (the flag is cleared), else
 * OME_OK.  Kernels never spin unboundedly; a wait that gives up marks its
 * result invalid through this flag instead of trapping. */
OME_API int ome_device_status(void* stream);

/* Failure-path self-test of the bounded device waits (no counterpart in the
 * reference; the reference's kernels have no device-side waits): launches on
 * `stream` one block whose thread waits on a shared-memory mbarrier that
 * nothing arrives on, gives up after `wait_ns` nanoseconds of %globaltimer
 * (clamped to [1 us, 1 s]), records the timeout flag exactly as a stalled
 * tensor-core kernel would, and returns.  The next ome_device_status on the
 * stream reports OME_TIMEOUT once; the context stays usable. */
OME_API int ome_selftest_wait_timeout(void* stream, uint64_t wait_ns);

/* Kernel timing (diagnostic; no counterpart in the reference).  While
 * enabled, the main kernel of every dispatch (the GEMM of a binary
 * contraction, the transpose of a permutation, the reduction of a sum, the
 * index kernel of loop_einsum) is bracketed by CUDA events on its own stream,
 * without synchronising.  ome_kernel_timing(n) with n > 0 starts the record
 * (cleared) after creating n event pairs up front, so that recording n
 * kernels creates no event; 0 stops it.  ome_kernel_times synchronises on the
 * recorded events
 * and writes up to `max` durations (ms, launch order) and kernel names
 * (static strings) to ms / names, and their number to *count. */
OME_API int ome_kernel_timing(int enable);
OME_API int ome_kernel_times(int32_t max, float* ms, const char** names, int32_t* count);

/* Message of the last failed call on this host thread ("" if none). */
OME_API const char* ome_last_error(void);

/* Create a context on `device` with a device workspace of `workspace_bytes`
 * (intermediates of plans and scratch of single calls).  Replaces the per-
 * intermediate CUDA.jl allocations (ext/CUDAExt.jl:34-47, :129-131).
 * A large FP32 GEMM whose BF16 operand terms do not fit the workspace puts
 * them in a second buffer that the context grows on demand (not during
 * stream capture, at most a quarter of the free device memory; growing
 * synchronises the device) and frees in ome_ctx_destroy. */
OME_API int ome_ctx_create(int device, size_t workspace_bytes, ome_ctx** out);
OME_API int ome_ctx_destroy(ome_ctx* ctx);
OME_API int ome_ctx_workspace_bytes(const ome_ctx* ctx, size_t* out);

/* Single contractions ------------------------------------------------------ */

/* einsum!(ixs, iy, xs, y, sx, sy, size_dict) for any number of inputs.
 * Replaces: the backend dispatch override ext/CUDAExt.jl:181-192 (binary),
 * the unary einsum! src/einsum.jl:84-101 with its rules src/unaryrules.jl,
 * and the n-ary fallback src/einsum.jl:47-50 -> loop_einsum!.
 * Dispatch: 1 input -> fused unary kernels; 2 inputs -> strided GEMM (no
 * permuted copies) or the index kernel; >= 3 inputs -> the index kernel. */
OME_API int ome_einsum(ome_ctx* ctx, void* stream, ome_dtype dtype, int32_t ninputs,
               const ome_tensor* xs, const ome_tensor* y, const void* sx,
               const void* sy, int32_t prec);

/* loop_einsum!(ixs, iy, xs, y, sx, sy, size_dict): the generic index-iterating
 * kernel regardless of shape.  Replaces src/loop_einsum.jl:21-45 and its GPU
 * form ext/CUDAExt.jl:60-113 (mapreducedim! over EinArray + expanddims!). */
OME_API int ome_loop_einsum(ome_ctx* ctx, void* stream, ome_dtype dtype, int32_t ninputs,
                    const ome_tensor* xs, const ome_tensor* y, const void* sx,
                    const void* sy);

/* einsum_grad(ixs, xs, iy, size_dict, dy, i) (src/autodiff.jl:24-30): the
 * gradient of einsum(ixs -> iy)(xs) with respect to input i (0-based):
 * dx <- conj(einsum((ixs with iy in place of ixs[i]) -> ixs[i])(xs with
 * conj(dy) in place of xs[i])).  dy carries iy as its labels; dx must have
 * xs[i]'s labels and extents (xs[i].data is not read and may be NULL).
 * Replaces the per-input pullback of rrule(einsum) (src/autodiff.jl:35-44). */
OME_API int ome_einsum_grad(ome_ctx* ctx, void* stream, ome_dtype dtype, int32_t ninputs,
                            const ome_tensor* xs, const ome_tensor* dy, int32_t i,
                            const ome_tensor* dx, int32_t prec);

/* Contraction trees (NestedEinsum / SlicedEinsum) -------------------------- */

/* A tree is given in post-order, root last.  Node j has node_nargs[j]
 * children; its child references are the next node_nargs[j] entries of
 * node_args: r >= 0 is node r, r < 0 is input tensor (-r - 1).  Its output
 * labels are the next node_niy[j] entries of node_iy.  The labels of input
 * tensor t are the next input_nlabels[t] entries of input_labels.  Extents:
 * label_ids[i] has extent label_extents[i].  Sliced labels (SlicedEinsum,
 * src/slicing.jl:10-13) are iterated in column-major order (first fastest).
 * Replaces einsum!/einsum(::NestedEinsum) (src/einsequence.jl:270-287,
 * ext/CUDAExt.jl:121-147) and the SlicedEinsum executors
 * (src/slicing.jl:112-137). */
OME_API int ome_plan_create(ome_ctx* ctx, ome_dtype dtype, int32_t ninputs,
                    const int32_t* input_nlabels, const int32_t* input_labels,
                    int32_t nnodes, const int32_t* node_nargs,
                    const int32_t* node_args, const int32_t* node_niy,
                    const int32_t* node_iy, int32_t nlabels,
                    const int32_t* label_ids, const int64_t* label_extents,
                    int32_t nsliced, const int32_t* sliced_labels, int32_t prec,
                    ome_plan** out);
OME_API int ome_plan_destroy(ome_plan* plan);

/* Peak workspace bytes the plan needs (forward only / forward+gradient). */
OME_API int ome_plan_peak_bytes(const ome_plan* plan, size_t* forward_bytes, size_t* grad_bytes);

/* Evaluate the tree: y <- sy*y + sx*tree(inputs).  inputs[t] are column-major
 * contiguous device buffers; y is column-major contiguous.  With slices, the
 * cross-slice sum is accumulated in FP64 for F32/F64 (C64 for C32). */
OME_API int ome_plan_execute(ome_ctx* ctx, ome_plan* plan, void* stream,
                     const void* const* inputs, void* y, const void* sx,
                     const void* sy);

/* Slice sharding (the slice loop of src/slicing.jl:118-137 split over ranks;
 * replaces the host-staged examples/slicing_multigpu.jl:54-75).  The slice
 * index space 0..nslices-1 is CartesianIndices order over the sliced labels,
 * first label fastest (src/slicing.jl:37-50).
 *
 * ome_plan_slice_count: number of slices (1 for an unsliced plan).
 * ome_plan_partial_info: the partial a range of slices produces -- dtype
 *   (F64 for F32/F64 plans with slices, C64 for C32 ones, the plan's dtype
 *   otherwise), its bytes (the full output, column-major contiguous) and how
 *   partials of different ranks combine: op 0 = elementwise sum, op 1 =
 *   elementwise max (Tropical max-plus, Bool or-and).
 * ome_plan_execute_slices: partial <- (+) over slices [begin, end) of the
 *   tree value, each at its sliced output positions (the algebra's zero
 *   elsewhere); sx/sy are not applied.
 * ome_plan_finish: y <- sy*y + sx*partial, rounded to the plan's dtype.
 * execute_slices(0, nslices) followed by finish equals ome_plan_execute. */
OME_API int ome_plan_slice_count(const ome_plan* plan, int64_t* nslices);
OME_API int ome_plan_partial_info(const ome_plan* plan, int* partial_dtype, size_t* partial_bytes,
                                  int* reduce_op);
OME_API int ome_plan_execute_slices(ome_ctx* ctx, ome_plan* plan, void* stream,
                                    const void* const* inputs, int64_t slice_begin,
                                    int64_t slice_end, void* partial);
OME_API int ome_plan_finish(ome_ctx* ctx, ome_plan* plan, void* stream, const void* partial,
                            void* y, const void* sx, const void* sy);

/* cost_and_gradient (src/bp.jl:122-130): forward with every intermediate kept
 * in the workspace, then einsum_grad (src/autodiff.jl:24-30) per node.
 * dy: the output cotangent (NULL = ones, requires a scalar output).  y
 * receives the forward value, dxs[t] the gradient of input t (column-major,
 * same shape as the input).  Slicing is not used for gradients, as in the
 * reference (src/bp.jl:26-28). */
OME_API int ome_plan_gradient(ome_ctx* ctx, ome_plan* plan, void* stream,
                      const void* const* inputs, const void* dy, void* y,
                      void* const* dxs);

/* Contraction-order search (host) ------------------------------------------
 *
 * TreeSA: simulated annealing over binary contraction trees, the method
 * OMEinsum re-exports from OMEinsumContractionOrders (src/contractionorder.jl:
 * 30-41).  ntensors tensors with nlabels[t] label ids each (concatenated in
 * `labels`, ids 0..nids-1, log2 extents in log2_sizes), output labels
 * out_labels.  init_tree / out_tree: ntensors-1 internal nodes in post-order,
 * two child refs each (r >= 0 internal node, r < 0 input tensor -r-1).
 * Moves rewrite (A, (B, C)) into ((A, B), C) or ((A, C), B); a move is
 * accepted with probability min(1, exp(-beta * dcost)), beta from beta_start
 * to beta_stop in steps of beta_step, niters sweeps over the nodes per beta,
 * cost = log2(sum 2^tc + rw_weight * 2^rw) + sc_weight * sum max(0, sc -
 * sc_target) over contractions.  ntrials independent trials (host threads,
 * seeds derived from `seed`); the best tree is returned with its (tc, sc, rw)
 * in log2 (out_complexity, 3 doubles; may be NULL). */
OME_API int ome_treesa(int32_t ntensors, const int32_t* nlabels, const int32_t* labels, int32_t nout,
                       const int32_t* out_labels, int32_t nids, const double* log2_sizes,
                       const int32_t* init_tree, double sc_target, double sc_weight, double rw_weight,
                       double beta_start, double beta_step, double beta_stop, int32_t niters,
                       int32_t ntrials, uint64_t seed, int32_t* out_tree, double* out_complexity);

/* Greedy pairwise order (OMEinsumContractionOrders' GreedyMethod): contract the
 * pair of live tensors that share a label (the two smallest when none do)
 * minimising size(result) - alpha * (size(a) + size(b)); ties at random, or
 * with temperature > 0 a pair drawn with Boltzmann weights.  nrepeat runs
 * (seeded from `seed`); the one with the smallest (tc, sc) is written to
 * out_tree in the ome_treesa format, its (tc, sc, rw) to out_complexity. */
OME_API int ome_greedy(int32_t ntensors, const int32_t* nlabels, const int32_t* labels, int32_t nout,
                       const int32_t* out_labels, int32_t nids, const double* log2_sizes, double alpha,
                       double temperature, int32_t nrepeat, uint64_t seed, int32_t* out_tree,
                       double* out_complexity);

/* Greedy slicer (the slicing loop of src/slicing.jl's SlicedEinsum with
 * OMEinsumContractionOrders' slicers as the reference uses them): slice, one
 * at a time, the label whose removal gives the smallest (space complexity,
 * time complexity + its log2 extent) until the largest intermediate of
 * `tree` (ome_treesa format) has at most 2^sc_target elements or max_slices
 * labels are sliced; `forbidden` (NULL or nids flags) excludes labels.  The
 * sliced label ids go to out_sliced in order, their number to *out_count. */
OME_API int ome_slice_greedy(int32_t ntensors, const int32_t* nlabels, const int32_t* labels, int32_t nout,
                             const int32_t* out_labels, int32_t nids, const double* log2_sizes,
                             const int32_t* tree, double sc_target, int32_t max_slices,
                             const int32_t* forbidden, int32_t* out_sliced, int32_t* out_count);

/* Batched contractions of uneven shapes (one grouped launch) ----------------
 *
 * `count` binary einsums y_i <- sy*y_i + sx*f(x1_i, x2_i) whose label groups
 * (outer1, outer2, inner, batch) each merge into one strided mode -- e.g.
 * every contraction of an MPS sweep.  ome_batch_create analyses them like
 * ome_einsum does (src/einsum.jl:139-211), uploads a problem table, and times
 * the candidate kernels on the batch (tile_config < 0; or pick 0..3);
 * ome_batch_run issues ONE persistent grouped kernel over all problems' tiles
 * (capturable in a CUDA graph).  Tensors are bound at creation: the buffers
 * must stay valid.  Replaces a loop of einsum! calls, one launch each. */
typedef struct ome_batch ome_batch;
OME_API int ome_batch_create(ome_ctx* ctx, void* stream, ome_dtype dtype, int32_t count,
                             const ome_tensor* x1s, const ome_tensor* x2s, const ome_tensor* ys,
                             int32_t tile_config, ome_batch** out);
OME_API int ome_batch_run(ome_ctx* ctx, ome_batch* batch, void* stream, const void* sx, const void* sy);
/* Chosen kernel (0: 32x32, 1: 64x32, 2: 64x64 CUDA-core tiles; 3: the tensor-core
 * grouped kernel, 128 x 128 tiles of BF16x6 split products, F32 and C32 only --
 * C32 as the real 2 x 2 embedding) and the autotuner's timings (us, 4 floats;
 * -1 for a kernel that is not a candidate for the dtype). */
OME_API int ome_batch_info(const ome_batch* batch, int32_t* tile_config, float* tuned_us);
OME_API int ome_batch_destroy(ome_batch* batch);

/* A CUDA graph of grouped launches (e.g. the two contractions of an MPS sweep
 * step), captured once and replayed with one call: replaces a loop of
 * ome_batch_run calls whose host launch cost would dominate small batches.
 * The graph runs batches[0..count) in order, each with its chosen kernel, with
 * scalars sxs[i] / sys[i] (NULL arrays or entries: 1 and 0 of the batch's
 * dtype).  The batches must outlive the graph; replays read the tensors bound
 * at batch creation.  Capture uses a private stream after synchronising
 * `stream`; ome_graph_launch enqueues one replay on `stream`. */
typedef struct ome_graph ome_graph;
OME_API int ome_batch_graph_create(ome_ctx* ctx, void* stream, int32_t count, ome_batch* const* batches,
                                   const void* const* sxs, const void* const* sys, ome_graph** out);
OME_API int ome_graph_launch(ome_graph* graph, void* stream);
OME_API int ome_graph_destroy(ome_graph* graph);

/* Serving: continuous batching of whole contraction-tree jobs --------------
 *
 * No counterpart in the reference, whose service would call
 * einsum(::NestedEinsum) or cost_and_gradient (src/einsequence.jl:270-287,
 * src/bp.jl:122-130) once per request.  A server keeps n_slots slots on one
 * device; each owns a stream, a host issue thread and a context whose
 * workspace is hbm_budget_bytes / n_slots (allocated on the slot's first job,
 * kept until ome_server_destroy).  Jobs are admitted in arrival order when a
 * slot is free and the plan's peak workspace bytes (ome_plan_peak_bytes:
 * forward, or forward+gradient for gradient jobs) fit a slot's share; a job
 * above a share but within the budget waits until every slot is idle and runs
 * alone in a workspace of its own size; jobs above the budget
 * (OME_JOB_REJECTED_MEMORY) or with more than max_job_work multiply-adds
 * (OME_JOB_REJECTED_WORK; max_job_work <= 0: no cap) are rejected at
 * admission.  Admission and retirement happen in ome_server_poll, which never
 * blocks on the device. */
typedef struct ome_server ome_server;
typedef enum {
  OME_JOB_COMPLETED = 0,
  OME_JOB_FAILED = 1,           /* status holds the error; ome_last_error() after poll names it */
  OME_JOB_REJECTED_MEMORY = 2,
  OME_JOB_REJECTED_WORK = 3
} ome_job_outcome;
typedef struct {
  int64_t id;
  int32_t outcome;              /* ome_job_outcome */
  int32_t status;               /* OME_OK for completed jobs */
  double arrival_s, admitted_s, done_s;   /* seconds since ome_server_create; admitted_s < 0 if never admitted */
} ome_server_job;
typedef struct {
  int64_t submitted, completed, failed, rejected_memory, rejected_work, queued, running;
  double p50_ms, p90_ms, p99_ms;          /* latency (arrival to completion seen by poll) of completed jobs */
  double jobs_per_s, makespan_s;          /* completed / (last completion - first arrival) */
} ome_serving_stats;
OME_API int ome_server_create(int device, int32_t n_slots, size_t hbm_budget_bytes, double max_job_work,
                              ome_server** out);
/* Queue a job: y <- tree(inputs) of the plan (dxs == NULL), or cost_and_gradient
 * (dxs[t] receives the gradient of input t; the plan runs unsliced).  inputs,
 * y and dxs are column-major contiguous device buffers of the plan's dtype;
 * they and the plan belong to the caller and must stay valid until poll
 * reports the job.  input_stream: the stream the inputs were written on (NULL
 * = the legacy default stream, as in every CUDA call); the job's kernels run
 * after the work queued on it at submit time -- the slots' streams are
 * non-blocking and would not otherwise wait for the default stream.
 * work: the job's multiply-adds, for the work cap.  Thread-safe with poll. */
OME_API int ome_server_submit(ome_server* server, ome_plan* plan, int32_t ninputs, const void* const* inputs,
                              void* y, void* const* dxs, double work, void* input_stream, int64_t* job_id);
/* Retire finished jobs, admit queued ones, and return up to max_jobs records
 * of jobs that finished or were rejected since the last poll (oldest first);
 * *running = jobs on the device. */
OME_API int ome_server_poll(ome_server* server, int32_t max_jobs, ome_server_job* jobs, int32_t* n_jobs,
                            int32_t* running);
OME_API int ome_server_stats(ome_server* server, ome_serving_stats* stats);
/* The server's clock: seconds since ome_server_create (the time base of
 * ome_server_job), for callers that account latency from their own arrivals. */
OME_API int ome_server_clock(const ome_server* server, double* seconds);
/* Waits (without a time limit) for every issued job, then frees the slots;
 * queued jobs are dropped. */
OME_API int ome_server_destroy(ome_server* server);

/* Allocation-free reduction --------------------------------------------------
 *
 * No counterpart in the reference.  y <- sy*y + sx*sum(x) where every label
 * of y is a label of x and the labels of x missing from y are summed (a Sum
 * or Tr einsum such as "ii->" or "ijk->j"; repeated input labels are
 * diagonals).  It runs the same two-pass split reduction as ome_einsum, but
 * keeps the partial sums in a fixed array inside the library instead of a
 * context workspace: it takes no context and allocates no device memory.
 * For callers that cannot let a library cudaMalloc: code whose device memory
 * is owned by its own allocator (CUDA.jl's pool, a serving process with a
 * fixed HBM arena), where an extra allocation would fail or fragment the
 * budget and cudaMalloc/cudaFree would synchronise the device.
 *
 * Limit: the partial sums (at least two per output element) must fit in
 * OME_NOALLOC_SCRATCH_BYTES, i.e. at most OME_NOALLOC_SCRATCH_BYTES /
 * (2 * element size) output elements; larger outputs are rejected with
 * OME_UNSUPPORTED.  Every GPU that loads the library holds the array until
 * the process exits.  The first call on a device looks up the array's device
 * address with that device current; make it before any stream capture.
 * All calls on a device share the array: calls that overlap on the GPU
 * (different streams or host threads) race and must be serialised. */
#define OME_NOALLOC_SCRATCH_BYTES (4u << 20)
OME_API int ome_reduce_noalloc(void* stream, ome_dtype dtype, const ome_tensor* x,
                               const ome_tensor* y, const void* sx, const void* sy);

#ifdef __cplusplus
}
#endif

#endif /* OME_B200_H */
