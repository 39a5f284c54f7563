// Launchers of libomeb200's kernels (host side).  Each returns the launch's
// cudaError_t; the argument blocks are defined in common.cuh.
#pragma once
#include "common.cuh"

namespace ome {

// Global count of kernel launches issued by the library.
unsigned long long launch_counter();
void count_launch(int n = 1);

// Diagnostic kernel timing: while enabled (ome_kernel_timing), a KernelTimer
// records CUDA events around the main kernel of a dispatch on its stream (no
// synchronisation); ome_kernel_times reads the durations afterwards.
void set_kernel_timing(int n);
int read_kernel_times(int max, float* ms, const char** names);
struct KernelTimer {
  KernelTimer(cudaStream_t s, const char* name);
  ~KernelTimer();
  cudaStream_t s;
  const char* name;
  int slot;
};

enum LoopMode { LOOP_THREAD = 0, LOOP_BLOCK = 1 };

// Generic sum-product (loop_einsum): mode LOOP_THREAD = one thread per output
// element; LOOP_BLOCK = one block per output (a.nsplit == 1) or nsplit blocks
// per output writing partials to a.partial, finished by launch_loop_finish.
cudaError_t launch_loop(ome_dtype dt, const LoopArgs& a, LoopMode mode, int grid, int block,
                        cudaStream_t s);
cudaError_t launch_loop_finish(ome_dtype dt, const LoopArgs& a, cudaStream_t s);
// No summed labels (ninner == 0): a block per segment of a row of y's
// fastest mode, 16-byte accesses where the strides allow.
cudaError_t launch_map_rows(ome_dtype dt, const LoopArgs& a, int num_sms, cudaStream_t s);
// Thread per output along y's fastest mode, summed space split over
// grid.y ranges of chunk (partials for launch_loop_finish when nsplit > 1).
// vec: V = 16 / element-size consecutive outputs per thread with 16-byte loads.
cudaError_t launch_loop_cols(ome_dtype dt, const LoopArgs& a, int64_t chunk, dim3 grid, bool vec, cudaStream_t s);
// One input, first inner mode contiguous, at most one more inner mode: block
// per (output, row split) with vector loads (vec) over rows of rchunk.
cudaError_t launch_reduce_contig(ome_dtype dt, const LoopArgs& a, bool vec, int64_t rchunk, int grid,
                                 cudaStream_t s);
// The same with one warp per output (many outputs).
cudaError_t launch_reduce_rows(ome_dtype dt, const LoopArgs& a, bool vec, int grid, cudaStream_t s);

// Permute / broadcast / identity copy with the αβ epilogue.
cudaError_t launch_perm(ome_dtype dt, const PermArgs& a, int num_sms, cudaStream_t s);

// y <- sy*y (or the algebra's zero when sy_zero) over a strided view.
cudaError_t launch_scale(ome_dtype dt, void* y, int nd, const int64_t* ext, const int64_t* str,
                         const Scalar& sy, int sy_zero, int num_sms, cudaStream_t s);

// CUDA-core strided batched GEMM over any algebra.
cudaError_t launch_gemm_simt(ome_dtype dt, const GemmArgs& g, cudaStream_t s);
// The same, with K split over blocks (partials in `workspace`, summed in
// split order) when the output tiles alone would leave most SMs idle.
cudaError_t launch_gemm_simt_ws(ome_dtype dt, const GemmArgs& g, void* workspace, size_t ws_bytes, int num_sms,
                                cudaStream_t s);
// FP32 batched GEMM with M, N <= 64 on CUDA cores (64 x 64 tiles, one per batch).
cudaError_t launch_gemm_simt_small_f32(const GemmArgs& g, cudaStream_t s);
// Batched GEMM with the batch mode contiguous in A, B and C and M, N <= 64
// (4 consecutive batches per CTA staged in shared memory, k_gemm_bstage);
// cudaErrorNotSupported if the shape differs.
bool gemm_bfast_applies(const GemmArgs& g);
cudaError_t launch_gemm_bfast(ome_dtype dt, const GemmArgs& g, cudaStream_t s);

// acc[i] (double / double2) += (double) src[i] for n elements, contiguous;
// FP64 cross-slice accumulation.  dt is the element type of src.
cudaError_t launch_acc64(ome_dtype dt, void* acc, const void* src, int64_t n, cudaStream_t s);
// y <- sx*(T)acc + sy*y over n contiguous elements (final slice write-back).
cudaError_t launch_acc64_store(ome_dtype dt, void* y, const void* acc, int64_t n, const Scalar& sx,
                               const Scalar& sy, int sy_zero, cudaStream_t s);

// acc (double / double2, strided view with nd modes) += src (contiguous, same
// mode order, column-major).
cudaError_t launch_acc64_strided(ome_dtype dt, void* acc, const void* src, int nd, const int64_t* ext,
                                 const int64_t* acc_str, cudaStream_t s);
// x <- conj(x) (complex dtypes) over n contiguous elements.
cudaError_t launch_conj(ome_dtype dt, void* x, int64_t n, cudaStream_t s);
// x <- one(T) over n contiguous elements.
cudaError_t launch_fill_one(ome_dtype dt, void* x, int64_t n, cudaStream_t s);

// Tensor-core FP32 GEMM from BF16 split products (tcgen05 + TMEM): nterms = 2
// (BF16x3, 3 MMAs per K step) or 3 (BF16x6, 6 MMAs, FP32-faithful).
// Returns cudaErrorNotSupported when the shape is outside the kernel's
// preconditions (the caller then uses the CUDA-core kernel).
cudaError_t launch_gemm_split(const GemmArgs& g, int nterms, void* workspace, size_t ws_bytes, int num_sms,
                              cudaStream_t s);
bool gemm_split_supported(const GemmArgs& g);
// Fill tab[0..M) and tab[M..M+N) with the C offsets of m and n and point
// g.m_tab_c / g.n_tab_c at them (for mode groups of several modes).
cudaError_t launch_c_offsets(GemmArgs& g, int64_t* tab, cudaStream_t s);
// Pre-split (packed BF16 terms) + bulk-copy-fed persistent GEMM; needs
// gemm_packed_bytes() of workspace, returns cudaErrorNotSupported otherwise
// (before launching anything).  ctab (M + N entries, or NULL): the C offset
// tables, filled by the pack launch and used by the GEMM's epilogue.
cudaError_t launch_gemm_packed(const GemmArgs& g, int nterms, void* workspace, size_t ws_bytes, int num_sms,
                               cudaStream_t s, int64_t* ctab);
size_t gemm_packed_bytes(const GemmArgs& g, int nterms, int num_sms);
// 2-SM tensor-core GEMM fed by TMA tensor maps over the FP32 operands (BF16
// terms formed in shared memory): single-mode M, N, K and batch groups, each
// operand contiguous along its row or K mode, 16-byte aligned.  Split-K
// partials go to `workspace`; cudaErrorNotSupported (nothing launched) when
// the shape or the workspace does not fit.
bool gemm_tma2_applies(const GemmArgs& g);
// Batches of FP32 GEMMs with M, N <= 64, K <= 256 and the batch mode
// contiguous in A, B and C (column-major bij,bjk->bik) on the tensor cores:
// two batches per block-diagonal 128 x 128 MMA, four per CTA, operands by TMA.
bool gemm_bdiag_applies(const GemmArgs& g);
cudaError_t launch_gemm_bdiag(const GemmArgs& g, int nterms, cudaStream_t s);
cudaError_t launch_gemm_tma2(const GemmArgs& g, int nterms, void* workspace, size_t ws_bytes, int num_sms,
                             cudaStream_t s);

// Read and clear the CUDA-core GEMM's split-partial self-check flag.
int simt_bounds_flag();
// One problem of a grouped launch: C[m,n,l] = sx * sum_k A[m,k,l] B[k,n,l]
// (+ sy*C), strides in elements; tile_begin / tiles_m / tiles_n depend on
// the tile shape of the kernel the table is built for.
struct GroupProblem {
  const void* a;
  const void* b;
  void* c;
  int64_t m, n, k, l;
  int64_t a_sm, a_sk, a_sl;
  int64_t b_sk, b_sn, b_sl;
  int64_t c_sm, c_sn, c_sl;
  int64_t tile_begin;  // first global tile index of this problem
  int32_t tiles_m, tiles_n;
  // the operand's K mode is contiguous and its rows start on 16 bytes
  // (vector loads of 4 complex / 8 real k by the tensor-core kernel)
  int32_t a_kvec, b_kvec;
};
// Grouped launch on the tensor cores (F32, or C32 through its real 2 x 2
// embedding): 128 x 128 tiles of the (embedded) output, BF16 split products
// (nterms 2 or 3) formed in shared memory; tiles_m counts 128 real rows
// (64 complex rows for C32).  cudaErrorNotSupported for other dtypes.
// Sets the kernel's shared-memory attribute (and so loads it); done by the
// first launch, and before a graph capture so that none happens inside it.
cudaError_t prepare_group_tc(ome_dtype dt, int nterms);
// tile_prob[t] is the problem that owns global tile t.
cudaError_t launch_group_tc(ome_dtype dt, int nterms, const GroupProblem* probs, const int32_t* tile_prob, int nprob,
                            int64_t tiles, int grid, const Scalar& sx, const Scalar& sy, int sy_zero, int sx_one,
                            cudaStream_t s);
// Synchronise s and read/clear the device timeout flag: 1 if a bounded wait
// gave up, 0 if not, -cudaError on failure.
int device_status(cudaStream_t s);
// One-block kernel whose bounded mbarrier wait runs out (failure-path test).
cudaError_t launch_selftest_wait(uint64_t wait_ns, cudaStream_t s);

}  // namespace ome
