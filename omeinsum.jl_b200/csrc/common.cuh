// Shared definitions of libomeb200: algebras (semirings), launch arguments,
// small device helpers.  Column-major, element-stride conventions of
// OMEinsum.jl (src/Core.jl:116-145 EinIndexer: offset = sum (i_d-1)*stride_d).
#pragma once

#include <atomic>
#include <utility>
#include <cuda_runtime.h>
#include <stdint.h>
#include <math.h>
#include "ome_b200.h"

namespace ome {

constexpr int MAXD = 64;     // max rank of a tensor at the ABI
constexpr int MAXM = 64;     // max merged modes in one kernel launch
constexpr int MAXIN = 8;     // max inputs of one index-kernel launch
constexpr int MAXG = 32;     // max merged modes per GEMM group (M, N, K, batch)

// ---------------------------------------------------------------------------
// element types
// ---------------------------------------------------------------------------
struct __align__(8) cf32 { float re, im; };
struct __align__(16) cf64 { double re, im; };

// Julia `max` on floats: NaN-propagating, +0.0 > -0.0.
template <class F>
__host__ __device__ __forceinline__ F julia_max(F a, F b) {
  if (a != a) return a;
  if (b != b) return b;
  if (b > a) return b;
  if (a > b) return a;
  return signbit(a) ? b : a;
}

// Each algebra: storage type T, zero/one, add (sum), mul (product), is_zero.
// Products of more than two factors are always evaluated left to right, as
// map_prod does (src/Core.jl:240-243).
struct AlgF32 {
  using T = float;
  static constexpr ome_dtype DT = OME_F32;
  __host__ __device__ static T zero() { return 0.f; }
  __host__ __device__ static T one() { return 1.f; }
  __host__ __device__ static T add(T a, T b) { return a + b; }
  __host__ __device__ static T mul(T a, T b) { return a * b; }
  __host__ __device__ static T fma(T a, T b, T c) { return fmaf(a, b, c); }
  __host__ __device__ static bool is_zero(T a) { return a == 0.f; }
  __host__ __device__ static bool is_one(T a) { return a == 1.f; }
};
struct AlgF64 {
  using T = double;
  static constexpr ome_dtype DT = OME_F64;
  __host__ __device__ static T zero() { return 0.0; }
  __host__ __device__ static T one() { return 1.0; }
  __host__ __device__ static T add(T a, T b) { return a + b; }
  __host__ __device__ static T mul(T a, T b) { return a * b; }
  __host__ __device__ static T fma(T a, T b, T c) { return ::fma(a, b, c); }
  __host__ __device__ static bool is_zero(T a) { return a == 0.0; }
  __host__ __device__ static bool is_one(T a) { return a == 1.0; }
};
struct AlgC32 {
  using T = cf32;
  static constexpr ome_dtype DT = OME_C32;
  __host__ __device__ static T zero() { return {0.f, 0.f}; }
  __host__ __device__ static T one() { return {1.f, 0.f}; }
  __host__ __device__ static T add(T a, T b) { return {a.re + b.re, a.im + b.im}; }
  __host__ __device__ static T mul(T a, T b) {
    return {a.re * b.re - a.im * b.im, a.re * b.im + a.im * b.re};
  }
  __host__ __device__ static T fma(T a, T b, T c) {
    return {fmaf(a.re, b.re, fmaf(-a.im, b.im, c.re)), fmaf(a.re, b.im, fmaf(a.im, b.re, c.im))};
  }
  __host__ __device__ static bool is_zero(T a) { return a.re == 0.f && a.im == 0.f; }
  __host__ __device__ static bool is_one(T a) { return a.re == 1.f && a.im == 0.f; }
};
struct AlgC64 {
  using T = cf64;
  static constexpr ome_dtype DT = OME_C64;
  __host__ __device__ static T zero() { return {0.0, 0.0}; }
  __host__ __device__ static T one() { return {1.0, 0.0}; }
  __host__ __device__ static T add(T a, T b) { return {a.re + b.re, a.im + b.im}; }
  __host__ __device__ static T mul(T a, T b) {
    return {a.re * b.re - a.im * b.im, a.re * b.im + a.im * b.re};
  }
  __host__ __device__ static T fma(T a, T b, T c) {
    return {::fma(a.re, b.re, ::fma(-a.im, b.im, c.re)), ::fma(a.re, b.im, ::fma(a.im, b.re, c.im))};
  }
  __host__ __device__ static bool is_zero(T a) { return a.re == 0.0 && a.im == 0.0; }
  __host__ __device__ static bool is_one(T a) { return a.re == 1.0 && a.im == 0.0; }
};
// Int64 with Julia's wrap-around: arithmetic through uint64.
struct AlgI64 {
  using T = long long;
  static constexpr ome_dtype DT = OME_I64;
  __host__ __device__ static T zero() { return 0; }
  __host__ __device__ static T one() { return 1; }
  __host__ __device__ static T add(T a, T b) {
    return (T)((unsigned long long)a + (unsigned long long)b);
  }
  __host__ __device__ static T mul(T a, T b) {
    return (T)((unsigned long long)a * (unsigned long long)b);
  }
  __host__ __device__ static T fma(T a, T b, T c) { return add(mul(a, b), c); }
  __host__ __device__ static bool is_zero(T a) { return a == 0; }
  __host__ __device__ static bool is_one(T a) { return a == 1; }
};
// Bool: OR-AND, one byte per element.
struct AlgBool {
  using T = unsigned char;
  static constexpr ome_dtype DT = OME_BOOL;
  __host__ __device__ static T zero() { return 0; }
  __host__ __device__ static T one() { return 1; }
  __host__ __device__ static T add(T a, T b) { return (T)((a | b) != 0); }
  __host__ __device__ static T mul(T a, T b) { return (T)((a != 0) & (b != 0)); }
  __host__ __device__ static T fma(T a, T b, T c) { return add(mul(a, b), c); }
  __host__ __device__ static bool is_zero(T a) { return a == 0; }
  __host__ __device__ static bool is_one(T a) { return a != 0; }
};
// Tropical max-plus (TropicalNumbers.jl): (+) = max, (*) = +, zero = -Inf, one = 0.
struct AlgTF32 {
  using T = float;
  static constexpr ome_dtype DT = OME_TROP_F32;
  __host__ __device__ static T zero() { return -INFINITY; }
  __host__ __device__ static T one() { return 0.f; }
  __host__ __device__ static T add(T a, T b) { return julia_max(a, b); }
  __host__ __device__ static T mul(T a, T b) { return a + b; }
  __host__ __device__ static T fma(T a, T b, T c) { return julia_max(a + b, c); }
  __host__ __device__ static bool is_zero(T a) { return a == -INFINITY; }
  __host__ __device__ static bool is_one(T a) { return a == 0.f; }
};
struct AlgTF64 {
  using T = double;
  static constexpr ome_dtype DT = OME_TROP_F64;
  __host__ __device__ static T zero() { return -INFINITY; }
  __host__ __device__ static T one() { return 0.0; }
  __host__ __device__ static T add(T a, T b) { return julia_max(a, b); }
  __host__ __device__ static T mul(T a, T b) { return a + b; }
  __host__ __device__ static T fma(T a, T b, T c) { return julia_max(a + b, c); }
  __host__ __device__ static bool is_zero(T a) { return a == -INFINITY; }
  __host__ __device__ static bool is_one(T a) { return a == 0.0; }
};

inline size_t dtype_size(ome_dtype d) {
  switch (d) {
    case OME_F32: return 4;
    case OME_F64: return 8;
    case OME_C32: return 8;
    case OME_C64: return 16;
    case OME_I64: return 8;
    case OME_BOOL: return 1;
    case OME_TROP_F32: return 4;
    case OME_TROP_F64: return 8;
  }
  return 0;
}

// Dispatch a templated call over the algebra of `dt`.
#define OME_DISPATCH(dt, ALG, ...)                      \
  switch (dt) {                                         \
    case OME_F32: { using ALG = ome::AlgF32; __VA_ARGS__; } break;  \
    case OME_F64: { using ALG = ome::AlgF64; __VA_ARGS__; } break;  \
    case OME_C32: { using ALG = ome::AlgC32; __VA_ARGS__; } break;  \
    case OME_C64: { using ALG = ome::AlgC64; __VA_ARGS__; } break;  \
    case OME_I64: { using ALG = ome::AlgI64; __VA_ARGS__; } break;  \
    case OME_BOOL: { using ALG = ome::AlgBool; __VA_ARGS__; } break; \
    case OME_TROP_F32: { using ALG = ome::AlgTF32; __VA_ARGS__; } break; \
    case OME_TROP_F64: { using ALG = ome::AlgTF64; __VA_ARGS__; } break; \
  }

// 16 raw bytes holding one scalar of any dtype (sx, sy).
// Raises kernel's dynamic shared-memory limit to `bytes` once per device
// (the attribute belongs to the device's context), safely from any host
// thread; `done` records the devices already set (bit = device ordinal).
template <class K>
inline cudaError_t set_smem_once(std::atomic<unsigned long long>& done, K* kernel, int bytes) {
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return e;
  const unsigned long long bit = 1ull << (dev & 63);
  if (done.load(std::memory_order_acquire) & bit) return cudaSuccess;
  e = cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes);
  if (e == cudaSuccess) done.fetch_or(bit, std::memory_order_release);
  return e;
}

struct Scalar {
  alignas(16) unsigned char b[16];
};
template <class T>
__host__ __device__ __forceinline__ T scalar_as(const Scalar& s) {
  T v;
  memcpy(&v, s.b, sizeof(T));
  return v;
}

// y <- sy*y + sx*f, or sx*f when sy is the algebra's zero (src/utils.jl:25-35).
template <class A>
__device__ __forceinline__ typename A::T epilogue(typename A::T f, const typename A::T* yp,
                                                  typename A::T sx, typename A::T sy,
                                                  bool sy_zero, bool sx_one) {
  typename A::T v = sx_one ? f : A::mul(sx, f);
  if (!sy_zero) v = A::add(A::mul(sy, *yp), v);
  return v;
}

// Warp shuffle for any trivially copyable T (split into 32-bit words).
template <class T>
__device__ __forceinline__ T shfl_down_any(T v, int d) {
  constexpr int W = (sizeof(T) + 3) / 4;
  uint32_t w[W];
  memset(w, 0, sizeof(w));
  memcpy(w, &v, sizeof(T));
#pragma unroll
  for (int i = 0; i < W; ++i) w[i] = __shfl_down_sync(0xffffffffu, w[i], d);
  T r;
  memcpy(&r, w, sizeof(T));
  return r;
}

// Block-wide reduction (result valid in thread 0).  blockDim.x multiple of 32.
template <class A>
__device__ typename A::T block_reduce(typename A::T v, typename A::T* sh /* >= 32 */) {
  for (int d = 16; d > 0; d >>= 1) v = A::add(v, shfl_down_any(v, d));
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  if (lane == 0) sh[wid] = v;
  __syncthreads();
  const int nw = (blockDim.x + 31) >> 5;
  if (wid == 0) {
    v = lane < nw ? sh[lane] : A::zero();
    for (int d = 16; d > 0; d >>= 1) v = A::add(v, shfl_down_any(v, d));
  }
  __syncthreads();
  return v;
}

// ---------------------------------------------------------------------------
// launch argument blocks (passed by value as kernel parameters)
// ---------------------------------------------------------------------------

// Generic index kernel (loop_einsum).  Modes [0, nout) are output modes,
// [nout, nout + ninner) inner (summed) modes.  str[0] holds y strides (0 for
// inner modes), str[1 + i] strides of input i (0 where the input lacks the
// label).  Step digits advance a mixed-radix inner counter by `step`.
struct LoopArgs {
  const void* x[MAXIN];
  void* y;
  void* partial;          // split mode: per (output, split) partial sums
  int nin, nout, ninner;
  int nsplit;             // >1: inner space split over nsplit blocks per output
  int64_t n_out, n_in;
  int64_t ext[MAXM];
  int64_t str[MAXIN + 1][MAXM];
  int32_t stepdig[MAXM];  // inner step (blockDim * nsplit) in mixed radix
  Scalar sx, sy;
  int sy_zero, sx_one;
};

// Permute / broadcast copy: y[modes] <- sx*x[modes] (+ sy*y).  Mode 0 is y's
// fastest mode; tmode (>0) is x's fastest mode for the tiled transpose, or -1.
// Division of n < 2^31 by an invariant d >= 1 with one multiply-high, add and
// shift (Granlund & Montgomery, "Division by invariant integers using
// multiplication", PLDI 1994, round-up multiplier m = floor(2^32 (2^l - d) / d) + 1,
// l = ceil(log2 d)).  (umulhi(n, m) + n) stays below 2^32 for n < 2^31.
struct FastDiv {
  uint32_t d, m, l;
};

static inline FastDiv make_fastdiv(uint32_t d) {
  uint32_t l = 0;
  while (l < 32 && ((uint64_t)1 << l) < d) ++l;
  const uint64_t m = (((uint64_t)1 << 32) * (((uint64_t)1 << l) - d)) / d + 1;
  return FastDiv{d, (uint32_t)m, l};
}

__device__ __forceinline__ uint32_t fast_div(uint32_t n, const FastDiv& f) {
  return (__umulhi(n, f.m) + n) >> f.l;
}

struct PermArgs {
  const void* x;
  void* y;
  int nd, tmode;
  int64_t n;
  int64_t ext[MAXM], xs[MAXM], ys[MAXM];
  Scalar sx, sy;
  int sy_zero, sx_one;
};

// Strided batched GEMM C[m,n,l] = sx * sum_k A[m,k,l] B[k,n,l] (+ sy*C) with
// every group given as merged modes (extent, strides).  No permuted copies.
struct GemmArgs {
  const void* A;
  const void* B;
  void* C;
  int64_t M, N, K, L;
  int nm, nn, nk, nl;
  int64_t m_ext[MAXG], m_sa[MAXG], m_sc[MAXG];
  int64_t n_ext[MAXG], n_sb[MAXG], n_sc[MAXG];
  int64_t k_ext[MAXG], k_sa[MAXG], k_sb[MAXG];
  int64_t l_ext[MAXG], l_sa[MAXG], l_sb[MAXG], l_sc[MAXG];
  int a_m_fast, b_n_fast;  // 1: the group's first mode is the operand's contiguous one
  Scalar sx, sy;
  int sy_zero, sx_one;
  // C offsets of every m and every n (device tables, or NULL): filled when a
  // group has several modes, so that epilogues index a table instead of
  // evaluating a mixed-radix offset per element
  const int64_t* m_tab_c;
  const int64_t* n_tab_c;
};

// Offset of flat index i over modes (column-major, first mode fastest).
__host__ __device__ __forceinline__ int64_t mode_offset(int64_t i, int n, const int64_t* ext,
                                                       const int64_t* str) {
  int64_t off = 0;
  for (int m = 0; m < n; ++m) {
    int64_t e = ext[m];
    int64_t q = i / e;
    off += (i - q * e) * str[m];
    i = q;
  }
  return off;
}

// Programmatic dependent launch: a kernel launched with the programmatic
// stream-serialisation attribute (launch_pdl) may start while the previous
// kernel in its stream finishes; it runs its set-up, then waits in
// griddep_wait until that kernel has completed and its writes are visible.
// The previous kernel lets it start once all its own blocks are running
// (griddep_launch_dependents).  Both are no-ops without the attribute.
__device__ __forceinline__ void griddep_wait() { asm volatile("griddepcontrol.wait;" ::: "memory"); }
__device__ __forceinline__ void griddep_launch_dependents() {
  asm volatile("griddepcontrol.launch_dependents;" ::: "memory");
}
template <class... KArgs, class... Args>
static cudaError_t launch_pdl(void (*kernel)(KArgs...), dim3 grid, dim3 block, size_t smem, cudaStream_t s,
                              Args&&... args) {
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = grid;
  cfg.blockDim = block;
  cfg.dynamicSmemBytes = smem;
  cfg.stream = s;
  cudaLaunchAttribute at[1];
  at[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
  at[0].val.programmaticStreamSerializationAllowed = 1;
  cfg.attrs = at;
  cfg.numAttrs = 1;
  return cudaLaunchKernelEx(&cfg, kernel, std::forward<Args>(args)...);
}

}  // namespace ome
