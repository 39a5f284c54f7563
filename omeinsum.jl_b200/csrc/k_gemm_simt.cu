// CUDA-core strided batched GEMM over any algebra.
//
// Replaces analyze_binary's permute -> reshape -> (batched) GEMM chain
// (src/einsum.jl:104-124, src/binaryrules.jl:46-61,94-141, src/utils.jl:162-177,
// ext/CUDAExt.jl:115-117,156-178) for the element types that have no
// tensor-core path (Int64, Bool, tropical, FP64, complex) and for the plain
// FP32 comparison path.  Operands are read in place through per-group mode
// strides, so no permuted copy is ever materialised; the output permutation
// is absorbed in the epilogue's strides.
#include <string.h>
#include "kernels.h"

namespace ome {

template <int ES> struct SimtCfg;                 // by element size
template <> struct SimtCfg<1> { static constexpr int BM = 128, BN = 128, BK = 8, TM = 8, TN = 8; };
template <> struct SimtCfg<4> { static constexpr int BM = 128, BN = 128, BK = 8, TM = 8, TN = 8; };
template <> struct SimtCfg<8> { static constexpr int BM = 64, BN = 64, BK = 8, TM = 4, TN = 4; };
template <> struct SimtCfg<16> { static constexpr int BM = 64, BN = 64, BK = 8, TM = 4, TN = 4; };
// 64 x 64 tiles for 4-byte types when M and N both fit in 64 (batched small
// GEMMs such as bij,bjk->bik with 64^3 per batch: a 128 x 128 tile would be
// three-quarters padding).
struct SimtSmall { static constexpr int BM = 64, BN = 64, BK = 8, TM = 4, TN = 4; };

__device__ __forceinline__ int64_t group_off(int64_t i, int n, const int64_t* ext, const int64_t* str) {
  if (n == 1) return i * str[0];
  return mode_offset(i, n, ext, str);
}

template <class A, class C = SimtCfg<sizeof(typename A::T)>>
__global__ void __launch_bounds__(256) k_gemm_simt(const __grid_constant__ GemmArgs g) {
  using T = typename A::T;
  constexpr int BM = C::BM, BN = C::BN, BK = C::BK, TM = C::TM, TN = C::TN;
  constexpr int NT = 256;
  constexpr int RA = BM * BK / NT, RB = BN * BK / NT;
  static_assert((BM / TM) * (BN / TN) == NT, "thread tile");
  __shared__ T As[2][BK][BM];
  __shared__ T Bs[2][BK][BN];
  __shared__ int64_t am[BM], bn[BN];

  const T* Ap = static_cast<const T*>(g.A);
  const T* Bp = static_cast<const T*>(g.B);
  T* Cp = static_cast<T*>(g.C);
  const T sx = scalar_as<T>(g.sx), sy = scalar_as<T>(g.sy);
  const int tid = threadIdx.x;
  const int tx = tid % (BN / TN), ty = tid / (BN / TN);
  const int64_t m0 = (int64_t)blockIdx.x * BM, n0 = (int64_t)blockIdx.y * BN;

  for (int64_t l = blockIdx.z; l < g.L; l += gridDim.z) {
    const int64_t la = mode_offset(l, g.nl, g.l_ext, g.l_sa);
    const int64_t lb = mode_offset(l, g.nl, g.l_ext, g.l_sb);
    const int64_t lc = mode_offset(l, g.nl, g.l_ext, g.l_sc);
    for (int i = tid; i < BM; i += NT)
      am[i] = (m0 + i < g.M) ? la + group_off(m0 + i, g.nm, g.m_ext, g.m_sa) : -1;
    for (int i = tid; i < BN; i += NT)
      bn[i] = (n0 + i < g.N) ? lb + group_off(n0 + i, g.nn, g.n_ext, g.n_sb) : -1;
    __syncthreads();

    T acc[TM][TN];
#pragma unroll
    for (int i = 0; i < TM; ++i)
#pragma unroll
      for (int j = 0; j < TN; ++j) acc[i][j] = A::zero();

    T ra[RA], rb[RB];
    auto load = [&](int64_t k0) {
#pragma unroll
      for (int r = 0; r < RA; ++r) {
        const int e = tid + NT * r;
        const int mm = g.a_m_fast ? e % BM : e / BK;
        const int kk = g.a_m_fast ? e / BM : e % BK;
        const int64_t k = k0 + kk;
        const int64_t base = am[mm];
        ra[r] = (base >= 0 && k < g.K) ? Ap[base + group_off(k, g.nk, g.k_ext, g.k_sa)] : A::zero();
      }
#pragma unroll
      for (int r = 0; r < RB; ++r) {
        const int e = tid + NT * r;
        const int nn = g.b_n_fast ? e % BN : e / BK;
        const int kk = g.b_n_fast ? e / BN : e % BK;
        const int64_t k = k0 + kk;
        const int64_t base = bn[nn];
        rb[r] = (base >= 0 && k < g.K) ? Bp[base + group_off(k, g.nk, g.k_ext, g.k_sb)] : A::zero();
      }
    };
    auto store = [&](int buf) {
#pragma unroll
      for (int r = 0; r < RA; ++r) {
        const int e = tid + NT * r;
        const int mm = g.a_m_fast ? e % BM : e / BK;
        const int kk = g.a_m_fast ? e / BM : e % BK;
        As[buf][kk][mm] = ra[r];
      }
#pragma unroll
      for (int r = 0; r < RB; ++r) {
        const int e = tid + NT * r;
        const int nn = g.b_n_fast ? e % BN : e / BK;
        const int kk = g.b_n_fast ? e / BN : e % BK;
        Bs[buf][kk][nn] = rb[r];
      }
    };

    load(0);
    store(0);
    __syncthreads();
    int buf = 0;
    for (int64_t k0 = 0; k0 < g.K; k0 += BK) {
      const bool more = k0 + BK < g.K;
      if (more) load(k0 + BK);
#pragma unroll
      for (int kk = 0; kk < BK; ++kk) {
        T a[TM], b[TN];
#pragma unroll
        for (int i = 0; i < TM; ++i) a[i] = As[buf][kk][ty * TM + i];
#pragma unroll
        for (int j = 0; j < TN; ++j) b[j] = Bs[buf][kk][tx * TN + j];
#pragma unroll
        for (int i = 0; i < TM; ++i)
#pragma unroll
          for (int j = 0; j < TN; ++j) acc[i][j] = A::fma(a[i], b[j], acc[i][j]);
      }
      if (more) store(buf ^ 1);
      __syncthreads();
      buf ^= 1;
    }

    int64_t cm[TM], cn[TN];
#pragma unroll
    for (int i = 0; i < TM; ++i) {
      const int64_t m = m0 + ty * TM + i;
      cm[i] = m < g.M ? group_off(m, g.nm, g.m_ext, g.m_sc) : -1;
    }
#pragma unroll
    for (int j = 0; j < TN; ++j) {
      const int64_t n = n0 + tx * TN + j;
      cn[j] = n < g.N ? group_off(n, g.nn, g.n_ext, g.n_sc) : -1;
    }
#pragma unroll
    for (int i = 0; i < TM; ++i)
#pragma unroll
      for (int j = 0; j < TN; ++j)
        if (cm[i] >= 0 && cn[j] >= 0) {
          T* cp = Cp + lc + cm[i] + cn[j];
          *cp = epilogue<A>(acc[i][j], cp, sx, sy, g.sy_zero, g.sx_one);
        }
    __syncthreads();
  }
}

template <class A>
static cudaError_t launch_gemm_simt_t(const GemmArgs& g, cudaStream_t s) {
  using C = SimtCfg<sizeof(typename A::T)>;
  const int64_t gm = (g.M + C::BM - 1) / C::BM, gn = (g.N + C::BN - 1) / C::BN;
  if (gm > 0x7fffffff || gn > 65535) return cudaErrorNotSupported;
  const int64_t gl = g.L < 65535 ? g.L : 65535;
  dim3 grid((unsigned)gm, (unsigned)gn, (unsigned)gl);
  KernelTimer kt(s, "k_gemm_simt");
  k_gemm_simt<A><<<grid, 256, 0, s>>>(g); count_launch();
  return cudaGetLastError();
}

// Batched GEMM whose batch mode is the contiguous one in A, B and C (Julia
// column-major `bij,bjk->bik`: b fastest) with small M, N: lane = one of 32
// consecutive batches, so every load and store of a warp is one contiguous
// 128-byte row; warp w of 4 owns 4 rows of the block's 16 x 4 output tile
// and keeps 4 x 4 accumulators (small tiles: enough warps in flight to hide
// the L2 latency of the K loop, which is unrolled by 4; the fastest of the
// tilings timed on b=512, 64^3); the 4 warps read the same B rows, which the
// L1 serves after the first.  Plain algebra arithmetic in K order.
template <class T> __device__ __forceinline__ T ld_ro(const T* p) { return *p; }
template <> __device__ __forceinline__ float ld_ro<float>(const float* p) { return __ldg(p); }
template <> __device__ __forceinline__ double ld_ro<double>(const double* p) { return __ldg(p); }

// FULL: M % 16 == 0, N % 4 == 0 and L % 32 == 0 (no bounds tests in the loop)
template <class A, bool FULL>
__global__ void __launch_bounds__(128) k_gemm_bfast(const __grid_constant__ GemmArgs g) {
  using T = typename A::T;
  constexpr int TN = 4, RM = 4, WARPS = 4;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int64_t b = (int64_t)blockIdx.x * 32 + lane;
  if (!FULL && b >= g.L) return;
  const int n0 = blockIdx.y * TN;
  const int m0 = blockIdx.z * (RM * WARPS) + warp * RM;
  // one mode per group, 32-bit strides inside a batch (checked by the host)
  const int sma = (int)g.m_sa[0], smc = (int)g.m_sc[0], snb = (int)g.n_sb[0], snc = (int)g.n_sc[0];
  const int ska = (int)g.k_sa[0], skb = (int)g.k_sb[0];
  const int M = (int)g.M, N = (int)g.N, K = (int)g.K;
  const T* __restrict__ ap = static_cast<const T*>(g.A) + mode_offset(b, g.nl, g.l_ext, g.l_sa) + (int64_t)m0 * sma;
  const T* __restrict__ bp = static_cast<const T*>(g.B) + mode_offset(b, g.nl, g.l_ext, g.l_sb) + (int64_t)n0 * snb;
  T* cp0 = static_cast<T*>(g.C) + mode_offset(b, g.nl, g.l_ext, g.l_sc) + (int64_t)m0 * smc + (int64_t)n0 * snc;
  T acc[RM][TN];
#pragma unroll
  for (int r = 0; r < RM; ++r)
#pragma unroll
    for (int c = 0; c < TN; ++c) acc[r][c] = A::zero();
#pragma unroll 4
  for (int k = 0; k < K; ++k) {
    T av[RM], bv[TN];
#pragma unroll
    for (int r = 0; r < RM; ++r) av[r] = (FULL || m0 + r < M) ? ld_ro(ap + r * sma) : A::zero();
#pragma unroll
    for (int c = 0; c < TN; ++c) bv[c] = (FULL || n0 + c < N) ? ld_ro(bp + c * snb) : A::zero();
#pragma unroll
    for (int r = 0; r < RM; ++r)
#pragma unroll
      for (int c = 0; c < TN; ++c) acc[r][c] = A::add(acc[r][c], A::mul(av[r], bv[c]));
    ap += ska;
    bp += skb;
  }
  const T sx = scalar_as<T>(g.sx), sy = scalar_as<T>(g.sy);
#pragma unroll
  for (int r = 0; r < RM; ++r)
#pragma unroll
    for (int c = 0; c < TN; ++c)
      if (FULL || (m0 + r < M && n0 + c < N)) {
        T* cp = cp0 + r * smc + c * snc;
        *cp = epilogue<A>(acc[r][c], cp, sx, sy, g.sy_zero, g.sx_one);
      }
}

bool gemm_bfast_applies(const GemmArgs& g) {
  auto small = [](int64_t ext, int64_t str) { return ext * (str < 0 ? -str : str) < ((int64_t)1 << 30); };
  return g.l_sa[0] == 1 && g.l_sb[0] == 1 && g.l_sc[0] == 1 && g.l_ext[0] >= 32 && g.M <= 64 && g.N <= 64 &&
         g.K <= 1024 && g.L >= 32 && (g.L + 31) / 32 <= 0x7fffffff && g.nm == 1 && g.nn == 1 && g.nk == 1 &&
         small(g.M, g.m_sa[0]) && small(g.M, g.m_sc[0]) && small(g.N, g.n_sb[0]) && small(g.N, g.n_sc[0]) &&
         small(g.K, g.k_sa[0]) && small(g.K, g.k_sb[0]);
}

cudaError_t launch_gemm_bfast(ome_dtype dt, const GemmArgs& g, cudaStream_t s) {
  if (g.M == 0 || g.N == 0 || g.L == 0) return cudaSuccess;
  if (!gemm_bfast_applies(g)) return cudaErrorNotSupported;
  const dim3 grid((unsigned)((g.L + 31) / 32), (unsigned)((g.N + 3) / 4), (unsigned)((g.M + 15) / 16));
  cudaError_t e = cudaErrorInvalidValue;
  const bool full = g.M % 16 == 0 && g.N % 4 == 0 && g.L % 32 == 0;
  KernelTimer kt(s, "k_gemm_bfast");
  OME_DISPATCH(dt, ALG, {
    if (full) k_gemm_bfast<ALG, true><<<grid, 128, 0, s>>>(g);
    else k_gemm_bfast<ALG, false><<<grid, 128, 0, s>>>(g);
    count_launch();
    e = cudaGetLastError();
  });
  return e;
}

cudaError_t launch_gemm_simt_small_f32(const GemmArgs& g, cudaStream_t s) {
  if (g.M == 0 || g.N == 0 || g.L == 0) return cudaSuccess;
  if (g.M > SimtSmall::BM || g.N > SimtSmall::BN) return cudaErrorNotSupported;
  const int64_t gl = g.L < 65535 ? g.L : 65535;
  KernelTimer kt(s, "k_gemm_simt");
  k_gemm_simt<AlgF32, SimtSmall><<<dim3(1, 1, (unsigned)gl), 256, 0, s>>>(g);
  count_launch();
  return cudaGetLastError();
}

cudaError_t launch_gemm_simt(ome_dtype dt, const GemmArgs& g, cudaStream_t s) {
  if (g.M == 0 || g.N == 0 || g.L == 0) return cudaSuccess;
  cudaError_t e = cudaErrorInvalidValue;
  OME_DISPATCH(dt, ALG, e = launch_gemm_simt_t<ALG>(g, s));
  return e;
}

}  // namespace ome
