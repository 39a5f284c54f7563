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

// Split along K (for grids too small to fill the GPU): blockIdx.z runs over
// L x S, block (l, sp) sums k in [sp * kchunk, (sp + 1) * kchunk) and writes
// its tile to partial[((sp * L + l) * M + m) * N + n]; k_simt_splitk_finish
// adds the S partials in split order and applies the epilogue.
struct SimtSplit {
  int S;               // 1: no split
  int64_t kchunk;
  void* partial;
  int64_t p_elems;     // partial capacity in elements (self-check)
};
// set (5) when a split partial's offset falls outside the scratch (self-check)
__device__ int g_ome_bounds_simt = 0;

template <class A, class C = SimtCfg<sizeof(typename A::T)>>
__global__ void __launch_bounds__(256) k_gemm_simt(const __grid_constant__ GemmArgs g,
                                                    const __grid_constant__ SimtSplit sp) {
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

  const int64_t zsteps = g.L * sp.S;
  for (int64_t z = blockIdx.z; z < zsteps; z += gridDim.z) {
    const int64_t l = z % g.L, spi = z / g.L;
    const int64_t kbeg = spi * sp.kchunk;
    const int64_t kend = sp.S > 1 ? min(g.K, kbeg + sp.kchunk) : g.K;
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
        ra[r] = (base >= 0 && k < kend) ? Ap[base + group_off(k, g.nk, g.k_ext, g.k_sa)] : A::zero();
      }
#pragma unroll
      for (int r = 0; r < RB; ++r) {
        const int e = tid + NT * r;
        const int nn = g.b_n_fast ? e % BN : e / BK;
        const int kk = g.b_n_fast ? e / BN : e % BK;
        const int64_t k = k0 + kk;
        const int64_t base = bn[nn];
        rb[r] = (base >= 0 && k < kend) ? Bp[base + group_off(k, g.nk, g.k_ext, g.k_sb)] : A::zero();
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

    load(kbeg);
    store(0);
    __syncthreads();
    int buf = 0;
    for (int64_t k0 = kbeg; k0 < kend; k0 += BK) {
      const bool more = k0 + BK < kend;
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
    if (sp.S > 1) {
      T* pp = static_cast<T*>(sp.partial) + (spi * g.L + l) * g.M * g.N;
#pragma unroll
      for (int i = 0; i < TM; ++i)
#pragma unroll
        for (int j = 0; j < TN; ++j) {
          const int64_t m = m0 + ty * TM + i, n = n0 + tx * TN + j;
          if (m < g.M && n < g.N) {
            const int64_t po = (spi * g.L + l) * g.M * g.N + m * g.N + n;
            if (po < sp.p_elems) pp[m * g.N + n] = acc[i][j];
            else atomicCAS(&g_ome_bounds_simt, 0, 5);
          }
        }
    } else {
#pragma unroll
      for (int i = 0; i < TM; ++i)
#pragma unroll
        for (int j = 0; j < TN; ++j)
          if (cm[i] >= 0 && cn[j] >= 0) {
            T* cp = Cp + lc + cm[i] + cn[j];
            *cp = epilogue<A>(acc[i][j], cp, sx, sy, g.sy_zero, g.sx_one);
          }
    }
    __syncthreads();
  }
}

// Sum the S split partials of every output in split order; αβ epilogue.
template <class A>
__global__ void __launch_bounds__(256) k_simt_splitk_finish(const __grid_constant__ GemmArgs g,
                                                             const __grid_constant__ SimtSplit sp) {
  using T = typename A::T;
  const T* pp = static_cast<const T*>(sp.partial);
  T* Cp = static_cast<T*>(g.C);
  const T sx = scalar_as<T>(g.sx), sy = scalar_as<T>(g.sy);
  const int64_t per = g.L * g.M * g.N;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < per; i += (int64_t)gridDim.x * blockDim.x) {
    T acc = pp[i];
    for (int s = 1; s < sp.S; ++s) acc = A::add(acc, pp[s * per + i]);
    const int64_t n = i % g.N, r = i / g.N, m = r % g.M, l = r / g.M;
    T* cp = Cp + mode_offset(l, g.nl, g.l_ext, g.l_sc) + group_off(m, g.nm, g.m_ext, g.m_sc) +
            group_off(n, g.nn, g.n_ext, g.n_sc);
    *cp = epilogue<A>(acc, cp, sx, sy, g.sy_zero, g.sx_one);
  }
}

template <class A>
static cudaError_t launch_gemm_simt_t(const GemmArgs& g, cudaStream_t s) {
  using C = SimtCfg<sizeof(typename A::T)>;
  const int64_t gm = (g.M + C::BM - 1) / C::BM, gn = (g.N + C::BN - 1) / C::BN;
  if (gm > 0x7fffffff || gn > 65535) return cudaErrorNotSupported;
  SimtSplit sp{1, g.K, nullptr, 0};
  const int64_t gl = g.L < 65535 ? g.L : 65535;
  dim3 grid((unsigned)gm, (unsigned)gn, (unsigned)gl);
  KernelTimer kt(s, "k_gemm_simt");
  k_gemm_simt<A><<<grid, 256, 0, s>>>(g, sp); count_launch();
  return cudaGetLastError();
}

// The same with K split over blocks when the tiles alone would leave most
// SMs idle (long K, few tiles) and the partials fit `workspace`.
template <class A>
static cudaError_t launch_gemm_simt_ws_t(const GemmArgs& g, void* workspace, size_t ws_bytes, int num_sms,
                                         cudaStream_t s) {
  using T = typename A::T;
  using C = SimtCfg<sizeof(T)>;
  const int64_t gm = (g.M + C::BM - 1) / C::BM, gn = (g.N + C::BN - 1) / C::BN;
  const int64_t blocks = gm * gn * g.L;
  int64_t S = 1;
  if (blocks < num_sms && g.K >= 1024 && gn <= 65535 && gm <= 0x7fffffff) {
    S = std::min<int64_t>((2 * (int64_t)num_sms + blocks - 1) / blocks, g.K / 256);
    S = std::min<int64_t>(S, 65535 / std::max<int64_t>(g.L, 1));
    while (S > 1 && (size_t)S * g.L * g.M * g.N * sizeof(T) > ws_bytes) --S;
  }
  if (S <= 1) return launch_gemm_simt_t<A>(g, s);
  const int64_t kchunk = (g.K + S - 1) / S;
  S = (g.K + kchunk - 1) / kchunk;
  SimtSplit sp{(int)S, kchunk, workspace, (int64_t)S * g.L * g.M * g.N};
  dim3 grid((unsigned)gm, (unsigned)gn, (unsigned)(g.L * S));
  {
    KernelTimer kt(s, "k_gemm_simt");
    k_gemm_simt<A><<<grid, 256, 0, s>>>(g, sp);
  }
  count_launch();
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return e;
  const int64_t per = g.L * g.M * g.N;
  const int64_t nb = std::min<int64_t>((per + 255) / 256, (int64_t)num_sms * 16);
  k_simt_splitk_finish<A><<<(unsigned)nb, 256, 0, s>>>(g, sp);
  count_launch();
  return cudaGetLastError();
}

// Batched GEMM whose batch mode is the contiguous one in A, B and C (Julia
// column-major `bij,bjk->bik`: b fastest) with small M, N (<= 64).  A CTA of
// 256 threads owns 4 consecutive batches and an NS-column slab of N (64:
// all of it, for 4-byte types with N > 32; otherwise 32); K runs in chunks of 16 staged in shared memory
// (two buffers, the next chunk's global loads in registers while the current
// one is multiplied).  Staging loads walk the batch mode fastest (4 batches =
// 16 contiguous bytes for 4-byte types), so each element of A and B leaves
// L2 once per slab instead of once per register tile; each thread keeps
// 8 x NS/8 accumulators of one batch and reads its operands from shared
// memory as 16-byte broadcasts (B in runs of 4 columns, conflict-free).  The tile leaves through shared memory too,
// batch mode fastest.  Plain algebra arithmetic in K order.
template <class T, int N>
__device__ __forceinline__ void lds_run(const T* p, T (&v)[N]) {
  if constexpr ((sizeof(T) * N) % 16 == 0) {
    constexpr int W = (int)(sizeof(T) * N / 16);
    uint4 w[W];
    const uint4* q = reinterpret_cast<const uint4*>(p);
#pragma unroll
    for (int i = 0; i < W; ++i) w[i] = q[i];
    memcpy(v, w, sizeof(v));
  } else {
#pragma unroll
    for (int i = 0; i < N; ++i) v[i] = p[i];
  }
}

template <int NS_> struct BsCfg {
  static constexpr int NB = 4, KC = 16, NS = NS_, MT = 64, NT = 256;
  static constexpr int TR = 8, TC = NS / 8;          // thread tile: rows x columns
  static constexpr int KSTEP = 64 / NS;              // B staging: k rows lk0, lk0 + KSTEP, ...
  // every offset the compute reads (8*tm, 4*tn, 32, the strides below) is a
  // multiple of 4 elements, so its runs are 16-byte aligned for 4-byte and
  // wider types
  static constexpr int A_B = KC * MT + 8;            // elements per batch in an A stage (padded)
  static constexpr int B_B = KC * NS + 8;            // elements per batch in a B stage
  static constexpr int STAGE = NB * (A_B + B_B);
  static constexpr int C_ROW = MT + 1;               // epilogue tile: [batch][n][m], padded rows
  static constexpr int C_B = NS * C_ROW + 8;
  static constexpr int ELEMS = 2 * STAGE > NB * C_B ? 2 * STAGE : NB * C_B;
};

template <class A, bool FULL, int NS_>
__global__ void __launch_bounds__(256, 1) k_gemm_bstage(const __grid_constant__ GemmArgs g) {
  using Cf = BsCfg<NS_>;
  constexpr int NB = Cf::NB, KC = Cf::KC, NS = Cf::NS, MT = Cf::MT, TR = Cf::TR, TC = Cf::TC;
  constexpr int KSTEP = Cf::KSTEP, A_B = Cf::A_B, B_B = Cf::B_B, STAGE = Cf::STAGE, C_ROW = Cf::C_ROW,
                C_B = Cf::C_B;
  using T = typename A::T;
  extern __shared__ __align__(16) unsigned char bs_raw[];
  T* sm = reinterpret_cast<T*>(bs_raw);
  const int t = threadIdx.x;
  const int64_t b0 = (int64_t)blockIdx.x * NB;
  const int n0 = blockIdx.y * NS;
  const int M = (int)g.M, N = (int)g.N, K = (int)g.K;
  const int sma = (int)g.m_sa[0], ska = (int)g.k_sa[0], snb = (int)g.n_sb[0], skb = (int)g.k_sb[0];
  // staging roles: batch lb of the group; A row lm (all 16 k of a chunk);
  // B column ln, k rows lk0 + KSTEP*q
  const int lb = t & 3, lm = t >> 2, ln = (t >> 2) % NS, lk0 = (t >> 2) / NS;
  const bool bok = FULL || b0 + lb < g.L;
  const T* ga = static_cast<const T*>(g.A);
  const T* gb = static_cast<const T*>(g.B);
  if (bok) {
    ga += mode_offset(b0 + lb, g.nl, g.l_ext, g.l_sa) + (int64_t)lm * sma;
    gb += mode_offset(b0 + lb, g.nl, g.l_ext, g.l_sb) + (int64_t)(n0 + ln) * snb + (int64_t)lk0 * skb;
  }
  const bool aok = bok && (FULL || lm < M), bnok = bok && (FULL || n0 + ln < N);
  T ra[KC], rb[KC / KSTEP];
  auto load = [&](int k0) {
#pragma unroll
    for (int q = 0; q < KC; ++q)
      ra[q] = aok && (FULL || k0 + q < K) ? ga[(int64_t)(k0 + q) * ska] : A::zero();
#pragma unroll
    for (int q = 0; q < KC / KSTEP; ++q)
      rb[q] = bnok && (FULL || k0 + lk0 + KSTEP * q < K) ? gb[(int64_t)(k0 + KSTEP * q) * skb] : A::zero();
  };
  auto store = [&](int st) {
    T* as = sm + st * STAGE + lb * A_B + lm;
    T* bsm = sm + st * STAGE + NB * A_B + lb * B_B + lk0 * NS + ln;
#pragma unroll
    for (int q = 0; q < KC; ++q) as[q * MT] = ra[q];
#pragma unroll
    for (int q = 0; q < KC / KSTEP; ++q) bsm[KSTEP * q * NS] = rb[q];
  };
  // 16-byte types (complex128) stage straight from global memory after the
  // multiply: the accumulators leave no registers for a prefetch
  constexpr bool PREF = sizeof(T) < 16;
  auto load_store = [&](int k0, int st) {
    T* as = sm + st * STAGE + lb * A_B + lm;
    T* bsm = sm + st * STAGE + NB * A_B + lb * B_B + lk0 * NS + ln;
#pragma unroll 4
    for (int q = 0; q < KC; ++q)
      as[q * MT] = aok && (FULL || k0 + q < K) ? ga[(int64_t)(k0 + q) * ska] : A::zero();
#pragma unroll 4
    for (int q = 0; q < KC / KSTEP; ++q)
      bsm[KSTEP * q * NS] =
          bnok && (FULL || k0 + lk0 + KSTEP * q < K) ? gb[(int64_t)(k0 + KSTEP * q) * skb] : A::zero();
  };
  // compute roles: batch cb, rows TR*tm.., columns 4*tn.. (and 32 + 4*tn..
  // for 8-column tiles: a warp's 16-byte reads of B stay in one 128-byte row
  // of banks)
  const int cb = t >> 6, tm = (t >> 3) & 7, tn = t & 7;
  T acc[TR][TC];
#pragma unroll
  for (int r = 0; r < TR; ++r)
#pragma unroll
    for (int c = 0; c < TC; ++c) acc[r][c] = A::zero();
  const int nchunks = (K + KC - 1) / KC;
  if (PREF) {
    load(0);
    store(0);
  } else {
    load_store(0, 0);
  }
  __syncthreads();
  for (int ch = 0; ch < nchunks; ++ch) {
    const int st = ch & 1;
    if (PREF && ch + 1 < nchunks) load((ch + 1) * KC);
    const T* as = sm + st * STAGE + cb * A_B + TR * tm;
    const T* bsm = sm + st * STAGE + NB * A_B + cb * B_B + 4 * tn;
#pragma unroll 2
    for (int kk = 0; kk < KC; ++kk) {
      T av[TR], bv[TC];
      lds_run(as + kk * MT, av);
#pragma unroll
      for (int h = 0; h < TC / 4; ++h) {
        T b4[4];
        lds_run(bsm + kk * NS + 32 * h, b4);
#pragma unroll
        for (int c = 0; c < 4; ++c) bv[4 * h + c] = b4[c];
      }
#pragma unroll
      for (int r = 0; r < TR; ++r)
#pragma unroll
        for (int c = 0; c < TC; ++c) acc[r][c] = A::add(acc[r][c], A::mul(av[r], bv[c]));
    }
    if (ch + 1 < nchunks) {
      if (PREF) store(st ^ 1);
      else load_store((ch + 1) * KC, st ^ 1);
    }
    __syncthreads();
  }
  // tile -> shared [batch][n][m] -> C with the batch mode fastest
  {
    T* cs = sm + cb * C_B + (4 * tn) * C_ROW + TR * tm;
#pragma unroll
    for (int c = 0; c < TC; ++c)
#pragma unroll
      for (int r = 0; r < TR; ++r) cs[((c >> 2) * 32 + (c & 3)) * C_ROW + r] = acc[r][c];
  }
  __syncthreads();
  if (!bok || !(FULL || lm < M)) return;
  const T sx = scalar_as<T>(g.sx), sy = scalar_as<T>(g.sy);
  T* cp = static_cast<T*>(g.C) + mode_offset(b0 + lb, g.nl, g.l_ext, g.l_sc) + (int64_t)lm * g.m_sc[0] +
          (int64_t)n0 * g.n_sc[0];
  const T* cs = sm + lb * C_B + lm;
  const int nn = FULL ? NS : min(NS, N - n0);
  for (int q = 0; q < nn; ++q) {
    T* yp = cp + (int64_t)q * g.n_sc[0];
    *yp = epilogue<A>(cs[q * C_ROW], yp, sx, sy, g.sy_zero, g.sx_one);
  }
}

bool gemm_bfast_applies(const GemmArgs& g) {
  auto small = [](int64_t ext, int64_t str) { return ext * (str < 0 ? -str : str) < ((int64_t)1 << 30); };
  return g.l_sa[0] == 1 && g.l_sb[0] == 1 && g.l_sc[0] == 1 && g.l_ext[0] >= 32 && g.M <= 64 && g.N <= 64 &&
         g.K <= 1024 && g.L >= 32 && (g.L + 31) / 32 <= 0x7fffffff && g.nm == 1 && g.nn == 1 && g.nk == 1 &&
         small(g.M, g.m_sa[0]) && small(g.M, g.m_sc[0]) && small(g.N, g.n_sb[0]) && small(g.N, g.n_sc[0]) &&
         small(g.K, g.k_sa[0]) && small(g.K, g.k_sb[0]);
}

template <class A, int NS>
static cudaError_t launch_gemm_bstage_t(const GemmArgs& g, cudaStream_t s) {
  using Cf = BsCfg<NS>;
  const size_t smem = (size_t)Cf::ELEMS * sizeof(typename A::T);
  static std::atomic<unsigned long long> attr_full{0}, attr_part{0};
  cudaError_t e = set_smem_once(attr_full, k_gemm_bstage<A, true, NS>, (int)smem);
  if (e == cudaSuccess) e = set_smem_once(attr_part, k_gemm_bstage<A, false, NS>, (int)smem);
  if (e != cudaSuccess) return e;
  const dim3 grid((unsigned)((g.L + Cf::NB - 1) / Cf::NB), (unsigned)((g.N + NS - 1) / NS));
  const bool full = g.M == Cf::MT && g.N % NS == 0 && g.K % Cf::KC == 0 && g.L % Cf::NB == 0;
  if (full) k_gemm_bstage<A, true, NS><<<grid, Cf::NT, smem, s>>>(g);
  else k_gemm_bstage<A, false, NS><<<grid, Cf::NT, smem, s>>>(g);
  count_launch();
  return cudaGetLastError();
}

// 64-column slabs (8 x 8 thread tiles) for types of at most 4 bytes; wider
// types keep 8 x 4 tiles, whose accumulators already fill the registers
template <class A>
static cudaError_t launch_gemm_bstage(const GemmArgs& g, cudaStream_t s) {
  if constexpr (sizeof(typename A::T) <= 4) {
    if (g.N > 32) return launch_gemm_bstage_t<A, 64>(g, s);
  }
  return launch_gemm_bstage_t<A, 32>(g, s);
}

cudaError_t launch_gemm_bfast(ome_dtype dt, const GemmArgs& g, cudaStream_t s) {
  if (g.M == 0 || g.N == 0 || g.L == 0) return cudaSuccess;
  if (!gemm_bfast_applies(g)) return cudaErrorNotSupported;
  cudaError_t e = cudaErrorInvalidValue;
  KernelTimer kt(s, "k_gemm_bstage");
  OME_DISPATCH(dt, ALG, e = launch_gemm_bstage<ALG>(g, s));
  return e;
}

cudaError_t launch_gemm_simt_small_f32(const GemmArgs& g, cudaStream_t s) {
  if (g.M == 0 || g.N == 0 || g.L == 0) return cudaSuccess;
  if (g.M > SimtSmall::BM || g.N > SimtSmall::BN) return cudaErrorNotSupported;
  const int64_t gl = g.L < 65535 ? g.L : 65535;
  KernelTimer kt(s, "k_gemm_simt");
  k_gemm_simt<AlgF32, SimtSmall><<<dim3(1, 1, (unsigned)gl), 256, 0, s>>>(g, SimtSplit{1, g.K, nullptr, 0});
  count_launch();
  return cudaGetLastError();
}

// Read and clear the split-partial self-check flag (0 = no violation).
int simt_bounds_flag() {
  int v = 0;
  if (cudaMemcpyFromSymbol(&v, g_ome_bounds_simt, sizeof(int)) != cudaSuccess) return 0;
  if (v) {
    const int zero = 0;
    cudaMemcpyToSymbol(g_ome_bounds_simt, &zero, sizeof(int));
  }
  return v;
}

cudaError_t launch_gemm_simt_ws(ome_dtype dt, const GemmArgs& g, void* workspace, size_t ws_bytes, int num_sms,
                                cudaStream_t s) {
  cudaError_t e = cudaErrorInvalidValue;
  OME_DISPATCH(dt, ALG, e = launch_gemm_simt_ws_t<ALG>(g, workspace, ws_bytes, num_sms, s));
  return e;
}

cudaError_t launch_gemm_simt(ome_dtype dt, const GemmArgs& g, cudaStream_t s) {
  if (g.M == 0 || g.N == 0 || g.L == 0) return cudaSuccess;
  cudaError_t e = cudaErrorInvalidValue;
  OME_DISPATCH(dt, ALG, e = launch_gemm_simt_t<ALG>(g, s));
  return e;
}

}  // namespace ome
