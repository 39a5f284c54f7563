// Tensor-core FP32 contraction from BF16 split products (sm_100a tcgen05):
// BF16x3 (2 terms per value, 3 MMAs) or BF16x6 (3 terms, 6 MMAs).
//
// Replaces the GEMM at the heart of OMEinsum's binary path
// (src/einsum.jl:104-124 -> src/binaryrules.jl mul!/_batched_gemm!, on GPU
// CUBLAS gemm / gemm_strided_batched, ext/CUDAExt.jl:115-117,156-178).
//
// Design:
//  * operands are read in place from the input tensors through per-group
//    mode strides (the permutation of simplifyto, src/einsum.jl:127-134, is
//    absorbed in the addressing; nothing is written back to HBM);
//  * 16 converter warps load FP32 from global memory (coalesced along the
//    operand's contiguous mode), split each value x into hi = bf16(x) and
//    lo = bf16(x - hi) (and a third term for BF16x6) and store them into shared memory in the UMMA K-major
//    no-swizzle canonical layout (8-row x 16-byte core matrices);
//    with two stages of loads in flight per thread;
//  * one elected thread of a seventeenth warp issues, per K=16 step, three
//    (BF16x3: hi*hi + hi*lo + lo*hi) or six (BF16x6: every term pair whose
//    orders sum below 3) tcgen05.mma kind::f16 accumulating in FP32 in
//    tensor memory; tcgen05.commit releases each shared-memory stage;
//  * TMEM holds two buffers of (main = t0*t0, cross = other term pairs)
//    accumulators; every CHUNK k-steps the converter warps drain the finished
//    buffer (tcgen05.ld) into FP32 running sums in shared memory with
//    round-to-nearest CUDA-core adds -- the tensor core's accumulation then
//    only ever spans CHUNK k-steps, which keeps BF16x6 FP32-faithful;
//  * the epilogue applies the y <- sy*y + sx*f epilogue through the
//    output's mode strides, or write a split-K partial that a second kernel
//    sums in a fixed order (deterministic);
//  * every mbarrier wait is bounded (about 2 s of %globaltimer); on expiry the
//    kernel records g_ome_timeout, stops waiting and frees its TMEM.
#include <cuda.h>
#include <cuda_bf16.h>
#include <string.h>
#include <mutex>
#include "kernels.h"

namespace ome {

__device__ int g_ome_timeout = 0;
// First kernel that found an output offset outside its view and skipped the
// store (self-check of the epilogues; 0 = none); read and cleared by
// device_status.
__device__ int g_ome_bounds = 0;
__device__ __forceinline__ bool in_bounds(int64_t off, int64_t hi, int id) {
  if (off >= 0 && off <= hi) return true;
  atomicCAS(&g_ome_bounds, 0, id);
  return false;
}

namespace tc {
constexpr int BM = 128, BN = 128, BK = 32;
constexpr int CHUNK = 8;                   // k-steps accumulated in TMEM between drains
constexpr int ACC_BYTES = BM * BN * 4;     // FP32 running sums in shared memory
template <int NT> struct Cfg {             // NT = bf16 terms per value (2: BF16x3, 3: BF16x6)
  static constexpr int STAGE_BYTES = 2 * NT * BM * BK * 2;   // A terms then B terms
  static constexpr int STAGES = NT == 2 ? 4 : 3;
  static constexpr int SMEM_BYTES = STAGES * STAGE_BYTES + ACC_BYTES + 256;
};
constexpr int PREF = 2;                    // stages of FP32 loads in flight per converter thread
constexpr int NCONV = 512;                 // converter + epilogue threads (16 warps)
constexpr int NTHREADS = NCONV + 32;       // + one MMA-issue warp
constexpr int TILE_BYTES = BM * BK * 2;    // one bf16 operand tile (one term): 8 KB
constexpr int TMEM_COLS = 512;            // 2 buffers x (main, cross-term) 128-column accumulators
constexpr unsigned long long WAIT_NS = 2000000000ull;
// kind::f16, BF16 x BF16 -> F32, K-major A and B, M = 128, N = 128
constexpr uint32_t IDESC = (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(BN >> 3) << 17) |
                           ((uint32_t)(BM >> 4) << 24);
}  // namespace tc

struct TcArgs {
  GemmArgs g;
  int S;               // K splits
  int64_t kchunk;      // K elements per split (multiple of BK)
  float* partial;      // S > 1: [S][L][N][M] partial sums
  int a_kfast, b_kfast;  // the operand's first K mode is contiguous and a multiple of 8 long
};

__device__ __forceinline__ uint32_t smem_u32(const void* p) {
  return (uint32_t)__cvta_generic_to_shared(p);
}
__device__ __forceinline__ uint64_t gtimer() {
  uint64_t t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}
__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}
__device__ __forceinline__ void mbar_arrive(uint64_t* bar) {
  asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_u32(bar)) : "memory");
}
__device__ __forceinline__ bool mbar_try_wait(uint64_t* bar, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
      "selp.u32 %0, 1, 0, p;\n\t}\n"
      : "=r"(ok)
      : "r"(smem_u32(bar)), "r"(parity)
      : "memory");
  return ok != 0;
}
// Bounded wait: false once the block has given up (abort flag set by any thread).
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, uint32_t parity, volatile int* abort_flag) {
  if (mbar_try_wait(bar, parity)) return true;
  const uint64_t t0 = gtimer();
  while (true) {
#pragma unroll 1
    for (int i = 0; i < 32; ++i)
      if (mbar_try_wait(bar, parity)) return true;
    if (*abort_flag) return false;
    if (gtimer() - t0 > tc::WAIT_NS) {
      *abort_flag = 1;
      atomicExch(&g_ome_timeout, 1);
      return false;
    }
  }
}
__device__ __forceinline__ void fence_proxy_async() {
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}
__device__ __forceinline__ void tc_fence_before() {
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
}
__device__ __forceinline__ void tc_fence_after() {
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
}
__device__ __forceinline__ uint64_t umma_desc(uint32_t saddr) {
  // K-major, no swizzle: LBO = 128 B between K-adjacent core matrices,
  // SBO = 512 B between 8-row groups (4 K-chunks of a BK=32 row group).
  return (uint64_t)((saddr >> 4) & 0x3FFF) | ((uint64_t)(128 >> 4) << 16) | ((uint64_t)(512 >> 4) << 32) |
         (1ull << 46);
}
__device__ __forceinline__ void umma_bf16(uint32_t d_tmem, uint64_t a, uint64_t b, uint32_t acc) {
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "setp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}\n" ::"r"(d_tmem),
      "l"(a), "l"(b), "r"(tc::IDESC), "r"(acc));
}
__device__ __forceinline__ void umma_commit(uint64_t* bar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
                   smem_u32(bar))
               : "memory");
}
__device__ __forceinline__ void tmem_ld16(uint32_t taddr, uint32_t (&r)[16]) {
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x16.b32 "
      "{%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
        "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
      : "r"(taddr));
  asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
}
__device__ __forceinline__ void tmem_ld32(uint32_t taddr, uint32_t (&r)[32]) {
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x32.b32 "
      "{%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15,"
      "%16,%17,%18,%19,%20,%21,%22,%23,%24,%25,%26,%27,%28,%29,%30,%31}, [%32];"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
        "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15]),
        "=r"(r[16]), "=r"(r[17]), "=r"(r[18]), "=r"(r[19]), "=r"(r[20]), "=r"(r[21]), "=r"(r[22]), "=r"(r[23]),
        "=r"(r[24]), "=r"(r[25]), "=r"(r[26]), "=r"(r[27]), "=r"(r[28]), "=r"(r[29]), "=r"(r[30]), "=r"(r[31])
      : "r"(taddr));
  asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
}

__device__ __forceinline__ int64_t goff(int64_t i, int n, const int64_t* ext, const int64_t* str) {
  if (n == 1) return i * str[0];
  return mode_offset(i, n, ext, str);
}

// C offsets of row m / column n (through the tables when present).
__device__ __forceinline__ int64_t c_moff(const GemmArgs& g, int64_t m) {
  return g.m_tab_c ? g.m_tab_c[m] : goff(m, g.nm, g.m_ext, g.m_sc);
}
__device__ __forceinline__ int64_t c_noff(const GemmArgs& g, int64_t n) {
  return g.n_tab_c ? g.n_tab_c[n] : goff(n, g.nn, g.n_ext, g.n_sc);
}

// Split 8 values into NT bf16 terms, x ~ t0 + t1 (+ t2): t0 = bf16_rn(x),
// t1 = bf16_rn(x - t0), t2 = bf16_rn(x - t0 - t1); 16 B per term.  Packed:
// one cvt.rn.bf16x2 per pair and term, terms widened back by bit shifts,
// residuals by one packed FMA each (exact).  Non-finite inputs give NaN
// residuals (the FP32 path keeps IEEE infinities).
template <int NT>
__device__ __forceinline__ void split8(const float (&v)[8], uint4 (&out)[NT]) {
  uint32_t w[NT][4];
#pragma unroll
  for (int p = 0; p < 4; ++p) {
    float2 r = make_float2(v[2 * p], v[2 * p + 1]);
#pragma unroll
    for (int t = 0; t < NT; ++t) {
      __nv_bfloat162 b = __float22bfloat162_rn(r);
      const uint32_t u = *reinterpret_cast<uint32_t*>(&b);
      w[t][p] = u;
      if (t + 1 < NT) {
        const float2 bf = make_float2(__uint_as_float(u << 16), __uint_as_float(u & 0xffff0000u));
        r = __ffma2_rn(bf, make_float2(-1.f, -1.f), r);
      }
    }
  }
#pragma unroll
  for (int t = 0; t < NT; ++t) out[t] = make_uint4(w[t][0], w[t][1], w[t][2], w[t][3]);
}

// Load one unit: 8 consecutive k (k0 .. k0+7) of one row.  rowoff < 0: a row
// beyond the extent (zeros).  kfast: the first K mode is contiguous and a
// multiple of 8 long, so the unit is 8 consecutive floats.
__device__ __forceinline__ void load_unit(const float* __restrict__ base, int64_t rowoff, int64_t k0, int64_t kend,
                                          int kfast, int nk, const int64_t* kext, const int64_t* kstr,
                                          float (&v)[8]) {
  if (rowoff < 0) {
#pragma unroll
    for (int i = 0; i < 8; ++i) v[i] = 0.f;
    return;
  }
  if (k0 + 8 <= kend) {
    if (kfast) {
      const float* p = base + rowoff + goff(k0, nk, kext, kstr);
      if ((reinterpret_cast<uintptr_t>(p) & 15) == 0) {
        const float4 a = __ldg(reinterpret_cast<const float4*>(p));
        const float4 b = __ldg(reinterpret_cast<const float4*>(p) + 1);
        v[0] = a.x; v[1] = a.y; v[2] = a.z; v[3] = a.w;
        v[4] = b.x; v[5] = b.y; v[6] = b.z; v[7] = b.w;
      } else {
#pragma unroll
        for (int i = 0; i < 8; ++i) v[i] = __ldg(p + i);
      }
      return;
    }
    if (nk == 1) {
      const int64_t sk = kstr[0];
      const float* p = base + rowoff + k0 * sk;
#pragma unroll
      for (int i = 0; i < 8; ++i) v[i] = __ldg(p + i * sk);
      return;
    }
  }
#pragma unroll
  for (int i = 0; i < 8; ++i) {
    const int64_t k = k0 + i;
    v[i] = k < kend ? __ldg(base + rowoff + goff(k, nk, kext, kstr)) : 0.f;
  }
}

__device__ __forceinline__ void sts128(uint32_t addr, const uint4& v) {
  asm volatile("st.shared.v4.b32 [%0], {%1, %2, %3, %4};" ::"r"(addr), "r"(v.x), "r"(v.y), "r"(v.z), "r"(v.w)
               : "memory");
}

template <int NT>
__global__ void __launch_bounds__(tc::NTHREADS, 1) k_gemm_bf16x3(const __grid_constant__ TcArgs t) {
  using namespace tc;
  constexpr int STAGES = Cfg<NT>::STAGES, STAGE_BYTES = Cfg<NT>::STAGE_BYTES;
  extern __shared__ __align__(1024) unsigned char smem[];
  float* acc = reinterpret_cast<float*>(smem + STAGES * STAGE_BYTES);   // [BN][BM] running sums
  uint64_t* full = reinterpret_cast<uint64_t*>(smem + STAGES * STAGE_BYTES + ACC_BYTES);
  uint64_t* empty = full + STAGES;
  uint64_t* chunk_done = empty + STAGES;   // [2]: a TMEM buffer's chunk of MMAs completed
  uint64_t* drained = chunk_done + 2;      // [2]: the converters have read that buffer
  uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(drained + 2);
  volatile int* abort_flag = reinterpret_cast<volatile int*>(tmem_slot + 1);

  const GemmArgs& g = t.g;
  const int tid = threadIdx.x;
  const int warp = tid >> 5, lane = tid & 31;
  const int64_t m0 = (int64_t)blockIdx.x * BM, n0 = (int64_t)blockIdx.y * BN;
  const int64_t z = blockIdx.z;
  const int64_t l = z / t.S;
  const int64_t split = z - l * t.S;
  const int64_t kbeg = split * t.kchunk;
  const int64_t kend = min(g.K, kbeg + t.kchunk);
  const int nkt = (int)((kend - kbeg + BK - 1) / BK);
  const int nchunks = (nkt + CHUNK - 1) / CHUNK;

  if (tid == 0) {
    for (int s = 0; s < STAGES; ++s) {
      mbar_init(&full[s], NCONV);
      mbar_init(&empty[s], 1);
    }
    for (int b = 0; b < 2; ++b) {
      mbar_init(&chunk_done[b], 1);
      mbar_init(&drained[b], NCONV);
    }
    *abort_flag = 0;
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  if (warp == NCONV / 32) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(tmem_slot)),
                 "r"(TMEM_COLS)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = *tmem_slot;
  // TMEM buffer b: main accumulator (t0*t0) at column 256b, cross terms at 256b + 128
  auto tmem_main = [&](int b) { return tmem + (uint32_t)(256 * b); };
  auto tmem_cross = [&](int b) { return tmem + (uint32_t)(256 * b + 128); };

  const float* Ap = static_cast<const float*>(g.A);
  const float* Bp = static_cast<const float*>(g.B);
  const int64_t la = mode_offset(l, g.nl, g.l_ext, g.l_sa);
  const int64_t lb = mode_offset(l, g.nl, g.l_ext, g.l_sb);

  if (warp < NCONV / 32) {
    // ---------------- converters ----------------
    // One unit (8 consecutive k of one row) of each operand per thread and
    // stage.  K-contiguous operand: a warp covers 8 rows x 4 k-chunks (each
    // row's 128 B read by 4 lanes); otherwise 32 consecutive rows of one
    // k-chunk.  Either way each quarter-warp stores 8 rows of one k-chunk =
    // one contiguous 128-byte core matrix (no bank conflicts).
    int arow, akc, brow, bkc;
    if (t.a_kfast) { arow = 8 * warp + (lane & 7); akc = lane >> 3; }
    else { arow = 32 * (warp & 3) + lane; akc = warp >> 2; }
    if (t.b_kfast) { brow = 8 * warp + (lane & 7); bkc = lane >> 3; }
    else { brow = 32 * (warp & 3) + lane; bkc = warp >> 2; }
    const int64_t am = m0 + arow, bn = n0 + brow;
    const int64_t aoff = am < g.M ? la + goff(am, g.nm, g.m_ext, g.m_sa) : -1;
    const int64_t boff = bn < g.N ? lb + goff(bn, g.nn, g.n_ext, g.n_sb) : -1;
    const uint32_t aso = (uint32_t)((((arow >> 3) * 4 + akc) * 8 + (arow & 7)) * 16);
    const uint32_t bso = (uint32_t)((((brow >> 3) * 4 + bkc) * 8 + (brow & 7)) * 16);
    const uint32_t sbase = smem_u32(smem);
    // accumulator lanes / columns of this thread (TMEM lane quarter = warp & 3)
    const int q = warp & 3, col = 32 * (warp >> 2);
    const int row = 32 * q + lane;

    // Drain chunk c: its TMEM buffer -> the FP32 running sums in shared memory
    // (round-to-nearest CUDA-core additions), then release the buffer.
    int drained_chunks = 0;
    auto drain = [&](int c) {
      const int b = c & 1;
      mbar_wait(&chunk_done[b], (uint32_t)((c >> 1) & 1), abort_flag);
      tc_fence_after();
#pragma unroll
      for (int h = 0; h < 2; ++h) {
        uint32_t rm[16], rc[16];
        __syncwarp();
        tmem_ld16(tmem_main(b) + ((uint32_t)(32 * q) << 16) + (uint32_t)(col + 16 * h), rm);
        tmem_ld16(tmem_cross(b) + ((uint32_t)(32 * q) << 16) + (uint32_t)(col + 16 * h), rc);
#pragma unroll
        for (int j = 0; j < 16; ++j) {
          const float v = __uint_as_float(rm[j]) + __uint_as_float(rc[j]);
          float* a = acc + (col + 16 * h + j) * BM + row;
          *a = c == 0 ? v : *a + v;
        }
      }
      tc_fence_before();
      mbar_arrive(&drained[b]);
    };

    float ring[PREF + 1][2][8];
    auto load_stage = [&](int kt, float (&dst)[2][8]) {
      if (kt < nkt) {
        const int64_t kb = kbeg + (int64_t)kt * BK;
        load_unit(Ap, aoff, kb + akc * 8, kend, t.a_kfast, g.nk, g.k_ext, g.k_sa, dst[0]);
        load_unit(Bp, boff, kb + bkc * 8, kend, t.b_kfast, g.nk, g.k_ext, g.k_sb, dst[1]);
      }
    };
    auto convert_stage = [&](int kt, const float (&src)[2][8]) {
      // chunk c - 2 must be drained before the MMAs of chunk c reuse its buffer
      if (kt % CHUNK == 0 && kt >= 2 * CHUNK) drain(drained_chunks++);
      const int s = kt % STAGES;
      if (kt >= STAGES) mbar_wait(&empty[s], (uint32_t)((kt / STAGES - 1) & 1), abort_flag);
      const uint32_t st = sbase + s * STAGE_BYTES;
      uint4 terms[NT];
      split8<NT>(src[0], terms);
#pragma unroll
      for (int u = 0; u < NT; ++u) sts128(st + u * TILE_BYTES + aso, terms[u]);
      split8<NT>(src[1], terms);
#pragma unroll
      for (int u = 0; u < NT; ++u) sts128(st + (NT + u) * TILE_BYTES + bso, terms[u]);
      fence_proxy_async();
      mbar_arrive(&full[s]);
    };
#pragma unroll
    for (int p = 0; p < PREF; ++p) load_stage(p, ring[p]);
    for (int kt = 0; kt < nkt; kt += PREF + 1) {
#pragma unroll
      for (int j = 0; j <= PREF; ++j) {
        if (kt + j < nkt) {
          load_stage(kt + j + PREF, ring[(j + PREF) % (PREF + 1)]);
          convert_stage(kt + j, ring[j]);
        }
      }
    }
    while (drained_chunks < nchunks) drain(drained_chunks++);
    // ---------------- epilogue ----------------
    const int64_t m = m0 + row;
    if (m < g.M) {
      const int64_t lc = mode_offset(l, g.nl, g.l_ext, g.l_sc);
      const int64_t cm = c_moff(g, m);
      float* Cp = static_cast<float*>(g.C);
      const float sx = scalar_as<float>(g.sx), sy = scalar_as<float>(g.sy);
#pragma unroll 4
      for (int j = 0; j < 32; ++j) {
        const int64_t n = n0 + col + j;
        if (n >= g.N) break;
        const float v = nchunks > 0 ? acc[(col + j) * BM + row] : 0.f;
        if (t.S > 1) {
          t.partial[((split * g.L + l) * g.N + n) * g.M + m] = v;
        } else {
          float* cp = Cp + lc + cm + c_noff(g, n);
          float o = g.sx_one ? v : sx * v;
          if (!g.sy_zero) o = fmaf(sy, *cp, o);
          *cp = o;
        }
      }
    }
  } else if (lane == 0) {
    // ---------------- MMA issue (one thread of the last warp) ----------------
    // Per K=16 step: t0*t0 into the chunk's main accumulator, the other term
    // pairs (i + j < NT) into its cross-term accumulator; each chunk starts
    // both from zero, so TMEM only ever sums CHUNK k-steps.
    const uint32_t sbase = smem_u32(smem);
    for (int kt = 0; kt < nkt; ++kt) {
      const int c = kt / CHUNK, b = c & 1;
      const bool first = kt % CHUNK == 0;
      if (first && c >= 2 && !mbar_wait(&drained[b], (uint32_t)(((c >> 1) - 1) & 1), abort_flag)) break;
      const int s = kt % STAGES;
      if (!mbar_wait(&full[s], (uint32_t)((kt / STAGES) & 1), abort_flag)) break;
      tc_fence_after();
      const uint32_t sb = sbase + s * STAGE_BYTES;
#pragma unroll
      for (int kk = 0; kk < 2; ++kk) {
        const uint32_t off = kk * 256;
        uint64_t ad[NT], bd[NT];
#pragma unroll
        for (int u = 0; u < NT; ++u) {
          ad[u] = umma_desc(sb + u * TILE_BYTES + off);
          bd[u] = umma_desc(sb + (NT + u) * TILE_BYTES + off);
        }
        const uint32_t keep = (first && kk == 0) ? 0u : 1u;
        umma_bf16(tmem_main(b), ad[0], bd[0], keep);
        bool first_cross = true;
#pragma unroll
        for (int d = 1; d < NT; ++d)
#pragma unroll
          for (int i = 0; i <= d; ++i) {
            umma_bf16(tmem_cross(b), ad[i], bd[d - i], first_cross ? keep : 1u);
            first_cross = false;
          }
      }
      umma_commit(&empty[s]);
      if (kt % CHUNK == CHUNK - 1 || kt == nkt - 1) umma_commit(&chunk_done[b]);
    }
  }
  tc_fence_before();
  __syncthreads();
  if (warp == NCONV / 32) {
    tc_fence_after();
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(TMEM_COLS) : "memory");
  }
}

// Sum the S partials of each output element in split order; αβ epilogue.
__global__ void __launch_bounds__(256) k_splitk_reduce(const __grid_constant__ TcArgs t) {
  const GemmArgs& g = t.g;
  const float sx = scalar_as<float>(g.sx), sy = scalar_as<float>(g.sy);
  float* Cp = static_cast<float*>(g.C);
  const int64_t total = g.M * g.N * g.L;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < total;
       i += (int64_t)gridDim.x * blockDim.x) {
    const int64_t m = i % g.M;
    const int64_t r = i / g.M;
    const int64_t n = r % g.N;
    const int64_t l = r / g.N;
    float acc = 0.f;
    for (int s = 0; s < t.S; ++s) acc += t.partial[((s * g.L + l) * g.N + n) * g.M + m];
    float* cp = Cp + mode_offset(l, g.nl, g.l_ext, g.l_sc) + c_moff(g, m) +
                c_noff(g, n);
    float o = g.sx_one ? acc : sx * acc;
    if (!g.sy_zero) o = fmaf(sy, *cp, o);
    *cp = o;
  }
}

// m -> C offset of m and n -> C offset of n for groups of several modes.
__global__ void __launch_bounds__(256) k_c_offsets(const __grid_constant__ GemmArgs g, int64_t* mt, int64_t* nt) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < g.M + g.N;
       i += (int64_t)gridDim.x * blockDim.x) {
    if (i < g.M) mt[i] = mode_offset(i, g.nm, g.m_ext, g.m_sc);
    else nt[i - g.M] = mode_offset(i - g.M, g.nn, g.n_ext, g.n_sc);
  }
}

cudaError_t launch_c_offsets(GemmArgs& g, int64_t* tab, cudaStream_t s) {
  const int64_t n = g.M + g.N;
  const int64_t nb = (n + 255) / 256;
  k_c_offsets<<<(unsigned)(nb < 4096 ? nb : 4096), 256, 0, s>>>(g, tab, tab + g.M);
  count_launch();
  g.m_tab_c = tab;
  g.n_tab_c = tab + g.M;
  return cudaGetLastError();
}

bool gemm_split_supported(const GemmArgs& g) {
  return g.M > 0 && g.N > 0 && g.K > 0 && g.L > 0 && g.M < (1ll << 31) && g.N < (1ll << 31) &&
         (g.M + tc::BM - 1) / tc::BM <= 0x7fffffff && (g.N + tc::BN - 1) / tc::BN <= 65535;
}

cudaError_t launch_gemm_split(const GemmArgs& g, int nterms, void* workspace, size_t ws_bytes, int num_sms,
                              cudaStream_t s) {
  using namespace tc;
  if (!gemm_split_supported(g) || (nterms != 2 && nterms != 3)) return cudaErrorNotSupported;
  static std::atomic<unsigned long long> attr2{0}, attr3{0};
  {
    const cudaError_t e = nterms == 2 ? set_smem_once(attr2, k_gemm_bf16x3<2>, Cfg<2>::SMEM_BYTES)
                                      : set_smem_once(attr3, k_gemm_bf16x3<3>, Cfg<3>::SMEM_BYTES);
    if (e != cudaSuccess) return e;
  }
  TcArgs t;
  memset(&t, 0, sizeof(t));
  t.g = g;
  t.a_kfast = g.k_sa[0] == 1 && g.k_ext[0] % 8 == 0;
  t.b_kfast = g.k_sb[0] == 1 && g.k_ext[0] % 8 == 0;
  const int64_t tm = (g.M + BM - 1) / BM, tn = (g.N + BN - 1) / BN;
  const int64_t tiles = tm * tn * g.L;
  // split K until the grid covers the SMs (one CTA per SM), keeping at
  // least 8 k-steps per split
  int64_t S = 1;
  const int64_t ksteps = (g.K + BK - 1) / BK;
  if (tiles < num_sms) {
    S = (num_sms + tiles - 1) / tiles;
    S = std::min<int64_t>(S, std::max<int64_t>(1, ksteps / 8));
  }
  int64_t kchunk = ((ksteps + S - 1) / S) * BK;
  S = (g.K + kchunk - 1) / kchunk;
  if (S > 1) {
    const size_t need = (size_t)S * g.L * g.M * g.N * sizeof(float);
    if (need > ws_bytes || g.L * S > 65535) {
      S = 1;
      kchunk = ksteps * BK;
    } else {
      t.partial = static_cast<float*>(workspace);
    }
  }
  if (S == 1 && g.L > 65535) return cudaErrorNotSupported;
  t.S = (int)S;
  t.kchunk = kchunk;
  dim3 grid((unsigned)tm, (unsigned)tn, (unsigned)(g.L * S));
  KernelTimer kt(s, "k_gemm_bf16x3");
  if (nterms == 2) k_gemm_bf16x3<2><<<grid, NTHREADS, Cfg<2>::SMEM_BYTES, s>>>(t);
  else k_gemm_bf16x3<3><<<grid, NTHREADS, Cfg<3>::SMEM_BYTES, s>>>(t);
  count_launch();
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess || S == 1) return e;
  const int64_t total = g.M * g.N * g.L;
  const int64_t nb = (total + 255) / 256;
  k_splitk_reduce<<<(unsigned)std::min<int64_t>(nb, (int64_t)num_sms * 16), 256, 0, s>>>(t);
  count_launch();
  return cudaGetLastError();
}

// ===========================================================================
// Pre-split operands + bulk-copy-fed persistent GEMM
// ===========================================================================
//
// k_pack_split writes each operand once as BF16 terms, already in the UMMA
// K-major canonical layout: for every (batch, 128-row tile, 32-wide k-step)
// one contiguous blob of NT 8 KB term tiles.  The GEMM then moves a whole
// stage with two cp.async.bulk copies (no tensor map, no converter warps):
//  * warp 8 lane 0 (producer) issues the bulk copies into a STAGES-deep ring,
//    completion counted by the stage's mbarrier (expect_tx);
//  * warp 9 allocates TMEM; its lane 0 issues the MMAs exactly as
//    k_gemm_bf16x3 does (main t0*t0 and cross-term accumulators, two TMEM
//    buffers, a fresh accumulation every CHUNK k-steps);
//  * warps 0-7 drain each finished chunk (tcgen05.ld) into FP32 running sums
//    held in registers (thread = one row x 64 columns), round-to-nearest
//    adds, and store the tile (αβ epilogue, or a split partial).
// The kernel is persistent over work units: the first F tiles (whole waves of
// the grid) are computed whole, the remaining tiles are cut into S K-splits so
// that the last wave fills the SMs; split partials are summed in split order
// by k_splitk_tiles (deterministic).  The chunk counter runs across units, so
// the epilogue of one unit overlaps the MMAs of the next.
namespace pk {
constexpr int BM = 128, BN = 128, BK = 32, CHUNK = 8;
constexpr int TILE_BYTES = BM * BK * 2;     // one term of one operand for one k-step
constexpr int NDRAIN = 256;                 // drain / epilogue warps 0-7
constexpr int NTHREADS = NDRAIN + 64;       // + producer warp 8 + MMA warp 9
constexpr int TMEM_COLS = 512;
template <int NT> struct Cfg {
  static constexpr int BLOB = NT * TILE_BYTES;
  static constexpr int STAGE_BYTES = 2 * BLOB;
  static constexpr int STAGES = NT == 2 ? 6 : 4;
  static constexpr int SMEM_BYTES = STAGES * STAGE_BYTES + 256;
};
}  // namespace pk

struct PackArgs {
  const float* X;
  unsigned char* P;   // [L][RT][NKT] blobs of NT x 8 KB
  int64_t* c_tab;     // C offset of every row (NULL: no table), from c_str
  int64_t R, K, L, RT, NKT;
  int nr, nk, nl, kfast;
  int64_t r_ext[MAXG], r_str[MAXG], k_ext[MAXG], k_str[MAXG], l_ext[MAXG], l_str[MAXG], c_str[MAXG];
};


struct PkArgs {
  GemmArgs g;                  // C, M, N, L and the epilogue
  const unsigned char* PA;     // packed A [L][TM][NKT]
  const unsigned char* PB;     // packed B [L][TN][NKT]
  float* partial;              // [(tiles - F) * S][BN][BM]
  int64_t TM, TN, NKT, tiles, F, ksplit, units;
  int S;
};

template <int NT>
__device__ __forceinline__ void pack_blob(const PackArgs& p, int64_t b, int warp, int lane) {
  using namespace pk;
  const int64_t kt = b % p.NKT;
  const int64_t r2 = b / p.NKT;
  const int64_t rt = r2 % p.RT;
  const int64_t l = r2 / p.RT;
  const int64_t loff = mode_offset(l, p.nl, p.l_ext, p.l_str);
  uint4* out = reinterpret_cast<uint4*>(p.P + b * (int64_t)(NT * TILE_BYTES));
  float v[2][8];
  int so[2];
#pragma unroll
  for (int j = 0; j < 2; ++j) {
    // the converter mapping of k_gemm_bf16x3 over 16 virtual warps: each
    // quarter-warp writes one contiguous 128-byte core matrix
    const int vw = warp + 8 * j;
    int row, kc;
    if (p.kfast) { row = 8 * vw + (lane & 7); kc = lane >> 3; }
    else { row = 32 * (vw & 3) + lane; kc = vw >> 2; }
    const int64_t r = rt * BM + row;
    const int64_t roff = r < p.R ? loff + goff(r, p.nr, p.r_ext, p.r_str) : -1;
    load_unit(p.X, roff, kt * BK + kc * 8, p.K, p.kfast, p.nk, p.k_ext, p.k_str, v[j]);
    so[j] = ((row >> 3) * 4 + kc) * 8 + (row & 7);
  }
#pragma unroll
  for (int j = 0; j < 2; ++j) {
    uint4 t[NT];
    split8<NT>(v[j], t);
#pragma unroll
    for (int u = 0; u < NT; ++u) out[u * (TILE_BYTES / 16) + so[j]] = t[u];
  }
}

// One launch packs A, then B, then fills the C offset tables of the rows of
// A (M) and B (N) when they are asked for: work unit = one blob or 256
// table entries, grid-stride over all of them.
template <int NT>
__global__ void __launch_bounds__(256) k_pack_split(const __grid_constant__ PackArgs pa,
                                                    const __grid_constant__ PackArgs pb) {
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int64_t na = pa.L * pa.RT * pa.NKT, nb = pb.L * pb.RT * pb.NKT;
  const int64_t ta = pa.c_tab ? (pa.R + 255) / 256 : 0, tb = pb.c_tab ? (pb.R + 255) / 256 : 0;
  const int64_t total = na + nb + ta + tb;
  for (int64_t u = blockIdx.x; u < total; u += gridDim.x) {
    if (u < na) {
      pack_blob<NT>(pa, u, warp, lane);
    } else if (u < na + nb) {
      pack_blob<NT>(pb, u - na, warp, lane);
    } else {
      const bool first = u < na + nb + ta;
      const PackArgs& p = first ? pa : pb;
      const int64_t i = (u - na - nb - (first ? 0 : ta)) * 256 + threadIdx.x;
      if (i < p.R) p.c_tab[i] = mode_offset(i, p.nr, p.r_ext, p.c_str);
    }
  }
}

__device__ __forceinline__ void mbar_expect_tx(uint64_t* bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes)
               : "memory");
}
__device__ __forceinline__ void bulk_g2s(uint32_t dst, const void* src, uint32_t bytes, uint64_t* bar) {
  asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(dst),
               "l"(src), "r"(bytes), "r"(smem_u32(bar))
               : "memory");
}
// Time-bounded wait that ignores the abort flag (used only to let this
// block's own asynchronous copies and MMAs finish before it exits).
__device__ __forceinline__ void mbar_wait_quiesce(uint64_t* bar, uint32_t parity) {
  const uint64_t t0 = gtimer();
  while (!mbar_try_wait(bar, parity))
    if (gtimer() - t0 > tc::WAIT_NS) {
      atomicExch(&g_ome_timeout, 1);
      return;
    }
}

template <int NT>
__global__ void __launch_bounds__(pk::NTHREADS, 1) k_gemm_packed(const __grid_constant__ PkArgs t) {
  using namespace pk;
  constexpr int STAGES = Cfg<NT>::STAGES, STAGE_BYTES = Cfg<NT>::STAGE_BYTES, BLOB = Cfg<NT>::BLOB;
  extern __shared__ __align__(1024) unsigned char smem[];
  uint64_t* full = reinterpret_cast<uint64_t*>(smem + STAGES * STAGE_BYTES);
  uint64_t* empty = full + STAGES;
  uint64_t* chunk_done = empty + STAGES;   // [2]
  uint64_t* drained = chunk_done + 2;      // [2]
  uint64_t* final_bar = drained + 2;
  uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(final_bar + 1);
  volatile int* abort_flag = reinterpret_cast<volatile int*>(tmem_slot + 1);

  const GemmArgs& g = t.g;
  const int tid = threadIdx.x;
  const int warp = tid >> 5, lane = tid & 31;
  if (tid == 0) {
    for (int s = 0; s < STAGES; ++s) {
      mbar_init(&full[s], 1);
      mbar_init(&empty[s], 1);
    }
    for (int b = 0; b < 2; ++b) {
      mbar_init(&chunk_done[b], 1);
      mbar_init(&drained[b], NDRAIN);
    }
    mbar_init(final_bar, 1);
    *abort_flag = 0;
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  if (warp == 9) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(tmem_slot)),
                 "r"(TMEM_COLS)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = *tmem_slot;
  auto tmem_main = [&](int b) { return tmem + (uint32_t)(256 * b); };
  auto tmem_cross = [&](int b) { return tmem + (uint32_t)(256 * b + 128); };
  const uint32_t sbase = smem_u32(smem);

  // unit u -> tile (l, mt, nt; mt fastest), k-step range, split slot (-1: whole)
  auto decode = [&](int64_t u, int64_t& l, int64_t& mt, int64_t& nt, int64_t& kb, int64_t& ke, int64_t& slot) {
    int64_t tile;
    if (u < t.F) {
      tile = u; kb = 0; ke = t.NKT; slot = -1;
    } else {
      const int64_t v = u - t.F;
      tile = t.F + v / t.S;
      kb = (v % t.S) * t.ksplit;
      ke = min(t.NKT, kb + t.ksplit);
      slot = v;
    }
    mt = tile % t.TM;
    const int64_t r = tile / t.TM;
    nt = r % t.TN;
    l = r / t.TN;
  };

  if (warp == 8) {
    // ---------------- producer: two bulk copies per stage ----------------
    if (lane == 0) {
      uint32_t it = 0;
      for (int64_t u = blockIdx.x; u < t.units; u += gridDim.x) {
        int64_t l, mt, nt, kb, ke, slot;
        decode(u, l, mt, nt, kb, ke, slot);
        const unsigned char* pa = t.PA + ((l * t.TM + mt) * t.NKT) * (int64_t)BLOB;
        const unsigned char* pb = t.PB + ((l * t.TN + nt) * t.NKT) * (int64_t)BLOB;
        bool ok = true;
        for (int64_t kt = kb; kt < ke; ++kt, ++it) {
          const int s = it % STAGES;
          if (it >= (uint32_t)STAGES && !mbar_wait(&empty[s], ((it / STAGES) - 1) & 1, abort_flag)) {
            ok = false;
            break;
          }
          mbar_expect_tx(&full[s], 2 * BLOB);
          bulk_g2s(sbase + s * STAGE_BYTES, pa + kt * BLOB, BLOB, &full[s]);
          bulk_g2s(sbase + s * STAGE_BYTES + BLOB, pb + kt * BLOB, BLOB, &full[s]);
        }
        if (!ok) break;
      }
      // the copies of the last STAGES issues must land before the block exits
      for (uint32_t i = it > (uint32_t)STAGES ? it - STAGES : 0; i < it; ++i)
        mbar_wait_quiesce(&full[i % STAGES], (i / STAGES) & 1);
    }
  } else if (warp == 9) {
    // ---------------- MMA issue ----------------
    if (lane == 0) {
      uint32_t it = 0, gc = 0;
      bool ok = true;
      for (int64_t u = blockIdx.x; u < t.units && ok; u += gridDim.x) {
        int64_t l, mt, nt, kb, ke, slot;
        decode(u, l, mt, nt, kb, ke, slot);
        const int nk = (int)(ke - kb);
        for (int j = 0; j < nk; ++j, ++it) {
          const uint32_t c = gc + j / CHUNK;
          const int b = c & 1;
          const bool first = j % CHUNK == 0;
          if (first && c >= 2 && !mbar_wait(&drained[b], ((c >> 1) - 1) & 1, abort_flag)) { ok = false; break; }
          const int s = it % STAGES;
          if (!mbar_wait(&full[s], (it / STAGES) & 1, abort_flag)) { ok = false; break; }
          tc_fence_after();
          const uint32_t sb = sbase + s * STAGE_BYTES;
#pragma unroll
          for (int kk = 0; kk < 2; ++kk) {
            const uint32_t off = kk * 256;
            uint64_t ad[NT], bd[NT];
#pragma unroll
            for (int q = 0; q < NT; ++q) {
              ad[q] = umma_desc(sb + q * TILE_BYTES + off);
              bd[q] = umma_desc(sb + BLOB + q * TILE_BYTES + off);
            }
            const uint32_t keep = (first && kk == 0) ? 0u : 1u;
            umma_bf16(tmem_main(b), ad[0], bd[0], keep);
            bool first_cross = true;
#pragma unroll
            for (int d = 1; d < NT; ++d)
#pragma unroll
              for (int i = 0; i <= d; ++i) {
                umma_bf16(tmem_cross(b), ad[i], bd[d - i], first_cross ? keep : 1u);
                first_cross = false;
              }
          }
          umma_commit(&empty[s]);
          if (j % CHUNK == CHUNK - 1 || j == nk - 1) umma_commit(&chunk_done[b]);
        }
        gc += (uint32_t)((nk + CHUNK - 1) / CHUNK);
      }
      // every MMA this thread issued must finish before TMEM is freed
      umma_commit(final_bar);
      mbar_wait_quiesce(final_bar, 0);
    }
  } else {
    // ---------------- drain + epilogue (warps 0-7) ----------------
    const int q = warp & 3, h = warp >> 2;
    const int row = 32 * q + lane;
    const int col0 = 64 * h;
    const uint32_t lane_off = (uint32_t)(32 * q) << 16;
    uint32_t gc = 0;
    const float sx = scalar_as<float>(g.sx), sy = scalar_as<float>(g.sy);
    float* Cp = static_cast<float*>(g.C);
    for (int64_t u = blockIdx.x; u < t.units; u += gridDim.x) {
      int64_t l, mt, nt, kb, ke, slot;
      decode(u, l, mt, nt, kb, ke, slot);
      const int nch = (int)((ke - kb + CHUNK - 1) / CHUNK);
      float sum[64];
#pragma unroll
      for (int j = 0; j < 64; ++j) sum[j] = 0.f;
      bool ok = true;
      for (int ci = 0; ci < nch; ++ci, ++gc) {
        const int b = gc & 1;
        if (!mbar_wait(&chunk_done[b], (gc >> 1) & 1, abort_flag)) { ok = false; break; }
        tc_fence_after();
#pragma unroll
        for (int hh = 0; hh < 4; ++hh) {
          uint32_t rm[16], rc[16];
          __syncwarp();
          tmem_ld16(tmem_main(b) + lane_off + (uint32_t)(col0 + 16 * hh), rm);
          tmem_ld16(tmem_cross(b) + lane_off + (uint32_t)(col0 + 16 * hh), rc);
#pragma unroll
          for (int j = 0; j < 16; ++j) {
            const float v = __uint_as_float(rm[j]) + __uint_as_float(rc[j]);
            sum[16 * hh + j] = ci == 0 ? v : sum[16 * hh + j] + v;
          }
        }
        tc_fence_before();
        mbar_arrive(&drained[b]);
      }
      if (!ok) break;
      if (slot >= 0) {
        float* pp = t.partial + (slot * BN + col0) * (int64_t)BM + row;
#pragma unroll
        for (int j = 0; j < 64; ++j) pp[(int64_t)j * BM] = sum[j];
      } else {
        const int64_t m = mt * BM + row;
        if (m < g.M) {
          const int64_t base = mode_offset(l, g.nl, g.l_ext, g.l_sc) + c_moff(g, m);
          const int64_t n0 = nt * BN + col0;
#pragma unroll
          for (int j = 0; j < 64; ++j) {
            const int64_t n = n0 + j;
            if (n < g.N) {
              float* cp = Cp + base + c_noff(g, n);
              float o = g.sx_one ? sum[j] : sx * sum[j];
              if (!g.sy_zero) o = fmaf(sy, *cp, o);
              *cp = o;
            }
          }
        }
      }
    }
  }
  tc_fence_before();
  __syncthreads();
  if (warp == 9) {
    tc_fence_after();
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(pk::TMEM_COLS) : "memory");
  }
}

// Sum the S split partials of each split tile in split order; αβ epilogue.
__global__ void __launch_bounds__(256) k_splitk_tiles(const __grid_constant__ PkArgs t) {
  using namespace pk;
  const GemmArgs& g = t.g;
  const float sx = scalar_as<float>(g.sx), sy = scalar_as<float>(g.sy);
  float* Cp = static_cast<float*>(g.C);
  const int64_t total = (t.tiles - t.F) * BM * BN;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < total;
       i += (int64_t)gridDim.x * blockDim.x) {
    const int64_t mloc = i % BM;
    const int64_t r = i / BM;
    const int64_t nloc = r % BN;
    const int64_t v = r / BN;
    const int64_t tile = t.F + v;
    const int64_t mt = tile % t.TM, r2 = tile / t.TM, nt = r2 % t.TN, l = r2 / t.TN;
    const int64_t m = mt * BM + mloc, n = nt * BN + nloc;
    if (m >= g.M || n >= g.N) continue;
    float acc = 0.f;
    for (int s = 0; s < t.S; ++s) acc += t.partial[((v * t.S + s) * BN + nloc) * BM + mloc];
    float* cp = Cp + mode_offset(l, g.nl, g.l_ext, g.l_sc) + c_moff(g, m) +
                c_noff(g, n);
    float o = g.sx_one ? acc : sx * acc;
    if (!g.sy_zero) o = fmaf(sy, *cp, o);
    *cp = o;
  }
}

static void pack_args(PackArgs& p, const float* X, unsigned char* P, int64_t R, int nr, const int64_t* r_ext,
                      const int64_t* r_str, const GemmArgs& g, const int64_t* k_str, const int64_t* l_str) {
  memset(&p, 0, sizeof(p));
  p.X = X;
  p.P = P;
  p.R = R;
  p.K = g.K;
  p.L = g.L;
  p.RT = (R + pk::BM - 1) / pk::BM;
  p.NKT = (g.K + pk::BK - 1) / pk::BK;
  p.nr = nr;
  p.nk = g.nk;
  p.nl = g.nl;
  for (int i = 0; i < nr; ++i) { p.r_ext[i] = r_ext[i]; p.r_str[i] = r_str[i]; }
  for (int i = 0; i < g.nk; ++i) { p.k_ext[i] = g.k_ext[i]; p.k_str[i] = k_str[i]; }
  for (int i = 0; i < g.nl; ++i) { p.l_ext[i] = g.l_ext[i]; p.l_str[i] = l_str[i]; }
  p.kfast = k_str[0] == 1 && g.k_ext[0] % 8 == 0;
}

size_t gemm_packed_bytes(const GemmArgs& g, int nterms, int num_sms) {
  using namespace pk;
  const int64_t TM = (g.M + BM - 1) / BM, TN = (g.N + BN - 1) / BN, NKT = (g.K + BK - 1) / BK;
  const size_t blob = (size_t)nterms * TILE_BYTES;
  // packed operands + at most one grid's worth of split partials
  return (size_t)g.L * (TM + TN) * NKT * blob + (size_t)num_sms * BM * BN * 4 + 1024;
}

cudaError_t launch_gemm_packed(const GemmArgs& g, int nterms, void* workspace, size_t ws_bytes, int num_sms,
                               cudaStream_t s, int64_t* ctab) {
  using namespace pk;
  if (!gemm_split_supported(g) || (nterms != 2 && nterms != 3)) return cudaErrorNotSupported;
  static std::atomic<unsigned long long> attr2{0}, attr3{0};
  {
    const cudaError_t e = nterms == 2 ? set_smem_once(attr2, k_gemm_packed<2>, Cfg<2>::SMEM_BYTES)
                                      : set_smem_once(attr3, k_gemm_packed<3>, Cfg<3>::SMEM_BYTES);
    if (e != cudaSuccess) return e;
  }
  const int64_t TM = (g.M + BM - 1) / BM, TN = (g.N + BN - 1) / BN, NKT = (g.K + BK - 1) / BK;
  const size_t blob = (size_t)nterms * TILE_BYTES;
  const size_t bytes_a = (size_t)g.L * TM * NKT * blob, bytes_b = (size_t)g.L * TN * NKT * blob;
  const int64_t tiles = g.L * TM * TN;
  const int64_t G = num_sms;
  // whole tiles for every complete wave; the rest split along K so that the
  // last wave covers the grid (at least 8 k-steps per split)
  int64_t F = tiles >= G ? (tiles / G) * G : 0;
  int64_t Rt = tiles - F;
  int64_t S = 1;
  if (Rt > 0) {
    S = std::max<int64_t>(1, G / Rt);
    S = std::min<int64_t>(S, std::max<int64_t>(1, NKT / 8));
  }
  const int64_t ksplit = (NKT + S - 1) / S;
  S = (NKT + ksplit - 1) / ksplit;
  if (S == 1) {
    F = tiles;
    Rt = 0;
  }
  const size_t bytes_p = (size_t)Rt * S * BM * BN * 4;
  if (bytes_a + bytes_b + bytes_p + 768 > ws_bytes) return cudaErrorNotSupported;
  unsigned char* w = static_cast<unsigned char*>(workspace);
  unsigned char* PA = w;
  unsigned char* PB = w + ((bytes_a + 255) & ~(size_t)255);
  float* part = reinterpret_cast<float*>(PB + ((bytes_b + 255) & ~(size_t)255));

  PackArgs pa, pb;
  pack_args(pa, static_cast<const float*>(g.A), PA, g.M, g.nm, g.m_ext, g.m_sa, g, g.k_sa, g.l_sa);
  pack_args(pb, static_cast<const float*>(g.B), PB, g.N, g.nn, g.n_ext, g.n_sb, g, g.k_sb, g.l_sb);
  if (ctab) {
    pa.c_tab = ctab;
    pb.c_tab = ctab + g.M;
    for (int i = 0; i < g.nm; ++i) pa.c_str[i] = g.m_sc[i];
    for (int i = 0; i < g.nn; ++i) pb.c_str[i] = g.n_sc[i];
  }
  const int64_t units = g.L * (TM + TN) * NKT + (ctab ? (g.M + 255) / 256 + (g.N + 255) / 256 : 0);
  const unsigned gp = (unsigned)std::min<int64_t>(units, (int64_t)num_sms * 8);
  if (nterms == 2) k_pack_split<2><<<gp, 256, 0, s>>>(pa, pb);
  else k_pack_split<3><<<gp, 256, 0, s>>>(pa, pb);
  count_launch();
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return e;

  PkArgs t;
  memset(&t, 0, sizeof(t));
  t.g = g;
  if (ctab) {
    t.g.m_tab_c = ctab;
    t.g.n_tab_c = ctab + g.M;
  }
  t.PA = PA;
  t.PB = PB;
  t.partial = part;
  t.TM = TM;
  t.TN = TN;
  t.NKT = NKT;
  t.tiles = tiles;
  t.F = F;
  t.S = (int)S;
  t.ksplit = ksplit;
  t.units = F + Rt * S;
  const unsigned grid = (unsigned)std::min<int64_t>(t.units, G);
  // plain launches: a GEMM block started early would hold its SM's shared
  // memory and TMEM while waiting, which stalls other streams' kernels
  {
    KernelTimer kt(s, "k_gemm_packed");
    if (nterms == 2) k_gemm_packed<2><<<grid, NTHREADS, Cfg<2>::SMEM_BYTES, s>>>(t);
    else k_gemm_packed<3><<<grid, NTHREADS, Cfg<3>::SMEM_BYTES, s>>>(t);
  }
  count_launch();
  e = cudaGetLastError();
  if (e != cudaSuccess || Rt == 0) return e;
  const int64_t total = Rt * BM * BN;
  const int64_t nb = (total + 255) / 256;
  k_splitk_tiles<<<(unsigned)std::min<int64_t>(nb, (int64_t)num_sms * 16), 256, 0, s>>>(t);
  count_launch();
  return cudaGetLastError();
}

// ---------------------------------------------------------------------------
// k_gemm_tma2: 2-SM tensor-core GEMM fed by tensor maps over the FP32 inputs.
//
// The operands are read in place, through TMA tensor maps whose dimensions
// and strides are the contraction's merged mode groups (the permutation of
// simplifyto, src/einsum.jl:127-134, lives in the maps: nothing is written
// back to HBM), and split into BF16 terms in shared memory.
//  * A cluster of two CTAs computes a 256 x 256 tile of C with
//    tcgen05.mma.cta_group::2 (M = 256, N = 256, K = 16): CTA r holds rows
//    128r..128r+127 of the A tile and columns 128r..128r+127 of the B tile;
//    its TMEM receives rows 128r.. of the accumulator, all 256 columns.
//  * Warp 16 (one thread) issues, per 32-wide k stage, the TMA loads of this
//    CTA's FP32 A and B tiles (128-byte swizzle, zero fill past the extents;
//    no multicast) into one of three FP32 stages.
//  * Warps 0-7 (A) and 8-15 (B) convert a stage into NT BF16 terms per value
//    in the UMMA K-major canonical layout (conflict-free shared-memory reads
//    and writes in both operand orientations), then arrive on the leader
//    CTA's term_full barrier (remote arrive, release at cluster scope).
//  * Warp 17 of the leader CTA issues the MMAs (main t0*t0 and cross-term
//    accumulators, 2 x 256 TMEM columns) and releases each term stage to both
//    CTAs with a multicast tcgen05.commit.
//  * Every CHS stages the 16 converter warps of both CTAs drain the
//    accumulators (tcgen05.ld) into FP32 running sums in registers with
//    round-to-nearest adds; the accumulators are single-buffered, so the
//    converters drain chunk c before they wait for a term stage whose MMAs
//    come after it (no cycle in the waits).
//  * Persistent over units: whole 256 x 256 tiles for the complete waves of
//    clusters, the last wave's tiles cut along K (partials summed in split
//    order by k_splitk_tiles2: deterministic).
//  * Every wait is bounded (tc::WAIT_NS); on expiry the CTA records the
//    timeout flag, stops waiting, lets its own copies and MMAs finish and
//    frees its TMEM.  Both CTAs meet at a final cluster barrier.
namespace t2 {
constexpr int BM = 128;                    // rows per CTA (256 per cluster tile)
constexpr int BK = 32;                     // k per stage
constexpr int CHS = 8;                     // stages per accumulator chunk (16 k-steps)
constexpr int F32_STAGES = 2;
constexpr int NSR = 32;                    // running sums per thread in registers (the other 32 in shared memory)
constexpr int F32_TILE = BM * BK * 4;      // 16 KB: one operand, one stage
constexpr int TERM_TILE = BM * BK * 2;     // 8 KB: one term of one operand
constexpr int NCONV = 512;                 // converter + drain warps 0-15
constexpr int NTHREADS = NCONV + 64;       // + TMA warp 16 + MMA warp 17
constexpr int TMEM_COLS = 512;
template <int NT> struct Cfg {
  static constexpr int F32_STAGE = 2 * F32_TILE;          // A tile, B tile
  static constexpr int TERM_STAGE = 2 * NT * TERM_TILE;   // A terms, B terms
  static constexpr int TSTAGES = NT == 2 ? 3 : 2;
  static constexpr int SUM_BYTES = NCONV * (64 - NSR) * 4;   // 64 KB of running sums
  static constexpr int BAR_BYTES = 256;
  static constexpr int SMEM_BYTES = F32_STAGES * F32_STAGE + TSTAGES * TERM_STAGE + SUM_BYTES + BAR_BYTES + 1024;
};
// kind::f16, BF16 x BF16 -> F32, K-major A and B, M = 256 (cta pair), N = 256
constexpr uint32_t IDESC = (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(256 >> 3) << 17) |
                           ((uint32_t)(256 >> 4) << 24);
}  // namespace t2

struct T2Args {
  GemmArgs g;
  float* partial;                  // [(tiles - F) * S][256][256]
  int TM, TN, NKT, tiles, F, ksplit, units, S;   // all below 2^31 (checked on the host)
  int64_t c_max, p_max;            // largest element offset of C and of the partials (self-check)
};

__device__ __forceinline__ uint32_t cluster_rank() {
  uint32_t r;
  asm volatile("mov.u32 %0, %%cluster_ctarank;" : "=r"(r));
  return r;
}
__device__ __forceinline__ void cluster_sync_all() {
  asm volatile("barrier.cluster.arrive.release.aligned;\n\tbarrier.cluster.wait.acquire.aligned;" ::: "memory");
}
// Address of the same shared-memory location in CTA `rank` of the cluster.
__device__ __forceinline__ uint32_t peer_addr(uint32_t a, uint32_t rank) {
  uint32_t r;
  asm volatile("mapa.shared::cluster.u32 %0, %1, %2;" : "=r"(r) : "r"(a), "r"(rank));
  return r;
}
// Arrive on an mbarrier of either CTA of the pair (default release at CTA
// scope: the data it publishes is this CTA's own shared memory, made visible
// to the tensor core by fence.proxy.async before the arrive; a cluster-scope
// release would cost a full fence per arrive).
__device__ __forceinline__ void mbar_arrive_remote(uint32_t cluster_addr) {
  asm volatile("mbarrier.arrive.shared::cluster.b64 _, [%0];" ::"r"(cluster_addr) : "memory");
}
__device__ __forceinline__ bool mbar_try_wait_cl(uint64_t* bar, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
      "selp.u32 %0, 1, 0, p;\n\t}\n"
      : "=r"(ok)
      : "r"(smem_u32(bar)), "r"(parity)
      : "memory");
  return ok != 0;
}
// Bounded wait on a barrier that both CTAs of the pair arrive on.
__device__ __forceinline__ bool mbar_wait_cl(uint64_t* bar, uint32_t parity, volatile int* abort_flag) {
  if (mbar_try_wait_cl(bar, parity)) return true;
  const uint64_t t0 = gtimer();
  while (true) {
#pragma unroll 1
    for (int i = 0; i < 32; ++i)
      if (mbar_try_wait_cl(bar, parity)) return true;
    if (*abort_flag) return false;
    if (gtimer() - t0 > tc::WAIT_NS) {
      *abort_flag = 1;
      atomicExch(&g_ome_timeout, 1);
      return false;
    }
  }
}
// 32-bit shared-address forms (fewer registers than generic pointers).
__device__ __forceinline__ bool mbar_try_wait32(uint32_t a, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
      "selp.u32 %0, 1, 0, p;\n\t}\n"
      : "=r"(ok)
      : "r"(a), "r"(parity)
      : "memory");
  return ok != 0;
}
__device__ __forceinline__ int ld_flag(uint32_t a) {
  int v;
  asm volatile("ld.volatile.shared.u32 %0, [%1];" : "=r"(v) : "r"(a) : "memory");
  return v;
}
__device__ __forceinline__ bool mbar_wait32(uint32_t a, uint32_t parity, uint32_t abort_a) {
  if (mbar_try_wait32(a, parity)) return true;
  const uint64_t t0 = gtimer();
  while (true) {
#pragma unroll 1
    for (int i = 0; i < 32; ++i)
      if (mbar_try_wait32(a, parity)) return true;
    if (ld_flag(abort_a)) return false;
    if (gtimer() - t0 > tc::WAIT_NS) {
      asm volatile("st.volatile.shared.u32 [%0], %1;" ::"r"(abort_a), "r"(1) : "memory");
      atomicExch(&g_ome_timeout, 1);
      return false;
    }
  }
}
__device__ __forceinline__ void mbar_arrive32(uint32_t a) {
  asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(a) : "memory");
}
__device__ __forceinline__ float lds32(uint32_t a) {
  float v;
  asm volatile("ld.shared.f32 %0, [%1];" : "=f"(v) : "r"(a));
  return v;
}
__device__ __forceinline__ void sts32(uint32_t a, float v) {
  asm volatile("st.shared.f32 [%0], %1;" ::"r"(a), "f"(v) : "memory");
}
__device__ __forceinline__ void tma_load_2d(uint32_t dst, const CUtensorMap* map, int x, int y, uint64_t* bar) {
  asm volatile(
      "cp.async.bulk.tensor.2d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3}], [%4];" ::
          "r"(dst), "l"(reinterpret_cast<uint64_t>(map)), "r"(x), "r"(y), "r"(smem_u32(bar))
      : "memory");
}
__device__ __forceinline__ void tma_load_3d(uint32_t dst, const CUtensorMap* map, int x, int y, int z,
                                            uint64_t* bar) {
  asm volatile(
      "cp.async.bulk.tensor.3d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4}], "
      "[%5];" ::"r"(dst),
      "l"(reinterpret_cast<uint64_t>(map)), "r"(x), "r"(y), "r"(z), "r"(smem_u32(bar))
      : "memory");
}
__device__ __forceinline__ void umma_bf16_pair(uint32_t d_tmem, uint64_t a, uint64_t b, uint32_t acc) {
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "setp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::2.kind::f16 [%0], %1, %2, %3, p;\n\t}\n" ::"r"(d_tmem),
      "l"(a), "l"(b), "r"(t2::IDESC), "r"(acc));
}
// Arrive (once) on the barrier at this shared-memory offset in the CTAs of
// `mask` when every tcgen05.mma this thread issued so far has completed.
__device__ __forceinline__ void umma_commit_pair(uint64_t* bar, uint16_t mask) {
  asm volatile(
      "tcgen05.commit.cta_group::2.mbarrier::arrive::one.shared::cluster.multicast::cluster.b64 [%0], %1;" ::"r"(
          smem_u32(bar)),
      "h"(mask)
      : "memory");
}
__device__ __forceinline__ void tmem_ld8(uint32_t taddr, uint32_t (&r)[8]) {
  asm volatile("tcgen05.ld.sync.aligned.32x32b.x8.b32 {%0,%1,%2,%3,%4,%5,%6,%7}, [%8];"
               : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7])
               : "r"(taddr));
  asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
}
__device__ __forceinline__ float4 lds128(uint32_t a) {
  float4 v;
  asm volatile("ld.shared.v4.f32 {%0,%1,%2,%3}, [%4];" : "=f"(v.x), "=f"(v.y), "=f"(v.z), "=f"(v.w) : "r"(a));
  return v;
}
__device__ __forceinline__ float2 lds64(uint32_t a) {
  float2 v;
  asm volatile("ld.shared.v2.f32 {%0,%1}, [%2];" : "=f"(v.x), "=f"(v.y) : "r"(a));
  return v;
}
// split8 with each term stored (16 bytes at dst + t * TERM_TILE) as soon as
// it is formed; v is overwritten by the residuals.  The rounding to BF16 is
// done with integer operations (round half away from zero: add half an ulp of
// the 8-bit significand, drop the low 16 bits), not with cvt, whose pipe
// would limit the converter warps; t + (v - t) == v exactly for any rounding
// of the leading term, so the split stays exact.  Non-finite inputs give
// NaN residuals.
template <int NT>
__device__ __forceinline__ void split8_store(float (&v)[8], uint32_t dst) {
#pragma unroll
  for (int t = 0; t < NT; ++t) {
    // the third term of a 3-term split is truncated: its error (below 2^-24
    // of the value) is under that of the products the split leaves out
    const uint32_t half = NT == 3 && t == 2 ? 0u : 0x8000u;
    uint32_t w[4];
#pragma unroll
    for (int p = 0; p < 4; ++p) {
      const uint32_t ra = __float_as_uint(v[2 * p]) + half;
      const uint32_t rb = __float_as_uint(v[2 * p + 1]) + half;
      w[p] = __byte_perm(ra, rb, 0x7632);   // (ra >> 16) | (rb & 0xffff0000)
      if (t + 1 < NT) {
        v[2 * p] -= __uint_as_float(ra & 0xffff0000u);
        v[2 * p + 1] -= __uint_as_float(rb & 0xffff0000u);
      }
    }
    sts128(dst + t * t2::TERM_TILE, make_uint4(w[0], w[1], w[2], w[3]));
  }
}

// Convert one operand's FP32 stage tile (128 rows x 32 k, TMA 128-byte
// swizzle) into NT BF16 term tiles (K-major canonical: 8-row x 16-byte core
// matrices, unit (row r, k-chunk c8) at ((r >> 3) * 4 + c8) * 128 + (r & 7) * 16).
// wl = warp within the operand's 8 warps; each thread converts 2 units.
// KMAJOR: the tile was loaded as one (32 k, 128 rows) box, row r at r * 128,
// 16-byte chunk c at (c ^ (r & 7)) * 16.  Otherwise as four (32 rows, 32 k)
// boxes (rows 32b.., 4 KB each), k-row k at k * 128, chunk c (4 rows) at
// (c ^ (k & 7)) * 16.
template <int NT, bool KMAJOR>
__device__ __forceinline__ void convert_tile(uint32_t f32, uint32_t terms, int wl, int lane) {
  if constexpr (KMAJOR) {
#pragma unroll
    for (int p = 0; p < 2; ++p) {
      const int r = 8 * (2 * wl + p) + (lane & 7);
      const int c8 = lane >> 3;
      const uint32_t base = f32 + (uint32_t)r * 128;
      const int sw = r & 7;
      const float4 v0 = lds128(base + ((uint32_t)((2 * c8) ^ sw) << 4));
      const float4 v1 = lds128(base + ((uint32_t)((2 * c8 + 1) ^ sw) << 4));
      float v[8] = {v0.x, v0.y, v0.z, v0.w, v1.x, v1.y, v1.z, v1.w};
      split8_store<NT>(v, terms + (uint32_t)(((r >> 3) * 4 + c8) * 128 + (r & 7) * 16));
    }
  } else {
    const int idx = 2 * wl + (lane >> 4);   // (box, k-chunk) of this half-warp
    const int b = idx >> 2, c8 = idx & 3;
    const int rp = lane & 15;               // row pair 2rp, 2rp + 1 of the box
    float va[8], vb[8];
#pragma unroll
    for (int kk = 0; kk < 8; ++kk) {
      const int k = 8 * c8 + kk;
      const uint32_t a = f32 + (uint32_t)(b * 4096 + k * 128 + ((((rp >> 1) ^ (k & 7))) << 4) + ((rp & 1) << 3));
      const float2 v = lds64(a);
      va[kk] = v.x;
      vb[kk] = v.y;
    }
    // the two rows are stored in an order rotated by lane group so that each
    // quarter-warp's 16-byte stores hit eight distinct bank groups
    const int sel = (rp >> 2) & 1;
    const int r0 = 32 * b + 2 * rp;
#pragma unroll
    for (int e = 0; e < 2; ++e) {
      const int which = e ^ sel;
      float v[8];
#pragma unroll
      for (int kk = 0; kk < 8; ++kk) v[kk] = which ? vb[kk] : va[kk];
      const int r = r0 + which;
      split8_store<NT>(v, terms + (uint32_t)(((r >> 3) * 4 + c8) * 128 + (r & 7) * 16));
    }
  }
}

template <int NT, bool AK, bool BKM>
__global__ void __cluster_dims__(2, 1, 1) __launch_bounds__(t2::NTHREADS, 1)
    k_gemm_tma2(const __grid_constant__ T2Args t, const __grid_constant__ CUtensorMap mapA,
                const __grid_constant__ CUtensorMap mapB) {
  using namespace t2;
  constexpr int TS = Cfg<NT>::TSTAGES, F32_STAGE = Cfg<NT>::F32_STAGE, TERM_STAGE = Cfg<NT>::TERM_STAGE;
  extern __shared__ __align__(1024) unsigned char smem_raw[];
  // 1024-byte aligned base for the 128-byte-swizzled TMA tiles (the same
  // offset in both CTAs of the pair, which the MMA descriptors rely on)
  const uint32_t raw = smem_u32(smem_raw);
  const uint32_t pad = (1024u - (raw & 1023u)) & 1023u;
  unsigned char* smem = smem_raw + pad;
  const uint32_t sbase = raw + pad;
  const uint32_t f32_base = sbase;
  const uint32_t term_base = sbase + F32_STAGES * F32_STAGE;
  uint64_t* bars = reinterpret_cast<uint64_t*>(smem + F32_STAGES * F32_STAGE + TS * TERM_STAGE + Cfg<NT>::SUM_BYTES);
  uint64_t* f32_full = bars;
  uint64_t* f32_empty = f32_full + F32_STAGES;
  uint64_t* term_full = f32_empty + F32_STAGES;   // used in the leader CTA
  uint64_t* term_empty = term_full + TS;
  uint64_t* chunk_done = term_empty + TS;
  uint64_t* drained = chunk_done + 1;             // used in the leader CTA
  uint64_t* final_bar = drained + 1;
  uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(final_bar + 1);
  volatile int* abort_flag = reinterpret_cast<volatile int*>(tmem_slot + 1);

  const GemmArgs& g = t.g;
  const int tid = threadIdx.x;
  const int warp = tid >> 5, lane = tid & 31;
  const uint32_t rank = cluster_rank();
  const int cid = blockIdx.x >> 1, ncl = gridDim.x >> 1;
  if (tid == 0) {
    for (int s = 0; s < F32_STAGES; ++s) {
      mbar_init(&f32_full[s], 1);
      mbar_init(&f32_empty[s], 16);
    }
    for (int s = 0; s < TS; ++s) {
      mbar_init(&term_full[s], 32);
      mbar_init(&term_empty[s], 1);
    }
    mbar_init(chunk_done, 1);
    mbar_init(drained, 32);
    mbar_init(final_bar, 1);
    *abort_flag = 0;
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  if (warp == 17) {
    asm volatile("tcgen05.alloc.cta_group::2.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(tmem_slot)),
                 "r"(TMEM_COLS)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::2.sync.aligned;" ::: "memory");
  }
  tc_fence_before();
  cluster_sync_all();   // both CTAs' barriers initialised and TMEM allocated
  tc_fence_after();
  const uint32_t tmem = *tmem_slot;
  const uint32_t tmem_main = tmem, tmem_cross = tmem + 256;

  auto decode = [&](int u, int& l, int& mt, int& nt, int& kb, int& ke, int& slot) {
    int tile;
    if (u < t.F) {
      tile = u; kb = 0; ke = t.NKT; slot = -1;
    } else {
      const int v = u - t.F;
      tile = t.F + v / t.S;
      kb = (v % t.S) * t.ksplit;
      ke = min(t.NKT, kb + t.ksplit);
      slot = v;
    }
    mt = tile % t.TM;
    const int r = tile / t.TM;
    nt = r % t.TN;
    l = r / t.TN;
  };

  if (warp == 16) {
    // ---------------- TMA producer ----------------
    if (lane == 0) {
      uint32_t it = 0;
      bool ok = true;
      for (int u = cid; u < t.units && ok; u += ncl) {
        int l, mt, nt, kb, ke, slot;
        decode(u, l, mt, nt, kb, ke, slot);
        const int ra = mt * 256 + (int)rank * BM, rb = nt * 256 + (int)rank * BM;
        for (int kt = kb; kt < ke; ++kt, ++it) {
          const int s = it % F32_STAGES;
          if (it >= (uint32_t)F32_STAGES && !mbar_wait(&f32_empty[s], ((it / F32_STAGES) - 1) & 1, abort_flag)) {
            ok = false;
            break;
          }
          mbar_expect_tx(&f32_full[s], 2 * F32_TILE);
          const uint32_t da = f32_base + s * F32_STAGE, db = da + F32_TILE;
          const int k0 = kt * BK;
          if (g.L > 1) {
            if (AK) tma_load_3d(da, &mapA, k0, ra, l, &f32_full[s]);
            else
              for (int i = 0; i < 4; ++i) tma_load_3d(da + i * 4096, &mapA, ra + 32 * i, k0, l, &f32_full[s]);
            if (BKM) tma_load_3d(db, &mapB, k0, rb, l, &f32_full[s]);
            else
              for (int i = 0; i < 4; ++i) tma_load_3d(db + i * 4096, &mapB, rb + 32 * i, k0, l, &f32_full[s]);
          } else {
            if (AK) tma_load_2d(da, &mapA, k0, ra, &f32_full[s]);
            else
              for (int i = 0; i < 4; ++i) tma_load_2d(da + i * 4096, &mapA, ra + 32 * i, k0, &f32_full[s]);
            if (BKM) tma_load_2d(db, &mapB, k0, rb, &f32_full[s]);
            else
              for (int i = 0; i < 4; ++i) tma_load_2d(db + i * 4096, &mapB, rb + 32 * i, k0, &f32_full[s]);
          }
        }
      }
      // this CTA's copies in flight must land before it exits
      for (uint32_t i = it > (uint32_t)F32_STAGES ? it - F32_STAGES : 0; i < it; ++i)
        mbar_wait_quiesce(&f32_full[i % F32_STAGES], (i / F32_STAGES) & 1);
    }
  } else if (warp == 17) {
    // ---------------- MMA issue (leader CTA) ----------------
    if (rank == 0 && lane == 0) {
      uint32_t it = 0, gc = 0;
      bool ok = true;
      for (int u = cid; u < t.units && ok; u += ncl) {
        int l, mt, nt, kb, ke, slot;
        decode(u, l, mt, nt, kb, ke, slot);
        const int nk = ke - kb;
        for (int j = 0; j < nk; ++j, ++it) {
          const bool first = j % CHS == 0;
          if (first && gc >= 1 && !mbar_wait_cl(drained, (gc - 1) & 1, abort_flag)) { ok = false; break; }
          const int ts = it % TS;
          if (!mbar_wait_cl(&term_full[ts], (it / TS) & 1, abort_flag)) { ok = false; break; }
          tc_fence_after();
          const uint32_t sa = term_base + ts * TERM_STAGE, sb = sa + NT * TERM_TILE;
#pragma unroll
          for (int kk = 0; kk < 2; ++kk) {
            const uint32_t off = kk * 256;
            uint64_t ad[NT], bd[NT];
#pragma unroll
            for (int q = 0; q < NT; ++q) {
              ad[q] = umma_desc(sa + q * TERM_TILE + off);
              bd[q] = umma_desc(sb + q * TERM_TILE + off);
            }
            const uint32_t keep = (first && kk == 0) ? 0u : 1u;
            umma_bf16_pair(tmem_main, ad[0], bd[0], keep);
            bool first_cross = true;
#pragma unroll
            for (int d = 1; d < NT; ++d)
#pragma unroll
              for (int i = 0; i <= d; ++i) {
                umma_bf16_pair(tmem_cross, ad[i], bd[d - i], first_cross ? keep : 1u);
                first_cross = false;
              }
          }
          umma_commit_pair(&term_empty[ts], 3);
          if (j % CHS == CHS - 1 || j == nk - 1) {
            umma_commit_pair(chunk_done, 3);
            ++gc;
          }
        }
      }
      // every MMA must finish before either CTA frees its TMEM
      umma_commit_pair(final_bar, 1);
      mbar_wait_quiesce(final_bar, 0);
      // and the peer's arrivals on this CTA's drained barrier must have
      // landed before this CTA's shared memory goes away
      if (gc >= 1) mbar_wait_quiesce(drained, (gc - 1) & 1);
    }
  } else if (warp < 16) {
    // ---------------- converters + drain + epilogue (warps 0-15) ----------------
    const int opnd = warp >> 3, wl = warp & 7;
    const int q = warp & 3, h = warp >> 2;
    const int row = 32 * q + lane;                    // accumulator row (TMEM lane) of this thread
    const int col0 = 64 * h;
    const uint32_t lane_off = (uint32_t)(32 * q) << 16;
    // barriers and flags by 32-bit shared address
    // every address is sbase (or the leader's base) plus a constant, so that
    // the offsets fold into the instructions instead of taking registers
    constexpr uint32_t O_BAR = F32_STAGES * F32_STAGE + TS * TERM_STAGE + Cfg<NT>::SUM_BYTES;
    constexpr uint32_t O_F32_FULL = O_BAR, O_F32_EMPTY = O_BAR + 8 * F32_STAGES;
    constexpr uint32_t O_TERM_FULL = O_BAR + 8 * 2 * F32_STAGES, O_TERM_EMPTY = O_TERM_FULL + 8 * TS;
    constexpr uint32_t O_CHUNK_DONE = O_TERM_EMPTY + 8 * TS, O_DRAINED = O_CHUNK_DONE + 8;
    constexpr uint32_t O_ABORT = O_DRAINED + 8 + 8 + 4;   // after final_bar and the TMEM slot
    const uint32_t lead = peer_addr(sbase, 0);            // the leader CTA's shared memory, cluster window
    // running sums of columns col0 .. col0+NSR-1 in registers, the others in
    // shared memory (thread-contiguous: conflict-free), element j at
    // ssum + j * NCONV * 4
    float sum[NSR];
#pragma unroll
    for (int j = 0; j < NSR; ++j) sum[j] = 0.f;
    const uint32_t ssum = sbase + (uint32_t)(F32_STAGES * F32_STAGE + TS * TERM_STAGE) + 4 * tid;
    // drain cursor: unit du, chunk dci of it, global chunk dgc, its first global stage dstage
    // (the unit's tile and split are decoded again where needed, which keeps
    // the cursor at four registers)
    int du = cid, dci = 0;
    uint32_t dgc = 0, dstage = 0;
    auto unit_stages = [&](int u) -> int {
      if (u < t.F) return t.NKT;
      const int kb = ((u - t.F) % t.S) * t.ksplit;
      return min(t.NKT, kb + t.ksplit) - kb;
    };
    bool ok = true;
    auto chunk_end = [&]() -> uint32_t { return dstage + (uint32_t)min((dci + 1) * CHS, unit_stages(du)); };
    auto drain_one = [&]() -> bool {
      if (!__all_sync(0xffffffffu, mbar_wait32(sbase + O_CHUNK_DONE, dgc & 1, sbase + O_ABORT))) return false;
      tc_fence_after();
#pragma unroll
      for (int hh = 0; hh < 8; ++hh) {
        uint32_t rm[8], rc[8];
        __syncwarp();
        tmem_ld8(tmem_main + lane_off + (uint32_t)(col0 + 8 * hh), rm);
        tmem_ld8(tmem_cross + lane_off + (uint32_t)(col0 + 8 * hh), rc);
#pragma unroll
        for (int j = 0; j < 8; ++j) {
          const float v = __uint_as_float(rm[j]) + __uint_as_float(rc[j]);
          const int c = 8 * hh + j;
          if (c < NSR) {
            sum[c] = dci == 0 ? v : sum[c] + v;
          } else {
            const uint32_t sp = ssum + (uint32_t)((c - NSR) * NCONV * 4);
            sts32(sp, dci == 0 ? v : lds32(sp) + v);
          }
        }
      }
      tc_fence_before();
      __syncwarp();
      if (lane == 0) mbar_arrive_remote(lead + O_DRAINED);
      ++dgc;
      ++dci;
      const int dn = unit_stages(du);
      if (dci * CHS >= dn) {
        // the unit is complete: epilogue
        int dl, dmt, dnt, dkb, dke, dslot;
        decode(du, dl, dmt, dnt, dkb, dke, dslot);
        if (dslot >= 0) {
          const int64_t po = ((int64_t)dslot * 256 + col0) * 256 + rank * BM + row;
          float* pp = t.partial + po;
          if (in_bounds(po + 63 * 256, t.p_max, 2))
#pragma unroll
            for (int j = 0; j < 64; ++j)
              pp[(int64_t)j * 256] = j < NSR ? sum[j] : lds32(ssum + (uint32_t)((j - NSR) * NCONV * 4));
        } else {
          const int64_t m = (int64_t)dmt * 256 + rank * BM + row;
          if (m < g.M) {
            const float sx = scalar_as<float>(g.sx), sy = scalar_as<float>(g.sy);
            const int64_t roff = (g.L > 1 ? (int64_t)dl * g.l_sc[0] : 0) + m * g.m_sc[0];
            float* crow = static_cast<float*>(g.C) + roff;
            const int64_t nsc = g.n_sc[0];
            const int n0 = dnt * 256 + col0;
#pragma unroll
            for (int j = 0; j < 64; ++j) {
              if (n0 + j < g.N && in_bounds(roff + (int64_t)(n0 + j) * nsc, t.c_max, 1)) {
                float* cp = crow + (int64_t)(n0 + j) * nsc;
                const float v = j < NSR ? sum[j] : lds32(ssum + (uint32_t)((j - NSR) * NCONV * 4));
                float o = g.sx_one ? v : sx * v;
                if (!g.sy_zero) o = fmaf(sy, *cp, o);
                *cp = o;
              }
            }
          }
        }
        dstage += (uint32_t)dn;
        dci = 0;
        du += ncl;
      }
      return true;
    };

    uint32_t it = 0;
    for (int u = cid; u < t.units && ok; u += ncl) {
      int l, mt, nt, kb, ke, slot;
      decode(u, l, mt, nt, kb, ke, slot);
      for (int kt = kb; kt < ke; ++kt, ++it) {
        // drain every chunk whose MMAs precede the term stage waited on below
        while (du < t.units && chunk_end() + (uint32_t)TS <= it) {
          if (!drain_one()) { ok = false; break; }
        }
        if (!ok) break;
        const int s = it % F32_STAGES, ts = it % TS;
        // warp-uniform decisions: the warp-synchronous operations below need every lane
        if (!__all_sync(0xffffffffu, mbar_wait32(sbase + O_F32_FULL + 8 * s, (it / F32_STAGES) & 1, sbase + O_ABORT))) {
          ok = false;
          break;
        }
        if (it >= (uint32_t)TS &&
            !__all_sync(0xffffffffu, mbar_wait32(sbase + O_TERM_EMPTY + 8 * ts, ((it / TS) - 1) & 1, sbase + O_ABORT))) {
          ok = false;
          break;
        }
        const uint32_t src = f32_base + s * F32_STAGE + opnd * F32_TILE;
        const uint32_t dst = term_base + ts * TERM_STAGE + opnd * NT * TERM_TILE;
        if (opnd == 0) convert_tile<NT, AK>(src, dst, wl, lane);
        else convert_tile<NT, BKM>(src, dst, wl, lane);
        fence_proxy_async();
        __syncwarp();
        if (lane == 0) {
          mbar_arrive32(sbase + O_F32_EMPTY + 8 * s);
          mbar_arrive_remote(lead + O_TERM_FULL + 8 * ts);
        }
      }
    }
    while (ok && du < t.units) ok = drain_one();
    // the multicast commits that free the last term stages arrive on this
    // CTA's barriers from the leader's tensor core: wait for them to land
    // before this CTA's shared memory can be reassigned
    if (tid == 0)
      for (uint32_t i = it > (uint32_t)TS ? it - TS : 0; i < it; ++i)
        mbar_wait_quiesce(&term_empty[i % TS], (i / TS) & 1);
  }
  tc_fence_before();
  __syncthreads();
  cluster_sync_all();   // the peer's drains and the leader's MMAs are over
  if (warp == 17) {
    tc_fence_after();
    asm volatile("tcgen05.dealloc.cta_group::2.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(t2::TMEM_COLS) : "memory");
  }
}

// Sum the S split partials of each split 256 x 256 tile in split order; αβ epilogue.
__global__ void __launch_bounds__(256) k_splitk_tiles2(const __grid_constant__ T2Args t) {
  const GemmArgs& g = t.g;
  const float sx = scalar_as<float>(g.sx), sy = scalar_as<float>(g.sy);
  float* Cp = static_cast<float*>(g.C);
  const int64_t total = (int64_t)(t.tiles - t.F) * 256 * 256;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < total;
       i += (int64_t)gridDim.x * blockDim.x) {
    const int64_t mloc = i % 256;
    const int64_t r = i / 256;
    const int64_t nloc = r % 256;
    const int64_t v = r / 256;
    const int64_t tile = t.F + v;
    const int64_t mt = tile % t.TM, r2 = tile / t.TM, nt = r2 % t.TN, l = r2 / t.TN;
    const int64_t m = mt * 256 + mloc, n = nt * 256 + nloc;
    if (m >= g.M || n >= g.N) continue;
    float acc = 0.f;
    if (!in_bounds(((v * t.S + t.S - 1) * 256 + nloc) * 256 + mloc, t.p_max, 3)) continue;
    for (int s = 0; s < t.S; ++s) acc += t.partial[((v * t.S + s) * 256 + nloc) * 256 + mloc];
    const int64_t co = (g.L > 1 ? l * g.l_sc[0] : 0) + m * g.m_sc[0] + n * g.n_sc[0];
    if (!in_bounds(co, t.c_max, 3)) continue;
    float* cp = Cp + co;
    float o = g.sx_one ? acc : sx * acc;
    if (!g.sy_zero) o = fmaf(sy, *cp, o);
    *cp = o;
  }
}

namespace {
typedef CUresult (*EncodeTiledFn)(CUtensorMap*, CUtensorMapDataType, cuuint32_t, void*, const cuuint64_t*,
                                  const cuuint64_t*, const cuuint32_t*, const cuuint32_t*, CUtensorMapInterleave,
                                  CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);
EncodeTiledFn encode_fn() {
  static EncodeTiledFn fn = nullptr;
  static std::once_flag once;
  std::call_once(once, [] {
    void* p = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      fn = reinterpret_cast<EncodeTiledFn>(p);
    else
      cudaGetLastError();
  });
  return fn;
}

// Tensor map over one FP32 operand: rows R (stride rs), K (stride ks), batch
// L (stride ls; L == 1: a 2-D map).  kmajor (ks == 1): box (32 k, 128 rows);
// otherwise (rs == 1): box (32 rows, 32 k).  128-byte swizzle, zero fill.
bool make_operand_map(CUtensorMap* map, const void* base, int64_t R, int64_t K, int64_t L, int64_t rs, int64_t ks,
                      int64_t ls, bool kmajor) {
  EncodeTiledFn fn = encode_fn();
  if (!fn) return false;
  cuuint64_t dims[3], strides[2];
  cuuint32_t box[3], estr[3] = {1, 1, 1};
  if (kmajor) {
    dims[0] = (cuuint64_t)K; dims[1] = (cuuint64_t)R;
    strides[0] = (cuuint64_t)rs * 4;
    box[0] = 32; box[1] = 128;
  } else {
    dims[0] = (cuuint64_t)R; dims[1] = (cuuint64_t)K;
    strides[0] = (cuuint64_t)ks * 4;
    box[0] = 32; box[1] = 32;
  }
  dims[2] = (cuuint64_t)L;
  strides[1] = (cuuint64_t)ls * 4;
  box[2] = 1;
  const cuuint32_t rank = L > 1 ? 3 : 2;
  CUresult r = fn(map, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, rank, const_cast<void*>(base), dims, strides, box, estr,
                  CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                  CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  return r == CUDA_SUCCESS;
}

template <int NT, bool AK, bool BKM>
cudaError_t launch_t2(const T2Args& t, const CUtensorMap& ma, const CUtensorMap& mb, int grid, cudaStream_t s) {
  static std::atomic<unsigned long long> attr{0};
  const cudaError_t e = set_smem_once(attr, k_gemm_tma2<NT, AK, BKM>, t2::Cfg<NT>::SMEM_BYTES);
  if (e != cudaSuccess) return e;
  k_gemm_tma2<NT, AK, BKM><<<grid, t2::NTHREADS, t2::Cfg<NT>::SMEM_BYTES, s>>>(t, ma, mb);
  return cudaGetLastError();
}
}  // namespace

bool gemm_tma2_applies(const GemmArgs& g) {
  if (g.nm != 1 || g.nn != 1 || g.nk != 1 || g.nl != 1) return false;
  if (g.M < 1 || g.N < 1 || g.K < 1 || g.L < 1) return false;
  if (g.M >= (1ll << 31) || g.N >= (1ll << 31) || g.K >= (1ll << 31) || g.L >= (1ll << 31)) return false;
  const bool ak = g.k_sa[0] == 1, ar = g.m_sa[0] == 1;
  const bool bk = g.k_sb[0] == 1, br = g.n_sb[0] == 1;
  if (!(ak || ar) || !(bk || br)) return false;
  // tensor-map rules: 16-byte aligned bases and non-unit strides of whole 16-byte units
  if ((reinterpret_cast<uintptr_t>(g.A) & 15) || (reinterpret_cast<uintptr_t>(g.B) & 15)) return false;
  const int64_t sa = ak ? g.m_sa[0] : g.k_sa[0], sb = bk ? g.n_sb[0] : g.k_sb[0];
  if (sa <= 0 || sb <= 0 || sa % 4 || sb % 4 || sa >= (1ll << 37) || sb >= (1ll << 37)) return false;
  if (g.L > 1 && (g.l_sa[0] <= 0 || g.l_sb[0] <= 0 || g.l_sa[0] % 4 || g.l_sb[0] % 4 ||
                  g.l_sa[0] >= (1ll << 37) || g.l_sb[0] >= (1ll << 37)))
    return false;
  return true;
}

size_t gemm_tma2_bytes(const GemmArgs& g, int num_sms) {
  (void)g;
  return (size_t)(num_sms / 2) * 256 * 256 * 4 + 1024;
}

cudaError_t launch_gemm_tma2(const GemmArgs& g, int nterms, void* workspace, size_t ws_bytes, int num_sms,
                             cudaStream_t s) {
  if ((nterms != 2 && nterms != 3) || !gemm_tma2_applies(g)) return cudaErrorNotSupported;
  const bool ak = g.k_sa[0] == 1, bk = g.k_sb[0] == 1;
  alignas(64) CUtensorMap ma, mb;
  if (!make_operand_map(&ma, g.A, g.M, g.K, g.L, g.m_sa[0], g.k_sa[0], g.L > 1 ? g.l_sa[0] : 0, ak) ||
      !make_operand_map(&mb, g.B, g.N, g.K, g.L, g.n_sb[0], g.k_sb[0], g.L > 1 ? g.l_sb[0] : 0, bk))
    return cudaErrorNotSupported;
  const int64_t TM = (g.M + 255) / 256, TN = (g.N + 255) / 256, NKT = (g.K + t2::BK - 1) / t2::BK;
  const int64_t tiles = g.L * TM * TN;
  const int64_t G = std::max(1, num_sms / 2);   // clusters of two CTAs
  int64_t F = tiles >= G ? (tiles / G) * G : 0;
  int64_t Rt = tiles - F;
  int64_t S = 1;
  if (Rt > 0) {
    S = std::max<int64_t>(1, G / Rt);
    S = std::min<int64_t>(S, std::max<int64_t>(1, NKT / 8));
  }
  const int64_t ksplit = (NKT + S - 1) / S;
  S = (NKT + ksplit - 1) / ksplit;
  if (S == 1) {
    F = tiles;
    Rt = 0;
  }
  const int64_t units = F + Rt * S;
  // the kernel's unit, tile and stage counters are 32-bit
  if (tiles >= (1ll << 30) || units >= (1ll << 30) || NKT >= (1ll << 30)) return cudaErrorNotSupported;
  const size_t bytes_p = (size_t)Rt * S * 256 * 256 * 4;
  if (bytes_p > ws_bytes) return cudaErrorNotSupported;
  T2Args t;
  memset(&t, 0, sizeof(t));
  t.g = g;
  t.TM = (int)TM;
  t.TN = (int)TN;
  t.NKT = (int)NKT;
  t.tiles = (int)tiles;
  t.partial = static_cast<float*>(workspace);
  t.F = (int)F;
  t.S = (int)S;
  t.ksplit = (int)ksplit;
  t.units = (int)units;
  t.c_max = (g.M - 1) * g.m_sc[0] + (g.N - 1) * g.n_sc[0] + (g.L > 1 ? (g.L - 1) * g.l_sc[0] : 0);
  t.p_max = (int64_t)(bytes_p / 4) - 1;
  const int grid = (int)(2 * std::min<int64_t>(units, G));
  cudaError_t e;
  {
    KernelTimer kt(s, "k_gemm_tma2");
    if (nterms == 3) {
      e = ak ? (bk ? launch_t2<3, true, true>(t, ma, mb, grid, s) : launch_t2<3, true, false>(t, ma, mb, grid, s))
             : (bk ? launch_t2<3, false, true>(t, ma, mb, grid, s) : launch_t2<3, false, false>(t, ma, mb, grid, s));
    } else {
      e = ak ? (bk ? launch_t2<2, true, true>(t, ma, mb, grid, s) : launch_t2<2, true, false>(t, ma, mb, grid, s))
             : (bk ? launch_t2<2, false, true>(t, ma, mb, grid, s) : launch_t2<2, false, false>(t, ma, mb, grid, s));
    }
  }
  count_launch();
  if (e != cudaSuccess || Rt == 0) return e;
  const int64_t total = Rt * 256 * 256;
  const int64_t nb = (total + 255) / 256;
  k_splitk_tiles2<<<(unsigned)std::min<int64_t>(nb, (int64_t)num_sms * 16), 256, 0, s>>>(t);
  count_launch();
  return cudaGetLastError();
}

// ---------------------------------------------------------------------------
// k_gemm_bdiag: batches of small FP32 GEMMs whose batch mode is contiguous in
// A, B and C (Julia column-major bij,bjk->bik: b fastest), on the tensor
// cores.
//
// Two batches share one 128 x 128 MMA as a block-diagonal product: the A
// operand stacks A_b (64 rows) over A_b' (64 rows), the B operand stacks
// B_b^T over B_b'^T, and the diagonal blocks of D are C_b and C_b' (the
// off-diagonal products are computed and discarded: the kernel is bound by
// HBM, not by the tensor pipe).  A CTA owns 4 consecutive batches (16 bytes
// of every (row, k) run, one TMA box of 4 x 64 x 32 per operand and k stage),
// converts each stage into NT BF16 terms per value in shared memory (the
// UMMA K-major layout; conflict-free reads and writes), and one thread of
// warp 8 issues the MMAs of both pairs into main (t0*t0) and cross
// accumulators (4 x 128 TMEM columns) and the next stage's TMA loads.  The
// tile leaves through shared memory with the batch mode fastest, as 16-byte
// stores with the αβ epilogue.  Every wait is bounded.
namespace bd {
constexpr int BK = 32, NB = 4;
constexpr int F32_TILE = NB * 64 * BK * 4;   // one operand, one stage: 32 KB ([k][row][b])
constexpr int TERM_TILE = 128 * BK * 2;      // one term of one operand of one pair: 8 KB
constexpr int NCONV = 512, NTHREADS = NCONV + 32;   // converter warps 0-15, control warp 16
constexpr int TMEM_COLS = 512;
template <int NT> struct Cfg {
  static constexpr int F32_STAGE = 2 * F32_TILE;                // A, B
  static constexpr int TERM_BYTES = 2 * 2 * NT * TERM_TILE;     // pairs x operands x terms
  static constexpr int SMEM_BYTES = 2 * F32_STAGE + TERM_BYTES + 256 + 128;
};
}  // namespace bd

static_assert(bd::TERM_TILE == t2::TERM_TILE, "split8_store's term stride");

struct BdArgs {
  GemmArgs g;
  int nk;        // k stages of 32
  int64_t c_max; // largest element offset of C (self-check)
};

template <int NT>
__global__ void __launch_bounds__(bd::NTHREADS, 1)
    k_gemm_bdiag(const __grid_constant__ BdArgs t, const __grid_constant__ CUtensorMap mapA,
                 const __grid_constant__ CUtensorMap mapB) {
  using namespace bd;
  constexpr int F32_STAGE = Cfg<NT>::F32_STAGE;
  extern __shared__ __align__(128) unsigned char bd_raw[];
  const uint32_t raw = smem_u32(bd_raw);
  const uint32_t pad = (128u - (raw & 127u)) & 127u;
  unsigned char* smem = bd_raw + pad;
  const uint32_t sbase = raw + pad;
  const uint32_t f32_base = sbase, term_base = sbase + 2 * F32_STAGE;
  uint64_t* bars = reinterpret_cast<uint64_t*>(smem + 2 * F32_STAGE + Cfg<NT>::TERM_BYTES);
  uint64_t* full = bars;            // [2] TMA stage landed
  uint64_t* conv_done = bars + 2;   // the 8 converter warps wrote a stage's terms
  uint64_t* mma_done = bars + 3;    // the MMAs of a stage completed
  uint64_t* final_bar = bars + 4;   // every MMA completed (before TMEM is freed)
  uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(bars + 5);
  volatile int* abort_flag = reinterpret_cast<volatile int*>(tmem_slot + 1);

  const GemmArgs& g = t.g;
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int b0 = blockIdx.x * NB;
  if (tid == 0) {
    mbar_init(&full[0], 1);
    mbar_init(&full[1], 1);
    mbar_init(conv_done, 16);
    mbar_init(mma_done, 1);
    mbar_init(final_bar, 1);
    *abort_flag = 0;
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  if (warp == 16) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(tmem_slot)),
                 "r"(TMEM_COLS)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = *tmem_slot;

  if (warp == 16) {
    // ---------------- TMA loads and MMA issue (one thread) ----------------
    if (lane == 0) {
      auto load = [&](int c) {
        const int s = c & 1;
        mbar_expect_tx(&full[s], 2 * F32_TILE);
        tma_load_3d(f32_base + s * F32_STAGE, &mapA, b0, 0, c * BK, &full[s]);
        tma_load_3d(f32_base + s * F32_STAGE + F32_TILE, &mapB, b0, 0, c * BK, &full[s]);
      };
      load(0);
      if (t.nk > 1) load(1);
      int issued = t.nk > 1 ? 2 : 1;
      bool ok = true;
      for (int c = 0; c < t.nk && ok; ++c) {
        if (!mbar_wait(conv_done, c & 1, abort_flag)) { ok = false; break; }
        tc_fence_after();
        // the converters are done with stage c & 1: the stage after next may land there
        if (c + 2 < t.nk) {
          load(c + 2);
          ++issued;
        }
#pragma unroll
        for (int p = 0; p < 2; ++p) {
          const uint32_t sa = term_base + (uint32_t)((p * 2 + 0) * NT * TERM_TILE);
          const uint32_t sb = term_base + (uint32_t)((p * 2 + 1) * NT * TERM_TILE);
          const uint32_t dmain = tmem + 256 * p, dcross = tmem + 256 * p + 128;
#pragma unroll
          for (int kk = 0; kk < 2; ++kk) {
            uint64_t ad[NT], bdsc[NT];
#pragma unroll
            for (int q = 0; q < NT; ++q) {
              ad[q] = umma_desc(sa + q * TERM_TILE + kk * 256);
              bdsc[q] = umma_desc(sb + q * TERM_TILE + kk * 256);
            }
            const uint32_t keep = (c == 0 && kk == 0) ? 0u : 1u;
            umma_bf16(dmain, ad[0], bdsc[0], keep);
            bool first_cross = true;
#pragma unroll
            for (int d = 1; d < NT; ++d)
#pragma unroll
              for (int i = 0; i <= d; ++i) {
                umma_bf16(dcross, ad[i], bdsc[d - i], first_cross ? keep : 1u);
                first_cross = false;
              }
          }
        }
        umma_commit(mma_done);
      }
      // every MMA this thread issued must finish before TMEM is freed, and
      // this CTA's copies in flight must land before it exits
      umma_commit(final_bar);
      mbar_wait_quiesce(final_bar, 0);
      for (int c = issued - 2 > 0 ? issued - 2 : 0; c < issued; ++c) mbar_wait_quiesce(&full[c & 1], (c >> 1) & 1);
    }
  } else {
    // ---------------- converters, then drain and epilogue (warps 0-15) ----------------
    // unit (row, 8 k at 8 * c8) of all 4 batches of operand op
    const int row = tid & 63, c8 = (tid >> 6) & 3, op = tid >> 8;
    bool ok = true;
    for (int c = 0; c < t.nk; ++c) {
      // warp-uniform decisions: the warp-synchronous operations below need every lane
      if (!__all_sync(0xffffffffu, mbar_wait(&full[c & 1], (c >> 1) & 1, abort_flag))) { ok = false; break; }
      if (c > 0 && !__all_sync(0xffffffffu, mbar_wait(mma_done, (c - 1) & 1, abort_flag))) {   // terms free again
        ok = false;
        break;
      }
      {
        const uint32_t src = f32_base + (c & 1) * F32_STAGE + op * F32_TILE;
        float v[NB][8];
#pragma unroll
        for (int kk = 0; kk < 8; ++kk) {
          const float4 w = lds128(src + (uint32_t)(((8 * c8 + kk) * 64 + row) * 16));
          v[0][kk] = w.x;
          v[1][kk] = w.y;
          v[2][kk] = w.z;
          v[3][kk] = w.w;
        }
#pragma unroll
        for (int b = 0; b < NB; ++b) {
          const int r = (b & 1) * 64 + row;
          const uint32_t dst = term_base + (uint32_t)((((b >> 1) * 2 + op) * NT) * TERM_TILE) +
                               (uint32_t)(((r >> 3) * 4 + c8) * 128 + (r & 7) * 16);
          split8_store<NT>(v[b], dst);   // term stride t2::TERM_TILE == bd::TERM_TILE
        }
      }
      fence_proxy_async();
      __syncwarp();
      if (lane == 0) mbar_arrive(conv_done);
    }
    // drain: warp w reads TMEM lanes 32 (w & 3).. of pair (w >> 2) & 1, 32 of
    // the columns (half w >> 3); row r of the pair's D is batch 2p + (r >> 6),
    // row r & 63; its diagonal block is columns 64 (r >> 6) ..
    if (ok) ok = __all_sync(0xffffffffu, mbar_wait(mma_done, (t.nk - 1) & 1, abort_flag));
    if (ok) {
      tc_fence_after();
      const int q = warp & 3, p = (warp >> 2) & 1, ch = warp >> 3;
      const int r = 32 * q + lane;
      const int bl = 2 * p + (r >> 6), i = r & 63;
      const uint32_t lane_off = (uint32_t)(32 * q) << 16;
      const uint32_t col = (uint32_t)(256 * p + 64 * (r >> 6) + 32 * ch);
      // staging [b][n][i] (i fastest) in the first FP32 stage, free by now
      float* cs = reinterpret_cast<float*>(smem);
#pragma unroll
      for (int h = 0; h < 4; ++h) {
        uint32_t rm[8], rc[8];
        __syncwarp();
        tmem_ld8(tmem + lane_off + col + 8 * h, rm);
        tmem_ld8(tmem + lane_off + col + 128 + 8 * h, rc);
#pragma unroll
        for (int j = 0; j < 8; ++j)
          cs[(bl * 64 + 32 * ch + 8 * h + j) * 64 + i] = __uint_as_float(rm[j]) + __uint_as_float(rc[j]);
      }
    }
    tc_fence_before();
    asm volatile("bar.sync 1, 512;" ::: "memory");   // the 16 converter warps only
    if (ok) {
      // 16-byte stores: 4 batches of one (row, column), batch mode fastest
      const float* cs = reinterpret_cast<const float*>(smem);
      const float sx = scalar_as<float>(g.sx), sy = scalar_as<float>(g.sy);
      float* Cp = static_cast<float*>(g.C);
      const int nb = min(NB, (int)(g.L - b0));
      for (int e = tid; e < 64 * 64; e += NCONV) {
        const int i = e & 63, n = e >> 6;
        if (i >= g.M || n >= g.N) continue;
        float o[NB];
#pragma unroll
        for (int b = 0; b < NB; ++b) {
          const float v = cs[(b * 64 + n) * 64 + i];
          o[b] = g.sx_one ? v : sx * v;
        }
        const int64_t co = b0 + (int64_t)i * g.m_sc[0] + (int64_t)n * g.n_sc[0];
        if (!in_bounds(co + nb - 1, t.c_max, 4)) continue;
        float* cp = Cp + co;
        if (nb == NB) {
          if (!g.sy_zero) {
            const float4 old = *reinterpret_cast<const float4*>(cp);
            o[0] = fmaf(sy, old.x, o[0]);
            o[1] = fmaf(sy, old.y, o[1]);
            o[2] = fmaf(sy, old.z, o[2]);
            o[3] = fmaf(sy, old.w, o[3]);
          }
          *reinterpret_cast<float4*>(cp) = make_float4(o[0], o[1], o[2], o[3]);
        } else {
          for (int b = 0; b < nb; ++b) cp[b] = g.sy_zero ? o[b] : fmaf(sy, cp[b], o[b]);
        }
      }
    }
  }
  tc_fence_before();
  __syncthreads();
  if (warp == 16) {
    tc_fence_after();
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(bd::TMEM_COLS) : "memory");
  }
}

namespace {
// 3-D FP32 tensor map, no swizzle: dims[0] is the contiguous mode; strides in
// bytes of dims 1 and 2.
bool make_map3(CUtensorMap* map, const void* base, const cuuint64_t (&dims)[3], const cuuint64_t (&strides)[2],
               const cuuint32_t (&box)[3]) {
  EncodeTiledFn fn = encode_fn();
  if (!fn) return false;
  cuuint32_t estr[3] = {1, 1, 1};
  CUresult r = fn(map, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 3, const_cast<void*>(base), dims, strides, box, estr,
                  CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
                  CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  return r == CUDA_SUCCESS;
}
}  // namespace

bool gemm_bdiag_applies(const GemmArgs& g) {
  if (g.nm != 1 || g.nn != 1 || g.nk != 1 || g.nl != 1) return false;
  if (g.l_sa[0] != 1 || g.l_sb[0] != 1 || g.l_sc[0] != 1) return false;
  if (g.M < 1 || g.M > 64 || g.N < 1 || g.N > 64 || g.K < 1 || g.K > 256 || g.L < 4 || g.L >= (1ll << 31))
    return false;
  const int64_t st[6] = {g.m_sa[0], g.k_sa[0], g.n_sb[0], g.k_sb[0], g.m_sc[0], g.n_sc[0]};
  for (int64_t v : st)
    if (v <= 0 || v % 4 || v >= (1ll << 37)) return false;
  return !((reinterpret_cast<uintptr_t>(g.A) | reinterpret_cast<uintptr_t>(g.B) | reinterpret_cast<uintptr_t>(g.C)) &
           15);
}

cudaError_t launch_gemm_bdiag(const GemmArgs& g, int nterms, cudaStream_t s) {
  if ((nterms != 2 && nterms != 3) || !gemm_bdiag_applies(g)) return cudaErrorNotSupported;
  alignas(64) CUtensorMap ma, mb;
  const cuuint32_t box[3] = {4, 64, 32};
  const cuuint64_t da[3] = {(cuuint64_t)g.L, (cuuint64_t)g.M, (cuuint64_t)g.K};
  const cuuint64_t sa[2] = {(cuuint64_t)g.m_sa[0] * 4, (cuuint64_t)g.k_sa[0] * 4};
  const cuuint64_t db[3] = {(cuuint64_t)g.L, (cuuint64_t)g.N, (cuuint64_t)g.K};
  const cuuint64_t sb[2] = {(cuuint64_t)g.n_sb[0] * 4, (cuuint64_t)g.k_sb[0] * 4};
  if (!make_map3(&ma, g.A, da, sa, box) || !make_map3(&mb, g.B, db, sb, box)) return cudaErrorNotSupported;
  BdArgs t;
  memset(&t, 0, sizeof(t));
  t.g = g;
  t.nk = (int)((g.K + bd::BK - 1) / bd::BK);
  t.c_max = (g.L - 1) + (g.M - 1) * g.m_sc[0] + (g.N - 1) * g.n_sc[0];
  const unsigned grid = (unsigned)((g.L + bd::NB - 1) / bd::NB);
  static std::atomic<unsigned long long> attr2{0}, attr3{0};
  cudaError_t e = nterms == 3 ? set_smem_once(attr3, k_gemm_bdiag<3>, bd::Cfg<3>::SMEM_BYTES)
                              : set_smem_once(attr2, k_gemm_bdiag<2>, bd::Cfg<2>::SMEM_BYTES);
  if (e != cudaSuccess) return e;
  {
    KernelTimer kt(s, "k_gemm_bdiag");
    if (nterms == 3) k_gemm_bdiag<3><<<grid, bd::NTHREADS, bd::Cfg<3>::SMEM_BYTES, s>>>(t, ma, mb);
    else k_gemm_bdiag<2><<<grid, bd::NTHREADS, bd::Cfg<2>::SMEM_BYTES, s>>>(t, ma, mb);
  }
  count_launch();
  return cudaGetLastError();
}

// ---------------------------------------------------------------------------
// k_group_tc: one persistent launch over the tiles of many uneven binary
// contractions (a grouped GEMM: the MPS transfer contractions of a sweep), on
// the tensor cores.
//
// Complex64 problems run as real GEMMs of their 2 x 2 embedding: with
// A' [(m, p), (k, q)] = (q == p ? Re A : (p == 0 ? -Im A : Im A))[m, k] and
// B' [(k, q), n] = (q == 0 ? Re B : Im B)[k, n], C' = A' B' holds
// C'[(m, 0), n] = Re C[m, n] and C'[(m, 1), n] = Im C[m, n] -- four real
// products per complex one, as many as the four real GEMMs, and C' is C's own
// interleaved storage.
//
// Warp roles (14 warps, one CTA per SM):
//   13     scheduler: walks this CTA's tiles (tile = blockIdx.x + j gridDim.x),
//          looks up each tile's problem in a host-built tile -> problem table
//          and stages the problem's descriptor and the tile's (l, m, n)
//          coordinates in a ring of shared-memory slots;
//   0-7    converters: load each 32-wide (real) k stage of a tile's A' and B'
//          straight from the strided inputs (the next stage's loads are in
//          flight while the current one is split), split it into NT BF16
//          terms and store them in the UMMA K-major layout;
//   12     MMA issue (lane 0): main and cross-term accumulators, two TMEM
//          buffers, a fresh accumulation every CHUNK stages;
//   8-11   drain (one warp per TMEM lane quarter): each finished chunk into FP32 running sums in shared
//          memory; the tile's last chunk goes straight from TMEM through the
//          alpha-beta epilogue to the output (complex: the two parts of an
//          element are neighbouring lanes).
// A tile's drain and epilogue overlap the next tile's loads and MMAs.  Every
// wait is bounded.
namespace gt {
constexpr int BM = 128, BN = 128, BK = 32, CHUNK = 8;
constexpr int TILE_BYTES = BM * BK * 2;      // one term of one operand, one stage: 8 KB
constexpr int NTHREADS = 14 * 32;            // at most 4 warps per SM quarter: 128 registers a thread
constexpr int ACC_BYTES = BM * BN * 4;
constexpr int TMEM_COLS = 512;
constexpr int NSLOT = 8;                     // scheduler ring
constexpr int SLOT_BYTES = 192;
constexpr int SLOT_USERS = 13;               // 8 converter warps + 4 drain warps + the MMA thread
template <int NT> struct Cfg {
  static constexpr int STAGE_BYTES = 2 * NT * TILE_BYTES;
  static constexpr int STAGES = NT == 2 ? 4 : 3;
  static constexpr int SMEM_BYTES = STAGES * STAGE_BYTES + ACC_BYTES + NSLOT * SLOT_BYTES + 512 + 128;
};
}  // namespace gt

// One staged tile: its problem and the tile's coordinates.
struct __align__(16) GtTile {
  GroupProblem p;
  int64_t li, mt, nt;
};
static_assert(sizeof(GtTile) <= gt::SLOT_BYTES, "scheduler slot");
static_assert(sizeof(GroupProblem) % 8 == 0 && sizeof(GroupProblem) / 8 <= 32, "descriptor copy by one warp");

struct GtArgs {
  const GroupProblem* probs;
  const int32_t* tile_prob;   // [tiles] owning problem of each global tile
  int nprob;
  int64_t tiles;
  Scalar sx, sy;
  int sy_zero, sx_one;
};

template <bool CPLX>
__device__ __forceinline__ int gt_stages(const GroupProblem& p) {
  const int64_t kr = CPLX ? 2 * p.k : p.k;   // real K of the (embedded) GEMM
  return (int)((kr + gt::BK - 1) / gt::BK);
}

static_assert(gt::TILE_BYTES == t2::TERM_TILE, "split8_store's term stride");

__device__ __forceinline__ void tmem_ld16_nw(uint32_t taddr, uint32_t (&r)[16]) {
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x16.b32 "
      "{%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
        "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
      : "r"(taddr));
}
__device__ __forceinline__ void tmem_wait_ld() { asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory"); }

// kind::f16 BF16 x BF16 -> F32, K-major A and B, M = 128, N = n (a multiple
// of 16 up to 256): a tile whose problem ends inside it multiplies only the
// columns it has.
__host__ __device__ constexpr uint32_t gt_idesc(uint32_t n) {
  return (1u << 4) | (1u << 7) | (1u << 10) | ((n >> 3) << 17) | ((uint32_t)(128 >> 4) << 24);
}
__device__ __forceinline__ void umma_bf16_i(uint32_t d_tmem, uint64_t a, uint64_t b, uint32_t idesc, uint32_t acc) {
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "setp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}\n" ::"r"(d_tmem),
      "l"(a), "l"(b), "r"(idesc), "r"(acc));
}
// Columns of tile nt that hold output (1..128).
__device__ __forceinline__ int gt_cols(const GtTile* ti) {
  const int64_t r = ti->p.n - ti->nt * 128;
  return r < 128 ? (int)r : 128;
}
static_assert(gt_idesc(128) == tc::IDESC, "instruction descriptor");

// Scheduler warp: stage every tile of this CTA, in order, in the slot ring.
__device__ __forceinline__ void gt_scheduler(const GtArgs& t, unsigned char* slots, uint64_t* sched_full,
                                             uint64_t* sched_empty, volatile int* abort_flag, int lane) {
  using namespace gt;
  uint32_t j = 0;
  for (int64_t tile = blockIdx.x; tile < t.tiles; tile += gridDim.x, ++j) {
    const int s = j % NSLOT;
    if (j >= (uint32_t)NSLOT &&
        !__all_sync(0xffffffffu, mbar_wait(&sched_empty[s], ((j / NSLOT) - 1) & 1, abort_flag)))
      return;
    const int pi = __ldg(t.tile_prob + tile);
    bool bad = pi < 0 || pi >= t.nprob;
    int64_t r = 0, tm = 1, per_l = 1;
    if (!bad) {
      const GroupProblem& p = t.probs[pi];
      r = tile - __ldg(&p.tile_begin);
      tm = __ldg(&p.tiles_m);
      per_l = tm * __ldg(&p.tiles_n);
      bad = per_l <= 0 || r < 0 || r >= per_l * __ldg(&p.l);
    }
    if (bad) {   // a table that does not match the problems: record it and stop
      if (lane == 0) {
        atomicCAS(&g_ome_bounds, 0, 5);
        *abort_flag = 1;
      }
      return;
    }
    GtTile* ti = reinterpret_cast<GtTile*>(slots + s * SLOT_BYTES);
    const uint64_t* src = reinterpret_cast<const uint64_t*>(t.probs + pi);
    if (lane < (int)(sizeof(GroupProblem) / 8)) reinterpret_cast<uint64_t*>(&ti->p)[lane] = __ldg(src + lane);
    if (lane == 0) {
      const int64_t li = r / per_l;
      r -= li * per_l;
      ti->li = li;
      ti->mt = r % tm;
      ti->nt = r / tm;
    }
    __syncwarp();
    if (lane == 0) mbar_arrive(&sched_full[s]);
  }
}

// One converter thread's share of one stage, in registers.
//   complex: A' rows 2m, 2m+1 from 4 complex k of one row m of A; B' from
//            2 x 4 complex k of one column n of B;
//   real:    2 x 8 k of one row of A and of one column of B.
template <bool CPLX> struct GtRegs;
template <> struct GtRegs<true> {
  float2 a[4], b[8];
  uint32_t ok;   // bit 0: the A row lies in the problem, bit 1: the B column does
};
template <> struct GtRegs<false> {
  float a[16], b[16];
  uint32_t ok;
};

// A converter thread's row of A and column of B in the current tile (null
// when outside the problem), K and the K strides, fixed for the tile's stages.
struct GtRows {
  const float* a;
  const float* b;
  int64_t K, ask, bsk;
  int akv, bkv;
};

template <bool CPLX>
__device__ __forceinline__ GtRows gt_rows(const GtTile* ti, int tid) {
  const GroupProblem& p = ti->p;
  constexpr int E = CPLX ? 2 : 1;   // floats per element
  const int64_t li = ti->li;
  const int64_t m = CPLX ? ti->mt * 64 + (tid & 63) : ti->mt * 128 + (tid & 127);
  const int64_t n = ti->nt * 128 + (tid & 127);
  GtRows w;
  w.a = m < p.m ? static_cast<const float*>(p.a) + E * (li * p.a_sl + m * p.a_sm) : nullptr;
  w.b = n < p.n ? static_cast<const float*>(p.b) + E * (li * p.b_sl + n * p.b_sn) : nullptr;
  w.K = p.k;
  w.ask = p.a_sk;
  w.bsk = p.b_sk;
  w.akv = p.a_kvec;
  w.bkv = p.b_kvec;
  return w;
}

// 4 complex (or 8 real) consecutive k of one operand row starting at k0:
// two 16-byte loads when the row is K-contiguous and 16-byte aligned (kvec)
// and the run lies inside K, element loads otherwise; zeros for a null row.
__device__ __forceinline__ void gt_ld4c(const float* rowf, int64_t sk, int64_t k0, int64_t K, int kvec,
                                        float2* out) {
  const float2* row = reinterpret_cast<const float2*>(rowf);
  if (!row) {
#pragma unroll
    for (int j = 0; j < 4; ++j) out[j] = make_float2(0.f, 0.f);
  } else if (kvec && k0 + 4 <= K) {
    const float4* q = reinterpret_cast<const float4*>(row + k0);
    const float4 u0 = __ldg(q), u1 = __ldg(q + 1);
    out[0] = make_float2(u0.x, u0.y);
    out[1] = make_float2(u0.z, u0.w);
    out[2] = make_float2(u1.x, u1.y);
    out[3] = make_float2(u1.z, u1.w);
  } else {
#pragma unroll
    for (int j = 0; j < 4; ++j) out[j] = k0 + j < K ? __ldg(row + (k0 + j) * sk) : make_float2(0.f, 0.f);
  }
}
__device__ __forceinline__ void gt_ld8r(const float* row, int64_t sk, int64_t k0, int64_t K, int kvec, float* out) {
  if (!row) {
#pragma unroll
    for (int j = 0; j < 8; ++j) out[j] = 0.f;
  } else if (kvec && k0 + 8 <= K) {
    const float4* q = reinterpret_cast<const float4*>(row + k0);
    const float4 u0 = __ldg(q), u1 = __ldg(q + 1);
    out[0] = u0.x; out[1] = u0.y; out[2] = u0.z; out[3] = u0.w;
    out[4] = u1.x; out[5] = u1.y; out[6] = u1.z; out[7] = u1.w;
  } else {
#pragma unroll
    for (int j = 0; j < 8; ++j) out[j] = k0 + j < K ? __ldg(row + (k0 + j) * sk) : 0.f;
  }
}

__device__ __forceinline__ void gt_load(const GtRows& w, int kt, int tid, GtRegs<true>& r) {
  r.ok = (w.a ? 1u : 0u) | (w.b ? 2u : 0u);
  gt_ld4c(w.a, w.ask, (int64_t)kt * 16 + 4 * (tid >> 6), w.K, w.akv, r.a);
#pragma unroll
  for (int u = 0; u < 2; ++u) gt_ld4c(w.b, w.bsk, (int64_t)kt * 16 + 4 * ((tid >> 7) + 2 * u), w.K, w.bkv, r.b + 4 * u);
}

__device__ __forceinline__ void gt_load(const GtRows& w, int kt, int tid, GtRegs<false>& r) {
  r.ok = (w.a ? 1u : 0u) | (w.b ? 2u : 0u);
#pragma unroll
  for (int u = 0; u < 2; ++u) {
    const int64_t k0 = (int64_t)kt * 32 + 8 * ((tid >> 7) + 2 * u);
    gt_ld8r(w.a, w.ask, k0, w.K, w.akv, r.a + 8 * u);
    gt_ld8r(w.b, w.bsk, k0, w.K, w.bkv, r.b + 8 * u);
  }
}

// The NT BF16 terms of x (each in the upper 16 bits of t[u]; low bits are
// rounding residue), by the integer rounding of split8_store.  The split is
// odd in x: the terms of -x are those of x with the sign bit flipped.
template <int NT>
__device__ __forceinline__ void split_terms(float x, uint32_t (&t)[NT]) {
#pragma unroll
  for (int u = 0; u < NT; ++u) {
    const uint32_t r = __float_as_uint(x) + (NT == 3 && u == 2 ? 0u : 0x8000u);   // last of 3: truncated
    t[u] = r;
    if (u + 1 < NT) x -= __uint_as_float(r & 0xffff0000u);
  }
}
__device__ __forceinline__ uint32_t pack_hi(uint32_t lo, uint32_t hi) { return __byte_perm(lo, hi, 0x7632); }

// Split one stage's registers into NT BF16 terms in the K-major core-matrix
// layout (8 rows x 16 bytes per core matrix; 4 k-chunks per 8-row group).
template <int NT>
__device__ __forceinline__ void gt_store(const GtRegs<true>& r, uint32_t st, int tid, int lane) {
  const int ml = tid & 63, c8 = tid >> 6;
  // Rows 2m = (re, -im) and 2m+1 = (im, re) of the embedding.  The thread
  // stores row 2m + firstp first (each quarter-warp's 16-byte stores then hit
  // eight distinct bank groups) as pairs (x, y); the other row's pairs are
  // (s y, -s x) with s = +1 for firstp = 1 and -1 for firstp = 0, i.e. the
  // same terms with the sign of one half flipped.
  // Rows outside the problem are not written: they only reach accumulator
  // rows and columns that are never stored.
  const int firstp = (lane >> 2) & 1;
  const uint32_t flip = firstp ? 0x80000000u : 0x00008000u;
  if (r.ok & 1u) {
  uint32_t tx[4][NT], ty[4][NT];
#pragma unroll
  for (int j = 0; j < 4; ++j) {
    split_terms<NT>(firstp ? r.a[j].y : r.a[j].x, tx[j]);
    split_terms<NT>(firstp ? r.a[j].x : -r.a[j].y, ty[j]);
  }
  const int r1 = 2 * ml + firstp, r2 = 2 * ml + (firstp ^ 1);
  const uint32_t o1 = st + (uint32_t)(((r1 >> 3) * 4 + c8) * 128 + (r1 & 7) * 16);
  const uint32_t o2 = st + (uint32_t)(((r2 >> 3) * 4 + c8) * 128 + (r2 & 7) * 16);
#pragma unroll
  for (int u = 0; u < NT; ++u) {
    sts128(o1 + u * gt::TILE_BYTES, make_uint4(pack_hi(tx[0][u], ty[0][u]), pack_hi(tx[1][u], ty[1][u]),
                                               pack_hi(tx[2][u], ty[2][u]), pack_hi(tx[3][u], ty[3][u])));
    sts128(o2 + u * gt::TILE_BYTES,
           make_uint4(pack_hi(ty[0][u], tx[0][u]) ^ flip, pack_hi(ty[1][u], tx[1][u]) ^ flip,
                      pack_hi(ty[2][u], tx[2][u]) ^ flip, pack_hi(ty[3][u], tx[3][u]) ^ flip));
  }
  }
  if (!(r.ok & 2u)) return;
  const int nl = tid & 127;
#pragma unroll
  for (int u = 0; u < 2; ++u) {
    const int c8b = (tid >> 7) + 2 * u;
    uint32_t tr[4][NT], tq[4][NT];
#pragma unroll
    for (int j = 0; j < 4; ++j) {
      split_terms<NT>(r.b[4 * u + j].x, tr[j]);
      split_terms<NT>(r.b[4 * u + j].y, tq[j]);
    }
    const uint32_t ob = st + gt::Cfg<NT>::STAGE_BYTES / 2 + (uint32_t)(((nl >> 3) * 4 + c8b) * 128 + (nl & 7) * 16);
#pragma unroll
    for (int t = 0; t < NT; ++t)
      sts128(ob + t * gt::TILE_BYTES, make_uint4(pack_hi(tr[0][t], tq[0][t]), pack_hi(tr[1][t], tq[1][t]),
                                                 pack_hi(tr[2][t], tq[2][t]), pack_hi(tr[3][t], tq[3][t])));
  }
}

template <int NT>
__device__ __forceinline__ void gt_store(const GtRegs<false>& r, uint32_t st, int tid, int lane) {
  (void)lane;
  const int rl = tid & 127;
#pragma unroll
  for (int u = 0; u < 2; ++u) {
    const int c8 = (tid >> 7) + 2 * u;
    const uint32_t so = (uint32_t)(((rl >> 3) * 4 + c8) * 128 + (rl & 7) * 16);
    float va[8], vb[8];
#pragma unroll
    for (int j = 0; j < 8; ++j) {
      va[j] = r.a[8 * u + j];
      vb[j] = r.b[8 * u + j];
    }
    // rows outside the problem only reach discarded accumulator rows / columns
    if (r.ok & 1u) split8_store<NT>(va, st + so);
    if (r.ok & 2u) split8_store<NT>(vb, st + gt::Cfg<NT>::STAGE_BYTES / 2 + so);
  }
}

// Wait for this CTA's tile j (tile index tl) in the scheduler ring and skip
// forward over tiles without k stages (K = 0: releasing their slots).
// 1: (j, tl, ti, nkt) is the next tile with stages; 0: none left; -1: aborted.
template <bool CPLX>
__device__ __forceinline__ int gt_next_tile(const GtArgs& t, unsigned char* slots, uint64_t* sched_full,
                                            uint64_t* sched_empty, volatile int* abort_flag, int lane,
                                            uint32_t& j, int64_t& tl, const GtTile*& ti, int& nkt) {
  using namespace gt;
  for (; tl < t.tiles; tl += gridDim.x, ++j) {
    const int s = j % NSLOT;
    if (!__all_sync(0xffffffffu, mbar_wait(&sched_full[s], (j / NSLOT) & 1, abort_flag))) return -1;
    ti = reinterpret_cast<const GtTile*>(slots + s * SLOT_BYTES);
    nkt = gt_stages<CPLX>(ti->p);
    if (nkt > 0) return 1;
    __syncwarp();
    if (lane == 0) mbar_arrive(&sched_empty[s]);
  }
  return 0;
}

// Converter warps 0-7: every stage of every tile of this CTA, in order.  A
// load cursor runs PD stages (of this tile or the following ones) ahead of
// the stage being split and stored, so PD stages of global loads are in
// flight while a thread converts.
template <bool CPLX>
struct GtCursor {
  uint32_t j;            // position of the cursor's tile in this CTA's sequence
  int64_t tile;
  const GtTile* ti;
  int nk, kt;
  bool more;
  GtRows w;
};

// Issue the loads of the cursor's stage into r, note whether it ends its tile
// (rel = the tile's slot, else -1) and step the cursor.  False when aborted.
template <bool CPLX>
__device__ __forceinline__ bool gt_issue(const GtArgs& t, unsigned char* slots, uint64_t* sched_full,
                                         uint64_t* sched_empty, volatile int* abort_flag, int tid, int lane,
                                         GtCursor<CPLX>& c, GtRegs<CPLX>& r, int& rel, bool& have) {
  have = c.more;
  if (!c.more) return true;
  gt_load(c.w, c.kt, tid, r);
  rel = c.kt + 1 == c.nk ? (int)(c.j % gt::NSLOT) : -1;
  if (++c.kt == c.nk) {
    ++c.j;
    c.tile += gridDim.x;
    c.kt = 0;
    const int rn = gt_next_tile<CPLX>(t, slots, sched_full, sched_empty, abort_flag, lane, c.j, c.tile, c.ti, c.nk);
    if (rn < 0) return false;
    c.more = rn == 1;
    if (c.more) c.w = gt_rows<CPLX>(c.ti, tid);
  }
  return true;
}

template <int NT, bool CPLX>
__device__ __forceinline__ void gt_converters(const GtArgs& t, uint32_t sbase, unsigned char* slots,
                                              uint64_t* sched_full, uint64_t* sched_empty, uint64_t* full,
                                              uint64_t* empty, volatile int* abort_flag, int warp, int lane) {
  using namespace gt;
  constexpr int STAGES = Cfg<NT>::STAGES, STAGE_BYTES = Cfg<NT>::STAGE_BYTES;
  constexpr int PD = CPLX ? 2 : 1;   // register budget: 24 floats a stage (complex), 32 (real)
  const int tid = warp * 32 + lane;
  GtCursor<CPLX> c;
  c.j = 0;
  c.tile = blockIdx.x;
  c.kt = 0;
  const int rc = gt_next_tile<CPLX>(t, slots, sched_full, sched_empty, abort_flag, lane, c.j, c.tile, c.ti, c.nk);
  if (rc <= 0) return;
  c.more = true;
  c.w = gt_rows<CPLX>(c.ti, tid);
  GtRegs<CPLX> r[PD + 1];
  int rel[PD + 1];
  bool have[PD + 1];
#pragma unroll
  for (int q = 0; q < PD; ++q)
    if (!gt_issue<CPLX>(t, slots, sched_full, sched_empty, abort_flag, tid, lane, c, r[q], rel[q], have[q])) return;
  uint32_t it = 0;
  while (have[0]) {
    if (!gt_issue<CPLX>(t, slots, sched_full, sched_empty, abort_flag, tid, lane, c, r[PD], rel[PD], have[PD]))
      return;
    const int s = it % STAGES;
    if (it >= (uint32_t)STAGES &&
        !__all_sync(0xffffffffu, mbar_wait(&empty[s], ((it / STAGES) - 1) & 1, abort_flag)))
      return;
    gt_store<NT>(r[0], sbase + s * STAGE_BYTES, tid, lane);
    fence_proxy_async();
    __syncwarp();
    if (lane == 0) mbar_arrive(&full[s]);
    ++it;
    if (rel[0] >= 0 && lane == 0) mbar_arrive(&sched_empty[rel[0]]);   // done with that tile's slot
#pragma unroll
    for (int q = 0; q < PD; ++q) {
      r[q] = r[q + 1];
      rel[q] = rel[q + 1];
      have[q] = have[q + 1];
    }
  }
}

// Write 16 columns (colbase .. +15 of the tile) of accumulator row `row`
// through the alpha-beta epilogue.  Complex: the row is real row 2m + part of
// the embedding; the element's other part is in the neighbouring lane, and
// each lane reads and writes only its own part.
template <bool CPLX>
__device__ __forceinline__ void gt_store_cols(const GtArgs& t, const GtTile* ti, int row, int colbase,
                                              const float (&v)[16]) {
  const GroupProblem& p = ti->p;
  const int64_t pm = p.m, pn = p.n, csm = p.c_sm, csn = p.c_sn, n0 = ti->nt * 128 + colbase;
  if constexpr (CPLX) {
    const cf32 sx = scalar_as<cf32>(t.sx), sy = scalar_as<cf32>(t.sy);
    const int part = row & 1;
    const int64_t m = ti->mt * 64 + (row >> 1);
    float* C = static_cast<float*>(p.c) + 2 * (ti->li * p.c_sl + m * csm) + part;
    const bool mrow = m < pm;
    if (t.sy_zero && sx.im == 0.f) {   // a real scale of each part: no exchange between the lanes
      if (!mrow) return;
      const int64_t nv = pn - n0;
      float* cp = C + 2 * n0 * csn;
#pragma unroll
      for (int j = 0; j < 16; ++j, cp += 2 * csn)
        if (j < nv) *cp = sx.re * v[j];
      return;
    }
#pragma unroll
    for (int j = 0; j < 16; ++j) {
      const int64_t n = n0 + j;
      const bool in = mrow && n < pn;   // the same for both lanes of an element
      float* cp = C + 2 * n * csn;
      const float y = in && !t.sy_zero ? *cp : 0.f;
      const float w = __shfl_xor_sync(0xffffffffu, v[j], 1), yo = __shfl_xor_sync(0xffffffffu, y, 1);
      if (in) {
        const float fr = part ? w : v[j], fi = part ? v[j] : w;
        const float yr = part ? yo : y, yi = part ? y : yo;
        float orr = t.sx_one ? fr : sx.re * fr - sx.im * fi;
        float oi = t.sx_one ? fi : sx.re * fi + sx.im * fr;
        if (!t.sy_zero) {
          orr += sy.re * yr - sy.im * yi;
          oi += sy.re * yi + sy.im * yr;
        }
        *cp = part ? oi : orr;
      }
    }
  } else {
    const float sx = scalar_as<float>(t.sx), sy = scalar_as<float>(t.sy);
    const int64_t m = ti->mt * 128 + row;
    if (m >= pm) return;
    const int64_t nv = pn - n0;
    float* cp = static_cast<float*>(p.c) + ti->li * p.c_sl + m * csm + n0 * csn;
    if (t.sy_zero) {
#pragma unroll
      for (int j = 0; j < 16; ++j, cp += csn)
        if (j < nv) *cp = sx * v[j];
    } else {
#pragma unroll
      for (int j = 0; j < 16; ++j, cp += csn)
        if (j < nv) *cp = fmaf(sy, *cp, sx * v[j]);
    }
  }
}

// Drain warps 8-11 (dw = warp - 8): thread = accumulator row 32 dw + lane
// (the TMEM lanes of its warp quarter), all 128 columns.
// Chunks before a tile's last go into the running sums; the last chunk is
// added to them and written out straight from TMEM.
template <int NT, bool CPLX>
__device__ __forceinline__ void gt_drain(const GtArgs& t, float* acc, uint32_t tmem, unsigned char* slots,
                                         uint64_t* sched_full, uint64_t* sched_empty, uint64_t* chunk_done,
                                         uint64_t* drained, volatile int* abort_flag, int dw, int lane) {
  using namespace gt;
  const int row = 32 * dw + lane;
  const uint32_t lane_off = (uint32_t)(32 * dw) << 16;
  uint32_t gc = 0, j = 0;
  for (int64_t tile = blockIdx.x; tile < t.tiles; tile += gridDim.x, ++j) {
    const int ss = j % NSLOT;
    if (!__all_sync(0xffffffffu, mbar_wait(&sched_full[ss], (j / NSLOT) & 1, abort_flag))) return;
    const GtTile* ti = reinterpret_cast<const GtTile*>(slots + ss * SLOT_BYTES);
    const int nch = (gt_stages<CPLX>(ti->p) + CHUNK - 1) / CHUNK;
    const int ngrp = (gt_cols(ti) + 15) >> 4;   // 16-column groups that hold output
    for (int ci = 0; ci < nch; ++ci, ++gc) {
      const int b = gc & 1;
      if (!__all_sync(0xffffffffu, mbar_wait(&chunk_done[b], (gc >> 1) & 1, abort_flag))) return;
      tc_fence_after();
      const bool last = ci + 1 == nch;
#pragma unroll 1
      for (int hh = 0; hh < ngrp; ++hh) {
        uint32_t rm[16], rc[16];
        const uint32_t col = (uint32_t)(16 * hh);
        tmem_ld16_nw(tmem + (uint32_t)(256 * b) + lane_off + col, rm);
        tmem_ld16_nw(tmem + (uint32_t)(256 * b + 128) + lane_off + col, rc);
        tmem_wait_ld();
        float v[16];
#pragma unroll
        for (int jj = 0; jj < 16; ++jj) {
          v[jj] = __uint_as_float(rm[jj]) + __uint_as_float(rc[jj]);
          float* a = acc + (col + jj) * BM + row;
          if (ci > 0) v[jj] += *a;
          if (!last) *a = v[jj];
        }
        if (last) gt_store_cols<CPLX>(t, ti, row, (int)col, v);
      }
      tc_fence_before();
      __syncwarp();
      if (lane == 0) mbar_arrive(&drained[b]);
    }
    if (nch == 0) {   // K = 0: the product is zero
      float v[16];
#pragma unroll
      for (int jj = 0; jj < 16; ++jj) v[jj] = 0.f;
#pragma unroll 1
      for (int hh = 0; hh < ngrp; ++hh) gt_store_cols<CPLX>(t, ti, row, 16 * hh, v);
    }
    __syncwarp();
    if (lane == 0) mbar_arrive(&sched_empty[ss]);
  }
}

template <int NT, bool CPLX>
__global__ void __launch_bounds__(gt::NTHREADS, 1) k_group_tc(const __grid_constant__ GtArgs t) {
  using namespace gt;
  constexpr int STAGES = Cfg<NT>::STAGES, STAGE_BYTES = Cfg<NT>::STAGE_BYTES;
  extern __shared__ __align__(128) unsigned char gt_raw[];
  const uint32_t raw = smem_u32(gt_raw);
  const uint32_t pad = (128u - (raw & 127u)) & 127u;
  unsigned char* smem = gt_raw + pad;
  const uint32_t sbase = raw + pad;
  float* acc = reinterpret_cast<float*>(smem + STAGES * STAGE_BYTES);   // [BN][BM] running sums
  unsigned char* slots = smem + STAGES * STAGE_BYTES + ACC_BYTES;       // scheduler ring
  uint64_t* full = reinterpret_cast<uint64_t*>(slots + NSLOT * SLOT_BYTES);
  uint64_t* empty = full + STAGES;
  uint64_t* chunk_done = empty + STAGES;   // [2]
  uint64_t* drained = chunk_done + 2;      // [2]
  uint64_t* final_bar = drained + 2;
  uint64_t* sched_full = final_bar + 1;    // [NSLOT]
  uint64_t* sched_empty = sched_full + NSLOT;
  uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(sched_empty + NSLOT);
  volatile int* abort_flag = reinterpret_cast<volatile int*>(tmem_slot + 1);
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  if (tid == 0) {
    for (int s = 0; s < STAGES; ++s) {
      mbar_init(&full[s], 8);
      mbar_init(&empty[s], 1);
    }
    for (int b = 0; b < 2; ++b) {
      mbar_init(&chunk_done[b], 1);
      mbar_init(&drained[b], 4);
    }
    mbar_init(final_bar, 1);
    for (int s = 0; s < NSLOT; ++s) {
      mbar_init(&sched_full[s], 1);
      mbar_init(&sched_empty[s], SLOT_USERS);
    }
    *abort_flag = 0;
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  if (warp == 12) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(tmem_slot)),
                 "r"(TMEM_COLS)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = *tmem_slot;

  if (warp < 8) {
    gt_converters<NT, CPLX>(t, sbase, slots, sched_full, sched_empty, full, empty, abort_flag, warp, lane);
  } else if (warp < 12) {
    gt_drain<NT, CPLX>(t, acc, tmem, slots, sched_full, sched_empty, chunk_done, drained, abort_flag, warp - 8,
                       lane);
  } else if (warp == 13) {
    gt_scheduler(t, slots, sched_full, sched_empty, abort_flag, lane);
  } else if (lane == 0) {
    // ---------------- MMA issue ----------------
    uint32_t it = 0, gc = 0, j = 0;
    bool ok = true;
    for (int64_t tile = blockIdx.x; tile < t.tiles && ok; tile += gridDim.x, ++j) {
      const int ss = j % NSLOT;
      if (!mbar_wait(&sched_full[ss], (j / NSLOT) & 1, abort_flag)) break;
      const GtTile* ti = reinterpret_cast<const GtTile*>(slots + ss * SLOT_BYTES);
      const int nkt = gt_stages<CPLX>(ti->p);
      const uint32_t idesc = gt_idesc((uint32_t)((gt_cols(ti) + 15) & ~15));
      mbar_arrive(&sched_empty[ss]);
      for (int kt = 0; kt < nkt; ++kt, ++it) {
        const uint32_t c = gc + kt / CHUNK;
        const int b = c & 1;
        const bool first = kt % CHUNK == 0;
        if (first && c >= 2 && !mbar_wait(&drained[b], ((c >> 1) - 1) & 1, abort_flag)) { ok = false; break; }
        const int s = it % STAGES;
        if (!mbar_wait(&full[s], (it / STAGES) & 1, abort_flag)) { ok = false; break; }
        tc_fence_after();
        const uint32_t sb = sbase + s * STAGE_BYTES;
#pragma unroll
        for (int kk = 0; kk < 2; ++kk) {
          const uint32_t off = kk * 256;
          uint64_t ad[NT], bdsc[NT];
#pragma unroll
          for (int u = 0; u < NT; ++u) {
            ad[u] = umma_desc(sb + u * TILE_BYTES + off);
            bdsc[u] = umma_desc(sb + (NT + u) * TILE_BYTES + off);
          }
          const uint32_t keep = (first && kk == 0) ? 0u : 1u;
          umma_bf16_i(tmem + (uint32_t)(256 * b), ad[0], bdsc[0], idesc, keep);
          bool first_cross = true;
#pragma unroll
          for (int d = 1; d < NT; ++d)
#pragma unroll
            for (int i = 0; i <= d; ++i) {
              umma_bf16_i(tmem + (uint32_t)(256 * b + 128), ad[i], bdsc[d - i], idesc, first_cross ? keep : 1u);
              first_cross = false;
            }
        }
        umma_commit(&empty[s]);
        if (kt % CHUNK == CHUNK - 1 || kt == nkt - 1) umma_commit(&chunk_done[b]);
      }
      gc += (uint32_t)((nkt + CHUNK - 1) / CHUNK);
    }
    umma_commit(final_bar);
    mbar_wait_quiesce(final_bar, 0);
  }
  tc_fence_before();
  __syncthreads();
  if (warp == 12) {
    tc_fence_after();
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(gt::TMEM_COLS) : "memory");
  }
}

namespace {
template <int NT, bool CPLX>
cudaError_t prepare_gt() {
  static std::atomic<unsigned long long> attr{0};
  return set_smem_once(attr, k_group_tc<NT, CPLX>, gt::Cfg<NT>::SMEM_BYTES);
}
template <int NT, bool CPLX>
cudaError_t launch_gt(const GtArgs& t, int grid, cudaStream_t s) {
  const cudaError_t e = prepare_gt<NT, CPLX>();
  if (e != cudaSuccess) return e;
  k_group_tc<NT, CPLX><<<grid, gt::NTHREADS, gt::Cfg<NT>::SMEM_BYTES, s>>>(t);
  return cudaGetLastError();
}
}  // namespace

cudaError_t prepare_group_tc(ome_dtype dt, int nterms) {
  if ((dt != OME_F32 && dt != OME_C32) || (nterms != 2 && nterms != 3)) return cudaErrorNotSupported;
  if (dt == OME_C32) return nterms == 3 ? prepare_gt<3, true>() : prepare_gt<2, true>();
  return nterms == 3 ? prepare_gt<3, false>() : prepare_gt<2, false>();
}

cudaError_t launch_group_tc(ome_dtype dt, int nterms, const GroupProblem* probs, const int32_t* tile_prob, int nprob,
                            int64_t tiles, int grid, const Scalar& sx, const Scalar& sy, int sy_zero, int sx_one,
                            cudaStream_t s) {
  if ((dt != OME_F32 && dt != OME_C32) || (nterms != 2 && nterms != 3) || !tile_prob) return cudaErrorNotSupported;
  if (tiles == 0) return cudaSuccess;
  GtArgs t;
  memset(&t, 0, sizeof(t));
  t.probs = probs;
  t.tile_prob = tile_prob;
  t.nprob = nprob;
  t.tiles = tiles;
  t.sx = sx;
  t.sy = sy;
  t.sy_zero = sy_zero;
  t.sx_one = sx_one;
  cudaError_t e;
  {
    KernelTimer kt(s, "k_group_tc");
    if (dt == OME_C32) e = nterms == 3 ? launch_gt<3, true>(t, grid, s) : launch_gt<2, true>(t, grid, s);
    else e = nterms == 3 ? launch_gt<3, false>(t, grid, s) : launch_gt<2, false>(t, grid, s);
  }
  count_launch();
  return e;
}

// One thread waits on an mbarrier that nothing arrives on, bounded by
// wait_ns; on expiry it records the timeout like any stalled wait and exits.
__global__ void k_selftest_wait(uint64_t wait_ns) {
  __shared__ __align__(8) uint64_t bar;
  if (threadIdx.x != 0) return;
  mbar_init(&bar, 1);
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  const uint64_t t0 = gtimer();
  while (!mbar_try_wait(&bar, 0)) {
    if (gtimer() - t0 > wait_ns) {
      atomicExch(&g_ome_timeout, 1);
      return;
    }
  }
}

cudaError_t launch_selftest_wait(uint64_t wait_ns, cudaStream_t s) {
  if (wait_ns < 1000) wait_ns = 1000;
  if (wait_ns > 1000000000ull) wait_ns = 1000000000ull;
  k_selftest_wait<<<1, 32, 0, s>>>(wait_ns);
  count_launch();
  return cudaGetLastError();
}

int device_status(cudaStream_t s) {
  cudaError_t e = cudaStreamSynchronize(s);
  if (e != cudaSuccess) return -(int)e;
  int flag = 0;
  e = cudaMemcpyFromSymbol(&flag, g_ome_timeout, sizeof(int));
  if (e != cudaSuccess) return -(int)e;
  if (flag) {
    const int zero = 0;
    cudaMemcpyToSymbol(g_ome_timeout, &zero, sizeof(int));
  }
  int bad = 0;
  e = cudaMemcpyFromSymbol(&bad, g_ome_bounds, sizeof(int));
  if (e != cudaSuccess) return -(int)e;
  if (!bad) bad = simt_bounds_flag();
  if (bad) {
    const int zero = 0;
    cudaMemcpyToSymbol(g_ome_bounds, &zero, sizeof(int));
    return 100 + bad;   // a kernel skipped an out-of-view store (its id)
  }
  return flag;
}

}  // namespace ome
