// Batched contractions of uneven shapes in one persistent grouped launch.
//
// Many small binary einsums (e.g. the 8192 MPS transfer contractions of one
// sweep) each reduce, after the same label analysis as the single-call path
// (analyze_binary, src/einsum.jl:139-211), to a strided GEMM
// C[m,n,l] = sx * sum_k A[m,k,l] B[k,n,l] (+ sy*C) with one merged mode per
// group.  Instead of one launch per contraction (what a loop over einsum!
// issues), the problems go into a device-side table and one persistent
// kernel walks the concatenated tile list; the host captures the launch in a
// CUDA graph.  The tile shape is chosen by timing the candidate shapes on the
// batch itself at creation (autotuning), cached in the batch.
#include <string.h>
#include <algorithm>
#include <vector>

#include "dispatch.h"

namespace ome {

template <int BM, int BN, int TM, int TN>
struct GroupCfg {
  static constexpr int NT = (BM / TM) * (BN / TN);
  static constexpr int BK = 8;
};

// One CTA per tile in a grid-stride loop over all problems' tiles.
template <class A, int BM, int BN, int TM, int TN>
__global__ void __launch_bounds__((BM / TM) * (BN / TN)) k_group_gemm(const GroupProblem* __restrict__ probs,
                                                                      int nprob, int64_t total_tiles, Scalar sxs,
                                                                      Scalar sys, int sy_zero, int sx_one) {
  using T = typename A::T;
  constexpr int NT = (BM / TM) * (BN / TN), BK = 8;
  __shared__ T As[BK][BM];
  __shared__ T Bs[BK][BN];
  const T sx = scalar_as<T>(sxs), sy = scalar_as<T>(sys);
  const int tid = threadIdx.x;
  const int tx = tid % (BN / TN), ty = tid / (BN / TN);
  for (int64_t tile = blockIdx.x; tile < total_tiles; tile += gridDim.x) {
    // problem owning this tile (binary search on tile_begin)
    int lo = 0, hi = nprob - 1;
    while (lo < hi) {
      const int mid = (lo + hi + 1) >> 1;
      if (probs[mid].tile_begin <= tile) lo = mid;
      else hi = mid - 1;
    }
    const GroupProblem& p = probs[lo];
    int64_t r = tile - p.tile_begin;
    const int64_t per_l = (int64_t)p.tiles_m * p.tiles_n;
    const int64_t li = r / per_l;
    r -= li * per_l;
    const int64_t m0 = (r % p.tiles_m) * BM, n0 = (r / p.tiles_m) * BN;
    const T* Ap = static_cast<const T*>(p.a) + li * p.a_sl;
    const T* Bp = static_cast<const T*>(p.b) + li * p.b_sl;
    T* Cp = static_cast<T*>(p.c) + li * p.c_sl;
    T acc[TM][TN];
#pragma unroll
    for (int i = 0; i < TM; ++i)
#pragma unroll
      for (int j = 0; j < TN; ++j) acc[i][j] = A::zero();
    for (int64_t k0 = 0; k0 < p.k; k0 += BK) {
      for (int e = tid; e < BM * BK; e += NT) {
        const int mm = e % BM, kk = e / BM;
        const int64_t m = m0 + mm, k = k0 + kk;
        As[kk][mm] = (m < p.m && k < p.k) ? Ap[m * p.a_sm + k * p.a_sk] : A::zero();
      }
      for (int e = tid; e < BN * BK; e += NT) {
        const int kk = e % BK, nn = e / BK;
        const int64_t n = n0 + nn, k = k0 + kk;
        Bs[kk][nn] = (n < p.n && k < p.k) ? Bp[k * p.b_sk + n * p.b_sn] : A::zero();
      }
      __syncthreads();
#pragma unroll
      for (int kk = 0; kk < BK; ++kk) {
        T a[TM], b[TN];
#pragma unroll
        for (int i = 0; i < TM; ++i) a[i] = As[kk][ty + i * (BM / TM)];
#pragma unroll
        for (int j = 0; j < TN; ++j) b[j] = Bs[kk][tx + j * (BN / TN)];
#pragma unroll
        for (int i = 0; i < TM; ++i)
#pragma unroll
          for (int j = 0; j < TN; ++j) acc[i][j] = A::fma(a[i], b[j], acc[i][j]);
      }
      __syncthreads();
    }
#pragma unroll
    for (int i = 0; i < TM; ++i) {
      const int64_t m = m0 + ty + i * (BM / TM);
      if (m >= p.m) continue;
#pragma unroll
      for (int j = 0; j < TN; ++j) {
        const int64_t n = n0 + tx + j * (BN / TN);
        if (n >= p.n) continue;
        T* cp = Cp + m * p.c_sm + n * p.c_sn;
        *cp = epilogue<A>(acc[i][j], cp, sx, sy, sy_zero, sx_one);
      }
    }
  }
}

// candidate tile shapes (BM, BN, TM, TN) of the CUDA-core kernel, then the
// tensor-core kernel (k_group_tc, 128 x 128 tiles of the real-embedded
// output; F32 and C32 only)
constexpr int NCFG = 4, CFG_TC = 3;
static const int kCfg[NCFG][4] = {{32, 32, 2, 2}, {64, 32, 4, 2}, {64, 64, 4, 4}, {128, 128, 0, 0}};

static bool tc_dtype(ome_dtype dt) { return dt == OME_F32 || dt == OME_C32; }

template <class A>
static cudaError_t launch_group_t(int cfg, const GroupProblem* d, int n, int64_t tiles, int grid, const Scalar& sx,
                                  const Scalar& sy, int syz, int sxo, cudaStream_t s) {
  switch (cfg) {
    case 0: k_group_gemm<A, 32, 32, 2, 2><<<grid, 256, 0, s>>>(d, n, tiles, sx, sy, syz, sxo); break;
    case 1: k_group_gemm<A, 64, 32, 4, 2><<<grid, 256, 0, s>>>(d, n, tiles, sx, sy, syz, sxo); break;
    default: k_group_gemm<A, 64, 64, 4, 4><<<grid, 256, 0, s>>>(d, n, tiles, sx, sy, syz, sxo); break;
  }
  count_launch();
  return cudaGetLastError();
}

}  // namespace ome

using namespace ome;

struct ome_batch {
  ome_dtype dt;
  int nprob;
  int cfg;
  int device;
  int num_sms;
  std::vector<GroupProblem> host[NCFG];   // per tile shape (tile_begin differs)
  GroupProblem* dev[NCFG] = {nullptr, nullptr, nullptr, nullptr};
  int64_t tiles[NCFG] = {0, 0, 0, 0};
  float tuned_us[NCFG] = {0, 0, 0, 0};
  std::vector<int32_t> tile_prob_host;     // tensor-core tiles: owning problem of each tile
  int32_t* tile_prob = nullptr;
};

static void free_batch(ome_batch* b) {
  for (int c = 0; c < NCFG; ++c)
    if (b->dev[c]) cudaFree(b->dev[c]);
  if (b->tile_prob) cudaFree(b->tile_prob);
  delete b;
}

namespace {

int find_lab(const HView& v, int32_t l) {
  for (int d = 0; d < v.nd; ++d)
    if (v.lab[d] == l) return d;
  return -1;
}

// Reduce one binary einsum to a single-mode-per-group strided GEMM.
int to_problem(const HView& x1v, const HView& x2v, const HView& yv, GroupProblem& p) {
  HView x1, x2, y;
  int rc = unique_view(x1v, x1);
  if (rc) return rc;
  rc = unique_view(x2v, x2);
  if (rc) return rc;
  rc = unique_view(yv, y);
  if (rc) return rc;
  if (y.nd != yv.nd) return set_err(OME_UNSUPPORTED, "batched contractions: repeated output labels");
  struct G {
    int n = 0;
    int64_t ext = 1, s[3] = {0, 0, 0};
    bool add(int64_t e, int64_t a, int64_t b, int64_t c) {
      if (e == 1) return true;
      if (n == 0) {
        ext = e; s[0] = a; s[1] = b; s[2] = c; n = 1;
        return true;
      }
      // merge when the new mode continues the existing one in every tensor
      if (a == s[0] * ext && b == s[1] * ext && c == s[2] * ext) { ext *= e; return true; }
      if (s[0] == a * e && s[1] == b * e && s[2] == c * e) { s[0] = a; s[1] = b; s[2] = c; ext *= e; return true; }
      return false;
    }
  } gm, gn, gk, gl;
  for (int d = 0; d < y.nd; ++d) {
    const int32_t l = y.lab[d];
    const int k1 = find_lab(x1, l), k2 = find_lab(x2, l);
    bool ok;
    if (k1 >= 0 && k2 >= 0) ok = gl.add(y.ext[d], x1.str[k1], x2.str[k2], y.str[d]);
    else if (k1 >= 0) ok = gm.add(y.ext[d], x1.str[k1], 0, y.str[d]);
    else if (k2 >= 0) ok = gn.add(y.ext[d], 0, x2.str[k2], y.str[d]);
    else return set_err(OME_UNSUPPORTED, "batched contractions: output label %d not in the inputs", l);
    if (!ok) return set_err(OME_UNSUPPORTED, "batched contractions: a label group does not merge into one mode");
  }
  for (int d = 0; d < x1.nd; ++d) {
    const int32_t l = x1.lab[d];
    const int k2 = find_lab(x2, l);
    if (find_lab(y, l) >= 0) continue;
    if (k2 < 0) return set_err(OME_UNSUPPORTED, "batched contractions: label %d summed on one side only", l);
    if (!gk.add(x1.ext[d], x1.str[d], x2.str[k2], 0))
      return set_err(OME_UNSUPPORTED, "batched contractions: inner labels do not merge into one mode");
  }
  for (int d = 0; d < x2.nd; ++d)
    if (find_lab(y, x2.lab[d]) < 0 && find_lab(x1, x2.lab[d]) < 0)
      return set_err(OME_UNSUPPORTED, "batched contractions: label %d summed on one side only", x2.lab[d]);
  p.a = x1.data;
  p.b = x2.data;
  p.c = y.data;
  p.m = gm.ext; p.n = gn.ext; p.k = gk.ext; p.l = gl.ext;
  p.a_sm = gm.s[0]; p.c_sm = gm.s[2];
  p.b_sn = gn.s[1]; p.c_sn = gn.s[2];
  p.a_sk = gk.s[0]; p.b_sk = gk.s[1];
  p.a_sl = gl.s[0]; p.b_sl = gl.s[1]; p.c_sl = gl.s[2];
  return OME_OK;
}

// 1 when an operand's K mode is contiguous and every row it reads starts on
// 16 bytes (per16 elements per 16 bytes).
int32_t kvec_ok(const void* base, int64_t sk, int64_t s_row, int64_t rows, int64_t s_l, int64_t l, int per16) {
  if (sk != 1 || (reinterpret_cast<uintptr_t>(base) & 15u) != 0) return 0;
  if (rows > 1 && s_row % per16 != 0) return 0;
  if (l > 1 && s_l % per16 != 0) return 0;
  return 1;
}

// Loads the kernel of config cfg (and sets its attributes) without launching it.
cudaError_t prepare_cfg(ome_dtype dt, int cfg) {
  if (cfg == CFG_TC) return prepare_group_tc(dt, 3);
  cudaFuncAttributes fa;
  cudaError_t e = cudaSuccess;
  OME_DISPATCH(dt, ALG, {
    switch (cfg) {
      case 0: e = cudaFuncGetAttributes(&fa, k_group_gemm<ALG, 32, 32, 2, 2>); break;
      case 1: e = cudaFuncGetAttributes(&fa, k_group_gemm<ALG, 64, 32, 4, 2>); break;
      default: e = cudaFuncGetAttributes(&fa, k_group_gemm<ALG, 64, 64, 4, 4>); break;
    }
  });
  return e;
}

cudaError_t launch_cfg(ome_batch* b, int cfg, const Scalar& sx, const Scalar& sy, cudaStream_t s) {
  const int64_t tiles = b->tiles[cfg];
  if (tiles == 0) return cudaSuccess;
  const int grid = (int)std::min<int64_t>(tiles, (int64_t)b->num_sms * 8);
  const int syz = scalar_is_zero(b->dt, sy), sxo = scalar_is_one(b->dt, sx);
  if (cfg == CFG_TC)
    return launch_group_tc(b->dt, 3, b->dev[cfg], b->tile_prob, b->nprob, tiles,
                           (int)std::min<int64_t>(tiles, b->num_sms), sx, sy, syz, sxo, s);
  cudaError_t e = cudaErrorInvalidValue;
  OME_DISPATCH(b->dt, ALG, e = launch_group_t<ALG>(cfg, b->dev[cfg], b->nprob, tiles, grid, sx, sy, syz, sxo, s));
  return e;
}

}  // namespace

extern "C" {

int ome_batch_create(ome_ctx* ctx, void* stream, ome_dtype dtype, int32_t count, const ome_tensor* x1s,
                     const ome_tensor* x2s, const ome_tensor* ys, int32_t tile_config, ome_batch** out) {
  if (!ctx || !x1s || !x2s || !ys || !out || count < 1) return set_err(OME_INVALID_ARGUMENT, "bad arguments");
  if ((int)dtype < 0 || (int)dtype > OME_TROP_F64) return set_err(OME_INVALID_ARGUMENT, "unknown dtype");
  *out = nullptr;
  auto b = new ome_batch();
  b->dt = dtype;
  b->nprob = count;
  b->device = ctx->device;
  b->num_sms = ctx->num_sms;
  std::vector<GroupProblem> probs(count);
  for (int i = 0; i < count; ++i) {
    HView x1, x2, y;
    int rc = view_from_tensor(x1s[i], x1, "x1");
    if (!rc) rc = view_from_tensor(x2s[i], x2, "x2");
    if (!rc) rc = view_from_tensor(ys[i], y, "y");
    if (!rc) rc = to_problem(x1, x2, y, probs[i]);
    if (rc) {
      delete b;
      return rc;
    }
    GroupProblem& p = probs[i];
    const int per16 = dtype == OME_C32 ? 2 : 4;
    p.a_kvec = p.b_kvec = 0;
    if (tc_dtype(dtype)) {
      p.a_kvec = kvec_ok(p.a, p.a_sk, p.a_sm, p.m, p.a_sl, p.l, per16);
      p.b_kvec = kvec_ok(p.b, p.b_sk, p.b_sn, p.n, p.b_sl, p.l, per16);
    }
  }
  for (int c = 0; c < NCFG; ++c) {
    b->host[c] = probs;
    int64_t t = 0;
    for (auto& p : b->host[c]) {
      // the tensor-core tiles count rows of the real embedding (two per complex row)
      const int64_t rows = c == CFG_TC && dtype == OME_C32 ? 2 * p.m : p.m;
      p.tiles_m = (int32_t)((rows + kCfg[c][0] - 1) / kCfg[c][0]);
      p.tiles_n = (int32_t)((p.n + kCfg[c][1] - 1) / kCfg[c][1]);
      p.tile_begin = t;
      t += (int64_t)p.tiles_m * p.tiles_n * p.l;
    }
    b->tiles[c] = t;
    cudaError_t e = cudaMalloc(&b->dev[c], sizeof(GroupProblem) * (size_t)count);
    if (e == cudaSuccess)
      e = cudaMemcpyAsync(b->dev[c], b->host[c].data(), sizeof(GroupProblem) * (size_t)count,
                          cudaMemcpyHostToDevice, static_cast<cudaStream_t>(stream));
    if (e == cudaSuccess && c == CFG_TC && tc_dtype(dtype)) {
      b->tile_prob_host.resize((size_t)t);
      for (int i = 0; i < count; ++i) {
        const GroupProblem& p = b->host[c][i];
        const int64_t n = (int64_t)p.tiles_m * p.tiles_n * p.l;
        std::fill_n(b->tile_prob_host.begin() + p.tile_begin, n, (int32_t)i);
      }
      e = cudaMalloc(&b->tile_prob, sizeof(int32_t) * std::max<size_t>((size_t)t, 1));
      if (e == cudaSuccess && t > 0)
        e = cudaMemcpyAsync(b->tile_prob, b->tile_prob_host.data(), sizeof(int32_t) * (size_t)t,
                            cudaMemcpyHostToDevice, static_cast<cudaStream_t>(stream));
    }
    if (e != cudaSuccess) {
      free_batch(b);
      return cuda_err(e, "batch table");
    }
  }
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  if (tile_config == CFG_TC && !tc_dtype(dtype)) {
    free_batch(b);
    return set_err(OME_UNSUPPORTED, "the tensor-core grouped launch takes Float32 and ComplexF32 only");
  }
  if (tile_config >= 0 && tile_config < NCFG) {
    b->cfg = tile_config;
  } else {
    // autotune: time every tile shape on this batch (outputs are overwritten later)
    const Scalar one = scalar_one(dtype), zero = scalar_zero(dtype);
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    float best = 1e30f;
    b->cfg = NCFG - 1;
    for (int c = 0; c < NCFG; ++c) {
      if (c == CFG_TC && !tc_dtype(dtype)) {
        b->tuned_us[c] = -1.f;   // not a candidate for this dtype
        continue;
      }
      launch_cfg(b, c, one, zero, s);  // warm-up
      cudaEventRecord(e0, s);
      for (int r = 0; r < 3; ++r) launch_cfg(b, c, one, zero, s);
      cudaEventRecord(e1, s);
      cudaEventSynchronize(e1);
      float ms = 0.f;
      cudaEventElapsedTime(&ms, e0, e1);
      b->tuned_us[c] = ms * 1e3f / 3.f;
      if (ms < best) {
        best = ms;
        b->cfg = c;
      }
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) {
      free_batch(b);
      return cuda_err(e, "batch autotune");
    }
  }
  *out = b;
  return OME_OK;
}

int ome_batch_run(ome_ctx* ctx, ome_batch* b, void* stream, const void* sx, const void* sy) {
  if (!ctx || !b || !sx || !sy) return set_err(OME_INVALID_ARGUMENT, "NULL argument");
  return cuda_err(launch_cfg(b, b->cfg, scalar_from(b->dt, sx), scalar_from(b->dt, sy),
                             static_cast<cudaStream_t>(stream)),
                  "batched contraction");
}

int ome_batch_info(const ome_batch* b, int32_t* tile_config, float* tuned_us) {
  if (!b) return set_err(OME_INVALID_ARGUMENT, "NULL batch");
  if (tile_config) *tile_config = b->cfg;
  if (tuned_us)
    for (int c = 0; c < NCFG; ++c) tuned_us[c] = b->tuned_us[c];
  return OME_OK;
}

// A CUDA graph of grouped launches, captured on a private stream (the
// caller's stream is never put in capture mode).
struct ome_graph {
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t exec = nullptr;
};

int ome_batch_graph_create(ome_ctx* ctx, void* stream, int32_t count, ome_batch* const* batches,
                           const void* const* sxs, const void* const* sys, ome_graph** out) {
  if (!ctx || !batches || !out || count < 1) return set_err(OME_INVALID_ARGUMENT, "bad arguments");
  *out = nullptr;
  for (int i = 0; i < count; ++i)
    if (!batches[i]) return set_err(OME_INVALID_ARGUMENT, "NULL batch %d", i);
  // the batches' tables were uploaded on their creation streams
  cudaError_t e = cudaStreamSynchronize(static_cast<cudaStream_t>(stream));
  if (e != cudaSuccess) return cuda_err(e, "graph capture");
  for (int i = 0; i < count; ++i) {
    e = prepare_cfg(batches[i]->dt, batches[i]->cfg);
    if (e != cudaSuccess) return cuda_err(e, "graph capture: loading a kernel");
  }
  cudaStream_t cs = nullptr;
  e = cudaStreamCreateWithFlags(&cs, cudaStreamNonBlocking);
  if (e != cudaSuccess) return cuda_err(e, "graph capture stream");
  e = cudaStreamBeginCapture(cs, cudaStreamCaptureModeThreadLocal);
  cudaError_t le = cudaSuccess;
  if (e == cudaSuccess) {
    for (int i = 0; i < count && le == cudaSuccess; ++i) {
      ome_batch* b = batches[i];
      const Scalar sx = sxs && sxs[i] ? scalar_from(b->dt, sxs[i]) : scalar_one(b->dt);
      const Scalar sy = sys && sys[i] ? scalar_from(b->dt, sys[i]) : scalar_zero(b->dt);
      le = launch_cfg(b, b->cfg, sx, sy, cs);
    }
    cudaGraph_t g = nullptr;
    e = cudaStreamEndCapture(cs, &g);   // always ends the capture
    auto gr = new ome_graph();
    gr->graph = g;
    if (e == cudaSuccess && le == cudaSuccess) e = cudaGraphInstantiate(&gr->exec, g, 0);
    if (e != cudaSuccess || le != cudaSuccess) {
      if (gr->exec) cudaGraphExecDestroy(gr->exec);
      if (g) cudaGraphDestroy(g);
      delete gr;
      cudaStreamDestroy(cs);
      return cuda_err(le != cudaSuccess ? le : e, "graph capture");
    }
    *out = gr;
  }
  cudaStreamDestroy(cs);
  return e == cudaSuccess ? OME_OK : cuda_err(e, "graph capture");
}

int ome_graph_launch(ome_graph* g, void* stream) {
  if (!g || !g->exec) return set_err(OME_INVALID_ARGUMENT, "NULL graph");
  return cuda_err(cudaGraphLaunch(g->exec, static_cast<cudaStream_t>(stream)), "graph launch");
}

int ome_graph_destroy(ome_graph* g) {
  if (!g) return OME_OK;
  if (g->exec) cudaGraphExecDestroy(g->exec);
  if (g->graph) cudaGraphDestroy(g->graph);
  delete g;
  return OME_OK;
}

int ome_batch_destroy(ome_batch* b) {
  if (!b) return OME_OK;
  free_batch(b);
  return OME_OK;
}

}  // extern "C"
