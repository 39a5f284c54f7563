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
};

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

// candidate tile shapes (BM, BN, TM, TN)
constexpr int NCFG = 3;
static const int kCfg[NCFG][4] = {{32, 32, 2, 2}, {64, 32, 4, 2}, {64, 64, 4, 4}};

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
  GroupProblem* dev[NCFG] = {nullptr, nullptr, nullptr};
  int64_t tiles[NCFG] = {0, 0, 0};
  float tuned_us[NCFG] = {0, 0, 0};
};

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

cudaError_t launch_cfg(ome_batch* b, int cfg, const Scalar& sx, const Scalar& sy, cudaStream_t s) {
  const int64_t tiles = b->tiles[cfg];
  if (tiles == 0) return cudaSuccess;
  const int grid = (int)std::min<int64_t>(tiles, (int64_t)b->num_sms * 8);
  const int syz = scalar_is_zero(b->dt, sy), sxo = scalar_is_one(b->dt, sx);
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
  }
  for (int c = 0; c < NCFG; ++c) {
    b->host[c] = probs;
    int64_t t = 0;
    for (auto& p : b->host[c]) {
      p.tiles_m = (int32_t)((p.m + kCfg[c][0] - 1) / kCfg[c][0]);
      p.tiles_n = (int32_t)((p.n + kCfg[c][1] - 1) / kCfg[c][1]);
      p.tile_begin = t;
      t += (int64_t)p.tiles_m * p.tiles_n * p.l;
    }
    b->tiles[c] = t;
    cudaError_t e = cudaMalloc(&b->dev[c], sizeof(GroupProblem) * (size_t)count);
    if (e == cudaSuccess)
      e = cudaMemcpyAsync(b->dev[c], b->host[c].data(), sizeof(GroupProblem) * (size_t)count,
                          cudaMemcpyHostToDevice, static_cast<cudaStream_t>(stream));
    if (e != cudaSuccess) {
      for (int q = 0; q <= c; ++q)
        if (b->dev[q]) cudaFree(b->dev[q]);
      delete b;
      return cuda_err(e, "batch table");
    }
  }
  cudaStream_t s = static_cast<cudaStream_t>(stream);
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
      for (int q = 0; q < NCFG; ++q) cudaFree(b->dev[q]);
      delete b;
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

int ome_batch_destroy(ome_batch* b) {
  if (!b) return OME_OK;
  for (int c = 0; c < NCFG; ++c)
    if (b->dev[c]) cudaFree(b->dev[c]);
  delete b;
  return OME_OK;
}

}  // extern "C"
