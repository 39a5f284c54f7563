// C ABI entry points and the single-contraction dispatcher of libomeb200.
//
// einsum! semantics follow OMEinsum.jl: unary (src/einsum.jl:84-101 with the
// rules of src/unaryrules.jl), binary (src/einsum.jl:104-211 +
// src/binaryrules.jl) and n-ary (src/einsum.jl:47-50 -> loop_einsum!).  The
// B200 design differs from the reference's in how, not what:
//  * repeated input labels (Diag) become diagonal views (summed strides) --
//    no compactify! copy;
//  * labels only on the output (Repeat) become stride-0 input modes;
//  * repeated output labels (Duplicate) become a diagonal view of y after a
//    one-pass y <- sy*y (or zero) over the off-diagonal entries;
//  * binary contractions run as a strided GEMM whose mode strides absorb
//    simplifyto's permutations (src/einsum.jl:127-134) and the output
//    permutation, so no permuted temporary is written to HBM; dangling
//    labels (summed on one side only) are pre-reduced as the reference does.
#include <stdarg.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <algorithm>
#include <string>
#include <vector>

#include "dispatch.h"

namespace ome {

static thread_local std::string g_err;

int set_err(int code, const char* fmt, ...) {
  char buf[1024];
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(buf, sizeof(buf), fmt, ap);
  va_end(ap);
  g_err = buf;
  return code;
}

int cuda_err(cudaError_t e, const char* what) {
  if (e == cudaSuccess) return OME_OK;
  if (e == cudaErrorMemoryAllocation) return set_err(OME_OUT_OF_MEMORY, "%s: %s", what, cudaGetErrorString(e));
  return set_err(OME_CUDA_ERROR, "%s: %s", what, cudaGetErrorString(e));
}

#define OME_CK(call)                                   \
  do {                                                 \
    int rc_ = (call);                                  \
    if (rc_ != OME_OK) return rc_;                     \
  } while (0)
#define OME_CUDA(call, what)                           \
  do {                                                 \
    cudaError_t e_ = (call);                           \
    if (e_ != cudaSuccess) return cuda_err(e_, what);  \
  } while (0)

// ----------------------------------------------------------------------------
// dispatch trace: OME_TRACE=1 in the environment logs every dispatch decision
// with its device time (events + synchronize, so only for diagnosis)
// ----------------------------------------------------------------------------

static int trace_on() {
  static int v = -1;
  if (v < 0) {
    const char* e = getenv("OME_TRACE");
    v = (e && e[0] && e[0] != '0') ? 1 : 0;
  }
  return v;
}
static thread_local char g_trace[256];
static void trace_path(const char* fmt, ...) {
  if (!trace_on()) return;
  va_list ap;
  va_start(ap, fmt);
  // a "  -> route" tag is appended to the shape already recorded
  const size_t at = (fmt[0] == ' ' && fmt[1] == ' ' && fmt[2] == '-') ? strlen(g_trace) : 0;
  vsnprintf(g_trace + at, sizeof(g_trace) - at, fmt, ap);
  va_end(ap);
}

void* ws_alloc(ome_ctx* c, size_t bytes) {
  size_t off = (c->ws_top + 255) & ~(size_t)255;
  if (off + bytes > c->ws_bytes) return nullptr;
  c->ws_top = off + bytes;
  return c->ws + off;
}

// ----------------------------------------------------------------------------
// scalars
// ----------------------------------------------------------------------------

Scalar scalar_from(ome_dtype dt, const void* p) {
  Scalar s;
  memset(&s, 0, sizeof(s));
  memcpy(s.b, p, dtype_size(dt));
  return s;
}
bool scalar_is_zero(ome_dtype dt, const Scalar& v) {
  bool r = false;
  OME_DISPATCH(dt, ALG, r = ALG::is_zero(scalar_as<typename ALG::T>(v)));
  return r;
}
bool scalar_is_one(ome_dtype dt, const Scalar& v) {
  bool r = false;
  OME_DISPATCH(dt, ALG, r = ALG::is_one(scalar_as<typename ALG::T>(v)));
  return r;
}
Scalar scalar_one(ome_dtype dt) {
  Scalar s;
  memset(&s, 0, sizeof(s));
  OME_DISPATCH(dt, ALG, { typename ALG::T v = ALG::one(); memcpy(s.b, &v, sizeof(v)); });
  return s;
}
Scalar scalar_zero(ome_dtype dt) {
  Scalar s;
  memset(&s, 0, sizeof(s));
  OME_DISPATCH(dt, ALG, { typename ALG::T v = ALG::zero(); memcpy(s.b, &v, sizeof(v)); });
  return s;
}

// ----------------------------------------------------------------------------
// views
// ----------------------------------------------------------------------------

int view_from_tensor(const ome_tensor& t, HView& v, const char* what) {
  if (t.ndim < 0 || t.ndim > MAXD)
    return set_err(OME_INVALID_ARGUMENT, "%s: rank %d outside [0, %d]", what, t.ndim, MAXD);
  if (t.ndim > 0 && (!t.dims || !t.labels))
    return set_err(OME_INVALID_ARGUMENT, "%s: dims and labels are required", what);
  v.data = static_cast<char*>(t.data);
  v.nd = t.ndim;
  int64_t s = 1;
  for (int d = 0; d < t.ndim; ++d) {
    if (t.dims[d] < 0) return set_err(OME_INVALID_ARGUMENT, "%s: negative extent", what);
    v.ext[d] = t.dims[d];
    v.str[d] = t.strides ? t.strides[d] : s;
    v.lab[d] = t.labels[d];
    s *= t.dims[d];
  }
  return OME_OK;
}

int unique_view(const HView& v, HView& u) {
  u.data = v.data;
  u.nd = 0;
  for (int d = 0; d < v.nd; ++d) {
    int k = 0;
    for (; k < u.nd; ++k)
      if (u.lab[k] == v.lab[d]) break;
    if (k < u.nd) {
      if (u.ext[k] != v.ext[d])
        return set_err(OME_DIMENSION_MISMATCH, "label %d = %lld or %lld)?", v.lab[d],
                       (long long)u.ext[k], (long long)v.ext[d]);
      u.str[k] += v.str[d];
    } else {
      u.lab[u.nd] = v.lab[d];
      u.ext[u.nd] = v.ext[d];
      u.str[u.nd] = v.str[d];
      u.nd++;
    }
  }
  return OME_OK;
}

static int find_lab(const HView& v, int32_t l) {
  for (int d = 0; d < v.nd; ++d)
    if (v.lab[d] == l) return d;
  return -1;
}

static int64_t numel(const HView& v) {
  int64_t n = 1;
  for (int d = 0; d < v.nd; ++d) n *= v.ext[d];
  return n;
}

// ----------------------------------------------------------------------------
// mode tables: one row per label, one stride column per tensor
// ----------------------------------------------------------------------------

struct Modes {
  int n = 0, nt = 0;
  int64_t ext[2 * MAXD];
  int64_t str[MAXIN + 1][2 * MAXD];

  void add(int64_t e, const int64_t* s) {
    ext[n] = e;
    for (int t = 0; t < nt; ++t) str[t][n] = s[t];
    n++;
  }
  int64_t total() const {
    int64_t p = 1;
    for (int i = 0; i < n; ++i) p *= ext[i];
    return p;
  }
  // Drop unit modes; stable sort by |stride of tensor key| (zero strides last);
  // merge neighbours whose strides are consistent in every tensor.
  void normalize(int key) {
    int w = 0;
    for (int i = 0; i < n; ++i) {
      if (ext[i] == 1) continue;
      ext[w] = ext[i];
      for (int t = 0; t < nt; ++t) str[t][w] = str[t][i];
      w++;
    }
    n = w;
    std::vector<int> idx(n);
    for (int i = 0; i < n; ++i) idx[i] = i;
    auto k = [&](int i) -> uint64_t {
      int64_t s = str[key][i];
      if (s == 0) return ~0ull;
      return (uint64_t)(s < 0 ? -s : s);
    };
    std::stable_sort(idx.begin(), idx.end(), [&](int a, int b) { return k(a) < k(b); });
    int64_t e2[2 * MAXD], s2[MAXIN + 1][2 * MAXD];
    for (int i = 0; i < n; ++i) {
      e2[i] = ext[idx[i]];
      for (int t = 0; t < nt; ++t) s2[t][i] = str[t][idx[i]];
    }
    int m = 0;
    for (int i = 0; i < n; ++i) {
      if (m > 0) {
        bool ok = true;
        for (int t = 0; t < nt && ok; ++t) ok = s2[t][i] == str[t][m - 1] * ext[m - 1];
        if (ok) {
          ext[m - 1] *= e2[i];
          continue;
        }
      }
      ext[m] = e2[i];
      for (int t = 0; t < nt; ++t) str[t][m] = s2[t][i];
      m++;
    }
    n = m;
  }
};

// ----------------------------------------------------------------------------
// generic index kernel
// ----------------------------------------------------------------------------

static int run_loop(ome_ctx* ctx, cudaStream_t s, ome_dtype dt, int nin, const HView* xu,
                    const HView& yu, const Scalar& sx, const Scalar& sy, bool sy_zero) {
  if (nin < 1 || nin > MAXIN)
    return set_err(OME_UNSUPPORTED, "the index kernel takes 1..%d inputs, got %d", MAXIN, nin);
  Modes outer, inner;
  outer.nt = inner.nt = nin + 1;
  int64_t st[MAXIN + 1];
  for (int d = 0; d < yu.nd; ++d) {
    st[0] = yu.str[d];
    for (int i = 0; i < nin; ++i) {
      int k = find_lab(xu[i], yu.lab[d]);
      st[1 + i] = k >= 0 ? xu[i].str[k] : 0;
    }
    outer.add(yu.ext[d], st);
  }
  std::vector<int32_t> seen;
  for (int i = 0; i < nin; ++i)
    for (int d = 0; d < xu[i].nd; ++d) {
      const int32_t l = xu[i].lab[d];
      if (find_lab(yu, l) >= 0 || std::find(seen.begin(), seen.end(), l) != seen.end()) continue;
      if ((int)seen.size() >= 2 * MAXD)
        return set_err(OME_UNSUPPORTED, "index kernel: more than %d summed labels", 2 * MAXD);
      seen.push_back(l);
      st[0] = 0;
      for (int j = 0; j < nin; ++j) {
        int k = find_lab(xu[j], l);
        st[1 + j] = k >= 0 ? xu[j].str[k] : 0;
      }
      inner.add(xu[i].ext[d], st);
    }
  const int64_t n_out = outer.total(), n_in = inner.total();
  if (n_out == 0) return OME_OK;
  outer.normalize(0);
  inner.normalize(1);
  // one contiguous summed run per output and too few outputs to fill the
  // GPU (`ijk->k` once i and j merge): view the run as rows (a divisor of its
  // length in [512, 4096], a multiple of 16 if there is one) so that the
  // row-split reduction spreads each output over many blocks
  // inputs whose first summed mode has stride 0 or 1, at least one of them 1:
  // the contiguous reductions below read rows of that mode
  bool rowwise = nin <= 3 && inner.n >= 1;
  bool any_unit = false;
  for (int k = 0; k < nin && rowwise; ++k) {
    rowwise = inner.str[1 + k][0] == 0 || inner.str[1 + k][0] == 1;
    any_unit = any_unit || inner.str[1 + k][0] == 1;
  }
  rowwise = rowwise && any_unit;
  if (rowwise && inner.n == 1 && inner.ext[0] >= 16384 && n_out < (int64_t)ctx->num_sms * 16 &&
      outer.n + 2 <= MAXM) {
    const int64_t E = inner.ext[0];
    int64_t row = 0;
    for (int pass = 0; pass < 2 && !row; ++pass)
      for (int64_t r = 4096; r >= 512; --r)
        if (E % r == 0 && (pass == 1 || r % 16 == 0)) {
          row = r;
          break;
        }
    if (row) {
      inner.n = 2;
      inner.ext[0] = row;
      inner.ext[1] = E / row;
      for (int t = 0; t < inner.nt; ++t) inner.str[t][1] = inner.str[t][0] * row;
    }
  }
  if (outer.n + inner.n > MAXM)
    return set_err(OME_UNSUPPORTED, "index kernel: %d modes after merging exceed %d", outer.n + inner.n, MAXM);

  LoopArgs a;
  memset(&a, 0, sizeof(a));
  for (int i = 0; i < nin; ++i) a.x[i] = xu[i].data;
  a.y = yu.data;
  a.nin = nin;
  a.nout = outer.n;
  a.ninner = inner.n;
  a.n_out = n_out;
  a.n_in = n_in;
  for (int m = 0; m < outer.n; ++m) {
    a.ext[m] = outer.ext[m];
    for (int t = 0; t <= nin; ++t) a.str[t][m] = outer.str[t][m];
  }
  for (int m = 0; m < inner.n; ++m) {
    a.ext[outer.n + m] = inner.ext[m];
    for (int t = 0; t <= nin; ++t) a.str[t][outer.n + m] = inner.str[t][m];
  }
  a.sx = sx;
  a.sy = sy;
  a.sy_zero = sy_zero;
  a.sx_one = scalar_is_one(dt, sx);
  a.nsplit = 1;

  const int sms = ctx->num_sms;
  // no summed labels (Hadamard and outer products, broadcast products): rows
  // of y's fastest mode
  if (inner.n == 0 && outer.n >= 1) {
    trace_path("map_rows nin=%d n_out=%lld modes=%d", nin, (long long)n_out, outer.n);
    return cuda_err(launch_map_rows(dt, a, sms, s), "map kernel");
  }
  // one input whose first summed mode is contiguous: row-vectorised reduction
  if (rowwise && (inner.n == 1 || inner.n == 2) && inner.ext[0] >= 32) {
    const int64_t R = inner.n == 2 ? inner.ext[1] : 1;
    const size_t es = dtype_size(dt);
    const int64_t V = (int64_t)(16 / es);
    bool vec = inner.ext[0] % V == 0;
    for (int k = 0; k < nin && vec; ++k) {
      if (inner.str[1 + k][0] == 0) continue;   // read once per row
      vec = ((uintptr_t)xu[k].data % 16) == 0;
      for (int m = 0; m < outer.n && vec; ++m) vec = (outer.str[1 + k][m] * (int64_t)es) % 16 == 0;
      if (inner.n == 2) vec = vec && (inner.str[1 + k][1] * (int64_t)es) % 16 == 0;
    }
    // many outputs: a warp per output
    if (n_out >= (int64_t)sms * 64) {
      const int grid = (int)std::min<int64_t>((n_out + 7) / 8, (int64_t)sms * 128);
      trace_path("reduce_rows n_out=%lld n_in=%lld modes=%d+%d vec=%d", (long long)n_out, (long long)n_in,
                 outer.n, inner.n, (int)vec);
      return cuda_err(launch_reduce_rows(dt, a, vec, grid, s), "reduce kernel");
    }
    int64_t nsplit = 1;
    const int64_t target = (int64_t)sms * 16;
    if (n_out < target) nsplit = std::min<int64_t>((target + n_out - 1) / n_out, R);
    int64_t rchunk = (R + nsplit - 1) / nsplit;
    nsplit = (R + rchunk - 1) / rchunk;
    if (nsplit > 1) {
      a.partial = ws_alloc(ctx, (size_t)(n_out * nsplit) * es);
      if (!a.partial) {
        nsplit = 1;
        rchunk = R;
      }
    }
    a.nsplit = (int)nsplit;
    const int grid = (int)std::min<int64_t>(n_out * nsplit, (int64_t)sms * 32);
    trace_path("reduce_contig n_out=%lld n_in=%lld modes=%d+%d nsplit=%lld vec=%d", (long long)n_out,
               (long long)n_in, outer.n, inner.n, (long long)nsplit, (int)vec);
    OME_CK(cuda_err(launch_reduce_contig(dt, a, vec, rchunk, grid, s), "reduce kernel"));
    if (nsplit > 1) OME_CK(cuda_err(launch_loop_finish(dt, a, s), "reduce finish"));
    return OME_OK;
  }
  // summed modes strided while y's fastest mode is contiguous in the first
  // input (GEMV `ij,j->i`, `ijk->ik`): a thread per output along that mode,
  // coalesced across the warp, the summed space split over enough ranges to
  // give every SM 8 blocks
  if (inner.n >= 1 && outer.n >= 1 && outer.str[1][0] == 1 && inner.str[1][0] != 1 && n_in > 16 && n_out >= 256) {
    // 16-byte accesses along the outputs: y contiguous there, every input
    // contiguous or constant there, all offsets the threads reach aligned
    const size_t es = dtype_size(dt);
    const int64_t V = es <= 8 && 16 % es == 0 ? (int64_t)(16 / es) : 1;
    bool vec = V > 1 && outer.str[0][0] == 1 && outer.ext[0] % V == 0 && ((uintptr_t)yu.data % 16) == 0;
    for (int m = 1; m < outer.n && vec; ++m) vec = (outer.str[0][m] * (int64_t)es) % 16 == 0;
    for (int k = 0; k < nin && vec; ++k) {
      const int64_t s0 = outer.str[1 + k][0];
      if (s0 == 0) continue;
      vec = s0 == 1 && ((uintptr_t)xu[k].data % 16) == 0;
      for (int m = 1; m < outer.n && vec; ++m) vec = (outer.str[1 + k][m] * (int64_t)es) % 16 == 0;
      for (int m = 0; m < inner.n && vec; ++m) vec = (inner.str[1 + k][m] * (int64_t)es) % 16 == 0;
    }
    const int64_t bx = (n_out / (vec ? V : 1) + 255) / 256;
    const int64_t target = (int64_t)sms * 8;
    int64_t nsplit = 1;
    if (bx < target) nsplit = std::min<int64_t>((target + bx - 1) / bx, std::max<int64_t>(1, n_in / 64));
    int64_t chunk = (n_in + nsplit - 1) / nsplit;
    nsplit = (n_in + chunk - 1) / chunk;
    if (nsplit > 1) {
      a.partial = ws_alloc(ctx, (size_t)(n_out * nsplit) * es);
      if (!a.partial) {
        nsplit = 1;
        chunk = n_in;
      }
    }
    a.nsplit = (int)nsplit;
    const dim3 grid((unsigned)std::min<int64_t>(bx, (int64_t)sms * 32), (unsigned)nsplit);
    trace_path("loop_cols nin=%d n_out=%lld n_in=%lld modes=%d+%d nsplit=%lld vec=%d", nin, (long long)n_out,
               (long long)n_in, outer.n, inner.n, (long long)nsplit, (int)vec);
    OME_CK(cuda_err(launch_loop_cols(dt, a, chunk, grid, vec, s), "index kernel"));
    if (nsplit > 1) OME_CK(cuda_err(launch_loop_finish(dt, a, s), "index kernel finish"));
    return OME_OK;
  }
  const bool thread_mode = n_in <= 16 || n_out >= (int64_t)sms * 512;
  if (thread_mode) {
    trace_path("loop_thread nin=%d n_out=%lld n_in=%lld modes=%d+%d", nin, (long long)n_out, (long long)n_in,
               outer.n, inner.n);
    const int64_t nb = (n_out + 255) / 256;
    const int grid = (int)std::min<int64_t>(nb, (int64_t)sms * 16);
    return cuda_err(launch_loop(dt, a, LOOP_THREAD, grid, 256, s), "index kernel");
  }
  const int block = 256;
  int64_t nsplit = 1;
  const int64_t target = (int64_t)sms * 8;
  if (n_out < target) {
    nsplit = (target + n_out - 1) / n_out;
    nsplit = std::min<int64_t>(nsplit, std::max<int64_t>(1, n_in / (block * 2)));
  }
  if (nsplit > 1) {
    a.partial = ws_alloc(ctx, (size_t)(n_out * nsplit) * dtype_size(dt));
    if (!a.partial) nsplit = 1;
  }
  a.nsplit = (int)nsplit;
  // step = block * nsplit in the inner mixed radix (last digit unbounded)
  int64_t step = (int64_t)block * nsplit;
  for (int m = 0; m < inner.n; ++m) {
    if (m == inner.n - 1) {
      a.stepdig[m] = (int32_t)std::min<int64_t>(step, 0x7fffffff);
    } else {
      a.stepdig[m] = (int32_t)(step % inner.ext[m]);
      step /= inner.ext[m];
    }
  }
  const int64_t nblocks = n_out * nsplit;
  const int grid = (int)std::min<int64_t>(nblocks, (int64_t)sms * 32);
  trace_path("loop_block nin=%d n_out=%lld n_in=%lld modes=%d+%d nsplit=%lld", nin, (long long)n_out,
             (long long)n_in, outer.n, inner.n, (long long)nsplit);
  OME_CK(cuda_err(launch_loop(dt, a, LOOP_BLOCK, grid, block, s), "index kernel"));
  if (nsplit > 1) OME_CK(cuda_err(launch_loop_finish(dt, a, s), "index kernel finish"));
  return OME_OK;
}

// ----------------------------------------------------------------------------
// unary: permute / broadcast copy, or reduction
// ----------------------------------------------------------------------------

static int run_unary(ome_ctx* ctx, cudaStream_t s, ome_dtype dt, const HView& xu, const HView& yu,
                     const Scalar& sx, const Scalar& sy, bool sy_zero) {
  bool reduced = false;
  for (int d = 0; d < xu.nd; ++d)
    if (find_lab(yu, xu.lab[d]) < 0 && xu.ext[d] != 1) reduced = true;
  if (reduced || xu.nd == 0 && false) return run_loop(ctx, s, dt, 1, &xu, yu, sx, sy, sy_zero);
  // labels of x not in y have extent 1 here (or 0, then y gets sy*y + sx*zero)
  for (int d = 0; d < xu.nd; ++d)
    if (find_lab(yu, xu.lab[d]) < 0 && xu.ext[d] == 0) return run_loop(ctx, s, dt, 1, &xu, yu, sx, sy, sy_zero);
  Modes md;
  md.nt = 2;  // 0: y, 1: x
  int64_t st[2];
  for (int d = 0; d < yu.nd; ++d) {
    int k = find_lab(xu, yu.lab[d]);
    st[0] = yu.str[d];
    st[1] = k >= 0 ? xu.str[k] : 0;
    md.add(yu.ext[d], st);
  }
  const int64_t n = md.total();
  if (n == 0) return OME_OK;
  md.normalize(0);
  if (md.n > MAXM) return run_loop(ctx, s, dt, 1, &xu, yu, sx, sy, sy_zero);
  PermArgs a;
  memset(&a, 0, sizeof(a));
  a.x = xu.data;
  a.y = yu.data;
  a.nd = md.n;
  a.n = n;
  for (int m = 0; m < md.n; ++m) {
    a.ext[m] = md.ext[m];
    a.ys[m] = md.str[0][m];
    a.xs[m] = md.str[1][m];
  }
  if (md.n == 0) {  // scalar
    a.nd = 1;
    a.ext[0] = 1;
    a.xs[0] = a.ys[0] = 1;
  }
  a.sx = sx;
  a.sy = sy;
  a.sy_zero = sy_zero;
  a.sx_one = scalar_is_one(dt, sx);
  a.tmode = -1;
  // x's contiguous mode, if it is not y's fastest mode -> tiled transpose
  int p = -1;
  for (int m = 0; m < a.nd; ++m)
    if (a.xs[m] == 1 || a.xs[m] == -1) { p = m; break; }
  if (p > 0 && (a.xs[0] > 1 || a.xs[0] < -1) && a.ext[0] >= 4 && a.ext[p] >= 4) a.tmode = p;
  trace_path("permute n=%lld modes=%d tmode=%d", (long long)n, a.nd, a.tmode);
  return cuda_err(launch_perm(dt, a, ctx->num_sms, s), "permute kernel");
}

// ----------------------------------------------------------------------------
// binary: strided GEMM or index kernel
// ----------------------------------------------------------------------------

static int reduce_dangling(ome_ctx* ctx, cudaStream_t s, ome_dtype dt, HView& xu, const HView& other,
                           const HView& yu) {
  HView r;
  r.nd = 0;
  bool any = false;
  int64_t n = 1;
  for (int d = 0; d < xu.nd; ++d) {
    if (find_lab(other, xu.lab[d]) < 0 && find_lab(yu, xu.lab[d]) < 0) {
      any = true;
      continue;
    }
    r.lab[r.nd] = xu.lab[d];
    r.ext[r.nd] = xu.ext[d];
    r.str[r.nd] = n;
    n *= xu.ext[d];
    r.nd++;
  }
  if (!any) return OME_OK;
  r.data = static_cast<char*>(ws_alloc(ctx, (size_t)std::max<int64_t>(n, 1) * dtype_size(dt)));
  if (!r.data)
    return set_err(OME_OUT_OF_MEMORY, "workspace too small for a dangling-label reduction (%lld elements)",
                   (long long)n);
  OME_CK(run_loop(ctx, s, dt, 1, &xu, r, scalar_one(dt), scalar_zero(dt), true));
  xu = r;
  return OME_OK;
}

// Tensor-core kernel for an FP32 GEMM: 2 = the 2-SM kernel fed by tensor
// maps over the FP32 operands (k_gemm_tma2), 1 = pre-split operands +
// bulk-copy persistent kernel (k_gemm_packed), 0 = in-kernel converters
// (k_gemm_bf16x3).  The environment variable OME_GEMM=tma|packed|fused
// overrides the shape rule (a kernel whose preconditions fail falls through
// to the next).
static int gemm_kernel_choice(const GemmArgs& g) {
  static const int forced = [] {
    const char* e = getenv("OME_GEMM");
    if (!e) return -1;
    if (!strcmp(e, "tma")) return 2;
    if (!strcmp(e, "packed")) return 1;
    if (!strcmp(e, "fused")) return 0;
    return -1;
  }();
  if (forced >= 0) return forced;
  const double flops = 2.0 * (double)g.M * (double)g.N * (double)g.K * (double)g.L;
  // 256 x 256 cluster tiles: worth it once a few waves of k-steps are there
  if (gemm_tma2_applies(g) && g.M >= 128 && g.N >= 128 && g.K >= 256 && flops >= 2e8) return 2;
  // pre-splitting pays for itself on large GEMMs with a long K only (two
  // extra HBM passes over the operands; with a short K the output dominates)
  return g.M >= 256 && g.N >= 256 && g.K >= 512 && flops >= 1e9 ? 1 : 0;
}

// Scratch of `need` bytes for a packed GEMM whose operands do not fit the
// workspace: the context's overflow buffer, grown (64 MiB granules) when it
// is smaller, but never during stream capture and never past a quarter of
// the free device memory.  Growing waits for the device (the old buffer may
// still be read by earlier launches).  nullptr: use the in-kernel-converter
// GEMM instead.
static void* overflow_scratch(ome_ctx* ctx, size_t need, cudaStream_t s) {
  if (need <= ctx->ovf_bytes) return ctx->ovf;
  cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
  if (cudaStreamIsCapturing(s, &cs) != cudaSuccess || cs != cudaStreamCaptureStatusNone) {
    cudaGetLastError();
    return nullptr;
  }
  size_t fr = 0, tot = 0;
  if (cudaMemGetInfo(&fr, &tot) != cudaSuccess) {
    cudaGetLastError();
    return nullptr;
  }
  const size_t gran = (size_t)64 << 20;
  const size_t want = (need + gran - 1) / gran * gran;
  if (want > (fr + ctx->ovf_bytes) / 4) return nullptr;
  if (ctx->ovf) {
    if (cudaDeviceSynchronize() != cudaSuccess) return nullptr;
    cudaFree(ctx->ovf);
    ctx->ovf = nullptr;
    ctx->ovf_bytes = 0;
  }
  if (cudaMalloc(&ctx->ovf, want) != cudaSuccess) {
    cudaGetLastError();
    ctx->ovf = nullptr;
    return nullptr;
  }
  ctx->ovf_bytes = want;
  return ctx->ovf;
}

static int run_binary(ome_ctx* ctx, cudaStream_t s, ome_dtype dt, HView x1, HView x2, const HView& yu,
                      const Scalar& sx, const Scalar& sy, bool sy_zero, int prec) {
  OME_CK(reduce_dangling(ctx, s, dt, x1, x2, yu));
  OME_CK(reduce_dangling(ctx, s, dt, x2, x1, yu));
  // group tables: M (y, A), N (y, B), K (A, B), L (y, A, B)
  Modes gm, gn, gk, gl;
  gm.nt = 2; gn.nt = 2; gk.nt = 2; gl.nt = 3;
  int64_t st[3];
  for (int d = 0; d < yu.nd; ++d) {
    const int32_t l = yu.lab[d];
    const int k1 = find_lab(x1, l), k2 = find_lab(x2, l);
    if (k1 >= 0 && k2 >= 0) {
      st[0] = x1.str[k1]; st[1] = x2.str[k2]; st[2] = yu.str[d];
      gl.add(yu.ext[d], st);
    } else if (k2 >= 0) {
      st[0] = x2.str[k2]; st[1] = yu.str[d];
      gn.add(yu.ext[d], st);
    } else {  // in x1 only, or broadcast (stride 0 in A)
      st[0] = k1 >= 0 ? x1.str[k1] : 0; st[1] = yu.str[d];
      gm.add(yu.ext[d], st);
    }
  }
  for (int d = 0; d < x1.nd; ++d) {
    const int32_t l = x1.lab[d];
    const int k2 = find_lab(x2, l);
    if (k2 >= 0 && find_lab(yu, l) < 0) {
      st[0] = x1.str[d]; st[1] = x2.str[k2];
      gk.add(x1.ext[d], st);
    }
  }
  const int64_t M = gm.total(), N = gn.total(), K = gk.total(), L = gl.total();
  if (M * N * L == 0) return OME_OK;
  const bool gemm_shape = M >= 16 && N >= 16 && K >= 8;
  if (gemm_shape) {
    gm.normalize(0);
    gn.normalize(0);
    // K order: A's contiguous mode first if A is K-contiguous, else B's
    bool a_kfast = false;
    for (int i = 0; i < gk.n; ++i)
      if (gk.str[0][i] == 1) a_kfast = true;
    gk.normalize(a_kfast ? 0 : 1);
    gl.normalize(2);
  }
  if (gemm_shape && gm.n <= MAXG && gn.n <= MAXG && gk.n <= MAXG && gl.n <= MAXG) {
    GemmArgs g;
    memset(&g, 0, sizeof(g));
    g.A = x1.data;
    g.B = x2.data;
    g.C = yu.data;
    g.M = M; g.N = N; g.K = K; g.L = L;
    g.nm = gm.n; g.nn = gn.n; g.nk = gk.n; g.nl = gl.n;
    for (int i = 0; i < gm.n; ++i) { g.m_ext[i] = gm.ext[i]; g.m_sa[i] = gm.str[0][i]; g.m_sc[i] = gm.str[1][i]; }
    for (int i = 0; i < gn.n; ++i) { g.n_ext[i] = gn.ext[i]; g.n_sb[i] = gn.str[0][i]; g.n_sc[i] = gn.str[1][i]; }
    for (int i = 0; i < gk.n; ++i) { g.k_ext[i] = gk.ext[i]; g.k_sa[i] = gk.str[0][i]; g.k_sb[i] = gk.str[1][i]; }
    for (int i = 0; i < gl.n; ++i) {
      g.l_ext[i] = gl.ext[i]; g.l_sa[i] = gl.str[0][i]; g.l_sb[i] = gl.str[1][i]; g.l_sc[i] = gl.str[2][i];
    }
    // empty groups: one unit mode so that offsets evaluate to 0
    if (g.nm == 0) { g.nm = 1; g.m_ext[0] = 1; }
    if (g.nn == 0) { g.nn = 1; g.n_ext[0] = 1; }
    if (g.nk == 0) { g.nk = 1; g.k_ext[0] = 1; }
    if (g.nl == 0) { g.nl = 1; g.l_ext[0] = 1; }
    g.a_m_fast = g.m_sa[0] == 1;
    g.b_n_fast = g.n_sb[0] == 1;
    g.sx = sx;
    g.sy = sy;
    g.sy_zero = sy_zero;
    g.sx_one = scalar_is_one(dt, sx);
    trace_path("gemm M=%lld N=%lld K=%lld L=%lld modes=%d/%d/%d/%d afast=%d bfast=%d prec=%d", (long long)M,
               (long long)N, (long long)K, (long long)L, gm.n, gn.n, gk.n, gl.n, g.a_m_fast, g.b_n_fast, prec);
    // batches of small GEMMs with the batch mode innermost in every tensor
    // (column-major bij,bjk->bik): lanes over consecutive batches
    if (dt == OME_F32 && prec != OME_PREC_FP32 && gemm_bdiag_applies(g)) {
      cudaError_t e = launch_gemm_bdiag(g, prec == OME_PREC_BF16X3 ? 2 : 3, s);
      if (e != cudaErrorNotSupported) {
        trace_path("  -> batch-innermost tensor cores");
        return cuda_err(e, "batch-innermost tensor-core gemm");
      }
      cudaGetLastError();
    }
    if (gemm_bfast_applies(g)) {
      trace_path("  -> batch-innermost");
      return cuda_err(launch_gemm_bfast(dt, g, s), "batch-innermost gemm");
    }
    // FP32 batches of small GEMMs (M, N <= 64; tensor-core tiles would be mostly
    // padding with a few k-steps each): plain FP32 on CUDA cores
    if (dt == OME_F32 && M <= 64 && N <= 64 && L >= 8) {
      trace_path("  -> simt 64x64");
      return cuda_err(launch_gemm_simt_small_f32(g, s), "simt small gemm");
    }
    if (dt == OME_F32 && prec != OME_PREC_FP32 && gemm_split_supported(g)) {
      // output mode groups of several modes: C offset tables for the epilogues
      // (filled by the packed GEMM's pack launch, else by their own kernel)
      int64_t* tab = nullptr;
      if (g.nm > 1 || g.nn > 1) tab = static_cast<int64_t*>(ws_alloc(ctx, (size_t)(M + N) * sizeof(int64_t)));
      size_t avail = ctx->ws_bytes > ctx->ws_top ? ctx->ws_bytes - ((ctx->ws_top + 255) & ~(size_t)255) : 0;
      void* w = avail ? ctx->ws + ((ctx->ws_top + 255) & ~(size_t)255) : nullptr;
      const int nterms = prec == OME_PREC_BF16X3 ? 2 : 3;
      const int choice = gemm_kernel_choice(g);
      if (choice == 2) {
        cudaError_t e = launch_gemm_tma2(g, nterms, w, avail, ctx->num_sms, s);
        if (e != cudaErrorNotSupported) {
          trace_path("  -> tma2");
          return cuda_err(e, "tma bf16 split gemm");
        }
        cudaGetLastError();
      }
      if (choice >= 1) {
        void* pw = w;
        size_t pavail = avail;
        const size_t need = gemm_packed_bytes(g, nterms, ctx->num_sms);
        if (need > avail) {
          pw = overflow_scratch(ctx, need, s);
          pavail = pw ? ctx->ovf_bytes : 0;
        }
        cudaError_t e = pw ? launch_gemm_packed(g, nterms, pw, pavail, ctx->num_sms, s, tab) : cudaErrorNotSupported;
        if (e != cudaErrorNotSupported) {
          trace_path("  -> packed");
          return cuda_err(e, "packed bf16 split gemm");
        }
        cudaGetLastError();
      }
      if (tab) OME_CK(cuda_err(launch_c_offsets(g, tab, s), "offset tables"));
      trace_path("  -> tc");
      cudaError_t e = launch_gemm_split(g, nterms, w, avail, ctx->num_sms, s);
      if (e != cudaErrorNotSupported) return cuda_err(e, "bf16 split gemm");
      cudaGetLastError();
    }
    trace_path("  -> simt");
    // split-K partials (long K, few tiles) go to the free workspace above ws_top
    const size_t off = (ctx->ws_top + 255) & ~(size_t)255;
    const size_t free_bytes = ctx->ws_bytes > off ? ctx->ws_bytes - off : 0;
    return cuda_err(launch_gemm_simt_ws(dt, g, free_bytes ? ctx->ws + off : nullptr, free_bytes, ctx->num_sms, s),
                    "simt gemm");
  }
  HView xs[2] = {x1, x2};
  if (trace_on()) {
    char buf[96];
    snprintf(buf, sizeof(buf), " [binary M=%lld N=%lld K=%lld L=%lld]", (long long)M, (long long)N, (long long)K,
             (long long)L);
    int rc = run_loop(ctx, s, dt, 2, xs, yu, sx, sy, sy_zero);
    strncat(g_trace, buf, sizeof(g_trace) - strlen(g_trace) - 1);
    return rc;
  }
  return run_loop(ctx, s, dt, 2, xs, yu, sx, sy, sy_zero);
}

// ----------------------------------------------------------------------------
// einsum on labelled views
// ----------------------------------------------------------------------------

static int einsum_views_impl(ome_ctx* ctx, cudaStream_t s, ome_dtype dt, int nin, const HView* xs,
                             const HView& y, const Scalar& sx, const Scalar& sy_in, int prec, bool loop_only) {
  if (nin < 1) return set_err(OME_INVALID_ARGUMENT, "number of input tensors must be greater than 0");
  if (nin > MAXIN) return set_err(OME_UNSUPPORTED, "at most %d input tensors per contraction", MAXIN);
  // size dict consistency (get_size_dict!, src/interfaces.jl:75-94)
  std::vector<std::pair<int32_t, int64_t>> sd;
  auto check = [&](int32_t l, int64_t e) -> int {
    for (auto& p : sd)
      if (p.first == l) {
        if (p.second != e)
          return set_err(OME_DIMENSION_MISMATCH, "label %d = %lld or %lld)?", l, (long long)p.second, (long long)e);
        return OME_OK;
      }
    sd.push_back({l, e});
    return OME_OK;
  };
  for (int i = 0; i < nin; ++i)
    for (int d = 0; d < xs[i].nd; ++d) OME_CK(check(xs[i].lab[d], xs[i].ext[d]));
  for (int d = 0; d < y.nd; ++d) OME_CK(check(y.lab[d], y.ext[d]));

  HView xu[MAXIN], yu;
  for (int i = 0; i < nin; ++i) OME_CK(unique_view(xs[i], xu[i]));
  OME_CK(unique_view(y, yu));
  if (numel(y) == 0) return OME_OK;

  Scalar sy = sy_in;
  bool sy_zero = scalar_is_zero(dt, sy);
  if (scalar_is_zero(dt, sx)) {  // @addmul! iszero(b): y <- sy*y
    if (!sy_zero && scalar_is_one(dt, sy)) return OME_OK;
    return cuda_err(launch_scale(dt, y.data, y.nd, y.ext, y.str, sy, sy_zero, ctx->num_sms, s), "scale");
  }
  if (yu.nd < y.nd) {
    // repeated output labels: off-diagonal entries <- sy*y (or zero); the
    // diagonal view then accumulates onto the scaled values.
    if (!(!sy_zero && scalar_is_one(dt, sy)))
      OME_CK(cuda_err(launch_scale(dt, y.data, y.nd, y.ext, y.str, sy, sy_zero, ctx->num_sms, s), "scale"));
    sy = scalar_one(dt);
  }
  if (loop_only || nin >= 3) return run_loop(ctx, s, dt, nin, xu, yu, sx, sy, sy_zero);
  if (nin == 1) return run_unary(ctx, s, dt, xu[0], yu, sx, sy, sy_zero);
  return run_binary(ctx, s, dt, xu[0], xu[1], yu, sx, sy, sy_zero, prec);
}

int einsum_views(ome_ctx* ctx, cudaStream_t s, ome_dtype dt, int nin, const HView* xs, const HView& y,
                 const Scalar& sx, const Scalar& sy, int prec, bool loop_only) {
  if (!trace_on()) return einsum_views_impl(ctx, s, dt, nin, xs, y, sx, sy, prec, loop_only);
  g_trace[0] = 0;
  cudaEvent_t e0, e1;
  cudaEventCreate(&e0);
  cudaEventCreate(&e1);
  cudaEventRecord(e0, s);
  const int rc = einsum_views_impl(ctx, s, dt, nin, xs, y, sx, sy, prec, loop_only);
  cudaEventRecord(e1, s);
  const cudaError_t se = cudaEventSynchronize(e1);
  float ms = 0.f;
  cudaEventElapsedTime(&ms, e0, e1);
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  fprintf(stderr, "[ome] dt=%d nin=%d ranks=", (int)dt, nin);
  for (int i = 0; i < nin; ++i) fprintf(stderr, "%d,", xs[i].nd);
  fprintf(stderr, "%d us=%.1f err=%d %s\n", y.nd, ms * 1e3, (int)se, g_trace);
  return rc;
}

}  // namespace ome

using namespace ome;

// ============================================================================
// C ABI
// ============================================================================

extern "C" {

int ome_version(void) { return 1; }

unsigned long long ome_launch_count(void) { return ome::launch_counter(); }

int ome_device_status(void* stream) {
  const int r = ome::device_status(static_cast<cudaStream_t>(stream));
  if (r < 0) return cuda_err((cudaError_t)(-r), "device status");
  if (r > 100)
    return set_err(OME_CUDA_ERROR, "kernel self-check %d: an output offset outside the view was skipped", r - 100);
  if (r > 0) return set_err(OME_TIMEOUT, "a device-side wait gave up (bounded wait expired)");
  return OME_OK;
}

int ome_kernel_timing(int enable) {
  set_kernel_timing(enable);
  return OME_OK;
}

int ome_kernel_times(int32_t max, float* ms, const char** names, int32_t* count) {
  if (max < 0 || (max > 0 && (!ms || !names)) || !count) return set_err(OME_INVALID_ARGUMENT, "NULL argument");
  *count = read_kernel_times(max, ms, names);
  return OME_OK;
}

int ome_selftest_wait_timeout(void* stream, uint64_t wait_ns) {
  return cuda_err(launch_selftest_wait(wait_ns, static_cast<cudaStream_t>(stream)), "self-test kernel");
}

const char* ome_last_error(void) { return g_err.c_str(); }

int ome_ctx_create(int device, size_t workspace_bytes, ome_ctx** out) {
  if (!out) return set_err(OME_INVALID_ARGUMENT, "out is NULL");
  *out = nullptr;
  int ndev = 0;
  OME_CUDA(cudaGetDeviceCount(&ndev), "cudaGetDeviceCount");
  if (device < 0 || device >= ndev) return set_err(OME_INVALID_ARGUMENT, "device %d of %d", device, ndev);
  OME_CUDA(cudaSetDevice(device), "cudaSetDevice");
  ome_ctx* c = new ome_ctx();
  c->device = device;
  cudaDeviceGetAttribute(&c->num_sms, cudaDevAttrMultiProcessorCount, device);
  c->ws = nullptr;
  c->ws_bytes = workspace_bytes;
  c->ws_top = 0;
  c->ovf = nullptr;
  c->ovf_bytes = 0;
  if (workspace_bytes) {
    cudaError_t e = cudaMalloc(&c->ws, workspace_bytes);
    if (e != cudaSuccess) {
      delete c;
      return cuda_err(e, "workspace cudaMalloc");
    }
  }
  *out = c;
  return OME_OK;
}

int ome_ctx_destroy(ome_ctx* ctx) {
  if (!ctx) return OME_OK;
  if (ctx->ws) cudaFree(ctx->ws);
  if (ctx->ovf) cudaFree(ctx->ovf);
  delete ctx;
  return OME_OK;
}

int ome_ctx_workspace_bytes(const ome_ctx* ctx, size_t* out) {
  if (!ctx || !out) return set_err(OME_INVALID_ARGUMENT, "NULL argument");
  *out = ctx->ws_bytes;
  return OME_OK;
}

static int einsum_entry(ome_ctx* ctx, void* stream, ome_dtype dtype, int32_t ninputs, const ome_tensor* xs,
                        const ome_tensor* y, const void* sx, const void* sy, int32_t prec, bool loop_only) {
  if (!ctx || !y || !sx || !sy || (ninputs > 0 && !xs)) return set_err(OME_INVALID_ARGUMENT, "NULL argument");
  if ((int)dtype < 0 || (int)dtype > OME_TROP_F64) return set_err(OME_INVALID_ARGUMENT, "unknown dtype %d", (int)dtype);
  if (ninputs < 1) return set_err(OME_INVALID_ARGUMENT, "number of input tensors must be greater than 0");
  if (ninputs > MAXIN) return set_err(OME_UNSUPPORTED, "at most %d input tensors per contraction", MAXIN);
  HView xv[MAXIN], yv;
  for (int i = 0; i < ninputs; ++i) OME_CK(view_from_tensor(xs[i], xv[i], "input"));
  OME_CK(view_from_tensor(*y, yv, "output"));
  ctx->ws_top = 0;
  return einsum_views(ctx, static_cast<cudaStream_t>(stream), dtype, ninputs, xv, yv, scalar_from(dtype, sx),
                      scalar_from(dtype, sy), prec, loop_only);
}

int ome_einsum(ome_ctx* ctx, void* stream, ome_dtype dtype, int32_t ninputs, const ome_tensor* xs,
               const ome_tensor* y, const void* sx, const void* sy, int32_t prec) {
  return einsum_entry(ctx, stream, dtype, ninputs, xs, y, sx, sy, prec, false);
}

int ome_loop_einsum(ome_ctx* ctx, void* stream, ome_dtype dtype, int32_t ninputs, const ome_tensor* xs,
                    const ome_tensor* y, const void* sx, const void* sy) {
  return einsum_entry(ctx, stream, dtype, ninputs, xs, y, sx, sy, OME_PREC_FP32, true);
}

// einsum_grad (src/autodiff.jl:24-30): dx <- conj(einsum(ixs with iy in place
// of ixs[i] -> ixs[i])(xs with conj(dy) in place of xs[i])).  For complex
// dtypes conj(dy) goes to a column-major workspace copy and the result is
// conjugated in place (through a workspace copy when dx is strided).
int ome_einsum_grad(ome_ctx* ctx, void* stream, ome_dtype dtype, int32_t ninputs, const ome_tensor* xs,
                    const ome_tensor* dy, int32_t i, const ome_tensor* dx, int32_t prec) {
  if (!ctx || !xs || !dy || !dx) return set_err(OME_INVALID_ARGUMENT, "NULL argument");
  if ((int)dtype < 0 || (int)dtype > OME_TROP_F64) return set_err(OME_INVALID_ARGUMENT, "unknown dtype %d", (int)dtype);
  if (ninputs < 1) return set_err(OME_INVALID_ARGUMENT, "number of input tensors must be greater than 0");
  if (ninputs > MAXIN) return set_err(OME_UNSUPPORTED, "at most %d input tensors per contraction", MAXIN);
  if (i < 0 || i >= ninputs) return set_err(OME_INVALID_ARGUMENT, "input index %d outside [0, %d)", i, ninputs);
  if (xs[i].ndim != dx->ndim) return set_err(OME_INVALID_ARGUMENT, "the gradient must have the rank of input %d", i);
  for (int d = 0; d < dx->ndim; ++d) {
    if (!xs[i].labels || !dx->labels || xs[i].labels[d] != dx->labels[d])
      return set_err(OME_INVALID_ARGUMENT, "the gradient's labels must be those of input %d", i);
    if (xs[i].dims && xs[i].dims[d] != dx->dims[d])
      return set_err(OME_DIMENSION_MISMATCH, "label %d = %lld or %lld)?", dx->labels[d],
                     (long long)xs[i].dims[d], (long long)dx->dims[d]);
  }
  HView xv[MAXIN], dyv, dxv;
  for (int k = 0; k < ninputs; ++k)
    if (k != i) OME_CK(view_from_tensor(xs[k], xv[k], "input"));
  OME_CK(view_from_tensor(*dy, dyv, "cotangent"));
  OME_CK(view_from_tensor(*dx, dxv, "gradient"));
  ctx->ws_top = 0;
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  const Scalar one = scalar_one(dtype), zero = scalar_zero(dtype);
  const bool cplx = dtype == OME_C32 || dtype == OME_C64;
  const size_t es = dtype_size(dtype);
  auto contiguous_copy = [&](const HView& v, HView& c) -> int {
    c = v;
    int64_t st = 1;
    for (int d = 0; d < v.nd; ++d) {
      c.str[d] = st;
      st *= v.ext[d];
    }
    c.data = static_cast<char*>(ws_alloc(ctx, (size_t)std::max<int64_t>(st, 1) * es));
    if (!c.data) return set_err(OME_OUT_OF_MEMORY, "workspace too small for a gradient temporary (%lld elements)",
                                (long long)st);
    return OME_OK;
  };
  if (cplx) {
    HView c;
    OME_CK(contiguous_copy(dyv, c));
    OME_CK(einsum_views(ctx, s, dtype, 1, &dyv, c, one, zero, prec, false));
    OME_CK(cuda_err(launch_conj(dtype, c.data, std::max<int64_t>(numel(c), 1), s), "conj"));
    xv[i] = c;
  } else {
    xv[i] = dyv;
  }
  bool dense = true;
  {
    int64_t st = 1;
    for (int d = 0; d < dxv.nd; ++d) {
      if (dxv.ext[d] > 1 && dxv.str[d] != st) dense = false;
      st *= dxv.ext[d];
    }
  }
  HView out = dxv;
  if (cplx && !dense) OME_CK(contiguous_copy(dxv, out));
  OME_CK(einsum_views(ctx, s, dtype, ninputs, xv, out, one, zero, prec, false));
  if (cplx) {
    OME_CK(cuda_err(launch_conj(dtype, out.data, std::max<int64_t>(numel(out), 1), s), "conj"));
    if (!dense) OME_CK(einsum_views(ctx, s, dtype, 1, &out, dxv, one, zero, prec, false));
  }
  return OME_OK;
}

}  // extern "C"
