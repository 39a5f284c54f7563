// Index-iterating kernels of libomeb200:
//  * k_loop_thread / k_loop_block / k_loop_finish: the generic sum-product
//    over labelled strided inputs (loop_einsum!, src/loop_einsum.jl:21-45;
//    GPU form ext/CUDAExt.jl:60-113).  Also serves Sum (src/unaryrules.jl:30-40),
//    Tr (:22-26) on a diagonal view, GEMV/dot/outer/Hadamard-shaped binary
//    rules and the n-ary fallback.
//  * k_transpose / k_map_rows / k_copy: Permutedims via tensorpermute!
//    (src/utils.jl:122-156), Repeat (src/unaryrules.jl:44-58, stride-0 input
//    modes) and Identity; k_map_rows also runs contractions without summed
//    labels (Hadamard and outer products);
//  * k_reduce_contig / k_reduce_rows / k_loop_cols: Sum and sum-products
//    whose summed or output modes are contiguous (dot, GEMV, column sums).
//  * k_scale, k_acc64*: αβ pre-pass and FP64 cross-slice accumulation.
#include <string.h>
#include <mutex>
#include <vector>
#include "kernels.h"

namespace ome {

// Largest |offset| reachable over the modes (sum of (ext-1)*|stride|).
static int64_t max_offset(int nd, const int64_t* ext, const int64_t* str) {
  int64_t m = 0;
  for (int i = 0; i < nd; ++i) m += (ext[i] > 0 ? ext[i] - 1 : 0) * (str[i] < 0 ? -str[i] : str[i]);
  return m;
}

static unsigned long long g_launches = 0;
unsigned long long launch_counter() { return __atomic_load_n(&g_launches, __ATOMIC_RELAXED); }
void count_launch(int n) { __atomic_fetch_add(&g_launches, (unsigned long long)n, __ATOMIC_RELAXED); }

// ---------------------------------------------------------------------------
// diagnostic kernel timing
// ---------------------------------------------------------------------------
struct TimedKernel {
  int ev;   // index of its event pair in the pool
  const char* name;
};
static std::mutex g_tmu;
static bool g_timing = false;
static std::vector<std::pair<cudaEvent_t, cudaEvent_t>> g_pool;   // created once, reused
static std::vector<TimedKernel> g_timed;
static const size_t kMaxTimed = 1 << 16;

static bool grow_pool(size_t n) {
  while (g_pool.size() < n) {
    cudaEvent_t b, e;
    if (cudaEventCreate(&b) != cudaSuccess) { cudaGetLastError(); return false; }
    if (cudaEventCreate(&e) != cudaSuccess) { cudaEventDestroy(b); cudaGetLastError(); return false; }
    g_pool.push_back({b, e});
  }
  return true;
}

KernelTimer::KernelTimer(cudaStream_t s_, const char* name_) : s(s_), name(name_), slot(-1) {
  std::lock_guard<std::mutex> lk(g_tmu);
  if (!g_timing || g_timed.size() >= kMaxTimed) return;
  const int idx = (int)g_timed.size();
  if (!grow_pool((size_t)idx + 1)) return;
  cudaEventRecord(g_pool[idx].first, s);
  g_timed.push_back({idx, name});
  slot = idx;
}

KernelTimer::~KernelTimer() {
  if (slot < 0) return;
  std::lock_guard<std::mutex> lk(g_tmu);
  if (slot < (int)g_timed.size()) cudaEventRecord(g_pool[g_timed[slot].ev].second, s);
}

void set_kernel_timing(int n) {
  std::lock_guard<std::mutex> lk(g_tmu);
  g_timed.clear();
  g_timing = n > 0;
  if (n > 0) grow_pool(std::min((size_t)n, kMaxTimed));
}

int read_kernel_times(int max, float* ms, const char** names) {
  std::lock_guard<std::mutex> lk(g_tmu);
  int n = 0;
  for (auto& t : g_timed) {
    if (n >= max) break;
    float v = -1.f;
    const auto& ev = g_pool[t.ev];
    if (cudaEventSynchronize(ev.second) == cudaSuccess) cudaEventElapsedTime(&v, ev.first, ev.second);
    cudaGetLastError();
    ms[n] = v;
    names[n] = t.name;
    ++n;
  }
  return n;
}

// ---------------------------------------------------------------------------
// generic loop kernel
// ---------------------------------------------------------------------------

template <class A, int NIN>
__device__ __forceinline__ typename A::T loop_prod(const LoopArgs& a, const int64_t* off) {
  using T = typename A::T;
  const int nin = NIN > 0 ? NIN : a.nin;
  T p = static_cast<const T*>(a.x[0])[off[0]];
#pragma unroll
  for (int i = 1; i < (NIN > 0 ? NIN : MAXIN); ++i) {
    if (i < nin) p = A::mul(p, static_cast<const T*>(a.x[i])[off[i]]);
  }
  return p;
}

// Decompose output index o over the output modes; fills input offsets.
template <int NIN>
__device__ __forceinline__ int64_t loop_outer_offsets(const LoopArgs& a, int64_t o, int64_t* off) {
  const int nin = NIN > 0 ? NIN : a.nin;
  int64_t yoff = 0;
#pragma unroll
  for (int i = 0; i < (NIN > 0 ? NIN : MAXIN); ++i) off[i] = 0;
  for (int m = 0; m < a.nout; ++m) {
    const int64_t e = a.ext[m];
    const int64_t q = o / e;
    const int64_t d = o - q * e;
    o = q;
    yoff += d * a.str[0][m];
#pragma unroll
    for (int i = 0; i < (NIN > 0 ? NIN : MAXIN); ++i)
      if (i < nin) off[i] += d * a.str[1 + i][m];
  }
  return yoff;
}

// One thread per output element; the first inner mode is a plain loop, the
// remaining inner modes an odometer (no divisions in the inner loop).
template <class A, int NIN>
__global__ void __launch_bounds__(256) k_loop_thread(const __grid_constant__ LoopArgs a) {
  using T = typename A::T;
  constexpr int NI = NIN > 0 ? NIN : MAXIN;
  const int nin = NIN > 0 ? NIN : a.nin;
  const T sx = scalar_as<T>(a.sx), sy = scalar_as<T>(a.sy);
  const int m0 = a.nout;
  const int64_t e0 = a.ninner > 0 ? a.ext[m0] : 1;
  for (int64_t o = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; o < a.n_out;
       o += (int64_t)gridDim.x * blockDim.x) {
    int64_t off[NI];
    const int64_t yoff = loop_outer_offsets<NIN>(a, o, off);
    T acc = A::zero();
    if (a.n_in > 0) {
      int64_t s0[NI];
#pragma unroll
      for (int i = 0; i < NI; ++i) s0[i] = (i < nin && a.ninner > 0) ? a.str[1 + i][m0] : 0;
      int dig[MAXM];
      for (int m = 0; m < a.ninner; ++m) dig[m] = 0;
      while (true) {
        int64_t o2[NI];
#pragma unroll
        for (int i = 0; i < NI; ++i) o2[i] = off[i];
        for (int64_t j = 0; j < e0; ++j) {
          acc = A::add(acc, loop_prod<A, NIN>(a, o2));
#pragma unroll
          for (int i = 0; i < NI; ++i) o2[i] += s0[i];
        }
        int m = 1;
        for (; m < a.ninner; ++m) {
          const int mm = m0 + m;
          dig[m]++;
#pragma unroll
          for (int i = 0; i < NI; ++i)
            if (i < nin) off[i] += a.str[1 + i][mm];
          if (dig[m] < a.ext[mm]) break;
#pragma unroll
          for (int i = 0; i < NI; ++i)
            if (i < nin) off[i] -= a.ext[mm] * a.str[1 + i][mm];
          dig[m] = 0;
        }
        if (m >= a.ninner) break;
      }
    }
    T* yp = static_cast<T*>(a.y) + yoff;
    *yp = epilogue<A>(acc, yp, sx, sy, a.sy_zero, a.sx_one);
  }
}

// Sum-products whose summed modes are strided while y's fastest mode is
// contiguous in the inputs (GEMV `ij,j->i`, `ijk->ik`): a thread per output,
// consecutive threads on consecutive outputs (each load is coalesced across
// the warp), the summed space cut into nsplit ranges (blockIdx.y), each
// walked by an odometer; split partials go to a.partial[o * nsplit + s] for
// k_loop_finish.
template <class A, int NIN, bool VEC>
__global__ void __launch_bounds__(256) k_loop_cols(const __grid_constant__ LoopArgs a, int64_t chunk) {
  using T = typename A::T;
  constexpr int NI = NIN > 0 ? NIN : MAXIN;
  constexpr int V = VEC ? (int)(16 / sizeof(T)) : 1;   // consecutive outputs per thread
  const int nin = NIN > 0 ? NIN : a.nin;
  const T sx = scalar_as<T>(a.sx), sy = scalar_as<T>(a.sy);
  griddep_launch_dependents();
  const int64_t split = blockIdx.y;
  const int64_t jb = split * chunk;
  const int64_t je = min(a.n_in, jb + chunk);
  const int64_t ngroups = a.n_out / V;
  for (int64_t g = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; g < ngroups;
       g += (int64_t)gridDim.x * blockDim.x) {
    const int64_t o = g * V;
    int64_t off[NI];
    const int64_t yoff = loop_outer_offsets<NIN>(a, o, off);
    int64_t dig[MAXM];
    int64_t j = jb;
    for (int m = 0; m < a.ninner; ++m) {
      const int mm = a.nout + m;
      const int64_t e = a.ext[mm];
      const int64_t q = j / e;
      dig[m] = j - q * e;
      j = q;
#pragma unroll
      for (int i = 0; i < NI; ++i)
        if (i < nin) off[i] += dig[m] * a.str[1 + i][mm];
    }
    // U steps at a time: the odometer first records the U offsets, then all
    // their loads are issued, then they are added in order (the sum order is
    // the sequential one)
    constexpr int U = VEC ? 4 : 8;
    T acc[V];
#pragma unroll
    for (int v = 0; v < V; ++v) acc[v] = A::zero();
    for (int64_t jj = jb; jj < je; jj += U) {
      int64_t o2[U][NI];
#pragma unroll
      for (int u = 0; u < U; ++u) {
#pragma unroll
        for (int i = 0; i < NI; ++i) o2[u][i] = off[i];
        if (jj + u + 1 < je) {
          for (int m = 0; m < a.ninner; ++m) {
            const int mm = a.nout + m;
#pragma unroll
            for (int i = 0; i < NI; ++i)
              if (i < nin) off[i] += a.str[1 + i][mm];
            if (++dig[m] < a.ext[mm]) break;
#pragma unroll
            for (int i = 0; i < NI; ++i)
              if (i < nin) off[i] -= a.ext[mm] * a.str[1 + i][mm];
            dig[m] = 0;
          }
        }
      }
      T val[U][V];
#pragma unroll
      for (int u = 0; u < U; ++u) {
        if constexpr (VEC) {
          if (jj + u >= je) break;
#pragma unroll
          for (int i = 0; i < NI; ++i) {
            if (i >= nin) break;
            const T* xi = static_cast<const T*>(a.x[i]) + o2[u][i];
            T w[V];
            if (a.str[1 + i][0] == 0) {
              const T c = xi[0];
#pragma unroll
              for (int v = 0; v < V; ++v) w[v] = c;
            } else {
              const uint4 w4 = __ldg(reinterpret_cast<const uint4*>(xi));
              memcpy(w, &w4, sizeof(w4));
            }
#pragma unroll
            for (int v = 0; v < V; ++v) val[u][v] = i == 0 ? w[v] : A::mul(val[u][v], w[v]);
          }
        } else {
          val[u][0] = jj + u < je ? loop_prod<A, NIN>(a, o2[u]) : A::zero();
        }
      }
#pragma unroll
      for (int u = 0; u < U; ++u)
        if (jj + u < je)
#pragma unroll
          for (int v = 0; v < V; ++v) acc[v] = A::add(acc[v], val[u][v]);
    }
#pragma unroll
    for (int v = 0; v < V; ++v) {
      if (a.nsplit == 1) {
        T* yp = static_cast<T*>(a.y) + yoff + v;
        *yp = epilogue<A>(acc[v], yp, sx, sy, a.sy_zero, a.sx_one);
      } else {
        static_cast<T*>(a.partial)[(o + v) * a.nsplit + split] = acc[v];
      }
    }
  }
}

template <class A, bool VEC>
static void launch_loop_cols_v(const LoopArgs& a, int64_t chunk, dim3 grid, cudaStream_t s) {
  switch (a.nin) {
    case 1: k_loop_cols<A, 1, VEC><<<grid, 256, 0, s>>>(a, chunk); break;
    case 2: k_loop_cols<A, 2, VEC><<<grid, 256, 0, s>>>(a, chunk); break;
    case 3: k_loop_cols<A, 3, VEC><<<grid, 256, 0, s>>>(a, chunk); break;
    default: k_loop_cols<A, 0, VEC><<<grid, 256, 0, s>>>(a, chunk); break;
  }
}

template <class A>
static cudaError_t launch_loop_cols_t(const LoopArgs& a, int64_t chunk, dim3 grid, bool vec, cudaStream_t s) {
  KernelTimer kt(s, "k_loop_cols");
  if constexpr (sizeof(typename A::T) <= 8 && 16 % sizeof(typename A::T) == 0) {
    if (vec) launch_loop_cols_v<A, true>(a, chunk, grid, s);
    else launch_loop_cols_v<A, false>(a, chunk, grid, s);
  } else {
    launch_loop_cols_v<A, false>(a, chunk, grid, s);
  }
  count_launch();
  return cudaGetLastError();
}

cudaError_t launch_loop_cols(ome_dtype dt, const LoopArgs& a, int64_t chunk, dim3 grid, bool vec, cudaStream_t s) {
  cudaError_t e = cudaErrorInvalidValue;
  OME_DISPATCH(dt, ALG, e = launch_loop_cols_t<ALG>(a, chunk, grid, vec, s));
  return e;
}

// Inner counter advanced by a fixed step given as mixed-radix digits.
template <int NIN>
struct InnerCursor {
  int64_t dig[MAXM];
  __device__ __forceinline__ void init(const LoopArgs& a, int64_t j, int64_t* off) {
    const int nin = NIN > 0 ? NIN : a.nin;
    for (int m = 0; m < a.ninner; ++m) {
      const int mm = a.nout + m;
      const int64_t e = a.ext[mm];
      const int64_t q = j / e;
      const int64_t d = j - q * e;
      j = q;
      dig[m] = d;
#pragma unroll
      for (int i = 0; i < (NIN > 0 ? NIN : MAXIN); ++i)
        if (i < nin) off[i] += d * a.str[1 + i][mm];
    }
  }
  __device__ __forceinline__ void advance(const LoopArgs& a, int64_t* off) {
    const int nin = NIN > 0 ? NIN : a.nin;
    int carry = 0;
    for (int m = 0; m < a.ninner; ++m) {
      const int mm = a.nout + m;
      int64_t nd = dig[m] + a.stepdig[m] + carry;
      const int64_t e = a.ext[mm];
      carry = nd >= e;
      if (carry) nd -= e;
      const int64_t delta = nd - dig[m];
      dig[m] = nd;
#pragma unroll
      for (int i = 0; i < (NIN > 0 ? NIN : MAXIN); ++i)
        if (i < nin) off[i] += delta * a.str[1 + i][mm];
    }
  }
};

// One block per output element (nsplit == 1), or nsplit blocks per output
// each summing a strided share of the inner space into a.partial.
template <class A, int NIN>
__global__ void __launch_bounds__(256) k_loop_block(const __grid_constant__ LoopArgs a) {
  using T = typename A::T;
  griddep_launch_dependents();   // the finish pass (if any) may start its set-up
  constexpr int NI = NIN > 0 ? NIN : MAXIN;
  constexpr int U = 4;
  __shared__ T sh[32];
  const T sx = scalar_as<T>(a.sx), sy = scalar_as<T>(a.sy);
  const int64_t step = (int64_t)blockDim.x * a.nsplit;
  const int64_t nblocks = a.n_out * a.nsplit;
  for (int64_t b = blockIdx.x; b < nblocks; b += gridDim.x) {
    const int64_t o = b / a.nsplit;
    const int64_t split = b - o * a.nsplit;
    int64_t off[NI];
    const int64_t yoff = loop_outer_offsets<NIN>(a, o, off);
    T acc = A::zero();
    int64_t j = split * blockDim.x + threadIdx.x;
    if (j < a.n_in) {
      InnerCursor<NIN> cur;
      cur.init(a, j, off);
      while (j < a.n_in) {
        T v[U];
#pragma unroll
        for (int u = 0; u < U; ++u) {
          if (j < a.n_in) {
            v[u] = loop_prod<A, NIN>(a, off);
            j += step;
            if (j < a.n_in) cur.advance(a, off);
          } else {
            v[u] = A::zero();
          }
        }
#pragma unroll
        for (int u = 0; u < U; ++u) acc = A::add(acc, v[u]);
      }
    }
    acc = block_reduce<A>(acc, sh);
    if (threadIdx.x == 0) {
      if (a.nsplit == 1) {
        T* yp = static_cast<T*>(a.y) + yoff;
        *yp = epilogue<A>(acc, yp, sx, sy, a.sy_zero, a.sx_one);
      } else {
        static_cast<T*>(a.partial)[b] = acc;
      }
    }
  }
}

// Sum the nsplit partials of each output in a fixed order and apply the αβ
// epilogue (deterministic two-pass reduction).
template <class A>
__global__ void __launch_bounds__(256) k_loop_finish(const __grid_constant__ LoopArgs a) {
  using T = typename A::T;
  griddep_wait();   // the partials of the previous kernel
  const T sx = scalar_as<T>(a.sx), sy = scalar_as<T>(a.sy);
  for (int64_t o = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; o < a.n_out;
       o += (int64_t)gridDim.x * blockDim.x) {
    int64_t yoff = 0, r = o;
    for (int m = 0; m < a.nout; ++m) {
      const int64_t e = a.ext[m];
      const int64_t q = r / e;
      yoff += (r - q * e) * a.str[0][m];
      r = q;
    }
    const T* p = static_cast<const T*>(a.partial) + o * a.nsplit;
    T acc = A::zero();
    for (int s = 0; s < a.nsplit; ++s) acc = A::add(acc, p[s]);
    T* yp = static_cast<T*>(a.y) + yoff;
    *yp = epilogue<A>(acc, yp, sx, sy, a.sy_zero, a.sx_one);
  }
}

// Reduction of one input whose first summed mode is contiguous (Sum over a
// leading dimension, src/unaryrules.jl:30-40).  Inner space = E0 contiguous
// elements x R rows (at most one more summed mode, row stride rs).  One block
// per (output, row split); 16-byte vector loads when VEC (every row start
// 16-byte aligned and E0 a multiple of the vector width), 4 loads in flight.
// Values of the NIN inputs at one unit (V consecutive elements of a row):
// inputs with stride 1 along the row are read (16-byte loads when VEC),
// stride-0 inputs give their row value; the product is left to right.
template <class A, int NIN, bool VEC, int V>
__device__ __forceinline__ void row_unit(const typename A::T* const (&xr)[NIN], const int (&s0)[NIN], int64_t c,
                                         typename A::T (&out)[V]) {
  using T = typename A::T;
#pragma unroll
  for (int k = 0; k < NIN; ++k) {
    T v[V];
    if (s0[k] == 0) {
      const T c0 = xr[k][0];
#pragma unroll
      for (int j = 0; j < V; ++j) v[j] = c0;
    } else if constexpr (VEC) {
      const uint4 w = __ldg(reinterpret_cast<const uint4*>(xr[k] + c * V));
      memcpy(v, &w, sizeof(w));
    } else {
      v[0] = xr[k][c];
    }
#pragma unroll
    for (int j = 0; j < V; ++j) out[j] = k == 0 ? v[j] : A::mul(out[j], v[j]);
  }
}

template <class A, int NIN, bool VEC, class I>
__global__ void __launch_bounds__(256) k_reduce_contig(const __grid_constant__ LoopArgs a, int64_t rchunk,
                                                       FastDiv chdiv) {
  griddep_launch_dependents();   // the finish pass (if any) may start its set-up
  using T = typename A::T;
  constexpr int V = VEC ? (16 / sizeof(T) > 0 ? 16 / sizeof(T) : 1) : 1;
  constexpr int U = NIN == 1 ? 8 : 4;
  __shared__ T sh[32];
  const T sx = scalar_as<T>(a.sx), sy = scalar_as<T>(a.sy);
  const int64_t e0 = a.ext[a.nout];
  const int64_t R = a.ninner > 1 ? a.ext[a.nout + 1] : 1;
  int s0[NIN];
  int64_t rs[NIN];
#pragma unroll
  for (int k = 0; k < NIN; ++k) {
    s0[k] = (int)a.str[1 + k][a.nout];
    rs[k] = a.ninner > 1 ? a.str[1 + k][a.nout + 1] : 0;
  }
  const int64_t chunks = e0 / V;              // vector units per row
  const int64_t nblocks = a.n_out * a.nsplit;
  for (int64_t b = blockIdx.x; b < nblocks; b += gridDim.x) {
    const int64_t o = b / a.nsplit;
    const int64_t split = b - o * a.nsplit;
    int64_t off[NIN];
    const int64_t yoff = loop_outer_offsets<NIN>(a, o, off);
    const int64_t rbeg = split * rchunk;
    const int64_t rend = min(R, rbeg + rchunk);
    // offsets inside one split in I (int32 when the split's span fits)
    const I units = (I)((rend - rbeg) * chunks);
    const I ich = (I)chunks;
    const T* xb[NIN];
#pragma unroll
    for (int k = 0; k < NIN; ++k) xb[k] = static_cast<const T*>(a.x[k]) + off[k] + rbeg * rs[k];
    T acc = A::zero();
    for (I u0 = threadIdx.x; u0 < units; u0 += (I)blockDim.x * U) {
      T part[U][V];
#pragma unroll
      for (int j = 0; j < U; ++j) {
        const I u = u0 + (I)j * (I)blockDim.x;
        if (u < units) {
          I r;
          if constexpr (sizeof(I) == 4) r = (I)fast_div((uint32_t)u, chdiv);
          else r = u / ich;
          const I c = u - r * ich;
          const T* xr[NIN];
#pragma unroll
          for (int k = 0; k < NIN; ++k) xr[k] = xb[k] + (I)(r * (I)rs[k]);
          row_unit<A, NIN, VEC, V>(xr, s0, (int64_t)c, part[j]);
        } else {
#pragma unroll
          for (int v = 0; v < V; ++v) part[j][v] = A::zero();
        }
      }
#pragma unroll
      for (int j = 0; j < U; ++j)
#pragma unroll
        for (int v = 0; v < V; ++v) acc = A::add(acc, part[j][v]);
    }
    acc = block_reduce<A>(acc, sh);
    if (threadIdx.x == 0) {
      if (a.nsplit == 1) {
        T* yp = static_cast<T*>(a.y) + yoff;
        *yp = epilogue<A>(acc, yp, sx, sy, a.sy_zero, a.sx_one);
      } else {
        static_cast<T*>(a.partial)[b] = acc;
      }
    }
  }
}

// The same reduction when there are many outputs (column sums of a tall
// column-major array, `ijk->jk`; GEMV `ji,j->i`): one warp per output, lanes
// along the contiguous row with 16-byte loads (4 per lane in flight), the
// optional second summed mode as an outer loop, then a shuffle reduction.
// Every lane runs the same row and round counts, so the whole warp reaches
// the shuffles.
template <class A, int NIN, bool VEC>
__global__ void __launch_bounds__(256) k_reduce_rows(const __grid_constant__ LoopArgs a) {
  using T = typename A::T;
  constexpr int V = VEC ? (16 / sizeof(T) > 0 ? 16 / sizeof(T) : 1) : 1;
  constexpr int U = 4;
  const T sx = scalar_as<T>(a.sx), sy = scalar_as<T>(a.sy);
  const int64_t e0 = a.ext[a.nout];
  const int64_t R = a.ninner > 1 ? a.ext[a.nout + 1] : 1;
  int s0[NIN];
  int64_t rs[NIN];
#pragma unroll
  for (int k = 0; k < NIN; ++k) {
    s0[k] = (int)a.str[1 + k][a.nout];
    rs[k] = a.ninner > 1 ? a.str[1 + k][a.nout + 1] : 0;
  }
  const int64_t chunks = e0 / V;
  const int lane = threadIdx.x & 31;
  const int64_t nw = (int64_t)gridDim.x * (blockDim.x >> 5);
  for (int64_t o = (int64_t)blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5); o < a.n_out; o += nw) {
    int64_t off[NIN];
    const int64_t yoff = loop_outer_offsets<NIN>(a, o, off);
    T acc = A::zero();
    for (int64_t r = 0; r < R; ++r) {
      const T* xr[NIN];
#pragma unroll
      for (int k = 0; k < NIN; ++k) xr[k] = static_cast<const T*>(a.x[k]) + off[k] + r * rs[k];
      for (int64_t c0 = lane; c0 - lane < chunks; c0 += 32 * U) {
        T part[U][V];
#pragma unroll
        for (int j = 0; j < U; ++j) {
          const int64_t c = c0 + 32 * j;
          if (c < chunks) {
            row_unit<A, NIN, VEC, V>(xr, s0, c, part[j]);
          } else {
#pragma unroll
            for (int v = 0; v < V; ++v) part[j][v] = A::zero();
          }
        }
#pragma unroll
        for (int j = 0; j < U; ++j)
#pragma unroll
          for (int v = 0; v < V; ++v) acc = A::add(acc, part[j][v]);
      }
    }
    for (int d = 16; d > 0; d >>= 1) acc = A::add(acc, shfl_down_any(acc, d));
    if (lane == 0) {
      T* yp = static_cast<T*>(a.y) + yoff;
      *yp = epilogue<A>(acc, yp, sx, sy, a.sy_zero, a.sx_one);
    }
  }
}

template <class A, int NIN>
static void launch_reduce_rows_n(const LoopArgs& a, bool vec, int grid, cudaStream_t s) {
  if (vec) k_reduce_rows<A, NIN, true><<<grid, 256, 0, s>>>(a);
  else k_reduce_rows<A, NIN, false><<<grid, 256, 0, s>>>(a);
}

template <class A>
static cudaError_t launch_reduce_rows_t(const LoopArgs& a, bool vec, int grid, cudaStream_t s) {
  KernelTimer kt(s, "k_reduce_rows");
  if (a.nin == 1) launch_reduce_rows_n<A, 1>(a, vec, grid, s);
  else if (a.nin == 2) launch_reduce_rows_n<A, 2>(a, vec, grid, s);
  else launch_reduce_rows_n<A, 3>(a, vec, grid, s);
  count_launch();
  return cudaGetLastError();
}

cudaError_t launch_reduce_rows(ome_dtype dt, const LoopArgs& a, bool vec, int grid, cudaStream_t s) {
  cudaError_t e = cudaErrorInvalidValue;
  OME_DISPATCH(dt, ALG, e = launch_reduce_rows_t<ALG>(a, vec, grid, s));
  return e;
}

template <class A, int NIN>
static void launch_reduce_contig_n(const LoopArgs& a, bool vec, bool small, int64_t rchunk, FastDiv chdiv, int grid,
                                   cudaStream_t s) {
  if (vec) {
    if (small) k_reduce_contig<A, NIN, true, int32_t><<<grid, 256, 0, s>>>(a, rchunk, chdiv);
    else k_reduce_contig<A, NIN, true, int64_t><<<grid, 256, 0, s>>>(a, rchunk, chdiv);
  } else {
    if (small) k_reduce_contig<A, NIN, false, int32_t><<<grid, 256, 0, s>>>(a, rchunk, chdiv);
    else k_reduce_contig<A, NIN, false, int64_t><<<grid, 256, 0, s>>>(a, rchunk, chdiv);
  }
}

template <class A>
static cudaError_t launch_reduce_contig_t(const LoopArgs& a, bool vec, int64_t rchunk, int grid, cudaStream_t s) {
  const int64_t R = a.ninner > 1 ? a.ext[a.nout + 1] : 1;
  bool small = R * a.ext[a.nout] < ((int64_t)1 << 30);
  for (int k = 0; k < a.nin; ++k) {
    const int64_t rs = a.ninner > 1 ? a.str[1 + k][a.nout + 1] : 0;
    small = small && rchunk * (rs > 0 ? rs : 1) + a.ext[a.nout] < ((int64_t)1 << 30);
  }
  constexpr int V = 16 / sizeof(typename A::T) > 0 ? 16 / sizeof(typename A::T) : 1;
  const FastDiv chdiv = make_fastdiv((uint32_t)(small ? a.ext[a.nout] / (vec ? V : 1) : 1));
  KernelTimer kt(s, "k_reduce_contig");
  if (a.nin == 1) launch_reduce_contig_n<A, 1>(a, vec, small, rchunk, chdiv, grid, s);
  else if (a.nin == 2) launch_reduce_contig_n<A, 2>(a, vec, small, rchunk, chdiv, grid, s);
  else launch_reduce_contig_n<A, 3>(a, vec, small, rchunk, chdiv, grid, s);
  count_launch();
  return cudaGetLastError();
}

cudaError_t launch_reduce_contig(ome_dtype dt, const LoopArgs& a, bool vec, int64_t rchunk, int grid,
                                 cudaStream_t s) {
  cudaError_t e = cudaErrorInvalidValue;
  OME_DISPATCH(dt, ALG, e = launch_reduce_contig_t<ALG>(a, vec, rchunk, grid, s));
  return e;
}

// Contractions without summed labels (Hadamard and outer products,
// broadcast products, Repeat copies): y = sx * (x1 * x2 * ...) (+ sy * y),
// products left to right.  A block takes a segment of one row of y's fastest
// mode (mode 0); the row's offsets come from one mixed-radix decomposition
// per segment instead of one per element.  VEC: mode 0 has stride 1 in y and
// stride 0 or 1 in every input, and all row starts it touches are 16-byte
// aligned (checked by the host): 16-byte loads and stores, a stride-0 input
// read once per vector.
constexpr int MAP_U = 4;   // vectors per thread per segment (at most)
template <class A, int NIN, bool VEC>
__global__ void __launch_bounds__(256) k_map_rows(const __grid_constant__ LoopArgs a, int64_t nseg, int nu) {
  using T = typename A::T;
  constexpr int V = VEC ? (int)(16 / sizeof(T)) : 1;
  constexpr int NI = NIN > 0 ? NIN : MAXIN;
  const int nin = NIN > 0 ? NIN : a.nin;
  const T sx = scalar_as<T>(a.sx), sy = scalar_as<T>(a.sy);
  const int64_t e0 = a.ext[0];
  const int64_t items = (a.n_out / e0) * nseg;
  for (int64_t w = blockIdx.x; w < items; w += gridDim.x) {
    const int64_t r = w / nseg, sg = w - r * nseg;
    int64_t yoff = 0, off[NI];
#pragma unroll
    for (int k = 0; k < NI; ++k) off[k] = 0;
    int64_t q = r;
    for (int m = 1; m < a.nout; ++m) {
      const int64_t e = a.ext[m];
      const int64_t qq = q / e;
      const int64_t d = q - qq * e;
      q = qq;
      yoff += d * a.str[0][m];
#pragma unroll
      for (int k = 0; k < NI; ++k)
        if (k < nin) off[k] += d * a.str[1 + k][m];
    }
    T* yr = static_cast<T*>(a.y) + yoff;
    const int64_t ys = a.str[0][0];
#pragma unroll
    for (int u = 0; u < MAP_U; ++u) {
      const int64_t i = (sg * nu * 256 + (int64_t)u * 256 + threadIdx.x) * V;
      if (u >= nu || i >= e0) break;
      T p[V];
#pragma unroll
      for (int k = 0; k < NI; ++k) {
        if (k >= nin) break;
        const T* xk = static_cast<const T*>(a.x[k]) + off[k];
        const int64_t xs = a.str[1 + k][0];
        T v[V];
        if constexpr (VEC) {
          if (xs == 0) {
            const T c = xk[0];
#pragma unroll
            for (int j = 0; j < V; ++j) v[j] = c;
          } else {
            const uint4 w4 = __ldg(reinterpret_cast<const uint4*>(xk + i));
            memcpy(v, &w4, sizeof(w4));
          }
        } else {
          v[0] = xk[i * xs];
        }
#pragma unroll
        for (int j = 0; j < V; ++j) p[j] = k == 0 ? v[j] : A::mul(p[j], v[j]);
      }
      if constexpr (VEC) {
        T* yp = yr + i;
        T old[V];
        if (!a.sy_zero) {
          const uint4 w4 = *reinterpret_cast<const uint4*>(yp);
          memcpy(old, &w4, sizeof(w4));
        }
#pragma unroll
        for (int j = 0; j < V; ++j) p[j] = epilogue<A>(p[j], old + j, sx, sy, a.sy_zero, a.sx_one);
        uint4 w4;
        memcpy(&w4, p, sizeof(w4));
        *reinterpret_cast<uint4*>(yp) = w4;
      } else {
        T* yp = yr + i * ys;
        *yp = epilogue<A>(p[0], yp, sx, sy, a.sy_zero, a.sx_one);
      }
    }
  }
}

template <class A, bool VEC>
static void launch_map_rows_v(const LoopArgs& a, int64_t nseg, int nu, int grid, cudaStream_t s) {
  switch (a.nin) {
    case 1: k_map_rows<A, 1, VEC><<<grid, 256, 0, s>>>(a, nseg, nu); break;
    case 2: k_map_rows<A, 2, VEC><<<grid, 256, 0, s>>>(a, nseg, nu); break;
    case 3: k_map_rows<A, 3, VEC><<<grid, 256, 0, s>>>(a, nseg, nu); break;
    default: k_map_rows<A, 0, VEC><<<grid, 256, 0, s>>>(a, nseg, nu); break;
  }
  count_launch();
}

// VEC when the element size divides 16 bytes (at least 2 per vector), mode 0
// is contiguous in y and contiguous or broadcast in every input, its extent is
// a multiple of the vector and every row start it touches is 16-byte aligned.
static bool map_vec_ok(const LoopArgs& a, size_t es) {
  if (es > 8 || 16 % es != 0) return false;
  const int64_t V = (int64_t)(16 / es);
  if (a.str[0][0] != 1 || a.ext[0] % V != 0 || (uintptr_t)a.y % 16 != 0) return false;
  for (int m = 1; m < a.nout; ++m)
    if ((a.str[0][m] * (int64_t)es) % 16 != 0) return false;
  for (int k = 0; k < a.nin; ++k) {
    const int64_t xs = a.str[1 + k][0];
    if (xs == 0) continue;
    if (xs != 1 || (uintptr_t)a.x[k] % 16 != 0) return false;
    for (int m = 1; m < a.nout; ++m)
      if ((a.str[1 + k][m] * (int64_t)es) % 16 != 0) return false;
  }
  return true;
}

template <class A>
static cudaError_t launch_map_rows_t(const LoopArgs& a, int num_sms, cudaStream_t s) {
  const bool vec = map_vec_ok(a, sizeof(typename A::T));
  const int64_t V = vec ? (int64_t)(16 / sizeof(typename A::T)) : 1;
  const int64_t rows = a.n_out / a.ext[0];
  // segments of MAP_U vectors per thread, or of one when that leaves fewer
  // than 8 blocks per SM (short rows: a diagonal, a small tensor)
  int nu = MAP_U;
  if (rows * ((a.ext[0] + MAP_U * 256 * V - 1) / (MAP_U * 256 * V)) < (int64_t)num_sms * 8) nu = 1;
  const int64_t seg = (int64_t)nu * 256 * V;
  const int64_t nseg = (a.ext[0] + seg - 1) / seg;
  const int64_t items = rows * nseg;
  const int grid = (int)std::min<int64_t>(items, (int64_t)num_sms * 32);
  KernelTimer kt(s, "k_map_rows");
  if constexpr (sizeof(typename A::T) <= 8 && 16 % sizeof(typename A::T) == 0) {
    if (vec) launch_map_rows_v<A, true>(a, nseg, nu, grid, s);
    else launch_map_rows_v<A, false>(a, nseg, nu, grid, s);
  } else {
    launch_map_rows_v<A, false>(a, nseg, nu, grid, s);
  }
  return cudaGetLastError();
}

cudaError_t launch_map_rows(ome_dtype dt, const LoopArgs& a, int num_sms, cudaStream_t s) {
  if (a.n_out == 0) return cudaSuccess;
  cudaError_t e = cudaErrorInvalidValue;
  OME_DISPATCH(dt, ALG, e = launch_map_rows_t<ALG>(a, num_sms, s));
  return e;
}

template <class A>
static cudaError_t launch_loop_t(const LoopArgs& a, LoopMode mode, int grid, int block,
                                 cudaStream_t s) {
  if (mode == LOOP_THREAD) {
    switch (a.nin) {
      case 1: k_loop_thread<A, 1><<<grid, block, 0, s>>>(a); count_launch(); break;
      case 2: k_loop_thread<A, 2><<<grid, block, 0, s>>>(a); count_launch(); break;
      case 3: k_loop_thread<A, 3><<<grid, block, 0, s>>>(a); count_launch(); break;
      default: k_loop_thread<A, 0><<<grid, block, 0, s>>>(a); count_launch(); break;
    }
  } else {
    switch (a.nin) {
      case 1: k_loop_block<A, 1><<<grid, block, 0, s>>>(a); count_launch(); break;
      case 2: k_loop_block<A, 2><<<grid, block, 0, s>>>(a); count_launch(); break;
      case 3: k_loop_block<A, 3><<<grid, block, 0, s>>>(a); count_launch(); break;
      default: k_loop_block<A, 0><<<grid, block, 0, s>>>(a); count_launch(); break;
    }
  }
  return cudaGetLastError();
}

cudaError_t launch_loop(ome_dtype dt, const LoopArgs& a, LoopMode mode, int grid, int block,
                        cudaStream_t s) {
  cudaError_t e = cudaErrorInvalidValue;
  KernelTimer kt(s, mode == LOOP_BLOCK ? "k_loop_block" : "k_loop_thread");
  OME_DISPATCH(dt, ALG, e = launch_loop_t<ALG>(a, mode, grid, block, s));
  return e;
}

cudaError_t launch_loop_finish(ome_dtype dt, const LoopArgs& a, cudaStream_t s) {
  const int64_t nb = (a.n_out + 255) / 256;
  const int grid = (int)(nb < 4096 ? nb : 4096);
  cudaError_t e = cudaErrorInvalidValue;
  OME_DISPATCH(dt, ALG, e = launch_pdl(k_loop_finish<ALG>, dim3(grid), dim3(256), 0, s, a); count_launch());
  return e;
}

// ---------------------------------------------------------------------------
// permute / broadcast copy
// ---------------------------------------------------------------------------

// Tile transpose between y's fastest mode (mode 0) and x's fastest mode
// (tmode); every other mode is a batch index.  Tile = 32 (x-fast) x TY
// (y-fast).  Reads are coalesced along x's contiguous mode, writes along y's;
// each thread keeps TY/8 elements in flight.  256 threads = 32 x 8.
template <class A, int TY>
__global__ void __launch_bounds__(256) k_transpose(const __grid_constant__ PermArgs a) {
  using T = typename A::T;
  __shared__ T tile[TY][33];
  const T sx = scalar_as<T>(a.sx), sy = scalar_as<T>(a.sy);
  const int tmode = a.tmode;
  const int64_t e0 = a.ext[0], et = a.ext[tmode];
  const int64_t t0 = (e0 + TY - 1) / TY, tt = (et + 31) >> 5;
  const int64_t nbatch = a.n / (e0 * et);
  const int64_t ntiles = t0 * tt * nbatch;
  const int tx = threadIdx.x & 31, ty = threadIdx.x >> 5;
  const T* x = static_cast<const T*>(a.x);
  T* y = static_cast<T*>(a.y);
  const int64_t xs0 = a.xs[0], xst = a.xs[tmode], ys0 = a.ys[0], yst = a.ys[tmode];
  for (int64_t tid = blockIdx.x; tid < ntiles; tid += gridDim.x) {
    int64_t r = tid;
    const int64_t i0 = r % t0;
    r /= t0;
    const int64_t it = r % tt;
    r /= tt;
    int64_t xb = 0, yb = 0;
    for (int m = 1; m < a.nd; ++m) {
      if (m == tmode) continue;
      const int64_t e = a.ext[m];
      const int64_t q = r / e;
      const int64_t d = r - q * e;
      r = q;
      xb += d * a.xs[m];
      yb += d * a.ys[m];
    }
    const int64_t p = it * 32 + tx;
    const bool pin = p < et;
    const T* xp = x + xb + p * xst;
    T v[TY / 8];
#pragma unroll
    for (int k = 0; k < TY / 8; ++k) {
      const int64_t q = i0 * TY + ty + 8 * k;
      v[k] = (pin && q < e0) ? xp[q * xs0] : A::zero();
    }
#pragma unroll
    for (int k = 0; k < TY / 8; ++k) tile[ty + 8 * k][tx] = v[k];
    __syncthreads();
#pragma unroll
    for (int h = 0; h < TY / 32; ++h) {
      const int64_t q = i0 * TY + 32 * h + tx;
      if (q < e0) {
        T* yq = y + yb + q * ys0;
#pragma unroll
        for (int k = 0; k < 4; ++k) {
          const int64_t pp = it * 32 + ty + 8 * k;
          if (pp < et) {
            T* yp = yq + pp * yst;
            *yp = epilogue<A>(tile[32 * h + tx][ty + 8 * k], yp, sx, sy, a.sy_zero, a.sx_one);
          }
        }
      }
    }
    __syncthreads();
  }
}

// The same tile transpose when the element count and every offset of x and y
// fit in 31 bits: offsets in int32 and the per-tile decomposition of the tile
// index into (y-fast tile, x-fast tile, batch digits) by invariant-divisor
// multiplies instead of 64-bit divides (the decomposition otherwise costs more
// instructions than the 2048-element tile's loads and stores).
struct TransArgs {
  const void* x;
  void* y;
  Scalar sx, sy;
  int sy_zero, sx_one;
  int nb;                           // batch modes
  int32_t e0, et, xs0, xst, ys0, yst;
  uint32_t ntiles;
  FastDiv t0, tt;
  FastDiv bdiv[MAXM];
  int32_t bxs[MAXM], bys[MAXM];
  // k_transpose_v4 only: pa_shift > 0 when the tile's x-fast index runs over
  // two modes adjacent in x (x's contiguous mode of extent 2^pa_shift and the
  // next one), so that x rows are 256 bytes long although x's contiguous mode
  // is shorter; y row of index pp: (pp mod 2^pa_shift) * yst + (pp >> pa_shift) * ysb
  int32_t pa_shift, ysb;
};

template <class A, int TY>
__global__ void __launch_bounds__(256) k_transpose32(const __grid_constant__ TransArgs a) {
  using T = typename A::T;
  __shared__ T tile[TY][33];
  const T sx = scalar_as<T>(a.sx), sy = scalar_as<T>(a.sy);
  const int tx = threadIdx.x & 31, ty = threadIdx.x >> 5;
  const T* x = static_cast<const T*>(a.x);
  T* y = static_cast<T*>(a.y);
  for (uint32_t tid = blockIdx.x; tid < a.ntiles; tid += gridDim.x) {
    uint32_t r = tid;
    uint32_t q = fast_div(r, a.t0);
    const int32_t i0 = (int32_t)(r - q * a.t0.d);
    r = q;
    q = fast_div(r, a.tt);
    const int32_t it = (int32_t)(r - q * a.tt.d);
    r = q;
    int32_t xb = 0, yb = 0;
    for (int m = 0; m < a.nb; ++m) {
      q = fast_div(r, a.bdiv[m]);
      const int32_t d = (int32_t)(r - q * a.bdiv[m].d);
      r = q;
      xb += d * a.bxs[m];
      yb += d * a.bys[m];
    }
    const int32_t p = it * 32 + tx;
    const bool pin = p < a.et;
    const T* xp = x + xb + p * a.xst;
    const int32_t qb = i0 * TY + ty;
    T v[TY / 8];
#pragma unroll
    for (int k = 0; k < TY / 8; ++k) {
      const int32_t qq = qb + 8 * k;
      v[k] = (pin && qq < a.e0) ? xp[qq * a.xs0] : A::zero();
    }
#pragma unroll
    for (int k = 0; k < TY / 8; ++k) tile[ty + 8 * k][tx] = v[k];
    __syncthreads();
#pragma unroll
    for (int h = 0; h < TY / 32; ++h) {
      const int32_t qq = i0 * TY + 32 * h + tx;
      if (qq < a.e0) {
        T* yq = y + yb + qq * a.ys0;
#pragma unroll
        for (int k = 0; k < 4; ++k) {
          const int32_t pp = it * 32 + ty + 8 * k;
          if (pp < a.et) {
            T* yp = yq + pp * a.yst;
            *yp = epilogue<A>(tile[32 * h + tx][ty + 8 * k], yp, sx, sy, a.sy_zero, a.sx_one);
          }
        }
      }
    }
    __syncthreads();
  }
}

// 4-byte elements, both contiguous modes a multiple of 4 long and every other
// stride a multiple of 4 (16-byte aligned rows): the same transpose on 64 x 64
// tiles with 16-byte accesses on both sides -- each thread reads four float4
// along x's contiguous mode and writes four float4 along y's, a quarter of
// the memory instructions of k_transpose32 and twice its bytes in flight.
// Shared tile pitch 65 words: at most 2-way bank conflicts on either side.
template <class A, int PW>
__global__ void __launch_bounds__(256) k_transpose_v4(const __grid_constant__ TransArgs a) {
  using T = typename A::T;
  static_assert(sizeof(T) == 4, "4-byte elements");
  constexpr int QH = 64;                   // tile extent along y's contiguous mode
  constexpr int LC = PW / 4, LR = 256 / LC, LP = QH / LR;   // load: float4 columns, rows/pass, passes
  constexpr int SC = QH / 4, SR = 256 / SC, SP = PW / SR;   // store: the same for y's side
  __shared__ T tile[PW][QH + 1];           // [x-fast p][y-fast q]
  const T sx = scalar_as<T>(a.sx), sy = scalar_as<T>(a.sy);
  const int lc4 = (threadIdx.x % LC) * 4, lr = threadIdx.x / LC;
  const int sc4 = (threadIdx.x % SC) * 4, sr = threadIdx.x / SC;
  const T* x = static_cast<const T*>(a.x);
  T* y = static_cast<T*>(a.y);
  // tile tid -> y-fast tile i0, x-fast tile it, batch offsets xb / yb
  auto decode = [&](uint32_t tid, int32_t& i0, int32_t& it, int32_t& xb, int32_t& yb) {
    uint32_t rr = tid;
    uint32_t q = fast_div(rr, a.t0);
    i0 = (int32_t)(rr - q * a.t0.d);
    rr = q;
    q = fast_div(rr, a.tt);
    it = (int32_t)(rr - q * a.tt.d);
    rr = q;
    xb = 0;
    yb = 0;
    for (int m = 0; m < a.nb; ++m) {
      q = fast_div(rr, a.bdiv[m]);
      const int32_t d = (int32_t)(rr - q * a.bdiv[m].d);
      rr = q;
      xb += d * a.bxs[m];
      yb += d * a.bys[m];
    }
  };
  // load: rows = y-fast index (x stride xs0), float4 along x-fast p
  auto load = [&](int32_t i0, int32_t it, int32_t xb, uint4 (&v)[LP]) {
    const int32_t p = it * PW + lc4;
#pragma unroll
    for (int k = 0; k < LP; ++k) {
      const int32_t qq = i0 * QH + lr + LR * k;
      if (p < a.et && qq < a.e0) v[k] = __ldg(reinterpret_cast<const uint4*>(x + xb + qq * a.xs0 + p));
      else v[k] = make_uint4(0, 0, 0, 0);
    }
  };
  auto put = [&](const uint4 (&v)[LP]) {
#pragma unroll
    for (int k = 0; k < LP; ++k) {
      const T* e = reinterpret_cast<const T*>(&v[k]);
#pragma unroll
      for (int i = 0; i < 4; ++i) tile[lc4 + i][lr + LR * k] = e[i];
    }
  };
  // store: rows = x-fast index (y stride yst), float4 along y-fast q
  auto store = [&](int32_t i0, int32_t it, int32_t yb) {
    const int32_t qs = i0 * QH + sc4;
#pragma unroll
    for (int k = 0; k < SP; ++k) {
      const int32_t pp = it * PW + sr + SR * k;
      if (pp < a.et && qs < a.e0) {
        const int32_t row = a.pa_shift ? (pp & ((1 << a.pa_shift) - 1)) * a.yst + (pp >> a.pa_shift) * a.ysb
                                       : pp * a.yst;
        T* yp = y + yb + row + qs;
        T o[4];
#pragma unroll
        for (int i = 0; i < 4; ++i) o[i] = tile[sr + SR * k][sc4 + i];
        if (!(a.sx_one && a.sy_zero)) {
          T old[4];
          if (!a.sy_zero) {
            const uint4 w = *reinterpret_cast<const uint4*>(yp);
            memcpy(old, &w, 16);
          }
#pragma unroll
          for (int i = 0; i < 4; ++i) o[i] = epilogue<A>(o[i], old + i, sx, sy, a.sy_zero, a.sx_one);
        }
        uint4 w;
        memcpy(&w, o, 16);
        *reinterpret_cast<uint4*>(yp) = w;
      }
    }
  };
  if constexpr (PW == 64) {
    // 256-byte rows: the next tile's loads are issued before this tile's
    // stores, so a block always has reads in flight (6% faster on 2- to
    // 4-mode transposes than loading at the top of the loop)
    uint32_t tid = blockIdx.x;
    if (tid >= a.ntiles) return;
    int32_t i0, it, xb, yb;
    decode(tid, i0, it, xb, yb);
    uint4 v[LP];
    load(i0, it, xb, v);
    for (; tid < a.ntiles; tid += gridDim.x) {
      put(v);
      __syncthreads();
      const uint32_t nt = tid + gridDim.x;
      int32_t ni0 = 0, nit = 0, nxb = 0, nyb = 0;
      if (nt < a.ntiles) {
        decode(nt, ni0, nit, nxb, nyb);
        load(ni0, nit, nxb, v);
      }
      store(i0, it, yb);
      __syncthreads();
      i0 = ni0;
      it = nit;
      xb = nxb;
      yb = nyb;
    }
  } else {
    // 128-byte rows (a tile's 64 x rows each hit their own DRAM page): the
    // early loads cost 3% here, so each tile loads at the top of the loop
    for (uint32_t tid = blockIdx.x; tid < a.ntiles; tid += gridDim.x) {
      int32_t i0, it, xb, yb;
      decode(tid, i0, it, xb, yb);
      uint4 v[LP];
      load(i0, it, xb, v);
      put(v);
      __syncthreads();
      store(i0, it, yb);
      __syncthreads();
    }
  }
}

// Elementwise copy in y order (x's fastest mode is y's, or x is broadcast).
template <class A>
__global__ void __launch_bounds__(256) k_copy(const __grid_constant__ PermArgs a) {
  using T = typename A::T;
  const T sx = scalar_as<T>(a.sx), sy = scalar_as<T>(a.sy);
  const T* x = static_cast<const T*>(a.x);
  T* y = static_cast<T*>(a.y);
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < a.n;
       i += (int64_t)gridDim.x * blockDim.x) {
    int64_t r = i, xo = 0, yo = 0;
    for (int m = 0; m < a.nd; ++m) {
      const int64_t e = a.ext[m];
      const int64_t q = r / e;
      const int64_t d = r - q * e;
      r = q;
      xo += d * a.xs[m];
      yo += d * a.ys[m];
    }
    T* yp = y + yo;
    *yp = epilogue<A>(x[xo], yp, sx, sy, a.sy_zero, a.sx_one);
  }
}

// Contiguous 1-mode copy with 16-byte vectors (both unit stride, aligned).
template <class A>
__global__ void __launch_bounds__(256) k_copy_vec(const __grid_constant__ PermArgs a) {
  using T = typename A::T;
  constexpr int V = 16 / sizeof(T);
  const T sx = scalar_as<T>(a.sx), sy = scalar_as<T>(a.sy);
  const int64_t nv = a.n / V;
  const uint4* x = static_cast<const uint4*>(a.x);
  uint4* y = static_cast<uint4*>(a.y);
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < nv;
       i += (int64_t)gridDim.x * blockDim.x) {
    uint4 xv = x[i];
    if (!(a.sx_one && a.sy_zero)) {
      uint4 yv;
      if (!a.sy_zero) yv = y[i];
      T* xe = reinterpret_cast<T*>(&xv);
      T* ye = reinterpret_cast<T*>(&yv);
#pragma unroll
      for (int v = 0; v < V; ++v) xe[v] = epilogue<A>(xe[v], ye + v, sx, sy, a.sy_zero, a.sx_one);
    }
    y[i] = xv;
  }
  // tail
  const T* xs = static_cast<const T*>(a.x);
  T* ys = static_cast<T*>(a.y);
  for (int64_t i = nv * V + blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < a.n;
       i += (int64_t)gridDim.x * blockDim.x) {
    ys[i] = epilogue<A>(xs[i], ys + i, sx, sy, a.sy_zero, a.sx_one);
  }
}

template <class A>
static cudaError_t launch_perm_t(const PermArgs& a, int num_sms, cudaStream_t s) {
  using T = typename A::T;
  if (a.n == 0) return cudaSuccess;
  const int maxgrid = num_sms * 16;
  if (a.tmode > 0) {
    constexpr int TY = sizeof(T) <= 4 ? 64 : 32;
    const int64_t tiles = ((a.ext[0] + TY - 1) / TY) * ((a.ext[a.tmode] + 31) / 32) *
                          (a.n / (a.ext[0] * a.ext[a.tmode]));
    const int grid = (int)(tiles < maxgrid ? tiles : maxgrid);
    if (a.n < ((int64_t)1 << 31) && tiles < ((int64_t)1 << 31) &&
        max_offset(a.nd, a.ext, a.xs) < ((int64_t)1 << 31) &&
        max_offset(a.nd, a.ext, a.ys) < ((int64_t)1 << 31)) {
      TransArgs t;
      t.x = a.x; t.y = a.y; t.sx = a.sx; t.sy = a.sy; t.sy_zero = a.sy_zero; t.sx_one = a.sx_one;
      t.e0 = (int32_t)a.ext[0]; t.et = (int32_t)a.ext[a.tmode];
      t.xs0 = (int32_t)a.xs[0]; t.xst = (int32_t)a.xs[a.tmode];
      t.ys0 = (int32_t)a.ys[0]; t.yst = (int32_t)a.ys[a.tmode];
      t.ntiles = (uint32_t)tiles;
      t.t0 = make_fastdiv((uint32_t)((a.ext[0] + TY - 1) / TY));
      t.tt = make_fastdiv((uint32_t)((a.ext[a.tmode] + 31) / 32));
      t.nb = 0;
      for (int m = 1; m < a.nd; ++m) {
        if (m == a.tmode) continue;
        t.bdiv[t.nb] = make_fastdiv((uint32_t)a.ext[m]);
        t.bxs[t.nb] = (int32_t)a.xs[m];
        t.bys[t.nb] = (int32_t)a.ys[m];
        ++t.nb;
      }
      bool v4 = sizeof(T) == 4 && a.xs[a.tmode] == 1 && a.ys[0] == 1 && a.ext[0] % 4 == 0 &&
                a.ext[a.tmode] % 4 == 0 && (uintptr_t)a.x % 16 == 0 && (uintptr_t)a.y % 16 == 0 &&
                a.xs[0] % 4 == 0 && a.ys[a.tmode] % 4 == 0;
      for (int m = 0; m < t.nb && v4; ++m) v4 = t.bxs[m] % 4 == 0 && t.bys[m] % 4 == 0;
      t.pa_shift = 0;
      t.ysb = 0;
      if constexpr (sizeof(T) == 4) {
        if (v4) {
          // x's contiguous mode of 8, 16 or 32 elements followed in x by a
          // batch mode (x stride = its extent): tile over both, 256-byte x rows
          const int64_t ec = a.ext[a.tmode];
          int merge = -1;
          if (ec >= 8 && ec <= 32 && (ec & (ec - 1)) == 0)
            for (int m = 0; m < t.nb; ++m)
              if (t.bxs[m] == ec && ec * (int64_t)t.bdiv[m].d >= 64 && t.bys[m] % 4 == 0) {
                merge = m;
                break;
              }
          if (merge >= 0) {
            t.pa_shift = ec == 8 ? 3 : ec == 16 ? 4 : 5;
            t.ysb = t.bys[merge];
            t.et = (int32_t)(ec * t.bdiv[merge].d);
            for (int m = merge; m + 1 < t.nb; ++m) {
              t.bdiv[m] = t.bdiv[m + 1];
              t.bxs[m] = t.bxs[m + 1];
              t.bys[m] = t.bys[m + 1];
            }
            --t.nb;
          }
          const int64_t et = t.et;
          const int pw = et <= 32 ? 32 : 64;   // tile width along x's contiguous run
          const int64_t tiles4 = ((a.ext[0] + 63) / 64) * ((et + pw - 1) / pw) * (a.n / (a.ext[0] * et));
          t.ntiles = (uint32_t)tiles4;
          t.t0 = make_fastdiv((uint32_t)((a.ext[0] + 63) / 64));
          t.tt = make_fastdiv((uint32_t)((et + pw - 1) / pw));
          const int grid4 = (int)(tiles4 < maxgrid ? tiles4 : maxgrid);
          KernelTimer kt(s, "k_transpose_v4");
          if (pw == 32) k_transpose_v4<A, 32><<<grid4, 256, 0, s>>>(t);
          else k_transpose_v4<A, 64><<<grid4, 256, 0, s>>>(t);
          count_launch();
          return cudaGetLastError();
        }
      }
      KernelTimer kt(s, "k_transpose32");
      k_transpose32<A, TY><<<grid, 256, 0, s>>>(t);
    } else {
      KernelTimer kt(s, "k_transpose");
      k_transpose<A, TY><<<grid, 256, 0, s>>>(a);
    }
    count_launch();
  } else if (a.nd == 1 && a.xs[0] == 1 && a.ys[0] == 1 && sizeof(T) <= 16 && 16 % sizeof(T) == 0 &&
             ((uintptr_t)a.x % 16) == 0 && ((uintptr_t)a.y % 16) == 0) {
    const int64_t nb = (a.n / (16 / sizeof(T)) + 255) / 256;
    const int grid = (int)(nb < 1 ? 1 : (nb < maxgrid ? nb : maxgrid));
    KernelTimer kt(s, "k_copy_vec");
    k_copy_vec<A><<<grid, 256, 0, s>>>(a); count_launch();
  } else if (a.nd >= 1) {
    // general copy / broadcast (Repeat): the row kernel over y's fastest mode
    LoopArgs l;
    memset(&l, 0, sizeof(l));
    l.x[0] = a.x;
    l.y = a.y;
    l.nin = 1;
    l.nout = a.nd;
    l.ninner = 0;
    l.n_out = a.n;
    l.n_in = 1;
    for (int m = 0; m < a.nd; ++m) {
      l.ext[m] = a.ext[m];
      l.str[0][m] = a.ys[m];
      l.str[1][m] = a.xs[m];
    }
    l.sx = a.sx;
    l.sy = a.sy;
    l.sy_zero = a.sy_zero;
    l.sx_one = a.sx_one;
    return launch_map_rows_t<A>(l, num_sms, s);
  } else {
    const int64_t nb = (a.n + 255) / 256;
    const int grid = (int)(nb < maxgrid ? nb : maxgrid);
    KernelTimer kt(s, "k_copy");
    k_copy<A><<<grid, 256, 0, s>>>(a); count_launch();
  }
  return cudaGetLastError();
}

cudaError_t launch_perm(ome_dtype dt, const PermArgs& a, int num_sms, cudaStream_t s) {
  cudaError_t e = cudaErrorInvalidValue;
  OME_DISPATCH(dt, ALG, e = launch_perm_t<ALG>(a, num_sms, s));
  return e;
}

// ---------------------------------------------------------------------------
// scale pre-pass (outputs with repeated labels)
// ---------------------------------------------------------------------------

template <class A>
__global__ void __launch_bounds__(256) k_scale(const __grid_constant__ PermArgs a) {
  using T = typename A::T;
  const T sy = scalar_as<T>(a.sy);
  T* y = static_cast<T*>(a.y);
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < a.n;
       i += (int64_t)gridDim.x * blockDim.x) {
    int64_t r = i, yo = 0;
    for (int m = 0; m < a.nd; ++m) {
      const int64_t e = a.ext[m];
      const int64_t q = r / e;
      yo += (r - q * e) * a.ys[m];
      r = q;
    }
    y[yo] = a.sy_zero ? A::zero() : A::mul(sy, y[yo]);
  }
}

cudaError_t launch_scale(ome_dtype dt, void* y, int nd, const int64_t* ext, const int64_t* str,
                         const Scalar& sy, int sy_zero, int num_sms, cudaStream_t s) {
  PermArgs a;
  memset(&a, 0, sizeof(a));
  a.y = y;
  a.nd = nd;
  a.n = 1;
  for (int m = 0; m < nd; ++m) {
    a.ext[m] = ext[m];
    a.ys[m] = str[m];
    a.n *= ext[m];
  }
  a.sy = sy;
  a.sy_zero = sy_zero;
  if (a.n == 0) return cudaSuccess;
  const int64_t nb = (a.n + 255) / 256;
  const int maxgrid = num_sms * 16;
  const int grid = (int)(nb < maxgrid ? nb : maxgrid);
  cudaError_t e = cudaErrorInvalidValue;
  OME_DISPATCH(dt, ALG, k_scale<ALG><<<grid, 256, 0, s>>>(a); count_launch(); e = cudaGetLastError());
  return e;
}

// ---------------------------------------------------------------------------
// FP64 cross-slice accumulation
// ---------------------------------------------------------------------------

template <class T, class W>
__global__ void __launch_bounds__(256) k_acc64(W* acc, const T* src, int64_t n) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x)
    acc[i] += (W)src[i];
}
__global__ void __launch_bounds__(256) k_acc64_c(double2* acc, const cf32* src, int64_t n) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x) {
    acc[i].x += (double)src[i].re;
    acc[i].y += (double)src[i].im;
  }
}

cudaError_t launch_acc64(ome_dtype dt, void* acc, const void* src, int64_t n, cudaStream_t s) {
  const int64_t nb = (n + 255) / 256;
  const int grid = (int)(nb < 2048 ? (nb < 1 ? 1 : nb) : 2048);
  switch (dt) {
    case OME_F32: k_acc64<float, double><<<grid, 256, 0, s>>>((double*)acc, (const float*)src, n); count_launch(); break;
    case OME_F64: k_acc64<double, double><<<grid, 256, 0, s>>>((double*)acc, (const double*)src, n); count_launch(); break;
    case OME_C32: k_acc64_c<<<grid, 256, 0, s>>>((double2*)acc, (const cf32*)src, n); count_launch(); break;
    default: return cudaErrorInvalidValue;
  }
  return cudaGetLastError();
}

template <class A, class W>
__global__ void __launch_bounds__(256) k_acc64_store(typename A::T* y, const W* acc, int64_t n,
                                                     Scalar sxs, Scalar sys, int sy_zero) {
  using T = typename A::T;
  const T sx = scalar_as<T>(sxs), sy = scalar_as<T>(sys);
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x) {
    T f;
    if constexpr (sizeof(W) == 16) {
      f.re = (decltype(f.re))acc[i].x;
      f.im = (decltype(f.im))acc[i].y;
    } else {
      f = (T)acc[i];
    }
    y[i] = epilogue<A>(f, y + i, sx, sy, sy_zero, false);
  }
}

cudaError_t launch_acc64_store(ome_dtype dt, void* y, const void* acc, int64_t n, const Scalar& sx,
                               const Scalar& sy, int sy_zero, cudaStream_t s) {
  const int64_t nb = (n + 255) / 256;
  const int grid = (int)(nb < 2048 ? (nb < 1 ? 1 : nb) : 2048);
  switch (dt) {
    case OME_F32:
      k_acc64_store<AlgF32, double><<<grid, 256, 0, s>>>((float*)y, (const double*)acc, n, sx, sy, sy_zero); count_launch();
      break;
    case OME_F64:
      k_acc64_store<AlgF64, double><<<grid, 256, 0, s>>>((double*)y, (const double*)acc, n, sx, sy, sy_zero); count_launch();
      break;
    case OME_C32:
      k_acc64_store<AlgC32, double2><<<grid, 256, 0, s>>>((cf32*)y, (const double2*)acc, n, sx, sy, sy_zero); count_launch();
      break;
    default: return cudaErrorInvalidValue;
  }
  return cudaGetLastError();
}

template <class W, class T>
__global__ void __launch_bounds__(256) k_acc64_strided(char* acc, const T* src, PermArgs a) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < a.n;
       i += (int64_t)gridDim.x * blockDim.x) {
    int64_t r = i, yo = 0;
    for (int m = 0; m < a.nd; ++m) {
      const int64_t e = a.ext[m];
      const int64_t q = r / e;
      yo += (r - q * e) * a.ys[m];
      r = q;
    }
    W* w = reinterpret_cast<W*>(acc) + yo;
    if constexpr (sizeof(W) == 16) {
      w->x += (double)src[i].re;
      w->y += (double)src[i].im;
    } else {
      *w += (double)src[i];
    }
  }
}

cudaError_t launch_acc64_strided(ome_dtype dt, void* acc, const void* src, int nd, const int64_t* ext,
                                 const int64_t* acc_str, cudaStream_t s) {
  PermArgs a;
  memset(&a, 0, sizeof(a));
  a.nd = nd;
  a.n = 1;
  for (int m = 0; m < nd; ++m) {
    a.ext[m] = ext[m];
    a.ys[m] = acc_str[m];
    a.n *= ext[m];
  }
  if (a.n == 0) return cudaSuccess;
  const int64_t nb = (a.n + 255) / 256;
  const int grid = (int)(nb < 2048 ? nb : 2048);
  switch (dt) {
    case OME_F32: k_acc64_strided<double, float><<<grid, 256, 0, s>>>((char*)acc, (const float*)src, a); count_launch(); break;
    case OME_F64: k_acc64_strided<double, double><<<grid, 256, 0, s>>>((char*)acc, (const double*)src, a); count_launch(); break;
    case OME_C32: k_acc64_strided<double2, cf32><<<grid, 256, 0, s>>>((char*)acc, (const cf32*)src, a); count_launch(); break;
    default: return cudaErrorInvalidValue;
  }
  return cudaGetLastError();
}

template <class T>
__global__ void __launch_bounds__(256) k_conj(T* x, int64_t n) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x)
    x[i].im = -x[i].im;
}

cudaError_t launch_conj(ome_dtype dt, void* x, int64_t n, cudaStream_t s) {
  if (n == 0) return cudaSuccess;
  const int64_t nb = (n + 255) / 256;
  const int grid = (int)(nb < 2048 ? nb : 2048);
  if (dt == OME_C32) {
    k_conj<cf32><<<grid, 256, 0, s>>>((cf32*)x, n);
  } else if (dt == OME_C64) {
    k_conj<cf64><<<grid, 256, 0, s>>>((cf64*)x, n);
  } else {
    return cudaSuccess;
  }
  count_launch();
  return cudaGetLastError();
}

template <class A>
__global__ void __launch_bounds__(256) k_fill_one(typename A::T* x, int64_t n) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x)
    x[i] = A::one();
}

cudaError_t launch_fill_one(ome_dtype dt, void* x, int64_t n, cudaStream_t s) {
  if (n == 0) return cudaSuccess;
  const int64_t nb = (n + 255) / 256;
  const int grid = (int)(nb < 2048 ? nb : 2048);
  cudaError_t e = cudaErrorInvalidValue;
  OME_DISPATCH(dt, ALG, k_fill_one<ALG><<<grid, 256, 0, s>>>((typename ALG::T*)x, n); count_launch(); e = cudaGetLastError());
  return e;
}

}  // namespace ome
