// ome_reduce_noalloc: the two-pass split reduction (k_loop_block writing
// per-split partial sums, then k_loop_finish adding them in a fixed order)
// with its partial sums kept in a fixed array inside this library instead of
// a context workspace, so that the call allocates no device memory.
//
// Who needs it: callers whose device memory belongs entirely to their own
// allocator -- CUDA.jl's memory pool, or a serving process that has carved a
// fixed HBM budget into its own arena -- and which therefore cannot let a
// library call cudaMalloc / cudaFree (those calls also synchronise the
// device, which such callers avoid on their hot path).
//
// The array holds OME_NOALLOC_SCRATCH_BYTES; every GPU that loads the library
// keeps it until the process exits.  In host code the array's name is only a
// host-side stand-in: the device address is looked up once per device with
// cudaGetSymbolAddress, with that device current, by the first call made on
// that device (make that first call before any stream capture).  The address
// is cached for the life of the process: after cudaDeviceReset the library's
// module is loaded again at another address, so this entry point must not be
// used across a cudaDeviceReset of a device it has already run on.  All calls
// on a device share the array and it keeps the last call's contents; the
// first pass overwrites every partial the second pass reads, so nothing has
// to be cleared, but calls that overlap on the GPU (several streams, or
// several host threads) race on it and must be serialised by the caller.
#include <string.h>
#include <algorithm>
#include <mutex>
#include <vector>

#include "dispatch.h"

static __device__ __align__(256) unsigned char g_noalloc_scratch[OME_NOALLOC_SCRATCH_BYTES];

namespace {

std::mutex g_noalloc_mu;
void* g_noalloc_addr[128] = {nullptr};
int g_noalloc_sms[128] = {0};

// Device address of the scratch array for the current device (set-up on first use).
int noalloc_setup(int dev, void** addr, int* sms) {
  if (dev < 0 || dev >= 128) return ome::set_err(OME_UNSUPPORTED, "device index %d out of range", dev);
  std::lock_guard<std::mutex> lk(g_noalloc_mu);
  if (!g_noalloc_addr[dev]) {
    void* p = nullptr;
    cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (e != cudaSuccess) return ome::cuda_err(e, "cudaGetSymbolAddress(no-alloc scratch)");
    int n = 0;
    e = cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev);
    if (e != cudaSuccess) return ome::cuda_err(e, "cudaDeviceGetAttribute");
    g_noalloc_addr[dev] = p;
    g_noalloc_sms[dev] = n;
  }
  *addr = g_noalloc_addr[dev];
  *sms = g_noalloc_sms[dev];
  return OME_OK;
}

int find(const ome::HView& v, int32_t l) {
  for (int d = 0; d < v.nd; ++d)
    if (v.lab[d] == l) return d;
  return -1;
}

}  // namespace

extern "C" int ome_reduce_noalloc(void* stream, ome_dtype dtype, const ome_tensor* x, const ome_tensor* y,
                                  const void* sxp, const void* syp) {
  using namespace ome;
  if (!x || !y || !sxp || !syp) return set_err(OME_INVALID_ARGUMENT, "NULL argument");
  if ((int)dtype < 0 || (int)dtype > OME_TROP_F64) return set_err(OME_INVALID_ARGUMENT, "unknown dtype %d", (int)dtype);
  HView xv, yv, xu, yu;
  int rc = view_from_tensor(*x, xv, "input");
  if (rc) return rc;
  rc = view_from_tensor(*y, yv, "output");
  if (rc) return rc;
  rc = unique_view(xv, xu);
  if (rc) return rc;
  rc = unique_view(yv, yu);
  if (rc) return rc;
  if (yu.nd != yv.nd) return set_err(OME_INVALID_ARGUMENT, "repeated output labels are not supported here");
  for (int d = 0; d < yu.nd; ++d) {
    const int k = find(xu, yu.lab[d]);
    if (k < 0) return set_err(OME_INVALID_ARGUMENT, "output label %d is not an input label", yu.lab[d]);
    if (xu.ext[k] != yu.ext[d])
      return set_err(OME_DIMENSION_MISMATCH, "label %d: input extent %lld, output extent %lld", yu.lab[d],
                     (long long)xu.ext[k], (long long)yu.ext[d]);
  }
  int dev = 0;
  cudaError_t ce = cudaGetDevice(&dev);
  if (ce != cudaSuccess) return cuda_err(ce, "cudaGetDevice");
  void* scratch = nullptr;
  int sms = 0;
  rc = noalloc_setup(dev, &scratch, &sms);
  if (rc) return rc;

  // modes: output labels (y order), then summed labels of x
  LoopArgs a;
  memset(&a, 0, sizeof(a));
  int64_t n_out = 1, n_in = 1;
  int no = 0;
  for (int d = 0; d < yu.nd; ++d) {
    if (yu.ext[d] == 1) continue;
    if (no >= MAXM) return set_err(OME_UNSUPPORTED, "too many output modes");
    a.ext[no] = yu.ext[d];
    a.str[0][no] = yu.str[d];
    a.str[1][no] = xu.str[find(xu, yu.lab[d])];
    n_out *= yu.ext[d];
    ++no;
  }
  int ni = 0;
  for (int d = 0; d < xu.nd; ++d) {
    if (find(yu, xu.lab[d]) >= 0) continue;
    n_in *= xu.ext[d];
    if (xu.ext[d] == 1) continue;
    if (no + ni >= MAXM) return set_err(OME_UNSUPPORTED, "too many modes");
    a.ext[no + ni] = xu.ext[d];
    a.str[0][no + ni] = 0;
    a.str[1][no + ni] = xu.str[d];
    ++ni;
  }
  if (n_out == 0) return OME_OK;
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  if (n_in == 0) {
    // a summed label of extent 0: the sum is the algebra's zero, so
    // y <- sy*y (zero when sy is zero); no partial sums are needed
    const Scalar sy = scalar_from(dtype, syp);
    return cuda_err(launch_scale(dtype, yu.data, yu.nd, yu.ext, yu.str, sy, scalar_is_zero(dtype, sy) ? 1 : 0, sms, s),
                    "no-alloc reduction (empty sum)");
  }
  const size_t es = dtype_size(dtype);
  const size_t cap = OME_NOALLOC_SCRATCH_BYTES;
  if ((size_t)n_out * 2 * es > cap)
    return set_err(OME_UNSUPPORTED,
                   "ome_reduce_noalloc: %lld outputs need %zu bytes of partial sums; the fixed scratch holds %zu "
                   "bytes (at most %zu outputs of this type)",
                   (long long)n_out, (size_t)n_out * 2 * es, cap, cap / (2 * es));
  // at least two splits per output (so that the reduction always goes
  // through the scratch), about 8 blocks per SM in total
  int64_t nsplit = std::max<int64_t>(2, ((int64_t)sms * 8 + n_out - 1) / n_out);
  nsplit = std::min<int64_t>(nsplit, std::max<int64_t>(2, n_in / 512));
  nsplit = std::min<int64_t>(nsplit, (int64_t)(cap / ((size_t)n_out * es)));
  a.x[0] = xu.data;
  a.y = yu.data;
  a.partial = scratch;
  a.nin = 1;
  a.nout = no;
  a.ninner = ni;
  a.n_out = n_out;
  a.n_in = n_in;
  a.nsplit = (int)nsplit;
  a.sx = scalar_from(dtype, sxp);
  a.sy = scalar_from(dtype, syp);
  a.sy_zero = scalar_is_zero(dtype, a.sy);
  a.sx_one = scalar_is_one(dtype, a.sx);
  const int block = 256;
  int64_t step = (int64_t)block * nsplit;
  for (int m = 0; m < ni; ++m) {
    if (m == ni - 1) {
      a.stepdig[m] = (int32_t)std::min<int64_t>(step, 0x7fffffff);
    } else {
      a.stepdig[m] = (int32_t)(step % a.ext[no + m]);
      step /= a.ext[no + m];
    }
  }
  const int grid = (int)std::min<int64_t>(n_out * nsplit, (int64_t)sms * 32);
  rc = cuda_err(launch_loop(dtype, a, LOOP_BLOCK, grid, block, s), "no-alloc reduction");
  if (rc) return rc;
  return cuda_err(launch_loop_finish(dtype, a, s), "no-alloc reduction finish");
}
