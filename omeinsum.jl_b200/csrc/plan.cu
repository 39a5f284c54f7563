// Contraction-tree plans: NestedEinsum / SlicedEinsum execution and
// cost_and_gradient on the device.
//
// Reference behaviour restated:
//  * post-order evaluation of a NestedEinsum (src/einsequence.jl:270-287;
//    GPU form ext/CUDAExt.jl:121-147); intermediates live in the context's
//    workspace at offsets planned from their lifetimes instead of per-node
//    allocations and unsafe_free! (active_free);
//  * SlicedEinsum (src/slicing.jl:104-137): slices in CartesianIndices order
//    over the sliced labels (first label fastest, :37-71); each slice's leaves
//    are strided VIEWS of the inputs (no take_slice copies, :78-85); the
//    cross-slice sum is accumulated in FP64 for F32/F64/C32 (the reference
//    accumulates in the eltype); other eltypes accumulate in place;
//  * cost_and_gradient (src/bp.jl:122-130): cached forward pass, then
//    einsum_grad per child (src/autodiff.jl:24-30: conj(dy) replaces the
//    child's input, the child's labels become the output, result conjugated).
#include <string.h>
#include <algorithm>
#include <cmath>
#include <map>
#include <vector>

#include "dispatch.h"

using namespace ome;

namespace {

struct PNode {
  std::vector<int> args;           // >= 0 node, < 0 input (-r-1)
  std::vector<int32_t> iy;         // output labels
  std::vector<int32_t> iy_s;       // output labels without sliced labels
  int64_t numel_s = 1, numel = 1;  // output elements (sliced / full)
  size_t off_fwd = 0;              // workspace offset in sliced forward
  size_t off_keep = 0;             // offset of the forward value when all are kept
  size_t off_grad = 0;             // offset of the gradient buffer
  int parent = -1;
};

}  // namespace

struct ome_plan {
  ome_dtype dt;
  int prec;
  int ninputs;
  std::vector<std::vector<int32_t>> in_labels;
  std::map<int32_t, int64_t> ext;
  std::vector<int32_t> sliced;
  int64_t nslices = 1;
  std::vector<PNode> nodes;
  bool acc64 = false;
  size_t acc_off = 0, tmp_off = 0;  // FP64 accumulator and root temporary (sliced)
  size_t dy_off = 0;                        // root cotangent buffer (gradient)
  size_t arena_bytes = 0, grad_arena = 0;  // planned buffers (forward / gradient)
  size_t fwd_bytes = 0, grad_bytes = 0;     // plus per-node dispatch scratch
  size_t esize = 0;
};

namespace {

struct Interval {
  size_t off, size;
};

// First-fit offset allocator over live intervals (256-byte aligned).
struct Arena {
  std::vector<std::pair<size_t, size_t>> live;  // (off, size)
  size_t peak = 0;
  size_t alloc(size_t bytes) {
    bytes = (bytes + 255) & ~(size_t)255;
    if (bytes == 0) bytes = 256;
    std::sort(live.begin(), live.end());
    size_t off = 0;
    for (auto& p : live) {
      if (p.first >= off + bytes) break;
      off = std::max(off, p.first + p.second);
    }
    live.push_back({off, bytes});
    peak = std::max(peak, off + bytes);
    return off;
  }
  void release(size_t off) {
    for (size_t i = 0; i < live.size(); ++i)
      if (live[i].first == off) {
        live.erase(live.begin() + i);
        return;
      }
  }
};

bool contains(const std::vector<int32_t>& v, int32_t l) { return std::find(v.begin(), v.end(), l) != v.end(); }

// Column-major contiguous view with labels `labs`; labels in `drop` are
// fixed at index `fix` (their stride folded into the base offset) and removed.
HView make_view(const ome_plan* p, char* base, const std::vector<int32_t>& labs, const std::vector<int32_t>& drop,
                const std::vector<int64_t>& fix) {
  HView v;
  v.data = base;
  v.nd = 0;
  int64_t s = 1;
  int64_t off = 0;
  for (int32_t l : labs) {
    const int64_t e = p->ext.at(l);
    auto it = std::find(drop.begin(), drop.end(), l);
    if (it != drop.end()) {
      off += fix[it - drop.begin()] * s;
    } else {
      v.lab[v.nd] = l;
      v.ext[v.nd] = e;
      v.str[v.nd] = s;
      v.nd++;
    }
    s *= e;
  }
  v.data = base + off * (int64_t)p->esize;
  return v;
}

std::vector<int32_t> child_labels(const ome_plan* p, int ref, bool sliced) {
  if (ref >= 0) return sliced ? p->nodes[ref].iy_s : p->nodes[ref].iy;
  const auto& l = p->in_labels[-ref - 1];
  if (!sliced) return l;
  std::vector<int32_t> r;
  for (int32_t x : l)
    if (!contains(p->sliced, x)) r.push_back(x);
  return r;
}

// Memory order of intermediates.  An intermediate's label order is internal to
// the plan (only the root's is the caller's), so each binary node lays out its
// children for itself, as analyze_binary's canonical orders do
// (src/einsum.jl:139-185; OMEinsumContractionOrders' optimize_permute):
// x1 = [outer1 (output order), inner, batch (output order)],
// x2 = [inner, outer2 (output order), batch (output order)], with one inner
// order shared by both (a leaf child's, if either child is a leaf).  Mode
// groups of the strided GEMM then merge into one or a few modes.  Top-down:
// a parent's order is final before its children are arranged.
void canonical_orders(ome_plan* p) {
  const int nn = (int)p->nodes.size();
  for (int j = nn - 1; j >= 0; --j) {
    PNode& n = p->nodes[j];
    if (n.args.size() != 2) continue;
    const int r1 = n.args[0], r2 = n.args[1];
    const std::vector<int32_t> L1 = r1 >= 0 ? p->nodes[r1].iy : p->in_labels[-r1 - 1];
    const std::vector<int32_t> L2 = r2 >= 0 ? p->nodes[r2].iy : p->in_labels[-r2 - 1];
    const std::vector<int32_t>& y = n.iy;
    std::vector<int32_t> o1, o2, batch, inner, d1, d2;
    for (int32_t l : y) {
      const bool a = contains(L1, l), b = contains(L2, l);
      if (a && b) batch.push_back(l);
      else if (a) o1.push_back(l);
      else if (b) o2.push_back(l);
    }
    const std::vector<int32_t>& ref = (r1 < 0 || r2 >= 0) ? L1 : L2;  // a leaf's order if there is one
    for (int32_t l : ref)
      if (contains(L1, l) && contains(L2, l) && !contains(y, l)) inner.push_back(l);
    for (int32_t l : L1)
      if (!contains(L2, l) && !contains(y, l)) d1.push_back(l);
    for (int32_t l : L2)
      if (!contains(L1, l) && !contains(y, l)) d2.push_back(l);
    auto rebuild = [&](int r, const std::vector<std::vector<int32_t>>& parts) {
      std::vector<int32_t> v;
      for (auto& q : parts) v.insert(v.end(), q.begin(), q.end());
      PNode& c = p->nodes[r];
      if (v.size() != c.iy.size()) return;  // not a permutation of the child's labels: keep
      c.iy = v;
      c.iy_s.clear();
      for (int32_t l : v)
        if (!contains(p->sliced, l)) c.iy_s.push_back(l);
    };
    if (r1 >= 0) rebuild(r1, {o1, inner, batch, d1});
    if (r2 >= 0) rebuild(r2, {inner, o2, batch, d2});
  }
}

}  // namespace

extern "C" {

int ome_plan_create(ome_ctx* ctx, ome_dtype dtype, int32_t ninputs, const int32_t* input_nlabels,
                    const int32_t* input_labels, int32_t nnodes, const int32_t* node_nargs, const int32_t* node_args,
                    const int32_t* node_niy, const int32_t* node_iy, int32_t nlabels, const int32_t* label_ids,
                    const int64_t* label_extents, int32_t nsliced, const int32_t* sliced_labels, int32_t prec,
                    ome_plan** out) {
  (void)ctx;
  if (!out) return set_err(OME_INVALID_ARGUMENT, "out is NULL");
  *out = nullptr;
  if ((int)dtype < 0 || (int)dtype > OME_TROP_F64) return set_err(OME_INVALID_ARGUMENT, "unknown dtype");
  if (ninputs < 1 || nnodes < 1) return set_err(OME_INVALID_ARGUMENT, "empty tree");
  auto p = new ome_plan();
  p->dt = dtype;
  p->prec = prec;
  p->esize = dtype_size(dtype);
  p->ninputs = ninputs;
  for (int i = 0; i < nlabels; ++i) {
    if (label_extents[i] < 0) {
      delete p;
      return set_err(OME_INVALID_ARGUMENT, "negative extent for label %d", label_ids[i]);
    }
    p->ext[label_ids[i]] = label_extents[i];
  }
  int pos = 0;
  for (int t = 0; t < ninputs; ++t) {
    std::vector<int32_t> l(input_labels + pos, input_labels + pos + input_nlabels[t]);
    pos += input_nlabels[t];
    for (int32_t x : l)
      if (!p->ext.count(x)) {
        delete p;
        return set_err(OME_INVALID_ARGUMENT, "label %d of input %d has no extent", x, t);
      }
    p->in_labels.push_back(l);
  }
  for (int i = 0; i < nsliced; ++i) {
    if (!p->ext.count(sliced_labels[i])) {
      delete p;
      return set_err(OME_INVALID_ARGUMENT, "sliced label %d has no extent", sliced_labels[i]);
    }
    p->sliced.push_back(sliced_labels[i]);
    p->nslices *= p->ext[sliced_labels[i]];
  }
  std::vector<int> input_used(ninputs, 0);
  int apos = 0, ypos = 0;
  p->nodes.resize(nnodes);
  for (int j = 0; j < nnodes; ++j) {
    PNode& n = p->nodes[j];
    for (int a = 0; a < node_nargs[j]; ++a) {
      const int r = node_args[apos++];
      if (r >= 0) {
        if (r >= j || p->nodes[r].parent != -1) {
          delete p;
          return set_err(OME_INVALID_ARGUMENT, "node %d: child %d is not an earlier unused node", j, r);
        }
        p->nodes[r].parent = j;
      } else {
        const int t = -r - 1;
        if (t >= ninputs || input_used[t]) {
          delete p;
          return set_err(OME_INVALID_ARGUMENT, "node %d: bad or repeated input %d", j, t);
        }
        input_used[t] = 1;
      }
      n.args.push_back(r);
    }
    if (n.args.empty()) {
      delete p;
      return set_err(OME_INVALID_ARGUMENT, "node %d has no children", j);
    }
    for (int a = 0; a < node_niy[j]; ++a) {
      const int32_t l = node_iy[ypos++];
      if (!p->ext.count(l)) {
        delete p;
        return set_err(OME_INVALID_ARGUMENT, "output label %d of node %d has no extent", l, j);
      }
      n.iy.push_back(l);
      if (!contains(p->sliced, l)) n.iy_s.push_back(l);
    }
    for (int32_t l : n.iy) n.numel *= p->ext[l];
    for (int32_t l : n.iy_s) n.numel_s *= p->ext[l];
  }
  canonical_orders(p);
  for (int t = 0; t < ninputs; ++t)
    if (!input_used[t]) {
      delete p;
      return set_err(OME_INVALID_ARGUMENT, "input %d is not used by the tree", t);
    }
  for (int j = 0; j < nnodes - 1; ++j)
    if (p->nodes[j].parent < 0) {
      delete p;
      return set_err(OME_INVALID_ARGUMENT, "node %d is not reachable from the root", j);
    }
  // forward arena (sliced shapes), liveness: a node's output dies when its
  // parent ran.  The FP64 cross-slice accumulator lives through every slice,
  // so it is reserved first and never shared with a node buffer.
  const int root = nnodes - 1;
  const bool sliced = !p->sliced.empty();
  p->acc64 = sliced && (dtype == OME_F32 || dtype == OME_F64 || dtype == OME_C32);
  Arena ar;
  if (p->acc64) p->acc_off = ar.alloc((size_t)p->nodes[root].numel * (dtype == OME_C32 ? 16 : 8));
  for (int j = 0; j < root; ++j) {
    PNode& n = p->nodes[j];
    n.off_fwd = ar.alloc((size_t)n.numel_s * p->esize);
    for (int r : n.args)
      if (r >= 0) ar.release(p->nodes[r].off_fwd);
  }
  // the root's temporary is written after every other node of the slice ran
  // (its children are still live here, so it cannot overlap them)
  if (p->acc64) p->tmp_off = ar.alloc((size_t)p->nodes[root].numel_s * p->esize);
  p->arena_bytes = ar.peak;
  // per-node dispatch scratch: dangling-label reductions (bounded by the
  // children's sizes), split-reduction partials and GEMM workspace; sliced
  // sizes for the forward plan, full sizes for the (unsliced) gradient
  // FP32 binary nodes that the dispatcher sends to the packed-operand
  // tensor-core GEMM (M, N >= 256, K >= 512, >= 1 GFLOP) need their BF16
  // terms in the workspace: L * (M/128 + N/128 tiles) * K/32 k-steps * 24 KB,
  // plus split partials and offset tables (at most 2 GB here; a node that
  // needs more takes its terms from the context's overflow scratch)
  auto packed_gemm_bytes = [&](int j, bool use_sliced) -> size_t {
    const PNode& n = p->nodes[j];
    if (dtype != OME_F32 || prec == OME_PREC_FP32 || n.args.size() != 2) return 0;
    auto labs = [&](int r) -> std::vector<int32_t> {
      std::vector<int32_t> v;
      if (r >= 0) {
        v = use_sliced ? p->nodes[r].iy_s : p->nodes[r].iy;
      } else {
        for (int32_t l : p->in_labels[-r - 1])
          if (!(use_sliced && contains(p->sliced, l))) v.push_back(l);
      }
      return v;
    };
    const std::vector<int32_t> a = labs(n.args[0]), b = labs(n.args[1]);
    const std::vector<int32_t>& y = use_sliced ? n.iy_s : n.iy;
    double M = 1, N = 1, K = 1, L = 1;
    std::vector<int32_t> seen;
    for (const auto* v : {&a, &b})
      for (int32_t l : *v) {
        if (contains(seen, l)) continue;
        seen.push_back(l);
        const bool ia = contains(a, l), ib = contains(b, l), iy = contains(y, l);
        const double e = (double)p->ext[l];
        if (ia && ib && iy) L *= e;
        else if (ia && ib) K *= e;
        else if (ia && iy) M *= e;
        else if (ib && iy) N *= e;
      }
    if (M < 256 || N < 256 || K < 512 || 2.0 * M * N * K * L < 1e9) return 0;
    const double bytes = L * (std::ceil(M / 128) + std::ceil(N / 128)) * std::ceil(K / 32) * 3 * 8192 +
                         148.0 * 128 * 128 * 4 + (M + N) * 8 + 4096;
    return bytes <= (double)((size_t)2 << 30) ? (size_t)bytes : 0;
  };
  auto scratch_bound = [&](bool use_sliced) {
    size_t scratch = 0;
    for (int j = 0; j < nnodes; ++j) {
      size_t sj = 0;
      for (int r : p->nodes[j].args) {
        int64_t c = 1;
        if (r >= 0) {
          c = use_sliced ? p->nodes[r].numel_s : p->nodes[r].numel;
        } else {
          for (int32_t l : p->in_labels[-r - 1])
            if (!(use_sliced && contains(p->sliced, l))) c *= p->ext[l];
        }
        sj += ((size_t)c * p->esize + 255) & ~(size_t)255;
      }
      sj += packed_gemm_bytes(j, use_sliced);
      scratch = std::max(scratch, sj);
    }
    return scratch + ((size_t)64 << 20);
  };
  const size_t scratch = scratch_bound(true), scratch_grad = scratch_bound(false);
  p->fwd_bytes = ((p->arena_bytes + 255) & ~(size_t)255) + scratch;
  // gradient arena: all forward values kept (unsliced) plus one gradient each
  size_t g = 0;
  for (int j = 0; j < root; ++j) {
    PNode& n = p->nodes[j];
    n.off_keep = g;
    g += ((size_t)n.numel * p->esize + 255) & ~(size_t)255;
  }
  for (int j = 0; j < root; ++j) {
    PNode& n = p->nodes[j];
    n.off_grad = g;
    g += ((size_t)n.numel * p->esize + 255) & ~(size_t)255;
  }
  p->dy_off = g;
  p->grad_arena = g + ((size_t)p->nodes[root].numel * p->esize + 511);
  p->grad_bytes = ((p->grad_arena + 255) & ~(size_t)255) + scratch_grad;
  *out = p;
  return OME_OK;
}

int ome_plan_destroy(ome_plan* plan) {
  delete plan;
  return OME_OK;
}

int ome_plan_peak_bytes(const ome_plan* plan, size_t* forward_bytes, size_t* grad_bytes) {
  if (!plan) return set_err(OME_INVALID_ARGUMENT, "plan is NULL");
  if (forward_bytes) *forward_bytes = plan->fwd_bytes;
  if (grad_bytes) *grad_bytes = plan->grad_bytes;
  return OME_OK;
}

}  // extern "C"

namespace {

// Run one node: inputs from children (workspace or leaf views), output view y.
int run_node(ome_ctx* ctx, ome_plan* p, cudaStream_t s, int j, const void* const* inputs, bool sliced,
             const std::vector<int64_t>& fix, size_t (*off_of)(const PNode&), const HView& y, const Scalar& sx,
             const Scalar& sy, size_t scratch_base) {
  const PNode& n = p->nodes[j];
  HView xs[MAXIN];
  const int nin = (int)n.args.size();
  if (nin > MAXIN) return set_err(OME_UNSUPPORTED, "node %d has %d children (max %d)", j, nin, MAXIN);
  static const std::vector<int32_t> none;
  static const std::vector<int64_t> nofix;
  for (int a = 0; a < nin; ++a) {
    const int r = n.args[a];
    if (r >= 0) {
      xs[a] = make_view(p, ctx->ws + off_of(p->nodes[r]), sliced ? p->nodes[r].iy_s : p->nodes[r].iy, none, nofix);
    } else {
      const int t = -r - 1;
      xs[a] = make_view(p, (char*)inputs[t], p->in_labels[t], sliced ? p->sliced : none, sliced ? fix : nofix);
    }
  }
  ctx->ws_top = scratch_base;
  return einsum_views(ctx, s, p->dt, nin, xs, y, sx, sy, p->prec, false);
}

size_t off_fwd_of(const PNode& n) { return n.off_fwd; }
size_t off_keep_of(const PNode& n) { return n.off_keep; }


// Slices [b, e) of the tree, each root result added at its sliced output
// positions: into the F64/C64 buffer `acc` for acc64 plans (the root goes to
// the temporary first), else straight into the plan-dtype output `acc` with
// root scale sx and sy = one (the caller initialised or prescaled it).
int run_slices(ome_ctx* ctx, ome_plan* p, cudaStream_t s, const void* const* inputs, int64_t b, int64_t e,
               char* acc, const Scalar& sx) {
  const ome_dtype dt = p->dt;
  const Scalar one = scalar_one(dt), zero = scalar_zero(dt);
  const int root = (int)p->nodes.size() - 1;
  const PNode& rn = p->nodes[root];
  const size_t scratch = (p->arena_bytes + 255) & ~(size_t)255;
  static const std::vector<int32_t> none;
  static const std::vector<int64_t> nofix;
  std::vector<int64_t> fix(p->sliced.size(), 0);
  for (int64_t sl = b; sl < e; ++sl) {
    int64_t r = sl;
    for (size_t i = 0; i < p->sliced.size(); ++i) {
      const int64_t ext = p->ext[p->sliced[i]];
      fix[i] = r % ext;
      r /= ext;
    }
    for (int j = 0; j < root; ++j) {
      HView v = make_view(p, ctx->ws + p->nodes[j].off_fwd, p->nodes[j].iy_s, none, nofix);
      int rc = run_node(ctx, p, s, j, inputs, true, fix, off_fwd_of, v, one, zero, scratch);
      if (rc) return rc;
    }
    if (p->acc64) {
      HView tv = make_view(p, ctx->ws + p->tmp_off, rn.iy_s, none, nofix);
      int rc = run_node(ctx, p, s, root, inputs, true, fix, off_fwd_of, tv, one, zero, scratch);
      if (rc) return rc;
      // acc[slice positions] += temp
      const size_t w = dt == OME_C32 ? 16 : 8;
      HView av = make_view(p, acc, rn.iy, p->sliced, fix);
      // the accumulator view has element size w: rescale its base offset
      const int64_t eoff = (av.data - acc) / (int64_t)p->esize;
      char* abase = acc + eoff * (int64_t)w;
      rc = cuda_err(launch_acc64_strided(dt, abase, tv.data, av.nd, av.ext, av.str, s), "acc64");
      if (rc) return rc;
    } else {
      HView yv = make_view(p, acc, rn.iy, p->sliced, fix);
      int rc = run_node(ctx, p, s, root, inputs, true, fix, off_fwd_of, yv, sx, one, scratch);
      if (rc) return rc;
    }
  }
  return OME_OK;
}

}  // namespace

extern "C" {

int ome_plan_execute(ome_ctx* ctx, ome_plan* p, void* stream, const void* const* inputs, void* y, const void* sxp,
                     const void* syp) {
  if (!ctx || !p || !inputs || !y || !sxp || !syp) return set_err(OME_INVALID_ARGUMENT, "NULL argument");
  if (ctx->ws_bytes < p->fwd_bytes)
    return set_err(OME_OUT_OF_MEMORY, "plan needs %zu workspace bytes, context has %zu", p->fwd_bytes, ctx->ws_bytes);
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  const ome_dtype dt = p->dt;
  const Scalar sx = scalar_from(dt, sxp), sy = scalar_from(dt, syp);
  const Scalar one = scalar_one(dt), zero = scalar_zero(dt);
  const int root = (int)p->nodes.size() - 1;
  const PNode& rn = p->nodes[root];
  const size_t scratch = (p->arena_bytes + 255) & ~(size_t)255;
  static const std::vector<int32_t> none;
  static const std::vector<int64_t> nofix;

  if (p->sliced.empty()) {
    for (int j = 0; j < root; ++j) {
      HView v = make_view(p, ctx->ws + p->nodes[j].off_fwd, p->nodes[j].iy, none, nofix);
      int rc = run_node(ctx, p, s, j, inputs, false, nofix, off_fwd_of, v, one, zero, scratch);
      if (rc) return rc;
    }
    HView yv = make_view(p, (char*)y, rn.iy, none, nofix);
    return run_node(ctx, p, s, root, inputs, false, nofix, off_fwd_of, yv, sx, sy, scratch);
  }

  // sliced: y <- sy*y first unless accumulating in FP64
  HView yfull = make_view(p, (char*)y, rn.iy, none, nofix);
  if (p->acc64) {
    const size_t w = dt == OME_C32 ? 16 : 8;
    int rc = cuda_err(cudaMemsetAsync(ctx->ws + p->acc_off, 0, (size_t)rn.numel * w, s), "memset");
    if (rc) return rc;
  } else {
    const bool syz = scalar_is_zero(dt, sy);
    if (!(scalar_is_one(dt, sy))) {
      int rc = cuda_err(launch_scale(dt, y, yfull.nd, yfull.ext, yfull.str, sy, syz, ctx->num_sms, s), "scale");
      if (rc) return rc;
    }
  }
  int rc = run_slices(ctx, p, s, inputs, 0, p->nslices, p->acc64 ? ctx->ws + p->acc_off : (char*)y, sx);
  if (rc) return rc;
  if (p->acc64) {
    return cuda_err(launch_acc64_store(dt, y, ctx->ws + p->acc_off, rn.numel, sx, sy, scalar_is_zero(dt, sy), s),
                    "acc64 store");
  }
  return OME_OK;
}

int ome_plan_slice_count(const ome_plan* p, int64_t* nslices) {
  if (!p || !nslices) return set_err(OME_INVALID_ARGUMENT, "NULL argument");
  *nslices = p->nslices;
  return OME_OK;
}

int ome_plan_partial_info(const ome_plan* p, int* partial_dtype, size_t* partial_bytes, int* reduce_op) {
  if (!p) return set_err(OME_INVALID_ARGUMENT, "plan is NULL");
  const int root = (int)p->nodes.size() - 1;
  const int64_t n = p->nodes[root].numel;
  ome_dtype pd = p->dt;
  if (p->acc64) pd = p->dt == OME_C32 ? OME_C64 : OME_F64;
  if (partial_dtype) *partial_dtype = (int)pd;
  if (partial_bytes) *partial_bytes = (size_t)n * dtype_size(pd);
  if (reduce_op) *reduce_op = (p->dt == OME_BOOL || p->dt == OME_TROP_F32 || p->dt == OME_TROP_F64) ? 1 : 0;
  return OME_OK;
}

int ome_plan_execute_slices(ome_ctx* ctx, ome_plan* p, void* stream, const void* const* inputs,
                            int64_t slice_begin, int64_t slice_end, void* partial) {
  if (!ctx || !p || !inputs || !partial) return set_err(OME_INVALID_ARGUMENT, "NULL argument");
  if (slice_begin < 0 || slice_end < slice_begin || slice_end > p->nslices)
    return set_err(OME_INVALID_ARGUMENT, "slice range [%lld, %lld) outside [0, %lld)", (long long)slice_begin,
                   (long long)slice_end, (long long)p->nslices);
  if (ctx->ws_bytes < p->fwd_bytes)
    return set_err(OME_OUT_OF_MEMORY, "plan needs %zu workspace bytes, context has %zu", p->fwd_bytes, ctx->ws_bytes);
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  const int root = (int)p->nodes.size() - 1;
  const PNode& rn = p->nodes[root];
  if (p->acc64) {
    const size_t w = p->dt == OME_C32 ? 16 : 8;
    int rc = cuda_err(cudaMemsetAsync(partial, 0, (size_t)rn.numel * w, s), "memset");
    if (rc) return rc;
  } else {
    static const std::vector<int32_t> none;
    static const std::vector<int64_t> nofix;
    HView pv = make_view(p, (char*)partial, rn.iy, none, nofix);
    int rc = cuda_err(launch_scale(p->dt, partial, pv.nd, pv.ext, pv.str, scalar_zero(p->dt), 1, ctx->num_sms, s),
                      "fill");
    if (rc) return rc;
  }
  return run_slices(ctx, p, s, inputs, slice_begin, slice_end, (char*)partial, scalar_one(p->dt));
}

int ome_plan_finish(ome_ctx* ctx, ome_plan* p, void* stream, const void* partial, void* y, const void* sxp,
                    const void* syp) {
  if (!ctx || !p || !partial || !y || !sxp || !syp) return set_err(OME_INVALID_ARGUMENT, "NULL argument");
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  const ome_dtype dt = p->dt;
  const Scalar sx = scalar_from(dt, sxp), sy = scalar_from(dt, syp);
  const int root = (int)p->nodes.size() - 1;
  const PNode& rn = p->nodes[root];
  if (p->acc64)
    return cuda_err(launch_acc64_store(dt, y, partial, rn.numel, sx, sy, scalar_is_zero(dt, sy), s), "acc64 store");
  static const std::vector<int32_t> none;
  static const std::vector<int64_t> nofix;
  HView xv = make_view(p, (char*)partial, rn.iy, none, nofix);
  HView yv = make_view(p, (char*)y, rn.iy, none, nofix);
  ctx->ws_top = 0;
  return einsum_views(ctx, s, dt, 1, &xv, yv, sx, sy, p->prec, false);
}

}  // extern "C"

namespace ome {
cudaError_t launch_conj(ome_dtype dt, void* x, int64_t n, cudaStream_t s);
cudaError_t launch_fill_one(ome_dtype dt, void* x, int64_t n, cudaStream_t s);
ome_dtype plan_dtype(const ome_plan* p) { return p->dt; }
int plan_ninputs(const ome_plan* p) { return p->ninputs; }
}

extern "C" {

int ome_plan_gradient(ome_ctx* ctx, ome_plan* p, void* stream, const void* const* inputs, const void* dy, void* y,
                      void* const* dxs) {
  if (!ctx || !p || !inputs || !y || !dxs) return set_err(OME_INVALID_ARGUMENT, "NULL argument");
  if (ctx->ws_bytes < p->grad_bytes)
    return set_err(OME_OUT_OF_MEMORY, "gradient needs %zu workspace bytes, context has %zu", p->grad_bytes,
                   ctx->ws_bytes);
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  const ome_dtype dt = p->dt;
  const bool cplx = dt == OME_C32 || dt == OME_C64;
  const Scalar one = scalar_one(dt), zero = scalar_zero(dt);
  const int root = (int)p->nodes.size() - 1;
  const PNode& rn = p->nodes[root];
  static const std::vector<int32_t> none;
  static const std::vector<int64_t> nofix;
  const size_t scratch = (p->grad_arena + 255) & ~(size_t)255;
  // forward, every value kept
  for (int j = 0; j < root; ++j) {
    HView v = make_view(p, ctx->ws + p->nodes[j].off_keep, p->nodes[j].iy, none, nofix);
    int rc = run_node(ctx, p, s, j, inputs, false, nofix, off_keep_of, v, one, zero, scratch);
    if (rc) return rc;
  }
  HView yv = make_view(p, (char*)y, rn.iy, none, nofix);
  int rc = run_node(ctx, p, s, root, inputs, false, nofix, off_keep_of, yv, one, zero, scratch);
  if (rc) return rc;
  // root cotangent: ones (init_gradient, src/bp.jl:133-138) or the caller's dy
  char* dy_root;
  ctx->ws_top = scratch;
  dy_root = ctx->ws + p->dy_off;
  if (dy) {
    rc = cuda_err(cudaMemcpyAsync(dy_root, dy, (size_t)rn.numel * p->esize, cudaMemcpyDeviceToDevice, s), "copy dy");
    if (rc) return rc;
  } else {
    if (rn.numel != 1) return set_err(OME_INVALID_ARGUMENT, "The output must be a scalar! Or you need to feed the gradient manually.");
    rc = cuda_err(launch_fill_one(dt, dy_root, 1, s), "fill");
    if (rc) return rc;
  }
  const size_t scratch2 = ctx->ws_top;
  // reverse sweep
  for (int j = root; j >= 0; --j) {
    const PNode& n = p->nodes[j];
    char* gj = j == root ? dy_root : ctx->ws + n.off_grad;
    // conj(dy) in place (complex): gradients are conj(einsum(.., conj(dy), ..))
    const int nin = (int)n.args.size();
    for (int i = 0; i < nin; ++i) {
      HView xs[MAXIN];
      for (int a = 0; a < nin; ++a) {
        const int r = n.args[a];
        if (a == i) {
          xs[a] = make_view(p, gj, n.iy, none, nofix);
        } else if (r >= 0) {
          xs[a] = make_view(p, ctx->ws + p->nodes[r].off_keep, p->nodes[r].iy, none, nofix);
        } else {
          xs[a] = make_view(p, (char*)inputs[-r - 1], p->in_labels[-r - 1], none, nofix);
        }
      }
      const int r = n.args[i];
      char* dst = r >= 0 ? ctx->ws + p->nodes[r].off_grad : (char*)dxs[-r - 1];
      const std::vector<int32_t>& labs = r >= 0 ? p->nodes[r].iy : p->in_labels[-r - 1];
      const int64_t cnt = r >= 0 ? p->nodes[r].numel : [&] {
        int64_t c = 1;
        for (int32_t l : labs) c *= p->ext[l];
        return c;
      }();
      HView dv = make_view(p, dst, labs, none, nofix);
      if (cplx) {
        rc = cuda_err(launch_conj(dt, gj, j == root ? rn.numel : n.numel, s), "conj");
        if (rc) return rc;
      }
      ctx->ws_top = scratch2;
      rc = einsum_views(ctx, s, dt, nin, xs, dv, one, zero, p->prec, false);
      if (rc) return rc;
      if (cplx) {
        rc = cuda_err(launch_conj(dt, gj, j == root ? rn.numel : n.numel, s), "conj");
        if (rc) return rc;
        rc = cuda_err(launch_conj(dt, dst, cnt, s), "conj");
        if (rc) return rc;
      }
    }
  }
  return OME_OK;
}

}  // extern "C"
