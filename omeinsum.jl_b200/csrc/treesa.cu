// Contraction-order search by simulated annealing over binary contraction
// trees ("TreeSA"), host code.
//
// OMEinsum re-exports TreeSA from its dependency OMEinsumContractionOrders
// (src/contractionorder.jl:30-41; compat 1.1 in the reference's
// Project.toml, not vendored).  This file restates the published method
// (Kalachev, Panteleev, Yung, "Recursive multi-tensor contraction for XEB
// verification of quantum circuits", 2021: local rewrites of a binary tree,
// Metropolis acceptance, inverse temperature swept upwards) in our own code:
//
//  * a node's output labels depend only on the set of leaves under it:
//    out(n) = sub(n) & outside(n), sub = labels of the leaves under n,
//    outside = labels of every other leaf plus the network's output labels;
//  * a move rewrites P = (A, (B, C)) into ((A, B), C) or ((A, C), B) (and the
//    mirror cases); only the new inner node's leaf set changes, so a move
//    touches two contractions: the inner node and P;
//  * cost = log2(sum over contractions of 2^tc + rw_weight * 2^rw)
//          + sc_weight * sum over contractions of max(0, sc - sc_target),
//    tc = log2 of the product of the extents of the labels a contraction
//    touches, sc = log2 of its output size, rw = log2 of (inputs + output);
//  * every trial starts from the given tree, ends with sweeps at zero
//    temperature (improvements only) and keeps its best tree; the best trial
//    (lowest cost) is returned.  Trials run on host threads.
#include <math.h>
#include <stdint.h>
#include <string.h>
#include <algorithm>
#include <random>
#include <thread>
#include <vector>
#include "ome_b200.h"

namespace {

constexpr int MAXW = 8;   // up to 512 labels

struct Bits {
  uint64_t w[MAXW];
};

struct Net {
  int T = 0, W = 0, L = 0;
  std::vector<Bits> leaf;    // labels of each input tensor
  Bits out{};                // labels of the network's output
  std::vector<double> lsz;   // log2 extent per label
  bool uniform = true;
  double u = 0;              // the common log2 extent when uniform
};

struct Tree {
  // internal nodes 0..T-2; child refs: >= 0 internal node, < 0 leaf -r-1
  std::vector<int> left, right, parent;
  int root = 0;
  std::vector<Bits> sub, outside, outb;   // internal nodes
  std::vector<double> tc, sc, rw;         // per internal node
};

inline Bits bor(const Bits& a, const Bits& b, int W) {
  Bits r{};
  for (int i = 0; i < W; ++i) r.w[i] = a.w[i] | b.w[i];
  return r;
}
inline Bits band(const Bits& a, const Bits& b, int W) {
  Bits r{};
  for (int i = 0; i < W; ++i) r.w[i] = a.w[i] & b.w[i];
  return r;
}
inline double lsum(const Net& n, const Bits& b) {
  if (n.uniform) {
    int c = 0;
    for (int i = 0; i < n.W; ++i) c += __builtin_popcountll(b.w[i]);
    return c * n.u;
  }
  double s = 0;
  for (int i = 0; i < n.W; ++i) {
    uint64_t x = b.w[i];
    while (x) {
      const int k = __builtin_ctzll(x);
      s += n.lsz[i * 64 + k];
      x &= x - 1;
    }
  }
  return s;
}

struct Score {
  double sc_target, sc_weight, rw_weight;
};

inline const Bits& sub_of(const Net& n, const Tree& t, int r) { return r >= 0 ? t.sub[r] : n.leaf[-r - 1]; }
inline const Bits& out_of(const Net& n, const Tree& t, int r) { return r >= 0 ? t.outb[r] : n.leaf[-r - 1]; }
inline double sc_of(const Net& n, const Tree& t, int r) { return r >= 0 ? t.sc[r] : lsum(n, n.leaf[-r - 1]); }

// contraction cost terms of internal node j from its children's outputs
inline void node_cost(const Net& n, const Tree& t, int j, const Bits& o, double& tc, double& sc, double& rw) {
  const Bits& a = out_of(n, t, t.left[j]);
  const Bits& b = out_of(n, t, t.right[j]);
  tc = lsum(n, bor(a, b, n.W));
  sc = lsum(n, o);
  const double sa = sc_of(n, t, t.left[j]), sb = sc_of(n, t, t.right[j]);
  const double m = std::max(sa, std::max(sb, sc));
  rw = m + log2(exp2(sa - m) + exp2(sb - m) + exp2(sc - m));
}

// sub / outside / out / costs of every internal node from the structure
void recompute(const Net& n, Tree& t) {
  const int NI = n.T - 1;
  std::vector<int> order;   // post-order
  order.reserve(NI);
  std::vector<std::pair<int, int>> st;
  st.push_back({t.root, 0});
  while (!st.empty()) {
    auto& [j, k] = st.back();
    if (k == 0) {
      k = 1;
      if (t.left[j] >= 0) st.push_back({t.left[j], 0});
    } else if (k == 1) {
      k = 2;
      if (t.right[j] >= 0) st.push_back({t.right[j], 0});
    } else {
      order.push_back(j);
      st.pop_back();
    }
  }
  for (int j : order) t.sub[j] = bor(sub_of(n, t, t.left[j]), sub_of(n, t, t.right[j]), n.W);
  t.outside[t.root] = n.out;
  for (int idx = NI - 1; idx >= 0; --idx) {   // reverse post-order: parents first
    const int j = order[idx];
    for (int side = 0; side < 2; ++side) {
      const int c = side ? t.right[j] : t.left[j];
      const int o = side ? t.left[j] : t.right[j];
      if (c >= 0) t.outside[c] = bor(t.outside[j], sub_of(n, t, o), n.W);
    }
  }
  for (int j : order) t.outb[j] = band(t.sub[j], t.outside[j], n.W);
  for (int j : order) node_cost(n, t, j, t.outb[j], t.tc[j], t.sc[j], t.rw[j]);
}

double total_cost(const Net& n, const Tree& t, const Score& s, double* S_out, double* Q_out) {
  double S = 0, Q = 0;
  for (int j = 0; j < n.T - 1; ++j) {
    S += exp2(t.tc[j]) + s.rw_weight * exp2(t.rw[j]);
    Q += std::max(0.0, t.sc[j] - s.sc_target);
  }
  if (S_out) *S_out = S;
  if (Q_out) *Q_out = Q;
  return log2(S) + s.sc_weight * Q;
}

void anneal(const Net& n, Tree& t, const Score& s, double b0, double db, double b1, int niters, uint64_t seed,
            Tree& best, double& best_cost) {
  std::mt19937_64 rng(seed);
  std::uniform_real_distribution<double> U(0.0, 1.0);
  const int NI = n.T - 1;
  recompute(n, t);
  double S, Q;
  double cost = total_cost(n, t, s, &S, &Q);
  best = t;
  best_cost = cost;
  std::vector<int> nodes(NI);
  for (int j = 0; j < NI; ++j) nodes[j] = j;
  // the temperature schedule, then 2 * niters sweeps at zero temperature
  // (improvements only) so that every trial ends in a local minimum
  const int nb = (int)floor((b1 - b0) / db + 1e-9) + 1;
  for (int bi = 0; bi <= nb; ++bi) {
    const double beta = bi < nb ? b0 + bi * db : INFINITY;
    for (int it = 0; it < (bi < nb ? niters : 2 * niters); ++it) {
      std::shuffle(nodes.begin(), nodes.end(), rng);
      for (int P : nodes) {
        // candidate rewrites at P: the inner child X = (B, C) and the other child A
        int opts[4][2];   // (which side holds X, which of X's children pairs with A)
        int no = 0;
        for (int side = 0; side < 2; ++side) {
          const int X = side ? t.right[P] : t.left[P];
          if (X < 0) continue;
          opts[no][0] = side; opts[no][1] = 0; ++no;
          opts[no][0] = side; opts[no][1] = 1; ++no;
        }
        if (no == 0) continue;
        const int pick = (int)(U(rng) * no) % no;
        const int side = opts[pick][0], keep = opts[pick][1];
        const int X = side ? t.right[P] : t.left[P];
        const int A = side ? t.left[P] : t.right[P];
        const int B = keep ? t.right[X] : t.left[X];   // goes into the new inner node with A
        const int Cc = keep ? t.left[X] : t.right[X];  // becomes P's other child
        // new inner node (A, B) reuses X's slot
        const Bits nsub = bor(sub_of(n, t, A), sub_of(n, t, B), n.W);
        const Bits nout_side = bor(t.outside[P], sub_of(n, t, Cc), n.W);
        const Bits nout = band(nsub, nout_side, n.W);
        // costs of the rewritten pair
        const int oldL[2] = {t.left[X], t.left[P]}, oldR[2] = {t.right[X], t.right[P]};
        const double old_c = exp2(t.tc[X]) + s.rw_weight * exp2(t.rw[X]) + exp2(t.tc[P]) + s.rw_weight * exp2(t.rw[P]);
        const double old_q = std::max(0.0, t.sc[X] - s.sc_target) + std::max(0.0, t.sc[P] - s.sc_target);
        const Bits sv_sub = t.sub[X], sv_out = t.outb[X], sv_outside = t.outside[X];
        const double sv[6] = {t.tc[X], t.sc[X], t.rw[X], t.tc[P], t.sc[P], t.rw[P]};
        t.left[X] = A; t.right[X] = B;
        t.left[P] = X; t.right[P] = Cc;
        t.sub[X] = nsub; t.outb[X] = nout; t.outside[X] = nout_side;
        node_cost(n, t, X, nout, t.tc[X], t.sc[X], t.rw[X]);
        node_cost(n, t, P, t.outb[P], t.tc[P], t.sc[P], t.rw[P]);
        const double new_c = exp2(t.tc[X]) + s.rw_weight * exp2(t.rw[X]) + exp2(t.tc[P]) + s.rw_weight * exp2(t.rw[P]);
        const double new_q = std::max(0.0, t.sc[X] - s.sc_target) + std::max(0.0, t.sc[P] - s.sc_target);
        const double S2 = std::max(S + new_c - old_c, 1e-300);
        const double Q2 = Q + new_q - old_q;
        const double cost2 = log2(S2) + s.sc_weight * Q2;
        const double d = cost2 - cost;
        if (d < 0 || (d == 0 && beta < INFINITY) || (beta < INFINITY && U(rng) < exp(-beta * d))) {
          // accepted: fix parent links and the outside sets below the new node
          if (A >= 0) t.parent[A] = X;
          if (B >= 0) t.parent[B] = X;
          if (Cc >= 0) t.parent[Cc] = P;
          t.parent[X] = P;
          if (A >= 0) t.outside[A] = bor(nout_side, sub_of(n, t, B), n.W);
          if (B >= 0) t.outside[B] = bor(nout_side, sub_of(n, t, A), n.W);
          if (Cc >= 0) t.outside[Cc] = bor(t.outside[P], nsub, n.W);
          S = S2;
          Q = Q2;
          cost = cost2;
          if (cost < best_cost - 1e-12) {
            best = t;
            best_cost = cost;
          }
        } else {
          t.left[X] = oldL[0]; t.right[X] = oldR[0];
          t.left[P] = oldL[1]; t.right[P] = oldR[1];
          t.sub[X] = sv_sub; t.outb[X] = sv_out; t.outside[X] = sv_outside;
          t.tc[X] = sv[0]; t.sc[X] = sv[1]; t.rw[X] = sv[2];
          t.tc[P] = sv[3]; t.sc[P] = sv[4]; t.rw[P] = sv[5];
        }
      }
      // drop the rounding of the running sums once per sweep
      cost = total_cost(n, t, s, &S, &Q);
    }
  }
  recompute(n, best);
  best_cost = total_cost(n, best, s, nullptr, nullptr);
}

}  // namespace

extern "C" {

int ome_treesa(int32_t ntensors, const int32_t* nlabels, const int32_t* labels, int32_t nout,
               const int32_t* out_labels, int32_t nids, const double* log2_sizes, const int32_t* init_tree,
               double sc_target, double sc_weight, double rw_weight, double beta_start, double beta_step,
               double beta_stop, int32_t niters, int32_t ntrials, uint64_t seed, int32_t* out_tree,
               double* out_complexity) {
  if (ntensors < 2 || !nlabels || !labels || !log2_sizes || !init_tree || !out_tree) return OME_INVALID_ARGUMENT;
  if (nids < 1 || nids > 64 * MAXW) return OME_UNSUPPORTED;
  if (!(beta_step > 0) || beta_stop < beta_start || niters < 1 || ntrials < 1) return OME_INVALID_ARGUMENT;
  Net n;
  n.T = ntensors;
  n.L = nids;
  n.W = (nids + 63) / 64;
  n.lsz.assign(log2_sizes, log2_sizes + nids);
  n.u = n.lsz[0];
  for (double v : n.lsz) n.uniform = n.uniform && v == n.u;
  n.leaf.resize(ntensors);
  int64_t pos = 0;
  for (int t = 0; t < ntensors; ++t) {
    memset(&n.leaf[t], 0, sizeof(Bits));
    for (int k = 0; k < nlabels[t]; ++k) {
      const int l = labels[pos++];
      if (l < 0 || l >= nids) return OME_INVALID_ARGUMENT;
      n.leaf[t].w[l >> 6] |= 1ull << (l & 63);
    }
  }
  memset(&n.out, 0, sizeof(Bits));
  for (int k = 0; k < nout; ++k) {
    const int l = out_labels[k];
    if (l < 0 || l >= nids) return OME_INVALID_ARGUMENT;
    n.out.w[l >> 6] |= 1ull << (l & 63);
  }
  const int NI = ntensors - 1;
  Tree t0;
  t0.left.resize(NI); t0.right.resize(NI); t0.parent.assign(NI, -1);
  t0.sub.resize(NI); t0.outside.resize(NI); t0.outb.resize(NI);
  t0.tc.resize(NI); t0.sc.resize(NI); t0.rw.resize(NI);
  std::vector<int> used(ntensors, 0);
  for (int j = 0; j < NI; ++j) {
    for (int side = 0; side < 2; ++side) {
      const int r = init_tree[2 * j + side];
      if (r >= 0) {
        if (r >= j) return OME_INVALID_ARGUMENT;   // post-order: children first
        if (t0.parent[r] != -1) return OME_INVALID_ARGUMENT;
        t0.parent[r] = j;
      } else {
        const int leaf = -r - 1;
        if (leaf >= ntensors || used[leaf]) return OME_INVALID_ARGUMENT;
        used[leaf] = 1;
      }
      (side ? t0.right : t0.left)[j] = r;
    }
  }
  for (int t = 0; t < ntensors; ++t)
    if (!used[t]) return OME_INVALID_ARGUMENT;
  t0.root = NI - 1;
  const Score s{sc_target, sc_weight, rw_weight};
  std::vector<Tree> bests(ntrials);
  std::vector<double> costs(ntrials, INFINITY);
  const unsigned hw = std::max(1u, std::thread::hardware_concurrency());
  for (int base = 0; base < ntrials; base += (int)hw) {
    std::vector<std::thread> th;
    for (int k = base; k < std::min(ntrials, base + (int)hw); ++k)
      th.emplace_back([&, k] {
        Tree t = t0;
        anneal(n, t, s, beta_start, beta_step, beta_stop, niters, seed + 0x9E3779B97F4A7C15ull * (uint64_t)(k + 1),
               bests[k], costs[k]);
      });
    for (auto& x : th) x.join();
  }
  const int kb = (int)(std::min_element(costs.begin(), costs.end()) - costs.begin());
  const Tree& b = bests[kb];
  // post-order renumbering of the best tree
  std::vector<int> order;
  std::vector<std::pair<int, int>> st;
  st.push_back({b.root, 0});
  while (!st.empty()) {
    auto& [j, k] = st.back();
    if (k == 0) {
      k = 1;
      if (b.left[j] >= 0) st.push_back({b.left[j], 0});
    } else if (k == 1) {
      k = 2;
      if (b.right[j] >= 0) st.push_back({b.right[j], 0});
    } else {
      order.push_back(j);
      st.pop_back();
    }
  }
  std::vector<int> newid(NI);
  for (int i = 0; i < NI; ++i) newid[order[i]] = i;
  for (int i = 0; i < NI; ++i) {
    const int j = order[i];
    const int l = b.left[j], r = b.right[j];
    out_tree[2 * i] = l >= 0 ? newid[l] : l;
    out_tree[2 * i + 1] = r >= 0 ? newid[r] : r;
  }
  if (out_complexity) {
    double S = 0, sc = 0, R = 0;
    for (int j = 0; j < NI; ++j) {
      S += exp2(b.tc[j]);
      R += exp2(b.rw[j]);
      sc = std::max(sc, b.sc[j]);
    }
    out_complexity[0] = log2(S);
    out_complexity[1] = sc;
    out_complexity[2] = log2(R);
  }
  return OME_OK;
}

// Greedy slicer: given a tree (ome_treesa format), repeatedly slice the label
// (extent set to 1) that gives the smallest (space complexity, time
// complexity + log2 extent of the label) until the largest intermediate fits
// 2^sc_target elements or max_slices labels are sliced.  Node label sets are
// computed once; a candidate only re-sums costs.
int ome_slice_greedy(int32_t ntensors, const int32_t* nlabels, const int32_t* labels, int32_t nout,
                     const int32_t* out_labels, int32_t nids, const double* log2_sizes, const int32_t* tree,
                     double sc_target, int32_t max_slices, const int32_t* forbidden, int32_t* out_sliced,
                     int32_t* out_count) {
  if (ntensors < 2 || !nlabels || !labels || !log2_sizes || !tree || !out_sliced || !out_count)
    return OME_INVALID_ARGUMENT;
  if (nids < 1 || nids > 64 * MAXW) return OME_UNSUPPORTED;
  Net n;
  n.T = ntensors;
  n.L = nids;
  n.W = (nids + 63) / 64;
  n.lsz.assign(log2_sizes, log2_sizes + nids);
  n.uniform = false;
  n.leaf.resize(ntensors);
  int64_t pos = 0;
  for (int t = 0; t < ntensors; ++t) {
    memset(&n.leaf[t], 0, sizeof(Bits));
    for (int k = 0; k < nlabels[t]; ++k) {
      const int l = labels[pos++];
      if (l < 0 || l >= nids) return OME_INVALID_ARGUMENT;
      n.leaf[t].w[l >> 6] |= 1ull << (l & 63);
    }
  }
  memset(&n.out, 0, sizeof(Bits));
  for (int k = 0; k < nout; ++k) {
    const int l = out_labels[k];
    if (l < 0 || l >= nids) return OME_INVALID_ARGUMENT;
    n.out.w[l >> 6] |= 1ull << (l & 63);
  }
  const int NI = ntensors - 1;
  Tree t;
  t.left.resize(NI); t.right.resize(NI); t.parent.assign(NI, -1);
  t.sub.resize(NI); t.outside.resize(NI); t.outb.resize(NI);
  t.tc.resize(NI); t.sc.resize(NI); t.rw.resize(NI);
  std::vector<int> used(ntensors, 0);
  for (int j = 0; j < NI; ++j)
    for (int side = 0; side < 2; ++side) {
      const int r = tree[2 * j + side];
      if (r >= 0) {
        if (r >= j || t.parent[r] != -1) return OME_INVALID_ARGUMENT;
        t.parent[r] = j;
      } else {
        const int leaf = -r - 1;
        if (leaf >= ntensors || used[leaf]) return OME_INVALID_ARGUMENT;
        used[leaf] = 1;
      }
      (side ? t.right : t.left)[j] = r;
    }
  for (int x = 0; x < ntensors; ++x)
    if (!used[x]) return OME_INVALID_ARGUMENT;
  t.root = NI - 1;
  recompute(n, t);
  // per node: the labels it touches (children's outputs) and its output
  std::vector<Bits> touch(NI);
  Bits any{};
  for (int j = 0; j < NI; ++j) {
    touch[j] = bor(out_of(n, t, t.left[j]), out_of(n, t, t.right[j]), n.W);
    any = bor(any, touch[j], n.W);
  }
  auto eval = [&](double& sc, double& tc) {
    double S = 0;
    sc = 0;
    for (int j = 0; j < NI; ++j) {
      S += exp2(lsum(n, touch[j]));
      sc = std::max(sc, lsum(n, t.outb[j]));
    }
    tc = log2(S);
  };
  int cnt = 0;
  while (cnt < max_slices) {
    double sc, tc;
    eval(sc, tc);
    if (sc <= sc_target + 1e-9) break;
    int best = -1;
    double bsc = INFINITY, bkey = INFINITY;
    for (int l = 0; l < nids; ++l) {
      if (!(any.w[l >> 6] >> (l & 63) & 1) || n.lsz[l] <= 0 || (forbidden && forbidden[l])) continue;
      const double keep = n.lsz[l];
      n.lsz[l] = 0;
      double sc2, tc2;
      eval(sc2, tc2);
      n.lsz[l] = keep;
      const double key = tc2 + keep;
      if (sc2 < bsc - 1e-12 || (fabs(sc2 - bsc) <= 1e-12 && key < bkey - 1e-12)) {
        bsc = sc2;
        bkey = key;
        best = l;
      }
    }
    if (best < 0) break;
    n.lsz[best] = 0;
    out_sliced[cnt++] = best;
  }
  *out_count = cnt;
  return OME_OK;
}

// Greedy pairwise order (the GreedyMethod of OMEinsumContractionOrders,
// restated): repeatedly contract the pair of live tensors that share a label
// (the two smallest tensors when none do) minimising
// size(result) - alpha * (size(a) + size(b)); ties broken at random, or, with
// temperature > 0, a pair drawn with weight exp(-(cost - min) / (temperature *
// max(|min|, 1))).  nrepeat runs; the one with the smallest (tc, sc) is
// returned in the ome_treesa tree format.
int ome_greedy(int32_t ntensors, const int32_t* nlabels, const int32_t* labels, int32_t nout,
               const int32_t* out_labels, int32_t nids, const double* log2_sizes, double alpha,
               double temperature, int32_t nrepeat, uint64_t seed, int32_t* out_tree, double* out_complexity) {
  if (ntensors < 2 || !nlabels || !labels || !log2_sizes || !out_tree) return OME_INVALID_ARGUMENT;
  if (nids < 1 || nids > 64 * MAXW) return OME_UNSUPPORTED;
  Net n;
  n.T = ntensors;
  n.L = nids;
  n.W = (nids + 63) / 64;
  n.lsz.assign(log2_sizes, log2_sizes + nids);
  n.u = n.lsz[0];
  for (double v : n.lsz) n.uniform = n.uniform && v == n.u;
  n.leaf.resize(ntensors);
  int64_t pos = 0;
  for (int t = 0; t < ntensors; ++t) {
    memset(&n.leaf[t], 0, sizeof(Bits));
    for (int k = 0; k < nlabels[t]; ++k) {
      const int l = labels[pos++];
      if (l < 0 || l >= nids) return OME_INVALID_ARGUMENT;
      n.leaf[t].w[l >> 6] |= 1ull << (l & 63);
    }
  }
  memset(&n.out, 0, sizeof(Bits));
  for (int k = 0; k < nout; ++k) {
    const int l = out_labels[k];
    if (l < 0 || l >= nids) return OME_INVALID_ARGUMENT;
    n.out.w[l >> 6] |= 1ull << (l & 63);
  }
  const int NI = ntensors - 1;
  std::mt19937_64 rng(seed);
  std::uniform_real_distribution<double> U(0.0, 1.0);
  std::vector<int32_t> best_tree;
  double best_tc = INFINITY, best_sc = INFINITY, best_rw = 0;
  for (int rep = 0; rep < std::max(1, nrepeat); ++rep) {
    // live slots: label bitset, tree ref; per-label number of live slots holding it
    std::vector<Bits> lab(n.leaf);
    std::vector<int> ref(ntensors), alive(ntensors, 1);
    for (int t = 0; t < ntensors; ++t) ref[t] = -t - 1;
    std::vector<int> cnt(nids, 0);
    for (int t = 0; t < ntensors; ++t)
      for (int l = 0; l < nids; ++l)
        if (lab[t].w[l >> 6] >> (l & 63) & 1) ++cnt[l];
    std::vector<int32_t> tree;
    tree.reserve(2 * NI);
    double S = 0, R = 0, sc = 0;
    auto result = [&](int a, int b) {
      Bits u = bor(lab[a], lab[b], n.W), r{};
      for (int i = 0; i < n.W; ++i) {
        uint64_t x = u.w[i];
        while (x) {
          const int k = __builtin_ctzll(x);
          const int l = i * 64 + k;
          const int inside = (int)(lab[a].w[i] >> k & 1) + (int)(lab[b].w[i] >> k & 1);
          if ((n.out.w[i] >> k & 1) || cnt[l] > inside) r.w[i] |= 1ull << k;
          x &= x - 1;
        }
      }
      return r;
    };
    int live = ntensors;
    while (live > 1) {
      // candidate pairs: live slots sharing a label
      std::vector<std::pair<int, int>> cand;
      for (int a = 0; a < ntensors; ++a) {
        if (!alive[a]) continue;
        for (int b = a + 1; b < ntensors; ++b) {
          if (!alive[b]) continue;
          bool share = false;
          for (int i = 0; i < n.W && !share; ++i) share = (lab[a].w[i] & lab[b].w[i]) != 0;
          if (share) cand.push_back({a, b});
        }
      }
      if (cand.empty()) {
        int s1 = -1, s2 = -1;
        for (int a = 0; a < ntensors; ++a) {
          if (!alive[a]) continue;
          if (s1 < 0 || lsum(n, lab[a]) < lsum(n, lab[s1])) { s2 = s1; s1 = a; }
          else if (s2 < 0 || lsum(n, lab[a]) < lsum(n, lab[s2])) s2 = a;
        }
        cand.push_back({std::min(s1, s2), std::max(s1, s2)});
      }
      std::vector<double> cost(cand.size());
      double cmin = INFINITY;
      for (size_t i = 0; i < cand.size(); ++i) {
        const int a = cand[i].first, b = cand[i].second;
        cost[i] = exp2(lsum(n, result(a, b))) - alpha * (exp2(lsum(n, lab[a])) + exp2(lsum(n, lab[b])));
        cmin = std::min(cmin, cost[i]);
      }
      size_t pick = 0;
      if (temperature > 0) {
        double tot = 0;
        std::vector<double> w(cand.size());
        for (size_t i = 0; i < cand.size(); ++i) tot += (w[i] = exp(-(cost[i] - cmin) / (temperature * std::max(fabs(cmin), 1.0))));
        double x = U(rng) * tot;
        for (pick = 0; pick + 1 < cand.size() && x >= w[pick]; ++pick) x -= w[pick];
      } else {
        std::vector<size_t> ties;
        for (size_t i = 0; i < cand.size(); ++i)
          if (cost[i] == cmin) ties.push_back(i);
        pick = ties[(size_t)(U(rng) * ties.size()) % ties.size()];
      }
      const int a = cand[pick].first, b = cand[pick].second;
      const Bits r = result(a, b);
      const double tcn = lsum(n, bor(lab[a], lab[b], n.W)), scn = lsum(n, r);
      const double sa = lsum(n, lab[a]), sb = lsum(n, lab[b]);
      S += exp2(tcn);
      R += exp2(sa) + exp2(sb) + exp2(scn);
      sc = std::max(sc, scn);
      tree.push_back(ref[a]);
      tree.push_back(ref[b]);
      for (int l = 0; l < nids; ++l) {
        cnt[l] -= (int)(lab[a].w[l >> 6] >> (l & 63) & 1) + (int)(lab[b].w[l >> 6] >> (l & 63) & 1);
        cnt[l] += (int)(r.w[l >> 6] >> (l & 63) & 1);
      }
      lab[a] = r;
      ref[a] = (int)(tree.size() / 2) - 1;
      alive[b] = 0;
      --live;
    }
    const double tc = log2(S);
    if (tc < best_tc - 1e-12 || (fabs(tc - best_tc) <= 1e-12 && sc < best_sc)) {
      best_tc = tc;
      best_sc = sc;
      best_rw = log2(R);
      best_tree = tree;
    }
  }
  for (int i = 0; i < 2 * NI; ++i) out_tree[i] = best_tree[i];
  if (out_complexity) {
    out_complexity[0] = best_tc;
    out_complexity[1] = best_sc;
    out_complexity[2] = best_rw;
  }
  return OME_OK;
}

}  // extern "C"
