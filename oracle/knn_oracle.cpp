// ORACLE -- test infrastructure only. Not part of the shipped library.
//
// CPU restatement of the approximate k-NN graph path of gosteq/Approximate-CUDA-kNN
// (euclideandistancematrixgpu.cu), made deterministic so that the GPU plain-FP32
// path can be checked against it bit for bit:
//
//   points -> random-projection trees -> leaf-block all-pairs k-NN
//          -> neighbour-of-neighbour propagation (Jacobi) -> k-NN graph
//
// plus an FP64 exact brute-force k-NN used as the recall / distance-error yardstick,
// and the learned split network's forward pass and triplet-loss gradient in
// FP64 (no reference counterpart; the tests pin it by central finite
// differences, then check the GPU backward kernels against it).
//
// Parity: the reference ships no tests, golden vectors or fixtures, and its GPU
// output is non-deterministic (atomic scatter order, atomic tie fill, unstable
// std::sort).  Parity of THIS restatement with the reference is therefore pinned
// only through the hand-built known-answer cases under tests/ (analytic grids,
// duplicates, ties, N = k+1, d = 1, d = 257) and the FP64 exact k-NN; the
// reference's own sm_100a build is compared by recall only.
//
// Deterministic rules (each departs from the reference only where the reference
// is non-deterministic or undefined):
//   * tree split (.cu:2138-2181, .cu:2291-2365): direction v = x[p2] - x[p1] for
//     two member positions p1 != p2 drawn from a counter hash of
//     (seed, tree, level, node) instead of one shared rand() pair per level;
//     side chosen by rank of (projection, point id) against the node median
//     (the reference splits at projection 0) and a STABLE partition instead of
//     the atomicInc scatter (.cu:2205-2260).  Node j of level l always covers
//     leaf-order positions [floor(j*n/2^l), floor((j+1)*n/2^l)).
//   * start node (.cu:87-105): the smallest ancestor of the leaf with >= k+1
//     points; its position range is the candidate block.
//   * candidate set of the initial k-NN (.cu:166-192): union over trees of the
//     blocks, minus the point itself; k smallest by (key, id)
//     instead of the histogram select with arbitrary tie fill (.cu:300-410).
//   * propagation (.cu:1078-1101, .cu:1937-1977): C_i = N(N(i)) minus {i},
//     new N(i) = k smallest of N(i) u C_i by (key, id), Jacobi double buffer.
//   * distance formulas (.cu:243-273, .cu:540-570, .cu:840-881): single-precision
//     fused multiply-add in the reference's order (sequential within 256-dim
//     chunks, chunk partials added to a running total).  Keys: squared L2 for
//     EUCLIDEAN (reported as sqrt), L1 for TAXICAB (the reference stores sqrt(L1);
//     the ranking is the same), 1 - cos for COSINE, with 1 for a zero-norm row.
//
// Build: see oracle/Makefile (g++ -O3 -fopenmp -ffp-contract=off).
#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <vector>
#include <omp.h>

namespace {

constexpr int kEuclidean = 0;
constexpr int kTaxicab = 1;
constexpr int kCosine = 2;

// ---------------------------------------------------------------- hashing --
inline uint64_t splitmix64(uint64_t x) {
  x += 0x9E3779B97F4A7C15ull;
  uint64_t z = x;
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
  return z ^ (z >> 31);
}

// Two distinct member positions of a node of n >= 2 points
// (replaces rand() pair of .cu:2329-2333 / .cu:2589).
inline void pivot_positions(uint64_t seed, int tree, int level, int64_t node, int64_t n,
                            int64_t* p1, int64_t* p2) {
  uint64_t z = splitmix64(seed + 0x9E3779B97F4A7C15ull * (uint64_t)(tree + 1));
  z = splitmix64(z ^ (((uint64_t)level << 40) | (uint64_t)node));
  int64_t a = (int64_t)((z & 0xFFFFFFFFull) % (uint64_t)n);
  int64_t b = (int64_t)((z >> 32) % (uint64_t)n);
  if (a == b) b = (a + 1) % n;
  *p1 = a;
  *p2 = b;
}

// ------------------------------------------------------------ tree shape --
inline int tree_depth(int64_t n, int leaf) {
  int l = 0;
  while (((n + (int64_t(1) << l) - 1) >> l) > leaf) ++l;
  return l;
}
inline int64_t node_lo(int64_t n, int level, int64_t j) {
  return (int64_t)(((unsigned __int128)j * (unsigned __int128)n) >> level);
}

// ------------------------------------------------------------- ordering --
inline uint32_t orderable(float f) {
  uint32_t u;
  std::memcpy(&u, &f, 4);
  return (u & 0x80000000u) ? ~u : (u | 0x80000000u);
}
inline uint64_t proj_key(float proj, int32_t id) {
  return ((uint64_t)orderable(proj) << 32) | (uint32_t)id;
}

struct Cand {
  float key;
  int32_t id;
};
inline bool cand_less(const Cand& a, const Cand& b) {
  if (a.key < b.key) return true;
  if (b.key < a.key) return false;
  return (uint32_t)a.id < (uint32_t)b.id;
}

// ------------------------------------------------------------ projection --
// Projection x . v in the GPU's grouped order: G lanes (power of two, <= 4,
// covering ceil(d/4) float4 chunks), lane l accumulates chunks l, l+G, ...
// with fmaf, then an xor butterfly over the G lanes.
inline int proj_group(int d) {
  int nc = (d + 3) / 4;
  int g = 1;
  while (g < nc && g < 4) g <<= 1;
  return g;
}
float project(const float* x, const float* v, int d) {
  const int G = proj_group(d);
  const int nc = (d + 3) / 4;
  float p[32];
  for (int l = 0; l < G; ++l) {
    float acc = 0.0f;
    for (int c = l; c < nc; c += G)
      for (int e = 0; e < 4; ++e) {
        int dim = 4 * c + e;
        if (dim < d) acc = std::fmaf(x[dim], v[dim], acc);
      }
    p[l] = acc;
  }
  for (int off = G / 2; off >= 1; off >>= 1) {
    float q[32];
    for (int l = 0; l < G; ++l) q[l] = p[l] + p[l ^ off];
    for (int l = 0; l < G; ++l) p[l] = q[l];
  }
  return p[0];
}

// ------------------------------------------------------------- distances --
// Reference order: sequential over each 256-dim chunk, chunk partial added to
// the running total (.cu:243-264).
float key_euclid(const float* a, const float* b, int d) {
  float total = 0.0f;
  for (int c0 = 0; c0 < d; c0 += 256) {
    float part = 0.0f;
    int c1 = std::min(d, c0 + 256);
    for (int i = c0; i < c1; ++i) {
      float df = a[i] - b[i];
      part = std::fmaf(df, df, part);
    }
    total = total + part;
  }
  return total;
}
float key_taxicab(const float* a, const float* b, int d) {
  float total = 0.0f;
  for (int c0 = 0; c0 < d; c0 += 256) {
    float part = 0.0f;
    int c1 = std::min(d, c0 + 256);
    for (int i = c0; i < c1; ++i) part = part + std::fabs(a[i] - b[i]);
    total = total + part;
  }
  return total;
}
float dot_chunked(const float* a, const float* b, int d) {
  float total = 0.0f;
  for (int c0 = 0; c0 < d; c0 += 256) {
    float part = 0.0f;
    int c1 = std::min(d, c0 + 256);
    for (int i = c0; i < c1; ++i) part = std::fmaf(a[i], b[i], part);
    total = total + part;
  }
  return total;
}
inline float key_cosine_from(float dot, float na, float nb) {
  if (na == 0.0f || nb == 0.0f) return 1.0f;
  return 1.0f - dot / (na * nb);
}

// Sums of one query row against eight candidate rows at once: eight
// independent sums, each in the order of key_euclid / key_taxicab /
// dot_chunked (sequential within 256-dim chunks, chunk partials added to the
// total), so every result has the bits of the one-pair function.
template <int METRIC>
void sums8(const float* a, const float* const* b, int d, float* out) {
  float total[8] = {0, 0, 0, 0, 0, 0, 0, 0};
  for (int c0 = 0; c0 < d; c0 += 256) {
    float part[8] = {0, 0, 0, 0, 0, 0, 0, 0};
    const int c1 = std::min(d, c0 + 256);
    for (int i = c0; i < c1; ++i) {
      const float av = a[i];
      for (int j = 0; j < 8; ++j) {
        if (METRIC == kEuclidean) {
          const float df = av - b[j][i];
          part[j] = std::fmaf(df, df, part[j]);
        } else if (METRIC == kTaxicab) {
          part[j] = part[j] + std::fabs(av - b[j][i]);
        } else {
          part[j] = std::fmaf(av, b[j][i], part[j]);
        }
      }
    }
    for (int j = 0; j < 8; ++j) total[j] = total[j] + part[j];
  }
  for (int j = 0; j < 8; ++j) out[j] = total[j];
}

struct Data {
  const float* X;
  int64_t n;
  int d;
  int metric;
  std::vector<float> norms;  // cosine only
  const float* row(int64_t i) const { return X + (size_t)i * (size_t)d; }
  float key(int64_t i, int64_t j) const {
    if (metric == kEuclidean) return key_euclid(row(i), row(j), d);
    if (metric == kTaxicab) return key_taxicab(row(i), row(j), d);
    return key_cosine_from(dot_chunked(row(i), row(j), d), norms[i], norms[j]);
  }
  // out[c] = key(i, ids[c]) for c < m, eight candidates at a time
  void keys(int64_t i, const int32_t* ids, int64_t m, float* out) const {
    int64_t c = 0;
    const float* b[8];
    for (; c + 8 <= m; c += 8) {
      for (int j = 0; j < 8; ++j) b[j] = row(ids[c + j]);
      if (metric == kEuclidean) sums8<kEuclidean>(row(i), b, d, out + c);
      else if (metric == kTaxicab) sums8<kTaxicab>(row(i), b, d, out + c);
      else {
        sums8<kCosine>(row(i), b, d, out + c);
        for (int j = 0; j < 8; ++j) out[c + j] = key_cosine_from(out[c + j], norms[i], norms[ids[c + j]]);
      }
    }
    for (; c < m; ++c) out[c] = key(i, ids[c]);
  }
};

// Candidates (ids, keys) that can still enter a full sorted list of k: those
// below its last entry (the rest cannot be among the k best of the union).
void add_below_tail(const std::vector<Cand>& list, int k, const int32_t* ids, const float* keys, int64_t m,
                    std::vector<Cand>& add) {
  add.clear();
  const bool full = (int)list.size() >= k;
  for (int64_t c = 0; c < m; ++c) {
    const Cand cd{keys[c], ids[c]};
    if (!full || cand_less(cd, list[k - 1])) add.push_back(cd);
  }
}

void prepare(Data& D) {
  if (D.metric == kCosine) {
    D.norms.resize(D.n);
#pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < D.n; ++i) D.norms[i] = std::sqrt(dot_chunked(D.row(i), D.row(i), D.d));
  }
}

// ------------------------------------------------------------ tree build --
void build_tree(const Data& D, int tree, int leaf, uint64_t seed, int32_t* perm) {
  const int64_t n = D.n;
  const int d = D.d;
  const int depth = tree_depth(n, leaf);
  for (int64_t i = 0; i < n; ++i) perm[i] = (int32_t)i;
  std::vector<float> v(d);
  std::vector<uint64_t> keys;
  std::vector<int32_t> tmp;
  for (int l = 0; l < depth; ++l) {
    const int64_t nodes = int64_t(1) << l;
    for (int64_t j = 0; j < nodes; ++j) {
      const int64_t lo = node_lo(n, l, j), hi = node_lo(n, l, j + 1);
      const int64_t mid = node_lo(n, l + 1, 2 * j + 1);
      const int64_t cnt = hi - lo;
      if (cnt < 2) continue;
      int64_t p1, p2;
      pivot_positions(seed, tree, l, j, cnt, &p1, &p2);
      const float* xa = D.row(perm[lo + p1]);
      const float* xb = D.row(perm[lo + p2]);
      for (int e = 0; e < d; ++e) v[e] = xb[e] - xa[e];
      keys.resize(cnt);
      for (int64_t p = 0; p < cnt; ++p) {
        int32_t id = perm[lo + p];
        keys[p] = proj_key(project(D.row(id), v.data(), d), id);
      }
      // pivot = (mid-lo)-th smallest key; left = keys strictly below it.
      std::vector<uint64_t> sorted(keys);
      const int64_t nl = mid - lo;
      std::nth_element(sorted.begin(), sorted.begin() + nl, sorted.end());
      const uint64_t pivot = sorted[nl];
      tmp.resize(cnt);
      int64_t wl = 0, wr = nl;
      for (int64_t p = 0; p < cnt; ++p) {
        if (keys[p] < pivot) tmp[wl++] = perm[lo + p];
        else tmp[wr++] = perm[lo + p];
      }
      std::memcpy(perm + lo, tmp.data(), cnt * sizeof(int32_t));
    }
  }
}

// ------------------------------------------------------------ top-k merge --
// list: sorted, unique; add: arbitrary; result: k smallest unique by (key,id).
void merge_topk(std::vector<Cand>& list, std::vector<Cand>& add, int k) {
  add.insert(add.end(), list.begin(), list.end());
  std::sort(add.begin(), add.end(), cand_less);
  list.clear();
  for (const Cand& c : add) {
    if (!list.empty() && list.back().id == c.id) continue;
    list.push_back(c);
    if ((int)list.size() == k) break;
  }
}

// ------------------------------------------------ reference-rule trees --
// The split of buildUpTheTrees (euclideandistancematrixgpu.cu:2138-2181,
// :2291-2365, :2478-2487) made deterministic: per level two draws shared by
// every node (p1 = R1 % c, p2 = R2 % c, p2 = (p1+1) % c if equal), side by
// the sign of the sequential fused sum x . (x[p2] - x[p1]) (left when < 0),
// p1 forced left and p2 right, stable partition, nodes of at most `leaf`
// points stop.
struct FNodeO {
  int64_t lo, hi, parent;
  bool split;
};

uint32_t faithful_draw(uint64_t seed, int tree, int level, int which) {
  const uint64_t h = splitmix64(seed ^ splitmix64(0xF417F01ull + (uint64_t)tree * 0x9E3779B97F4A7C15ull +
                                                  (uint64_t)level * 0xD1B54A32D192ED03ull + (uint64_t)which));
  return (uint32_t)(h & 0x7FFFFFFFu);
}

void build_tree_faithful(const Data& D, int tree, int leaf, uint64_t seed, int32_t* perm,
                         std::vector<FNodeO>& nodes) {
  const int64_t n = D.n;
  const int d = D.d;
  for (int64_t i = 0; i < n; ++i) perm[i] = (int32_t)i;
  nodes.clear();
  nodes.push_back({0, n, -1, false});
  std::vector<int64_t> active;
  if (n > leaf) active.push_back(0);
  std::vector<int32_t> tmp;
  std::vector<float> diff(d);
  int level = 0;
  while (!active.empty()) {
    std::vector<int64_t> next;
    for (int64_t a : active) {
      const int64_t lo = nodes[a].lo, hi = nodes[a].hi, cnt = hi - lo;
      int64_t p1 = 0, p2 = 0;
      if (cnt > 1) {
        p1 = faithful_draw(seed, tree, level, 1) % (uint64_t)cnt;
        p2 = faithful_draw(seed, tree, level, 2) % (uint64_t)cnt;
        if (p1 == p2) p2 = (p1 + 1) % cnt;
      }
      const float* xa = D.row(perm[lo + p1]);
      const float* xb = D.row(perm[lo + p2]);
      for (int c = 0; c < d; ++c) diff[c] = xb[c] - xa[c];
      tmp.clear();
      std::vector<int32_t> right;
      for (int64_t p = lo; p < hi; ++p) {
        const float* x = D.row(perm[p]);
        float acc = 0.0f;
        for (int c = 0; c < d; ++c) acc = std::fmaf(x[c], diff[c], acc);
        bool left = acc < 0.0f;
        if (p == lo + p1) left = true;
        if (p == lo + p2) left = false;
        if (left) tmp.push_back(perm[p]);
        else right.push_back(perm[p]);
      }
      const int64_t nl = (int64_t)tmp.size();
      for (int32_t v : right) tmp.push_back(v);
      std::memcpy(perm + lo, tmp.data(), sizeof(int32_t) * (size_t)cnt);
      nodes[a].split = true;
      const int64_t L = (int64_t)nodes.size();
      nodes.push_back({lo, lo + nl, a, false});
      nodes.push_back({lo + nl, hi, a, false});
      if (nl > leaf) next.push_back(L);
      if (hi - lo - nl > leaf) next.push_back(L + 1);
    }
    active.swap(next);
    ++level;
  }
}

}  // namespace

extern "C" {

int oracle_tree_depth(int64_t n, int32_t leaf) { return tree_depth(n, leaf); }

float oracle_project(const float* x, const float* v, int32_t d) { return project(x, v, d); }

float oracle_pair_key(const float* a, const float* b, int32_t d, int32_t metric) {
  if (metric == kEuclidean) return key_euclid(a, b, d);
  if (metric == kTaxicab) return key_taxicab(a, b, d);
  float na = std::sqrt(dot_chunked(a, a, d)), nb = std::sqrt(dot_chunked(b, b, d));
  return key_cosine_from(dot_chunked(a, b, d), na, nb);
}

// perm: [trees][n] leaf order of each tree.
int oracle_build_trees(const float* X, int64_t n, int32_t d, int32_t trees, int32_t leaf,
                       uint64_t seed, int32_t* perm, int32_t nthreads) {
  if (!X || n < 1 || d < 1 || trees < 1 || leaf < 1 || !perm) return -1;
  if (nthreads > 0) omp_set_num_threads(nthreads);
  Data D{X, n, d, kEuclidean, {}};
#pragma omp parallel for schedule(dynamic, 1)
  for (int t = 0; t < trees; ++t) build_tree(D, t, leaf, seed, perm + (size_t)t * n);
  return 0;
}

// Initial k-NN from given trees. out_key holds keys (squared L2 / L1 / 1-cos).
// Trees with global indices tree_offset + t * tree_stride (a rank's share of a
// sharded build); oracle_build_trees is offset 0, stride 1.
int oracle_build_trees_ex(const float* X, int64_t n, int32_t d, int32_t trees, int32_t leaf, uint64_t seed,
                          int32_t tree_offset, int32_t tree_stride, int32_t* perm, int32_t nthreads) {
  if (!X || n < 1 || d < 1 || trees < 1 || leaf < 1 || !perm || tree_offset < 0 || tree_stride < 1) return -1;
  if (nthreads > 0) omp_set_num_threads(nthreads);
  Data D{X, n, d, kEuclidean, {}};
#pragma omp parallel for schedule(dynamic, 1)
  for (int t = 0; t < trees; ++t) build_tree(D, tree_offset + t * tree_stride, leaf, seed, perm + (size_t)t * n);
  return 0;
}
int oracle_leaf_stage(const float* X, int64_t n, int32_t d, int32_t k, int32_t trees,
                      int32_t leaf, int32_t metric, const int32_t* perm, int32_t* out_idx,
                      float* out_key, int32_t nthreads) {
  if (!X || n < 1 || d < 1 || k < 1 || n <= k || trees < 1 || leaf < 1) return -1;
  if (nthreads > 0) omp_set_num_threads(nthreads);
  Data D{X, n, d, metric, {}};
  prepare(D);
  const int depth = tree_depth(n, leaf);
  const int64_t nleaves = int64_t(1) << depth;
  std::vector<std::vector<Cand>> lists(n);
  for (int t = 0; t < trees; ++t) {
    const int32_t* pm = perm + (size_t)t * n;
#pragma omp parallel for schedule(dynamic, 16)
    for (int64_t j = 0; j < nleaves; ++j) {
      const int64_t lo = node_lo(n, depth, j), hi = node_lo(n, depth, j + 1);
      int bl = depth;
      int64_t bj = j;
      while (bl > 0 && node_lo(n, bl, bj + 1) - node_lo(n, bl, bj) < k + 1) {
        --bl;
        bj >>= 1;
      }
      const int64_t blo = node_lo(n, bl, bj), bhi = node_lo(n, bl, bj + 1);
      std::vector<Cand> add;
      std::vector<int32_t> ids;
      std::vector<float> keys;
      for (int64_t q = lo; q < hi; ++q) {
        const int32_t i = pm[q];
        ids.clear();
        for (int64_t c = blo; c < bhi; ++c)
          if (pm[c] != i) ids.push_back(pm[c]);
        keys.resize(ids.size());
        D.keys(i, ids.data(), (int64_t)ids.size(), keys.data());
        add_below_tail(lists[i], k, ids.data(), keys.data(), (int64_t)ids.size(), add);
        merge_topk(lists[i], add, k);
      }
    }
  }
  for (int64_t i = 0; i < n; ++i)
    for (int s = 0; s < k; ++s) {
      out_idx[i * k + s] = lists[i][s].id;
      out_key[i * k + s] = lists[i][s].key;
    }
  return 0;
}

// One Jacobi propagation step on keys.
int oracle_propagate(const float* X, int64_t n, int32_t d, int32_t k, int32_t metric,
                     const int32_t* idx_in, const float* key_in, int32_t* idx_out,
                     float* key_out, int32_t nthreads) {
  if (!X || n < 1 || d < 1 || k < 1) return -1;
  if (nthreads > 0) omp_set_num_threads(nthreads);
  Data D{X, n, d, metric, {}};
  prepare(D);
#pragma omp parallel
  {
    std::vector<Cand> list, add;
    std::vector<int32_t> ids, fresh;
    std::vector<float> keys;
#pragma omp for schedule(dynamic, 64)
    for (int64_t i = 0; i < n; ++i) {
      list.clear();
      for (int s = 0; s < k; ++s) list.push_back({key_in[i * k + s], idx_in[i * k + s]});
      ids.clear();
      for (int s = 0; s < k; ++s) {
        const int32_t a = idx_in[i * k + s];
        for (int r = 0; r < k; ++r) {
          const int32_t jj = idx_in[(int64_t)a * k + r];
          if (jj == (int32_t)i) continue;
          ids.push_back(jj);
        }
      }
      std::sort(ids.begin(), ids.end());
      ids.erase(std::unique(ids.begin(), ids.end()), ids.end());
      fresh.clear();
      for (int32_t jj : ids) {
        bool in_list = false;
        for (int s = 0; s < k; ++s) in_list |= (list[s].id == jj);
        if (!in_list) fresh.push_back(jj);
      }
      keys.resize(fresh.size());
      D.keys(i, fresh.data(), (int64_t)fresh.size(), keys.data());
      add_below_tail(list, k, fresh.data(), keys.data(), (int64_t)fresh.size(), add);
      merge_topk(list, add, k);
      for (int s = 0; s < k; ++s) {
        idx_out[i * k + s] = list[s].id;
        key_out[i * k + s] = list[s].key;
      }
    }
  }
  return 0;
}

// Key -> reported distance (sqrt for EUCLIDEAN).
void oracle_finalize(int64_t count, int32_t metric, const float* key, float* dist) {
  for (int64_t i = 0; i < count; ++i) dist[i] = metric == kEuclidean ? std::sqrt(key[i]) : key[i];
}

// Whole path: trees -> leaf stage -> props x propagation -> sorted (dist, idx).
int oracle_knn_build(const float* X, int64_t n, int32_t d, int32_t k, int32_t trees,
                     int32_t leaf, int32_t props, int32_t metric, uint64_t seed,
                     int32_t* out_idx, float* out_dist, int32_t nthreads) {
  if (!X || !out_idx || !out_dist) return -1;
  if (n < 1 || d < 1 || k < 1 || trees < 1 || leaf < 1 || props < 0) return -1;
  if (metric < 0 || metric > 2) return -1;
  if (n <= k) return -2;
  std::vector<int32_t> perm((size_t)trees * n);
  int rc = oracle_build_trees(X, n, d, trees, leaf, seed, perm.data(), nthreads);
  if (rc) return rc;
  std::vector<int32_t> ia((size_t)n * k), ib((size_t)n * k);
  std::vector<float> ka((size_t)n * k), kb((size_t)n * k);
  rc = oracle_leaf_stage(X, n, d, k, trees, leaf, metric, perm.data(), ia.data(), ka.data(),
                         nthreads);
  if (rc) return rc;
  for (int p = 0; p < props; ++p) {
    rc = oracle_propagate(X, n, d, k, metric, ia.data(), ka.data(), ib.data(), kb.data(),
                          nthreads);
    if (rc) return rc;
    ia.swap(ib);
    ka.swap(kb);
  }
  std::memcpy(out_idx, ia.data(), ia.size() * sizeof(int32_t));
  oracle_finalize((int64_t)ka.size(), metric, ka.data(), out_dist);
  return 0;
}

// FP64 exact k-NN of the given query ids against all n points (self excluded),
// ties by index.  dist: sqrt(sum sq) / sum |.| / 1 - cos, in double.
// The whole build with reference-rule trees: leaves are the nodes that were
// not split; a leaf's block is its smallest ancestor-or-self with at least
// k+1 points.
int oracle_knn_build_faithful(const float* X, int64_t n, int32_t d, int32_t k, int32_t trees, int32_t leaf,
                              int32_t props, int32_t metric, uint64_t seed, int32_t* out_idx, float* out_dist,
                              int32_t nthreads) {
  if (!X || !out_idx || !out_dist || n < 1 || d < 1 || k < 1 || trees < 1 || leaf < 1 || props < 0) return -1;
  if (metric < 0 || metric > 2) return -1;
  if (n <= k) return -2;
  if (nthreads > 0) omp_set_num_threads(nthreads);
  Data D{X, n, d, metric, {}};
  prepare(D);
  std::vector<int32_t> perm((size_t)trees * n);
  std::vector<std::vector<FNodeO>> nodes(trees);
#pragma omp parallel for schedule(dynamic, 1)
  for (int t = 0; t < trees; ++t) build_tree_faithful(D, t, leaf, seed, perm.data() + (size_t)t * n, nodes[t]);
  std::vector<std::vector<Cand>> lists(n);
  for (int t = 0; t < trees; ++t) {
    const int32_t* pm = perm.data() + (size_t)t * n;
    std::vector<int64_t> leaves;
    for (int64_t j = 0; j < (int64_t)nodes[t].size(); ++j)
      if (!nodes[t][j].split) leaves.push_back(j);
#pragma omp parallel for schedule(dynamic, 16)
    for (int64_t li = 0; li < (int64_t)leaves.size(); ++li) {
      const FNodeO& lf = nodes[t][leaves[li]];
      int64_t b = leaves[li];
      while (nodes[t][b].hi - nodes[t][b].lo < k + 1 && nodes[t][b].parent >= 0) b = nodes[t][b].parent;
      const int64_t blo = nodes[t][b].lo, bhi = nodes[t][b].hi;
      std::vector<Cand> add;
      for (int64_t q = lf.lo; q < lf.hi; ++q) {
        const int32_t i = pm[q];
        add.clear();
        for (int64_t c = blo; c < bhi; ++c) {
          const int32_t jj = pm[c];
          if (jj == i) continue;
          add.push_back({D.key(i, jj), jj});
        }
        merge_topk(lists[i], add, k);
      }
    }
  }
  std::vector<int32_t> ia((size_t)n * k), ib((size_t)n * k);
  std::vector<float> ka((size_t)n * k), kb((size_t)n * k);
  for (int64_t i = 0; i < n; ++i)
    for (int s = 0; s < k; ++s) {
      ia[i * k + s] = lists[i][s].id;
      ka[i * k + s] = lists[i][s].key;
    }
  for (int p = 0; p < props; ++p) {
    int rc = oracle_propagate(X, n, d, k, metric, ia.data(), ka.data(), ib.data(), kb.data(), nthreads);
    if (rc) return rc;
    ia.swap(ib);
    ka.swap(kb);
  }
  std::memcpy(out_idx, ia.data(), ia.size() * sizeof(int32_t));
  oracle_finalize((int64_t)ka.size(), metric, ka.data(), out_dist);
  return 0;
}

int oracle_exact_knn(const float* X, int64_t n, int32_t d, int32_t k, int32_t metric,
                     const int64_t* queries, int64_t nq, int32_t* out_idx, double* out_dist,
                     int32_t nthreads) {
  if (!X || n < 1 || d < 1 || k < 1 || n <= k || !queries || nq < 0) return -1;
  if (nthreads > 0) omp_set_num_threads(nthreads);
  std::vector<double> norms;
  if (metric == kCosine) {
    norms.resize(n);
#pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < n; ++i) {
      double s = 0;
      for (int e = 0; e < d; ++e) s += (double)X[i * d + e] * (double)X[i * d + e];
      norms[i] = std::sqrt(s);
    }
  }
#pragma omp parallel
  {
    std::vector<std::pair<double, int32_t>> all(n);
#pragma omp for schedule(dynamic, 4)
    for (int64_t qi = 0; qi < nq; ++qi) {
      const int64_t q = queries[qi];
      const float* a = X + q * d;
      int64_t m = 0;
      for (int64_t j = 0; j < n; ++j) {
        if (j == q) continue;
        const float* b = X + j * d;
        double s = 0;
        if (metric == kEuclidean) {
          for (int e = 0; e < d; ++e) {
            double t = (double)a[e] - (double)b[e];
            s += t * t;
          }
          s = std::sqrt(s);
        } else if (metric == kTaxicab) {
          for (int e = 0; e < d; ++e) s += std::fabs((double)a[e] - (double)b[e]);
        } else {
          for (int e = 0; e < d; ++e) s += (double)a[e] * (double)b[e];
          double den = norms[q] * norms[j];
          s = den == 0.0 ? 1.0 : 1.0 - s / den;
        }
        all[m++] = {s, (int32_t)j};
      }
      std::partial_sort(all.begin(), all.begin() + k, all.begin() + m);
      for (int s = 0; s < k; ++s) {
        out_idx[qi * k + s] = all[s].second;
        out_dist[qi * k + s] = all[s].first;
      }
    }
  }
  return 0;
}

// FP64 distance of given pairs (i, j) (for the distance-error report).
int oracle_pair_dist_fp64(const float* X, int64_t n, int32_t d, int32_t metric,
                          const int64_t* qi, const int32_t* cj, int64_t count, double* out) {
  if (!X || n < 1 || d < 1) return -1;
#pragma omp parallel for schedule(static)
  for (int64_t p = 0; p < count; ++p) {
    const float* a = X + qi[p] * d;
    const float* b = X + (int64_t)cj[p] * d;
    double s = 0;
    if (metric == kEuclidean) {
      for (int e = 0; e < d; ++e) {
        double t = (double)a[e] - (double)b[e];
        s += t * t;
      }
      s = std::sqrt(s);
    } else if (metric == kTaxicab) {
      for (int e = 0; e < d; ++e) s += std::fabs((double)a[e] - (double)b[e]);
    } else {
      double aa = 0, bb = 0;
      for (int e = 0; e < d; ++e) {
        s += (double)a[e] * (double)b[e];
        aa += (double)a[e] * (double)a[e];
        bb += (double)b[e] * (double)b[e];
      }
      double den = std::sqrt(aa) * std::sqrt(bb);
      s = den == 0.0 ? 1.0 : 1.0 - s / den;
    }
    out[p] = s;
  }
  return 0;
}

// ---- learned split network, FP64 -------------------------------------------
// f(x) = W2 gelu(W1 x + b1) + b2 on already-standardised rows x [d];
// params = W1 [256][d], b1 [256], W2 [64][256], b2 [64].
static const int kOH = 256, kOE = 64;

static double o_gelu(double a) {
  const double c = 0.7978845608028654, u = c * (a + 0.044715 * a * a * a);
  return 0.5 * a * (1.0 + std::tanh(u));
}
static double o_gelu_grad(double a) {
  const double c = 0.7978845608028654, u = c * (a + 0.044715 * a * a * a), t = std::tanh(u);
  return 0.5 * (1.0 + t) + 0.5 * a * (1.0 - t * t) * c * (1.0 + 3.0 * 0.044715 * a * a);
}

// Z [m][64] = f(rows) for m rows [m][d].
int oracle_mlp_forward(const float* params, int32_t d, const float* rows, int64_t m, double* Z) {
  const float* W1 = params;
  const float* b1 = W1 + (size_t)kOH * d;
  const float* W2 = b1 + kOH;
  const float* b2 = W2 + (size_t)kOE * kOH;
  std::vector<double> g(kOH);
  for (int64_t r = 0; r < m; ++r) {
    const float* x = rows + r * d;
    for (int h = 0; h < kOH; ++h) {
      double a = b1[h];
      for (int c = 0; c < d; ++c) a += (double)W1[(size_t)h * d + c] * x[c];
      g[h] = o_gelu(a);
    }
    for (int e = 0; e < kOE; ++e) {
      double z = b2[e];
      for (int h = 0; h < kOH; ++h) z += (double)W2[(size_t)e * kOH + h] * g[h];
      Z[r * kOE + e] = z;
    }
  }
  return 0;
}

// Mean triplet loss over B triplets of rows [3B][d] (anchors, positives,
// negatives) and its gradient with respect to params.
int oracle_mlp_loss_grad(const float* params, int32_t d, const float* rows, int32_t B, double margin,
                         double* grad, double* loss, double* hinge) {
  const float* W1 = params;
  const float* W2 = W1 + (size_t)kOH * d + kOH;
  const size_t np = (size_t)kOH * d + kOH + (size_t)kOE * kOH + kOE;
  double* gW1 = grad;
  double* gb1 = gW1 + (size_t)kOH * d;
  double* gW2 = gb1 + kOH;
  double* gb2 = gW2 + (size_t)kOE * kOH;
  std::fill(grad, grad + np, 0.0);
  const int R = 3 * B;
  std::vector<double> A((size_t)R * kOH), G((size_t)R * kOH), Z((size_t)R * kOE), dZ((size_t)R * kOE, 0.0);
  const float* b1 = W1 + (size_t)kOH * d;
  const float* b2 = W2 + (size_t)kOE * kOH;
  for (int r = 0; r < R; ++r) {
    const float* x = rows + (size_t)r * d;
    for (int h = 0; h < kOH; ++h) {
      double a = b1[h];
      for (int c = 0; c < d; ++c) a += (double)W1[(size_t)h * d + c] * x[c];
      A[(size_t)r * kOH + h] = a;
      G[(size_t)r * kOH + h] = o_gelu(a);
    }
    for (int e = 0; e < kOE; ++e) {
      double z = b2[e];
      for (int h = 0; h < kOH; ++h) z += (double)W2[(size_t)e * kOH + h] * G[(size_t)r * kOH + h];
      Z[(size_t)r * kOE + e] = z;
    }
  }
  double L = 0.0;
  for (int b = 0; b < B; ++b) {
    const double* za = &Z[(size_t)b * kOE];
    const double* zp = &Z[(size_t)(B + b) * kOE];
    const double* zn = &Z[(size_t)(2 * B + b) * kOE];
    double dap = 0, dan = 0;
    for (int e = 0; e < kOE; ++e) {
      dap += (za[e] - zp[e]) * (za[e] - zp[e]);
      dan += (za[e] - zn[e]) * (za[e] - zn[e]);
    }
    const double l = margin + dap - dan;
    if (hinge) hinge[b] = l;
    if (l <= 0) continue;
    L += l / B;
    const double s = 2.0 / B;
    for (int e = 0; e < kOE; ++e) {
      const double u = za[e] - zp[e], w = za[e] - zn[e];
      dZ[(size_t)b * kOE + e] += s * (u - w);
      dZ[(size_t)(B + b) * kOE + e] += -s * u;
      dZ[(size_t)(2 * B + b) * kOE + e] += s * w;
    }
  }
  *loss = L;
  std::vector<double> dA(kOH);
  for (int r = 0; r < R; ++r) {
    const double* dz = &dZ[(size_t)r * kOE];
    for (int e = 0; e < kOE; ++e) {
      gb2[e] += dz[e];
      for (int h = 0; h < kOH; ++h) gW2[(size_t)e * kOH + h] += dz[e] * G[(size_t)r * kOH + h];
    }
    for (int h = 0; h < kOH; ++h) {
      double s = 0;
      for (int e = 0; e < kOE; ++e) s += dz[e] * W2[(size_t)e * kOH + h];
      dA[h] = s * o_gelu_grad(A[(size_t)r * kOH + h]);
      gb1[h] += dA[h];
    }
    const float* x = rows + (size_t)r * d;
    for (int h = 0; h < kOH; ++h)
      for (int c = 0; c < d; ++c) gW1[(size_t)h * d + c] += dA[h] * x[c];
  }
  return 0;
}

}  // extern "C"
