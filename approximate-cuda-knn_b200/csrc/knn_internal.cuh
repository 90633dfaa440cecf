// Internal device/host definitions shared by the k-NN graph kernels.
//
// Arithmetic conventions (all translation units are built with --fmad=false so
// that only the explicit __fmaf_rn below are fused; sqrt and division are IEEE):
//   * pair keys: squared L2 (EUCLIDEAN), L1 (TAXICAB), 1 - cos (COSINE), summed
//     sequentially within 256-dim chunks and chunk partials added to a running
//     total -- the summation order of the reference's distance loops
//     (euclideandistancematrixgpu.cu:243-264, :540-556, :840-868);
//   * projections for the tree splits: grouped float4 lanes + xor butterfly
//     (proj_group / group_project below);
//   * candidate order: (key, id) ascending, ids compared unsigned.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include "../../include/knn.h"

namespace knn {

constexpr int kWarp = 32;
constexpr uint32_t kIdMask = 0x7FFFFFFFu;  // id bits; bit 31 = "new" flag
constexpr uint32_t kNoId = 0xFFFFFFFFu;
constexpr int kMaxK = 128;

// --------------------------------------------------------------- hashing --
__host__ __device__ __forceinline__ uint64_t splitmix64(uint64_t x) {
  x += 0x9E3779B97F4A7C15ull;
  uint64_t z = x;
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
  return z ^ (z >> 31);
}

// Two distinct member positions of a node with n >= 2 points; replaces the
// per-level rand() pair of euclideandistancematrixgpu.cu:2329-2333.
__host__ __device__ __forceinline__ void pivot_positions(uint64_t seed, int tree, int level,
                                                         int64_t node, int64_t n, int64_t* p1,
                                                         int64_t* p2) {
  uint64_t z = splitmix64(seed + 0x9E3779B97F4A7C15ull * (uint64_t)(tree + 1));
  z = splitmix64(z ^ (((uint64_t)level << 40) | (uint64_t)node));
  int64_t a = (int64_t)((z & 0xFFFFFFFFull) % (uint64_t)n);
  int64_t b = (int64_t)((z >> 32) % (uint64_t)n);
  if (a == b) b = (a + 1) % n;
  *p1 = a;
  *p2 = b;
}

// ------------------------------------------------------------ tree shape --
// Node j of level l covers leaf-order positions [lo(l,j), lo(l,j+1)).
// n < 2^31 and level <= 31 keep every product below 2^63.
__host__ __device__ __forceinline__ int64_t node_lo(int64_t n, int level, int64_t j) {
  return (int64_t)(((uint64_t)j * (uint64_t)n) >> level);
}
// Node of level l that contains position p: the largest j with lo(l,j) <= p,
// i.e. ceil((p+1) 2^l / n) - 1.
__host__ __device__ __forceinline__ int64_t node_of(int64_t n, int level, int64_t p) {
  const uint64_t num = (uint64_t)(p + 1) << level;
  return (int64_t)((num + (uint64_t)n - 1) / (uint64_t)n) - 1;
}
inline int tree_depth(int64_t n, int leaf) {
  int l = 0;
  while (((n + (int64_t(1) << l) - 1) >> l) > leaf) ++l;
  return l;
}

// ------------------------------------------------------------------ scan --
// Block-wide exclusive scan of one value per thread; returns the exclusive
// prefix and writes the block total to *total.
__device__ __forceinline__ int64_t block_excl_scan(int64_t v, int64_t* warp_sums, int64_t* total) {
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5, nw = blockDim.x >> 5;
  int64_t incl = v;
#pragma unroll
  for (int off = 1; off < 32; off <<= 1) {
    int64_t o = __shfl_up_sync(0xFFFFFFFFu, incl, off);
    if (lane >= off) incl += o;
  }
  if (lane == 31) warp_sums[w] = incl;
  __syncthreads();
  if (w == 0) {
    int64_t s = lane < nw ? warp_sums[lane] : 0;
    int64_t si = s;
#pragma unroll
    for (int off = 1; off < 32; off <<= 1) {
      int64_t o = __shfl_up_sync(0xFFFFFFFFu, si, off);
      if (lane >= off) si += o;
    }
    if (lane < nw) warp_sums[lane] = si - s;
    if (lane == 31) warp_sums[32] = si;
  }
  __syncthreads();
  const int64_t r = warp_sums[w] + incl - v;
  *total = warp_sums[32];
  __syncthreads();
  return r;
}

// ------------------------------------------------------------- segments --
// A batch of independent point sets concatenated in one array.  Segment a
// holds the global positions / ids [off, off + n) and its trees have `depth`
// levels; ids in neighbour lists stay global while the batch is built.
// Segments are sorted by n descending (so by depth descending): the segments
// still splitting at level l are a prefix of the table.  leaf_base = leaves
// per tree of the segments before this one.
struct SegEntry {
  int64_t off, n;
  uint64_t seed;
  int64_t leaf_base;
  int32_t depth, pad;
};

struct SegView {
  const SegEntry* table;  // device; null: one segment {0, n0, seed0, depth0}
  const int32_t* seg_of;  // device [ntot]: segment of each point; null with one segment
  int count;
  int64_t n0;
  uint64_t seed0;
  int depth0;

  __device__ __forceinline__ SegEntry get(int a) const {
    if (table) return table[a];
    SegEntry e;
    e.off = 0;
    e.n = n0;
    e.seed = seed0;
    e.leaf_base = 0;
    e.depth = depth0;
    e.pad = 0;
    return e;
  }
  __device__ __forceinline__ int of(int64_t i) const { return seg_of ? seg_of[i] : 0; }
  // The segment holding flat leaf index b (per tree); *j = the leaf in it.
  __device__ __forceinline__ SegEntry leaf(int64_t b, int64_t* j) const {
    if (!table) {
      *j = b;
      return get(0);
    }
    int lo = 0, hi = count - 1;  // last segment with leaf_base <= b
    while (lo < hi) {
      const int mid = (lo + hi + 1) >> 1;
      if (table[mid].leaf_base <= b) lo = mid;
      else hi = mid - 1;
    }
    const SegEntry e = table[lo];
    *j = b - e.leaf_base;
    return e;
  }
};

inline SegView single_segment(int64_t n, uint64_t seed, int depth) {
  SegView v;
  v.table = nullptr;
  v.seg_of = nullptr;
  v.count = 1;
  v.n0 = n;
  v.seed0 = seed;
  v.depth0 = depth;
  return v;
}

// Global positions of leaf j of segment e and of its block, the smallest
// ancestor holding at least k+1 points (the climb of
// euclideandistancematrixgpu.cu:87-105).
__device__ __forceinline__ void leaf_block(const SegEntry& e, int64_t j, int k, int64_t* lo, int64_t* hi,
                                           int64_t* blo, int64_t* bhi) {
  *lo = e.off + node_lo(e.n, e.depth, j);
  *hi = e.off + node_lo(e.n, e.depth, j + 1);
  int bl = e.depth;
  int64_t bj = j;
  while (bl > 0 && node_lo(e.n, bl, bj + 1) - node_lo(e.n, bl, bj) < k + 1) {
    --bl;
    bj >>= 1;
  }
  *blo = e.off + node_lo(e.n, bl, bj);
  *bhi = e.off + node_lo(e.n, bl, bj + 1);
}

// -------------------------------------------------------------- ordering --
__host__ __device__ __forceinline__ uint32_t orderable(float f) {
#ifdef __CUDA_ARCH__
  uint32_t u = __float_as_uint(f);
#else
  uint32_t u;
  memcpy(&u, &f, 4);
#endif
  return (u & 0x80000000u) ? ~u : (u | 0x80000000u);
}
__host__ __device__ __forceinline__ uint64_t proj_key(float proj, uint32_t id) {
  return ((uint64_t)orderable(proj) << 32) | id;
}
__device__ __forceinline__ bool cand_less(float ka, uint32_t ia, float kb, uint32_t ib) {
  return ka < kb || (!(kb < ka) && (ia & kIdMask) < (ib & kIdMask));
}

// ------------------------------------------------------------ projection --
__host__ __device__ __forceinline__ int proj_group(int d) {
  int nc = (d + 3) / 4;
  int g = 1;
  while (g < nc && g < 4) g <<= 1;
  return g;
}

// x . v over dpad (multiple of 4, zero padded) dims by a group of G lanes.
// Every lane of the group returns the same value.
template <int G>
__device__ __forceinline__ float group_project(const float* __restrict__ x,
                                               const float* __restrict__ v, int dpad, int gl) {
  const float4* x4 = reinterpret_cast<const float4*>(x);
  const float4* v4 = reinterpret_cast<const float4*>(v);
  const int nc = dpad >> 2;
  float acc = 0.0f;
  for (int c = gl; c < nc; c += G) {
    float4 a = __ldg(x4 + c);
    float4 b = v4[c];
    acc = __fmaf_rn(a.x, b.x, acc);
    acc = __fmaf_rn(a.y, b.y, acc);
    acc = __fmaf_rn(a.z, b.z, acc);
    acc = __fmaf_rn(a.w, b.w, acc);
  }
#pragma unroll
  for (int off = G / 2; off >= 1; off >>= 1) acc = __fadd_rn(acc, __shfl_xor_sync(0xFFFFFFFFu, acc, off, G));
  return acc;
}

// Four projections of one row at once (directions v[0..3]), each summed in
// group_project's order, so each equals group_project's result bit for bit;
// the four chains and their loads overlap.
template <int G>
__device__ __forceinline__ void group_project4(const float* __restrict__ x, const float* const (&v)[4], int dpad,
                                               int gl, float (&out)[4]) {
  const float4* x4 = reinterpret_cast<const float4*>(x);
  const int nc = dpad >> 2;
  float acc[4] = {0.0f, 0.0f, 0.0f, 0.0f};
  for (int c = gl; c < nc; c += G) {
    const float4 a = __ldg(x4 + c);
    float4 b[4];
#pragma unroll
    for (int u = 0; u < 4; ++u) b[u] = __ldg(reinterpret_cast<const float4*>(v[u]) + c);
#pragma unroll
    for (int u = 0; u < 4; ++u) {
      acc[u] = __fmaf_rn(a.x, b[u].x, acc[u]);
      acc[u] = __fmaf_rn(a.y, b[u].y, acc[u]);
      acc[u] = __fmaf_rn(a.z, b[u].z, acc[u]);
      acc[u] = __fmaf_rn(a.w, b[u].w, acc[u]);
    }
  }
#pragma unroll
  for (int off = G / 2; off >= 1; off >>= 1)
#pragma unroll
    for (int u = 0; u < 4; ++u) acc[u] = __fadd_rn(acc[u], __shfl_xor_sync(0xFFFFFFFFu, acc[u], off, G));
#pragma unroll
  for (int u = 0; u < 4; ++u) out[u] = acc[u];
}

// ------------------------------------------------------------- pair keys --
__device__ __forceinline__ float cosine_key(float dot, float na, float nb) {
  if (na == 0.0f || nb == 0.0f) return 1.0f;
  return __fsub_rn(1.0f, __fdiv_rn(dot, __fmul_rn(na, nb)));
}

// Per-dim accumulation step of each metric.
template <int METRIC>
__device__ __forceinline__ float acc_step(float q, float c, float part) {
  if (METRIC == KNN_METRIC_EUCLIDEAN) {
    float df = __fsub_rn(q, c);
    return __fmaf_rn(df, df, part);
  } else if (METRIC == KNN_METRIC_TAXICAB) {
    return __fadd_rn(part, fabsf(__fsub_rn(q, c)));
  } else {
    return __fmaf_rn(q, c, part);
  }
}

// Sequential 256-chunked key between two rows (thread-local), used for norms.
__device__ __forceinline__ float self_dot_chunked(const float* __restrict__ a, int d) {
  float total = 0.0f;
  for (int c0 = 0; c0 < d; c0 += 256) {
    float part = 0.0f;
    int c1 = min(d, c0 + 256);
    for (int i = c0; i < c1; ++i) part = __fmaf_rn(a[i], a[i], part);
    total = __fadd_rn(total, part);
  }
  return total;
}

// ------------------------------------------------------ warp top-k lists --
// A sorted list of 32*KPL (key, id) entries held by one warp: entry e lives in
// register e/32 of lane e%32.  Bit 31 of an id is a caller-defined flag and is
// ignored by comparisons.  K is float (keys) or double (exact k-NN).
__device__ __forceinline__ bool cand_less(double ka, uint32_t ia, double kb, uint32_t ib) {
  return ka < kb || (!(kb < ka) && (ia & kIdMask) < (ib & kIdMask));
}

template <int KPL, typename K = float>
struct WarpList {
  K key[KPL];
  uint32_t id[KPL];
};

template <typename K>
__device__ __forceinline__ void cmp_swap_lane(K& k, uint32_t& id, int mask, bool up) {
  // Exchange with lane ^ mask; the lower lane keeps the smaller when `up`.
  const int lane = threadIdx.x & 31;
  const K ok = __shfl_xor_sync(0xFFFFFFFFu, k, mask);
  const uint32_t oid = __shfl_xor_sync(0xFFFFFFFFu, id, mask);
  const bool lower = (lane & mask) == 0;
  const bool take_small = (lower == up);
  if (take_small ? cand_less(ok, oid, k, id) : cand_less(k, id, ok, oid)) {
    k = ok;
    id = oid;
  }
}

// Bitonic merge of a bitonic 32-sequence (one entry per lane) into ascending order.
template <typename K>
__device__ __forceinline__ void warp_bitonic_merge32(K& k, uint32_t& id) {
#pragma unroll
  for (int m = 16; m >= 1; m >>= 1) cmp_swap_lane(k, id, m, true);
}

// Full bitonic sort of 32 entries (one per lane), ascending.
template <typename K>
__device__ __forceinline__ void warp_bitonic_sort32(K& k, uint32_t& id) {
  const int lane = threadIdx.x & 31;
#pragma unroll
  for (int size = 2; size <= 32; size <<= 1) {
    const bool up = (lane & size) == 0;
#pragma unroll
    for (int m = size >> 1; m >= 1; m >>= 1) cmp_swap_lane(k, id, m, up);
  }
}

// Merge two ascending 32-lists a and b: a <- 32 smallest, b <- 32 largest.
template <typename K>
__device__ __forceinline__ void warp_merge_pair(K& ak, uint32_t& ai, K& bk, uint32_t& bi) {
  const int lane = threadIdx.x & 31;
  const K rk = __shfl_sync(0xFFFFFFFFu, bk, 31 - lane);
  const uint32_t ri = __shfl_sync(0xFFFFFFFFu, bi, 31 - lane);
  const K lk = ak;
  const uint32_t li = ai;
  // min(a, reversed b) and max(a, reversed b) are both bitonic.
  if (cand_less(rk, ri, lk, li)) {
    ak = rk;
    ai = ri;
    bk = lk;
    bi = li;
  } else {
    ak = lk;
    ai = li;
    bk = rk;
    bi = ri;
  }
  warp_bitonic_merge32(ak, ai);
  warp_bitonic_merge32(bk, bi);
}

// a <- the 32 smallest of two ascending 32-lists a and b (b is left as is).
template <typename K>
__device__ __forceinline__ void warp_merge_lower(K& ak, uint32_t& ai, K bk, uint32_t bi) {
  const int lane = threadIdx.x & 31;
  const K rk = __shfl_sync(0xFFFFFFFFu, bk, 31 - lane);
  const uint32_t ri = __shfl_sync(0xFFFFFFFFu, bi, 31 - lane);
  if (cand_less(rk, ri, ak, ai)) {  // min(a, reversed b) is bitonic
    ak = rk;
    ai = ri;
  }
  warp_bitonic_merge32(ak, ai);
}

// Insert 32 candidates (one per lane, unsorted, +inf for none) into the list,
// keeping its 32*KPL smallest.  The 32*KPL smallest of list u candidates are
// the first KPL-1 registers plus the 32 smallest of (last register u
// candidates); that block is then merged down through the sorted registers.
template <int KPL, typename K>
__device__ __forceinline__ void warp_list_insert(WarpList<KPL, K>& L, K ck, uint32_t ci) {
  const int lane = threadIdx.x & 31;
  warp_bitonic_sort32(ck, ci);
  const K rk = __shfl_sync(0xFFFFFFFFu, ck, 31 - lane);
  const uint32_t ri = __shfl_sync(0xFFFFFFFFu, ci, 31 - lane);
  K& tk = L.key[KPL - 1];
  uint32_t& ti = L.id[KPL - 1];
  if (cand_less(rk, ri, tk, ti)) {
    tk = rk;
    ti = ri;
  }
  warp_bitonic_merge32(tk, ti);
#pragma unroll
  for (int r = KPL - 2; r >= 0; --r) warp_merge_pair(L.key[r], L.id[r], L.key[r + 1], L.id[r + 1]);
}

// One-register list (32 entries, ascending across lanes): insert the
// warp-uniform candidate (c, i).  The lanes whose entry is greater than the
// candidate form a suffix; its first lane takes the candidate, the suffix
// shifts up one lane and lane 31's entry drops out.
__device__ __forceinline__ void warp_insert1(float& lk, uint32_t& li, float c, uint32_t i) {
  const int lane = threadIdx.x & 31;
  const uint32_t after = __ballot_sync(0xFFFFFFFFu, cand_less(c, i, lk, li));
  const float uk = __shfl_up_sync(0xFFFFFFFFu, lk, 1);
  const uint32_t ui = __shfl_up_sync(0xFFFFFFFFu, li, 1);
  if (after) {
    const int pos = __ffs(after) - 1;
    if (lane > pos) {
      lk = uk;
      li = ui;
    } else if (lane == pos) {
      lk = c;
      li = i;
    }
  }
}

// Insert one warp-uniform candidate: entries from its rank on shift down one
// slot and the last entry drops out.  ~10 instructions per register.
template <int KPL, typename K>
__device__ __forceinline__ void warp_list_insert_one(WarpList<KPL, K>& L, K ck, uint32_t ci) {
  const int lane = threadIdx.x & 31;
  int pos = 0;
#pragma unroll
  for (int r = 0; r < KPL; ++r) pos += __popc(__ballot_sync(0xFFFFFFFFu, cand_less(L.key[r], L.id[r], ck, ci)));
#pragma unroll
  for (int r = KPL - 1; r >= 0; --r) {
    K up_k = __shfl_up_sync(0xFFFFFFFFu, L.key[r], 1);
    uint32_t up_i = __shfl_up_sync(0xFFFFFFFFu, L.id[r], 1);
    if (r > 0) {
      const K pk = __shfl_sync(0xFFFFFFFFu, L.key[r - 1], 31);
      const uint32_t pi = __shfl_sync(0xFFFFFFFFu, L.id[r - 1], 31);
      if (lane == 0) {
        up_k = pk;
        up_i = pi;
      }
    }
    const int e = r * 32 + lane;
    if (e > pos) {
      L.key[r] = up_k;
      L.id[r] = up_i;
    } else if (e == pos) {
      L.key[r] = ck;
      L.id[r] = ci;
    }
  }
}

// Insert the candidates of the lanes in `bal` (one per lane): one at a time
// when there are few, else by bitonic sort + merge.
template <int KPL, typename K>
__device__ __forceinline__ void warp_list_insert_lanes(WarpList<KPL, K>& L, uint32_t bal, K ck,
                                                       uint32_t ci, K inf_key) {
  if (__popc(bal) <= 3) {
    while (bal) {
      const int src = __ffs(bal) - 1;
      bal &= bal - 1;
      const K k1 = __shfl_sync(0xFFFFFFFFu, ck, src);
      const uint32_t i1 = __shfl_sync(0xFFFFFFFFu, ci, src);
      warp_list_insert_one(L, k1, i1);
    }
  } else {
    const bool mine = (bal >> (threadIdx.x & 31)) & 1u;
    warp_list_insert(L, mine ? ck : inf_key, mine ? ci : kNoId);
  }
}

// Entry e of the list (broadcast to all lanes).
template <int KPL, typename K>
__device__ __forceinline__ void warp_list_get(const WarpList<KPL, K>& L, int e, K& k, uint32_t& id) {
  const int r = e >> 5, src = e & 31;
  K kk = 0;
  uint32_t ii = 0;
#pragma unroll
  for (int q = 0; q < KPL; ++q)
    if (q == r) {
      kk = L.key[q];
      ii = L.id[q];
    }
  k = __shfl_sync(0xFFFFFFFFu, kk, src);
  id = __shfl_sync(0xFFFFFFFFu, ii, src);
}

// True when id (bits 0..30) equals the id of any of the first k list entries.
template <int KPL, typename K>
__device__ __forceinline__ bool warp_list_contains(const WarpList<KPL, K>& L, uint32_t id, int k) {
  bool hit = false;
  const uint32_t want = id & kIdMask;
#pragma unroll
  for (int r = 0; r < KPL; ++r) {
#pragma unroll 8
    for (int src = 0; src < 32; ++src) {
      const uint32_t o = __shfl_sync(0xFFFFFFFFu, L.id[r], src);
      hit |= ((o & kIdMask) == want) && (r * 32 + src < k);
    }
  }
  return hit;
}

inline int kpl_for(int k) { return k <= 32 ? 1 : (k <= 64 ? 2 : 4); }

}  // namespace knn
