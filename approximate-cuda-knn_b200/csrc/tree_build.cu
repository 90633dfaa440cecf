// Random-projection tree build, all trees level by level.
//
// Replaces buildUpTheTrees + makePartitionOfLeaf0..9
// (euclideandistancematrixgpu.cu:2130-2405, :2407-2686).  Differences by design:
//   * a tree is only a permutation of point ids (its leaf order); node j of
//     level l covers positions [floor(j n / 2^l), floor((j+1) n / 2^l)), so no
//     node records, no host round trip of the trees (.cu:2642-2655) and no
//     per-level host sync on a "there was a split" flag (.cu:2602-2604);
//   * split direction v = x[p2] - x[p1] of two member points (as .cu:2145-2160)
//     with p1, p2 drawn per node from a counter hash instead of one rand() pair
//     per level (.cu:2329-2333);
//   * the split is at the node median of (projection, id) -- a per-node radix
//     select -- followed by a stable partition, instead of the sign test against
//     0 (.cu:2160) and the atomicInc scatter (.cu:2205-2260).
// Every kernel is deterministic; the tree equals the CPU restatement's.
#include "knn_internal.cuh"
#include "knn_kernels.cuh"

namespace knn {

// One warp per (active segment, tree, node) of `level`: direction
// x[b] - x[a] of two member points.  Global positions index the perm rows.
__global__ void k_directions(const float* __restrict__ X, int dpad, int64_t ntot, int level,
                             int trees, const int32_t* __restrict__ perm, float* __restrict__ dirs,
                             SegView segs, int active, int tree_offset, int tree_stride) {
  const int64_t nodes = int64_t(1) << level;
  const int64_t gw = (int64_t)(blockIdx.x * (blockDim.x >> 5)) + (threadIdx.x >> 5);
  const int lane = threadIdx.x & 31;
  if (gw >= nodes * trees * active) return;
  const int a = (int)(gw / (nodes * trees));
  const int64_t r = gw - (int64_t)a * nodes * trees;
  const int t = (int)(r / nodes);
  const int64_t j = r - (int64_t)t * nodes;
  const SegEntry e = segs.get(a);
  const int64_t lo = e.off + node_lo(e.n, level, j), hi = e.off + node_lo(e.n, level, j + 1);
  const int64_t cnt = hi - lo;
  float4* v4 = reinterpret_cast<float4*>(dirs + (size_t)gw * dpad);
  const int nc = dpad >> 2;
  if (cnt < 2) {
    for (int c = lane; c < nc; c += 32) v4[c] = make_float4(0.f, 0.f, 0.f, 0.f);
    return;
  }
  int64_t p1, p2;
  pivot_positions(e.seed, tree_offset + t * tree_stride, level, j, cnt, &p1, &p2);
  const int32_t ia = perm[(size_t)t * ntot + lo + p1];
  const int32_t ib = perm[(size_t)t * ntot + lo + p2];
  const float4* xa = reinterpret_cast<const float4*>(X + (size_t)ia * dpad);
  const float4* xb = reinterpret_cast<const float4*>(X + (size_t)ib * dpad);
  for (int c = lane; c < nc; c += 32) {
    float4 u = __ldg(xa + c), w = __ldg(xb + c);
    v4[c] = make_float4(__fsub_rn(w.x, u.x), __fsub_rn(w.y, u.y), __fsub_rn(w.z, u.z),
                        __fsub_rn(w.w, u.w));
  }
}

// Keys of every (tree, position): (orderable projection << 32) | id, computed
// point-major: a group of G lanes takes one point, reads its row once (the
// re-reads for the other trees hit L1) and projects it on the direction of the
// node it occupies in each tree (recorded by the previous level's split).  The
// rows thus cross HBM once per level instead of once per tree and level; the
// directions (a few MB per level) come from L2.
template <int G>
__global__ void __launch_bounds__(256) k_project(const float* __restrict__ X, int dpad, int64_t ntot,
                                                 int level, int trees,
                                                 const int32_t* __restrict__ inv,
                                                 const int32_t* __restrict__ node,
                                                 const float* __restrict__ dirs,
                                                 uint64_t* __restrict__ keys, SegView segs, int active) {
  const int64_t nodes = int64_t(1) << level;
  constexpr int PER_WARP = 32 / G;
  const int lane = threadIdx.x & 31;
  const int gl = lane % G;
  const int64_t warps = (int64_t)gridDim.x * (blockDim.x >> 5);
  for (int64_t base = ((int64_t)blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5)) * PER_WARP;
       base < ntot; base += warps * PER_WARP) {
    const int64_t i0 = base + lane / G;
    const int64_t i = i0 < ntot ? i0 : ntot - 1;
    int a = segs.of(i);
    // every lane takes part in the group's shuffles; points of segments that
    // stopped splitting project on a valid direction and store nothing
    const bool valid = i0 < ntot && a < active;
    if (a >= active) a = 0;
    const float* row = X + (size_t)i * dpad;
    // four trees at a time: their index loads, direction loads and sums overlap
    for (int t0 = 0; t0 < trees; t0 += 4) {
      const int nt = min(4, trees - t0);  // warp-uniform
      int64_t p[4];
      const float* v[4];
#pragma unroll
      for (int u = 0; u < 4; ++u) {
        const int t = t0 + (u < nt ? u : 0);  // past the last tree: a valid direction, result unused
        p[u] = inv[(size_t)t * ntot + i];
        const int64_t j = valid ? node[(size_t)t * ntot + i] : 0;
        v[u] = dirs + (((size_t)a * trees + t) * nodes + j) * dpad;
      }
      float proj[4];
      group_project4<G>(row, v, dpad, gl, proj);
#pragma unroll
      for (int u = 0; u < 4; ++u)
        if (u < nt && valid && gl == 0) keys[(size_t)(t0 + u) * ntot + p[u]] = proj_key(proj[u], (uint32_t)i);
    }
  }
}

// ---------------------------------------------------------------- select --
// rank-th smallest (0-based) of cnt distinct 64-bit keys, MSB-first 8-bit
// radix select by the whole block.  Keys may live in shared or global memory.
__device__ uint64_t block_radix_select(const uint64_t* K, int64_t cnt, int64_t rank,
                                       uint32_t* hist /*256*/, uint64_t* sh /*4*/) {
  const int tid = threadIdx.x;
  uint64_t prefix = 0;
  for (int pass = 0; pass < 8; ++pass) {
    const int shift = 56 - 8 * pass;
    for (int b = tid; b < 256; b += blockDim.x) hist[b] = 0;
    __syncthreads();
    for (int64_t i = tid; i < cnt; i += blockDim.x) {
      const uint64_t key = K[i];
      if (pass == 0 || (key >> (shift + 8)) == (prefix >> (shift + 8)))
        atomicAdd(&hist[(key >> shift) & 255u], 1u);
    }
    __syncthreads();
    if (tid < 32) {
      uint32_t h[8];
      uint32_t s = 0;
#pragma unroll
      for (int q = 0; q < 8; ++q) {
        h[q] = hist[tid * 8 + q];
        s += h[q];
      }
      uint32_t incl = s;
#pragma unroll
      for (int off = 1; off < 32; off <<= 1) {
        uint32_t o = __shfl_up_sync(0xFFFFFFFFu, incl, off);
        if (tid >= off) incl += o;
      }
      int64_t c = (int64_t)(incl - s);
#pragma unroll
      for (int q = 0; q < 8; ++q) {
        if (c <= rank && rank < c + (int64_t)h[q]) {
          sh[0] = (uint64_t)(tid * 8 + q);
          sh[1] = (uint64_t)c;
          sh[2] = (uint64_t)h[q];
        }
        c += h[q];
      }
    }
    __syncthreads();
    const uint64_t bin = sh[0];
    const int64_t below = (int64_t)sh[1];
    const uint64_t inbin = sh[2];
    prefix |= bin << shift;
    rank -= below;
    if (pass == 7) return prefix;
    if (inbin == 1) {
      __syncthreads();
      for (int64_t i = tid; i < cnt; i += blockDim.x) {
        const uint64_t key = K[i];
        if ((key >> shift) == (prefix >> shift)) sh[3] = key;
      }
      __syncthreads();
      return sh[3];
    }
    __syncthreads();
  }
  return prefix;  // not reached
}

// One block per (active segment, tree, node) of `level`: median select +
// stable partition of the node's positions into perm_out, keeping the inverse
// permutation `inv` (point id -> global position) and each point's node of the
// next level current.  Blocks past the active ones copy the whole range of a
// (segment, tree) that no longer splits, so both perm buffers stay complete.
// SMEM_KEYS: node keys staged in shared memory (count <= kSplitSmemKeys).
template <bool SMEM_KEYS>
__global__ void __launch_bounds__(1024) k_split(int64_t ntot, int level, int trees, SegView segs, int active,
                                                const uint64_t* __restrict__ keys,
                                                const int32_t* __restrict__ perm,
                                                int32_t* __restrict__ perm_out,
                                                int32_t* __restrict__ inv,
                                                int32_t* __restrict__ node) {
  extern __shared__ uint64_t dyn_keys[];
  __shared__ uint32_t hist[256];
  __shared__ uint64_t sh[4];
  __shared__ int64_t warp_sums[33];
  const int64_t nodes = int64_t(1) << level;
  const int64_t s = blockIdx.x;
  const int64_t split_blocks = (int64_t)active * trees * nodes;
  if (s >= split_blocks) {  // copy a finished (segment, tree)
    const int64_t c = s - split_blocks;
    const int a = active + (int)(c / trees);
    const int t = (int)(c % trees);
    const SegEntry e = segs.get(a);
    const int32_t* Pin = perm + (size_t)t * ntot + e.off;
    int32_t* Pout = perm_out + (size_t)t * ntot + e.off;
    for (int64_t i = threadIdx.x; i < e.n; i += blockDim.x) Pout[i] = Pin[i];
    return;
  }
  const int a = (int)(s / (nodes * trees));
  const int64_t r = s - (int64_t)a * nodes * trees;
  const int t = (int)(r / nodes);
  const int64_t j = r - (int64_t)t * nodes;
  const SegEntry e = segs.get(a);
  const int64_t lo = e.off + node_lo(e.n, level, j), hi = e.off + node_lo(e.n, level, j + 1);
  const int64_t mid = e.off + node_lo(e.n, level + 1, 2 * j + 1);
  const int64_t cnt = hi - lo, nl = mid - lo;
  const uint64_t* K = keys + (size_t)t * ntot + lo;
  const int32_t* Pin = perm + (size_t)t * ntot + lo;
  int32_t* Pout = perm_out + (size_t)t * ntot + lo;
  if (cnt < 2 || nl <= 0 || nl >= cnt) {
    for (int64_t i = threadIdx.x; i < cnt; i += blockDim.x) {
      const int32_t id = Pin[i];
      Pout[i] = id;
      node[(size_t)t * ntot + id] = (int32_t)(lo + i < mid ? 2 * j : 2 * j + 1);
    }
    return;
  }
  const uint64_t* KS = K;
  if (SMEM_KEYS) {
    for (int64_t i = threadIdx.x; i < cnt; i += blockDim.x) dyn_keys[i] = K[i];
    __syncthreads();
    KS = dyn_keys;
  }
  const uint64_t pivot = block_radix_select(KS, cnt, nl, hist, sh);
  // Stable partition, ITEMS consecutive positions per thread per tile.
  constexpr int ITEMS = 4;
  const int64_t tile = (int64_t)blockDim.x * ITEMS;
  int64_t left_base = 0;
  for (int64_t t0 = 0; t0 < cnt; t0 += tile) {
    const int64_t p0 = t0 + (int64_t)threadIdx.x * ITEMS;
    bool f[ITEMS];
    int c = 0;
#pragma unroll
    for (int q = 0; q < ITEMS; ++q) {
      const int64_t p = p0 + q;
      f[q] = p < cnt && KS[p] < pivot;
      c += f[q];
    }
    int64_t total;
    int64_t before = block_excl_scan(c, warp_sums, &total) + left_base;
#pragma unroll
    for (int q = 0; q < ITEMS; ++q) {
      const int64_t p = p0 + q;
      if (p < cnt) {
        const int64_t dst = f[q] ? before : nl + (p - before);
        if (dst >= 0 && dst < cnt) {  // exactly nl keys are below the pivot
          const int32_t id = Pin[p];
          Pout[dst] = id;
          inv[(size_t)t * ntot + id] = (int32_t)(lo + dst);
          node[(size_t)t * ntot + id] = (int32_t)(f[q] ? 2 * j : 2 * j + 1);
        }
        before += f[q];
      }
    }
    left_base += total;
  }
}

// ------------------------------------------------------ multi-block split --
// The top levels hold few nodes with many points each (level 0: one node of
// all n points per tree), too few blocks for the GPU.  There every node is
// spread over blocks of kMChunk keys: an MSB radix select over global
// 256-bin histograms (one histogram pass and one select step per 8-bit
// digit; a node stops once its target bucket holds a single key), then a
// count pass and a stable scatter pass.  The pivot is the same order
// statistic and the partition the same stable one as k_split's, so the trees
// are identical.
struct MSplitNode {
  uint64_t prefix;  // known high digits of the pivot
  int64_t rank;     // rank of the pivot among keys sharing those digits
  int32_t shift;    // digits at and above `shift` are known
  int32_t state;    // 0 selecting, 1 pivot known, 2 node not split (copy)
};

__device__ __forceinline__ void msplit_node(const SegView& segs, int level, int trees, int64_t s,
                                            int64_t* lo, int64_t* hi, int64_t* mid, int* t, int64_t* j) {
  const int64_t nodes = int64_t(1) << level;
  const int a = (int)(s / (nodes * trees));
  const int64_t r = s - (int64_t)a * nodes * trees;
  *t = (int)(r / nodes);
  *j = r - (int64_t)(*t) * nodes;
  const SegEntry e = segs.get(a);
  *lo = e.off + node_lo(e.n, level, *j);
  *hi = e.off + node_lo(e.n, level, *j + 1);
  *mid = e.off + node_lo(e.n, level + 1, 2 * (*j) + 1);
}

__global__ void k_msplit_init(SegView segs, int level, int trees, MSplitNode* st, uint32_t* hist) {
  const int64_t s = blockIdx.x;
  int64_t lo, hi, mid, j;
  int t;
  msplit_node(segs, level, trees, s, &lo, &hi, &mid, &t, &j);
  const int64_t cnt = hi - lo, nl = mid - lo;
  if (threadIdx.x == 0) {
    st[s].prefix = 0;
    st[s].rank = nl;
    st[s].shift = 64;
    st[s].state = (cnt < 2 || nl <= 0 || nl >= cnt) ? 2 : 0;
  }
  for (int b = threadIdx.x; b < 256; b += blockDim.x) hist[s * 256 + b] = 0;
}

// One digit: block (b, s) histograms chunk b of node s.
__global__ void __launch_bounds__(256) k_msplit_hist(SegView segs, int level, int trees, int64_t ntot, int pass,
                                                     const uint64_t* __restrict__ keys,
                                                     const MSplitNode* __restrict__ st, uint32_t* __restrict__ hist) {
  __shared__ uint32_t h[256];
  const int64_t s = blockIdx.y;
  const MSplitNode nd = st[s];
  if (nd.state != 0) return;
  int64_t lo, hi, mid, j;
  int t;
  msplit_node(segs, level, trees, s, &lo, &hi, &mid, &t, &j);
  const int64_t c0 = lo + (int64_t)blockIdx.x * kMChunk;
  if (c0 >= hi) return;
  const int64_t c1 = min(hi, c0 + kMChunk);
  h[threadIdx.x] = 0;
  __syncthreads();
  const int shift = 56 - 8 * pass;
  const uint64_t* K = keys + (size_t)t * ntot;
  for (int64_t i = c0 + threadIdx.x; i < c1; i += blockDim.x) {
    const uint64_t key = K[i];
    if (pass == 0 || (key >> (shift + 8)) == (nd.prefix >> (shift + 8))) atomicAdd(&h[(key >> shift) & 255u], 1u);
  }
  __syncthreads();
  const uint32_t v = h[threadIdx.x];
  if (v) atomicAdd(&hist[s * 256 + threadIdx.x], v);
}

// One digit: the bucket holding the target rank; histogram cleared for the next digit.
__global__ void __launch_bounds__(256) k_msplit_select(int pass, MSplitNode* __restrict__ st, uint32_t* __restrict__ hist) {
  __shared__ uint32_t sum[8];
  const int64_t s = blockIdx.x;
  const MSplitNode nd = st[s];
  if (nd.state != 0) return;
  const int tid = threadIdx.x, lane = tid & 31, w = tid >> 5;
  const uint32_t v = hist[s * 256 + tid];
  uint32_t incl = v;
#pragma unroll
  for (int off = 1; off < 32; off <<= 1) {
    const uint32_t o = __shfl_up_sync(0xFFFFFFFFu, incl, off);
    if (lane >= off) incl += o;
  }
  if (lane == 31) sum[w] = incl;
  __syncthreads();
  uint32_t before = 0;
  for (int q = 0; q < w; ++q) before += sum[q];
  const int64_t excl = (int64_t)before + incl - v;
  const int shift = 56 - 8 * pass;
  if (v > 0 && excl <= nd.rank && nd.rank < excl + (int64_t)v) {
    MSplitNode out = nd;
    out.prefix = nd.prefix | ((uint64_t)tid << shift);
    out.rank = nd.rank - excl;
    out.shift = shift;
    out.state = (v == 1 || pass == 7) ? 1 : 0;
    st[s] = out;
  }
  hist[s * 256 + tid] = 0;
}

__device__ __forceinline__ bool msplit_less(uint64_t key, const MSplitNode& nd) {
  return (key >> nd.shift) < (nd.prefix >> nd.shift);
}

// Keys below the pivot in chunk b of node s.
__global__ void __launch_bounds__(256) k_msplit_count(SegView segs, int level, int trees, int64_t ntot,
                                                      const uint64_t* __restrict__ keys,
                                                      const MSplitNode* __restrict__ st, int32_t* __restrict__ lcount,
                                                      int nchunks) {
  __shared__ int32_t red[8];
  const int64_t s = blockIdx.y;
  const MSplitNode nd = st[s];
  int64_t lo, hi, mid, j;
  int t;
  msplit_node(segs, level, trees, s, &lo, &hi, &mid, &t, &j);
  const int64_t c0 = lo + (int64_t)blockIdx.x * kMChunk;
  const int64_t c1 = min(hi, c0 + kMChunk);
  const uint64_t* K = keys + (size_t)t * ntot;
  int32_t c = 0;
  if (nd.state == 1)
    for (int64_t i = c0 + threadIdx.x; i < c1; i += blockDim.x) c += msplit_less(K[i], nd) ? 1 : 0;
#pragma unroll
  for (int off = 16; off >= 1; off >>= 1) c += __shfl_xor_sync(0xFFFFFFFFu, c, off);
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = c;
  __syncthreads();
  if (threadIdx.x == 0) {
    int32_t tot = 0;
    for (int q = 0; q < (int)(blockDim.x >> 5); ++q) tot += red[q];
    lcount[s * nchunks + blockIdx.x] = tot;
  }
}

// Stable scatter of chunk b of node s: left keys after the left keys of the
// chunks before it, right keys after nl and the right keys before them.
__global__ void __launch_bounds__(256) k_msplit_scatter(SegView segs, int level, int trees, int64_t ntot,
                                                        const uint64_t* __restrict__ keys,
                                                        const MSplitNode* __restrict__ st,
                                                        const int32_t* __restrict__ lcount, int nchunks,
                                                        const int32_t* __restrict__ perm,
                                                        int32_t* __restrict__ perm_out, int32_t* __restrict__ inv,
                                                        int32_t* __restrict__ node) {
  __shared__ int64_t warp_sums[33];
  __shared__ int64_t base_sh;
  const int64_t s = blockIdx.y;
  const MSplitNode nd = st[s];
  int64_t lo, hi, mid, j;
  int t;
  msplit_node(segs, level, trees, s, &lo, &hi, &mid, &t, &j);
  const int64_t c0 = lo + (int64_t)blockIdx.x * kMChunk;
  if (c0 >= hi) return;
  const int64_t c1 = min(hi, c0 + kMChunk);
  const int32_t* Pin = perm + (size_t)t * ntot;
  int32_t* Pout = perm_out + (size_t)t * ntot;
  int32_t* Node = node + (size_t)t * ntot;
  int32_t* Inv = inv + (size_t)t * ntot;
  if (nd.state == 2) {  // not split: copy, children by position
    for (int64_t i = c0 + threadIdx.x; i < c1; i += blockDim.x) {
      const int32_t id = Pin[i];
      Pout[i] = id;
      Node[id] = (int32_t)(i < mid ? 2 * j : 2 * j + 1);
    }
    return;
  }
  if (threadIdx.x == 0) {
    int64_t b = 0;
    for (int q = 0; q < (int)blockIdx.x; ++q) b += lcount[s * nchunks + q];
    base_sh = b;
  }
  __syncthreads();
  const int64_t nl = mid - lo;
  const uint64_t* K = keys + (size_t)t * ntot;
  constexpr int ITEMS = 4;
  const int64_t tile = (int64_t)blockDim.x * ITEMS;
  int64_t left_base = base_sh;  // left keys before this tile, over the whole node
  for (int64_t t0 = c0; t0 < c1; t0 += tile) {
    const int64_t p0 = t0 + (int64_t)threadIdx.x * ITEMS;
    bool f[ITEMS];
    int c = 0;
#pragma unroll
    for (int q = 0; q < ITEMS; ++q) {
      const int64_t p = p0 + q;
      f[q] = p < c1 && msplit_less(K[p], nd);
      c += f[q];
    }
    int64_t total;
    int64_t before = block_excl_scan(c, warp_sums, &total) + left_base;
#pragma unroll
    for (int q = 0; q < ITEMS; ++q) {
      const int64_t p = p0 + q;
      if (p < c1) {
        const int64_t rel = p - lo;
        const int64_t dst = f[q] ? before : nl + (rel - before);
        if (dst >= 0 && dst < hi - lo) {
          const int32_t id = Pin[p];
          Pout[lo + dst] = id;
          Inv[id] = (int32_t)(lo + dst);
          Node[id] = (int32_t)(f[q] ? 2 * j : 2 * j + 1);
        }
        before += f[q];
      }
    }
    left_base += total;
  }
}

// Ranges of the (segment, tree) pairs that no longer split, copied as they are.
__global__ void k_copy_finished(SegView segs, int active, int trees, int64_t ntot, const int32_t* __restrict__ perm,
                                int32_t* __restrict__ perm_out) {
  const int a = active + (int)(blockIdx.x / trees);
  const int t = (int)(blockIdx.x % trees);
  const SegEntry e = segs.get(a);
  for (int64_t i = threadIdx.x; i < e.n; i += blockDim.x)
    perm_out[(size_t)t * ntot + e.off + i] = perm[(size_t)t * ntot + e.off + i];
}

// ------------------------------------------------------------------ host --
size_t msplit_scratch_bytes(int64_t max_node_points) {
  const int64_t chunks = (max_node_points + kMChunk - 1) / kMChunk;
  return sizeof(MSplitNode) * kMSplitMaxNodes + sizeof(uint32_t) * 256 * kMSplitMaxNodes +
         sizeof(int32_t) * (size_t)kMSplitMaxNodes * (size_t)(chunks > 0 ? chunks : 1);
}

size_t tree_dir_nodes(const SegEntry* hsegs, int nseg, int trees) {
  size_t best = 1;
  const int maxdepth = hsegs[0].depth;
  for (int l = 0; l < maxdepth; ++l) {
    int active = 0;
    while (active < nseg && hsegs[active].depth > l) ++active;
    const size_t v = (size_t)active * (size_t)trees << l;
    if (v > best) best = v;
  }
  return best;
}

int tree_build(const TreeArgs& a, LaunchLog& log) {
  const int64_t ntot = a.n;
  cudaStream_t st = a.stream;
  static bool attr_set[64] = {false};
  int dev = 0;
  cudaGetDevice(&dev);
  if (!attr_set[dev & 63]) {
    cudaFuncSetAttribute(k_split<true>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                         kSplitSmemKeys * (int)sizeof(uint64_t));
    attr_set[dev & 63] = true;
  }
  // identity order for every tree
  k_iota<<<(unsigned)((a.trees * ntot + 255) / 256), 256, 0, st>>>(a.perm, ntot, a.trees);
  k_iota<<<(unsigned)((a.trees * ntot + 255) / 256), 256, 0, st>>>(a.inv, ntot, a.trees);
  cudaMemsetAsync(a.node, 0, sizeof(int32_t) * (size_t)a.trees * ntot, st);  // all in the root
  log.add(2);
  int32_t* cur = a.perm;
  int32_t* alt = a.perm_alt;
  const int G = proj_group(a.d);
  const int maxdepth = a.hsegs[0].depth;
  for (int l = 0; l < maxdepth; ++l) {
    int active = 0;
    while (active < a.nseg && a.hsegs[active].depth > l) ++active;
    const int64_t nodes = int64_t(1) << l;
    const int64_t segs = nodes * a.trees * active;
    k_directions<<<(unsigned)((segs + 7) / 8), 256, 0, st>>>(a.X, a.dpad, ntot, l, a.trees, cur, a.dirs,
                                                             a.segs, active, a.tree_offset,
                                                             a.tree_stride > 0 ? a.tree_stride : 1);
    const int per_block = 8 * (32 / G);
    int64_t blocks = (ntot + per_block - 1) / per_block;
    if (blocks > 148LL * 64) blocks = 148LL * 64;
    switch (G) {
      case 1: k_project<1><<<(unsigned)blocks, 256, 0, st>>>(a.X, a.dpad, ntot, l, a.trees, a.inv, a.node, a.dirs, a.keys, a.segs, active); break;
      case 2: k_project<2><<<(unsigned)blocks, 256, 0, st>>>(a.X, a.dpad, ntot, l, a.trees, a.inv, a.node, a.dirs, a.keys, a.segs, active); break;
      case 4: k_project<4><<<(unsigned)blocks, 256, 0, st>>>(a.X, a.dpad, ntot, l, a.trees, a.inv, a.node, a.dirs, a.keys, a.segs, active); break;
      case 8: k_project<8><<<(unsigned)blocks, 256, 0, st>>>(a.X, a.dpad, ntot, l, a.trees, a.inv, a.node, a.dirs, a.keys, a.segs, active); break;
      case 16: k_project<16><<<(unsigned)blocks, 256, 0, st>>>(a.X, a.dpad, ntot, l, a.trees, a.inv, a.node, a.dirs, a.keys, a.segs, active); break;
      default: k_project<32><<<(unsigned)blocks, 256, 0, st>>>(a.X, a.dpad, ntot, l, a.trees, a.inv, a.node, a.dirs, a.keys, a.segs, active); break;
    }
    // the largest active segment is the first
    const int64_t maxcnt = (a.hsegs[0].n + nodes - 1) / nodes;
    int threads = (int)((maxcnt + 3) / 4);
    threads = ((threads + 31) / 32) * 32;
    if (threads < 64) threads = 64;
    if (threads > 1024) threads = 1024;
    const unsigned grid = (unsigned)(segs + (int64_t)(a.nseg - active) * a.trees);
    if (a.msplit && segs <= kMSplitMaxNodes && maxcnt > 2 * kMChunk) {
      const int nchunks = (int)((maxcnt + kMChunk - 1) / kMChunk);
      MSplitNode* mst = static_cast<MSplitNode*>(a.msplit);
      uint32_t* hist = reinterpret_cast<uint32_t*>(mst + kMSplitMaxNodes);
      int32_t* lcount = reinterpret_cast<int32_t*>(hist + (size_t)kMSplitMaxNodes * 256);
      const dim3 g2((unsigned)nchunks, (unsigned)segs);
      k_msplit_init<<<(unsigned)segs, 256, 0, st>>>(a.segs, l, a.trees, mst, hist);
      for (int pass = 0; pass < 8; ++pass) {
        k_msplit_hist<<<g2, 256, 0, st>>>(a.segs, l, a.trees, ntot, pass, a.keys, mst, hist);
        k_msplit_select<<<(unsigned)segs, 256, 0, st>>>(pass, mst, hist);
      }
      k_msplit_count<<<g2, 256, 0, st>>>(a.segs, l, a.trees, ntot, a.keys, mst, lcount, nchunks);
      k_msplit_scatter<<<g2, 256, 0, st>>>(a.segs, l, a.trees, ntot, a.keys, mst, lcount, nchunks, cur, alt, a.inv,
                                           a.node);
      if (a.nseg > active)
        k_copy_finished<<<(unsigned)((a.nseg - active) * a.trees), 256, 0, st>>>(a.segs, active, a.trees, ntot, cur,
                                                                               alt);
      log.add(19 + (a.nseg > active ? 1 : 0));
    } else if (maxcnt <= kSplitSmemKeys) {
      k_split<true><<<grid, threads, (size_t)maxcnt * sizeof(uint64_t), st>>>(ntot, l, a.trees, a.segs, active, a.keys, cur, alt, a.inv, a.node);
      log.add(1);
    } else {
      k_split<false><<<grid, threads, 0, st>>>(ntot, l, a.trees, a.segs, active, a.keys, cur, alt, a.inv, a.node);
      log.add(1);
    }
    log.add(2);
    int32_t* tmp = cur;
    cur = alt;
    alt = tmp;
  }
  if (cur != a.perm) {
    cudaMemcpyAsync(a.perm, cur, sizeof(int32_t) * (size_t)a.trees * ntot, cudaMemcpyDeviceToDevice, st);
  }
  return cudaPeekAtLastError() == cudaSuccess ? KNN_OK : KNN_ERR_CUDA;
}

__global__ void k_iota(int32_t* perm, int64_t n, int trees) {
  const int64_t g = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (g < (int64_t)trees * n) perm[g] = (int32_t)(g % n);
}

}  // namespace knn
