// Reference-rule trees (knn_options.split_rule = KNN_SPLIT_REFERENCE).
//
// The split of buildUpTheTrees / makePartitionOfLeaf1..3
// (euclideandistancematrixgpu.cu:2138-2181, :2291-2365, :2478-2487), kept
// deterministic:
//   * per level two integers R1, R2 shared by every node of the level (the
//     reference draws them with rand(); here a counter hash of (seed, tree,
//     level)); a node of c > leaf points takes positions p1 = R1 % c and
//     p2 = R2 % c (p2 = (p1 + 1) % c when they coincide);
//   * a member x goes left when sum_dim x[dim] * (x[p2][dim] - x[p1][dim]) < 0,
//     summed over the dimensions in order with a fused multiply-add (the
//     hyperplane passes through the origin); the point at p1 goes left and the
//     one at p2 right whatever their sums;
//   * the node's positions are partitioned stably (lefts first, each side in
//     its previous order) instead of the atomic scatter (.cu:2205-2260);
//   * nodes of at most `leaf` points stop; the tree ends when no node splits.
// Node sizes then depend on the data, so each level runs on an explicit list
// of splitting nodes, and the host reads the left counts back once per level
// to form the next list (the reference syncs once per level as well,
// .cu:2602-2604).  The leaf blocks of the leaf stage come from the node
// records (smallest ancestor of a leaf with at least k+1 points).
#include <algorithm>
#include <vector>

#include "knn_internal.cuh"
#include "knn_kernels.cuh"

namespace knn {

namespace {
constexpr int kFChunk = 1024;  // positions per block
}

// Block (b, s): sides of positions [lo + b*kFChunk, ...) of splitting node s
// (1 = left).
__global__ void __launch_bounds__(256) k_faithful_side(const float* __restrict__ X, int d, int dpad, int64_t ntot,
                                                       const FNode* __restrict__ nodes, const int32_t* __restrict__ perm,
                                                       uint8_t* __restrict__ side) {
  const FNode nd = nodes[blockIdx.y];
  const int64_t c0 = nd.lo + (int64_t)blockIdx.x * kFChunk;
  if (c0 >= nd.hi) return;
  const int64_t c1 = min(nd.hi, c0 + kFChunk);
  const int32_t* P = perm + (size_t)nd.tree * ntot;
  const float* xa = X + (size_t)P[nd.lo + nd.p1] * dpad;
  const float* xb = X + (size_t)P[nd.lo + nd.p2] * dpad;
  for (int64_t p = c0 + threadIdx.x; p < c1; p += blockDim.x) {
    const float* x = X + (size_t)P[p] * dpad;
    float acc = 0.f;
    for (int c = 0; c < d; ++c) acc = __fmaf_rn(x[c], __fsub_rn(xb[c], xa[c]), acc);
    uint8_t left = acc < 0.f ? 1 : 0;
    if (p == nd.lo + nd.p1) left = 1;
    if (p == nd.lo + nd.p2) left = 0;
    side[(size_t)nd.tree * ntot + p] = left;
  }
}

// Left positions in chunk b of node s.
__global__ void __launch_bounds__(256) k_faithful_count(int64_t ntot, const FNode* __restrict__ nodes,
                                                        const uint8_t* __restrict__ side, int32_t* __restrict__ lcount) {
  __shared__ int32_t red[8];
  const FNode nd = nodes[blockIdx.y];
  const int64_t c0 = nd.lo + (int64_t)blockIdx.x * kFChunk;
  if (c0 >= nd.hi) return;  // past this node's chunks (uniform in the block)
  const int64_t c1 = min(nd.hi, c0 + kFChunk);
  int32_t c = 0;
  for (int64_t p = c0 + threadIdx.x; p < c1; p += blockDim.x) c += side[(size_t)nd.tree * ntot + p];
#pragma unroll
  for (int off = 16; off >= 1; off >>= 1) c += __shfl_xor_sync(0xFFFFFFFFu, c, off);
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = c;
  __syncthreads();
  if (threadIdx.x == 0) {
    int32_t t = 0;
    for (int q = 0; q < (int)(blockDim.x >> 5); ++q) t += red[q];
    lcount[(size_t)nd.cbase + blockIdx.x] = t;
  }
}

// Stable partition of chunk b of node s into perm_out; the node's left count
// (all chunks) to nleft[s].
__global__ void __launch_bounds__(256) k_faithful_scatter(int64_t ntot, const FNode* __restrict__ nodes,
                                                          const uint8_t* __restrict__ side,
                                                          const int32_t* __restrict__ lcount,
                                                          const int32_t* __restrict__ perm, int32_t* __restrict__ perm_out,
                                                          int64_t* __restrict__ nleft) {
  __shared__ int64_t warp_sums[33];
  __shared__ int64_t base[2];
  const int64_t s = blockIdx.y;
  const FNode nd = nodes[s];
  const int64_t c0 = nd.lo + (int64_t)blockIdx.x * kFChunk;
  if (c0 >= nd.hi) return;
  const int64_t c1 = min(nd.hi, c0 + kFChunk);
  const int chunks = (int)((nd.hi - nd.lo + kFChunk - 1) / kFChunk);
  if (threadIdx.x == 0) {
    int64_t before = 0, total = 0;
    for (int q = 0; q < chunks; ++q) {
      const int64_t v = lcount[(size_t)nd.cbase + q];
      if (q < (int)blockIdx.x) before += v;
      total += v;
    }
    base[0] = before;
    base[1] = total;
    if (blockIdx.x == 0) nleft[s] = total;
  }
  __syncthreads();
  const int64_t nl = base[1];
  const int32_t* P = perm + (size_t)nd.tree * ntot;
  int32_t* Q = perm_out + (size_t)nd.tree * ntot;
  const uint8_t* S = side + (size_t)nd.tree * ntot;
  constexpr int ITEMS = 4;
  const int64_t tile = (int64_t)blockDim.x * ITEMS;
  int64_t left_base = base[0];
  for (int64_t t0 = c0; t0 < c1; t0 += tile) {
    const int64_t p0 = t0 + (int64_t)threadIdx.x * ITEMS;
    bool f[ITEMS];
    int c = 0;
#pragma unroll
    for (int q = 0; q < ITEMS; ++q) {
      const int64_t p = p0 + q;
      f[q] = p < c1 && S[p] != 0;
      c += f[q];
    }
    int64_t total;
    int64_t before = block_excl_scan(c, warp_sums, &total) + left_base;
#pragma unroll
    for (int q = 0; q < ITEMS; ++q) {
      const int64_t p = p0 + q;
      if (p < c1) {
        const int64_t rel = p - nd.lo;
        const int64_t dst = f[q] ? before : nl + (rel - before);
        if (dst >= 0 && dst < nd.hi - nd.lo) Q[nd.lo + dst] = P[p];
        before += f[q];
      }
    }
    left_base += total;
  }
}

uint32_t faithful_draw(uint64_t seed, int tree, int level, int which) {
  const uint64_t h = splitmix64(seed ^ splitmix64(0xF417F01ull + (uint64_t)tree * 0x9E3779B97F4A7C15ull +
                                                  (uint64_t)level * 0xD1B54A32D192ED03ull + (uint64_t)which));
  return (uint32_t)(h & 0x7FFFFFFFu);
}

void faithful_pivots(uint64_t seed, int tree, int level, int64_t cnt, int32_t* p1, int32_t* p2) {
  if (cnt <= 1) {
    *p1 = *p2 = 0;
    return;
  }
  *p1 = (int32_t)(faithful_draw(seed, tree, level, 1) % (uint64_t)cnt);
  *p2 = (int32_t)(faithful_draw(seed, tree, level, 2) % (uint64_t)cnt);
  if (*p1 == *p2) *p2 = (int32_t)((*p1 + 1) % cnt);
}

int faithful_tree_build(const FaithfulArgs& a, FaithfulTrees* out, LaunchLog& log) {
  cudaStream_t st = a.stream;
  const int64_t n = a.n;
  out->nodes.clear();
  // node records: (tree, lo, hi, parent); the roots first
  std::vector<FNode> active;
  for (int t = 0; t < a.trees; ++t) {
    FNode r{};
    r.tree = t;
    r.lo = 0;
    r.hi = n;
    r.parent = -1;
    r.id = (int64_t)out->nodes.size();
    out->nodes.push_back(r);
    if (n > a.leaf) active.push_back(r);
  }
  k_iota<<<(unsigned)((a.trees * n + 255) / 256), 256, 0, st>>>(a.perm, n, a.trees);
  log.add();
  int32_t* cur = a.perm;
  int32_t* alt = a.perm_alt;
  std::vector<int64_t> nl;
  int level = 0;
  while (!active.empty()) {
    if (level >= kFaithfulMaxLevels) return KNN_ERR_UNSUPPORTED;
    const int S = (int)active.size();
    int64_t maxcnt = 0;
    size_t chunks = 0;
    for (auto& nd : active) {
      faithful_pivots(a.seed, a.tree_offset + nd.tree * (a.tree_stride > 0 ? a.tree_stride : 1), level,
                      nd.hi - nd.lo, &nd.p1, &nd.p2);
      maxcnt = std::max(maxcnt, nd.hi - nd.lo);
      nd.cbase = (int32_t)chunks;
      chunks += (size_t)((nd.hi - nd.lo + kFChunk - 1) / kFChunk);
    }
    const int nchunks = (int)((maxcnt + kFChunk - 1) / kFChunk);
    if ((size_t)S > a.node_cap || chunks > a.count_cap) return KNN_ERR_UNSUPPORTED;
    if (cudaMemcpyAsync(a.dnodes, active.data(), sizeof(FNode) * S, cudaMemcpyHostToDevice, st) != cudaSuccess ||
        cudaMemcpyAsync(alt, cur, sizeof(int32_t) * (size_t)a.trees * n, cudaMemcpyDeviceToDevice, st) != cudaSuccess)
      return KNN_ERR_CUDA;
    const dim3 g((unsigned)nchunks, (unsigned)S);
    k_faithful_side<<<g, 256, 0, st>>>(a.X, a.d, a.dpad, n, a.dnodes, cur, a.side);
    k_faithful_count<<<g, 256, 0, st>>>(n, a.dnodes, a.side, a.lcount);
    k_faithful_scatter<<<g, 256, 0, st>>>(n, a.dnodes, a.side, a.lcount, cur, alt, a.nleft);
    log.add(3);
    nl.resize(S);
    if (cudaMemcpyAsync(nl.data(), a.nleft, sizeof(int64_t) * S, cudaMemcpyDeviceToHost, st) != cudaSuccess ||
        cudaStreamSynchronize(st) != cudaSuccess)
      return KNN_ERR_CUDA;
    std::vector<FNode> next;
    for (int s = 0; s < S; ++s) {
      const FNode& p = active[s];
      FNode L{}, R{};
      L.tree = R.tree = p.tree;
      L.parent = R.parent = p.id;
      L.lo = p.lo;
      L.hi = p.lo + nl[s];
      R.lo = L.hi;
      R.hi = p.hi;
      L.id = (int64_t)out->nodes.size();
      out->nodes.push_back(L);
      R.id = (int64_t)out->nodes.size();
      out->nodes.push_back(R);
      out->split.resize(out->nodes.size(), 0);
      out->split[p.id] = 1;
      if (L.hi - L.lo > a.leaf) next.push_back(L);
      if (R.hi - R.lo > a.leaf) next.push_back(R);
    }
    std::swap(cur, alt);
    active.swap(next);
    ++level;
  }
  out->split.resize(out->nodes.size(), 0);
  if (cur != a.perm &&
      cudaMemcpyAsync(a.perm, cur, sizeof(int32_t) * (size_t)a.trees * n, cudaMemcpyDeviceToDevice, st) != cudaSuccess)
    return KNN_ERR_CUDA;
  out->levels = level;
  return cudaPeekAtLastError() == cudaSuccess ? KNN_OK : KNN_ERR_CUDA;
}

// Leaf blocks per tree: (lo, hi, blo, bhi) of every leaf in position order,
// the block being the smallest ancestor-or-self with at least k+1 points.
void faithful_leaf_table(const FaithfulTrees& T, int trees, int k, std::vector<int64_t>* table,
                         std::vector<int64_t>* offset, std::vector<int64_t>* count) {
  table->clear();
  offset->assign(trees, 0);
  count->assign(trees, 0);
  std::vector<std::vector<const FNode*>> leaves(trees);
  for (const auto& nd : T.nodes)
    if (!T.split[nd.id]) leaves[nd.tree].push_back(&nd);
  for (int t = 0; t < trees; ++t) {
    std::sort(leaves[t].begin(), leaves[t].end(), [](const FNode* a, const FNode* b) { return a->lo < b->lo; });
    (*offset)[t] = (int64_t)table->size() / 4;
    for (const FNode* lf : leaves[t]) {
      if (lf->hi <= lf->lo) continue;
      const FNode* b = lf;
      while (b->hi - b->lo < k + 1 && b->parent >= 0) b = &T.nodes[b->parent];
      table->push_back(lf->lo);
      table->push_back(lf->hi);
      table->push_back(b->lo);
      table->push_back(b->hi);
      ++(*count)[t];
    }
  }
}

}  // namespace knn
