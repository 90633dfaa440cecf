// Initial k-NN over leaf blocks, plain FP32 on CUDA cores.
//
// Replaces findGraphTraversalStartPoint + findInitialStateOfAproximated{Euclidean,
// Taxicab,Cosine}KNN (euclideandistancematrixgpu.cu:87-105, :107-1031).  The
// reference unions every tree's block of a point in an N-byte bitmap, scans the
// bitmap per point and selects k with a histogram; here each (tree, leaf) block
// is split into tile jobs of 64 query rows against all the block's candidates:
// the rows are staged in shared memory 32 dims at a
// time, every (query, candidate) key of the block is computed by a 4x4 register
// tile per thread in the reference's summation order, and each query's k best
// are merged into its running sorted list by one warp (bitonic sort + merge via
// shuffles).  Taking the k best of every tree in turn and dropping ids already
// listed gives the k best of the union, so no bitmap is needed.
//
// Two result-neutral shortcuts: where every leaf is its own block, each tile
// pair of a leaf is computed once and merged into both sides (k_leaf_pair; the
// keys are symmetric bit for bit), and on sparse rows a tile reads only the dims
// that are non-zero in some of its rows (the left-out terms are exact zeros).
//
// The block of a leaf is its smallest ancestor holding at least k+1 points
// (the climb of .cu:87-105); all points of a leaf share it.
#include "knn_internal.cuh"
#include "knn_kernels.cuh"

namespace knn {

namespace {
constexpr int kDC = 32;     // dims staged per chunk
}  // namespace

// Register tile of R consecutive floats from shared memory (R = 2 or 4).
template <int R>
__device__ __forceinline__ void load_r(const float* p, float (&v)[R]) {
  if constexpr (R == 4) {
    const float4 t = *reinterpret_cast<const float4*>(p);
    v[0] = t.x; v[1] = t.y; v[2] = t.z; v[3] = t.w;
  } else {
    const float2 t = *reinterpret_cast<const float2*>(p);
    v[0] = t.x; v[1] = t.y;
  }
}

// ------------------------------------------------------------ sparse rows --
// A dim where every row of a leaf block is zero adds an exact +0 to each of the
// block's EUCLIDEAN and TAXICAB sums ((0-0)^2 and |0-0|, added to a partial sum
// that is never negative), so leaving it out keeps every key's bits.  Per leaf
// block: a bit mask of the dims that are non-zero in some row, then the list of
// those dims with the 256-dim groups kept apart (each group's dims padded with
// -1 to whole 32-dim chunks), so that the per-group partial sums are formed over
// the same terms in the same order as over all dims.
constexpr int kDimRows = 1024;  // rows of a leaf block per mask block

// grid (leaf, row part); mask [leaves][W] zeroed beforehand, W = dpad / 32 + 1.
// Thread t of the block tests dims t, t + 256, ...: warp w's 32 lanes cover one
// mask word, so each warp ORs whole words.
__global__ void __launch_bounds__(256) k_leaf_dim_mask(const float* __restrict__ X, int dpad, SegView segs,
                                                       int k, const int32_t* __restrict__ perm,
                                                       uint32_t* __restrict__ mask, int W) {
  const int64_t leaf = blockIdx.x;
  int64_t j, lo, hi, blo, bhi;
  const SegEntry seg = segs.leaf(leaf, &j);
  leaf_block(seg, j, k, &lo, &hi, &blo, &bhi);
  for (int64_t r0 = blo + (int64_t)blockIdx.y * kDimRows; r0 < bhi; r0 += (int64_t)gridDim.y * kDimRows) {
    const int64_t r1 = min(bhi, r0 + kDimRows);
    for (int dim0 = 0; dim0 < dpad; dim0 += 256) {
      const int dim = dim0 + (int)threadIdx.x;
      bool nz = false;
      if (dim < dpad) {
        int64_t r = r0;
        for (; r + 4 <= r1 && !nz; r += 4) {  // four rows in flight
          const int32_t p0 = __ldg(perm + r), p1 = __ldg(perm + r + 1);
          const int32_t p2 = __ldg(perm + r + 2), p3 = __ldg(perm + r + 3);
          const float v0 = __ldg(X + (size_t)p0 * dpad + dim), v1 = __ldg(X + (size_t)p1 * dpad + dim);
          const float v2 = __ldg(X + (size_t)p2 * dpad + dim), v3 = __ldg(X + (size_t)p3 * dpad + dim);
          nz = (v0 != 0.f) | (v1 != 0.f) | (v2 != 0.f) | (v3 != 0.f);
        }
        for (; r < r1 && !nz; ++r) nz = __ldg(X + (size_t)__ldg(perm + r) * dpad + dim) != 0.f;
      }
      const uint32_t bits = __ballot_sync(0xFFFFFFFFu, nz);
      if ((threadIdx.x & 31) == 0 && bits) atomicOr(mask + leaf * W + (dim >> 5), bits);
    }
  }
}

// The dims set in mask words word(0..W) into out, one warp: every 256-dim group's
// dims in increasing order (lane l holds dims 256 g + 8 l .. + 7 of group g),
// padded with -1 to a multiple of 32 entries.  Returns the chunks of 32, or -1
// when the list saves no chunk over the ceil(d / 32) chunks of all dims.
template <typename LT, typename MaskFn>
__device__ __forceinline__ int warp_dim_list(MaskFn word, int W, int d, int dpad, LT* out) {
  const int lane = threadIdx.x & 31;
  int pos = 0;
  for (int g = 0; g * 256 < dpad; ++g) {
    const int w = 8 * g + (lane >> 2);
    const uint32_t bits = w < W ? (word(w) >> (8 * (lane & 3))) & 0xFFu : 0u;
    const int c = __popc(bits);
    int incl = c;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const int v = __shfl_up_sync(0xFFFFFFFFu, incl, o);
      if (lane >= o) incl += v;
    }
    const int total = __shfl_sync(0xFFFFFFFFu, incl, 31);
    int at = pos + incl - c;
    for (uint32_t b = bits; b; b &= b - 1) out[at++] = (LT)(256 * g + 8 * lane + (__ffs(b) - 1));
    const int padded = (total + 31) & ~31;
    for (int e = total + lane; e < padded; e += 32) out[pos + e] = (LT)-1;
    pos += padded;
  }
  return pos / 32 < (d + 31) / 32 ? pos / 32 : -1;
}

// Dim lists are 16-bit (dims below 32768), in global memory (a leaf block's
// list) or shared memory (a tile pair's): generic loads serve both.
__device__ __forceinline__ int4 load_dims4(const int16_t* p) {
  const short4 v = *reinterpret_cast<const short4*>(p);
  return make_int4(v.x, v.y, v.z, v.w);
}
__device__ __forceinline__ int load_dim(const int16_t* p) { return *p; }

// One warp per leaf: the listed dims of every 256-dim group in increasing order,
// each group padded with -1 to a multiple of 32 entries; dnch[leaf] = chunks of
// 32, or -1 when the list saves no chunk over the ceil(d / 32) chunks of all dims
// (the block then reads rows whole).
__global__ void __launch_bounds__(256) k_leaf_dim_list(const uint32_t* __restrict__ mask, int W, int d, int dpad,
                                                       int64_t leaves, int16_t* __restrict__ dlist,
                                                       int32_t* __restrict__ dnch, int lmax) {
  const int64_t leaf = (int64_t)blockIdx.x * 8 + (threadIdx.x >> 5);
  const int lane = threadIdx.x & 31;
  if (leaf >= leaves) return;
  const uint32_t* m = mask + leaf * W;
  const int nch = warp_dim_list<int16_t>([&](int w) { return m[w]; }, W, d, dpad, dlist + leaf * lmax);
  if (lane == 0) dnch[leaf] = nch;
}

// Tiles of rows with one zero pattern read fewer dims than tiles that mix
// patterns, and a leaf's graph does not depend on the order of its positions.
// So, with tile pairs, each tree's leaves are ordered by a bucket of the rows'
// non-zero patterns and each tile pair reads the union of its two tiles' dims.
constexpr int kBucketBits = 8;
constexpr int kMaxListDims = 4096;  // padded dims of a tile pair's list in shared memory

// bucket[row]: the top 8 bits of a hash of the row's non-zero pattern (one
// ballot word per 32 dims).  One warp per row.  *zeros (cleared beforehand)
// becomes 1 when some row has a zero among its d dims: without one, every tile
// reads rows whole, and the order and masks below are skipped.
__global__ void __launch_bounds__(256) k_row_bucket(const float* __restrict__ X, int64_t n, int d, int dpad,
                                                    uint8_t* __restrict__ bucket, uint32_t* __restrict__ zeros) {
  const int64_t row = (int64_t)blockIdx.x * 8 + (threadIdx.x >> 5);
  const int lane = threadIdx.x & 31;
  if (row >= n) return;
  const float* x = X + (size_t)row * dpad;
  uint64_t h = 0x9E3779B97F4A7C15ull;
  int nnz = 0;
  for (int d0 = 0; d0 < dpad; d0 += 32) {
    const bool nz = d0 + lane < d && x[d0 + lane] != 0.f;
    const uint32_t w = __ballot_sync(0xFFFFFFFFu, nz);
    h = (h ^ w) * 0x100000001B3ull;
    h ^= h >> 29;
    nnz += __popc(w);
  }
  if (lane == 0) {
    bucket[row] = (uint8_t)(h >> (64 - kBucketBits));
    if (nnz < d && *reinterpret_cast<volatile uint32_t*>(zeros) == 0u) atomicOr(zeros, 1u);
  }
}

// Each leaf's positions stably ordered by bucket.  One block of 1024 threads
// per leaf; warp w takes the w-th of 32 equal ranges of the leaf's positions,
// counts them per bucket, and scatters them in order after the prefix over
// (bucket, warp); tmp holds the new order until it is copied back.
__global__ void __launch_bounds__(1024) k_leaf_bucket_sort(int32_t* __restrict__ perm, SegView segs, int k,
                                                           const uint8_t* __restrict__ bucket,
                                                           int32_t* __restrict__ tmp,
                                                           const uint32_t* __restrict__ zeros) {
  constexpr int NB = 1 << kBucketBits;
  __shared__ int cnt[32][NB];
  __shared__ int tot[NB];
  if (*zeros == 0u) return;  // no zero anywhere: nothing to order
  const int64_t leaf = blockIdx.x;
  int64_t j, lo, hi, blo, bhi;
  const SegEntry seg = segs.leaf(leaf, &j);
  leaf_block(seg, j, k, &lo, &hi, &blo, &bhi);
  const int n = (int)(hi - lo);
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int per = (n + 31) / 32;
  const int r0 = min(n, warp * per), r1 = min(n, r0 + per);
  for (int e = threadIdx.x; e < 32 * NB; e += 1024) (&cnt[0][0])[e] = 0;
  __syncthreads();
  for (int r = r0 + lane; r < r1; r += 32) atomicAdd(&cnt[warp][bucket[perm[lo + r]]], 1);
  __syncthreads();
  if (threadIdx.x < NB) {
    int t = 0;
    for (int w = 0; w < 32; ++w) t += cnt[w][threadIdx.x];
    tot[threadIdx.x] = t;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    int run = 0;
    for (int b = 0; b < NB; ++b) {
      const int t = tot[b];
      tot[b] = run;
      run += t;
    }
  }
  __syncthreads();
  if (threadIdx.x < NB) {
    int run = tot[threadIdx.x];
    for (int w = 0; w < 32; ++w) {
      const int c = cnt[w][threadIdx.x];
      cnt[w][threadIdx.x] = run;
      run += c;
    }
  }
  __syncthreads();
  for (int c0 = r0; c0 < r1; c0 += 32) {
    const int r = c0 + lane;
    const bool valid = r < r1;
    const int32_t id = valid ? perm[lo + r] : -1;
    const int b = valid ? (int)bucket[id] : NB;
    const uint32_t peers = __match_any_sync(0xFFFFFFFFu, b);
    const int rank = __popc(peers & ((1u << lane) - 1u));
    if (valid) tmp[lo + cnt[warp][b] + rank] = id;
    __syncwarp();
    if (valid && rank == 0) cnt[warp][b] += __popc(peers);
    __syncwarp();
  }
  __syncthreads();
  for (int r = threadIdx.x; r < n; r += 1024) perm[lo + r] = tmp[lo + r];
}

// tmask[leaf][t][0..W): the dims non-zero in some row of the leaf's tile t
// (TILE positions), W = ceil(dpad / 32) words, every word written; word W: the
// 32-dim chunks of the tile's own list (each 256-dim group padded), so that a
// pair with a tile whose list saves nothing skips building one.  grid (leaf, tile).
__global__ void __launch_bounds__(256) k_tile_dim_mask(const float* __restrict__ X, int dpad, SegView segs, int k,
                                                       const int32_t* __restrict__ perm, int tile, int tpl,
                                                       uint32_t* __restrict__ tmask, int W,
                                                       const uint32_t* __restrict__ zeros) {
  __shared__ int gcount;
  int chunks = 0;  // thread 0
  if (*zeros == 0u) return;  // no zero anywhere: the pairs read rows whole
  const int64_t leaf = blockIdx.x;
  int64_t j, lo, hi, blo, bhi;
  const SegEntry seg = segs.leaf(leaf, &j);
  leaf_block(seg, j, k, &lo, &hi, &blo, &bhi);
  const int64_t r0 = lo + (int64_t)blockIdx.y * tile;
  if (r0 >= hi) return;
  const int64_t r1 = min(hi, r0 + tile);
  uint32_t* out = tmask + ((size_t)leaf * tpl + blockIdx.y) * (W + 1);
  for (int dim0 = 0; dim0 < dpad; dim0 += 256) {  // one 256-dim group per pass
    const int dim = dim0 + (int)threadIdx.x;
    if (threadIdx.x == 0) gcount = 0;
    __syncthreads();
    bool nz = false;
    if (dim < dpad)
      for (int64_t r = r0; r < r1 && !nz; ++r) nz = __ldg(X + (size_t)__ldg(perm + r) * dpad + dim) != 0.f;
    const uint32_t bits = __ballot_sync(0xFFFFFFFFu, nz);
    if ((threadIdx.x & 31) == 0 && dim < dpad) {
      out[dim >> 5] = bits;
      if (bits) atomicAdd(&gcount, __popc(bits));
    }
    __syncthreads();
    if (threadIdx.x == 0) chunks += (gcount + 31) / 32;
  }
  if (threadIdx.x == 0) out[W] = (uint32_t)chunks;
}


// Keys of one TILE x TILE tile: rows qid[0..mq) against columns cid[0..mc)
// (ids; -1 past the end), 16 x 16 threads each holding an R x R register
// tile, R = TILE / 16.  Each key is summed over the block's chunks of 32 dims
// (all dims, or the listed non-zero dims dl of a sparse block) in the
// reference's order: a sequential partial per 256-dim group, added to the
// total at the group's end.  Ks receives the keys, +inf outside mq x mc.
template <int METRIC, int TILE>
__device__ __forceinline__ void tile_keys(const float* __restrict__ X, int dpad, const int16_t* dl,
                                          int nchunks, int mq, int mc, const int32_t* qid, const int32_t* cid,
                                          const float* qnorm, const float* cnorm, float (*Qs)[TILE + 4],
                                          float (*Cs)[TILE + 4], float (*Ks)[TILE + 1]) {
  constexpr int R = TILE / 16;
  const int tid = threadIdx.x, ty = tid >> 4, tx = tid & 15;
  float part[R][R], total[R][R];
#pragma unroll
  for (int a = 0; a < R; ++a)
#pragma unroll
    for (int b = 0; b < R; ++b) {
      part[a][b] = 0.f;
      total[a][b] = 0.f;
    }
  for (int ch = 0; ch < nchunks; ++ch) {
    const int cd = ch * kDC;
#pragma unroll
    for (int h = 0; h < TILE / 32; ++h) {
      const int f = tid + h * 256;
      const int r = f >> 3, c4 = f & 7;
      float4 qv = make_float4(0.f, 0.f, 0.f, 0.f), cv = qv;
      if (dl) {  // four listed dims (-1: padding, read as zero)
        const int4 dm = load_dims4(dl + cd + 4 * c4);
        if (r < mq) {
          const float* row = X + (size_t)qid[r] * dpad;
          if (dm.x >= 0) qv.x = __ldg(row + dm.x);
          if (dm.y >= 0) qv.y = __ldg(row + dm.y);
          if (dm.z >= 0) qv.z = __ldg(row + dm.z);
          if (dm.w >= 0) qv.w = __ldg(row + dm.w);
        }
        if (r < mc) {
          const float* row = X + (size_t)cid[r] * dpad;
          if (dm.x >= 0) cv.x = __ldg(row + dm.x);
          if (dm.y >= 0) cv.y = __ldg(row + dm.y);
          if (dm.z >= 0) cv.z = __ldg(row + dm.z);
          if (dm.w >= 0) cv.w = __ldg(row + dm.w);
        }
      } else {
        const int dim = cd + 4 * c4;
        if (r < mq && dim < dpad) qv = __ldg(reinterpret_cast<const float4*>(X + (size_t)qid[r] * dpad + dim));
        if (r < mc && dim < dpad) cv = __ldg(reinterpret_cast<const float4*>(X + (size_t)cid[r] * dpad + dim));
      }
      Qs[4 * c4 + 0][r] = qv.x;
      Qs[4 * c4 + 1][r] = qv.y;
      Qs[4 * c4 + 2][r] = qv.z;
      Qs[4 * c4 + 3][r] = qv.w;
      Cs[4 * c4 + 0][r] = cv.x;
      Cs[4 * c4 + 1][r] = cv.y;
      Cs[4 * c4 + 2][r] = cv.z;
      Cs[4 * c4 + 3][r] = cv.w;
    }
    __syncthreads();
#pragma unroll 8
    for (int dd = 0; dd < kDC; ++dd) {
      float qa[R], cb[R];
      load_r<R>(&Qs[dd][ty * R], qa);
      load_r<R>(&Cs[dd][tx * R], cb);
#pragma unroll
      for (int a = 0; a < R; ++a)
#pragma unroll
        for (int b = 0; b < R; ++b) part[a][b] = acc_step<METRIC>(qa[a], cb[b], part[a][b]);
    }
    // end of a 256-dim group: its partial sum joins the total
    const bool gend = ch == nchunks - 1 ||
                      (dl ? (load_dim(dl + cd + kDC) >> 8) != (load_dim(dl + cd) >> 8) : ((cd + kDC) & 255) == 0);
    if (gend) {
#pragma unroll
      for (int a = 0; a < R; ++a)
#pragma unroll
        for (int b = 0; b < R; ++b) {
          total[a][b] = __fadd_rn(total[a][b], part[a][b]);
          part[a][b] = 0.f;
        }
    }
    __syncthreads();
  }
  const float kInf = __int_as_float(0x7F800000);
#pragma unroll
  for (int a = 0; a < R; ++a)
#pragma unroll
    for (int b = 0; b < R; ++b) {
      const int qq = ty * R + a, cc = tx * R + b;
      float key = total[a][b];
      if (METRIC == KNN_METRIC_COSINE) key = cosine_key(key, qnorm[qq], cnorm[cc]);
      Ks[qq][cc] = (qq < mq && cc < mc) ? key : kInf;
    }
}

// Merge rows rowid[0..mrow) of a tile into their running sorted lists against
// the tile's columns colid[0..mcol): keys Ks[row][col], or Ks[col][row] when
// TRANS (the tile read from its other side: every key is symmetric in its two
// points, bit for bit).  One warp per row: bitonic insertion via shuffles.
template <int KPL, int TILE, bool TRANS>
__device__ __forceinline__ void merge_rows(int k, int mrow, int mcol, const int32_t* rowid, const int32_t* colid,
                                           const float (*Ks)[TILE + 1], float* __restrict__ rkey,
                                           uint32_t* __restrict__ rid) {
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const float kInf = __int_as_float(0x7F800000);
  for (int rr = warp; rr < mrow; rr += 8) {
    const uint32_t i = (uint32_t)rowid[rr];
    WarpList<KPL> L;
#pragma unroll
    for (int r = 0; r < KPL; ++r) {
      const int e = r * 32 + lane;
      if (e < k) {
        L.key[r] = rkey[(size_t)i * k + e];
        L.id[r] = rid[(size_t)i * k + e];
      } else {
        L.key[r] = kInf;
        L.id[r] = kNoId;
      }
    }
    for (int cb = 0; cb < mcol; cb += 32) {
      const int c = cb + lane;
      const bool inrange = c < mcol;
      const float ck = inrange ? (TRANS ? Ks[c][rr] : Ks[rr][c]) : kInf;
      const uint32_t ci = inrange ? (uint32_t)colid[c] : kNoId;
      float tk;
      uint32_t ti;
      warp_list_get(L, k - 1, tk, ti);
      bool pass = inrange && ci != i && cand_less(ck, ci, tk, ti);
      if (!__any_sync(0xFFFFFFFFu, pass)) continue;
      const bool dup = warp_list_contains(L, ci, k);
      pass = pass && !dup;
      if (!__any_sync(0xFFFFFFFFu, pass)) continue;
      warp_list_insert(L, pass ? ck : kInf, pass ? ci : kNoId);
    }
#pragma unroll
    for (int r = 0; r < KPL; ++r) {
      const int e = r * 32 + lane;
      if (e < k) {
        rkey[(size_t)i * k + e] = L.key[r];
        rid[(size_t)i * k + e] = L.id[r];
      }
    }
  }
}

// Every key is summed over dims in the same order whatever the tile, and each
// row's list is the k best of the union under (key, id), so all TILE variants
// (and the pair schedule below) give identical lists.
template <int METRIC, int KPL, int TILE>
__global__ void __launch_bounds__(256, TILE == 64 ? 4 : 5) k_leaf(const float* __restrict__ X, int d, int dpad,
                                              SegView segs, const int64_t* __restrict__ ftab, int k,
                                              const int32_t* __restrict__ perm,
                                              const float* __restrict__ norms,
                                              float* __restrict__ rkey, uint32_t* __restrict__ rid,
                                              unsigned long long* __restrict__ pair_counter,
                                              const int16_t* __restrict__ dlist,
                                              const int32_t* __restrict__ dnch, int lmax) {
  constexpr int kTile = TILE;
  static_assert(TILE == 32 || TILE == 64, "tile of 32 or 64");
  __shared__ __align__(16) float Qs[kDC][TILE + 4];
  __shared__ __align__(16) float Cs[kDC][TILE + 4];
  __shared__ float Ks[kTile][kTile + 1];
  __shared__ int32_t qid[kTile], cid[kTile];
  __shared__ float qnorm[kTile], cnorm[kTile];

  // block = (leaf, query tile): the 64-row (or 32-row) query tiles of a large
  // leaf spread over gridDim.y, and each query row's list is read and written
  // by one block only
  const int64_t leaf = blockIdx.x;
  int64_t lo, hi, blo, bhi;
  if (ftab) {  // explicit leaf table (reference-rule trees)
    const int64_t* e = ftab + 4 * leaf;
    lo = e[0];
    hi = e[1];
    blo = e[2];
    bhi = e[3];
  } else {
    int64_t j;
    const SegEntry seg = segs.leaf(leaf, &j);
    leaf_block(seg, j, k, &lo, &hi, &blo, &bhi);
  }
  const int nq = (int)(hi - lo);
  const int nb = (int)(bhi - blo);
  const int tid = threadIdx.x;
  // sparse rows: this block's non-zero dims, 32 per chunk (null: all dims)
  const int16_t* dl = nullptr;
  int nchunks = (d + kDC - 1) / kDC;
  if (METRIC != KNN_METRIC_COSINE && dlist && dnch[leaf] >= 0) {
    dl = dlist + leaf * lmax;
    nchunks = dnch[leaf];
  }

  for (int q0 = (int)blockIdx.y * kTile; q0 < nq; q0 += (int)gridDim.y * kTile) {
    if (pair_counter && tid == 0)
      atomicAdd(pair_counter, (unsigned long long)min(kTile, nq - q0) * (unsigned long long)(nb - 1));
    const int mq = min(kTile, nq - q0);
    if (tid < kTile) {
      const int32_t id = tid < mq ? perm[lo + q0 + tid] : -1;
      qid[tid] = id;
      if (METRIC == KNN_METRIC_COSINE) qnorm[tid] = id >= 0 ? norms[id] : 0.f;
    }
    for (int c0 = 0; c0 < nb; c0 += kTile) {
      const int mc = min(kTile, nb - c0);
      if (tid < kTile) {
        const int32_t id = tid < mc ? perm[blo + c0 + tid] : -1;
        cid[tid] = id;
        if (METRIC == KNN_METRIC_COSINE) cnorm[tid] = id >= 0 ? norms[id] : 0.f;
      }
      __syncthreads();
      tile_keys<METRIC, TILE>(X, dpad, dl, nchunks, mq, mc, qid, cid, qnorm, cnorm, Qs, Cs, Ks);
      __syncthreads();
      merge_rows<KPL, TILE, false>(k, mq, mc, qid, cid, Ks, rkey, rid);
      __syncthreads();
    }
  }
}

// Tile pairs of a leaf that is its own block (queries = candidates): the key of
// (q, c) equals the key of (c, q) bit for bit (the terms are |q-c|, (q-c)^2 or
// q*c in the same dim order), so each unordered pair of a leaf's T tiles is
// computed once and merged into both tiles' rows.  The pairs are scheduled in
// rounds by the circle method over T' = T rounded up to even: in round r < T'-1
// pair i is (r, T'-1) for i = 0, else ((r + i) mod (T'-1), (r - i) mod (T'-1));
// the pairs of one round are disjoint, so each row's list is read and written
// by one block per round.  Round T'-1 takes the diagonal tiles (t, t).  Pairs
// with a tile past the leaf's own T are skipped.  One launch per round.
// Sparse rows: with tmask (per-tile dim masks, W words each, tpl tiles per
// leaf) a block reads the union of its two tiles' non-zero dims, listed in
// shared memory; else with dlist the leaf block's list.
template <int METRIC, int KPL, int TILE>
__global__ void __launch_bounds__(256, TILE == 64 ? 4 : 5) k_leaf_pair(
    const float* __restrict__ X, int d, int dpad, SegView segs, int k, const int32_t* __restrict__ perm,
    const float* __restrict__ norms, float* __restrict__ rkey, uint32_t* __restrict__ rid,
    unsigned long long* __restrict__ pair_counter, const int16_t* __restrict__ dlist,
    const int32_t* __restrict__ dnch, int lmax, const uint32_t* __restrict__ tmask, int tpl, int W,
    const uint32_t* __restrict__ zeros, int round, int tpr) {
  static_assert(TILE == 32 || TILE == 64, "tile of 32 or 64");
  __shared__ __align__(16) float Qs[kDC][TILE + 4];
  __shared__ __align__(16) float Cs[kDC][TILE + 4];
  __shared__ float Ks[TILE][TILE + 1];
  __shared__ int32_t qid[TILE], cid[TILE];
  __shared__ float qnorm[TILE], cnorm[TILE];
  __shared__ __align__(16) int16_t sl[METRIC == KNN_METRIC_COSINE ? 4 : kMaxListDims];
  __shared__ int snch;

  const int64_t leaf = blockIdx.x;
  int64_t j, lo, hi, blo, bhi;
  const SegEntry seg = segs.leaf(leaf, &j);
  leaf_block(seg, j, k, &lo, &hi, &blo, &bhi);  // the host launches this only when blo = lo, bhi = hi
  const int n = (int)(hi - lo);
  const int T = (n + TILE - 1) / TILE;
  int a, b;
  if (round == tpr - 1) {
    a = b = (int)blockIdx.y;
  } else {
    const int m = tpr - 1;
    const int i = (int)blockIdx.y;
    a = i == 0 ? round : (round + i) % m;
    b = i == 0 ? m : (round - i + m) % m;
  }
  if (a >= T || b >= T) return;
  const int tid = threadIdx.x;
  const int16_t* dl = nullptr;
  int nchunks = (d + kDC - 1) / kDC;
  if (METRIC != KNN_METRIC_COSINE && dlist && !tmask && dnch[leaf] >= 0) {
    dl = dlist + leaf * lmax;
    nchunks = dnch[leaf];
  }
  // the union of two tiles' dims lists no fewer chunks than either tile's own
  // list, so a pair with a tile whose list saves nothing reads rows whole
  const uint32_t* ma = tmask ? tmask + ((size_t)leaf * tpl + a) * (W + 1) : nullptr;
  const uint32_t* mb = tmask ? tmask + ((size_t)leaf * tpl + b) * (W + 1) : nullptr;
  const bool listed = METRIC != KNN_METRIC_COSINE && tmask && *zeros != 0u && (int)__ldg(ma + W) < nchunks &&
                      (int)__ldg(mb + W) < nchunks;  // block-uniform
  if (listed) {
    if (tid < 32) {
      const int nch = warp_dim_list<int16_t>([&](int w) { return __ldg(ma + w) | __ldg(mb + w); }, W, d, dpad, sl);
      if (tid == 0) snch = nch;
    }
    __syncthreads();
    if (snch >= 0) {
      nchunks = snch;
      dl = sl;
    }
  }
  const int mq = min(TILE, n - a * TILE), mc = min(TILE, n - b * TILE);
  if (pair_counter && tid == 0)
    atomicAdd(pair_counter, a == b ? (unsigned long long)mq * (unsigned long long)(mq - 1)
                                   : 2ull * (unsigned long long)mq * (unsigned long long)mc);
  if (tid < TILE) {
    const int32_t qi = tid < mq ? perm[lo + a * TILE + tid] : -1;
    const int32_t ci = tid < mc ? perm[lo + b * TILE + tid] : -1;
    qid[tid] = qi;
    cid[tid] = ci;
    if (METRIC == KNN_METRIC_COSINE) {
      qnorm[tid] = qi >= 0 ? norms[qi] : 0.f;
      cnorm[tid] = ci >= 0 ? norms[ci] : 0.f;
    }
  }
  __syncthreads();
  tile_keys<METRIC, TILE>(X, dpad, dl, nchunks, mq, mc, qid, cid, qnorm, cnorm, Qs, Cs, Ks);
  __syncthreads();
  merge_rows<KPL, TILE, false>(k, mq, mc, qid, cid, Ks, rkey, rid);
  if (a != b) merge_rows<KPL, TILE, true>(k, mc, mq, cid, qid, Ks, rkey, rid);
}

// Rounds of the pair schedule for leaves of at most maxleaf points: T' = the
// tiles of the largest leaf rounded up to even; 0 when the schedule does not
// apply (a leaf of one tile, or more tiles than a grid dimension holds).
template <int TILE>
static int pair_tiles(int64_t maxleaf) {
  const int64_t t = (maxleaf + TILE - 1) / TILE;
  const int64_t tp = (t + 1) / 2 * 2;
  return (t >= 2 && tp <= 65535) ? (int)tp : 0;
}

// Sparse tile pairs: each leaf's positions ordered by row bucket, then the
// dim masks of its tiles (two launches before the rounds).
template <int TILE>
static int sparse_tile_masks(const LeafArgs& a, int32_t* perm, int64_t leaves, int tpl, int W) {
  k_leaf_bucket_sort<<<(unsigned)leaves, 1024, 0, a.stream>>>(perm, a.segs, a.k, a.bucket, a.sort_tmp,
                                                               a.zeros);
  k_tile_dim_mask<<<dim3((unsigned)leaves, (unsigned)tpl), 256, 0, a.stream>>>(a.X, a.dpad, a.segs, a.k, perm, TILE,
                                                                               tpl, a.tmask, W, a.zeros);
  return 2;
}

template <int METRIC, int TILE>
static int launch_leaf_tile(const LeafArgs& a, const int32_t* perm, const int64_t* ftab, int64_t leaves, int kpl,
                            const int16_t* dlist, int32_t* perm_w) {
  if (leaves <= 0) return 0;
  const int tpr = (a.pairs && !ftab) ? pair_tiles<TILE>(a.maxleaf) : 0;
  if (tpr) {
    const int tpl = (int)((a.maxleaf + TILE - 1) / TILE);
    const int W = (a.dpad + 31) / 32;
    int extra = 0;
    const uint32_t* tmask = nullptr;
    if (METRIC != KNN_METRIC_COSINE && a.tmask && perm_w && a.dpad <= kMaxListDims) {
      extra = sparse_tile_masks<TILE>(a, perm_w, leaves, tpl, W);
      tmask = a.tmask;
      dlist = nullptr;
    }
    for (int r = 0; r < tpr; ++r) {
      const dim3 grid((unsigned)leaves, (unsigned)(r == tpr - 1 ? tpr : tpr / 2));
      if (kpl == 1)
        k_leaf_pair<METRIC, 1, TILE><<<grid, 256, 0, a.stream>>>(a.X, a.d, a.dpad, a.segs, a.k, perm, a.norms, a.rkey,
                                                                  a.rid, a.pair_counter, dlist, a.dnch, a.lmax, tmask,
                                                                  tpl, W, a.zeros, r, tpr);
      else if (kpl == 2)
        k_leaf_pair<METRIC, 2, TILE><<<grid, 256, 0, a.stream>>>(a.X, a.d, a.dpad, a.segs, a.k, perm, a.norms, a.rkey,
                                                                  a.rid, a.pair_counter, dlist, a.dnch, a.lmax, tmask,
                                                                  tpl, W, a.zeros, r, tpr);
      else
        k_leaf_pair<METRIC, 4, TILE><<<grid, 256, 0, a.stream>>>(a.X, a.d, a.dpad, a.segs, a.k, perm, a.norms, a.rkey,
                                                                  a.rid, a.pair_counter, dlist, a.dnch, a.lmax, tmask,
                                                                  tpl, W, a.zeros, r, tpr);
    }
    return tpr + extra;
  }
  const int64_t qtiles = (a.maxleaf + TILE - 1) / TILE;
  dim3 grid((unsigned)leaves, (unsigned)std::min<int64_t>(qtiles, 65535));
  if (kpl == 1)
    k_leaf<METRIC, 1, TILE><<<grid, 256, 0, a.stream>>>(a.X, a.d, a.dpad, a.segs, ftab, a.k, perm, a.norms, a.rkey, a.rid, a.pair_counter, dlist, a.dnch, a.lmax);
  else if (kpl == 2)
    k_leaf<METRIC, 2, TILE><<<grid, 256, 0, a.stream>>>(a.X, a.d, a.dpad, a.segs, ftab, a.k, perm, a.norms, a.rkey, a.rid, a.pair_counter, dlist, a.dnch, a.lmax);
  else
    k_leaf<METRIC, 4, TILE><<<grid, 256, 0, a.stream>>>(a.X, a.d, a.dpad, a.segs, ftab, a.k, perm, a.norms, a.rkey, a.rid, a.pair_counter, dlist, a.dnch, a.lmax);
  return 1;
}

template <int METRIC>
static void launch_leaf_metric(const LeafArgs& a, int t, int kpl, LaunchLog& log) {
  const int32_t* perm = a.perm + (size_t)t * a.n;
  const int64_t* ftab = a.ftable ? a.ftable + 4 * a.foff[t] : nullptr;
  const int64_t leaves = a.ftable ? a.fcount[t] : a.leaves;
  const int16_t* dlist = nullptr;
  int32_t* perm_w = a.perm_w ? a.perm_w + (size_t)t * a.n : nullptr;
  if (a.dlist && !a.tmask && !ftab && METRIC != KNN_METRIC_COSINE && leaves > 0) {
    const int W = a.dpad / 32 + 1;
    cudaMemsetAsync(a.dmask, 0, sizeof(uint32_t) * (size_t)leaves * W, a.stream);
    const int64_t splits = (std::max(a.maxblock, a.maxleaf) + kDimRows - 1) / kDimRows;
    k_leaf_dim_mask<<<dim3((unsigned)leaves, (unsigned)std::min<int64_t>(splits, 65535)), 256, 0, a.stream>>>(
        a.X, a.dpad, a.segs, a.k, perm, a.dmask, W);
    k_leaf_dim_list<<<(unsigned)((leaves + 7) / 8), 256, 0, a.stream>>>(a.dmask, W, a.d, a.dpad, leaves,
                                                                        a.dlist, a.dnch, a.lmax);
    log.add(3);
    dlist = a.dlist;
  }
  const int launches = a.tile == 32 ? launch_leaf_tile<METRIC, 32>(a, perm, ftab, leaves, kpl, dlist, perm_w)
                                    : launch_leaf_tile<METRIC, 64>(a, perm, ftab, leaves, kpl, dlist, perm_w);
  log.add(launches);
}

// One launch per tree: a point sits in one leaf per tree, so the leaves of a
// tree update disjoint lists, and stream order serialises the trees.
int leaf_stage(const LeafArgs& a, LaunchLog& log) {
  const int kpl = kpl_for(a.k);
  if (a.tmask && a.bucket && a.n > 0) {
    cudaMemsetAsync(a.zeros, 0, sizeof(uint32_t), a.stream);
    k_row_bucket<<<(unsigned)((a.n + 7) / 8), 256, 0, a.stream>>>(a.X, a.n, a.d, a.dpad, a.bucket, a.zeros);
    log.add();
  }
  for (int t = a.first_tree; t < a.first_tree + a.trees; ++t) {
    if (a.kev) cudaEventRecord(a.kev[2 * (t - a.first_tree)], a.stream);
    if (a.metric == KNN_METRIC_EUCLIDEAN) launch_leaf_metric<KNN_METRIC_EUCLIDEAN>(a, t, kpl, log);
    else if (a.metric == KNN_METRIC_TAXICAB) launch_leaf_metric<KNN_METRIC_TAXICAB>(a, t, kpl, log);
    else launch_leaf_metric<KNN_METRIC_COSINE>(a, t, kpl, log);
    if (a.kev) cudaEventRecord(a.kev[2 * (t - a.first_tree) + 1], a.stream);
  }
  return cudaPeekAtLastError() == cudaSuccess ? KNN_OK : KNN_ERR_CUDA;
}

}  // namespace knn
