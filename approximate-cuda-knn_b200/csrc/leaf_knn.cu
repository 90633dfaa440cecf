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

// TILE x TILE (query x candidate) tiles, 16 x 16 threads each holding an
// R x R register tile, R = TILE / 16.  Every key is summed over dims in the
// same order whatever the tile, and each row's list is the k best of the
// union under (key, id), so all TILE variants give identical lists.
template <int METRIC, int KPL, int TILE>
__global__ void __launch_bounds__(256, TILE == 64 ? 4 : 5) k_leaf(const float* __restrict__ X, int d, int dpad,
                                              SegView segs, const int64_t* __restrict__ ftab, int k,
                                              const int32_t* __restrict__ perm,
                                              const float* __restrict__ norms,
                                              float* __restrict__ rkey, uint32_t* __restrict__ rid,
                                              unsigned long long* __restrict__ pair_counter) {
  constexpr int kTile = TILE;
  constexpr int kSP = TILE + 4;
  constexpr int R = TILE / 16;
  static_assert(R == 2 || R == 4, "tile of 32 or 64");
  __shared__ __align__(16) float Qs[kDC][kSP];
  __shared__ __align__(16) float Cs[kDC][kSP];
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

  const int tid = threadIdx.x, ty = tid >> 4, tx = tid & 15;
  const int warp = tid >> 5, lane = tid & 31;
  const float kInf = __int_as_float(0x7F800000);
  const int nchunks = (d + kDC - 1) / kDC;

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
        for (int h = 0; h < kTile / 32; ++h) {
          const int f = tid + h * 256;
          const int r = f >> 3, c4 = f & 7;
          const int dim = cd + 4 * c4;
          float4 qv = make_float4(0.f, 0.f, 0.f, 0.f), cv = qv;
          if (r < mq && dim < dpad) qv = __ldg(reinterpret_cast<const float4*>(X + (size_t)qid[r] * dpad + dim));
          if (r < mc && dim < dpad) cv = __ldg(reinterpret_cast<const float4*>(X + (size_t)cid[r] * dpad + dim));
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
        if (((cd + kDC) & 255) == 0 || ch == nchunks - 1) {
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
#pragma unroll
      for (int a = 0; a < R; ++a)
#pragma unroll
        for (int b = 0; b < R; ++b) {
          const int qq = ty * R + a, cc = tx * R + b;
          float key = total[a][b];
          if (METRIC == KNN_METRIC_COSINE) key = cosine_key(key, qnorm[qq], cnorm[cc]);
          Ks[qq][cc] = (qq < mq && cc < mc) ? key : kInf;
        }
      __syncthreads();

      // Merge every query row of the tile into its running list.
      for (int qq = warp; qq < mq; qq += 8) {
        const uint32_t i = (uint32_t)qid[qq];
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
        for (int cb = 0; cb < mc; cb += 32) {
          const int c = cb + lane;
          const bool inrange = c < mc;
          const float ck = inrange ? Ks[qq][c] : kInf;
          const uint32_t ci = inrange ? (uint32_t)cid[c] : kNoId;
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
      __syncthreads();
    }
  }
}

template <int METRIC, int TILE>
static void launch_leaf_tile(const LeafArgs& a, const int32_t* perm, const int64_t* ftab, int64_t leaves, int kpl) {
  if (leaves <= 0) return;
  const int64_t qtiles = (a.maxleaf + TILE - 1) / TILE;
  dim3 grid((unsigned)leaves, (unsigned)std::min<int64_t>(qtiles, 65535));
  if (kpl == 1)
    k_leaf<METRIC, 1, TILE><<<grid, 256, 0, a.stream>>>(a.X, a.d, a.dpad, a.segs, ftab, a.k, perm, a.norms, a.rkey, a.rid, a.pair_counter);
  else if (kpl == 2)
    k_leaf<METRIC, 2, TILE><<<grid, 256, 0, a.stream>>>(a.X, a.d, a.dpad, a.segs, ftab, a.k, perm, a.norms, a.rkey, a.rid, a.pair_counter);
  else
    k_leaf<METRIC, 4, TILE><<<grid, 256, 0, a.stream>>>(a.X, a.d, a.dpad, a.segs, ftab, a.k, perm, a.norms, a.rkey, a.rid, a.pair_counter);
}

template <int METRIC>
static void launch_leaf_metric(const LeafArgs& a, int t, int kpl) {
  const int32_t* perm = a.perm + (size_t)t * a.n;
  const int64_t* ftab = a.ftable ? a.ftable + 4 * a.foff[t] : nullptr;
  const int64_t leaves = a.ftable ? a.fcount[t] : a.leaves;
  if (a.tile == 32) launch_leaf_tile<METRIC, 32>(a, perm, ftab, leaves, kpl);
  else launch_leaf_tile<METRIC, 64>(a, perm, ftab, leaves, kpl);
}

// One launch per tree: a point sits in one leaf per tree, so the leaves of a
// tree update disjoint lists, and stream order serialises the trees.
int leaf_stage(const LeafArgs& a, LaunchLog& log) {
  const int kpl = kpl_for(a.k);
  for (int t = a.first_tree; t < a.first_tree + a.trees; ++t) {
    if (a.kev) cudaEventRecord(a.kev[2 * (t - a.first_tree)], a.stream);
    if (a.metric == KNN_METRIC_EUCLIDEAN) launch_leaf_metric<KNN_METRIC_EUCLIDEAN>(a, t, kpl);
    else if (a.metric == KNN_METRIC_TAXICAB) launch_leaf_metric<KNN_METRIC_TAXICAB>(a, t, kpl);
    else launch_leaf_metric<KNN_METRIC_COSINE>(a, t, kpl);
    if (a.kev) cudaEventRecord(a.kev[2 * (t - a.first_tree) + 1], a.stream);
    log.add();
  }
  return cudaPeekAtLastError() == cudaSuccess ? KNN_OK : KNN_ERR_CUDA;
}

}  // namespace knn
