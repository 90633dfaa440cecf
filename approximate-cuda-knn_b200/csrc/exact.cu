// Exact k-NN in FP64 on the GPU: the yardstick of recall and distance error.
// No counterpart in the reference (which never checks its own output; its
// VALIDATION file is written unconditionally, euclideandistancematrixgpu.cu:2967-2971).
//
// Arithmetic matches a plain sequential double loop without contraction:
//   L2:  sqrt(sum (a-b)^2),  L1: sum |a-b|,  COS: 1 - sum ab / (sqrt(sum a^2) sqrt(sum b^2))
// and ties break by index, so the result equals a CPU double-precision brute force.
//
// Layout: a block owns 64 queries and one slice of the points; the 64x64
// distance tile is built by a 4x4 register tile per thread (points staged 8
// dims at a time in shared memory), each warp keeps the sorted k best of 8
// queries in registers.  A second kernel merges the slices.
#include "knn_internal.cuh"
#include "knn_kernels.cuh"

namespace knn {

namespace {
constexpr int kET = 64;
constexpr int kEDC = 8;  // keeps the static shared memory under 48 KB
}  // namespace

__global__ void k_exact_norms(const float* __restrict__ X, int64_t n, int d, int dpad,
                              double* __restrict__ out) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const float* a = X + (size_t)i * dpad;
  double s = 0.0;
  for (int e = 0; e < d; ++e) s = __dadd_rn(s, __dmul_rn((double)a[e], (double)a[e]));
  out[i] = sqrt(s);
}

template <int METRIC, int KPL>
__global__ void __launch_bounds__(256) k_exact(const float* __restrict__ X, int64_t n, int d,
                                               int dpad, int k, const int64_t* __restrict__ queries,
                                               int64_t nq, const double* __restrict__ norms,
                                               int64_t slice, double* __restrict__ part_dist,
                                               uint32_t* __restrict__ part_idx) {
  __shared__ double Qs[kEDC][kET + 1];
  __shared__ double Cs[kEDC][kET + 1];
  __shared__ double Ks[kET][kET + 1];
  __shared__ int64_t qrow[kET];
  const int tid = threadIdx.x, ty = tid >> 4, tx = tid & 15, warp = tid >> 5, lane = tid & 31;
  const int64_t q0 = (int64_t)blockIdx.x * kET;
  const int mq = (int)min((int64_t)kET, nq - q0);
  const int64_t c_begin = (int64_t)blockIdx.y * slice;
  const int64_t c_end = min(n, c_begin + slice);
  const double kInf = __longlong_as_double(0x7FF0000000000000LL);
  if (tid < kET) qrow[tid] = tid < mq ? queries[q0 + tid] : -1;
  __syncthreads();

  WarpList<KPL, double> L[8];
#pragma unroll
  for (int s = 0; s < 8; ++s)
#pragma unroll
    for (int r = 0; r < KPL; ++r) {
      L[s].key[r] = kInf;
      L[s].id[r] = kNoId;
    }

  for (int64_t c0 = c_begin; c0 < c_end; c0 += kET) {
    const int mc = (int)min((int64_t)kET, c_end - c0);
    double acc[4][4];
#pragma unroll
    for (int a = 0; a < 4; ++a)
#pragma unroll
      for (int b = 0; b < 4; ++b) acc[a][b] = 0.0;
    for (int cd = 0; cd < d; cd += kEDC) {
      for (int f = tid; f < kET * kEDC; f += 256) {
        const int r = f / kEDC, e = f % kEDC;
        const int dim = cd + e;
        double qv = 0.0, cv = 0.0;
        if (r < mq && dim < d) qv = (double)X[(size_t)qrow[r] * dpad + dim];
        if (r < mc && dim < d) cv = (double)X[(size_t)(c0 + r) * dpad + dim];
        Qs[e][r] = qv;
        Cs[e][r] = cv;
      }
      __syncthreads();
      const int lim = min(kEDC, d - cd);
      for (int e = 0; e < lim; ++e) {
        double qa[4], cb[4];
#pragma unroll
        for (int a = 0; a < 4; ++a) qa[a] = Qs[e][ty * 4 + a];
#pragma unroll
        for (int b = 0; b < 4; ++b) cb[b] = Cs[e][tx * 4 + b];
#pragma unroll
        for (int a = 0; a < 4; ++a)
#pragma unroll
          for (int b = 0; b < 4; ++b) {
            if (METRIC == KNN_METRIC_EUCLIDEAN) {
              const double t = __dsub_rn(qa[a], cb[b]);
              acc[a][b] = __dadd_rn(acc[a][b], __dmul_rn(t, t));
            } else if (METRIC == KNN_METRIC_TAXICAB) {
              acc[a][b] = __dadd_rn(acc[a][b], fabs(__dsub_rn(qa[a], cb[b])));
            } else {
              acc[a][b] = __dadd_rn(acc[a][b], __dmul_rn(qa[a], cb[b]));
            }
          }
      }
      __syncthreads();
    }
#pragma unroll
    for (int a = 0; a < 4; ++a)
#pragma unroll
      for (int b = 0; b < 4; ++b) {
        const int qq = ty * 4 + a, cc = tx * 4 + b;
        double v = acc[a][b];
        if (METRIC == KNN_METRIC_EUCLIDEAN) v = sqrt(v);
        if (METRIC == KNN_METRIC_COSINE && qq < mq && cc < mc) {
          const double den = __dmul_rn(norms[qrow[qq]], norms[c0 + cc]);
          v = den == 0.0 ? 1.0 : __dsub_rn(1.0, __ddiv_rn(v, den));
        }
        const bool ok = qq < mq && cc < mc && qrow[qq] != c0 + cc;
        Ks[qq][cc] = ok ? v : kInf;
      }
    __syncthreads();
#pragma unroll
    for (int s = 0; s < 8; ++s) {
      const int qq = warp * 8 + s;
      if (qq >= mq) continue;
      for (int cb = 0; cb < mc; cb += 32) {
        const int c = cb + lane;
        const double ck = c < mc ? Ks[qq][c] : kInf;
        const uint32_t ci = c < mc ? (uint32_t)(c0 + c) : kNoId;
        double tk;
        uint32_t ti;
        warp_list_get(L[s], k - 1, tk, ti);
        const bool pass = ck < kInf && cand_less(ck, ci, tk, ti);
        if (__any_sync(0xFFFFFFFFu, pass)) warp_list_insert(L[s], pass ? ck : kInf, pass ? ci : kNoId);
      }
    }
    __syncthreads();
  }
  // partial result of this slice: [slice][query][k]
#pragma unroll
  for (int s = 0; s < 8; ++s) {
    const int qq = warp * 8 + s;
    if (qq >= mq) continue;
    const size_t row = ((size_t)blockIdx.y * nq + (q0 + qq)) * k;
#pragma unroll
    for (int r = 0; r < KPL; ++r) {
      const int e = r * 32 + lane;
      if (e < k) {
        part_dist[row + e] = L[s].key[r];
        part_idx[row + e] = L[s].id[r];
      }
    }
  }
}

// One warp per query: k best over the slices.
template <int KPL>
__global__ void k_exact_merge(int64_t nq, int k, int slices, const double* __restrict__ part_dist,
                              const uint32_t* __restrict__ part_idx, double* __restrict__ out_dist,
                              int32_t* __restrict__ out_idx) {
  const int64_t q = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int lane = threadIdx.x & 31;
  if (q >= nq) return;
  const double kInf = __longlong_as_double(0x7FF0000000000000LL);
  WarpList<KPL, double> L;
#pragma unroll
  for (int r = 0; r < KPL; ++r) {
    L.key[r] = kInf;
    L.id[r] = kNoId;
  }
  for (int s = 0; s < slices; ++s) {
    const size_t row = ((size_t)s * nq + q) * k;
    for (int e0 = 0; e0 < k; e0 += 32) {
      const int e = e0 + lane;
      const double ck = e < k ? part_dist[row + e] : kInf;
      const uint32_t ci = e < k ? part_idx[row + e] : kNoId;
      const bool pass = ck < kInf;
      if (__any_sync(0xFFFFFFFFu, pass)) warp_list_insert(L, pass ? ck : kInf, pass ? ci : kNoId);
    }
  }
#pragma unroll
  for (int r = 0; r < KPL; ++r) {
    const int e = r * 32 + lane;
    if (e < k) {
      out_dist[q * k + e] = L.key[r];
      out_idx[q * k + e] = (int32_t)L.id[r];
    }
  }
}

int exact_fp64(const float* X, int64_t n, int d, int dpad, int k, int metric,
               const int64_t* queries, int64_t nq, double* norms, double* part_dist,
               uint32_t* part_idx, int slices, double* out_dist, int32_t* out_idx,
               cudaStream_t st) {
  if (metric == KNN_METRIC_COSINE)
    k_exact_norms<<<(unsigned)((n + 127) / 128), 128, 0, st>>>(X, n, d, dpad, norms);
  const int64_t slice = (n + slices - 1) / slices;
  dim3 grid((unsigned)((nq + kET - 1) / kET), (unsigned)slices);
  const int kpl = kpl_for(k);
#define KNN_EXACT(M, KP) k_exact<M, KP><<<grid, 256, 0, st>>>(X, n, d, dpad, k, queries, nq, norms, slice, part_dist, part_idx)
#define KNN_EXACT_M(M) \
  do { if (kpl == 1) KNN_EXACT(M, 1); else if (kpl == 2) KNN_EXACT(M, 2); else KNN_EXACT(M, 4); } while (0)
  if (metric == KNN_METRIC_EUCLIDEAN) KNN_EXACT_M(KNN_METRIC_EUCLIDEAN);
  else if (metric == KNN_METRIC_TAXICAB) KNN_EXACT_M(KNN_METRIC_TAXICAB);
  else KNN_EXACT_M(KNN_METRIC_COSINE);
#undef KNN_EXACT_M
#undef KNN_EXACT
  const unsigned mb = (unsigned)((nq * 32 + 255) / 256);
  if (kpl == 1) k_exact_merge<1><<<mb, 256, 0, st>>>(nq, k, slices, part_dist, part_idx, out_dist, out_idx);
  else if (kpl == 2) k_exact_merge<2><<<mb, 256, 0, st>>>(nq, k, slices, part_dist, part_idx, out_dist, out_idx);
  else k_exact_merge<4><<<mb, 256, 0, st>>>(nq, k, slices, part_dist, part_idx, out_dist, out_idx);
  return cudaPeekAtLastError() == cudaSuccess ? KNN_OK : KNN_ERR_CUDA;
}

}  // namespace knn
