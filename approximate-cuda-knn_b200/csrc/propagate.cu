// Neighbour propagation, one Jacobi step: N'(i) = k best of N(i) u N(N(i)) \ {i}.
//
// Replaces propagate{Euclidean,Taxicab,Cosine}Kernel and the host loop
// (euclideandistancematrixgpu.cu:1033-1935, :1937-1977).  The reference marks
// N(N(i)) in an N-byte bitmap per point, clears N(i) and i, scans the bitmap and
// histogram-selects; here one warp owns one point:
//   * candidates come from the k lists of its neighbours (coalesced 4k-byte
//     reads) and are deduplicated in a per-warp shared-memory hash set that
//     is seeded with i and N(i);
//   * candidate rows are staged 64 dims at a time into shared memory with
//     cp.async (16-byte, xor-swizzled so the per-lane row reads are
//     conflict-free) and each lane computes one key in the reference's order;
//   * survivors are merged into the warp-held sorted list (bitonic via shuffles).
// "New" flags: a pair (a, j) is skipped when a was already in N(i) and j already
// in N(a) before the previous step.  Such a j was a candidate of i in that step
// and lost to k better entries (or is listed), and N(i) only improves, so it
// cannot enter now: the result is identical to evaluating every pair.
#include "knn_internal.cuh"
#include "knn_kernels.cuh"

namespace knn {

namespace {
constexpr int kPropMaxWarps = 8;
constexpr size_t kPropSmemBudget = 200 * 1024;
constexpr int kDCH = 64;  // dims staged per chunk (16 float4)

__device__ __forceinline__ bool hash_insert(int32_t* H, int hbits, int32_t id) {
  const uint32_t size = 1u << hbits;
  uint32_t slot = ((uint32_t)id * 2654435761u) >> (32 - hbits);
  for (uint32_t probe = 0; probe < size; ++probe) {
    const int32_t prev = atomicCAS(&H[slot], -1, id);
    if (prev == -1) return true;
    if (prev == id) return false;
    slot = (slot + 1) & (size - 1);
  }
  return false;  // unreachable: the table holds twice the most insertions
}

__device__ __forceinline__ void cp_async16(void* smem, const void* gmem, int src_bytes) {
  const uint32_t s = (uint32_t)__cvta_generic_to_shared(smem);
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;\n" ::"r"(s), "l"(gmem), "r"(src_bytes));
}
__device__ __forceinline__ void cp_async_wait_all() {
  asm volatile("cp.async.commit_group;\n" ::);
  asm volatile("cp.async.wait_group 0;\n" ::);
}

}  // namespace

int prop_hash_bits(int k) {
  const int need = 2 * (k * k + k + 1);
  int b = 5;
  while ((1 << b) < need) ++b;
  return b;
}

size_t prop_warp_bytes(int k, int dpad) {
  const size_t h = (size_t)4 << prop_hash_bits(k);
  const size_t q = 64 * 4;
  const size_t xq = (size_t)dpad * 4;
  const size_t rows = 32 * kDCH * 4;
  size_t b = h + q + xq + rows;
  return (b + 15) & ~(size_t)15;
}

template <int METRIC, int KPL>
__global__ void __launch_bounds__(kPropMaxWarps * 32) k_propagate(
    const float* __restrict__ X, int64_t n, int64_t r0, int64_t cnt, int d, int dpad, int k, int kw, int hbits,
    size_t warp_bytes, const float* __restrict__ norms, const int32_t* __restrict__ order,
    const float* __restrict__ key_in, const uint32_t* __restrict__ id_in,
    const uint32_t* __restrict__ flags_in, float* __restrict__ key_out,
    uint32_t* __restrict__ id_out, uint32_t* __restrict__ flags_out,
    unsigned long long* __restrict__ cand_counter) {
  extern __shared__ __align__(16) unsigned char smem[];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  unsigned char* base = smem + (size_t)warp * warp_bytes;
  const int hsize = 1 << hbits;
  int32_t* H = reinterpret_cast<int32_t*>(base);
  uint32_t* Q = reinterpret_cast<uint32_t*>(base + (size_t)4 * hsize);
  float* xq = reinterpret_cast<float*>(base + (size_t)4 * hsize + 256);
  float* rows = xq + dpad;
  const float kInf = __int_as_float(0x7F800000);
  const uint32_t lt_mask = (1u << lane) - 1u;
  unsigned long long evaluated = 0;

  const int wpb = blockDim.x >> 5;
  const int64_t nwarps = (int64_t)gridDim.x * wpb;
  // points (or order positions) r0 .. r0 + cnt - 1
  for (int64_t w = (int64_t)blockIdx.x * wpb + warp; w < cnt; w += nwarps) {
    const int32_t i = order ? order[r0 + w] : (int32_t)(r0 + w);
    WarpList<KPL> L;
    uint32_t oid[KPL];
    bool oflag[KPL];
#pragma unroll
    for (int r = 0; r < KPL; ++r) {
      const int e = r * 32 + lane;
      if (e < k) {
        L.key[r] = key_in[(size_t)i * k + e];
        // an id outside [0, n) is an empty entry: kept out of the list and
        // never followed
        const uint32_t u = id_in[(size_t)i * k + e] & kIdMask;
        const bool ok = u < (uint64_t)n;
        L.key[r] = ok ? L.key[r] : kInf;
        L.id[r] = ok ? u : kNoId;
        oid[r] = ok ? u : kNoId;
        oflag[r] = flags_in ? ((flags_in[(size_t)i * kw + r] >> lane) & 1u) : true;
      } else {
        L.key[r] = kInf;
        L.id[r] = kNoId;
        oid[r] = kNoId;
        oflag[r] = false;
      }
    }
    for (int s = lane; s < hsize; s += 32) H[s] = -1;
    const float4* xr = reinterpret_cast<const float4*>(X + (size_t)i * dpad);
    for (int c = lane; c < (dpad >> 2); c += 32) reinterpret_cast<float4*>(xq)[c] = __ldg(xr + c);
    __syncwarp();
    if (lane == 0) hash_insert(H, hbits, i);
#pragma unroll
    for (int r = 0; r < KPL; ++r)
      if (r * 32 + lane < k && oid[r] != kNoId) hash_insert(H, hbits, (int32_t)oid[r]);
    __syncwarp();
    const float ni = (METRIC == KNN_METRIC_COSINE) ? norms[i] : 0.f;

    int qn = 0;
    auto process = [&](int m) {
      // keys of the m queued candidates, one per lane
      const int32_t cj = lane < m ? (int32_t)Q[lane] : 0;
      float total = 0.f, part = 0.f;
      for (int cd = 0; cd < d; cd += kDCH) {
        // stage rows: 16 float4 per row, 2 rows per warp step
        const int half = lane >> 4, c4 = lane & 15;
        const int dim = cd + 4 * c4;
        for (int r = half; r < m; r += 2) {
          const int32_t jid = (int32_t)Q[r];
          const float* src = X + (size_t)jid * dpad + (dim < dpad ? dim : 0);
          float* dst = rows + r * kDCH + ((c4 ^ (r & 7)) << 2);
          cp_async16(dst, src, dim < dpad ? 16 : 0);
        }
        cp_async_wait_all();
        __syncwarp();
        if (lane < m) {
          const float* myrow = rows + lane * kDCH;
          const int lim = min(kDCH, d - cd);
          for (int q4 = 0; q4 < (lim + 3) >> 2; ++q4) {
            const float4 cv = *reinterpret_cast<const float4*>(myrow + ((q4 ^ (lane & 7)) << 2));
            const float4 qv = *reinterpret_cast<const float4*>(xq + cd + 4 * q4);
            part = acc_step<METRIC>(qv.x, cv.x, part);
            part = acc_step<METRIC>(qv.y, cv.y, part);
            part = acc_step<METRIC>(qv.z, cv.z, part);
            part = acc_step<METRIC>(qv.w, cv.w, part);
          }
          if (((cd + kDCH) & 255) == 0 || cd + kDCH >= d) {
            total = __fadd_rn(total, part);
            part = 0.f;
          }
        }
        __syncwarp();
      }
      float key = total;
      if (METRIC == KNN_METRIC_COSINE) key = lane < m ? cosine_key(total, ni, norms[cj]) : kInf;
      float tk;
      uint32_t ti;
      warp_list_get(L, k - 1, tk, ti);
      const bool pass = lane < m && cand_less(key, (uint32_t)cj, tk, ti);
      if (lane == 0) evaluated += (unsigned long long)m;
      if (__any_sync(0xFFFFFFFFu, pass))
        warp_list_insert(L, pass ? key : kInf, pass ? ((uint32_t)cj | 0x80000000u) : kNoId);
    };

    for (int s = 0; s < k; ++s) {
      // entry s of the old list and its flag, broadcast
      const int rr = s >> 5, src = s & 31;
      uint32_t av = 0;
      int fv = 0;
#pragma unroll
      for (int r = 0; r < KPL; ++r)
        if (r == rr) {
          av = oid[r];
          fv = oflag[r] ? 1 : 0;
        }
      const uint32_t a = __shfl_sync(0xFFFFFFFFu, av, src);
      const bool af = __shfl_sync(0xFFFFFFFFu, fv, src) != 0;
      if (a == kNoId) continue;  // warp-uniform
      for (int r0 = 0; r0 < k; r0 += 32) {
        const int e = r0 + lane;
        bool cand = false;
        int32_t jj = 0;
        if (e < k) {
          jj = (int32_t)(id_in[(size_t)a * k + e] & kIdMask);
          const bool jf = flags_in ? ((flags_in[(size_t)a * kw + (r0 >> 5)] >> lane) & 1u) : true;
          cand = (af || jf) && (int64_t)jj < n && hash_insert(H, hbits, jj);
        }
        const uint32_t bal = __ballot_sync(0xFFFFFFFFu, cand);
        if (cand) Q[qn + __popc(bal & lt_mask)] = (uint32_t)jj;
        qn += __popc(bal);
        __syncwarp();
        if (qn >= 32) {
          process(32);
          const uint32_t carry = lane < qn - 32 ? Q[32 + lane] : 0;
          __syncwarp();
          if (lane < qn - 32) Q[lane] = carry;
          qn -= 32;
          __syncwarp();
        }
      }
    }
    if (qn > 0) process(qn);

#pragma unroll
    for (int r = 0; r < KPL; ++r) {
      const int e = r * 32 + lane;
      if (e < k) {
        key_out[(size_t)i * k + e] = L.key[r];
        id_out[(size_t)i * k + e] = L.id[r] & kIdMask;
      }
      const uint32_t fl = __ballot_sync(0xFFFFFFFFu, e < k && (L.id[r] >> 31));
      if (lane == 0 && r < kw) flags_out[(size_t)i * kw + r] = fl;
    }
    __syncwarp();
  }
  if (cand_counter && lane == 0 && evaluated) atomicAdd(cand_counter, evaluated);
}

template <int METRIC>
static void launch_prop_metric(const PropArgs& a, int kpl, int hbits, size_t wb, int wpb,
                               unsigned grid) {
  const int kw = (a.k + 31) / 32;
  const int64_t r0 = a.r0, cnt = (a.r1 > 0 ? a.r1 : a.n) - a.r0;
  const size_t smem = wb * wpb;
#define KNN_PROP_LAUNCH(KP)                                                                       \
  do {                                                                                            \
    cudaFuncSetAttribute(k_propagate<METRIC, KP>, cudaFuncAttributeMaxDynamicSharedMemorySize,    \
                         (int)kPropSmemBudget);                                                   \
    k_propagate<METRIC, KP><<<grid, wpb * 32, smem, a.stream>>>(                                  \
        a.X, a.n, r0, cnt, a.d, a.dpad, a.k, kw, hbits, wb, a.norms, a.order, a.key_in, a.id_in,  \
        a.flags_in, a.key_out, a.id_out, a.flags_out, a.cand_counter);                            \
  } while (0)
  if (kpl == 1) KNN_PROP_LAUNCH(1);
  else if (kpl == 2) KNN_PROP_LAUNCH(2);
  else KNN_PROP_LAUNCH(4);
#undef KNN_PROP_LAUNCH
}

int propagate_step(const PropArgs& a, LaunchLog& log) {
  const int kpl = kpl_for(a.k);
  const int hbits = prop_hash_bits(a.k);
  const size_t wb = prop_warp_bytes(a.k, a.dpad);
  int wpb = (int)(kPropSmemBudget / wb);
  if (wpb > kPropMaxWarps) wpb = kPropMaxWarps;
  if (wpb < 1) return KNN_ERR_UNSUPPORTED;
  if (a.warps > 0 && a.warps < wpb) wpb = a.warps;  // a tuned block size (results identical)
  int dev = 0, sms = 148;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  int per_sm = (int)((220 * 1024) / (wb * wpb));
  if (per_sm < 1) per_sm = 1;
  const int64_t cnt = (a.r1 > 0 ? a.r1 : a.n) - a.r0;
  if (cnt <= 0) return KNN_OK;
  const int64_t want = (cnt + wpb - 1) / wpb;
  const int64_t cap = (int64_t)sms * per_sm;
  const unsigned grid = (unsigned)(want < cap ? want : cap);
  if (a.metric == KNN_METRIC_EUCLIDEAN) launch_prop_metric<KNN_METRIC_EUCLIDEAN>(a, kpl, hbits, wb, wpb, grid);
  else if (a.metric == KNN_METRIC_TAXICAB) launch_prop_metric<KNN_METRIC_TAXICAB>(a, kpl, hbits, wb, wpb, grid);
  else launch_prop_metric<KNN_METRIC_COSINE>(a, kpl, hbits, wb, wpb, grid);
  log.add();
  return cudaPeekAtLastError() == cudaSuccess ? KNN_OK : KNN_ERR_CUDA;
}

}  // namespace knn
