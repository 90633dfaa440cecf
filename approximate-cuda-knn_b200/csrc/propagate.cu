// Neighbour propagation, one Jacobi step: N'(i) = k best of N(i) u N(N(i)) \ {i}.
//
// Replaces propagate{Euclidean,Taxicab,Cosine}Kernel and the host loop
// (euclideandistancematrixgpu.cu:1033-1935, :1937-1977).  The reference marks
// N(N(i)) in an N-byte bitmap per point, clears N(i) and i, scans the bitmap and
// histogram-selects; here one warp owns one point:
//   * the k x k neighbour-of-neighbour ids are read all at once (four loads in
//     flight per lane), deduplicated in a per-warp shared-memory hash set
//     seeded with i and N(i), and compacted into a candidate array;
//   * the candidates' rows are staged by cp.async in 256-byte row slices (32
//     rows per stage, padded pitch so the per-lane row reads are conflict-free
//     at compile-time offsets); FP16 inputs are gathered as FP16 (the
//     conversion to FP32 is exact, so the keys are unchanged);
//   * each lane computes one key in the reference's order and the batch's
//     survivors are merged into the warp-held sorted list (bitonic via shuffles).
// "New" flags: a pair (a, j) is skipped when a was already in N(i) and j already
// in N(a) before the previous step.  Such a j was a candidate of i in that step
// and lost to k better entries (or is listed), and N(i) only improves, so it
// cannot enter now: the result is identical to evaluating every pair.  The
// candidate set does not depend on the order of discovery, and the list keeps
// the k best of the set by (key, id), so the result does not either.
#include <cuda_fp16.h>

#include <type_traits>

#include "knn_internal.cuh"
#include "knn_kernels.cuh"

namespace knn {

namespace {
constexpr int kPropMaxWarps = 8;
constexpr size_t kPropSmemBudget = 200 * 1024;
constexpr int kSliceBytes = 256;  // bytes of one candidate row per stage (16 x 16 B)
constexpr int kRowStride = kSliceBytes + 16;  // padded row pitch of the staging buffer
constexpr int kGatherUnroll = 4;  // neighbour-list entries in flight per lane

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
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::); }
template <int N>
__device__ __forceinline__ void cp_async_wait() {
  asm volatile("cp.async.wait_group %0;\n" ::"n"(N) : "memory");
}

inline int round_up(int v, int m) { return (v + m - 1) / m * m; }

}  // namespace

int prop_hash_bits(int k) {
  const int need = 2 * (k * k + k + 1);
  int b = 5;
  while ((1 << b) < need) ++b;
  return b;
}

// hash set (with two buffers: also the second row-slice buffer, since the
// hash is done with before the first row is staged) | candidates [k*k] | N(i)
// ids and flags | query row (float, d rounded to 8) | the row-slice buffer
// (32 rows, padded pitch)
size_t prop_region0_bytes(int k, int nbuf) {
  const size_t h = (size_t)4 << prop_hash_bits(k);
  return nbuf == 2 ? std::max(h, (size_t)32 * kRowStride) : h;
}
size_t prop_warp_bytes(int k, int d, int nbuf) {
  size_t b = prop_region0_bytes(k, nbuf) + (size_t)4 * round_up(k * k, 32) + (size_t)8 * round_up(k, 32) +
             (size_t)4 * round_up(d, 8) + (size_t)32 * kRowStride;
  return (b + 15) & ~(size_t)15;
}

// HALF: rows are FP16 [n][ldr] (ldr % 8 == 0), else float32 [n][ldr] (ldr % 4 == 0);
// zero padded beyond d.  NBUF 2: the next stage's row slices load while the
// current stage is summed (used where the second buffer costs no warps per SM).
template <int METRIC, int KPL, bool HALF, int NBUF>
__global__ void __launch_bounds__(kPropMaxWarps * 32) k_propagate(
    const void* __restrict__ Xrows, int ldr, int64_t n, int64_t r0, int64_t cnt, int d, int k, int kw, int hbits,
    size_t warp_bytes, size_t region0, const float* __restrict__ norms, const int32_t* __restrict__ order,
    const float* __restrict__ key_in, const uint32_t* __restrict__ id_in,
    const uint32_t* __restrict__ flags_in, float* __restrict__ key_out,
    uint32_t* __restrict__ id_out, uint32_t* __restrict__ flags_out,
    unsigned long long* __restrict__ cand_counter) {
  using Elem = typename std::conditional<HALF, __half, float>::type;
  constexpr int kEPU = 16 / sizeof(Elem);            // elements per 16-byte unit
  constexpr int kCH = kSliceBytes / sizeof(Elem);    // dims per row slice (divides 256)
  extern __shared__ __align__(16) unsigned char smem[];
  const Elem* X = static_cast<const Elem*>(Xrows);
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  unsigned char* base = smem + (size_t)warp * warp_bytes;
  const int hsize = 1 << hbits;
  const int kk = k * k;
  const int kr = (k + 31) & ~31;
  const int dq = (d + 7) & ~7;
  int32_t* H = reinterpret_cast<int32_t*>(base);
  uint32_t* Q = reinterpret_cast<uint32_t*>(base + region0);
  uint32_t* nbid = Q + ((kk + 31) & ~31);
  uint32_t* nbfl = nbid + kr;
  float* xq = reinterpret_cast<float*>(nbfl + kr);
  unsigned char* rows1 = reinterpret_cast<unsigned char*>(xq + dq);  // [32][kRowStride]
  unsigned char* rows0 = NBUF == 2 ? base : rows1;                    // over the hash set
  const float kInf = __int_as_float(0x7F800000);
  const uint32_t lt_mask = (1u << lane) - 1u;
  const int nch = (d + kCH - 1) / kCH;
  unsigned long long evaluated = 0;

  const int wpb = blockDim.x >> 5;
  const int64_t nwarps = (int64_t)gridDim.x * wpb;
  // points (or order positions) r0 .. r0 + cnt - 1
  for (int64_t w = (int64_t)blockIdx.x * wpb + warp; w < cnt; w += nwarps) {
    const int32_t i = order ? order[r0 + w] : (int32_t)(r0 + w);
    WarpList<KPL> L;
#pragma unroll
    for (int r = 0; r < KPL; ++r) {
      const int e = r * 32 + lane;
      uint32_t nid = kNoId, nfl = 0;
      if (e < k) {
        L.key[r] = key_in[(size_t)i * k + e];
        // an id outside [0, n) is an empty entry: kept out of the list and
        // never followed
        const uint32_t u = id_in[(size_t)i * k + e] & kIdMask;
        const bool ok = u < (uint64_t)n;
        L.key[r] = ok ? L.key[r] : kInf;
        L.id[r] = ok ? u : kNoId;
        nid = ok ? u : kNoId;
        nfl = flags_in ? ((flags_in[(size_t)i * kw + r] >> lane) & 1u) : 1u;
      } else {
        L.key[r] = kInf;
        L.id[r] = kNoId;
      }
      if (e < kr) {
        nbid[e] = nid;
        nbfl[e] = nfl;
      }
    }
    for (int s = lane; s < hsize; s += 32) H[s] = -1;
    {
      const Elem* xr = X + (size_t)i * ldr;
      for (int c = lane; c < dq; c += 32) xq[c] = c < d ? (float)xr[c] : 0.f;
    }
    __syncwarp();
    if (lane == 0) hash_insert(H, hbits, i);
#pragma unroll
    for (int r = 0; r < KPL; ++r)
      if (r * 32 + lane < k && L.id[r] != kNoId) hash_insert(H, hbits, (int32_t)L.id[r]);
    __syncwarp();
    const float ni = (METRIC == KNN_METRIC_COSINE) ? norms[i] : 0.f;

    // candidates: entry (s, t) of the flattened k x k neighbour lists, lane-strided
    int qn = 0;
    for (int e0 = 0; e0 < kk; e0 += 32 * kGatherUnroll) {
      uint32_t jj[kGatherUnroll];
      bool ok[kGatherUnroll];
#pragma unroll
      for (int u = 0; u < kGatherUnroll; ++u) {
        const int e = e0 + u * 32 + lane;
        jj[u] = 0;
        ok[u] = false;
        if (e < kk) {
          const int s = e / k, t = e - s * k;
          const uint32_t a = nbid[s];
          if (a != kNoId) {
            jj[u] = id_in[(size_t)a * k + t] & kIdMask;
            const bool jf = flags_in ? ((flags_in[(size_t)a * kw + (t >> 5)] >> (t & 31)) & 1u) : true;
            ok[u] = (nbfl[s] != 0 || jf) && (int64_t)jj[u] < n;
          }
        }
      }
#pragma unroll
      for (int u = 0; u < kGatherUnroll; ++u) {
        const bool cand = ok[u] && hash_insert(H, hbits, (int32_t)jj[u]);
        const uint32_t bal = __ballot_sync(0xFFFFFFFFu, cand);
        if (cand) Q[qn + __popc(bal & lt_mask)] = jj[u];
        qn += __popc(bal);
      }
    }
    __syncwarp();

    // keys of the candidates, 32 per batch, one row slice of kSliceBytes per
    // stage; rows are kRowStride apart, so lane r's 16-byte loads of unit q
    // (address r * 272 + 16 q) fall in distinct bank groups within each
    // 8-lane phase and the unit offsets are compile-time constants
    const int stages = ((qn + 31) >> 5) * nch;
    const int half = lane >> 4, c16 = lane & 15;
    // stage t: rows 32 b .. of the candidates, dims c * kCH .. of each, into buffer t mod NBUF
    auto stage_rows = [&](int t) {
      const int b = t / nch, c = t - b * nch;
      const int m = min(32, qn - 32 * b);
      const int dim = c * kCH + kEPU * c16;
      const bool ok = dim < ldr;
      unsigned char* buf = (NBUF == 2 && (t & 1)) ? rows1 : rows0;
      for (int r = half; r < m; r += 2) {
        const uint32_t jid = Q[32 * b + r];
        cp_async16(buf + r * kRowStride + c16 * 16, X + (size_t)jid * ldr + (ok ? dim : 0), ok ? 16 : 0);
      }
      cp_async_commit();
    };
    float total = 0.f, part = 0.f;
    if (NBUF == 2 && stages > 0) stage_rows(0);
    for (int t = 0; t < stages; ++t) {
      const int b = t / nch, c = t - b * nch;
      const int m = min(32, qn - 32 * b);
      const int cd = c * kCH;
      if (NBUF == 2) {
        if (t + 1 < stages) {
          stage_rows(t + 1);  // its buffer was last read in stage t - 1, before that stage's closing syncwarp
          cp_async_wait<1>();
        } else {
          cp_async_wait<0>();
        }
      } else {
        stage_rows(t);
        cp_async_wait<0>();
      }
      __syncwarp();
      const unsigned char* rows = (NBUF == 2 && (t & 1)) ? rows1 : rows0;
      if (lane < m) {
        const unsigned char* myrow = rows + lane * kRowStride;
        const int nu = (min(kCH, d - cd) + kEPU - 1) / kEPU;  // 16-byte units holding dims
        const float* qx = xq + cd;
#pragma unroll
        for (int q = 0; q < kCH / kEPU; ++q) {
          if (q < nu) {
            const uint4 raw = *reinterpret_cast<const uint4*>(myrow + q * 16);
            if (HALF) {
              const __half2* h2 = reinterpret_cast<const __half2*>(&raw);
#pragma unroll
              for (int e = 0; e < 4; ++e) {
                const float2 cv = __half22float2(h2[e]);
                part = acc_step<METRIC>(qx[kEPU * q + 2 * e], cv.x, part);
                part = acc_step<METRIC>(qx[kEPU * q + 2 * e + 1], cv.y, part);
              }
            } else {
              const float4 cv = *reinterpret_cast<const float4*>(&raw);
              const float4 qv = *reinterpret_cast<const float4*>(qx + kEPU * q);
              part = acc_step<METRIC>(qv.x, cv.x, part);
              part = acc_step<METRIC>(qv.y, cv.y, part);
              part = acc_step<METRIC>(qv.z, cv.z, part);
              part = acc_step<METRIC>(qv.w, cv.w, part);
            }
          }
        }
        if (((cd + kCH) & 255) == 0 || cd + kCH >= d) {
          total = __fadd_rn(total, part);
          part = 0.f;
        }
      }
      __syncwarp();  // the buffer is refilled by the next stage
      if (c == nch - 1) {
        const int32_t cj = lane < m ? (int32_t)Q[32 * b + lane] : 0;
        float key = total;
        if (METRIC == KNN_METRIC_COSINE) key = lane < m ? cosine_key(total, ni, norms[cj]) : kInf;
        float tk;
        uint32_t ti;
        warp_list_get(L, k - 1, tk, ti);
        const bool pass = lane < m && cand_less(key, (uint32_t)cj, tk, ti);
        if (lane == 0) evaluated += (unsigned long long)m;
        if (__any_sync(0xFFFFFFFFu, pass))
          warp_list_insert(L, pass ? key : kInf, pass ? ((uint32_t)cj | 0x80000000u) : kNoId);
        total = 0.f;
        part = 0.f;
      }
    }

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

template <int METRIC, bool HALF, int NBUF>
static void launch_prop_metric(const PropArgs& a, int kpl, int hbits, size_t wb, int wpb, unsigned grid) {
  const int kw = (a.k + 31) / 32;
  const int64_t r0 = a.r0, cnt = (a.r1 > 0 ? a.r1 : a.n) - a.r0;
  const size_t smem = wb * wpb;
  const void* rows = HALF ? static_cast<const void*>(a.Xh) : static_cast<const void*>(a.X);
  const int ldr = HALF ? a.ldh : a.dpad;
  const size_t region0 = prop_region0_bytes(a.k, NBUF);
#define KNN_PROP_LAUNCH(KP)                                                                                \
  do {                                                                                                     \
    cudaFuncSetAttribute(k_propagate<METRIC, KP, HALF, NBUF>, cudaFuncAttributeMaxDynamicSharedMemorySize, \
                         (int)kPropSmemBudget);                                                            \
    k_propagate<METRIC, KP, HALF, NBUF><<<grid, wpb * 32, smem, a.stream>>>(                               \
        rows, ldr, a.n, r0, cnt, a.d, a.k, kw, hbits, wb, region0, a.norms, a.order, a.key_in, a.id_in,    \
        a.flags_in, a.key_out, a.id_out, a.flags_out, a.cand_counter);                                     \
  } while (0)
  if (kpl == 1) KNN_PROP_LAUNCH(1);
  else if (kpl == 2) KNN_PROP_LAUNCH(2);
  else KNN_PROP_LAUNCH(4);
#undef KNN_PROP_LAUNCH
}

template <int METRIC>
static void launch_prop_rows(const PropArgs& a, int kpl, int hbits, size_t wb, int wpb, unsigned grid, int nbuf) {
  if (nbuf == 2) {
    if (a.Xh) launch_prop_metric<METRIC, true, 2>(a, kpl, hbits, wb, wpb, grid);
    else launch_prop_metric<METRIC, false, 2>(a, kpl, hbits, wb, wpb, grid);
  } else {
    if (a.Xh) launch_prop_metric<METRIC, true, 1>(a, kpl, hbits, wb, wpb, grid);
    else launch_prop_metric<METRIC, false, 1>(a, kpl, hbits, wb, wpb, grid);
  }
}

int propagate_step(const PropArgs& a, LaunchLog& log) {
  const int kpl = kpl_for(a.k);
  const int hbits = prop_hash_bits(a.k);
  size_t wb = prop_warp_bytes(a.k, a.d, 1);
  int wpb = (int)(kPropSmemBudget / wb);
  if (wpb > kPropMaxWarps) wpb = kPropMaxWarps;
  if (wpb < 1) return KNN_ERR_UNSUPPORTED;
  if (a.warps > 0 && a.warps < wpb) wpb = a.warps;  // a tuned block size (results identical)
  int dev = 0, sms = 148;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  int per_sm = (int)((220 * 1024) / (wb * wpb));
  if (per_sm < 1) per_sm = 1;
  // a second row-slice buffer where it leaves the warps per SM as they are
  // (the results do not depend on it)
  int nbuf = 1;
  const size_t wb2 = prop_warp_bytes(a.k, a.d, 2);
  if (wb2 * wpb <= kPropSmemBudget && (int)((220 * 1024) / (wb2 * wpb)) >= per_sm) {
    nbuf = 2;
    wb = wb2;
  }
  const int64_t cnt = (a.r1 > 0 ? a.r1 : a.n) - a.r0;
  if (cnt <= 0) return KNN_OK;
  const int64_t want = (cnt + wpb - 1) / wpb;
  const int64_t cap = (int64_t)sms * per_sm;
  const unsigned grid = (unsigned)(want < cap ? want : cap);
  if (a.metric == KNN_METRIC_EUCLIDEAN) launch_prop_rows<KNN_METRIC_EUCLIDEAN>(a, kpl, hbits, wb, wpb, grid, nbuf);
  else if (a.metric == KNN_METRIC_TAXICAB) launch_prop_rows<KNN_METRIC_TAXICAB>(a, kpl, hbits, wb, wpb, grid, nbuf);
  else launch_prop_rows<KNN_METRIC_COSINE>(a, kpl, hbits, wb, wpb, grid, nbuf);
  log.add();
  return cudaPeekAtLastError() == cudaSuccess ? KNN_OK : KNN_ERR_CUDA;
}

}  // namespace knn
