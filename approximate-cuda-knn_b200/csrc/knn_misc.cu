// Small element-wise kernels around the k-NN stages.
#include <cuda_bf16.h>
#include <cuda_fp16.h>

#include "knn_internal.cuh"
#include "knn_kernels.cuh"

namespace knn {

// Every list slot empty (+inf, no id), every flag "new".  Plays the role of
// stubInitializationKernel (euclideandistancematrixgpu.cu:2110-2117), whose
// stub is (id -1, distance 100000).
__global__ void k_init_lists(float* key, uint32_t* id, int64_t count) {
  const int64_t g = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (g < count) {
    key[g] = __int_as_float(0x7F800000);
    id[g] = kNoId;
  }
}

__global__ void k_set_flags(uint32_t* flags, int64_t n, int k, int kw) {
  const int64_t g = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (g < n * kw) {
    const int w = (int)(g % kw);
    const int bits = min(32, k - 32 * w);
    flags[g] = bits >= 32 ? 0xFFFFFFFFu : ((1u << bits) - 1u);
  }
}

// |x| in the reference's summation order (used for 1 - cos).
__global__ void k_norms(const float* __restrict__ X, int64_t n, int d, int dpad, float* __restrict__ norms) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) norms[i] = __fsqrt_rn(self_dot_chunked(X + (size_t)i * dpad, d));
}

// Rows of any input element type -> zero-padded float32 rows of dpad floats.
template <typename T>
__device__ __forceinline__ float to_f32(T v);
template <>
__device__ __forceinline__ float to_f32<float>(float v) { return v; }
template <>
__device__ __forceinline__ float to_f32<__half>(__half v) { return __half2float(v); }
template <>
__device__ __forceinline__ float to_f32<__nv_bfloat16>(__nv_bfloat16 v) { return __bfloat162float(v); }

template <typename T>
__global__ void k_pad_rows(const T* __restrict__ src, int64_t n, int d, int64_t ld,
                           float* __restrict__ dst, int dpad) {
  const int64_t g = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (g >= n * dpad) return;
  const int64_t i = g / dpad;
  const int c = (int)(g - i * dpad);
  dst[g] = c < d ? to_f32<T>(src[i * ld + c]) : 0.0f;
}

// FP16 rows [n][ld] -> [n][dh] (dh % 8 == 0), zero padded.
__global__ void k_pad_rows_f16(const __half* __restrict__ src, int64_t n, int d, int64_t ld,
                               __half* __restrict__ dst, int dh) {
  const int64_t g = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (g >= n * dh) return;
  const int64_t i = g / dh;
  const int c = (int)(g - i * dh);
  dst[g] = c < d ? src[i * ld + c] : __float2half_rn(0.0f);
}

// Rows of many device point sets into one padded float32 array: block (x, y)
// copies rows y, y + gridDim.y, ... of set x.
template <typename T>
__global__ void k_gather_sets(const RowSource* __restrict__ sets, int d, float* __restrict__ dst, int dpad) {
  const RowSource s = sets[blockIdx.x];
  const T* src = static_cast<const T*>(s.src);
  for (int64_t i = blockIdx.y; i < s.n; i += gridDim.y) {
    float* out = dst + (size_t)(s.off + i) * dpad;
    for (int c = threadIdx.x; c < dpad; c += blockDim.x) out[c] = c < d ? to_f32<T>(src[i * d + c]) : 0.0f;
  }
}

__global__ void k_finalize(const float* __restrict__ key, const uint32_t* __restrict__ id,
                           int64_t count, int metric, float* __restrict__ dist,
                           int32_t* __restrict__ idx) {
  const int64_t g = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (g < count) {
    const float kv = key[g];
    dist[g] = metric == KNN_METRIC_EUCLIDEAN ? __fsqrt_rn(kv) : kv;
    idx[g] = (int32_t)(id[g] & kIdMask);
  }
}

// Batches: ids become local to their segment (the point's own), as above.
__global__ void k_finalize_local(const float* __restrict__ key, const uint32_t* __restrict__ id,
                                 int64_t ntot, int k, int metric, const int32_t* __restrict__ seg_of,
                                 const SegEntry* __restrict__ segs, float* __restrict__ dist,
                                 int32_t* __restrict__ idx) {
  const int64_t g = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (g < ntot * k) {
    const int64_t off = segs[seg_of[g / k]].off;
    const float kv = key[g];
    dist[g] = metric == KNN_METRIC_EUCLIDEAN ? __fsqrt_rn(kv) : kv;
    idx[g] = (int32_t)((int64_t)(id[g] & kIdMask) - off);
  }
}

// Warp per point: the k best distinct ids by (key, id) over `lists` sorted
// candidate lists [lists][n][k] (id < 0: empty).  A list holds an id once, so
// an id met again comes from another list and is dropped.
template <int KPL>
__global__ void k_merge_lists(const int32_t* __restrict__ idx, const float* __restrict__ key, int lists, int64_t n,
                              int k, int32_t* __restrict__ idx_out, float* __restrict__ key_out) {
  const int lane = threadIdx.x & 31;
  const int64_t w0 = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int64_t nw = ((int64_t)gridDim.x * blockDim.x) >> 5;
  const float kInf = __int_as_float(0x7F800000);
  for (int64_t i = w0; i < n; i += nw) {
    WarpList<KPL> L;
#pragma unroll
    for (int r = 0; r < KPL; ++r) {
      L.key[r] = kInf;
      L.id[r] = kNoId;
    }
    for (int l = 0; l < lists; ++l) {
      const size_t row = ((size_t)l * n + i) * k;
      for (int c0 = 0; c0 < k; c0 += 32) {
        const int e = c0 + lane;
        const int32_t id = e < k ? idx[row + e] : -1;
        const float ck = id >= 0 ? key[row + e] : kInf;
        const uint32_t ci = id >= 0 ? (uint32_t)id : kNoId;
        float tk;
        uint32_t ti;
        warp_list_get(L, k - 1, tk, ti);
        bool pass = id >= 0 && cand_less(ck, ci, tk, ti);
        if (!__any_sync(0xFFFFFFFFu, pass)) continue;
        // every lane takes part in the id check's shuffles
        const bool dup = warp_list_contains(L, ci, k);
        pass = pass && !dup;
        if (!__any_sync(0xFFFFFFFFu, pass)) continue;
        warp_list_insert(L, pass ? ck : kInf, pass ? ci : kNoId);
      }
    }
#pragma unroll
    for (int r = 0; r < KPL; ++r) {
      const int e = r * 32 + lane;
      if (e < k) {
        idx_out[(size_t)i * k + e] = L.id[r] == kNoId ? -1 : (int32_t)(L.id[r] & kIdMask);
        key_out[(size_t)i * k + e] = L.key[r];
      }
    }
  }
}

// seg_of[i] = segment of global position i; block per segment.
__global__ void k_fill_seg_of(const SegEntry* __restrict__ segs, int32_t* __restrict__ seg_of) {
  const SegEntry e = segs[blockIdx.x];
  for (int64_t i = threadIdx.x; i < e.n; i += blockDim.x) seg_of[e.off + i] = (int32_t)blockIdx.x;
}

__global__ void k_keys_from_dist(const float* __restrict__ dist, int64_t count, int metric,
                                 float* __restrict__ key) {
  const int64_t g = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (g < count) {
    const float v = dist[g];
    key[g] = metric == KNN_METRIC_EUCLIDEAN ? __fmul_rn(v, v) : v;
  }
}

static inline unsigned blocks_for(int64_t count, int threads) {
  return (unsigned)((count + threads - 1) / threads);
}

void launch_init_lists(float* key, uint32_t* id, uint32_t* flags, int64_t n, int k, int kw,
                       cudaStream_t st) {
  k_init_lists<<<blocks_for(n * k, 256), 256, 0, st>>>(key, id, n * k);
  if (flags) k_set_flags<<<blocks_for(n * kw, 256), 256, 0, st>>>(flags, n, k, kw);
}
void launch_set_flags(uint32_t* flags, int64_t n, int k, int kw, cudaStream_t st) {
  k_set_flags<<<blocks_for(n * kw, 256), 256, 0, st>>>(flags, n, k, kw);
}
void launch_norms(const float* X, int64_t n, int d, int dpad, float* norms, cudaStream_t st) {
  k_norms<<<blocks_for(n, 128), 128, 0, st>>>(X, n, d, dpad, norms);
}
void launch_pad_rows(const void* src, int dtype, int64_t n, int d, int64_t ld, float* dst,
                     int dpad, cudaStream_t st) {
  const unsigned b = blocks_for(n * dpad, 256);
  if (dtype == KNN_F16)
    k_pad_rows<__half><<<b, 256, 0, st>>>(static_cast<const __half*>(src), n, d, ld, dst, dpad);
  else if (dtype == KNN_BF16)
    k_pad_rows<__nv_bfloat16><<<b, 256, 0, st>>>(static_cast<const __nv_bfloat16*>(src), n, d, ld, dst, dpad);
  else
    k_pad_rows<float><<<b, 256, 0, st>>>(static_cast<const float*>(src), n, d, ld, dst, dpad);
}
void launch_pad_rows_f16(const void* src, int64_t n, int d, int64_t ld, void* dst, int dh, cudaStream_t st) {
  k_pad_rows_f16<<<blocks_for(n * dh, 256), 256, 0, st>>>(static_cast<const __half*>(src), n, d, ld,
                                                           static_cast<__half*>(dst), dh);
}
void launch_finalize(const float* key, const uint32_t* id, int64_t n, int k, int metric,
                     float* out_dist, int32_t* out_idx, cudaStream_t st) {
  k_finalize<<<blocks_for(n * k, 256), 256, 0, st>>>(key, id, n * k, metric, out_dist, out_idx);
}
void launch_finalize_local(const float* key, const uint32_t* id, int64_t ntot, int k, int metric,
                           const int32_t* seg_of, const SegEntry* segs, float* out_dist, int32_t* out_idx,
                           cudaStream_t st) {
  k_finalize_local<<<blocks_for(ntot * k, 256), 256, 0, st>>>(key, id, ntot, k, metric, seg_of, segs, out_dist,
                                                               out_idx);
}
void launch_gather_sets(const RowSource* sets, int count, int dtype, int d, float* dst, int dpad,
                        cudaStream_t st) {
  dim3 grid((unsigned)count, 128);
  const int threads = dpad >= 128 ? 128 : 64;
  if (dtype == KNN_F16) k_gather_sets<__half><<<grid, threads, 0, st>>>(sets, d, dst, dpad);
  else if (dtype == KNN_BF16) k_gather_sets<__nv_bfloat16><<<grid, threads, 0, st>>>(sets, d, dst, dpad);
  else k_gather_sets<float><<<grid, threads, 0, st>>>(sets, d, dst, dpad);
}
void launch_merge_lists(const int32_t* idx, const float* key, int lists, int64_t n, int k, int32_t* idx_out,
                        float* key_out, cudaStream_t st) {
  const unsigned grid = blocks_for(n * 32, 256);
  const int kpl = kpl_for(k);
  if (kpl == 1) k_merge_lists<1><<<grid, 256, 0, st>>>(idx, key, lists, n, k, idx_out, key_out);
  else if (kpl == 2) k_merge_lists<2><<<grid, 256, 0, st>>>(idx, key, lists, n, k, idx_out, key_out);
  else k_merge_lists<4><<<grid, 256, 0, st>>>(idx, key, lists, n, k, idx_out, key_out);
}
void launch_fill_seg_of(const SegEntry* segs, int count, int32_t* seg_of, cudaStream_t st) {
  k_fill_seg_of<<<(unsigned)count, 256, 0, st>>>(segs, seg_of);
}
void launch_keys_from_dist(const float* dist, int64_t count, int metric, float* key,
                           cudaStream_t st) {
  k_keys_from_dist<<<blocks_for(count, 256), 256, 0, st>>>(dist, count, metric, key);
}

// ------------------------------------------- reference normalisation (CLI) --
// Step 1 (normalizeDataStep1, euclideandistancematrixgpu.cu:19-42): one thread
// per dimension sums the column sequentially in float, divides by n and
// subtracts.  Row-major here, so the column walk is strided.
__global__ void k_norm_step1(float* X, int64_t n, int d) {
  const int dim = blockIdx.x * blockDim.x + threadIdx.x;
  if (dim >= d) return;
  float mean = 0.0f;
  for (int64_t i = 0; i < n; ++i) mean = __fadd_rn(mean, X[i * d + dim]);
  mean = __fdiv_rn(mean, (float)n);
  for (int64_t i = 0; i < n; ++i) X[i * d + dim] = __fsub_rn(X[i * d + dim], mean);
}
// Step 2 (normalizeDataStep2, .cu:44-85): a single 256-thread block; thread t
// covers dimension t only (the reference's `if` is not a loop), takes the
// largest |x| of its dimension, thread 0 takes the largest over the 256
// slots, and dimensions < 256 are divided by it.
__global__ void k_norm_step2(float* X, int64_t n, int d) {
  __shared__ float mx[256];
  __shared__ float mglobal;
  const int t = threadIdx.x;
  mx[t] = 0.0f;
  if (t == 0) mglobal = 0.0f;
  __syncthreads();
  if (t < d) {
    float m = 0.0f;
    for (int64_t i = 0; i < n; ++i) m = fmaxf(fabsf(X[i * d + t]), m);
    mx[t] = m;
  }
  __syncthreads();
  if (t == 0) {
    float g = 0.0f;
    for (int q = 0; q < 256; ++q) g = fmaxf(g, mx[q]);
    mglobal = g;
  }
  __syncthreads();
  if (t < d) {
    const float g = mglobal;
    for (int64_t i = 0; i < n; ++i) X[i * d + t] = __fdiv_rn(X[i * d + t], g);
  }
}
void launch_normalize_reference(float* X, int64_t n, int d, cudaStream_t st) {
  k_norm_step1<<<(d + 255) / 256, 256, 0, st>>>(X, n, d);
  k_norm_step2<<<1, 256, 0, st>>>(X, n, d);
}

}  // namespace knn
