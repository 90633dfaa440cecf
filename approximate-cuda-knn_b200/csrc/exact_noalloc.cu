// Allocation-free variant of the FP64 exact k-NN (knn_exact_fp64_noalloc).
//
// Some callers cannot allocate device memory once they are running: a serving
// process whose whole device memory is handed to its own pool at start-up, or
// a latency-critical thread that must not pay the device-wide synchronisation
// that cudaMalloc/cudaFree can imply.  For them this entry point works from
// caller-owned inputs and outputs plus one fixed scratch area compiled into the
// library: a file-scope __device__ array of kNoAllocScratchBytes (16 MiB) that
// every GPU loading the library keeps until the process exits.
//
// Rules of use:
//   * all pointers are device pointers; the call runs on `stream` and returns
//     after that stream has finished the work (it reads back one status word);
//   * the first call on a device looks up the array's device address with
//     cudaGetSymbolAddress (once per device, with that device current), so make
//     that first call before any stream capture begins;
//   * with CUDA's lazy module loading (the default) the array itself is
//     reserved on a device only when this code first runs there, so a caller
//     that hands its device memory to a pool at start-up makes one warm-up call
//     on each device before that; if the reservation fails the call returns
//     KNN_ERR_OOM with a message saying so;
//   * every call shares the one array and leaves its contents behind: calls
//     that overlap on the GPU (two streams, two host threads) race on it;
//   * requests whose scratch would not fit are rejected with KNN_ERR_ARGS.
// Nothing here calls cudaMalloc, cudaFree or any allocating library routine.
#include <mutex>
#include <string>

#include "knn_internal.cuh"
#include "knn_kernels.cuh"

namespace knn {
int exact_fp64(const float* X, int64_t n, int d, int dpad, int k, int metric,
               const int64_t* queries, int64_t nq, double* norms, double* part_dist,
               uint32_t* part_idx, int slices, double* out_dist, int32_t* out_idx,
               cudaStream_t st);
void set_last_error(const std::string& what);
}  // namespace knn

namespace {

constexpr size_t kNoAllocScratchBytes = size_t(16) << 20;
constexpr int kMaxDevices = 64;

// The scratch.  In host code `g_noalloc_scratch` is only a stand-in symbol, not
// a device address; kernels get the address looked up below.
__device__ __align__(256) unsigned char g_noalloc_scratch[kNoAllocScratchBytes];

std::mutex g_setup_mutex;
unsigned char* g_scratch_addr[kMaxDevices] = {};

inline size_t align256(size_t b) { return (b + 255) & ~size_t(255); }

// Copies the query ids into the scratch, replacing any id outside [0, n) by 0
// and raising the status word, so the exact kernels never read out of bounds.
__global__ void k_sanitize_queries(const int64_t* __restrict__ q, int64_t nq, int64_t n,
                                   int64_t* __restrict__ out, int* __restrict__ status) {
  const int64_t g = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (g >= nq) return;
  const int64_t v = q[g];
  const bool ok = v >= 0 && v < n;
  out[g] = ok ? v : 0;
  if (!ok) atomicExch(status, 1);
}

int fail(int code, const std::string& msg) {
  knn::set_last_error(msg);
  return code;
}

int scratch_for_device(unsigned char** out) {
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return fail(KNN_ERR_NO_DEVICE, std::string("cudaGetDevice: ") + cudaGetErrorString(e));
  if (dev < 0 || dev >= kMaxDevices) return fail(KNN_ERR_UNSUPPORTED, "device ordinal too large");
  std::lock_guard<std::mutex> lock(g_setup_mutex);
  if (!g_scratch_addr[dev]) {
    void* p = nullptr;
    e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (e == cudaErrorMemoryAllocation) {
      cudaGetLastError();
      return fail(KNN_ERR_OOM,
                  "the 16 MiB scratch of knn_exact_fp64_noalloc could not be reserved on this device; make a "
                  "first call on each device before device memory is handed to a pool");
    }
    if (e != cudaSuccess || !p)
      return fail(KNN_ERR_CUDA, std::string("cudaGetSymbolAddress: ") + cudaGetErrorString(e));
    g_scratch_addr[dev] = static_cast<unsigned char*>(p);
  }
  *out = g_scratch_addr[dev];
  return KNN_OK;
}

}  // namespace

extern "C" int knn_exact_fp64_noalloc(const float* points, int64_t n, int32_t d, int32_t k,
                                      int32_t metric, const int64_t* queries, int64_t nq,
                                      int32_t* out_idx, double* out_dist, void* stream) {
  if (!points || !queries || !out_idx || !out_dist) return fail(KNN_ERR_ARGS, "NULL pointer");
  if (n < 1 || n >= (int64_t)INT32_MAX || d < 1 || k < 1 || k > KNN_MAX_K || nq < 1)
    return fail(KNN_ERR_ARGS, "size out of range");
  if (metric < 0 || metric > 2) return fail(KNN_ERR_ARGS, "unknown metric");
  if (n <= k) return fail(KNN_ERR_N_LE_K, "n must exceed k");

  // scratch layout: status | sanitized queries | row norms (COSINE) | per-slice lists
  const size_t b_status = 256;
  const size_t b_queries = align256((size_t)nq * sizeof(int64_t));
  const size_t b_norms = metric == KNN_METRIC_COSINE ? align256((size_t)n * sizeof(double)) : 0;
  const size_t per_slice = align256((size_t)nq * k * sizeof(double)) + align256((size_t)nq * k * sizeof(uint32_t));
  const size_t fixed = b_status + b_queries + b_norms;
  if (fixed + per_slice > kNoAllocScratchBytes)
    return fail(KNN_ERR_ARGS, "request needs " + std::to_string(fixed + per_slice) +
                                  " bytes of scratch; knn_exact_fp64_noalloc holds " +
                                  std::to_string(kNoAllocScratchBytes));
  unsigned char* base = nullptr;
  int rc = scratch_for_device(&base);
  if (rc) return rc;

  int dev = 0, sms = 148;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  const int64_t qtiles = (nq + 63) / 64;
  int64_t slices = (4LL * sms + qtiles - 1) / qtiles;
  if (slices > 64) slices = 64;
  if (slices > (n + 63) / 64) slices = (n + 63) / 64;
  const int64_t fit = (int64_t)((kNoAllocScratchBytes - fixed) / per_slice);
  if (slices > fit) slices = fit;
  if (slices < 1) slices = 1;

  int* status = reinterpret_cast<int*>(base);
  int64_t* q = reinterpret_cast<int64_t*>(base + b_status);
  double* norms = reinterpret_cast<double*>(base + b_status + b_queries);
  unsigned char* lists = base + fixed;
  double* part_dist = reinterpret_cast<double*>(lists);
  uint32_t* part_idx = reinterpret_cast<uint32_t*>(lists + align256((size_t)slices * nq * k * sizeof(double)));

  cudaStream_t st = static_cast<cudaStream_t>(stream);
  cudaError_t e = cudaMemsetAsync(status, 0, sizeof(int), st);  // the one word that must start at 0
  if (e != cudaSuccess) return fail(KNN_ERR_CUDA, std::string("cudaMemsetAsync: ") + cudaGetErrorString(e));
  k_sanitize_queries<<<(unsigned)((nq + 255) / 256), 256, 0, st>>>(queries, nq, n, q, status);
  rc = knn::exact_fp64(points, n, d, d, k, metric, q, nq, norms, part_dist, part_idx, (int)slices,
                       out_dist, out_idx, st);
  if (rc) {
    e = cudaGetLastError();
    return fail(KNN_ERR_CUDA, std::string("exact launch: ") + cudaGetErrorString(e));
  }
  int host_status = 0;
  e = cudaMemcpyAsync(&host_status, status, sizeof(int), cudaMemcpyDeviceToHost, st);
  if (e == cudaSuccess) e = cudaStreamSynchronize(st);
  if (e != cudaSuccess) return fail(KNN_ERR_CUDA, std::string("exact: ") + cudaGetErrorString(e));
  if (host_status) return fail(KNN_ERR_ARGS, "query id out of range");
  return KNN_OK;
}
