// C ABI of the k-NN graph builder: argument checks, device scratch, stage order.
//
// Replaces the orchestration of EuclideanDistanceMatrixGPU
// (euclideandistancematrixgpu.cu:2759-2819 initialize, :2861-2896 calculate,
// :2908-2915 the result copy of saveResultToResultFile).  The reference owns one
// pitched column-major copy of the points, per-block N-byte bitmaps
// (SMs*10*N bytes, .cu:2797) and candidate buffers; here the points are
// row-major and padded to whole float4s, and scratch is O(trees*n + n*k),
// owned by a reusable context.  Errors come back as status codes; nothing is
// printed and the device is never reset.
#include <cstdio>
#include <cstring>
#include <map>
#include <memory>
#include <string>
#include <vector>
#include <algorithm>

#include "knn_internal.cuh"
#include "knn_kernels.cuh"

namespace knn {
int exact_fp64(const float* X, int64_t n, int d, int dpad, int k, int metric,
               const int64_t* queries, int64_t nq, double* norms, double* part_dist,
               uint32_t* part_idx, int slices, double* out_dist, int32_t* out_idx,
               cudaStream_t st);
void launch_normalize_reference(float* X, int64_t n, int d, cudaStream_t st);
}  // namespace knn

namespace {

thread_local std::string g_last_error;

int fail(int code, const std::string& what) {
  g_last_error = what;
  return code;
}
int fail_cuda(cudaError_t e, const char* where) {
  g_last_error = std::string(where) + ": " + cudaGetErrorString(e);
  return e == cudaErrorMemoryAllocation ? KNN_ERR_OOM : KNN_ERR_CUDA;
}

#define KNN_CK(call)                                  \
  do {                                                \
    cudaError_t e_ = (call);                          \
    if (e_ != cudaSuccess) return fail_cuda(e_, #call); \
  } while (0)

struct Buffer {
  void* p = nullptr;
  size_t bytes = 0;
};

}  // namespace

namespace knn {
void set_last_error(const std::string& what) { g_last_error = what; }
}  // namespace knn

struct knn_context {
  int device = 0;
  cudaStream_t stream = nullptr;
  cudaEvent_t ev[8] = {};
  std::map<std::string, Buffer> bufs;
  // Bumped whenever a buffer moves: captured graphs of older generations hold
  // stale pointers and are not replayed.
  uint64_t generation = 0;
  // Captured batch pipelines by shape signature (see knn_build_batch).
  struct Captured {
    std::string sig;
    uint64_t generation;
    cudaGraphExec_t exec;
  };
  std::vector<Captured> graphs;
  std::vector<std::string> seen;
  // Autotuned launch shapes by workload key: (FP32 leaf tile, propagation warps).
  std::map<std::string, std::pair<int, int>> tuned;
  // Tuned sibling leaves per tensor-core tile, by workload key and precision.
  std::map<std::string, int> tuned_group;
  cudaEvent_t tev[2] = {};
  // Device error words: [0] is cleared at the start of every build and tells
  // the tensor-core tile kernels of that build to stop issuing work; [1] is
  // sticky -- set with [0] by a kernel whose bounded wait gave up, and cleared
  // only when a synchronising call or knn_context_status() reports it, so an
  // asynchronous build's failure reaches the caller.
  int* err_words = nullptr;
  // Test hook: the next build starts with both error words set.
  bool preset_err = false;
  // Events around each tree's leaf-tile kernel (statistics only), grown on demand.
  std::vector<cudaEvent_t> kev;
  cudaEvent_t* kernel_events(int trees) {
    while ((int)kev.size() < 2 * trees) {
      cudaEvent_t e = nullptr;
      if (cudaEventCreate(&e) != cudaSuccess) return nullptr;
      kev.push_back(e);
    }
    return kev.data();
  }

  // Device buffer `name` of at least `bytes`; grows by reallocation.
  int get(const char* name, size_t bytes, void** out) {
    Buffer& b = bufs[name];
    if (bytes == 0) bytes = 16;
    if (b.bytes < bytes) {
      if (b.p) {
        cudaError_t e = cudaFree(b.p);
        b.p = nullptr;
        b.bytes = 0;
        if (e != cudaSuccess) return fail_cuda(e, "cudaFree");
      }
      cudaError_t e = cudaMalloc(&b.p, bytes);
      if (e != cudaSuccess) {
        cudaGetLastError();
        return fail_cuda(e, (std::string("cudaMalloc ") + name).c_str());
      }
      b.bytes = bytes;
      ++generation;
    }
    *out = b.p;
    return KNN_OK;
  }
  template <typename T>
  int get(const char* name, size_t count, T** out) {
    void* p = nullptr;
    int rc = get(name, count * sizeof(T), &p);
    *out = static_cast<T*>(p);
    return rc;
  }
  int64_t bytes_held() const {
    int64_t s = 0;
    for (const auto& kv : bufs) s += (int64_t)kv.second.bytes;
    return s;
  }
  ~knn_context() {
    int cur = 0;
    if (cudaGetDevice(&cur) == cudaSuccess && cur != device) cudaSetDevice(device);
    for (auto& g : graphs) cudaGraphExecDestroy(g.exec);
    for (auto& kv : bufs)
      if (kv.second.p) cudaFree(kv.second.p);
    if (err_words) cudaFree(err_words);
    for (auto& e : ev)
      if (e) cudaEventDestroy(e);
    for (auto& e : tev)
      if (e) cudaEventDestroy(e);
    for (auto& e : kev)
      if (e) cudaEventDestroy(e);
    if (stream) cudaStreamDestroy(stream);
    if (cur != device) cudaSetDevice(cur);
  }
};

namespace {

int make_context(int device, knn_context** out) {
  int count = 0;
  cudaError_t e = cudaGetDeviceCount(&count);
  if (e != cudaSuccess || count == 0) {
    cudaGetLastError();
    return fail(KNN_ERR_NO_DEVICE, "no CUDA device");
  }
  if (device < 0) KNN_CK(cudaGetDevice(&device));
  if (device >= count) return fail(KNN_ERR_ARGS, "device ordinal out of range");
  KNN_CK(cudaSetDevice(device));
  std::unique_ptr<knn_context> c(new knn_context());
  c->device = device;
  KNN_CK(cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking));
  for (auto& ev : c->ev) KNN_CK(cudaEventCreate(&ev));
  for (auto& ev : c->tev) KNN_CK(cudaEventCreate(&ev));
  KNN_CK(cudaMalloc(&c->err_words, 2 * sizeof(int)));
  KNN_CK(cudaMemset(c->err_words, 0, 2 * sizeof(int)));
  *out = c.release();
  return KNN_OK;
}

thread_local std::map<int, std::unique_ptr<knn_context>> g_default;

int default_context(int device, knn_context** out) {
  if (device < 0) {
    cudaError_t e = cudaGetDevice(&device);
    if (e != cudaSuccess) {
      cudaGetLastError();
      return fail(KNN_ERR_NO_DEVICE, "no CUDA device");
    }
  }
  auto it = g_default.find(device);
  if (it != g_default.end()) {
    *out = it->second.get();
    return KNN_OK;
  }
  knn_context* c = nullptr;
  int rc = make_context(device, &c);
  if (rc) return rc;
  g_default[device].reset(c);
  *out = c;
  return KNN_OK;
}

int check_common(const void* points, int64_t n, int d, int k, int metric) {
  if (!points) return fail(KNN_ERR_ARGS, "points is NULL");
  if (n < 1 || n >= (int64_t)INT32_MAX) return fail(KNN_ERR_ARGS, "n out of range");
  if (d < 1) return fail(KNN_ERR_ARGS, "d must be >= 1");
  if (k < 1 || k > KNN_MAX_K) return fail(KNN_ERR_ARGS, "k must be in 1..KNN_MAX_K");
  if (metric < 0 || metric > 2) return fail(KNN_ERR_ARGS, "unknown metric");
  if (n <= k) return fail(KNN_ERR_N_LE_K, "n must exceed k");
  return KNN_OK;
}

inline int round4(int d) { return (d + 3) & ~3; }

struct Prepared {
  const float* X = nullptr;
  int dpad = 0;
  const void* Xh = nullptr;  // FP16 input: its rows zero padded to ldh (a multiple of 8), for gathers
  int ldh = 0;
};

// Points -> zero-padded float32 rows on the device.
int prepare_points(knn_context* C, const void* points, int64_t n, int d, const knn_options& o,
                   cudaStream_t st, Prepared* P, knn::LaunchLog& log) {
  const int dpad = round4(d);
  const int64_t ld = o.ld ? o.ld : d;
  if (ld < d) return fail(KNN_ERR_ARGS, "ld < d");
  P->dpad = dpad;
  const size_t esz = o.dtype == KNN_F32 ? 4 : 2;
  if (o.dtype == KNN_F16) {
    P->ldh = (d + 7) & ~7;
    if (o.points_on_device && ld == d && (d & 7) == 0 && ((uintptr_t)points & 15) == 0) P->Xh = points;
  }
  if (o.points_on_device) {
    if (o.dtype == KNN_F32 && ld == d && (d & 3) == 0 && ((uintptr_t)points & 15) == 0) {
      P->X = static_cast<const float*>(points);
      return KNN_OK;
    }
    float* X = nullptr;
    int rc = C->get("X", (size_t)n * dpad, &X);
    if (rc) return rc;
    knn::launch_pad_rows(points, o.dtype, n, d, ld, X, dpad, st);
    log.add();
    P->X = X;
    if (o.dtype == KNN_F16 && !P->Xh) {
      void* Xh = nullptr;
      rc = C->get("Xh", (size_t)n * P->ldh * 2, &Xh);
      if (rc) return rc;
      knn::launch_pad_rows_f16(points, n, d, ld, Xh, P->ldh, st);
      log.add();
      P->Xh = Xh;
    }
    return KNN_OK;
  }
  float* X = nullptr;
  int rc = C->get("X", (size_t)n * dpad, &X);
  if (rc) return rc;
  if (o.dtype == KNN_F32) {
    KNN_CK(cudaMemcpy2DAsync(X, (size_t)dpad * 4, points, (size_t)ld * 4, (size_t)d * 4, (size_t)n,
                             cudaMemcpyHostToDevice, st));
    if (dpad != d)
      KNN_CK(cudaMemset2DAsync(X + d, (size_t)dpad * 4, 0, (size_t)(dpad - d) * 4, (size_t)n, st));
  } else {
    void* stage = nullptr;
    rc = C->get("stage", (size_t)n * ld * esz, &stage);
    if (rc) return rc;
    KNN_CK(cudaMemcpyAsync(stage, points, (size_t)n * ld * esz, cudaMemcpyHostToDevice, st));
    knn::launch_pad_rows(stage, o.dtype, n, d, ld, X, dpad, st);
    log.add();
    if (o.dtype == KNN_F16) {
      void* Xh = nullptr;
      rc = C->get("Xh", (size_t)n * P->ldh * 2, &Xh);
      if (rc) return rc;
      knn::launch_pad_rows_f16(stage, n, d, ld, Xh, P->ldh, st);
      log.add();
      P->Xh = Xh;
    }
  }
  P->X = X;
  return KNN_OK;
}

struct Trees {
  int32_t* perm = nullptr;
  int depth = 0;
};

// Trees of a batch of segments (global positions), or of one point set.
int run_trees_segs(knn_context* C, const float* X, int64_t ntot, int d, int dpad, int trees,
                   const knn::SegView& segs, const knn::SegEntry* hsegs, int nseg, cudaStream_t st,
                   Trees* T, knn::LaunchLog& log, int tree_offset = 0, int tree_stride = 1) {
  knn::TreeArgs a{};
  a.tree_offset = tree_offset;
  a.tree_stride = tree_stride > 0 ? tree_stride : 1;
  a.X = X;
  a.n = ntot;
  a.d = d;
  a.dpad = dpad;
  a.trees = trees;
  a.segs = segs;
  a.hsegs = hsegs;
  a.nseg = nseg;
  int rc = C->get("perm", (size_t)trees * ntot, &a.perm);
  if (!rc) rc = C->get("perm_alt", (size_t)trees * ntot, &a.perm_alt);
  if (!rc) rc = C->get("perm_inv", (size_t)trees * ntot, &a.inv);
  if (!rc) rc = C->get("perm_node", (size_t)trees * ntot, &a.node);
  if (!rc) rc = C->get("keys", (size_t)trees * ntot, &a.keys);
  if (!rc) rc = C->get("dirs", knn::tree_dir_nodes(hsegs, nseg, trees) * dpad, &a.dirs);
  if (!rc) rc = C->get("msplit", knn::msplit_scratch_bytes(hsegs[0].n), &a.msplit);
  if (rc) return rc;
  a.stream = st;
  rc = knn::tree_build(a, log);
  if (rc) return fail_cuda(cudaGetLastError(), "tree build launch");
  T->perm = a.perm;
  T->depth = hsegs[0].depth;
  return KNN_OK;
}

int run_trees(knn_context* C, const float* X, int64_t n, int d, int dpad, int trees, int leaf,
              uint64_t seed, cudaStream_t st, Trees* T, knn::LaunchLog& log, int tree_offset = 0,
              int tree_stride = 1) {
  const int depth = knn::tree_depth(n, leaf);
  if (depth > 30) return fail(KNN_ERR_ARGS, "tree too deep (n / leaf too large)");
  knn::SegEntry e{};
  e.off = 0;
  e.n = n;
  e.seed = seed;
  e.leaf_base = 0;
  e.depth = depth;
  return run_trees_segs(C, X, n, d, dpad, trees, knn::single_segment(n, seed, depth), &e, 1, st, T, log,
                        tree_offset, tree_stride);
}

// Reference-rule trees (tree_faithful.cu); T->depth = levels built.
int run_faithful_trees(knn_context* C, const float* X, int64_t n, int d, int dpad, int trees, int leaf,
                       uint64_t seed, int tree_offset, int tree_stride, cudaStream_t st, Trees* T,
                       knn::FaithfulTrees* FT, knn::LaunchLog& log) {
  knn::FaithfulArgs a{};
  a.X = X;
  a.n = n;
  a.d = d;
  a.dpad = dpad;
  a.trees = trees;
  a.leaf = leaf;
  a.seed = seed;
  a.tree_offset = tree_offset;
  a.tree_stride = tree_stride;
  // splitting nodes per level: at most trees * n / (leaf + 1); chunk counts
  // sum to at most that plus trees * n / 1024
  a.node_cap = (size_t)trees * (size_t)(n / (leaf + 1) + 1);
  a.count_cap = a.node_cap + (size_t)trees * (size_t)(n / 1024 + 1);
  int rc = C->get("perm", (size_t)trees * n, &a.perm);
  if (!rc) rc = C->get("perm_alt", (size_t)trees * n, &a.perm_alt);
  if (!rc) rc = C->get("f_side", (size_t)trees * n, &a.side);
  if (!rc) rc = C->get("f_nodes", a.node_cap, &a.dnodes);
  if (!rc) rc = C->get("f_lcount", a.count_cap, &a.lcount);
  if (!rc) rc = C->get("f_nleft", a.node_cap, &a.nleft);
  if (rc) return rc;
  a.stream = st;
  rc = knn::faithful_tree_build(a, FT, log);
  if (rc == KNN_ERR_UNSUPPORTED) return fail(rc, "reference-rule tree deeper than the level limit");
  if (rc) return fail_cuda(cudaGetLastError(), "reference-rule tree build");
  T->perm = a.perm;
  T->depth = FT->levels;
  return KNN_OK;
}

struct Lists {
  float* key[2];
  uint32_t* id[2];
  uint32_t* flags[2];
  int cur = 0;
};

int get_lists(knn_context* C, int64_t n, int k, Lists* L) {
  const int kw = (k + 31) / 32;
  int rc = C->get("key0", (size_t)n * k, &L->key[0]);
  if (!rc) rc = C->get("key1", (size_t)n * k, &L->key[1]);
  if (!rc) rc = C->get("id0", (size_t)n * k, &L->id[0]);
  if (!rc) rc = C->get("id1", (size_t)n * k, &L->id[1]);
  if (!rc) rc = C->get("flags0", (size_t)n * kw, &L->flags[0]);
  if (!rc) rc = C->get("flags1", (size_t)n * kw, &L->flags[1]);
  L->cur = 0;
  return rc;
}

// Where the leaves of every tree lie: segments, leaf blocks per tree, largest leaf.
struct Layout {
  knn::SegView segs;
  int64_t leaves = 1, maxleaf = 1;
  int64_t maxblock = 0;  // bound on the points of a leaf block (0: unknown)
  int tc_group_max = 1;  // sibling leaves a tensor-core tile may hold (1, 2 or 4)
  bool own_blocks = false;  // every leaf holds k+1 points, so each leaf is its own block
  // reference-rule trees: explicit leaf table (device) and per-tree offsets / counts (host)
  const int64_t* ftable = nullptr;
  const int64_t* foff = nullptr;
  const int64_t* fcount = nullptr;
};

// Bound on the leaf blocks of a median tree of n points and this depth: node
// sizes at level l are floor or ceil of n / 2^l, and a leaf climbs at most to
// the deepest level whose smallest node holds k+1 points.
int64_t host_max_block(int64_t n, int depth, int k) {
  int l = depth;
  while (l > 0 && (n >> l) < k + 1) --l;
  return (n + (int64_t(1) << l) - 1) >> l;
}

// Largest group of sibling leaves (1, 2 or 4) that one 128-row tensor-core
// tile can take with every leaf its own block: leaves of at most 128 / G
// points, the smallest leaf of every segment (floor(n / 2^depth) points)
// holding k+1, and every segment at least log2 G levels deep so that groups
// never straddle two sets.
// Every leaf of every segment holds at least k+1 points (the smallest leaf of a
// median tree holds floor(n / 2^depth)), so no leaf block climbs above its leaf.
bool leaves_own_blocks(const knn::SegEntry* hsegs, int nseg, int k) {
  for (int i = 0; i < nseg; ++i)
    if ((hsegs[i].n >> hsegs[i].depth) < k + 1) return false;
  return true;
}

int tc_group_max(const knn::SegEntry* hsegs, int nseg, int k, int64_t maxleaf) {
  int g = 1;
  for (int cand = 2, lg = 1; cand <= 4; cand *= 2, ++lg) {
    if (maxleaf * cand > 128) break;
    bool ok = true;
    for (int i = 0; i < nseg && ok; ++i)
      ok = hsegs[i].depth >= lg && (hsegs[i].n >> hsegs[i].depth) >= k + 1;
    if (!ok) break;
    g = cand;
  }
  return g;
}

Layout single_layout(int64_t n, int depth) {
  Layout y;
  y.segs = knn::single_segment(n, 0, depth);
  y.leaves = int64_t(1) << depth;
  y.maxleaf = (n + y.leaves - 1) / y.leaves;
  return y;
}

int run_leaf(knn_context* C, const float* X, int64_t n, int d, int dpad, int k, int trees,
             const Layout& lay, int metric, const int32_t* perm, const float* norms, Lists* L,
             unsigned long long* counter, cudaStream_t st, knn::LaunchLog& log, int tile = 0,
             cudaEvent_t* kev = nullptr, bool sparse = false, bool pairs = false) {
  const int kw = (k + 31) / 32;
  knn::launch_init_lists(L->key[L->cur], L->id[L->cur], L->flags[L->cur], n, k, kw, st);
  log.add(2);
  knn::LeafArgs a{};
  a.X = X;
  a.n = n;
  a.d = d;
  a.dpad = dpad;
  a.k = k;
  a.trees = trees;
  a.segs = lay.segs;
  a.leaves = lay.leaves;
  a.maxleaf = lay.maxleaf;
  a.maxblock = lay.maxblock;
  a.metric = metric;
  a.perm = perm;
  a.norms = norms;
  a.rkey = L->key[L->cur];
  a.rid = L->id[L->cur];
  a.pair_counter = counter;
  a.tile = tile;
  a.kev = kev;
  a.ftable = lay.ftable;
  a.foff = lay.foff;
  a.fcount = lay.fcount;
  a.stream = st;
  a.pairs = pairs && lay.own_blocks && !lay.ftable;
  if (sparse && metric != KNN_METRIC_COSINE && !lay.ftable) {
    a.lmax = 256 * ((dpad + 255) / 256);
    int rc = C->get("dmask", (size_t)lay.leaves * (dpad / 32 + 1), &a.dmask);
    if (!rc) rc = C->get("dlist", (size_t)lay.leaves * a.lmax, &a.dlist);
    if (!rc) rc = C->get("dnch", (size_t)lay.leaves, &a.dnch);
    if (!rc && a.pairs && dpad <= 4096) {
      // tile pairs read the union of their two tiles' dims: the leaf stage
      // reorders positions within each leaf of the trees' order (context
      // scratch) by row bucket, which leaves every leaf's point set as it is
      a.perm_w = const_cast<int32_t*>(perm);
      rc = C->get("rbucket", (size_t)n, &a.bucket);
      if (!rc) rc = C->get("rzeros", 1, &a.zeros);
      if (!rc) rc = C->get("sort_tmp", (size_t)n, &a.sort_tmp);
      if (!rc)
        rc = C->get("tmask", (size_t)lay.leaves * ((lay.maxleaf + 31) / 32) * ((dpad + 31) / 32 + 1), &a.tmask);
    }
    if (rc) return rc;
  }
  int rc = knn::leaf_stage(a, log);
  if (rc) return fail_cuda(cudaGetLastError(), "leaf stage launch");
  return KNN_OK;
}

// Sparse-row leaf tiles (same keys, fewer dims read): forced on or off by the
// option, else on when leaves hold at least 1024 points, where the per-tree
// mask pass (one read of the points) is small beside the tiles.
bool use_sparse_dims(const knn_options& o, int metric, const Layout& lay, int dpad) {
  // dim lists are 16-bit
  if (metric == KNN_METRIC_COSINE || lay.ftable || o.sparse_dims < 0 || dpad > 32767) return false;
  return o.sparse_dims > 0 || lay.maxleaf >= 1024;
}

// Symmetric tile pairs (each key computed once for both of its points): on
// unless the option turns them off, wherever every leaf is its own block.
bool use_tile_pairs(const knn_options& o, const Layout& lay) {
  return o.tile_pairs >= 0 && lay.own_blocks && !lay.ftable;
}

// Mixed precision: BF16 or FP16 tensor-core tiles select each point's best min(2k, 32)
// approximate candidates over all trees; FP32 re-rank keeps the exact best k.
int run_leaf_umma(knn_context* C, const float* X, int64_t n, int d, int dpad, int k, int trees,
                  const Layout& lay, int metric, int precision, const int32_t* perm, const float* norms,
                  Lists* L, int* err_flag, cudaStream_t st, knn::LaunchLog& log, cudaEvent_t* kev = nullptr,
                  int tc_group = 1) {
  const int kw = (k + 31) / 32;
  const int kq = k <= 16 ? 2 * k : 32;
  const int Kp = ((d + 63) / 64) * 64;
  knn::UmmaLeafArgs a{};
  a.X = X;
  a.n = n;
  a.d = d;
  a.dpad = dpad;
  a.k = k;
  a.kq = kq;
  a.trees = trees;
  a.segs = lay.segs;
  a.leaves = lay.leaves;
  a.maxleaf = lay.maxleaf;
  a.maxblock = lay.maxblock > 0 ? lay.maxblock : INT64_MAX;
  a.tc_group = std::min(std::max(tc_group, 1), lay.tc_group_max);
  a.ftable = lay.ftable;
  a.foff = lay.foff;
  a.fcount = lay.fcount;
  a.metric = metric;
  a.perm = perm;
  a.norms = norms;
  a.err = err_flag;
  a.stream = st;
  a.kev = kev;
  a.rkey = L->key[L->cur];
  a.rid = L->id[L->cur];
  a.f16 = precision == KNN_PREC_F16_RERANK;
  int rc = C->get("Xb", (size_t)n * Kp * 2, &a.Xb);
  if (!rc) rc = C->get("maxabs", 1, &a.maxabs);
  if (!rc) rc = C->get("norms2", (size_t)n, &a.norms2);
  if (!rc && trees > 1) rc = C->get("linv", (size_t)n, &a.inv);
  if (!rc) rc = C->get("akey", (size_t)n * kq, &a.akey);
  if (!rc) rc = C->get("aid", (size_t)n * kq, &a.aid);
  if (rc) return rc;
  knn::launch_init_lists(a.akey, a.aid, nullptr, n, kq, 1, st);
  log.add();
  rc = knn::leaf_stage_umma(a, log);
  if (rc == KNN_ERR_UNSUPPORTED) return fail(rc, "tensor-core leaf stage: unsupported shape");
  if (rc) return fail_cuda(cudaGetLastError(), "tensor-core leaf stage launch");
  knn::launch_set_flags(L->flags[L->cur], n, k, kw, st);
  log.add();
  return KNN_OK;
}

int run_prop(const float* X, int64_t n, int d, int dpad, int k, int metric, const float* norms,
             const int32_t* order, Lists* L, bool with_flags, unsigned long long* counter,
             cudaStream_t st, knn::LaunchLog& log, int warps = 0, const void* Xh = nullptr, int ldh = 0) {
  knn::PropArgs a{};
  a.X = X;
  a.Xh = Xh;
  a.ldh = ldh;
  a.n = n;
  a.d = d;
  a.dpad = dpad;
  a.k = k;
  a.metric = metric;
  a.norms = norms;
  a.order = order;
  a.key_in = L->key[L->cur];
  a.id_in = L->id[L->cur];
  a.flags_in = with_flags ? L->flags[L->cur] : nullptr;
  a.key_out = L->key[1 - L->cur];
  a.id_out = L->id[1 - L->cur];
  a.flags_out = L->flags[1 - L->cur];
  a.cand_counter = counter;
  a.warps = warps;
  a.stream = st;
  int rc = knn::propagate_step(a, log);
  if (rc == KNN_ERR_UNSUPPORTED) return fail(rc, "propagation scratch exceeds shared memory (k or d too large)");
  if (rc) return fail_cuda(cudaGetLastError(), "propagation launch");
  L->cur = 1 - L->cur;
  return KNN_OK;
}

// ---------------------------------------------------------------- tuning --
// Launch shapes that do not change any result -- the FP32 leaf kernel's
// query x candidate tile and the propagation kernel's warps per block -- are
// picked by timing.  Each candidate runs twice on the call's own trees and
// lists (into the spare list buffers; the second run is timed with events) and
// the fastest is cached in the context per (metric, d, k, largest leaf).
// Tuning happens only in eagerly launched calls; captured graphs use the cache.
std::string tune_key(int metric, int d, int k, int64_t maxleaf) {
  return "m" + std::to_string(metric) + ":d" + std::to_string(d) + ":k" + std::to_string(k) + ":L" +
         std::to_string(maxleaf);
}

int time_since(knn_context* C, cudaStream_t st, float* ms) {
  KNN_CK(cudaEventRecord(C->tev[1], st));
  KNN_CK(cudaEventSynchronize(C->tev[1]));
  KNN_CK(cudaEventElapsedTime(ms, C->tev[0], C->tev[1]));
  return KNN_OK;
}

int tune_leaf_tile(knn_context* C, const float* X, int64_t n, int d, int dpad, int k, const Layout& lay,
                   int metric, const int32_t* perm, const float* norms, const Lists& L, cudaStream_t st,
                   bool sparse, bool pairs, int* best) {
  Lists S = L;
  S.cur = 1 - L.cur;  // scratch lists
  float best_ms = 3.4e38f;
  *best = 64;
  for (int tile : {64, 32}) {
    float ms = 0;
    for (int rep = 0; rep < 2; ++rep) {
      knn::LaunchLog tl;
      KNN_CK(cudaEventRecord(C->tev[0], st));
      int rc = run_leaf(C, X, n, d, dpad, k, 1, lay, metric, perm, norms, &S, nullptr, st, tl, tile, nullptr, sparse,
                        pairs);
      if (!rc) rc = time_since(C, st, &ms);
      if (rc) return rc;
    }
    if (ms < best_ms) {
      best_ms = ms;
      *best = tile;
    }
  }
  return KNN_OK;
}

int tune_prop_warps(knn_context* C, const float* X, int64_t n, int d, int dpad, int k, int metric,
                    const float* norms, const int32_t* order, Lists* L, cudaStream_t st, int* best) {
  const int cur = L->cur;
  float best_ms = 3.4e38f;
  *best = 0;
  for (int w : {8, 4, 2}) {
    float ms = 0;
    for (int rep = 0; rep < 2; ++rep) {
      knn::LaunchLog tl;
      KNN_CK(cudaEventRecord(C->tev[0], st));
      int rc = run_prop(X, n, d, dpad, k, metric, norms, order, L, true, nullptr, st, tl, w);
      L->cur = cur;  // the timing run's output is scratch
      if (!rc) rc = time_since(C, st, &ms);
      if (rc) return rc;
    }
    if (ms < best_ms) {
      best_ms = ms;
      *best = w;
    }
  }
  return KNN_OK;
}

// Leaf tile and propagation warps for this call: forced by the options,
// cached, or tuned now (when allowed).
struct Shapes {
  int leaf_tile = 0, prop_warps = 0;
  bool sparse = false;  // FP32 leaf tiles read each block's non-zero dims only
  bool pairs = false;   // FP32 leaf tiles computed once per tile pair
  int tc_group = 0;  // tensor-core tiles: sibling leaves per tile
};

// Sibling leaves per tensor-core tile (results identical for every choice):
// each allowed group is run twice over the first tree into the spare lists,
// the second run timed.
int tune_tc_group(knn_context* C, const float* X, int64_t n, int d, int dpad, int k, const Layout& lay,
                  int metric, int precision, const int32_t* perm, const float* norms, const Lists& L,
                  int* err_flag, cudaStream_t st, int* best) {
  Lists S = L;
  S.cur = 1 - L.cur;
  float best_ms = 3.4e38f;
  *best = lay.tc_group_max;
  for (int g = lay.tc_group_max; g >= 1; g /= 2) {
    float ms = 0;
    for (int rep = 0; rep < 2; ++rep) {
      knn::LaunchLog tl;
      KNN_CK(cudaEventRecord(C->tev[0], st));
      int rc = run_leaf_umma(C, X, n, d, dpad, k, 1, lay, metric, precision, perm, norms, &S, err_flag, st, tl,
                             nullptr, g);
      if (!rc) rc = time_since(C, st, &ms);
      if (rc) return rc;
    }
    if (ms < best_ms) {
      best_ms = ms;
      *best = g;
    }
  }
  return KNN_OK;
}

int pick_shapes(knn_context* C, const knn_options& o, bool may_tune, bool fp32_leaf, int props, const float* X,
                int64_t n, int d, int dpad, int k, const Layout& lay, int metric, const int32_t* perm,
                const float* norms, Lists* L, cudaStream_t st, Shapes* sh, bool* tune_prop_after,
                int* err_flag) {
  sh->leaf_tile = o.leaf_tile;
  sh->prop_warps = o.prop_warps;
  sh->sparse = fp32_leaf && use_sparse_dims(o, metric, lay, dpad);
  sh->pairs = fp32_leaf && use_tile_pairs(o, lay);
  *tune_prop_after = false;
  const std::string key = tune_key(metric, d, k, lay.maxleaf);
  if (!fp32_leaf) {
    // tensor-core tiles: forced, cached, tuned (eager calls with autotune), or the largest group
    const std::string gkey = key + ":q" + std::to_string(o.precision);
    auto gi = C->tuned_group.find(gkey);
    if (o.tc_group) sh->tc_group = o.tc_group;
    else if (gi != C->tuned_group.end()) sh->tc_group = gi->second;
    else if (o.autotune && may_tune && lay.tc_group_max > 1) {
      int rc = tune_tc_group(C, X, n, d, dpad, k, lay, metric, o.precision, perm, norms, *L, err_flag, st,
                             &sh->tc_group);
      if (rc) return rc;
      C->tuned_group[gkey] = sh->tc_group;
    } else {
      sh->tc_group = lay.tc_group_max;
    }
    sh->tc_group = std::min(sh->tc_group, lay.tc_group_max);
  }
  if (!o.autotune) return KNN_OK;
  auto it = C->tuned.find(key);
  if (it != C->tuned.end()) {
    if (!sh->leaf_tile) sh->leaf_tile = it->second.first;
    if (!sh->prop_warps) sh->prop_warps = it->second.second;
    if (!(fp32_leaf && sh->leaf_tile == 0) && !(props > 0 && sh->prop_warps == 0)) return KNN_OK;
  }
  if (!may_tune) return KNN_OK;
  if (fp32_leaf && !sh->leaf_tile) {
    int rc = tune_leaf_tile(C, X, n, d, dpad, k, lay, metric, perm, norms, *L, st, sh->sparse, sh->pairs,
                            &sh->leaf_tile);
    if (rc) return rc;
    C->tuned[key].first = sh->leaf_tile;
  }
  *tune_prop_after = props > 0 && !sh->prop_warps;
  return KNN_OK;
}

int finish_prop_tuning(knn_context* C, const knn_options& o, const float* X, int64_t n, int d, int dpad, int k,
                       int metric, const float* norms, const int32_t* order, Lists* L, int64_t maxleaf,
                       cudaStream_t st, Shapes* sh) {
  int rc = tune_prop_warps(C, X, n, d, dpad, k, metric, norms, order, L, st, &sh->prop_warps);
  if (rc) return rc;
  C->tuned[tune_key(metric, d, k, maxleaf)].second = sh->prop_warps;
  (void)o;
  return KNN_OK;
}

// Learned split network (mlp.cu): the plain graph of a strided sample of the
// points trains the MLP; the trees are then built on the embeddings of all
// points.  Sample graph: 8 trees, leaf 128, 2 propagations, 2k neighbours (at
// most 32), plain FP32.
constexpr int kMlpSampleDefault = 65536;
constexpr int kMlpStepsDefault = 300;
constexpr int kMlpBatch = 1024;
constexpr float kMlpLr = 1e-3f;
constexpr float kMlpMargin = 1.0f;
constexpr int kMlpGraphTrees = 8, kMlpGraphLeaf = 128, kMlpGraphProps = 2;
constexpr int64_t kMlpEmbedChunk = 65536;
constexpr uint64_t kMlpSeedSalt = 0x6C6561726E656421ull;

struct Learned {
  float* params = nullptr;
  float* mean = nullptr;
  float* inv_std = nullptr;
  float* loss = nullptr;
  int steps = 0;
};

int learn_network(knn_context* C, const float* X, int64_t n, int d, int dpad, int k, int metric,
                  uint64_t seed, const knn_options& o, cudaStream_t st, Learned* Lr, knn::LaunchLog& log) {
  int64_t ns = o.mlp_sample > 0 ? o.mlp_sample : kMlpSampleDefault;
  if (ns > n) ns = n;
  int gk = 2 * k;
  if (gk > 32) gk = 32;
  if (gk < 2) gk = 2;
  if (ns <= gk) return fail(KNN_ERR_ARGS, "learned splits: too few points for the training graph");
  const int steps = o.mlp_steps > 0 ? o.mlp_steps : kMlpStepsDefault;
  const uint64_t lseed = knn::splitmix64(seed ^ kMlpSeedSalt);

  float* Xs = nullptr;
  int rc = C->get("mlp_Xs", (size_t)ns * dpad, &Xs);
  if (rc) return rc;
  knn::launch_gather_sample(X, n, dpad, ns, Xs, st);
  log.add();
  float* norms = nullptr;
  if (metric == KNN_METRIC_COSINE) {
    rc = C->get("mlp_norms", (size_t)ns, &norms);
    if (rc) return rc;
    knn::launch_norms(Xs, ns, d, dpad, norms, st);
    log.add();
  }
  Trees T;
  rc = run_trees(C, Xs, ns, d, dpad, kMlpGraphTrees, kMlpGraphLeaf, lseed, st, &T, log);
  if (rc) return rc;
  Lists L;
  rc = get_lists(C, ns, gk, &L);
  if (!rc)
    rc = run_leaf(C, Xs, ns, d, dpad, gk, kMlpGraphTrees, single_layout(ns, T.depth), metric, T.perm, norms, &L,
                  nullptr, st, log);
  for (int p = 0; !rc && p < kMlpGraphProps; ++p)
    rc = run_prop(Xs, ns, d, dpad, gk, metric, norms, T.perm, &L, true, nullptr, st, log);
  if (rc) return rc;
  int32_t* graph = nullptr;
  float* gdist = nullptr;
  rc = C->get("mlp_graph", (size_t)ns * gk, &graph);
  if (!rc) rc = C->get("mlp_gdist", (size_t)ns * gk, &gdist);
  if (rc) return rc;
  knn::launch_finalize(L.key[L.cur], L.id[L.cur], ns, gk, metric, gdist, graph, st);
  log.add();

  knn::MlpTrainArgs a{};
  a.Xs = Xs;
  a.norms = norms;
  a.ns = ns;
  a.d = d;
  a.dpad = dpad;
  a.graph = graph;
  a.gk = gk;
  a.steps = steps;
  a.batch = kMlpBatch;
  a.lr = kMlpLr;
  a.margin = kMlpMargin;
  a.seed = lseed;
  a.stream = st;
  rc = C->get("mlp_params", knn::mlp_param_count(d), &a.params);
  if (!rc) rc = C->get("mlp_mean", (size_t)d, &a.mean);
  if (!rc) rc = C->get("mlp_inv_std", (size_t)d, &a.inv_std);
  if (!rc) rc = C->get("mlp_loss", (size_t)steps, &a.loss);
  if (!rc) rc = C->get("mlp_ws", knn::mlp_train_ws_floats(d, kMlpBatch), &a.ws);
  if (rc) return rc;
  rc = knn::mlp_train(a, log);
  if (rc) return fail_cuda(cudaGetLastError(), "learned split training launch");
  Lr->params = a.params;
  Lr->mean = a.mean;
  Lr->inv_std = a.inv_std;
  Lr->loss = a.loss;
  Lr->steps = steps;
  return KNN_OK;
}

int embed_points(knn_context* C, const float* X, const float* norms, int64_t n, int d, int dpad,
                 const float* params, const float* mean, const float* inv_std, cudaStream_t st, float** Z,
                 knn::LaunchLog& log) {
  float* ws = nullptr;
  const int64_t chunk = n < kMlpEmbedChunk ? n : kMlpEmbedChunk;
  int rc = C->get("mlp_Z", (size_t)n * knn::kMlpEmbed, Z);
  if (!rc) rc = C->get("mlp_embed_ws", knn::mlp_embed_ws_floats(d, chunk), &ws);
  if (rc) return rc;
  rc = knn::mlp_embed(X, norms, n, d, dpad, params, mean, inv_std, ws, chunk, *Z, st, log);
  if (rc) return fail_cuda(cudaGetLastError(), "learned split embedding launch");
  return KNN_OK;
}

int resolve_options(const knn_options* opt, knn_options* o) {
  knn_default_options(o);
  if (opt) {
    if (opt->struct_size != (int32_t)sizeof(knn_options))
      return fail(KNN_ERR_ARGS, "knn_options.struct_size mismatch");
    *o = *opt;
  }
  if (o->dtype < 0 || o->dtype > 2) return fail(KNN_ERR_ARGS, "unknown dtype");
  if (o->precision < 0 || o->precision > 2) return fail(KNN_ERR_ARGS, "unknown precision mode");
  if (o->learned_splits < 0 || o->learned_splits > 1) return fail(KNN_ERR_ARGS, "learned_splits must be 0 or 1");
  if (o->mlp_sample < 0 || o->mlp_steps < 0) return fail(KNN_ERR_ARGS, "negative learned-split setting");
  if (o->autotune < 0 || o->autotune > 1) return fail(KNN_ERR_ARGS, "autotune must be 0 or 1");
  if (o->leaf_tile != 0 && o->leaf_tile != 32 && o->leaf_tile != 64)
    return fail(KNN_ERR_ARGS, "leaf_tile must be 0, 32 or 64");
  if (o->prop_warps < 0 || o->prop_warps > 8) return fail(KNN_ERR_ARGS, "prop_warps must be in 0..8");
  if (o->tree_offset < 0 || o->tree_stride < 0) return fail(KNN_ERR_ARGS, "negative tree offset or stride");
  if (o->raw_keys < 0 || o->raw_keys > 1) return fail(KNN_ERR_ARGS, "raw_keys must be 0 or 1");
  if (o->split_rule < 0 || o->split_rule > 1) return fail(KNN_ERR_ARGS, "unknown split rule");
  if (o->tc_group != 0 && o->tc_group != 1 && o->tc_group != 2 && o->tc_group != 4)
    return fail(KNN_ERR_ARGS, "tc_group must be 0, 1, 2 or 4");
  if (o->split_rule == KNN_SPLIT_REFERENCE && o->learned_splits)
    return fail(KNN_ERR_UNSUPPORTED, "reference-rule splits and learned splits do not combine");
  return KNN_OK;
}

int enter_device(knn_context** ctx, const knn_options& o) {
  if (!*ctx) {
    int rc = default_context(o.device, ctx);
    if (rc) return rc;
  } else if (o.device >= 0 && o.device != (*ctx)->device) {
    return fail(KNN_ERR_ARGS, "context device differs from options.device");
  }
  KNN_CK(cudaSetDevice((*ctx)->device));
  return KNN_OK;
}

// Start of a build: clear the per-build error word (or set both words for the
// test hook) on the build's stream.
int reset_error_word(knn_context* C, cudaStream_t st) {
  if (C->preset_err) {
    C->preset_err = false;
    KNN_CK(cudaMemsetAsync(C->err_words, 0x01, 2 * sizeof(int), st));
  } else {
    KNN_CK(cudaMemsetAsync(C->err_words, 0, sizeof(int), st));
  }
  return KNN_OK;
}

// After the stream has finished: KNN_ERR_TIMEOUT (and the sticky word
// cleared) when a tile wait of this or an earlier asynchronous build gave up.
int check_error_words(knn_context* C) {
  int host[2] = {0, 0};
  KNN_CK(cudaMemcpy(host, C->err_words, sizeof(host), cudaMemcpyDeviceToHost));
  if (host[0] == 0 && host[1] == 0) return KNN_OK;
  // reported: clear both (the stream has finished, so no kernel of the build reads them)
  KNN_CK(cudaMemset(C->err_words, 0, 2 * sizeof(int)));
  return fail(KNN_ERR_TIMEOUT, "a tensor-core tile wait exceeded its time limit");
}

int build_impl(knn_context* C, const void* points, int64_t n, int32_t d, int32_t k,
               int32_t trees, int32_t leaf, int32_t props, int32_t metric, uint64_t seed,
               int32_t* out_idx, float* out_dist, const knn_options& o, knn_stats* stats) {
  cudaStream_t st = o.stream ? static_cast<cudaStream_t>(o.stream) : C->stream;
  knn::LaunchLog log;
  const bool timed = stats != nullptr;
  if (timed) KNN_CK(cudaEventRecord(C->ev[0], st));

  unsigned long long* counters = nullptr;
  int rc = C->get("counters", 2 + KNN_MAX_PROPS, &counters);
  if (rc) return rc;
  if (stats) KNN_CK(cudaMemsetAsync(counters, 0, sizeof(unsigned long long) * (2 + KNN_MAX_PROPS), st));

  Prepared P;
  rc = prepare_points(C, points, n, d, o, st, &P, log);
  if (rc) return rc;
  float* norms = nullptr;
  if (metric == KNN_METRIC_COSINE) {
    rc = C->get("norms", (size_t)n, &norms);
    if (rc) return rc;
    knn::launch_norms(P.X, n, d, P.dpad, norms, st);
    log.add();
  }
  if (timed) KNN_CK(cudaEventRecord(C->ev[1], st));

  Trees T;
  knn::FaithfulTrees FT;
  std::vector<int64_t> ftab_h, foff_h, fcount_h;
  const int64_t* ftab_d = nullptr;
  if (o.split_rule == KNN_SPLIT_REFERENCE) {
    rc = run_faithful_trees(C, P.X, n, d, P.dpad, trees, leaf, seed, o.tree_offset, o.tree_stride, st, &T, &FT,
                            log);
    if (rc) return rc;
    knn::faithful_leaf_table(FT, trees, k, &ftab_h, &foff_h, &fcount_h);
    int64_t* dt = nullptr;
    rc = C->get("ftable", ftab_h.size(), &dt);
    if (rc) return rc;
    KNN_CK(cudaMemcpyAsync(dt, ftab_h.data(), sizeof(int64_t) * ftab_h.size(), cudaMemcpyHostToDevice, st));
    ftab_d = dt;
  } else if (o.learned_splits) {
    // Trees on the learned 64-dim embedding; leaf and propagation on X.
    Learned Lr;
    rc = learn_network(C, P.X, n, d, P.dpad, k, metric, seed, o, st, &Lr, log);
    float* Z = nullptr;
    if (!rc) rc = embed_points(C, P.X, norms, n, d, P.dpad, Lr.params, Lr.mean, Lr.inv_std, st, &Z, log);
    if (rc) return rc;
    if (timed) KNN_CK(cudaEventRecord(C->ev[6], st));
    rc = run_trees(C, Z, n, knn::kMlpEmbed, knn::kMlpEmbed, trees, leaf, seed, st, &T, log);
  } else {
    rc = run_trees(C, P.X, n, d, P.dpad, trees, leaf, seed, st, &T, log, o.tree_offset, o.tree_stride);
  }
  if (rc) return rc;
  if (timed) KNN_CK(cudaEventRecord(C->ev[2], st));

  Lists L;
  rc = get_lists(C, n, k, &L);
  if (rc) return rc;
  int* err_flag = C->err_words;
  rc = reset_error_word(C, st);
  if (rc) return rc;
  const bool tensor_leaf = o.precision != KNN_PREC_FP32 && metric != KNN_METRIC_TAXICAB &&
                           d <= 256 && k <= 32;
  Layout lay = single_layout(n, T.depth);
  lay.maxblock = host_max_block(n, T.depth, k);
  {
    knn::SegEntry e{};
    e.n = n;
    e.depth = T.depth;
    lay.tc_group_max = tc_group_max(&e, 1, k, lay.maxleaf);
    lay.own_blocks = leaves_own_blocks(&e, 1, k);
  }
  if (ftab_d) {
    lay.ftable = ftab_d;
    lay.foff = foff_h.data();
    lay.fcount = fcount_h.data();
    lay.maxleaf = leaf;
    lay.tc_group_max = 1;
  }
  cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
  KNN_CK(cudaStreamIsCapturing(st, &cs));
  Shapes sh;
  bool tune_prop = false;
  rc = pick_shapes(C, o, cs == cudaStreamCaptureStatusNone, !tensor_leaf, props, P.X, n, d, P.dpad, k, lay,
                   metric, T.perm, norms, &L, st, &sh, &tune_prop, err_flag);
  if (rc) return rc;
  cudaEvent_t* kev = nullptr;  // per-tree tile-kernel events for the statistics
  if (timed && cs == cudaStreamCaptureStatusNone) {
    kev = C->kernel_events(trees);
    if (!kev) return fail_cuda(cudaGetLastError(), "event creation");
  }
  if (tensor_leaf) {
    rc = run_leaf_umma(C, P.X, n, d, P.dpad, k, trees, lay, metric, o.precision, T.perm, norms, &L, err_flag, st,
                       log, kev, sh.tc_group);
  } else {
    rc = run_leaf(C, P.X, n, d, P.dpad, k, trees, lay, metric, T.perm, norms, &L, stats ? counters : nullptr, st,
                  log, sh.leaf_tile, kev, sh.sparse, sh.pairs);
  }
  if (rc) return rc;
  if (tune_prop) {
    rc = finish_prop_tuning(C, o, P.X, n, d, P.dpad, k, metric, norms, T.perm, &L, lay.maxleaf, st, &sh);
    if (rc) return rc;
  }
  if (timed) KNN_CK(cudaEventRecord(C->ev[3], st));

  for (int p = 0; p < props; ++p) {
    rc = run_prop(P.X, n, d, P.dpad, k, metric, norms, T.perm, &L, true,
                  stats ? counters + 2 + p : nullptr, st, log, sh.prop_warps, P.Xh, P.ldh);
    if (rc) return rc;
  }
  if (timed) KNN_CK(cudaEventRecord(C->ev[4], st));

  // Finalise into the caller's buffers (or staging, then copy to the host).
  float* dd = out_dist;
  int32_t* di = out_idx;
  if (!o.outputs_on_device) {
    rc = C->get("out_dist", (size_t)n * k, &dd);
    if (!rc) rc = C->get("out_idx", (size_t)n * k, &di);
    if (rc) return rc;
  }
  // raw keys: no sqrt (the TAXICAB transform is the identity)
  knn::launch_finalize(L.key[L.cur], L.id[L.cur], n, k, o.raw_keys ? KNN_METRIC_TAXICAB : metric, dd, di, st);
  log.add();
  if (!o.outputs_on_device) {
    KNN_CK(cudaMemcpyAsync(out_dist, dd, sizeof(float) * (size_t)n * k, cudaMemcpyDeviceToHost, st));
    KNN_CK(cudaMemcpyAsync(out_idx, di, sizeof(int32_t) * (size_t)n * k, cudaMemcpyDeviceToHost, st));
  }
  if (timed) KNN_CK(cudaEventRecord(C->ev[5], st));
  KNN_CK(cudaPeekAtLastError());

  const bool async_ok = o.stream && o.outputs_on_device && !stats;
  if (!async_ok) {
    KNN_CK(cudaStreamSynchronize(st));
    rc = check_error_words(C);
    if (rc) return rc;
  }

  if (stats) {
    const int32_t sz = stats->struct_size;
    std::memset(stats, 0, sizeof(knn_stats));
    stats->struct_size = sz;
    stats->depth = T.depth;
    float ms = 0;
    KNN_CK(cudaEventElapsedTime(&ms, C->ev[0], C->ev[5]));
    stats->ms_total = ms;
    KNN_CK(cudaEventElapsedTime(&ms, C->ev[0], C->ev[1]));
    stats->ms_upload = ms;
    if (o.learned_splits) {
      KNN_CK(cudaEventElapsedTime(&ms, C->ev[1], C->ev[6]));
      stats->ms_learn = ms;
      KNN_CK(cudaEventElapsedTime(&ms, C->ev[6], C->ev[2]));
    } else {
      KNN_CK(cudaEventElapsedTime(&ms, C->ev[1], C->ev[2]));
    }
    stats->ms_trees = ms;
    KNN_CK(cudaEventElapsedTime(&ms, C->ev[2], C->ev[3]));
    stats->ms_leaf = ms;
    KNN_CK(cudaEventElapsedTime(&ms, C->ev[3], C->ev[4]));
    stats->ms_propagate = ms;
    KNN_CK(cudaEventElapsedTime(&ms, C->ev[4], C->ev[5]));
    stats->ms_download = ms;
    if (kev) {
      float sum = 0;
      for (int t = 0; t < trees; ++t) {
        KNN_CK(cudaEventElapsedTime(&ms, kev[2 * t], kev[2 * t + 1]));
        sum += ms;
      }
      stats->ms_leaf_tiles = sum;
    }
    stats->launches = log.count;
    stats->props_run = props;
    stats->leaf_tile = tensor_leaf ? 128 : (sh.leaf_tile ? sh.leaf_tile : 64);
    stats->leaf_path = tensor_leaf ? o.precision : 0;
    stats->tc_group = tensor_leaf ? std::min(std::max(sh.tc_group, 1), lay.tc_group_max) : 0;
    stats->leaf_fallback = (o.precision != KNN_PREC_FP32 && !tensor_leaf) ? 1 : 0;
    stats->sparse_dims = (!tensor_leaf && sh.sparse) ? 1 : 0;
    stats->tile_pairs = (!tensor_leaf && sh.pairs) ? 1 : 0;
    stats->prop_warps = sh.prop_warps;
    unsigned long long host[2 + KNN_MAX_PROPS];
    KNN_CK(cudaMemcpy(host, counters, sizeof(host), cudaMemcpyDeviceToHost));
    stats->leaf_pairs = (int64_t)host[0];
    for (int p = 0; p < props && p < KNN_MAX_PROPS; ++p) stats->prop_candidates[p] = (int64_t)host[2 + p];
  }
  return KNN_OK;
}

// ------------------------------------------------------------------ batch --
// Rows of one point set into the concatenated float32 array (dst already
// offset), zero padded to dpad.
int upload_rows(knn_context* C, const void* src, int64_t n, int d, int dtype, bool on_device, float* dst,
                int dpad, cudaStream_t st, knn::LaunchLog& log) {
  if (on_device) {
    knn::launch_pad_rows(src, dtype, n, d, d, dst, dpad, st);
    log.add();
    return KNN_OK;
  }
  if (dtype == KNN_F32) {
    KNN_CK(cudaMemcpy2DAsync(dst, (size_t)dpad * 4, src, (size_t)d * 4, (size_t)d * 4, (size_t)n,
                             cudaMemcpyHostToDevice, st));
    if (dpad != d)
      KNN_CK(cudaMemset2DAsync(dst + d, (size_t)dpad * 4, 0, (size_t)(dpad - d) * 4, (size_t)n, st));
    return KNN_OK;
  }
  void* stage = nullptr;
  int rc = C->get("stage", (size_t)n * d * 2, &stage);
  if (rc) return rc;
  KNN_CK(cudaMemcpyAsync(stage, src, (size_t)n * d * 2, cudaMemcpyHostToDevice, st));
  knn::launch_pad_rows(stage, dtype, n, d, d, dst, dpad, st);
  log.add();
  return KNN_OK;
}

// One group of datasets sharing d: concatenated rows, segment table sorted by
// n descending, one launch per stage for all of them.
struct BatchGroup {
  int d = 0, dpad = 0;
  int64_t ntot = 0;
  std::vector<int> order;                 // dataset indices, n descending
  std::vector<knn::SegEntry> hsegs;       // same order
  int64_t leaves = 0, maxleaf = 1;
};

BatchGroup make_group(const knn_dataset* sets, std::vector<int> idx, int d, int leaf) {
  BatchGroup g;
  g.d = d;
  g.dpad = round4(d);
  std::stable_sort(idx.begin(), idx.end(), [&](int a, int b) { return sets[a].n > sets[b].n; });
  g.order = idx;
  for (int i : idx) {
    knn::SegEntry e{};
    e.off = g.ntot;
    e.n = sets[i].n;
    e.seed = sets[i].seed;
    e.depth = knn::tree_depth(e.n, leaf);
    e.leaf_base = g.leaves;
    g.leaves += int64_t(1) << e.depth;
    const int64_t ml = (e.n + (int64_t(1) << e.depth) - 1) >> e.depth;
    if (ml > g.maxleaf) g.maxleaf = ml;
    g.ntot += e.n;
    g.hsegs.push_back(e);
  }
  return g;
}

// The device part of a group's build, from the uploaded rows and table to the
// finalised [ntot][k] lists with local ids.  Stream-ordered launches only
// (no allocation once the buffers exist), so it can be captured.
int group_compute(knn_context* C, const BatchGroup& g, int k, int trees, int props, int metric,
                  const knn_options& o, bool may_tune, const float* X, const knn::SegEntry* dsegs, int32_t* seg_of,
                  float* norms, int* err_flag, float* out_dist, int32_t* out_idx, cudaStream_t st,
                  knn::LaunchLog& log, bool stage_events = false) {
  const int precision = o.precision;
  if (stage_events) KNN_CK(cudaEventRecord(C->ev[1], st));
  const int nseg = (int)g.hsegs.size();
  knn::launch_fill_seg_of(dsegs, nseg, seg_of, st);
  log.add();
  if (metric == KNN_METRIC_COSINE) {
    knn::launch_norms(X, g.ntot, g.d, g.dpad, norms, st);
    log.add();
  }
  knn::SegView view;
  view.table = dsegs;
  view.seg_of = seg_of;
  view.count = nseg;
  view.n0 = g.ntot;
  view.seed0 = 0;
  view.depth0 = 0;
  Trees T;
  int rc = run_trees_segs(C, X, g.ntot, g.d, g.dpad, trees, view, g.hsegs.data(), nseg, st, &T, log);
  if (rc) return rc;
  if (stage_events) KNN_CK(cudaEventRecord(C->ev[2], st));
  Lists L;
  rc = get_lists(C, g.ntot, k, &L);
  if (rc) return rc;
  Layout lay;
  lay.segs = view;
  lay.leaves = g.leaves;
  lay.maxleaf = g.maxleaf;
  for (const auto& e : g.hsegs) lay.maxblock = std::max(lay.maxblock, host_max_block(e.n, e.depth, k));
  lay.tc_group_max = tc_group_max(g.hsegs.data(), (int)g.hsegs.size(), k, g.maxleaf);
  lay.own_blocks = leaves_own_blocks(g.hsegs.data(), (int)g.hsegs.size(), k);
  const bool tensor_leaf = precision != KNN_PREC_FP32 && metric != KNN_METRIC_TAXICAB && g.d <= 256 &&
                           k <= 32;
  Shapes sh;
  bool tune_prop = false;
  rc = pick_shapes(C, o, may_tune, !tensor_leaf, props, X, g.ntot, g.d, g.dpad, k, lay, metric, T.perm, norms, &L,
                   st, &sh, &tune_prop, err_flag);
  if (rc) return rc;
  if (tensor_leaf)
    rc = run_leaf_umma(C, X, g.ntot, g.d, g.dpad, k, trees, lay, metric, precision, T.perm, norms, &L, err_flag,
                       st, log, nullptr, sh.tc_group);
  else
    rc = run_leaf(C, X, g.ntot, g.d, g.dpad, k, trees, lay, metric, T.perm, norms, &L, nullptr, st, log,
                  sh.leaf_tile, nullptr, sh.sparse, sh.pairs);
  if (rc) return rc;
  if (tune_prop) {
    rc = finish_prop_tuning(C, o, X, g.ntot, g.d, g.dpad, k, metric, norms, T.perm, &L, lay.maxleaf, st, &sh);
    if (rc) return rc;
  }
  if (stage_events) KNN_CK(cudaEventRecord(C->ev[3], st));
  for (int p = 0; p < props; ++p) {
    rc = run_prop(X, g.ntot, g.d, g.dpad, k, metric, norms, T.perm, &L, true, nullptr, st, log, sh.prop_warps);
    if (rc) return rc;
  }
  if (stage_events) KNN_CK(cudaEventRecord(C->ev[4], st));
  knn::launch_finalize_local(L.key[L.cur], L.id[L.cur], g.ntot, k, metric, seg_of, dsegs, out_dist, out_idx, st);
  log.add();
  KNN_CK(cudaPeekAtLastError());
  return KNN_OK;
}

std::string group_signature(const BatchGroup& g, int k, int trees, int leaf, int props, int metric,
                            int precision) {
  std::string s = "d" + std::to_string(g.d) + ":k" + std::to_string(k) + ":t" + std::to_string(trees) + ":l" +
                  std::to_string(leaf) + ":p" + std::to_string(props) + ":m" + std::to_string(metric) + ":q" +
                  std::to_string(precision);
  for (const auto& e : g.hsegs) s += ":" + std::to_string(e.n) + "/" + std::to_string(e.seed);
  return s;
}

int batch_impl(knn_context* C, const knn_dataset* sets, int count, int32_t k, int32_t trees, int32_t leaf,
               int32_t props, int32_t metric, const knn_options& o, knn_stats* stats, bool use_graphs) {
  cudaStream_t st = o.stream ? static_cast<cudaStream_t>(o.stream) : C->stream;
  knn::LaunchLog log;
  const bool timed = stats != nullptr;
  if (timed) KNN_CK(cudaEventRecord(C->ev[0], st));
  std::map<int, std::vector<int>> by_d;
  for (int i = 0; i < count; ++i) by_d[sets[i].d].push_back(i);
  int max_depth = 0;
  int* err_flag = C->err_words;
  int rc = reset_error_word(C, st);
  if (rc) return rc;
  cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
  KNN_CK(cudaStreamIsCapturing(st, &cs));
  if (cs != cudaStreamCaptureStatusNone || timed) use_graphs = false;
  float stage_ms[3] = {0, 0, 0};

  for (auto& kv : by_d) {
    const BatchGroup g = make_group(sets, kv.second, kv.first, leaf);
    for (const auto& e : g.hsegs)
      if (e.depth > 30) return fail(KNN_ERR_ARGS, "tree too deep (n / leaf too large)");
    if (g.hsegs[0].depth > max_depth) max_depth = g.hsegs[0].depth;
    const int nseg = (int)g.hsegs.size();
    // buffers (all allocated before anything is captured)
    float *X = nullptr, *norms = nullptr, *od = nullptr;
    int32_t *seg_of = nullptr, *oi = nullptr;
    knn::SegEntry* dsegs = nullptr;
    rc = C->get("bX", (size_t)g.ntot * g.dpad, &X);
    if (!rc) rc = C->get("b_segs", (size_t)nseg, &dsegs);
    if (!rc) rc = C->get("b_seg_of", (size_t)g.ntot, &seg_of);
    if (!rc && metric == KNN_METRIC_COSINE) rc = C->get("norms", (size_t)g.ntot, &norms);
    if (!rc) rc = C->get("b_out_dist", (size_t)g.ntot * k, &od);
    if (!rc) rc = C->get("b_out_idx", (size_t)g.ntot * k, &oi);
    if (rc) return rc;
    // inputs: device sets in one gather launch, host sets by one copy each
    if (o.points_on_device) {
      std::vector<knn::RowSource> src(g.order.size());
      for (size_t a = 0; a < g.order.size(); ++a)
        src[a] = {sets[g.order[a]].points, g.hsegs[a].n, g.hsegs[a].off};
      knn::RowSource* dsrc = nullptr;
      rc = C->get("b_src", src.size(), &dsrc);
      if (rc) return rc;
      KNN_CK(cudaMemcpyAsync(dsrc, src.data(), sizeof(knn::RowSource) * src.size(), cudaMemcpyHostToDevice, st));
      knn::launch_gather_sets(dsrc, (int)src.size(), o.dtype, g.d, X, g.dpad, st);
      log.add();
    } else {
      for (size_t a = 0; a < g.order.size(); ++a) {
        const knn_dataset& ds = sets[g.order[a]];
        rc = upload_rows(C, ds.points, ds.n, g.d, o.dtype, false, X + (size_t)g.hsegs[a].off * g.dpad, g.dpad, st,
                         log);
        if (rc) return rc;
      }
    }
    KNN_CK(cudaMemcpyAsync(dsegs, g.hsegs.data(), sizeof(knn::SegEntry) * nseg, cudaMemcpyHostToDevice, st));
    // compute: replay a captured graph of this shape, capture it on its second
    // sighting, or launch directly
    const std::string sig = use_graphs ? group_signature(g, k, trees, leaf, props, metric, o.precision) : "";
    bool done = false;
    if (use_graphs) {
      for (auto& cg : C->graphs)
        if (cg.sig == sig && cg.generation == C->generation) {
          KNN_CK(cudaGraphLaunch(cg.exec, st));
          log.add(1);
          done = true;
          break;
        }
      if (!done && std::find(C->seen.begin(), C->seen.end(), sig) != C->seen.end()) {
        const uint64_t gen0 = C->generation;
        knn::LaunchLog glog;
        cudaGraph_t graph = nullptr;
        cudaGraphExec_t exec = nullptr;
        KNN_CK(cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal));
        const int crc = group_compute(C, g, k, trees, props, metric, o, false, X, dsegs, seg_of, norms,
                                      err_flag, od, oi, st, glog);
        cudaError_t e = cudaStreamEndCapture(st, &graph);
        if (crc == KNN_OK && e == cudaSuccess && C->generation == gen0) e = cudaGraphInstantiate(&exec, graph, 0);
        else if (e == cudaSuccess) e = cudaErrorStreamCaptureInvalidated;
        if (graph) cudaGraphDestroy(graph);
        cudaGetLastError();
        if (e == cudaSuccess) {
          // drop captures whose buffers have moved since, keep at most 16
          std::vector<knn_context::Captured> keep;
          for (auto& cg : C->graphs) {
            if (cg.generation == C->generation && keep.size() < 15) keep.push_back(cg);
            else cudaGraphExecDestroy(cg.exec);
          }
          C->graphs.swap(keep);
          C->graphs.push_back({sig, C->generation, exec});
          KNN_CK(cudaGraphLaunch(exec, st));
          log.add(1);
          done = true;
        }
      }
      if (!done && std::find(C->seen.begin(), C->seen.end(), sig) == C->seen.end()) {
        if (C->seen.size() >= 64) C->seen.erase(C->seen.begin());
        C->seen.push_back(sig);
      }
    }
    if (!done) {
      rc = group_compute(C, g, k, trees, props, metric, o, cs == cudaStreamCaptureStatusNone, X, dsegs, seg_of,
                         norms, err_flag, od, oi, st, log, timed);
      if (rc) return rc;
      if (timed) {  // stage times summed over the groups
        float a = 0, b = 0, c = 0;
        KNN_CK(cudaEventSynchronize(C->ev[4]));
        KNN_CK(cudaEventElapsedTime(&a, C->ev[1], C->ev[2]));
        KNN_CK(cudaEventElapsedTime(&b, C->ev[2], C->ev[3]));
        KNN_CK(cudaEventElapsedTime(&c, C->ev[3], C->ev[4]));
        stage_ms[0] += a;
        stage_ms[1] += b;
        stage_ms[2] += c;
      }
    }
    // outputs
    const cudaMemcpyKind kind = o.outputs_on_device ? cudaMemcpyDeviceToDevice : cudaMemcpyDeviceToHost;
    for (size_t a = 0; a < g.order.size(); ++a) {
      const knn_dataset& ds = sets[g.order[a]];
      const size_t off = (size_t)g.hsegs[a].off * k, cnt = (size_t)ds.n * k;
      KNN_CK(cudaMemcpyAsync(ds.out_dist, od + off, sizeof(float) * cnt, kind, st));
      KNN_CK(cudaMemcpyAsync(ds.out_idx, oi + off, sizeof(int32_t) * cnt, kind, st));
    }
  }
  if (timed) KNN_CK(cudaEventRecord(C->ev[5], st));
  const bool async_ok = o.stream && o.outputs_on_device && !stats;
  if (!async_ok) {
    KNN_CK(cudaStreamSynchronize(st));
    rc = check_error_words(C);
    if (rc) return rc;
  }
  if (stats) {
    const int32_t sz = stats->struct_size;
    std::memset(stats, 0, sizeof(knn_stats));
    stats->struct_size = sz;
    stats->depth = max_depth;
    float ms = 0;
    KNN_CK(cudaEventElapsedTime(&ms, C->ev[0], C->ev[5]));
    stats->ms_total = ms;
    stats->ms_trees = stage_ms[0];
    stats->ms_leaf = stage_ms[1];
    stats->ms_propagate = stage_ms[2];
    stats->launches = log.count;
    stats->props_run = props;
    // per group of equal d: tensor-core tiles when the request allows them
    for (const auto& kv : by_d) {
      const bool tc = o.precision != KNN_PREC_FP32 && metric != KNN_METRIC_TAXICAB && kv.first <= 256 && k <= 32;
      if (tc) stats->leaf_path = o.precision;
      if (o.precision != KNN_PREC_FP32 && !tc) stats->leaf_fallback = 1;
    }
  }
  return KNN_OK;
}

}  // namespace

extern "C" {

void knn_default_options(knn_options* opt) {
  if (!opt) return;
  std::memset(opt, 0, sizeof(*opt));
  opt->struct_size = (int32_t)sizeof(knn_options);
  opt->device = -1;
  opt->dtype = KNN_F32;
  opt->precision = KNN_PREC_FP32;
}

int knn_version(void) { return 100; }

int knn_device_capability(int32_t device, int32_t* major, int32_t* minor) {
  if (!major || !minor) return fail(KNN_ERR_ARGS, "NULL pointer");
  int count = 0;
  cudaError_t e = cudaGetDeviceCount(&count);
  if (e != cudaSuccess || count == 0) {
    cudaGetLastError();
    return fail(KNN_ERR_NO_DEVICE, "no CUDA device");
  }
  if (device < 0 || device >= count) return fail(KNN_ERR_ARGS, "device ordinal out of range");
  cudaDeviceProp p;
  e = cudaGetDeviceProperties(&p, device);
  if (e != cudaSuccess) return fail_cuda(e, "cudaGetDeviceProperties");
  *major = p.major;
  *minor = p.minor;
  return KNN_OK;
}

const char* knn_status_string(int status) {
  switch (status) {
    case KNN_OK: return "ok";
    case KNN_ERR_ARGS: return "invalid argument";
    case KNN_ERR_N_LE_K: return "n must exceed k";
    case KNN_ERR_OOM: return "out of memory";
    case KNN_ERR_CUDA: return "CUDA error";
    case KNN_ERR_TIMEOUT: return "device wait timed out";
    case KNN_ERR_UNSUPPORTED: return "unsupported request";
    case KNN_ERR_NO_DEVICE: return "no CUDA device";
    default: return "unknown status";
  }
}

const char* knn_last_error(void) { return g_last_error.c_str(); }

knn_context* knn_context_create(int32_t device) {
  knn_context* c = nullptr;
  if (make_context(device, &c)) return nullptr;
  return c;
}

void knn_context_destroy(knn_context* ctx) { delete ctx; }

int64_t knn_context_scratch_bytes(const knn_context* ctx) { return ctx ? ctx->bytes_held() : 0; }

int knn_context_status(knn_context* ctx, void* stream) {
  knn_options o;
  knn_default_options(&o);
  int rc = enter_device(&ctx, o);
  if (rc) return rc;
  KNN_CK(cudaStreamSynchronize(stream ? static_cast<cudaStream_t>(stream) : ctx->stream));
  return check_error_words(ctx);
}

int knn_test_fail_next_tile_wait(knn_context* ctx) {
  knn_options o;
  knn_default_options(&o);
  int rc = enter_device(&ctx, o);
  if (rc) return rc;
  ctx->preset_err = true;
  return KNN_OK;
}

int knn_build(const void* points, int64_t n, int32_t d, int32_t k, int32_t trees, int32_t leaf,
              int32_t props, int32_t metric, uint64_t seed, int32_t* out_idx, float* out_dist) {
  return knn_build_ex(nullptr, points, n, d, k, trees, leaf, props, metric, seed, out_idx,
                      out_dist, nullptr, nullptr);
}

int knn_build_ex(knn_context* ctx, const void* points, int64_t n, int32_t d, int32_t k,
                 int32_t trees, int32_t leaf, int32_t props, int32_t metric, uint64_t seed,
                 int32_t* out_idx, float* out_dist, const knn_options* opt, knn_stats* stats) {
  knn_options o;
  int rc = resolve_options(opt, &o);
  if (rc) return rc;
  rc = check_common(points, n, d, k, metric);
  if (rc) return rc;
  if (!out_idx || !out_dist) return fail(KNN_ERR_ARGS, "output pointer is NULL");
  if (trees < 1 || leaf < 1) return fail(KNN_ERR_ARGS, "trees and leaf must be >= 1");
  if (props < 0 || props > KNN_MAX_PROPS) return fail(KNN_ERR_ARGS, "props out of range");
  if (stats && stats->struct_size != (int32_t)sizeof(knn_stats))
    return fail(KNN_ERR_ARGS, "knn_stats.struct_size mismatch");
  rc = enter_device(&ctx, o);
  if (rc) return rc;
  return build_impl(ctx, points, n, d, k, trees, leaf, props, metric, seed, out_idx, out_dist, o,
                    stats);
}

int knn_build_batch(knn_context* ctx, const knn_dataset* sets, int32_t count, int32_t k, int32_t trees,
                    int32_t leaf, int32_t props, int32_t metric, const knn_options* opt, knn_stats* stats) {
  knn_options o;
  int rc = resolve_options(opt, &o);
  if (rc) return rc;
  if (!sets || count < 1) return fail(KNN_ERR_ARGS, "no datasets");
  if (k < 1 || k > KNN_MAX_K) return fail(KNN_ERR_ARGS, "k must be in 1..KNN_MAX_K");
  if (metric < 0 || metric > 2) return fail(KNN_ERR_ARGS, "unknown metric");
  if (trees < 1 || leaf < 1) return fail(KNN_ERR_ARGS, "trees and leaf must be >= 1");
  if (props < 0 || props > KNN_MAX_PROPS) return fail(KNN_ERR_ARGS, "props out of range");
  if (o.ld != 0) return fail(KNN_ERR_ARGS, "batches take contiguous rows (options.ld must be 0)");
  if (o.learned_splits) return fail(KNN_ERR_UNSUPPORTED, "learned splits are not available for batches");
  if (o.split_rule != 0) return fail(KNN_ERR_UNSUPPORTED, "reference-rule splits are not available for batches");
  if (stats && stats->struct_size != (int32_t)sizeof(knn_stats))
    return fail(KNN_ERR_ARGS, "knn_stats.struct_size mismatch");
  std::map<int, int64_t> per_d;
  for (int32_t i = 0; i < count; ++i) {
    const knn_dataset& ds = sets[i];
    if (!ds.points || !ds.out_idx || !ds.out_dist) return fail(KNN_ERR_ARGS, "dataset pointer is NULL");
    if (ds.d < 1) return fail(KNN_ERR_ARGS, "dataset d must be >= 1");
    if (ds.n < 1 || ds.n >= (int64_t)INT32_MAX) return fail(KNN_ERR_ARGS, "dataset n out of range");
    if (ds.n <= k) return fail(KNN_ERR_N_LE_K, "a dataset has n <= k");
    per_d[ds.d] += ds.n;
    if (per_d[ds.d] >= (int64_t)INT32_MAX) return fail(KNN_ERR_ARGS, "too many points of one d in the batch");
  }
  rc = enter_device(&ctx, o);
  if (rc) return rc;
  return batch_impl(ctx, sets, count, k, trees, leaf, props, metric, o, stats, true);
}

int knn_build_trees(knn_context* ctx, const float* points, int64_t n, int32_t d, int32_t trees,
                    int32_t leaf, uint64_t seed, int32_t* out_perm) {
  if (!points || !out_perm) return fail(KNN_ERR_ARGS, "NULL pointer");
  if (n < 1 || n >= (int64_t)INT32_MAX || d < 1 || trees < 1 || leaf < 1)
    return fail(KNN_ERR_ARGS, "size out of range");
  knn_options o;
  knn_default_options(&o);
  int rc = enter_device(&ctx, o);
  if (rc) return rc;
  cudaStream_t st = ctx->stream;
  knn::LaunchLog log;
  Prepared P;
  rc = prepare_points(ctx, points, n, d, o, st, &P, log);
  if (rc) return rc;
  Trees T;
  rc = run_trees(ctx, P.X, n, d, P.dpad, trees, leaf, seed, st, &T, log);
  if (rc) return rc;
  KNN_CK(cudaMemcpyAsync(out_perm, T.perm, sizeof(int32_t) * (size_t)trees * n, cudaMemcpyDeviceToHost, st));
  KNN_CK(cudaStreamSynchronize(st));
  return KNN_OK;
}

int knn_leaf_stage(knn_context* ctx, const float* points, int64_t n, int32_t d, int32_t k,
                   int32_t trees, int32_t leaf, int32_t metric, const int32_t* perm,
                   int32_t* out_idx, float* out_key) {
  int rc = check_common(points, n, d, k, metric);
  if (rc) return rc;
  if (!perm || !out_idx || !out_key || trees < 1 || leaf < 1) return fail(KNN_ERR_ARGS, "bad argument");
  const int depth = knn::tree_depth(n, leaf);
  if (depth > 30) return fail(KNN_ERR_ARGS, "tree too deep");
  knn_options o;
  knn_default_options(&o);
  rc = enter_device(&ctx, o);
  if (rc) return rc;
  cudaStream_t st = ctx->stream;
  knn::LaunchLog log;
  Prepared P;
  rc = prepare_points(ctx, points, n, d, o, st, &P, log);
  if (rc) return rc;
  int32_t* dperm = nullptr;
  rc = ctx->get("perm", (size_t)trees * n, &dperm);
  if (rc) return rc;
  KNN_CK(cudaMemcpyAsync(dperm, perm, sizeof(int32_t) * (size_t)trees * n, cudaMemcpyHostToDevice, st));
  float* norms = nullptr;
  if (metric == KNN_METRIC_COSINE) {
    rc = ctx->get("norms", (size_t)n, &norms);
    if (rc) return rc;
    knn::launch_norms(P.X, n, d, P.dpad, norms, st);
  }
  Lists L;
  rc = get_lists(ctx, n, k, &L);
  if (rc) return rc;
  rc = run_leaf(ctx, P.X, n, d, P.dpad, k, trees, single_layout(n, depth), metric, dperm, norms, &L, nullptr, st,
                log);
  if (rc) return rc;
  KNN_CK(cudaMemcpyAsync(out_key, L.key[L.cur], sizeof(float) * (size_t)n * k, cudaMemcpyDeviceToHost, st));
  int32_t* di = nullptr;
  rc = ctx->get("out_idx", (size_t)n * k, &di);
  if (rc) return rc;
  float* dd = nullptr;
  rc = ctx->get("out_dist", (size_t)n * k, &dd);
  if (rc) return rc;
  knn::launch_finalize(L.key[L.cur], L.id[L.cur], n, k, metric, dd, di, st);
  KNN_CK(cudaMemcpyAsync(out_idx, di, sizeof(int32_t) * (size_t)n * k, cudaMemcpyDeviceToHost, st));
  KNN_CK(cudaStreamSynchronize(st));
  return KNN_OK;
}

int knn_propagate_step(knn_context* ctx, const float* points, int64_t n, int32_t d, int32_t k,
                       int32_t metric, const int32_t* idx_in, const float* key_in,
                       int32_t* idx_out, float* key_out) {
  int rc = check_common(points, n, d, k, metric);
  if (rc) return rc;
  if (!idx_in || !key_in || !idx_out || !key_out) return fail(KNN_ERR_ARGS, "NULL pointer");
  for (int64_t g = 0; g < n * k; ++g)
    if (idx_in[g] < 0 || idx_in[g] >= n) return fail(KNN_ERR_ARGS, "neighbour id out of range");
  knn_options o;
  knn_default_options(&o);
  rc = enter_device(&ctx, o);
  if (rc) return rc;
  cudaStream_t st = ctx->stream;
  knn::LaunchLog log;
  Prepared P;
  rc = prepare_points(ctx, points, n, d, o, st, &P, log);
  if (rc) return rc;
  float* norms = nullptr;
  if (metric == KNN_METRIC_COSINE) {
    rc = ctx->get("norms", (size_t)n, &norms);
    if (rc) return rc;
    knn::launch_norms(P.X, n, d, P.dpad, norms, st);
  }
  Lists L;
  rc = get_lists(ctx, n, k, &L);
  if (rc) return rc;
  KNN_CK(cudaMemcpyAsync(L.key[0], key_in, sizeof(float) * (size_t)n * k, cudaMemcpyHostToDevice, st));
  KNN_CK(cudaMemcpyAsync(L.id[0], idx_in, sizeof(int32_t) * (size_t)n * k, cudaMemcpyHostToDevice, st));
  rc = run_prop(P.X, n, d, P.dpad, k, metric, norms, nullptr, &L, false, nullptr, st, log);
  if (rc) return rc;
  int32_t* di = nullptr;
  rc = ctx->get("out_idx", (size_t)n * k, &di);
  if (rc) return rc;
  float* dd = nullptr;
  rc = ctx->get("out_dist", (size_t)n * k, &dd);
  if (rc) return rc;
  // ids without flag bits; keys as they are
  knn::launch_finalize(L.key[L.cur], L.id[L.cur], n, k, KNN_METRIC_TAXICAB, dd, di, st);
  KNN_CK(cudaMemcpyAsync(key_out, dd, sizeof(float) * (size_t)n * k, cudaMemcpyDeviceToHost, st));
  KNN_CK(cudaMemcpyAsync(idx_out, di, sizeof(int32_t) * (size_t)n * k, cudaMemcpyDeviceToHost, st));
  KNN_CK(cudaStreamSynchronize(st));
  return KNN_OK;
}

int knn_exact_fp64(knn_context* ctx, const void* points, int64_t n, int32_t d, int32_t k,
                   int32_t metric, const int64_t* queries, int64_t nq, int32_t* out_idx,
                   double* out_dist, const knn_options* opt) {
  knn_options o;
  int rc = resolve_options(opt, &o);
  if (rc) return rc;
  rc = check_common(points, n, d, k, metric);
  if (rc) return rc;
  if (!queries || nq < 1 || !out_idx || !out_dist) return fail(KNN_ERR_ARGS, "bad query arguments");
  for (int64_t q = 0; q < nq; ++q)
    if (queries[q] < 0 || queries[q] >= n) return fail(KNN_ERR_ARGS, "query id out of range");
  rc = enter_device(&ctx, o);
  if (rc) return rc;
  cudaStream_t st = o.stream ? static_cast<cudaStream_t>(o.stream) : ctx->stream;
  knn::LaunchLog log;
  knn_options po = o;
  po.outputs_on_device = 0;
  Prepared P;
  rc = prepare_points(ctx, points, n, d, po, st, &P, log);
  if (rc) return rc;
  int dev_sms = 148;
  cudaDeviceGetAttribute(&dev_sms, cudaDevAttrMultiProcessorCount, ctx->device);
  const int64_t qtiles = (nq + 63) / 64;
  int slices = (int)((4LL * dev_sms + qtiles - 1) / qtiles);
  if (slices < 1) slices = 1;
  if (slices > 64) slices = 64;
  if ((int64_t)slices > (n + 63) / 64) slices = (int)((n + 63) / 64);
  int64_t* dq = nullptr;
  double* norms = nullptr;
  double* pd = nullptr;
  uint32_t* pi = nullptr;
  double* od = nullptr;
  int32_t* oi = nullptr;
  rc = ctx->get("ex_q", (size_t)nq, &dq);
  if (!rc) rc = ctx->get("ex_norms", (size_t)n, &norms);
  if (!rc) rc = ctx->get("ex_pd", (size_t)slices * nq * k, &pd);
  if (!rc) rc = ctx->get("ex_pi", (size_t)slices * nq * k, &pi);
  if (!rc) rc = ctx->get("ex_od", (size_t)nq * k, &od);
  if (!rc) rc = ctx->get("ex_oi", (size_t)nq * k, &oi);
  if (rc) return rc;
  KNN_CK(cudaMemcpyAsync(dq, queries, sizeof(int64_t) * (size_t)nq, cudaMemcpyHostToDevice, st));
  rc = knn::exact_fp64(P.X, n, d, P.dpad, k, metric, dq, nq, norms, pd, pi, slices, od, oi, st);
  if (rc) return fail_cuda(cudaGetLastError(), "exact launch");
  KNN_CK(cudaMemcpyAsync(out_dist, od, sizeof(double) * (size_t)nq * k, cudaMemcpyDeviceToHost, st));
  KNN_CK(cudaMemcpyAsync(out_idx, oi, sizeof(int32_t) * (size_t)nq * k, cudaMemcpyDeviceToHost, st));
  KNN_CK(cudaStreamSynchronize(st));
  return KNN_OK;
}

int knn_normalize_reference(float* points, int64_t n, int32_t d) {
  if (!points || n < 1 || d < 1) return fail(KNN_ERR_ARGS, "bad argument");
  knn_context* ctx = nullptr;
  knn_options o;
  knn_default_options(&o);
  int rc = enter_device(&ctx, o);
  if (rc) return rc;
  float* X = nullptr;
  rc = ctx->get("norm_X", (size_t)n * d, &X);
  if (rc) return rc;
  cudaStream_t st = ctx->stream;
  KNN_CK(cudaMemcpyAsync(X, points, sizeof(float) * (size_t)n * d, cudaMemcpyHostToDevice, st));
  knn::launch_normalize_reference(X, n, d, st);
  KNN_CK(cudaPeekAtLastError());
  KNN_CK(cudaMemcpyAsync(points, X, sizeof(float) * (size_t)n * d, cudaMemcpyDeviceToHost, st));
  KNN_CK(cudaStreamSynchronize(st));
  return KNN_OK;
}

int knn_merge_lists(knn_context* ctx, const int32_t* idx, const float* key, int32_t lists, int64_t n, int32_t k,
                    int32_t metric, int32_t as_distance, int32_t* idx_out, float* key_out,
                    const knn_options* opt) {
  knn_options o;
  int rc = resolve_options(opt, &o);
  if (rc) return rc;
  if (!idx || !key || !idx_out || !key_out) return fail(KNN_ERR_ARGS, "NULL pointer");
  if (lists < 1 || n < 1 || n >= (int64_t)INT32_MAX || k < 1 || k > KNN_MAX_K)
    return fail(KNN_ERR_ARGS, "size out of range");
  if (metric < 0 || metric > 2 || as_distance < 0 || as_distance > 1) return fail(KNN_ERR_ARGS, "bad metric or mode");
  rc = enter_device(&ctx, o);
  if (rc) return rc;
  cudaStream_t st = o.stream ? static_cast<cudaStream_t>(o.stream) : ctx->stream;
  const size_t in = (size_t)lists * n * k, out = (size_t)n * k;
  const int32_t* di = idx;
  const float* dk = key;
  int32_t* oi = idx_out;
  float* ok = key_out;
  if (!o.points_on_device) {
    int32_t* ti = nullptr;
    float* tk = nullptr;
    rc = ctx->get("ml_in_idx", in, &ti);
    if (!rc) rc = ctx->get("ml_in_key", in, &tk);
    if (!rc) rc = ctx->get("ml_out_idx", out, &oi);
    if (!rc) rc = ctx->get("ml_out_key", out, &ok);
    if (rc) return rc;
    KNN_CK(cudaMemcpyAsync(ti, idx, sizeof(int32_t) * in, cudaMemcpyHostToDevice, st));
    KNN_CK(cudaMemcpyAsync(tk, key, sizeof(float) * in, cudaMemcpyHostToDevice, st));
    di = ti;
    dk = tk;
  }
  knn::launch_merge_lists(di, dk, lists, n, k, oi, ok, st);
  if (as_distance) {  // keys -> distances (ids without flag bits already)
    knn::launch_finalize(ok, reinterpret_cast<const uint32_t*>(oi), n, k, metric, ok, oi, st);
  }
  KNN_CK(cudaPeekAtLastError());
  if (!o.points_on_device) {
    KNN_CK(cudaMemcpyAsync(idx_out, oi, sizeof(int32_t) * out, cudaMemcpyDeviceToHost, st));
    KNN_CK(cudaMemcpyAsync(key_out, ok, sizeof(float) * out, cudaMemcpyDeviceToHost, st));
  }
  KNN_CK(cudaStreamSynchronize(st));
  return KNN_OK;
}

int knn_propagate_range(knn_context* ctx, const void* points, int64_t n, int32_t d, int32_t k, int32_t metric,
                        int64_t r0, int64_t r1, const int32_t* idx_in, const float* key_in,
                        const uint32_t* flags_in, int32_t* idx_out, float* key_out, uint32_t* flags_out,
                        const knn_options* opt) {
  knn_options o;
  int rc = resolve_options(opt, &o);
  if (rc) return rc;
  rc = check_common(points, n, d, k, metric);
  if (rc) return rc;
  if (!idx_in || !key_in || !idx_out || !key_out || !flags_out) return fail(KNN_ERR_ARGS, "NULL pointer");
  if (r0 < 0 || r1 > n || r0 > r1) return fail(KNN_ERR_ARGS, "point range out of bounds");
  rc = enter_device(&ctx, o);
  if (rc) return rc;
  cudaStream_t st = o.stream ? static_cast<cudaStream_t>(o.stream) : ctx->stream;
  knn::LaunchLog log;
  Prepared P;
  rc = prepare_points(ctx, points, n, d, o, st, &P, log);
  if (rc) return rc;
  float* norms = nullptr;
  if (metric == KNN_METRIC_COSINE) {
    rc = ctx->get("norms", (size_t)n, &norms);
    if (rc) return rc;
    knn::launch_norms(P.X, n, d, P.dpad, norms, st);
  }
  if (r1 > r0) {
    knn::PropArgs a{};
    a.X = P.X;
    a.Xh = P.Xh;
    a.ldh = P.ldh;
    a.n = n;
    a.d = d;
    a.dpad = P.dpad;
    a.k = k;
    a.metric = metric;
    a.norms = norms;
    a.order = nullptr;
    a.key_in = key_in;
    a.id_in = reinterpret_cast<const uint32_t*>(idx_in);
    a.flags_in = flags_in;
    a.key_out = key_out;
    a.id_out = reinterpret_cast<uint32_t*>(idx_out);
    a.flags_out = flags_out;
    a.r0 = r0;
    a.r1 = r1;
    a.warps = o.prop_warps;
    a.stream = st;
    rc = knn::propagate_step(a, log);
    if (rc == KNN_ERR_UNSUPPORTED) return fail(rc, "propagation scratch exceeds shared memory (k or d too large)");
    if (rc) return fail_cuda(cudaGetLastError(), "propagation launch");
  }
  KNN_CK(cudaStreamSynchronize(st));
  return KNN_OK;
}

int64_t knn_mlp_param_count(int32_t d) {
  if (d < 1) return fail(KNN_ERR_ARGS, "d must be >= 1");
  return (int64_t)knn::mlp_param_count(d);
}

int knn_mlp_loss_grad(const float* params, int32_t d, const float* rows, int32_t batch, float margin,
                      float* grad, float* loss) {
  if (!params || !rows || !grad || !loss) return fail(KNN_ERR_ARGS, "NULL pointer");
  if (d < 1 || batch < 1) return fail(KNN_ERR_ARGS, "d and batch must be >= 1");
  knn_context* ctx = nullptr;
  knn_options o;
  knn_default_options(&o);
  int rc = enter_device(&ctx, o);
  if (rc) return rc;
  cudaStream_t st = ctx->stream;
  knn::LaunchLog log;
  const size_t np = knn::mlp_param_count(d);
  const size_t nr = (size_t)3 * batch * d;
  float *dp = nullptr, *dr = nullptr, *dg = nullptr, *ws = nullptr, *dl = nullptr;
  rc = ctx->get("mlpg_params", np, &dp);
  if (!rc) rc = ctx->get("mlpg_rows", nr, &dr);
  if (!rc) rc = ctx->get("mlpg_grad", np, &dg);
  if (!rc) rc = ctx->get("mlpg_ws", knn::mlp_fwd_bwd_ws_floats(d, batch), &ws);
  if (!rc) rc = ctx->get("mlpg_loss", 1, &dl);
  if (rc) return rc;
  KNN_CK(cudaMemcpyAsync(dp, params, sizeof(float) * np, cudaMemcpyHostToDevice, st));
  KNN_CK(cudaMemcpyAsync(dr, rows, sizeof(float) * nr, cudaMemcpyHostToDevice, st));
  KNN_CK(cudaMemsetAsync(dl, 0, sizeof(float), st));
  rc = knn::mlp_loss_grad(dp, d, dr, batch, margin, dg, ws, dl, st, log);
  if (rc) return fail_cuda(cudaGetLastError(), "learned split gradient launch");
  KNN_CK(cudaMemcpyAsync(grad, dg, sizeof(float) * np, cudaMemcpyDeviceToHost, st));
  KNN_CK(cudaMemcpyAsync(loss, dl, sizeof(float), cudaMemcpyDeviceToHost, st));
  KNN_CK(cudaStreamSynchronize(st));
  return KNN_OK;
}

int knn_mlp_train(knn_context* ctx, const void* points, int64_t n, int32_t d, int32_t k, int32_t metric,
                  uint64_t seed, const knn_options* opt, float* params, float* mean, float* inv_std,
                  float* loss_curve) {
  knn_options o;
  int rc = resolve_options(opt, &o);
  if (rc) return rc;
  rc = check_common(points, n, d, k, metric);
  if (rc) return rc;
  if (!params || !mean || !inv_std) return fail(KNN_ERR_ARGS, "output pointer is NULL");
  rc = enter_device(&ctx, o);
  if (rc) return rc;
  cudaStream_t st = o.stream ? static_cast<cudaStream_t>(o.stream) : ctx->stream;
  knn::LaunchLog log;
  Prepared P;
  rc = prepare_points(ctx, points, n, d, o, st, &P, log);
  if (rc) return rc;
  Learned Lr;
  rc = learn_network(ctx, P.X, n, d, P.dpad, k, metric, seed, o, st, &Lr, log);
  if (rc) return rc;
  KNN_CK(cudaMemcpyAsync(params, Lr.params, sizeof(float) * knn::mlp_param_count(d), cudaMemcpyDeviceToHost, st));
  KNN_CK(cudaMemcpyAsync(mean, Lr.mean, sizeof(float) * (size_t)d, cudaMemcpyDeviceToHost, st));
  KNN_CK(cudaMemcpyAsync(inv_std, Lr.inv_std, sizeof(float) * (size_t)d, cudaMemcpyDeviceToHost, st));
  if (loss_curve)
    KNN_CK(cudaMemcpyAsync(loss_curve, Lr.loss, sizeof(float) * (size_t)Lr.steps, cudaMemcpyDeviceToHost, st));
  KNN_CK(cudaStreamSynchronize(st));
  return KNN_OK;
}

int knn_mlp_embed(knn_context* ctx, const void* points, int64_t n, int32_t d, int32_t metric,
                  const float* params, const float* mean, const float* inv_std, const knn_options* opt,
                  float* out) {
  knn_options o;
  int rc = resolve_options(opt, &o);
  if (rc) return rc;
  if (!points || !params || !mean || !inv_std || !out) return fail(KNN_ERR_ARGS, "NULL pointer");
  if (n < 1 || n >= (int64_t)INT32_MAX || d < 1) return fail(KNN_ERR_ARGS, "size out of range");
  if (metric < 0 || metric > 2) return fail(KNN_ERR_ARGS, "unknown metric");
  rc = enter_device(&ctx, o);
  if (rc) return rc;
  cudaStream_t st = o.stream ? static_cast<cudaStream_t>(o.stream) : ctx->stream;
  knn::LaunchLog log;
  Prepared P;
  rc = prepare_points(ctx, points, n, d, o, st, &P, log);
  if (rc) return rc;
  const size_t np = knn::mlp_param_count(d);
  float *dp = nullptr, *dm = nullptr, *ds = nullptr;
  rc = ctx->get("mlpe_params", np, &dp);
  if (!rc) rc = ctx->get("mlpe_mean", (size_t)d, &dm);
  if (!rc) rc = ctx->get("mlpe_inv_std", (size_t)d, &ds);
  if (rc) return rc;
  KNN_CK(cudaMemcpyAsync(dp, params, sizeof(float) * np, cudaMemcpyHostToDevice, st));
  KNN_CK(cudaMemcpyAsync(dm, mean, sizeof(float) * (size_t)d, cudaMemcpyHostToDevice, st));
  KNN_CK(cudaMemcpyAsync(ds, inv_std, sizeof(float) * (size_t)d, cudaMemcpyHostToDevice, st));
  float* norms = nullptr;
  if (metric == KNN_METRIC_COSINE) {
    rc = ctx->get("norms", (size_t)n, &norms);
    if (rc) return rc;
    knn::launch_norms(P.X, n, d, P.dpad, norms, st);
  }
  float* Z = nullptr;
  rc = embed_points(ctx, P.X, norms, n, d, P.dpad, dp, dm, ds, st, &Z, log);
  if (rc) return rc;
  KNN_CK(cudaMemcpyAsync(out, Z, sizeof(float) * (size_t)n * knn::kMlpEmbed,
                         o.outputs_on_device ? cudaMemcpyDeviceToDevice : cudaMemcpyDeviceToHost, st));
  KNN_CK(cudaStreamSynchronize(st));
  return KNN_OK;
}

}  // extern "C"
