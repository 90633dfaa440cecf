/*
 * knn.h -- C ABI of the B200 approximate k-NN graph builder (libacknn.so).
 *
 * The builder replaces the compute span of the reference's class
 * EuclideanDistanceMatrixGPU (euclideandistancematrixgpu.h:50-63): everything
 * between the start and the end of calculate() (euclideandistancematrixgpu.cu:2861-2896),
 * i.e. normalisation-free tree build, initial k-NN and neighbour propagation.
 * The CLI, the CSV reader and the binary writer of the reference sit above
 * this ABI (see approximate-cuda-knn_b200/cli/hello.cpp).
 *
 * Conventions
 *   - Every function returns KNN_OK (0) or a negative KNN_ERR_* code; none
 *     prints, exits, or resets the device (the reference calls cudaDeviceReset
 *     in initialize/deinitialize, euclideandistancematrixgpu.cu:2775, :2856).
 *   - The caller owns points and outputs (host or device memory, see
 *     knn_options).  The library owns its scratch through a knn_context,
 *     reused across calls.  One context per host thread.
 *   - Output rows are sorted by (distance, index) ascending.  Distances are
 *     L2 for EUCLIDEAN, L1 for TAXICAB and 1 - cos for COSINE.
 *   - Plain-FP32 results are bit-identical to the CPU restatement under
 *     oracle/ (same trees, same neighbour lists, same distances).
 */
#ifndef ACKNN_KNN_H_
#define ACKNN_KNN_H_

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Metric codes, same values as DISTANCE_EUCLIDEAN / DISTANCE_TAXICAB /
 * DISTANCE_COSINE (euclideandistancematrixgpu.h:16-18). */
#define KNN_METRIC_EUCLIDEAN 0
#define KNN_METRIC_TAXICAB 1
#define KNN_METRIC_COSINE 2

/* Status codes.  The reference signals failure with a bool `true` and a
 * message on stdout (cucall.h:12-19); these codes replace both. */
#define KNN_OK 0
#define KNN_ERR_ARGS -1        /* a size, pointer or option is invalid        */
#define KNN_ERR_N_LE_K -2      /* n <= k: fewer than k other points exist       */
#define KNN_ERR_OOM -3         /* device or pinned allocation failed            */
#define KNN_ERR_CUDA -4        /* a CUDA call failed; see knn_last_error()      */
#define KNN_ERR_TIMEOUT -5     /* a bounded device-side wait gave up            */
#define KNN_ERR_UNSUPPORTED -6 /* valid request this build cannot serve        */
#define KNN_ERR_NO_DEVICE -7   /* no usable CUDA device                         */

/* Element types of the input points. */
#define KNN_F32 0
#define KNN_F16 1
#define KNN_BF16 2

/* Precision modes of the leaf stage. */
#define KNN_PREC_FP32 0        /* every key in FP32 CUDA-core arithmetic          */
#define KNN_PREC_BF16_RERANK 1 /* leaf blocks as BF16 tensor-core tiles in the
                                  |x|^2+|y|^2-2x.y form, each point's best 2k
                                  re-ranked with exact FP32 keys.  TAXICAB, and
                                  requests the tiles cannot hold, run the FP32
                                  leaf stage instead; knn_stats.leaf_path and
                                  leaf_fallback say which ran                     */
#define KNN_PREC_F16_RERANK 2  /* the same with FP16 tiles: 11 significant bits
                                  instead of 8, exact for FP16 input; EUCLIDEAN
                                  rows are scaled by a power of two into the FP16
                                  range inside the tile stage (keys are ranked
                                  the same; the re-rank uses the input rows)     */

/* Tree split rules.  MEDIAN: each node splits at the median of its points'
 * projections (balanced trees of static shape).  REFERENCE: the split of
 * buildUpTheTrees (euclideandistancematrixgpu.cu:2138-2181, :2291-2365): the
 * sign of x . (x[p2] - x[p1]) through the origin, positions p1, p2 drawn once
 * per level and shared by its nodes, p1 forced left and p2 right, nodes
 * split until they hold at most `leaf` points -- for like-for-like recall
 * comparisons with the reference (single builds only). */
#define KNN_SPLIT_MEDIAN 0
#define KNN_SPLIT_REFERENCE 1

#define KNN_MAX_K 128
#define KNN_MAX_PROPS 64

typedef struct knn_options {
  int32_t struct_size;       /* sizeof(knn_options)                                  */
  int32_t device;            /* CUDA device ordinal; -1: the current device          */
  int32_t points_on_device;  /* 1: `points` is a device pointer                       */
  int32_t outputs_on_device; /* 1: out_idx / out_dist are device pointers             */
  int32_t dtype;             /* KNN_F32 / KNN_F16 / KNN_BF16                           */
  int32_t precision;         /* KNN_PREC_*                                             */
  int32_t learned_splits;    /* 1: tree directions from the learned split network     */
  int32_t timing;            /* 1: record per-stage device times in knn_stats         */
  int64_t ld;                /* row stride of `points` in elements; 0 means d         */
  void* stream;              /* cudaStream_t; NULL: the context's own stream          */
  int32_t mlp_sample;        /* learned splits: points in the training sample (0: 65536) */
  int32_t mlp_steps;         /* learned splits: Adam steps (0: 300)                      */
  int32_t autotune;          /* 1: time the result-invariant launch shapes (FP32 leaf
                                tile, propagation warps) on the first eager call of a
                                workload and reuse the fastest from then on           */
  int32_t leaf_tile;         /* FP32 leaf tile 32 or 64 (0: tuned, else 64)              */
  int32_t prop_warps;        /* propagation warps per block 1..8 (0: tuned, else max)   */
  int32_t tree_offset;       /* sharded builds: local tree t is the global tree          */
  int32_t tree_stride;       /*   tree_offset + t * tree_stride (stride 0 means 1)       */
  int32_t raw_keys;          /* 1: out_dist receives the ranking keys (squared L2 for
                                EUCLIDEAN) instead of distances                       */
  int32_t split_rule;        /* KNN_SPLIT_MEDIAN (default) or KNN_SPLIT_REFERENCE     */
  int32_t tc_group;          /* tensor-core leaf tiles: sibling leaves per 128-row tile,
                                1, 2 or 4 (0: tuned with autotune, else the most that
                                fit); a row keeps its own leaf's columns, so results do
                                not depend on it; capped at what the leaves allow      */
  int32_t sparse_dims;       /* FP32 leaf tiles, EUCLIDEAN and TAXICAB, d < 32768: 1 each
                                tile reads only the dims that are non-zero in some of
                                its rows (with tile pairs: the union of the pair's two
                                tiles, each leaf's points ordered by zero pattern;
                                the left-out terms are exact zeros, so the keys keep
                                their bits); -1 never; 0 when leaves hold at least
                                1024 points                                           */
  int32_t tile_pairs;        /* FP32 leaf tiles where every leaf is its own block: each
                                key is computed once for both of its points (keys are
                                symmetric bit for bit, so the graph is the same); -1 off,
                                else on                                               */
} knn_options;

typedef struct knn_stats {
  int32_t struct_size;       /* sizeof(knn_stats)                                      */
  int32_t depth;             /* levels below the root in every tree                    */
  float ms_total;            /* device time of the call, first to last launch           */
  float ms_upload;           /* host->device copy and row padding                      */
  float ms_trees;            /* tree build                                             */
  float ms_leaf;             /* initial k-NN over leaf blocks                          */
  float ms_propagate;        /* all propagation iterations                             */
  float ms_download;         /* finalisation and device->host copy                     */
  int32_t launches;          /* kernels launched by the call                           */
  int32_t props_run;         /* propagation iterations run                             */
  int64_t leaf_pairs;        /* (query, candidate) keys evaluated by the leaf stage     */
  int64_t prop_candidates[KNN_MAX_PROPS]; /* keys evaluated per propagation iteration  */
  float ms_prop_iter[KNN_MAX_PROPS];      /* device time per propagation iteration     */
  float ms_learn;            /* learned splits: sample graph, training and embedding    */
  int32_t leaf_tile;         /* leaf tile used: 32/64 FP32, 128 tensor-core             */
  int32_t prop_warps;        /* propagation warps per block used (0: the default)       */
  float ms_leaf_tiles;       /* summed device time of the leaf-tile kernel launches     */
  int32_t leaf_path;         /* leaf stage that ran: 0 FP32 CUDA cores, 1 BF16 tensor-core
                                tiles, 2 FP16 tensor-core tiles                        */
  int32_t leaf_fallback;     /* 1: tensor-core precision was asked for, FP32 ran        */
  int32_t tc_group;          /* sibling leaves per tensor-core tile used (0: FP32 path) */
  int32_t sparse_dims;       /* 1: the FP32 leaf tiles read each block's non-zero dims
                                (knn_build_ex; 0 from knn_build_batch)               */
  int32_t tile_pairs;        /* 1: the FP32 leaf tiles ran as tile pairs (knn_build_ex) */
  int32_t reserved32;
  int64_t reserved[3];
} knn_stats;

typedef struct knn_context knn_context;

/* Fill `opt` with defaults: current device, host pointers, FP32 input, plain
 * precision, random-projection splits, no timing. */
void knn_default_options(knn_options* opt);

/* Library version as MAJOR*10000 + MINOR*100 + PATCH. */
int knn_version(void);

/* Text of a status code, and the message of the last failure on this thread. */
const char* knn_status_string(int status);
const char* knn_last_error(void);

/* Compute capability of `device`: KNN_OK, KNN_ERR_NO_DEVICE when the machine
 * has no CUDA device, KNN_ERR_ARGS when the ordinal does not exist.  Serves the
 * CLI's device check (main.cpp:53-70). */
int knn_device_capability(int32_t device, int32_t* major, int32_t* minor);

/* Context owning device scratch, stream and events on `device` (-1: current).
 * Returns NULL on failure (see knn_last_error). */
knn_context* knn_context_create(int32_t device);
void knn_context_destroy(knn_context* ctx);
/* Bytes of device scratch the context currently holds. */
int64_t knn_context_scratch_bytes(const knn_context* ctx);

/* Outcome of the context's asynchronous calls.  A build given a caller stream,
 * device outputs and no statistics returns as soon as its work is queued, so a
 * tensor-core tile wait that gives up inside it cannot change its return
 * value.  The failure is kept in a per-context error word that only a read
 * clears: this call waits for `stream` (NULL: the context's own stream), then
 * returns KNN_ERR_TIMEOUT once for every such failure since the last report,
 * else KNN_OK.  The next synchronising build on the context reports it too.
 * ctx NULL: the calling thread's default context of the current device. */
int knn_context_status(knn_context* ctx, void* stream);

/* Test hook: the next build on `ctx` (NULL: the thread's default context)
 * starts with its tile-wait error word already set, as if a wait had given
 * up.  Its tensor-core tile kernels then issue no MMA, free their tensor
 * memory and return, and the build returns KNN_ERR_TIMEOUT.  One-shot; the
 * build after it runs normally. */
int knn_test_fail_next_tile_wait(knn_context* ctx);

/*
 * knn_build -- the drop-in call.  Replaces EuclideanDistanceMatrixGPU::initialize
 * + calculate + the device->host copy of saveResultToResultFile
 * (euclideandistancematrixgpu.cu:2759-2819, :2861-2896, :2908-2915) for points
 * already in memory.
 *   points   host float32 [n][d], row-major
 *   k        neighbours per point (1..KNN_MAX_K), n must exceed k
 *   trees    random-projection trees (numberOfTrees, main.cpp:27)
 *   leaf     maximum points per leaf (minSize / numberOfElemsInLeaf, main.cpp:28)
 *   props    propagation iterations (numberOfPropagations, main.cpp:29)
 *   metric   KNN_METRIC_*
 *   seed     seed of the split choices
 *   out_idx  host int32 [n][k];  out_dist host float32 [n][k]
 * Uses a per-thread default context on the current device, plain FP32.
 */
int knn_build(const void* points, int64_t n, int32_t d, int32_t k, int32_t trees, int32_t leaf,
              int32_t props, int32_t metric, uint64_t seed, int32_t* out_idx, float* out_dist);

/* knn_build with an explicit context (NULL: per-thread default), options
 * (NULL: defaults) and optional statistics (NULL: none). */
int knn_build_ex(knn_context* ctx, const void* points, int64_t n, int32_t d, int32_t k,
                 int32_t trees, int32_t leaf, int32_t props, int32_t metric, uint64_t seed,
                 int32_t* out_idx, float* out_dist, const knn_options* opt, knn_stats* stats);

/*
 * knn_build_batch -- many independent point sets in one call (no counterpart
 * in the reference, which builds one set per process).  Sets of equal d are
 * concatenated and every stage runs once for all of them; each set's trees,
 * leaf blocks and propagation stay within the set, and its result equals a
 * knn_build_ex of that set alone with the same seed (bit for bit in plain
 * FP32).  The device work of a group of equal-d sets is captured as a CUDA
 * graph the second time the same shapes are seen and replayed after that.
 *   sets[i].points  [n][d] rows, host or device and element type per options
 *                   (options.ld must be 0);  out_idx int32 [n][k] (ids local to
 *                   the set) and out_dist float32 [n][k], host or device.
 * Learned splits are not available here (KNN_ERR_UNSUPPORTED).
 */
typedef struct knn_dataset {
  const void* points;
  int64_t n;
  int32_t d;
  int32_t reserved;
  uint64_t seed;
  int32_t* out_idx;
  float* out_dist;
} knn_dataset;

int knn_build_batch(knn_context* ctx, const knn_dataset* sets, int32_t count, int32_t k, int32_t trees,
                    int32_t leaf, int32_t props, int32_t metric, const knn_options* opt, knn_stats* stats);

/*
 * Sharded builds (several GPUs, one process each; no counterpart in the
 * reference).  Rank r of G builds the global trees r, r+G, ... with
 * knn_build_ex (tree_offset = r, tree_stride = G, raw_keys = 1, props = 0);
 * the G lists of every point are gathered and merged by knn_merge_lists (the
 * k best distinct ids of the union: the lists of all trees at once); each
 * propagation step then runs on a point range per rank (knn_propagate_range)
 * and the ranges are gathered.  The graph equals the single-GPU build's.
 *
 * knn_merge_lists: idx/key [lists][n][k] sorted lists (id < 0: empty) ->
 *   idx_out/key_out [n][k]; as_distance = 1 writes distances (sqrt of the key
 *   for EUCLIDEAN) instead of keys.  Device memory when
 *   options.points_on_device, else host.
 * knn_propagate_range: one Jacobi propagation step for the points
 *   [r0, r1); lists in device memory (idx/key [n][k] with keys, flags
 *   [n][ceil(k/32)] NEW bits or NULL for all new); rows outside the range of
 *   the outputs are left as they are.  Points per options.
 */
int knn_merge_lists(knn_context* ctx, const int32_t* idx, const float* key, int32_t lists, int64_t n, int32_t k,
                    int32_t metric, int32_t as_distance, int32_t* idx_out, float* key_out,
                    const knn_options* opt);
int knn_propagate_range(knn_context* ctx, const void* points, int64_t n, int32_t d, int32_t k, int32_t metric,
                        int64_t r0, int64_t r1, const int32_t* idx_in, const float* key_in,
                        const uint32_t* flags_in, int32_t* idx_out, float* key_out, uint32_t* flags_out,
                        const knn_options* opt);

/*
 * Stage entry points (host memory in and out), for stage-by-stage checks.
 *   knn_build_trees   leaf order of every tree: out_perm int32 [trees][n]
 *                     (replaces buildUpTheTrees, euclideandistancematrixgpu.cu:2407-2686)
 *   knn_leaf_stage    initial k-NN from given leaf orders; out_key holds keys
 *                     (squared L2 / L1 / 1-cos), rows sorted
 *                     (replaces findInitialKNN, euclideandistancematrixgpu.cu:2067-2107)
 *   knn_propagate_step one Jacobi propagation step on keys
 *                     (replaces one iteration of propagate, euclideandistancematrixgpu.cu:1937-1977)
 */
int knn_build_trees(knn_context* ctx, const float* points, int64_t n, int32_t d, int32_t trees,
                    int32_t leaf, uint64_t seed, int32_t* out_perm);
int knn_leaf_stage(knn_context* ctx, const float* points, int64_t n, int32_t d, int32_t k,
                   int32_t trees, int32_t leaf, int32_t metric, const int32_t* perm,
                   int32_t* out_idx, float* out_key);
int knn_propagate_step(knn_context* ctx, const float* points, int64_t n, int32_t d, int32_t k,
                       int32_t metric, const int32_t* idx_in, const float* key_in,
                       int32_t* idx_out, float* key_out);

/*
 * knn_exact_fp64 -- exact k-NN of `nq` query rows against all n points in
 * FP64 on the GPU (self excluded, ties by index).  The yardstick of recall and
 * distance error; no counterpart in the reference.
 *   points host or device (opt->points_on_device) float32 [n][d]
 *   queries host int64 [nq] row ids;  out_idx host int32 [nq][k];
 *   out_dist host float64 [nq][k] (L2 / L1 / 1-cos)
 */
int knn_exact_fp64(knn_context* ctx, const void* points, int64_t n, int32_t d, int32_t k,
                   int32_t metric, const int64_t* queries, int64_t nq, int32_t* out_idx,
                   double* out_dist, const knn_options* opt);

/*
 * knn_exact_fp64_noalloc -- knn_exact_fp64 for callers that cannot allocate
 * device memory while they run (a process whose device memory is all handed to
 * its own pool at start-up, or a thread that must not pay the device-wide
 * synchronisation cudaMalloc/cudaFree may bring).  No counterpart in the
 * reference.  It allocates nothing: its scratch is one 16 MiB array compiled
 * into the library, held by every GPU that loads it until the process exits.
 *   points  device float32 [n][d];  queries device int64 [nq];
 *   out_idx device int32 [nq][k];  out_dist device float64 [nq][k];
 *   stream  cudaStream_t (NULL: legacy default stream); the call returns once
 *           the stream has finished.
 * Results equal knn_exact_fp64's.  The first call on a device looks up the
 * scratch address, so make it before any stream capture; with CUDA's lazy
 * module loading that first call is also when the array is reserved on the
 * device, so a caller that hands its device memory to a pool makes one
 * warm-up call per device before that (a failed reservation returns
 * KNN_ERR_OOM).  All calls share the
 * scratch: calls that overlap on the GPU race.  Requests whose scratch exceeds
 * 16 MiB (about 16 bytes per (query, neighbour) pair, plus 8 bytes per point
 * for COSINE) return KNN_ERR_ARGS; so does a query id outside [0, n).
 */
int knn_exact_fp64_noalloc(const float* points, int64_t n, int32_t d, int32_t k, int32_t metric,
                           const int64_t* queries, int64_t nq, int32_t* out_idx,
                           double* out_dist, void* stream);

/*
 * knn_normalize_reference -- the reference's data normalisation
 * (normalizeDataStep1/2, euclideandistancematrixgpu.cu:19-85, run by calculate()
 * at :2869-2875) on host float32 [n][d] in place, on the GPU: subtract the
 * per-dimension mean, then divide dimensions 0..255 by the largest |x| seen
 * over dimensions 0..255 (dimensions >= 256 stay centred but unscaled, as in
 * the reference).  Used by the CLI only; knn_build never normalises.
 */
int knn_normalize_reference(float* points, int64_t n, int32_t d);

/*
 * Learned split network (options.learned_splits = 1).  No counterpart in the
 * reference, whose split directions are differences of raw points
 * (euclideandistancematrixgpu.cu:2138-2164).
 *
 *   f(x) = W2 gelu(W1 s(x) + b1) + b2,  s(x) = (u(x) - mean) * inv_std,
 *   u(x) = x/|x| for COSINE (a zero row stays zero), else x,
 *   gelu(a) = 0.5 a (1 + tanh(sqrt(2/pi) (a + 0.044715 a^3))),
 *   W1 [256][d], b1 [256], W2 [64][256], b2 [64]; the parameter vector is
 *   W1, b1, W2, b2 in that order, float32, knn_mlp_param_count(d) values.
 *
 * Training: the plain method builds a k-NN graph (2k neighbours, at most 32)
 * of a strided sample of options.mlp_sample points; each Adam step takes 1024
 * triplets (anchor, a graph neighbour of rank < k', a random point or a
 * neighbour of rank >= k', k' = half the graph width) and minimises
 *   mean max(0, margin + |f(a) - f(p)|^2 - |f(a) - f(n)|^2),  margin 1.
 * knn_build_ex then builds the trees on the 64-dim embeddings f(x) (split
 * directions f(x_p2) - f(x_p1)); leaf blocks and propagation rank the
 * original points as before.
 */
#define KNN_MLP_HIDDEN 256
#define KNN_MLP_EMBED 64
int64_t knn_mlp_param_count(int32_t d);
/* Mean triplet loss and its gradient for one batch: rows host float32
 * [3*batch][d], already standardised, anchors then positives then negatives;
 * grad host float32 [knn_mlp_param_count(d)]; loss host float32 [1]. */
int knn_mlp_loss_grad(const float* params, int32_t d, const float* rows, int32_t batch, float margin,
                      float* grad, float* loss);
/* Train the network as knn_build_ex does for these points (host outputs:
 * params, mean [d], inv_std [d], loss_curve [steps] or NULL). */
int knn_mlp_train(knn_context* ctx, const void* points, int64_t n, int32_t d, int32_t k, int32_t metric,
                  uint64_t seed, const knn_options* opt, float* params, float* mean, float* inv_std,
                  float* loss_curve);
/* out [n][64] = f(points) (host, or device with options.outputs_on_device);
 * for KNN_METRIC_COSINE the network input is the unit row x/|x|. */
int knn_mlp_embed(knn_context* ctx, const void* points, int64_t n, int32_t d, int32_t metric,
                  const float* params, const float* mean, const float* inv_std, const knn_options* opt,
                  float* out);

#ifdef __cplusplus
}
#endif

#endif /* ACKNN_KNN_H_ */
