// Host-side launchers of the k-NN graph stages and their argument blocks.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include <vector>

#include "knn_internal.cuh"

namespace knn {

// Keys of a node staged in shared memory by k_split when it has at most this
// many points (96 KB).
constexpr int kSplitSmemKeys = 12288;
// Multi-block splits (levels with at most kMSplitMaxNodes split nodes and more
// than 2 * kMChunk points in the largest): keys per block, and the scratch.
constexpr int kMChunk = 8192;
constexpr int kMSplitMaxNodes = 296;
size_t msplit_scratch_bytes(int64_t max_node_points);

// Counts kernel launches of one call.
struct LaunchLog {
  int count = 0;
  void add(int c = 1) { count += c; }
};

__global__ void k_iota(int32_t* perm, int64_t n, int trees);

// Points are row-major float32 [n][dpad], dpad % 4 == 0, zero padded, 16-byte
// aligned rows.
// Batches: n = total points of all segments; segs / hsegs describe them
// (device view and host copy, sorted by n descending).
struct TreeArgs {
  const float* X;
  int64_t n;
  int d, dpad;
  int trees;
  int tree_offset, tree_stride;  // local tree t is global tree tree_offset + t * tree_stride
  SegView segs;
  const SegEntry* hsegs;
  int nseg;
  int32_t* perm;      // [trees][n] out: leaf order
  int32_t* perm_alt;  // [trees][n] scratch
  int32_t* inv;       // [trees][n] scratch: position of each point
  int32_t* node;      // [trees][n] scratch: node of each point at the current level
  uint64_t* keys;     // [trees][n] scratch
  float* dirs;        // [tree_dir_nodes(...)][dpad] scratch
  void* msplit;       // msplit_scratch_bytes(largest segment) scratch, or null (single-block splits)
  cudaStream_t stream;
};
int tree_build(const TreeArgs& a, LaunchLog& log);
// Direction slots the deepest-populated level needs: max over levels l of
// (segments still splitting at l) * trees * 2^l.
size_t tree_dir_nodes(const SegEntry* hsegs, int nseg, int trees);

// Reference-rule trees (tree_faithful.cu): node records, split per level on
// an explicit list of splitting nodes.
constexpr int kFaithfulMaxLevels = 4096;
struct FNode {
  int64_t lo, hi, id, parent;
  int32_t tree, p1, p2, cbase;  // cbase: the node's first slot in the chunk counts
};
struct FaithfulArgs {
  const float* X;
  int64_t n;
  int d, dpad, trees, leaf;
  uint64_t seed;
  int tree_offset, tree_stride;  // local tree t is global tree tree_offset + t * tree_stride
  int32_t* perm;       // [trees][n] out: leaf order
  int32_t* perm_alt;   // [trees][n] scratch
  uint8_t* side;       // [trees][n] scratch
  FNode* dnodes;       // [node_cap] scratch
  size_t node_cap;
  int32_t* lcount;     // [count_cap] scratch
  size_t count_cap;
  int64_t* nleft;      // [node_cap] scratch
  cudaStream_t stream;
};
struct FaithfulTrees {
  std::vector<FNode> nodes;   // every node, roots first; id = index
  std::vector<uint8_t> split; // 1: the node was split
  int levels = 0;
};
int faithful_tree_build(const FaithfulArgs& a, FaithfulTrees* out, LaunchLog& log);
// (lo, hi, blo, bhi) per leaf, per tree in position order; offset / count in leaves.
void faithful_leaf_table(const FaithfulTrees& T, int trees, int k, std::vector<int64_t>* table,
                         std::vector<int64_t>* offset, std::vector<int64_t>* count);

// n = all points (a batch: of every segment); leaves = leaf blocks per tree.
// With ftable the leaves of tree t are the fcount[t] entries (lo, hi, blo,
// bhi) from entry foff[t] of ftable (device; foff and fcount on the host).
struct LeafArgs {
  const float* X;
  int64_t n;
  int d, dpad, k, trees, metric;
  SegView segs;
  int64_t leaves;
  int64_t maxleaf;       // points in the largest leaf (query tiles per leaf)
  int64_t maxblock;      // points in the largest leaf block (0: maxleaf)
  const int32_t* perm;   // [trees][n]
  const float* norms;    // [n] (COSINE) or null
  float* rkey;           // [n][k] in/out, sorted
  uint32_t* rid;         // [n][k] in/out
  unsigned long long* pair_counter;  // optional
  int tile;              // 32 or 64 (0: 64): query x candidate tile, results identical
  int first_tree;        // trees [first_tree, first_tree + trees) of perm
  cudaEvent_t* kev;      // [2 * trees] events around each tree's tile kernel, or null
  const int64_t* ftable;
  const int64_t* foff;
  const int64_t* fcount;
  // sparse rows (EUCLIDEAN / TAXICAB, median trees): per tree, each leaf block's
  // non-zero dims; null dlist: every block reads all dims
  uint32_t* dmask;       // [leaves][dpad / 32 + 1]
  int16_t* dlist;        // [leaves][lmax], dims below 32768
  int32_t* dnch;         // [leaves]
  int lmax;              // 256 * ceil(dpad / 256)
  // every leaf is its own block (at least k+1 points, median trees): each tile
  // pair of a leaf is computed once and merged into both sides (k_leaf_pair)
  bool pairs;
  // sparse rows with tile pairs: positions within each leaf reordered by row
  // bucket (perm_w: writable alias of perm), per-tile dim masks
  int32_t* perm_w;       // [trees][n] or null
  uint8_t* bucket;       // [n]
  uint32_t* zeros;       // [1]: some row has a zero among its d dims
  int32_t* sort_tmp;     // [n]
  uint32_t* tmask;       // [leaves][ceil(maxleaf / tile)][ceil(dpad / 32) + 1]
  cudaStream_t stream;
};
int leaf_stage(const LeafArgs& a, LaunchLog& log);

// Mixed-precision leaf stage (BF16 tensor-core tiles + FP32 re-rank).
struct UmmaLeafArgs {
  const float* X;        // padded float32 rows
  int64_t n;
  int d, dpad, k, kq, trees, metric;
  SegView segs;
  int64_t leaves, maxleaf;  // leaf blocks per tree; points in the largest leaf
  int64_t maxblock;         // points in the largest leaf block (median trees)
  int tc_group;             // sibling leaves per 128-row tile: 1, 2 or 4 (each leaf its own block)
  const int32_t* perm;   // [trees][n]
  const float* norms;    // [n] FP32 norms (COSINE) or null
  bool f16;              // operands FP16 (else BF16)
  void* Xb;              // [n][Kp] 16-bit operand scratch (Kp = d rounded up to 64)
  unsigned int* maxabs;  // [1] scratch: largest |x| (FP16 EUCLIDEAN row scale)
  float* norms2;         // [n] scratch
  int32_t* inv;          // [n] scratch: a tree's inverse order (null: duplicate checks in the merge)
  cudaEvent_t* kev;      // [2 * trees] events around each tree's tile kernel, or null
  float* akey;           // [n][kq] approximate lists (in: empty)
  uint32_t* aid;
  float* rkey;           // [n][k] out: exact keys, sorted
  uint32_t* rid;
  int* err;              // [2]: [0] stop word of this build, [1] sticky; both set when a bounded wait expires
  const int64_t* ftable; // as in LeafArgs
  const int64_t* foff;
  const int64_t* fcount;
  cudaStream_t stream;
};
int leaf_stage_umma(const UmmaLeafArgs& a, LaunchLog& log);

struct PropArgs {
  const float* X;
  const void* Xh;            // FP16 rows [n][ldh] (ldh % 8 == 0, zero padded), gathered instead of X; or null
  int ldh;
  int64_t n;
  int d, dpad, k, metric;
  const float* norms;
  const int32_t* order;  // query order (a tree's leaf order) or null
  const float* key_in;
  const uint32_t* id_in;
  const uint32_t* flags_in;  // [n][kw] or null: every entry new
  float* key_out;
  uint32_t* id_out;
  uint32_t* flags_out;       // [n][kw]
  unsigned long long* cand_counter;  // optional
  int warps;                 // warps per block (0: as many as shared memory allows, at most 8)
  int64_t r0, r1;            // process points (order positions) [r0, r1); r1 = 0: all n
  cudaStream_t stream;
};
int propagate_step(const PropArgs& a, LaunchLog& log);

// Learned split network d -> kMlpHidden -> kMlpEmbed (mlp.cu).  Parameter
// vector: W1 [H][d], b1 [H], W2 [E][H], b2 [E].
constexpr int kMlpHidden = 256;
constexpr int kMlpEmbed = 64;

struct MlpTrainArgs {
  const float* Xs;       // [ns][dpad] sample rows
  const float* norms;    // [ns] row norms (COSINE: the input is the unit row) or null
  int64_t ns;
  int d, dpad;
  const int32_t* graph;  // [ns][gk] k-NN graph of the sample (sample-local ids), rank order
  int gk;
  int steps, batch;      // Adam steps, triplets per step
  float lr, margin;
  uint64_t seed;
  float* params;         // out: [mlp_param_count(d)]
  float* mean;           // out: [d]
  float* inv_std;        // out: [d]
  float* loss;           // out: [steps] mean triplet loss per step
  float* ws;             // [mlp_train_ws_floats(d, batch)]
  cudaStream_t stream;
};
size_t mlp_param_count(int d);
size_t mlp_fwd_bwd_ws_floats(int d, int B);
size_t mlp_train_ws_floats(int d, int B);
size_t mlp_embed_ws_floats(int d, int64_t chunk);
int mlp_train(const MlpTrainArgs& a, LaunchLog& log);
// Z [n][kMlpEmbed] = f(X) in chunks of `chunk` rows; norms [n] (COSINE) or null.
int mlp_embed(const float* X, const float* norms, int64_t n, int d, int dpad, const float* params,
              const float* mean, const float* inv_std, float* ws, int64_t chunk, float* Z, cudaStream_t st,
              LaunchLog& log);
// One forward + backward of the triplet loss over 3B standardised rows.
int mlp_loss_grad(const float* params, int d, const float* rows, int B, float margin, float* grad, float* ws,
                  float* loss, cudaStream_t st, LaunchLog& log);
void launch_gather_sample(const float* X, int64_t n, int dpad, int64_t ns, float* Xs, cudaStream_t st);

// Helpers (knn_misc.cu).
void launch_init_lists(float* key, uint32_t* id, uint32_t* flags, int64_t n, int k, int kw,
                       cudaStream_t st);
void launch_set_flags(uint32_t* flags, int64_t n, int k, int kw, cudaStream_t st);
void launch_norms(const float* X, int64_t n, int d, int dpad, float* norms, cudaStream_t st);
void launch_pad_rows(const void* src, int dtype, int64_t n, int d, int64_t ld, float* dst,
                     int dpad, cudaStream_t st);
// FP16 rows [n][ld] -> zero-padded [n][dh] (dh % 8 == 0), for FP16 gathers.
void launch_pad_rows_f16(const void* src, int64_t n, int d, int64_t ld, void* dst, int dh, cudaStream_t st);
void launch_finalize(const float* key, const uint32_t* id, int64_t n, int k, int metric,
                     float* out_dist, int32_t* out_idx, cudaStream_t st);
void launch_keys_from_dist(const float* dist, int64_t count, int metric, float* key,
                           cudaStream_t st);
// Batches (segments): local ids at finalisation; segment of every point.
void launch_finalize_local(const float* key, const uint32_t* id, int64_t ntot, int k, int metric,
                           const int32_t* seg_of, const SegEntry* segs, float* out_dist, int32_t* out_idx,
                           cudaStream_t st);
void launch_fill_seg_of(const SegEntry* segs, int count, int32_t* seg_of, cudaStream_t st);
// out[i] = the k best distinct ids by (key, id) of `lists` candidate lists
// [lists][n][k] of each point (ids < 0 or keys +inf are empty entries).
void launch_merge_lists(const int32_t* idx, const float* key, int lists, int64_t n, int k, int32_t* idx_out,
                        float* key_out, cudaStream_t st);
// Device rows of several sets ([n][d], element type dtype) gathered into one
// padded array at row offsets `off`, in one launch.
struct RowSource {
  const void* src;
  int64_t n, off;
};
void launch_gather_sets(const RowSource* sets, int count, int dtype, int d, float* dst, int dpad,
                        cudaStream_t st);

}  // namespace knn
