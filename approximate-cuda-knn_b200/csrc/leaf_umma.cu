// Initial k-NN over leaf blocks on the 5th-generation tensor cores (tcgen05),
// for EUCLIDEAN and COSINE: the mixed-precision leaf stage.
//
// Same blocks and same union-over-trees rule as the FP32 leaf stage (which
// replaces findInitialStateOfAproximated*KNN, euclideandistancematrixgpu.cu:107-1031),
// but every (query, candidate) key of a block comes from one BF16 GEMM tile:
//     key ~= |x|^2 + |y|^2 - 2 x.y      (EUCLIDEAN, norms of the BF16 rows)
//     key ~= 1 - x.y                     (COSINE, rows normalised before rounding)
// with FP32 accumulation in tensor memory.  Each point keeps its best kq (2k,
// at most 32) approximate candidates over all trees; k_rerank then recomputes
// those kq keys exactly in FP32 (the reference's order) and keeps the best k.
// When the BF16 products and FP32 sums are exact (integer data below 2^8 per
// coordinate and 2^24 per sum, e.g. the integer-mixture workload) the result
// equals the FP32 leaf stage bit for bit.
//
// Tile: 128 queries x 128 candidates x Kp (Kp = d rounded up to 64, <= 256).
//   * operands: K-major, 128-byte swizzled shared-memory tiles (8-row atoms of
//     1024 B), filled by cp.async from the BF16 copy through the tree's order;
//   * MMA: tcgen05.mma.cta_group::1.kind::f16, M=128 N=128 K=16, issued by one
//     thread, accumulator 128 lanes x 128 columns of tensor memory, two
//     accumulators so that one tile's MMA overlaps the previous tile's rounds;
//   * completion: tcgen05.commit -> mbarrier, waited with an iteration limit
//     (on expiry the block records an error, drains, frees TMEM and returns);
//   * epilogue: per tile, tcgen05.ld 32x32b.x32 twice by all 8 warps (warp
//     w reads lane quarter w%4, two 32-column slices); three instructions per
//     key filter it against a slightly widened bound of the row's last entry
//     into a survivor bit mask, then (while the next tile's MMA runs) the warps
//     of each lane quarter read their rows' few survivors back from tensor
//     memory, compute their exact keys and insert them into the query's sorted
//     list (held in shared memory for the whole block) with one ballot and one
//     lane shift each.  Two block barriers per tile.
#include <cuda_bf16.h>
#include <cuda_fp16.h>

#include <algorithm>

#include "knn_internal.cuh"
#include "knn_kernels.cuh"

namespace knn {

namespace {
constexpr int kBM = 128;
constexpr int kBN = 128;
constexpr int kKC = 64;               // bf16 per 128-byte swizzled row
constexpr int kChunkBytes = kBM * 128; // one 128 x 64 bf16 operand chunk
constexpr uint32_t kTmemCols = 256;  // two 128-column accumulators
constexpr int kUThreads = 256;
constexpr int kRound = 64;          // tile columns per epilogue slice pair
constexpr int kBulkMerge = 12;      // first tree: survivors in a 32-column slice from which sort + merge pays
constexpr float kSlack = 4.76837158203125e-07f;  // 2^-21: filter widening, eight units of FP32 rounding
// Listed candidates inside the block, per row: sorted 16-bit column positions
// ending in kXEnd (blocks of up to kXMaxBlock columns).
constexpr int kXS = 33;
constexpr uint32_t kXEnd = 0xFFFFu;
constexpr int kXMaxBlock = 65000;
// First tree: blocks of at least kPrepassMin columns get a bounding pass; its
// group minima (64 per row, row stride kGS) use the list area.
constexpr int kPrepassMin = 1024;
constexpr int kGroups = 64;
constexpr int kGS = kGroups + 1;
constexpr int kLS = 33;              // list row stride (row owners hit distinct banks)
// A 128x128x256 tile finishes in about a microsecond; 2^16 polls with 32 ns
// sleeps (a few ms) is far beyond that, and keeps a failing launch short.
constexpr uint32_t kSpinLimit = 1u << 16;

// Instruction descriptor of kind::f16: D f32 (bits 4-5 = 1), A and B format
// at 7-9 and 10-12 (0 f16, 1 bf16; A and B always the same type), A and B
// K-major (15, 16 = 0), N>>3 at 17-22, M>>4 at 24-28.
constexpr uint32_t idesc_for(bool f16) {
  return (1u << 4) | ((f16 ? 0u : 1u) << 7) | ((f16 ? 0u : 1u) << 10) | ((uint32_t)(kBN >> 3) << 17) |
         ((uint32_t)(kBM >> 4) << 24);
}

__device__ __forceinline__ uint32_t smem_u32(const void* p) {
  return (uint32_t)__cvta_generic_to_shared(p);
}

// Shared-memory matrix descriptor, K-major, 128-byte swizzle: start address
// (>>4) in bits 0-13, leading offset 1 (unused for swizzled K-major) at 16-29,
// stride 1024 B (>>4 = 64) between 8-row atoms at 32-45, version 1 at 46-47,
// base offset 0, layout type 2 (SWIZZLE_128B) at 61-63.
__device__ __forceinline__ uint64_t desc_sw128(uint32_t saddr) {
  return (uint64_t)((saddr >> 4) & 0x3FFFu) | ((uint64_t)1 << 16) | ((uint64_t)64 << 32) |
         ((uint64_t)1 << 46) | ((uint64_t)2 << 61);
}

__device__ __forceinline__ void cp_async16(uint32_t dst, const void* src, int bytes) {
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;\n" ::"r"(dst), "l"(src), "r"(bytes));
}

__device__ __forceinline__ void mbar_init(uint32_t bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;\n" ::"r"(bar), "r"(count));
}

// Non-blocking test of phase completion.  (try_wait may suspend the thread for
// a system-dependent time per call, so counting try_wait calls bounds nothing;
// test_wait never suspends.)
__device__ __forceinline__ bool mbar_test_wait(uint32_t bar, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "mbarrier.test_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
      "selp.u32 %0, 1, 0, p;\n\t}\n"
      : "=r"(ok)
      : "r"(bar), "r"(parity)
      : "memory");
  return ok != 0;
}

// Waits for the phase with the given parity; false once kWaitNs of wall time
// (globaltimer) have passed.
constexpr uint64_t kWaitNs = 20ull * 1000 * 1000;  // 20 ms; a tile takes ~1 us
__device__ __forceinline__ uint64_t global_ns() {
  uint64_t t;
  asm volatile("mov.u64 %0, %%globaltimer;\n" : "=l"(t));
  return t;
}
__device__ __forceinline__ bool mbar_wait_bounded(uint32_t bar, uint32_t parity) {
  const uint64_t t0 = global_ns();
  for (uint32_t it = 0; it < kSpinLimit; ++it) {
    if (mbar_test_wait(bar, parity)) return true;
    if (it > 64) {
      __nanosleep(256);
      if (global_ns() - t0 > kWaitNs) return false;
    }
  }
  return false;
}

__device__ __forceinline__ void umma_f16(uint32_t tmem_d, uint64_t da, uint64_t db, uint32_t idesc,
                                         uint32_t accumulate) {
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "setp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t}\n" ::"r"(tmem_d),
      "l"(da), "l"(db), "r"(idesc), "r"(accumulate), "r"(0u), "r"(0u), "r"(0u), "r"(0u));
}

__device__ __forceinline__ void umma_commit(uint32_t bar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];\n" ::"r"(bar)
               : "memory");
}

__device__ __forceinline__ uint32_t tmem_ld1(uint32_t taddr) {
  uint32_t v;
  asm volatile("tcgen05.ld.sync.aligned.32x32b.x1.b32 {%0}, [%1];\n" : "=r"(v) : "r"(taddr));
  asm volatile("tcgen05.wait::ld.sync.aligned;\n" ::: "memory");
  return v;
}

__device__ __forceinline__ void tmem_ld32(uint32_t taddr, uint32_t (&v)[32]) {
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x32.b32 "
      "{%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15,"
      "%16,%17,%18,%19,%20,%21,%22,%23,%24,%25,%26,%27,%28,%29,%30,%31}, [%32];\n"
      : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]), "=r"(v[5]), "=r"(v[6]),
        "=r"(v[7]), "=r"(v[8]), "=r"(v[9]), "=r"(v[10]), "=r"(v[11]), "=r"(v[12]), "=r"(v[13]),
        "=r"(v[14]), "=r"(v[15]), "=r"(v[16]), "=r"(v[17]), "=r"(v[18]), "=r"(v[19]),
        "=r"(v[20]), "=r"(v[21]), "=r"(v[22]), "=r"(v[23]), "=r"(v[24]), "=r"(v[25]),
        "=r"(v[26]), "=r"(v[27]), "=r"(v[28]), "=r"(v[29]), "=r"(v[30]), "=r"(v[31])
      : "r"(taddr));
  asm volatile("tcgen05.wait::ld.sync.aligned;\n" ::: "memory");
}

// Stage 128 gathered rows (ids in `ids`, <0: zero row) of the 16-bit copy
// into a K-major 128B-swizzled operand of NCH 64-element chunks.  Thread t
// always stages the same 16-byte unit (t mod 8 NCH) of rows t / (8 NCH) + i *
// R, R = the rows one pass of the threads covers.
template <int NCH>
__device__ __forceinline__ void stage_operand(unsigned char* op, const uint16_t* __restrict__ Xb,
                                              const int32_t* ids) {
  constexpr int kUnitsPerRow = 8 * NCH;       // 16-byte units per row
  constexpr int kRowsPerPass = kUThreads / kUnitsPerRow;
  constexpr int kActive = kRowsPerPass * kUnitsPerRow;  // all 256 threads but for NCH = 3 (240)
  const uint32_t base = smem_u32(op);
  if (threadIdx.x < kActive) {
    const int c16 = threadIdx.x % kUnitsPerRow;
    const int chunk = c16 >> 3, w = c16 & 7;
    const int r0 = threadIdx.x / kUnitsPerRow;
#pragma unroll
    for (int r = r0; r < kBM; r += kRowsPerPass) {
      const uint32_t dst = base + chunk * kChunkBytes + r * 128 + ((w ^ (r & 7)) << 4);
      const int32_t id = ids[r];
      const uint16_t* src = Xb + (size_t)(id < 0 ? 0 : id) * (NCH * kKC) + c16 * 8;
      cp_async16(dst, src, id < 0 ? 0 : 16);
    }
  }
  asm volatile("cp.async.commit_group;\n" ::);
}

}  // namespace

// Ascending sort of one value per lane (bitonic network over the warp).
__device__ __forceinline__ uint32_t warp_sort32_u32(uint32_t v) {
  const int lane = threadIdx.x & 31;
#pragma unroll
  for (int size = 2; size <= 32; size <<= 1) {
#pragma unroll
    for (int m = size >> 1; m >= 1; m >>= 1) {
      const uint32_t o = __shfl_xor_sync(0xFFFFFFFFu, v, m);
      const bool keep_min = ((lane & size) == 0) == ((lane & m) == 0);
      v = keep_min ? min(v, o) : max(v, o);
    }
  }
  return v;
}

// One block per (leaf, 128-query tile), stepping over the block's 128-column
// candidate tiles.  The 128 queries' lists stay in shared memory for the whole
// block (read once, written once).  Each step empties one 128x128 tensor-core
// tile (tensor memory, two 128-column buffers):
//   * epilogue: thread (row, 32-column half) loads the products of its two
//     32-column slices (tcgen05.ld 32x32b.x32), filters them against a
//     conservative bound of the row's list tail at the step's start into
//     survivor bit masks (three instructions per key), drops the row's own
//     column and listed ids;
//   * merge: the warps of the rows' lane quarter insert each row's survivors,
//     reading their products back from tensor memory (tcgen05.ld x1 per
//     survivor, or x32 and a lane transpose for a bulk batch), computing the
//     exact keys and applying the exact (key, id) rule.
// The next step's operand is staged while the epilogue runs (its MMA has
// completed), and its MMA runs into the other tensor-memory buffer during
// the merge.  MMA issue, bounded waits and the tensor-memory loads follow the
// single-tile sequence that was checked on its own against a CPU product.
// FIRST: the launch of the first tree, whose lists start empty; a point then
// meets every candidate once, so no survivor can already be listed, and a
// 32-column slice with many survivors is sorted and merged into the list in one go.
// Blocks of kPrepassMin columns or more first run all tiles once (pass 0) to
// record each row's smallest exact key in each of kGroups column groups
// (32-column slices, wrapping); the kq-th smallest group minimum is the key of
// kq distinct candidates, so it bounds the kq-th key of the final list, and
// pass 1 filters against it from its first tile on.
// Later trees, with inv (the tree's inverse order): the block's columns that
// hold an id already in the row's list are found up front (inv of each listed
// id) and masked out of the survivors, so the merge needs no duplicate check;
// a candidate meets a row once per tree, so ids inserted during the block
// cannot come back.
template <int METRIC, bool FIRST, int NCH>
__global__ void __launch_bounds__(kUThreads, 2)
    k_leaf_tc(const uint16_t* __restrict__ Xb, uint32_t idesc, SegView segs,
              const int64_t* __restrict__ ftab, int k, int kq,
              int qtiles, int glog, const int32_t* __restrict__ perm, const int32_t* __restrict__ inv,
              const float* __restrict__ norms2, float* __restrict__ akey, uint32_t* __restrict__ aid,
              int* __restrict__ err) {
  extern __shared__ __align__(1024) unsigned char smem_raw[];
  unsigned char* smem = (unsigned char*)(((uintptr_t)smem_raw + 1023) & ~(uintptr_t)1023);
  constexpr int nchunks = NCH;
  unsigned char* opA = smem;
  unsigned char* opB = opA + nchunks * kChunkBytes;
  float* Lk = reinterpret_cast<float*>(opB + nchunks * kChunkBytes);  // [128][kLS] list keys
  uint32_t* Li = reinterpret_cast<uint32_t*>(Lk + kBM * kLS);         // [128][kLS] list ids
  int32_t* qid = reinterpret_cast<int32_t*>(Li + kBM * kLS);
  float* qn = reinterpret_cast<float*>(qid + kBM);
  int32_t* cid3 = reinterpret_cast<int32_t*>(qn + kBM);  // [3][128] candidate ids, slot = step mod 3
  float* cn3 = reinterpret_cast<float*>(cid3 + 3 * kBN);  // [3][128] norms (EUCLIDEAN) or 0; +inf: padding
  uint32_t* msk = reinterpret_cast<uint32_t*>(cn3 + 3 * kBN);  // [128][4] survivor bits of the step's tile
  float* cmax3 = reinterpret_cast<float*>(msk + kBM * 4);      // [3][4] largest candidate norm per warp
  uint16_t* xp = reinterpret_cast<uint16_t*>(cmax3 + 12);      // [128][kXS] listed columns
  float* tcap = reinterpret_cast<float*>(xp + kBM * kXS);      // [128] first tree: bound on the kq-th key
  // [128][2] grouped leaves: the row's own columns (in the listed-column area,
  // unused then: a grouped tile is one column tile, so xcl is off)
  int16_t* rcol = reinterpret_cast<int16_t*>(xp);
  uint64_t* mbar = reinterpret_cast<uint64_t*>(tcap + kBM);
  uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(mbar + 1);
  int* status = reinterpret_cast<int*>(tmem_slot + 1);

  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int64_t leaf = blockIdx.x / qtiles;
  const int qt = (int)(blockIdx.x - leaf * qtiles);
  int64_t lo, hi, blo, bhi;
  if (ftab) {  // explicit leaf table (reference-rule trees)
    const int64_t* e = ftab + 4 * leaf;
    lo = e[0];
    hi = e[1];
    blo = e[2];
    bhi = e[3];
  } else if (glog == 0) {
    int64_t j;
    const SegEntry seg = segs.leaf(leaf, &j);
    leaf_block(seg, j, k, &lo, &hi, &blo, &bhi);
  } else {
    // 2^glog sibling leaves, each its own block (the host checks that every
    // leaf holds k+1 points), as one tile: a row keeps only its own leaf's
    // columns (rcol)
    int64_t j;
    const SegEntry seg = segs.leaf(leaf << glog, &j);
    lo = blo = seg.off + node_lo(seg.n, seg.depth, j);
    hi = bhi = seg.off + node_lo(seg.n, seg.depth, j + (int64_t(1) << glog));
    if (threadIdx.x < kBM) {
      const int64_t p = lo + threadIdx.x;
      int64_t a = lo, b = lo;
      for (int g = 0; g < (1 << glog); ++g) {
        const int64_t e = seg.off + node_lo(seg.n, seg.depth, j + g + 1);
        if (p < e) {
          b = e;
          break;
        }
        a = e;
      }
      rcol[2 * threadIdx.x] = (int16_t)(a - blo);
      rcol[2 * threadIdx.x + 1] = (int16_t)(b - blo);
    }
  }
  const int nq = (int)(hi - lo);
  const int q0 = qt * kBM;
  if (q0 >= nq) return;  // whole block, before any barrier or allocation
  const int mq = min(kBM, nq - q0);
  const int nb = (int)(bhi - blo);
  const int ntiles = (nb + kBN - 1) / kBN;
  // Listed ids are located up front only in blocks of several tiles: in a
  // one-tile block the few survivors are cheaper to check by the merge's ballot.
  const bool xcl = !FIRST && inv != nullptr && nb > kBN && nb <= kXMaxBlock;  // block-uniform
  const bool pre = FIRST && nb >= kPrepassMin && glog == 0;
  const int nsteps = pre ? 2 * ntiles : ntiles;
  const float kInf = __int_as_float(0x7F800000);
  const float kMaxF = __int_as_float(0x7F7FFFFF);
  const uint32_t bar = smem_u32(mbar);
  float* gm = Lk;  // [128][kGS] group minima during pass 0 (spans Lk and Li)

  if (warp == 0) {
    if (lane == 0) {
      mbar_init(bar, 1);
      asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
      *status = 0;
    }
    __syncwarp();
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;\n" ::"r"(smem_u32(tmem_slot)),
                 "r"(kTmemCols));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;\n" ::);
  }
  if (tid < kBM) {
    const int32_t id = tid < mq ? perm[lo + q0 + tid] : -1;
    qid[tid] = id;
    qn[tid] = (METRIC == KNN_METRIC_EUCLIDEAN && id >= 0) ? norms2[id] : 0.f;
    tcap[tid] = kInf;
  }
  // candidates of step s (warps 0-3, whole warps) into slot s mod 3;
  // fetch_cols loads them into registers (a step ahead), put_cols stores them
  int32_t nid = -1;
  float nnv = 0.f;
  auto fetch_cols = [&](int s) {
    const int c0 = (s % ntiles) * kBN, mc = min(kBN, nb - c0);
    nid = tid < mc ? perm[blo + c0 + tid] : -1;
    nnv = (METRIC == KNN_METRIC_EUCLIDEAN && nid >= 0) ? norms2[nid] : 0.f;
  };
  auto put_cols = [&](int s) {
    cid3[(s % 3) * kBN + tid] = nid;
    cn3[(s % 3) * kBN + tid] = nid >= 0 ? nnv : kInf;
    // norms are >= 0, so their bit patterns order as unsigned integers
    const uint32_t wm = __reduce_max_sync(0xFFFFFFFFu, __float_as_uint(nnv));
    if (lane == 0) cmax3[(s % 3) * 4 + warp] = __uint_as_float(wm);
  };
  if (tid < kBN) {
    fetch_cols(0);
    put_cols(0);
    if (nsteps > 1) fetch_cols(1);
  }
  __syncthreads();
  stage_operand<NCH>(opA, Xb, qid);
  stage_operand<NCH>(opB, Xb, cid3);
  if (pre) {
    for (int e = tid; e < kBM * kGS; e += kUThreads) gm[e] = kInf;
  } else {
    // warp w: rows w + 8 i, lane s: entry s; all loads issued before use
    float lkr[kBM / 8];
    uint32_t lir[kBM / 8];
#pragma unroll
    for (int i = 0; i < kBM / 8; ++i) {
      const int32_t id = qid[warp + 8 * i];
      const bool live = id >= 0 && lane < kq;
      lkr[i] = live ? akey[(size_t)id * kq + lane] : kInf;
      lir[i] = live ? aid[(size_t)id * kq + lane] : kNoId;
    }
#pragma unroll
    for (int i = 0; i < kBM / 8; ++i) {
      Lk[(warp + 8 * i) * kLS + lane] = lkr[i];
      Li[(warp + 8 * i) * kLS + lane] = lir[i];
    }
    if (xcl) {
      // the listed ids' columns in this block, sorted per row: the 16 rows'
      // bitonic networks interleaved stage by stage, two rows' 16-bit
      // positions packed per register (halfword min / max)
      uint32_t pk[kBM / 16];
#pragma unroll
      for (int i = 0; i < kBM / 8; ++i) {
        uint32_t p = kXEnd;
        if (lir[i] != kNoId) {
          const int64_t q = (int64_t)inv[lir[i]] - blo;
          if (q >= 0 && q < nb) p = (uint32_t)q;
        }
        if (i & 1) pk[i >> 1] |= p << 16;
        else pk[i >> 1] = p;
      }
#pragma unroll
      for (int size = 2; size <= 32; size <<= 1) {
#pragma unroll
        for (int m = size >> 1; m >= 1; m >>= 1) {
          const bool keep_min = ((lane & size) == 0) == ((lane & m) == 0);
#pragma unroll
          for (int j = 0; j < kBM / 16; ++j) {
            const uint32_t o = __shfl_xor_sync(0xFFFFFFFFu, pk[j], m);
            pk[j] = keep_min ? __vminu2(pk[j], o) : __vmaxu2(pk[j], o);
          }
        }
      }
#pragma unroll
      for (int i = 0; i < kBM / 8; ++i) {
        xp[(warp + 8 * i) * kXS + lane] = (uint16_t)((i & 1) ? (pk[i >> 1] >> 16) : (pk[i >> 1] & 0xFFFFu));
        if (lane == 0) xp[(warp + 8 * i) * kXS + 32] = (uint16_t)kXEnd;
      }
    }
  }
  int xptr = 0;  // this thread's next entry of its row's listed columns

  // step 0's MMA
  asm volatile("cp.async.wait_all;\n" ::: "memory");
  asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory");
  asm volatile("tcgen05.fence::before_thread_sync;\n" ::: "memory");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory");
  const uint32_t tmem = *tmem_slot;
  auto issue_mma = [&](int s) {  // thread 0: operands staged, previous MMA waited for
    if (*reinterpret_cast<volatile int*>(err) != 0) {
      *status = 2;  // another block failed: issue nothing more
      return;
    }
    const uint32_t a0 = smem_u32(opA), b0 = smem_u32(opB);
    const uint32_t d = tmem + (uint32_t)((s & 1) * kBN);
    for (int ch = 0; ch < nchunks; ++ch)
#pragma unroll
      for (int kk = 0; kk < kKC / 16; ++kk) {
        const uint32_t off = ch * kChunkBytes + kk * 32;
        umma_f16(d, desc_sw128(a0 + off), desc_sw128(b0 + off), idesc, (ch | kk) != 0 ? 1u : 0u);
      }
    umma_commit(bar);
  };
  if (tid == 0) issue_mma(0);

  // Per step: [A] MMA(s) done -> stage B(s+1) -> epilogue over the tile's 128
  // columns (two 32-column slices per thread) -> [B] -> MMA(s+1) issued ->
  // merge of the step's survivors -> the next step's [A].  Candidate ids and
  // norms live in three slots (step s in slot s mod 3): the merge of step s
  // still reads its slot while step s+1 fills slot (s+2) mod 3.
  uint32_t phase = 0;
  for (int s = 0; s < nsteps; ++s) {
    const int pass = pre && s < ntiles ? 0 : 1;
    const int c0 = (s % ntiles) * kBN, mc = min(kBN, nb - c0);
    const bool has_next = s + 1 < nsteps;
    if (has_next && tid < kBN) {
      put_cols(s + 1);
      if (s + 2 < nsteps) fetch_cols(s + 2);
    }
    if (tid == 0 && *status == 0 && !mbar_wait_bounded(bar, phase)) {
      *status = 1;
      atomicExch(err, 1);     // this build's blocks stop issuing MMAs
      atomicOr(err + 1, 1);   // sticky until the host reports it
      mbar_wait_bounded(bar, phase);  // let the MMAs drain before TMEM is freed
    }
    phase ^= 1u;
    __syncthreads();  // [A]
    asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory");
    if (*status != 0) break;  // uniform: read after the barrier
    // step s's MMA has completed: B is free for step s + 1
    if (has_next) stage_operand<NCH>(opB, Xb, cid3 + ((s + 1) % 3) * kBN);
    const int32_t* cid = cid3 + (s % 3) * kBN;
    const float* cn = cn3 + (s % 3) * kBN;
    const float* cmx = cmax3 + (s % 3) * 4;
    const float cm = fmaxf(fmaxf(cmx[0], cmx[1]), fmaxf(cmx[2], cmx[3]));
    const uint32_t tbuf = tmem + (uint32_t)((s & 1) * kBN);
    const int quarter = warp & 3, half = warp >> 2;
    const uint32_t tq = tbuf + ((uint32_t)(quarter * 32) << 16);  // this warp's lane quarter
    const int r = quarter * 32 + lane;
    // the row's filter bound (pass 1), from its list tail at the step's start
    float thr = 0.f;
    if (pass == 1) {
      // Row filter, a superset of what the exact rule (key <= the row's
      // list tail tk) can admit: key' = |y|^2 - 2 x.y (EUCLIDEAN) or
      // -x.y (COSINE) against thr = tk - |x|^2 (or tk - 1) widened by
      // 2^-21 (|tk| + |x|^2 + max|y|^2), which bounds the rounding of
      // both the key and the threshold.  Padding columns have key' =
      // +inf, a row outside the block thr = -inf, a list with free slots
      // thr = FLT_MAX.  A bound from the step's start is looser than the
      // current tail, never tighter, so the filter stays a superset.
      const float tk = FIRST ? fminf(Lk[r * kLS + kq - 1], tcap[r]) : Lk[r * kLS + kq - 1];
      if (r >= mq) thr = -kInf;
      else if (tk == kInf) thr = kMaxF;
      else if (METRIC == KNN_METRIC_EUCLIDEAN) {
        const float myn = qn[r];
        thr = fminf((tk - myn) + kSlack * (fabsf(tk) + myn + cm), kMaxF);
      } else {
        thr = fminf((tk - 1.f) + kSlack * (fabsf(tk) + 2.f), kMaxF);
      }
    }
#pragma unroll 1
    for (int ri = 0; ri < 2; ++ri) {
      const int col0 = ri * kRound + half * 32;  // this thread's 32 columns
      if (ri * kRound >= mc) {                   // warp-uniform: no candidates in this round
        if (pass == 1) msk[r * 4 + ri * 2 + half] = 0u;
        continue;
      }
      uint32_t v[32];
      tmem_ld32(tq + (uint32_t)col0, v);
      const float4* cn4 = reinterpret_cast<const float4*>(cn + col0);
      if (FIRST && pass == 0) {
        // smallest exact key of these 32 columns (the row's own column
        // left out) into the slice's group
        const float myn = qn[r];
        const int64_t sb = (lo + q0 + r) - blo - c0 - col0;
        float m = kInf;
#pragma unroll
        for (int q = 0; q < 8; ++q) {
          const float4 c = cn4[q];
          const float cc[4] = {c.x, c.y, c.z, c.w};
#pragma unroll
          for (int e = 0; e < 4; ++e) {
            const float dot = __uint_as_float(v[4 * q + e]);
            const float key = METRIC == KNN_METRIC_EUCLIDEAN ? __fmaf_rn(-2.f, dot, __fadd_rn(myn, cc[e]))
                                                             : __fsub_rn(1.f + cc[e], dot);
            m = (sb == 4 * q + e) ? m : fminf(m, key);
          }
        }
        const int g = ((c0 / kBN) * 4 + ri * 2 + half) & (kGroups - 1);
        gm[r * kGS + g] = fminf(gm[r * kGS + g], m);
      } else {
        // bit j of neg = sign of thr - key'_j, shifted in from column 31 down
        uint32_t neg = 0;
#pragma unroll
        for (int q = 7; q >= 0; --q) {
          const float4 c = cn4[q];
          const float cc[4] = {c.x, c.y, c.z, c.w};
#pragma unroll
          for (int e = 3; e >= 0; --e) {
            const float dot = __uint_as_float(v[4 * q + e]);
            const float kp =
                METRIC == KNN_METRIC_EUCLIDEAN ? __fmaf_rn(-2.f, dot, cc[e]) : __fsub_rn(cc[e], dot);
            neg = __funnelshift_l(__float_as_uint(__fsub_rn(thr, kp)), neg, 1);
          }
        }
        uint32_t mask = ~neg;
        // the row's own point (its leaf lies inside the block) never survives
        const int64_t selfbit = (lo + q0 + r) - blo - c0 - col0;
        if (selfbit >= 0 && selfbit < 32) mask &= ~(1u << (int)selfbit);
        if (glog) {  // grouped leaves: the row's own leaf's columns only
          const int a = min(max((int)rcol[2 * r] - (c0 + col0), 0), 32);
          const int b = min(max((int)rcol[2 * r + 1] - (c0 + col0), 0), 32);
          mask &= (uint32_t)(((1ull << b) - 1ull) ^ ((1ull << a) - 1ull));
        }
        if (xcl) {
          // listed ids among these 32 columns: walk the row's sorted
          // positions (each thread's columns only increase)
          const int lo_c = c0 + col0;
          uint32_t ex = 0;
          int p = xp[r * kXS + xptr];
          while (p < lo_c + 32) {
            if (p >= lo_c) ex |= 1u << (p - lo_c);
            p = xp[r * kXS + (++xptr)];
          }
          mask &= ~ex;
        }
        msk[r * 4 + ri * 2 + half] = mask;
      }
    }
    // step s + 1's operand (staged since [A]) lands before [B]; its MMA is
    // issued after [B] and runs while this step's survivors are merged
    if (has_next) {
      asm volatile("cp.async.wait_all;\n" ::: "memory");
      asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory");
    }
    asm volatile("tcgen05.fence::before_thread_sync;\n" ::: "memory");
    __syncthreads();  // [B]
    asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory");
    if (has_next && tid == 0) issue_mma(s + 1);
    if (pass == 1) {
      // The quarter's rows with survivors (one ballot) alternate between
      // its two warps; survivors' products come from the warp's lane
      // quarter of tensor memory.
      const int rowq = quarter * 32 + lane;
      const bool has = rowq < mq && (msk[rowq * 4] | msk[rowq * 4 + 1] | msk[rowq * 4 + 2] | msk[rowq * 4 + 3]) != 0;
      const uint32_t all = __ballot_sync(0xFFFFFFFFu, has);
      const bool mine = has && (__popc(all & ((1u << lane) - 1u)) & 1) == half;
      uint32_t rows = __ballot_sync(0xFFFFFFFFu, mine);
      while (rows) {
        const int ql = __ffs(rows) - 1;  // row within the quarter
        const int qq = quarter * 32 + ql;
        rows &= rows - 1;
        float lk = Lk[qq * kLS + lane];
        uint32_t li = Li[qq * kLS + lane];
        const float myn = qn[qq];
#pragma unroll 1
        for (int h = 0; h < 4; ++h) {
          uint32_t bal = msk[qq * 4 + h];
          if (bal == 0) continue;
          const int cb = h * 32;  // the slice's first column in the tile
          if (FIRST && __popc(bal) >= kBulkMerge) {
            // lane j <- product of column cb + j of row qq
            uint32_t v[32];
            tmem_ld32(tq + (uint32_t)cb, v);
            float dot = 0.f;
#pragma unroll
            for (int j = 0; j < 32; ++j) {
              const float t = __shfl_sync(0xFFFFFFFFu, __uint_as_float(v[j]), ql);
              if (lane == j) dot = t;
            }
            float ck = kInf;
            uint32_t ci = kNoId;
            if ((bal >> lane) & 1u) {
              ck = METRIC == KNN_METRIC_EUCLIDEAN ? __fmaf_rn(-2.f, dot, __fadd_rn(myn, cn[cb + lane]))
                                                  : __fsub_rn(1.f, dot);
              ci = (uint32_t)cid[cb + lane];
            }
            warp_bitonic_sort32(ck, ci);
            warp_merge_lower(lk, li, ck, ci);
            continue;
          }
          while (bal) {
            const int j = __ffs(bal) - 1;
            bal &= bal - 1;
            const float dot = __shfl_sync(0xFFFFFFFFu, __uint_as_float(tmem_ld1(tq + (uint32_t)(cb + j))), ql);
            const float k1 = METRIC == KNN_METRIC_EUCLIDEAN ? __fmaf_rn(-2.f, dot, __fadd_rn(myn, cn[cb + j]))
                                                            : __fsub_rn(1.f, dot);
            const uint32_t i1 = (uint32_t)cid[cb + j];
            const bool dup = !FIRST && !xcl && __ballot_sync(0xFFFFFFFFu, lane < kq && li == i1) != 0;
            if (!dup) warp_insert1(lk, li, k1, i1);
          }
        }
        Lk[qq * kLS + lane] = lk;
        Li[qq * kLS + lane] = li;
      }
    }
    asm volatile("tcgen05.fence::before_thread_sync;\n" ::: "memory");
    if (FIRST && pass == 0 && s == ntiles - 1) {
      // bound per row: the kq-th smallest of its group minima (warp w: rows
      // w + 8 i, four rows' networks interleaved).  Each row's 64 minima:
      // lanes' first halves sorted ascending, second halves descending, their
      // lane-wise minima are the 32 smallest (a bitonic sequence), merged.
      // Then the lists start empty for pass 1.
      for (int i0 = 0; i0 < kBM / 8; i0 += 4) {
        float a[4], b[4];
#pragma unroll
        for (int i = 0; i < 4; ++i) {
          const int qq = warp + 8 * (i0 + i);
          a[i] = gm[qq * kGS + lane];
          b[i] = gm[qq * kGS + 32 + lane];
        }
#pragma unroll
        for (int size = 2; size <= 32; size <<= 1) {
#pragma unroll
          for (int m = size >> 1; m >= 1; m >>= 1) {
            const bool keep_min = ((lane & size) == 0) == ((lane & m) == 0);
#pragma unroll
            for (int i = 0; i < 4; ++i) {
              const float oa = __shfl_xor_sync(0xFFFFFFFFu, a[i], m);
              const float ob = __shfl_xor_sync(0xFFFFFFFFu, b[i], m);
              a[i] = keep_min ? fminf(a[i], oa) : fmaxf(a[i], oa);
              b[i] = keep_min ? fmaxf(b[i], ob) : fminf(b[i], ob);
            }
          }
        }
#pragma unroll
        for (int i = 0; i < 4; ++i) a[i] = fminf(a[i], b[i]);
#pragma unroll
        for (int m = 16; m >= 1; m >>= 1) {
          const bool keep_min = (lane & m) == 0;
#pragma unroll
          for (int i = 0; i < 4; ++i) {
            const float o = __shfl_xor_sync(0xFFFFFFFFu, a[i], m);
            a[i] = keep_min ? fminf(a[i], o) : fmaxf(a[i], o);
          }
        }
#pragma unroll
        for (int i = 0; i < 4; ++i) {
          const float t = __shfl_sync(0xFFFFFFFFu, a[i], kq - 1);
          if (lane == 0) tcap[warp + 8 * (i0 + i)] = t;
        }
      }
      __syncthreads();
      for (int e = tid; e < kBM * kLS; e += kUThreads) {
        Lk[e] = kInf;
        Li[e] = kNoId;
      }
    }
  }
  // the last step's merge is ordered before the write-back only by this barrier
  __syncthreads();
  if (*status == 0) {
    for (int e = tid; e < kBM * 32; e += kUThreads) {
      const int r = e >> 5, s = e & 31;
      const int32_t id = qid[r];
      if (id >= 0 && s < kq) {
        akey[(size_t)id * kq + s] = Lk[r * kLS + s];
        aid[(size_t)id * kq + s] = Li[r * kLS + s];
      }
    }
  }
  asm volatile("tcgen05.fence::before_thread_sync;\n" ::: "memory");
  __syncthreads();
  if (warp == 0) {
    __syncwarp();
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;\n" ::"r"(*tmem_slot), "r"(kTmemCols));
  }
}

// inv[order[i]] = i: the position of each point in a tree's order.
__global__ void k_inverse_order(const int32_t* __restrict__ order, int64_t n, int32_t* __restrict__ inv) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
    inv[order[i]] = (int32_t)i;
}

// Largest |x| over the rows (non-negative floats order as their bit patterns).
__global__ void k_max_abs(const float* __restrict__ X, int64_t count, unsigned int* __restrict__ out) {
  float m = 0.f;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < count; i += (int64_t)gridDim.x * blockDim.x)
    m = fmaxf(m, fabsf(X[i]));
  m = __uint_as_float(__reduce_max_sync(0xFFFFFFFFu, __float_as_uint(m)));
  if ((threadIdx.x & 31) == 0) atomicMax(out, __float_as_uint(m));
}

__device__ __forceinline__ uint16_t to_operand(float v, bool f16) {
  return f16 ? __half_as_ushort(__float2half_rn(v)) : __bfloat16_as_ushort(__float2bfloat16_rn(v));
}
__device__ __forceinline__ float from_operand(uint16_t b, bool f16) {
  return f16 ? __half2float(__ushort_as_half(b)) : __bfloat162float(__ushort_as_bfloat16(b));
}

// 16-bit operand copy: rows of Kp BF16 or FP16 values (zero padded), COSINE
// rows divided by their FP32 norm first; norms2 = |row|^2 of the rounded
// values (EUCLIDEAN).  FP16 EUCLIDEAN rows are first multiplied by the power
// of two 2^e that brings the largest |x| (maxabs) into [2^14, 2^15), inside
// the FP16 range: a power-of-two scale is exact, scales every key of the tile
// stage by the same 2^2e and so keeps its ranking (the re-rank uses X).
__global__ void k_to_operand(const float* __restrict__ X, int64_t n, int d, int dpad, int Kp, int metric, bool f16,
                             const unsigned int* __restrict__ maxabs, const float* __restrict__ norms,
                             uint16_t* __restrict__ Xb, float* __restrict__ norms2) {
  const int64_t row = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int lane = threadIdx.x & 31;
  if (row >= n) return;
  float scale = 1.f;
  if (metric == KNN_METRIC_COSINE) {
    const float nr = norms[row];
    scale = nr > 0.f ? __frcp_rn(nr) : 0.f;
  } else if (f16) {
    const float m = __uint_as_float(*maxabs);
    int e = 0;
    if (m > 0.f && m < __int_as_float(0x7F800000)) {
      frexpf(m, &e);  // m in [2^(e-1), 2^e)
      e = 15 - e;     // m * 2^(15-e) in [2^14, 2^15)
      e = max(-126, min(126, e));
    }
    scale = ldexpf(1.f, e);
  }
  float s = 0.f;
  for (int c = lane; c < Kp; c += 32) {
    const float v = c < d ? X[(size_t)row * dpad + c] : 0.f;
    const uint16_t b = to_operand(__fmul_rn(v, scale), f16);
    Xb[(size_t)row * Kp + c] = b;
    const float f = from_operand(b, f16);
    s = __fmaf_rn(f, f, s);
  }
#pragma unroll
  for (int off = 16; off >= 1; off >>= 1) s = __fadd_rn(s, __shfl_xor_sync(0xFFFFFFFFu, s, off));
  if (lane == 0) norms2[row] = s;
}

// Exact FP32 keys (the reference's order) of each point's kq approximate
// candidates; the best k become the list, all flagged new.  One warp per point:
// the candidate rows are staged 64 dims at a time by 16-byte cp.async into an
// xor-swizzled tile (lane r reads row r conflict-free), one lane per candidate.
template <int METRIC>
__global__ void __launch_bounds__(256) k_rerank(const float* __restrict__ X, int64_t n, int d, int dpad,
                                                int k, int kq, const float* __restrict__ norms,
                                                const uint32_t* __restrict__ aid,
                                                float* __restrict__ rkey, uint32_t* __restrict__ rid) {
  extern __shared__ __align__(16) float rsm[];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int64_t i = (int64_t)blockIdx.x * (blockDim.x >> 5) + warp;
  float* xq = rsm + (size_t)warp * (dpad + 32 * 64 + 32);
  float* rows = xq + dpad;
  uint32_t* ids = reinterpret_cast<uint32_t*>(rows + 32 * 64);
  if (i >= n) return;
  const float kInf = __int_as_float(0x7F800000);
  const float4* xr = reinterpret_cast<const float4*>(X + (size_t)i * dpad);
  for (int c = lane; c < (dpad >> 2); c += 32) reinterpret_cast<float4*>(xq)[c] = xr[c];
  const uint32_t cj = lane < kq ? aid[(size_t)i * kq + lane] : kNoId;
  const bool valid = cj != kNoId;
  ids[lane] = cj;
  __syncwarp();
  float total = 0.f, part = 0.f;
  const int half = lane >> 4, c4 = lane & 15;
  for (int cd = 0; cd < d; cd += 64) {
    const int dim = cd + 4 * c4;
    for (int r = half; r < 32; r += 2) {
      const uint32_t id = ids[r];
      const bool ok = id != kNoId && dim < dpad;
      const float* src = X + (size_t)(id != kNoId ? id : 0) * dpad + (dim < dpad ? dim : 0);
      cp_async16(smem_u32(rows + r * 64 + ((c4 ^ (r & 7)) << 2)), src, ok ? 16 : 0);
    }
    asm volatile("cp.async.commit_group;\n" ::);
    asm volatile("cp.async.wait_all;\n" ::: "memory");
    __syncwarp();
    const int lim = min(64, d - cd);
    const float* myrow = rows + lane * 64;
    for (int q4 = 0; q4 < (lim + 3) >> 2; ++q4) {
      const float4 cv = *reinterpret_cast<const float4*>(myrow + ((q4 ^ (lane & 7)) << 2));
      const float4 qv = *reinterpret_cast<const float4*>(xq + cd + 4 * q4);
      part = acc_step<METRIC>(qv.x, cv.x, part);
      part = acc_step<METRIC>(qv.y, cv.y, part);
      part = acc_step<METRIC>(qv.z, cv.z, part);
      part = acc_step<METRIC>(qv.w, cv.w, part);
    }
    if (((cd + 64) & 255) == 0 || cd + 64 >= d) {
      total = __fadd_rn(total, part);
      part = 0.f;
    }
    __syncwarp();
  }
  float key = total;
  if (METRIC == KNN_METRIC_COSINE) key = valid ? cosine_key(total, norms[i], norms[cj]) : kInf;
  if (!valid) key = kInf;
  float kk = key;
  uint32_t ii = valid ? cj : kNoId;
  warp_bitonic_sort32(kk, ii);
  if (lane < k) {
    rkey[(size_t)i * k + lane] = kk;
    rid[(size_t)i * k + lane] = ii;
  }
}

size_t umma_smem_bytes(int Kp) {
  // alignment slack + A + B + lists + (qid, qn) + two steps' (cid, cn) + survivor masks + two
  // steps' norm maxima + listed columns + first-tree bounds + barrier words
  return 1024 + 2 * (size_t)(Kp / kKC) * kChunkBytes + (size_t)kBM * kLS * 8 + (size_t)kBM * 8 +
         (size_t)kBN * 3 * 8 + (size_t)kBM * 4 * 4 + 48 + (size_t)kBM * kXS * 2 + (size_t)kBM * 4 + 64;
}

int leaf_stage_umma(const UmmaLeafArgs& a, LaunchLog& log) {
  const int Kp = ((a.d + kKC - 1) / kKC) * kKC;
  if (Kp > 256 || a.kq > 32 || a.kq < a.k) return KNN_ERR_UNSUPPORTED;
  cudaStream_t st = a.stream;
  uint16_t* Xb = static_cast<uint16_t*>(a.Xb);
  // operand copy (FP16 EUCLIDEAN: the largest |x| first, for the row scale)
  if (a.f16 && a.metric == KNN_METRIC_EUCLIDEAN) {
    cudaMemsetAsync(a.maxabs, 0, sizeof(unsigned int), st);
    const int64_t cnt = a.n * (int64_t)a.dpad;
    k_max_abs<<<(unsigned)std::min<int64_t>((cnt + 255) / 256, 148 * 8), 256, 0, st>>>(a.X, cnt, a.maxabs);
    log.add();
  }
  k_to_operand<<<(unsigned)((a.n * 32 + 255) / 256), 256, 0, st>>>(a.X, a.n, a.d, a.dpad, Kp, a.metric, a.f16,
                                                                    a.maxabs, a.norms, Xb, a.norms2);
  log.add();
  const uint32_t idesc = idesc_for(a.f16);
  const size_t smem = umma_smem_bytes(Kp);
  const int64_t leaves = a.leaves;
  // 2^glog sibling leaves per tile (the caller checks it is allowed)
  const int glog = a.tc_group >= 4 ? 2 : a.tc_group == 2 ? 1 : 0;
  if (glog && (a.ftable || (a.maxleaf << glog) > kBM)) return KNN_ERR_UNSUPPORTED;
  const int qtiles = glog ? 1 : (int)((a.maxleaf + kBM - 1) / kBM);
  for (int t = 0; t < a.trees; ++t) {
    const int32_t* perm = a.perm + (size_t)t * a.n;
    const int64_t* ftab = a.ftable ? a.ftable + 4 * a.foff[t] : nullptr;
    const int64_t tleaves = a.ftable ? a.fcount[t] : (leaves >> glog);
    if (tleaves <= 0) {
      if (a.kev) {
        cudaEventRecord(a.kev[2 * t], st);
        cudaEventRecord(a.kev[2 * t + 1], st);
      }
      continue;
    }
    const unsigned grid = (unsigned)(tleaves * qtiles);
    const int32_t* inv = nullptr;
    if (t > 0 && a.inv && (a.ftable || a.maxblock > kBN)) {
      k_inverse_order<<<(unsigned)std::min<int64_t>((a.n + 255) / 256, 148 * 16), 256, 0, st>>>(perm, a.n, a.inv);
      log.add();
      inv = a.inv;
    }
#define KNN_TC_LAUNCH_N(M, F, N)                                                                          \
  do {                                                                                                    \
    cudaFuncSetAttribute(k_leaf_tc<M, F, N>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);    \
    k_leaf_tc<M, F, N><<<grid, kUThreads, smem, st>>>(Xb, idesc, a.segs, ftab, a.k, a.kq, qtiles, glog, perm, \
                                                      inv, a.norms2, a.akey, a.aid, a.err);             \
  } while (0)
#define KNN_TC_LAUNCH(M, F)                    \
  do {                                         \
    if (Kp == 64) KNN_TC_LAUNCH_N(M, F, 1);    \
    else if (Kp == 128) KNN_TC_LAUNCH_N(M, F, 2); \
    else if (Kp == 192) KNN_TC_LAUNCH_N(M, F, 3); \
    else KNN_TC_LAUNCH_N(M, F, 4);             \
  } while (0)
    if (a.kev) cudaEventRecord(a.kev[2 * t], st);
    if (a.metric == KNN_METRIC_EUCLIDEAN) {
      if (t == 0) KNN_TC_LAUNCH(KNN_METRIC_EUCLIDEAN, true);
      else KNN_TC_LAUNCH(KNN_METRIC_EUCLIDEAN, false);
    } else {
      if (t == 0) KNN_TC_LAUNCH(KNN_METRIC_COSINE, true);
      else KNN_TC_LAUNCH(KNN_METRIC_COSINE, false);
    }
    if (a.kev) cudaEventRecord(a.kev[2 * t + 1], st);
#undef KNN_TC_LAUNCH
#undef KNN_TC_LAUNCH_N
    log.add();
  }
  const size_t rsm = (size_t)8 * (a.dpad + 32 * 64 + 32) * sizeof(float);
  const unsigned rgrid = (unsigned)((a.n + 7) / 8);
  if (a.metric == KNN_METRIC_EUCLIDEAN) {
    cudaFuncSetAttribute(k_rerank<KNN_METRIC_EUCLIDEAN>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)rsm);
    k_rerank<KNN_METRIC_EUCLIDEAN><<<rgrid, 256, rsm, st>>>(a.X, a.n, a.d, a.dpad, a.k, a.kq, a.norms, a.aid, a.rkey, a.rid);
  } else {
    cudaFuncSetAttribute(k_rerank<KNN_METRIC_COSINE>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)rsm);
    k_rerank<KNN_METRIC_COSINE><<<rgrid, 256, rsm, st>>>(a.X, a.n, a.d, a.dpad, a.k, a.kq, a.norms, a.aid, a.rkey, a.rid);
  }
  log.add();
  return cudaPeekAtLastError() == cudaSuccess ? KNN_OK : KNN_ERR_CUDA;
}

}  // namespace knn
