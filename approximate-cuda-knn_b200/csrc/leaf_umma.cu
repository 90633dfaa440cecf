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
//     thread, accumulator 128 lanes x 128 columns of tensor memory;
//   * completion: tcgen05.commit -> mbarrier, waited with an iteration limit
//     (on expiry the block records an error, drains, frees TMEM and returns);
//   * epilogue: per 64-column round, tcgen05.ld 32x32b.x32 by all 8 warps (warp
//     w reads lane quarter w%4, 32 columns); three instructions per key filter
//     it against a slightly widened bound of the row's current last entry into
//     a survivor bit mask, then one warp per row computes its few survivors'
//     keys and inserts them into that query's sorted list (held in shared
//     memory for the whole block) with one ballot and one lane shift each.
#include <cuda_bf16.h>

#include <algorithm>

#include "knn_internal.cuh"
#include "knn_kernels.cuh"

namespace knn {

namespace {
constexpr int kBM = 128;
constexpr int kBN = 128;
constexpr int kKC = 64;               // bf16 per 128-byte swizzled row
constexpr int kChunkBytes = kBM * 128; // one 128 x 64 bf16 operand chunk
constexpr uint32_t kTmemCols = 128;
constexpr int kUThreads = 256;
constexpr int kRound = 64;          // tile columns per epilogue round
constexpr int kBulkMerge = 12;      // first tree: survivors in a half round from which sort + merge pays
constexpr float kSlack = 4.76837158203125e-07f;  // 2^-21: filter widening, eight units of FP32 rounding
// Listed candidates inside the block, per row: sorted 16-bit column positions
// ending in kXEnd (blocks of up to kXMaxBlock columns).
constexpr int kXS = 34;
constexpr uint32_t kXEnd = 0xFFFFu;
constexpr int kXMaxBlock = 65000;
// First tree: blocks of at least kPrepassMin columns get a bounding pass; its
// group minima (64 per row, row stride kGS) use the list area.
constexpr int kPrepassMin = 1024;
constexpr int kGroups = 64;
constexpr int kGS = kGroups + 1;
// Round products live in the B-operand region once the tile's MMA has completed:
// 128 rows x 64 floats (32 KB).
constexpr int kKsBytes = kBM * kRound * 4;
constexpr int kLS = 33;              // list row stride (row owners hit distinct banks)
// A 128x128x256 tile finishes in about a microsecond; 2^16 polls with 32 ns
// sleeps (a few ms) is far beyond that, and keeps a failing launch short.
constexpr uint32_t kSpinLimit = 1u << 16;

// Instruction descriptor: D f32 (bits 4-5 = 1), A bf16 (7-9 = 1), B bf16
// (10-12 = 1), A and B K-major (15, 16 = 0), N>>3 at 17-22, M>>4 at 24-28.
constexpr uint32_t kIdesc = (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(kBN >> 3) << 17) |
                            ((uint32_t)(kBM >> 4) << 24);

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

__device__ __forceinline__ void umma_bf16(uint32_t tmem_d, uint64_t da, uint64_t db, uint32_t accumulate) {
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "setp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t}\n" ::"r"(tmem_d),
      "l"(da), "l"(db), "r"(kIdesc), "r"(accumulate), "r"(0u), "r"(0u), "r"(0u), "r"(0u));
}

__device__ __forceinline__ void umma_commit(uint32_t bar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];\n" ::"r"(bar)
               : "memory");
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

// Stage `rows` gathered rows (ids in `ids`, <0: zero row) of the BF16 copy into
// a K-major 128B-swizzled operand of Kp/64 chunks.
__device__ __forceinline__ void stage_operand(unsigned char* op, const __nv_bfloat16* __restrict__ Xb,
                                              int Kp, const int32_t* ids) {
  const int units = kBM * (Kp / 8);  // 16-byte units
  const uint32_t base = smem_u32(op);
  for (int u = threadIdx.x; u < units; u += kUThreads) {
    const int r = u / (Kp / 8);
    const int c16 = u - r * (Kp / 8);  // 16-byte unit along K
    const int chunk = c16 >> 3, w = c16 & 7;
    const uint32_t dst = base + chunk * kChunkBytes + r * 128 + ((w ^ (r & 7)) << 4);
    const int32_t id = ids[r];
    const __nv_bfloat16* src = Xb + (size_t)(id < 0 ? 0 : id) * Kp + c16 * 8;
    cp_async16(dst, src, id < 0 ? 0 : 16);
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

// One block per (leaf, 128-query tile).  The 128 queries' lists stay in shared
// memory for the whole loop over candidate tiles (read once, written once);
// each 128x128 tensor-core tile is emptied in two 64-column rounds: epilogue
// (tcgen05.ld, a conservative per-row filter packed into survivor bit masks,
// raw products parked in shared memory) then a per-row merge that computes the
// survivors' keys and applies the exact rule.  Prologue, MMA issue, bounded
// wait and the tensor-memory loads follow the single-tile sequence that was
// checked on its own against a CPU product.
// FIRST: the launch of the first tree, whose lists start empty; a point then
// meets every candidate once, so no survivor can already be listed, and a
// half round with many survivors is sorted and merged into the list in one go.
// Later trees, with inv (the tree's inverse order): the block's columns that
// hold an id already in the row's list are found up front (inv of each listed
// id) and masked out of the survivors, so the merge needs no duplicate check;
// a candidate meets a row once per tree, so ids inserted during the block
// cannot come back.
template <int METRIC, bool FIRST>
__global__ void __launch_bounds__(kUThreads, 2)
    k_leaf_tc(const __nv_bfloat16* __restrict__ Xb, int Kp, SegView segs, const int64_t* __restrict__ ftab, int k,
              int kq,
              int qtiles, const int32_t* __restrict__ perm, const int32_t* __restrict__ inv,
              const float* __restrict__ norms2, float* __restrict__ akey, uint32_t* __restrict__ aid,
              int* __restrict__ err) {
  extern __shared__ __align__(1024) unsigned char smem_raw[];
  unsigned char* smem = (unsigned char*)(((uintptr_t)smem_raw + 1023) & ~(uintptr_t)1023);
  const int nchunks = Kp / kKC;
  unsigned char* opA = smem;
  unsigned char* opB = opA + nchunks * kChunkBytes;
  const int bbytes = max(nchunks * kChunkBytes, kKsBytes);
  float* Ks = reinterpret_cast<float*>(opB);                           // round products (reuses B)
  float* Lk = reinterpret_cast<float*>(opB + bbytes);                  // [128][kLS] list keys
  uint32_t* Li = reinterpret_cast<uint32_t*>(Lk + kBM * kLS);         // [128][kLS] list ids
  int32_t* qid = reinterpret_cast<int32_t*>(Li + kBM * kLS);
  int32_t* cid = qid + kBM;
  float* qn = reinterpret_cast<float*>(cid + kBN);
  float* cn = qn + kBM;  // candidate norms (EUCLIDEAN) or 0; +inf for padding columns
  uint32_t* msk = reinterpret_cast<uint32_t*>(cn + kBN);  // [128][2] survivor bits of the round
  float* cmax = reinterpret_cast<float*>(msk + kBM * 2);  // [4] largest candidate norm per warp
  uint16_t* xp = reinterpret_cast<uint16_t*>(cmax + 4);   // [128][kXS] listed columns
  float* tcap = reinterpret_cast<float*>(xp + kBM * kXS);  // [128] first tree: bound on the kq-th key
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
  } else {
    int64_t j;
    const SegEntry seg = segs.leaf(leaf, &j);
    leaf_block(seg, j, k, &lo, &hi, &blo, &bhi);
  }
  const int nq = (int)(hi - lo);
  const int q0 = qt * kBM;
  if (q0 >= nq) return;  // whole block, before any barrier or allocation
  const int mq = min(kBM, nq - q0);
  const int nb = (int)(bhi - blo);
  const bool xcl = !FIRST && inv != nullptr && nb <= kXMaxBlock;  // block-uniform
  const float kInf = __int_as_float(0x7F800000);
  const float kMaxF = __int_as_float(0x7F7FFFFF);
  const uint32_t bar = smem_u32(mbar);

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
  }
  // First tree, blocks of kPrepassMin columns or more: pass 0 runs the tiles
  // once to record each row's smallest exact key in each of kGroups groups of
  // columns (32-column slices, wrapping).  The kq-th smallest group minimum is
  // the key of kq distinct candidates, so it bounds the kq-th key of the
  // final list; pass 1 filters against it from the first tile on, which
  // leaves a few dozen survivors per row instead of ~kq ln(columns / kq).
  const bool pre = FIRST && nb >= kPrepassMin;
  float* gm = Lk;  // [128][kGS] group minima during pass 0 (spans Lk and Li)
  if (tid < kBM) tcap[tid] = kInf;
  __syncthreads();
  if (pre) {
    for (int e = tid; e < kBM * kGS; e += kUThreads) gm[e] = kInf;
  } else {
    for (int e = tid; e < kBM * 32; e += kUThreads) {
      const int r = e >> 5, s = e & 31;
      const int32_t id = qid[r];
      const bool live = id >= 0 && s < kq;
      Lk[r * kLS + s] = live ? akey[(size_t)id * kq + s] : kInf;
      Li[r * kLS + s] = live ? aid[(size_t)id * kq + s] : kNoId;
    }
  }
  stage_operand(opA, Xb, Kp, qid);
  if (xcl) {
    // warp w: rows w, w + 8, ...; lane s: the row's s-th listed id
    uint32_t pos[kBM / 8];
#pragma unroll
    for (int i = 0; i < kBM / 8; ++i) {
      const int32_t id = qid[warp + 8 * i];
      pos[i] = (id >= 0 && lane < kq) ? aid[(size_t)id * kq + lane] : kNoId;
    }
#pragma unroll
    for (int i = 0; i < kBM / 8; ++i) {
      uint32_t p = kXEnd;
      if (pos[i] != kNoId) {
        const int64_t q = (int64_t)inv[pos[i]] - blo;
        if (q >= 0 && q < nb) p = (uint32_t)q;
      }
      pos[i] = p;
    }
#pragma unroll
    for (int i = 0; i < kBM / 8; ++i) {
      const uint32_t v = warp_sort32_u32(pos[i]);
      xp[(warp + 8 * i) * kXS + lane] = (uint16_t)v;
      if (lane == 0) xp[(warp + 8 * i) * kXS + 32] = (uint16_t)kXEnd;
    }
  }
  int xptr = 0;  // this thread's next entry of its row's listed columns

  uint32_t phase = 0;
  for (int pass = pre ? 0 : 1; pass < 2; ++pass) {
    for (int c0 = 0; c0 < nb; c0 += kBN) {
      const int mc = min(kBN, nb - c0);
      if (tid < kBN) {  // warps 0-3, whole warps
        const int32_t id = tid < mc ? perm[blo + c0 + tid] : -1;
        cid[tid] = id;
        const float nv = (METRIC == KNN_METRIC_EUCLIDEAN && id >= 0) ? norms2[id] : 0.f;
        cn[tid] = id >= 0 ? nv : kInf;
        // norms are >= 0, so their bit patterns order as unsigned integers
        const uint32_t wm = __reduce_max_sync(0xFFFFFFFFu, __float_as_uint(nv));
        if (lane == 0) cmax[warp] = __uint_as_float(wm);
      }
      __syncthreads();
      stage_operand(opB, Xb, Kp, cid);
      asm volatile("cp.async.wait_all;\n" ::: "memory");
      asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory");
      asm volatile("tcgen05.fence::before_thread_sync;\n" ::: "memory");
      __syncthreads();
      asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory");
      const uint32_t tmem = *tmem_slot;
      if (tid == 0) {
        if (*reinterpret_cast<volatile int*>(err) != 0) {
          *status = 2;  // another block failed: issue nothing more
        } else {
          const uint32_t a0 = smem_u32(opA), b0 = smem_u32(opB);
          for (int ch = 0; ch < nchunks; ++ch)
#pragma unroll
            for (int kk = 0; kk < kKC / 16; ++kk) {
              const uint32_t off = ch * kChunkBytes + kk * 32;
              umma_bf16(tmem, desc_sw128(a0 + off), desc_sw128(b0 + off), (ch | kk) != 0 ? 1u : 0u);
            }
          umma_commit(bar);
          if (!mbar_wait_bounded(bar, phase)) {
            *status = 1;
            atomicExch(err, 1);
            mbar_wait_bounded(bar, phase);  // let the MMAs drain before TMEM is freed
          }
        }
      }
      __syncthreads();
      phase ^= 1u;
      if (*status != 0) break;  // uniform: read after the barrier

      const float cm = fmaxf(fmaxf(cmax[0], cmax[1]), fmaxf(cmax[2], cmax[3]));
      for (int rb = 0; rb < mc; rb += kRound) {
        asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory");
        {
          const int quarter = warp & 3, half = warp >> 2;
          const int r = quarter * 32 + lane;
          const int col0 = rb + half * 32;
          uint32_t v[32];
          tmem_ld32(tmem + ((uint32_t)(quarter * 32) << 16) + (uint32_t)col0, v);
          if (FIRST && pass == 0) {
            // smallest exact key of these 32 columns (the row's own column
            // left out) into the slice's group
            const float4* cn4 = reinterpret_cast<const float4*>(cn + col0);
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
            const int g = ((c0 / kBN) * 4 + (rb / kRound) * 2 + half) & (kGroups - 1);
            gm[r * kGS + g] = fminf(gm[r * kGS + g], m);
          } else {
            // raw products for the merge: 16-byte chunks xor-swizzled by the row,
            // so that row-parallel writes and column-parallel reads hit distinct banks
            float4* ks4 = reinterpret_cast<float4*>(Ks) + r * (kRound / 4);
#pragma unroll
            for (int q = 0; q < 8; ++q)
              ks4[(half * 8 + q) ^ (r & 7)] = make_float4(__uint_as_float(v[4 * q]), __uint_as_float(v[4 * q + 1]),
                                                           __uint_as_float(v[4 * q + 2]), __uint_as_float(v[4 * q + 3]));
            // Row filter, a superset of what the exact rule (key <= the row's
            // current last entry tk) can admit: key' = |y|^2 - 2 x.y (EUCLIDEAN)
            // or -x.y (COSINE) against thr = tk - |x|^2 (or tk - 1) widened by
            // 2^-21 (|tk| + |x|^2 + max|y|^2), which bounds the rounding of both
            // the key and the threshold.  Padding columns have key' = +inf, a row
            // outside the block thr = -inf, a list with free slots thr = FLT_MAX.
            const float tk = FIRST ? fminf(Lk[r * kLS + kq - 1], tcap[r]) : Lk[r * kLS + kq - 1];
            float thr;
            if (r >= mq) thr = -kInf;
            else if (tk == kInf) thr = kMaxF;
            else if (METRIC == KNN_METRIC_EUCLIDEAN) {
              const float myn = qn[r];
              thr = fminf((tk - myn) + kSlack * (fabsf(tk) + myn + cm), kMaxF);
            } else {
              thr = fminf((tk - 1.f) + kSlack * (fabsf(tk) + 2.f), kMaxF);
            }
            // bit j of neg = sign of thr - key'_j, shifted in from column 31 down
            const float4* cn4 = reinterpret_cast<const float4*>(cn + col0);
            uint32_t neg = 0;
#pragma unroll
            for (int q = 7; q >= 0; --q) {
              const float4 c = cn4[q];
              const float cc[4] = {c.x, c.y, c.z, c.w};
#pragma unroll
              for (int e = 3; e >= 0; --e) {
                const float dot = __uint_as_float(v[4 * q + e]);
                const float kp = METRIC == KNN_METRIC_EUCLIDEAN ? __fmaf_rn(-2.f, dot, cc[e]) : __fsub_rn(cc[e], dot);
                neg = __funnelshift_l(__float_as_uint(__fsub_rn(thr, kp)), neg, 1);
              }
            }
            uint32_t mask = ~neg;
            // the row's own point (its leaf lies inside the block) never survives
            const int64_t selfbit = (lo + q0 + r) - blo - c0 - col0;
            if (selfbit >= 0 && selfbit < 32) mask &= ~(1u << (int)selfbit);
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
            msk[r * 2 + half] = mask;
          }
        }
        asm volatile("tcgen05.fence::before_thread_sync;\n" ::: "memory");
        __syncthreads();
        if (pass == 1) {
          // one warp per query row with survivors (found by one ballot over the
          // warp's 16 rows); lane l holds the round's columns l and 32 + l.  The
          // survivor's exact key is computed here; few survivors are placed one
          // by one by warp_insert1 (which drops a candidate behind all 32
          // entries), many (first tree) by one sort and merge.
          {
            const int myrow = warp + (kUThreads / 32) * (lane & 15);
            const bool has = lane < 16 && myrow < mq && (msk[myrow * 2] | msk[myrow * 2 + 1]) != 0;
            uint32_t rows = __ballot_sync(0xFFFFFFFFu, has);
            while (rows) {
              const int qq = warp + (kUThreads / 32) * (__ffs(rows) - 1);
              rows &= rows - 1;
              const uint32_t m0 = msk[qq * 2], m1 = msk[qq * 2 + 1];
              float lk = Lk[qq * kLS + lane];
              uint32_t li = Li[qq * kLS + lane];
              const float myn = qn[qq];
#pragma unroll
              for (int h = 0; h < 2; ++h) {
                uint32_t bal = h ? m1 : m0;
                if (bal == 0) continue;
                const int col = h * 32 + lane;
                float ck = kInf;
                uint32_t ci = kNoId;
                if ((bal >> lane) & 1u) {
                  const float dot = Ks[qq * kRound + ((((col >> 2) ^ (qq & 7)) << 2) | (col & 3))];
                  ck = METRIC == KNN_METRIC_EUCLIDEAN ? __fmaf_rn(-2.f, dot, __fadd_rn(myn, cn[rb + col]))
                                                      : __fsub_rn(1.f, dot);
                  ci = (uint32_t)cid[rb + col];
                }
                if (FIRST && __popc(bal) >= kBulkMerge) {
                  warp_bitonic_sort32(ck, ci);
                  warp_merge_lower(lk, li, ck, ci);
                  continue;
                }
                while (bal) {
                  const int src = __ffs(bal) - 1;
                  bal &= bal - 1;
                  const float k1 = __shfl_sync(0xFFFFFFFFu, ck, src);
                  const uint32_t i1 = __shfl_sync(0xFFFFFFFFu, ci, src);
                  const bool dup = !FIRST && !xcl && __ballot_sync(0xFFFFFFFFu, lane < kq && li == i1) != 0;
                  if (!dup) warp_insert1(lk, li, k1, i1);
                }
              }
              Lk[qq * kLS + lane] = lk;
              Li[qq * kLS + lane] = li;
            }
          }
          __syncthreads();
        }
      }
    }
    if (*status != 0) break;
    if (FIRST && pass == 0) {
      __syncthreads();
      // bound per row: the kq-th smallest of its group minima
      for (int qq = warp; qq < mq; qq += kUThreads / 32) {
        float a = gm[qq * kGS + lane], b = gm[qq * kGS + 32 + lane];
        uint32_t ia = lane, ib = 32 + lane;
        warp_bitonic_sort32(a, ia);
        warp_bitonic_sort32(b, ib);
        warp_merge_pair(a, ia, b, ib);
        const float t = __shfl_sync(0xFFFFFFFFu, a, kq - 1);
        if (lane == 0) tcap[qq] = t;
      }
      __syncthreads();
      for (int e = tid; e < kBM * kLS; e += kUThreads) {
        Lk[e] = kInf;
        Li[e] = kNoId;
      }
    }
  }
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

// BF16 operand copy: rows of Kp bf16 (zero padded), COSINE rows divided by
// their FP32 norm first; norms2 = |row|^2 of the BF16 values (EUCLIDEAN).
__global__ void k_to_bf16(const float* __restrict__ X, int64_t n, int d, int dpad, int Kp, int metric,
                          const float* __restrict__ norms, __nv_bfloat16* __restrict__ Xb,
                          float* __restrict__ norms2) {
  const int64_t row = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int lane = threadIdx.x & 31;
  if (row >= n) return;
  float scale = 1.f;
  if (metric == KNN_METRIC_COSINE) {
    const float nr = norms[row];
    scale = nr > 0.f ? __frcp_rn(nr) : 0.f;
  }
  float s = 0.f;
  for (int c = lane; c < Kp; c += 32) {
    const float v = c < d ? X[(size_t)row * dpad + c] : 0.f;
    const __nv_bfloat16 b = __float2bfloat16_rn(metric == KNN_METRIC_COSINE ? __fmul_rn(v, scale) : v);
    Xb[(size_t)row * Kp + c] = b;
    const float f = __bfloat162float(b);
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
  // alignment slack + A + B (also the round products) + lists + (qid, cid, qn, cn) + survivor
  // masks + per-warp norm maxima + listed columns + first-tree bounds + barrier words
  const size_t bbytes = std::max((size_t)(Kp / kKC) * kChunkBytes, (size_t)kKsBytes);
  return 1024 + (size_t)(Kp / kKC) * kChunkBytes + bbytes + (size_t)kBM * kLS * 8 +
         (size_t)(kBM + kBN) * 8 + (size_t)kBM * 2 * 4 + 16 + (size_t)kBM * kXS * 2 + (size_t)kBM * 4 + 64;
}

int leaf_stage_umma(const UmmaLeafArgs& a, LaunchLog& log) {
  const int Kp = ((a.d + kKC - 1) / kKC) * kKC;
  if (Kp > 256 || a.kq > 32 || a.kq < a.k) return KNN_ERR_UNSUPPORTED;
  cudaStream_t st = a.stream;
  __nv_bfloat16* Xb = static_cast<__nv_bfloat16*>(a.Xb);
  // operand copy
  k_to_bf16<<<(unsigned)((a.n * 32 + 255) / 256), 256, 0, st>>>(a.X, a.n, a.d, a.dpad, Kp, a.metric,
                                                                 a.norms, Xb, a.norms2);
  log.add();
  const size_t smem = umma_smem_bytes(Kp);
  const int64_t leaves = a.leaves;
  const int qtiles = (int)((a.maxleaf + kBM - 1) / kBM);
  for (int t = 0; t < a.trees; ++t) {
    const int32_t* perm = a.perm + (size_t)t * a.n;
    const int64_t* ftab = a.ftable ? a.ftable + 4 * a.foff[t] : nullptr;
    const int64_t tleaves = a.ftable ? a.fcount[t] : leaves;
    if (tleaves <= 0) continue;
    const unsigned grid = (unsigned)(tleaves * qtiles);
    const int32_t* inv = nullptr;
    if (t > 0 && a.inv) {
      k_inverse_order<<<(unsigned)std::min<int64_t>((a.n + 255) / 256, 148 * 16), 256, 0, st>>>(perm, a.n, a.inv);
      log.add();
      inv = a.inv;
    }
#define KNN_TC_LAUNCH(M, F)                                                                               \
  do {                                                                                                    \
    cudaFuncSetAttribute(k_leaf_tc<M, F>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);       \
    k_leaf_tc<M, F><<<grid, kUThreads, smem, st>>>(Xb, Kp, a.segs, ftab, a.k, a.kq, qtiles, perm, inv, a.norms2, \
                                                   a.akey, a.aid, a.err);                                \
  } while (0)
    if (a.metric == KNN_METRIC_EUCLIDEAN) {
      if (t == 0) KNN_TC_LAUNCH(KNN_METRIC_EUCLIDEAN, true);
      else KNN_TC_LAUNCH(KNN_METRIC_EUCLIDEAN, false);
    } else {
      if (t == 0) KNN_TC_LAUNCH(KNN_METRIC_COSINE, true);
      else KNN_TC_LAUNCH(KNN_METRIC_COSINE, false);
    }
#undef KNN_TC_LAUNCH
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
