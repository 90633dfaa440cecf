// Learned split directions.  A small MLP
//
//   f(x) = W2 gelu(W1 s(x) + b1) + b2,   d -> 256 -> 64,
//   s(x) = (u(x) - mean) * inv_std        (per-dimension, from the sample;
//                                          u(x) = x/|x| for COSINE, else x),
//   gelu(a) = 0.5 a (1 + tanh(sqrt(2/pi) (a + 0.044715 a^3)))
//
// is trained on the GPU with a triplet (contrastive) loss on the k-NN graph
// that the plain method builds for a sample of the points:
//
//   loss = mean_b max(0, margin + |f(a) - f(p)|^2 - |f(a) - f(n)|^2)
//
// (a: a sample point; p: one of its graph neighbours of rank < gk/2; n: either
// a random sample point or a graph neighbour of rank >= gk/2), with Adam.  The
// trees are then built on the 64-dim embeddings f(x), so every split
// direction f(x_p2) - f(x_p1) lives in the learned space; leaf blocks and
// propagation still rank the original rows with exact keys.  The reference has
// no counterpart: its split directions use raw coordinates
// (euclideandistancematrixgpu.cu:2138-2164), which stays the default here.
//
// Everything is FP32 on CUDA cores (a 64x64-tile GEMM with bias/GELU epilogue,
// split-K partials reduced in a fixed order so training is deterministic).
#include <cmath>
#include <cstring>

#include "knn_internal.cuh"
#include "knn_kernels.cuh"

namespace knn {

namespace {
constexpr int kGT = 64;    // GEMM tile (rows and columns)
constexpr int kGK = 16;    // GEMM k-chunk
constexpr int kSplitK = 8; // k-splits of the weight-gradient GEMMs
constexpr float kSqrt2OverPi = 0.7978845608028654f;
constexpr float kGeluC = 0.044715f;
constexpr float kB1 = 0.9f, kB2 = 0.999f, kEps = 1e-8f;
}  // namespace

__device__ __forceinline__ float gelu_f(float a) {
  const float u = kSqrt2OverPi * (a + kGeluC * a * a * a);
  return 0.5f * a * (1.0f + tanhf(u));
}
__device__ __forceinline__ float gelu_grad(float a) {
  const float u = kSqrt2OverPi * (a + kGeluC * a * a * a);
  const float t = tanhf(u);
  const float du = kSqrt2OverPi * (1.0f + 3.0f * kGeluC * a * a);
  return 0.5f * (1.0f + t) + 0.5f * a * (1.0f - t * t) * du;
}

// C[i][j] = sum_{k in split z} A(i,k) B(j,k) (+ bias[j]) (GELU; pre-activation
// to P), with A(i,k) = A[i*sai + k*sak] and B(j,k) = B[j*sbj + k*sbk].  With
// gridDim.z > 1 block z writes the partial sum of its k range to
// C + z * M * ldc and no epilogue is applied.
__global__ void __launch_bounds__(256) k_gemm(int M, int N, int K, const float* __restrict__ A, int64_t sai,
                                              int64_t sak, const float* __restrict__ B, int64_t sbj,
                                              int64_t sbk, const float* __restrict__ bias, float* __restrict__ C,
                                              int64_t ldc, float* __restrict__ P, int gelu) {
  __shared__ __align__(16) float As[kGK][kGT + 4];
  __shared__ __align__(16) float Bs[kGK][kGT + 4];
  const int tid = threadIdx.x, ty = tid >> 4, tx = tid & 15;
  const int i0 = blockIdx.y * kGT, j0 = blockIdx.x * kGT;
  const int kper = (((K + (int)gridDim.z - 1) / (int)gridDim.z) + kGK - 1) / kGK * kGK;
  const int kb = blockIdx.z * kper, ke = min(K, kb + kper);
  // Loads walk whichever index is unit-stride.
  const bool a_k_fast = sak <= sai, b_k_fast = sbk <= sbj;
  float acc[4][4] = {};
  for (int k0 = kb; k0 < ke; k0 += kGK) {
    for (int e = tid; e < kGT * kGK; e += 256) {
      int r, kk;
      if (a_k_fast) { r = e / kGK; kk = e % kGK; } else { r = e % kGT; kk = e / kGT; }
      const int gi = i0 + r, gk = k0 + kk;
      As[kk][r] = (gi < M && gk < ke) ? A[(int64_t)gi * sai + (int64_t)gk * sak] : 0.f;
      if (b_k_fast) { r = e / kGK; kk = e % kGK; } else { r = e % kGT; kk = e / kGT; }
      const int gj = j0 + r, gk2 = k0 + kk;
      Bs[kk][r] = (gj < N && gk2 < ke) ? B[(int64_t)gj * sbj + (int64_t)gk2 * sbk] : 0.f;
    }
    __syncthreads();
#pragma unroll
    for (int kk = 0; kk < kGK; ++kk) {
      const float4 a = *reinterpret_cast<const float4*>(&As[kk][ty * 4]);
      const float4 b = *reinterpret_cast<const float4*>(&Bs[kk][tx * 4]);
      const float av[4] = {a.x, a.y, a.z, a.w}, bv[4] = {b.x, b.y, b.z, b.w};
#pragma unroll
      for (int p = 0; p < 4; ++p)
#pragma unroll
        for (int q = 0; q < 4; ++q) acc[p][q] = __fmaf_rn(av[p], bv[q], acc[p][q]);
    }
    __syncthreads();
  }
  float* Cz = C + (int64_t)blockIdx.z * M * ldc;
  const bool epilogue = gridDim.z == 1;
#pragma unroll
  for (int p = 0; p < 4; ++p)
#pragma unroll
    for (int q = 0; q < 4; ++q) {
      const int i = i0 + ty * 4 + p, j = j0 + tx * 4 + q;
      if (i >= M || j >= N) continue;
      float v = acc[p][q];
      if (epilogue && bias) v = __fadd_rn(v, bias[j]);
      if (epilogue && gelu) {
        if (P) P[(int64_t)i * ldc + j] = v;
        v = gelu_f(v);
      }
      Cz[(int64_t)i * ldc + j] = v;
    }
}

// out[g] = sum_z part[z][g], in order z = 0..splits-1.
__global__ void k_sum_splits(const float* __restrict__ part, int splits, int64_t count, float* __restrict__ out) {
  const int64_t g = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (g >= count) return;
  float s = part[g];
  for (int z = 1; z < splits; ++z) s = __fadd_rn(s, part[(int64_t)z * count + g]);
  out[g] = s;
}

// Column sums of G [M][ld] (bias gradients), first pass: block (x, z) sums
// columns [32x, 32x+32) over rows [z*rows, (z+1)*rows), 8 row lanes per column
// combined in a fixed order; part[z][j].  k_sum_splits finishes.
constexpr int kColSplits = 16;
__global__ void __launch_bounds__(256) k_colsum_part(const float* __restrict__ G, int M, int N, int64_t ld,
                                                     float* __restrict__ part) {
  __shared__ float red[8][33];
  const int tx = threadIdx.x & 31, ty = threadIdx.x >> 5;
  const int j = blockIdx.x * 32 + tx;
  const int rows = (M + (int)gridDim.z - 1) / (int)gridDim.z;
  const int r0 = blockIdx.z * rows, r1 = min(M, r0 + rows);
  float s = 0.f;
  if (j < N)
    for (int i = r0 + ty; i < r1; i += 8) s = __fadd_rn(s, G[(int64_t)i * ld + j]);
  red[ty][tx] = s;
  __syncthreads();
  if (ty == 0 && j < N) {
    float t = red[0][tx];
    for (int q = 1; q < 8; ++q) t = __fadd_rn(t, red[q][tx]);
    part[(int64_t)blockIdx.z * N + j] = t;
  }
}

// dA = dG * gelu'(pre), elementwise (in place allowed)
__global__ void k_gelu_back(const float* __restrict__ pre, const float* dG, int64_t count, float* dA) {
  const int64_t g = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (g < count) dA[g] = __fmul_rn(dG[g], gelu_grad(pre[g]));
}

// Triplet loss over Z = [anchors; positives; negatives] (3B rows of E), warp
// per triplet.  dZ = gradient of the mean loss; hinge[b] = the triplet's loss.
__global__ void k_triplet(const float* __restrict__ Z, int B, int E, float margin, float* __restrict__ dZ,
                          float* __restrict__ hinge) {
  const int b = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
  const int lane = threadIdx.x & 31;
  if (b >= B) return;
  const float* za = Z + (int64_t)b * E;
  const float* zp = Z + (int64_t)(B + b) * E;
  const float* zn = Z + (int64_t)(2 * B + b) * E;
  float dap = 0.f, dan = 0.f;
  for (int e = lane; e < E; e += 32) {
    const float u = za[e] - zp[e], w = za[e] - zn[e];
    dap = __fmaf_rn(u, u, dap);
    dan = __fmaf_rn(w, w, dan);
  }
#pragma unroll
  for (int off = 16; off >= 1; off >>= 1) {
    dap += __shfl_xor_sync(0xFFFFFFFFu, dap, off);
    dan += __shfl_xor_sync(0xFFFFFFFFu, dan, off);
  }
  const float l = margin + dap - dan;
  const float s = l > 0.f ? 2.0f / (float)B : 0.f;
  // d/dza = 2(za-zp) - 2(za-zn), d/dzp = -2(za-zp), d/dzn = 2(za-zn)
  for (int e = lane; e < E; e += 32) {
    const float u = za[e] - zp[e], w = za[e] - zn[e];
    dZ[(int64_t)b * E + e] = s * (u - w);
    dZ[(int64_t)(B + b) * E + e] = -s * u;
    dZ[(int64_t)(2 * B + b) * E + e] = s * w;
  }
  if (lane == 0) hinge[b] = l > 0.f ? l : 0.f;
}

// loss[step ? *step : 0] = mean of hinge[0..B), summed in a fixed order (one
// block of 256).
__global__ void __launch_bounds__(256) k_loss_mean(const float* __restrict__ hinge, int B, const int* __restrict__ step,
                                                   float* __restrict__ loss) {
  __shared__ float red[256];
  float s = 0.f;
  for (int b = threadIdx.x; b < B; b += 256) s = __fadd_rn(s, hinge[b]);
  red[threadIdx.x] = s;
  __syncthreads();
  for (int w = 128; w >= 1; w >>= 1) {
    if ((int)threadIdx.x < w) red[threadIdx.x] = __fadd_rn(red[threadIdx.x], red[threadIdx.x + w]);
    __syncthreads();
  }
  if (threadIdx.x == 0) loss[step ? *step : 0] = red[0] / (float)B;
}

// Adam on the whole parameter vector; *step = step index (0-based).
__global__ void k_adam(float* __restrict__ w, const float* __restrict__ g, float* __restrict__ m,
                       float* __restrict__ v, int64_t count, float lr, const int* __restrict__ step) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= count) return;
  const float t = (float)(*step + 1);
  const float c1 = 1.0f - powf(kB1, t), c2 = 1.0f - powf(kB2, t);
  const float gi = g[i];
  const float mi = kB1 * m[i] + (1.f - kB1) * gi;
  const float vi = kB2 * v[i] + (1.f - kB2) * gi * gi;
  m[i] = mi;
  v[i] = vi;
  w[i] -= lr * (mi / c1) / (sqrtf(vi / c2) + kEps);
}

__global__ void k_step_advance(int* step) { *step += 1; }

// Row scale of the network input: 1/|x| for COSINE (norms given; a zero row
// stays zero), else 1.
__device__ __forceinline__ float unit_scale(const float* __restrict__ norms, int64_t i) {
  if (!norms) return 1.0f;
  const float nr = norms[i];
  return nr > 0.f ? __fdiv_rn(1.0f, nr) : 1.0f;
}

// Standardised rows of one triplet batch.  Row r < B: anchor a (random sample
// point); B <= r < 2B: positive, a graph neighbour of a of rank < half;
// 2B <= r: negative, a random sample point (even hash) or a graph neighbour of
// a of rank >= half (odd hash).  The step index is read on the device, so a
// replayed step draws fresh triplets.
__global__ void k_triplet_rows(const float* __restrict__ Xs, const float* __restrict__ norms, int dpad, int d,
                               int64_t ns, const int32_t* __restrict__ graph, int gk, int half, int B,
                               uint64_t seed, const int* __restrict__ step, const float* __restrict__ mean,
                               const float* __restrict__ inv_std, float* __restrict__ rows) {
  const int r = blockIdx.x;  // 0 .. 3B-1
  const int b = r % B, role = r / B;
  const uint64_t h = splitmix64(seed ^ splitmix64((uint64_t)(*step) * 0x9E3779B97F4A7C15ull + (uint64_t)b));
  const int64_t a = (int64_t)(h % (uint64_t)ns);
  int64_t src = a;
  if (role == 1) {
    const uint64_t h2 = splitmix64(h ^ 0x5851F42D4C957F2Dull);
    src = graph[a * gk + (int64_t)(h2 % (uint64_t)half)];
  } else if (role == 2) {
    const uint64_t h3 = splitmix64(h ^ 0x14057B7EF767814Full);
    if ((h3 & 1) == 0 || gk <= half)
      src = (int64_t)((h3 >> 1) % (uint64_t)ns);
    else
      src = graph[a * gk + half + (int64_t)((h3 >> 1) % (uint64_t)(gk - half))];
  }
  const float sc = unit_scale(norms, src);
  for (int c = threadIdx.x; c < d; c += blockDim.x)
    rows[(int64_t)r * d + c] = __fmul_rn(__fsub_rn(__fmul_rn(Xs[src * dpad + c], sc), mean[c]), inv_std[c]);
}

// Per-dimension mean and 1/std of the sample rows (one warp per dimension).
__global__ void k_standardise_stats(const float* __restrict__ Xs, const float* __restrict__ norms, int dpad, int d,
                                    int64_t ns, float* __restrict__ mean, float* __restrict__ inv_std) {
  const int c = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
  const int lane = threadIdx.x & 31;
  if (c >= d) return;
  double s = 0, s2 = 0;
  for (int64_t i = lane; i < ns; i += 32) {
    const double v = __fmul_rn(Xs[i * dpad + c], unit_scale(norms, i));
    s += v;
    s2 += v * v;
  }
#pragma unroll
  for (int off = 16; off >= 1; off >>= 1) {
    s += __shfl_xor_sync(0xFFFFFFFFu, s, off);
    s2 += __shfl_xor_sync(0xFFFFFFFFu, s2, off);
  }
  if (lane == 0) {
    const double mu = s / (double)ns;
    const double var = s2 / (double)ns - mu * mu;
    mean[c] = (float)mu;
    inv_std[c] = var > 1e-12 ? (float)(1.0 / sqrt(var)) : 1.0f;
  }
}

// Rows [r0, r0+m) of X, standardised, into a dense [m][d] block.
__global__ void k_standardise_rows(const float* __restrict__ X, const float* __restrict__ norms, int dpad, int d,
                                   int64_t r0, int m, const float* __restrict__ mean,
                                   const float* __restrict__ inv_std, float* __restrict__ out) {
  const int64_t g = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (g >= (int64_t)m * d) return;
  const int64_t r = g / d;
  const int c = (int)(g - r * d);
  const float sc = unit_scale(norms, r0 + r);
  out[g] = __fmul_rn(__fsub_rn(__fmul_rn(X[(size_t)(r0 + r) * dpad + c], sc), mean[c]), inv_std[c]);
}

// Gaussian initial weights (Box-Muller on a splitmix64 stream) times `scale`.
__global__ void k_init_normal(float* __restrict__ w, int64_t count, float scale, uint64_t seed) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= count) return;
  const uint64_t h = splitmix64(seed + (uint64_t)i * 0x9E3779B97F4A7C15ull);
  const float u1 = ((float)((h >> 40) & 0xFFFFFF) + 1.0f) / 16777217.0f;
  const float u2 = (float)((h >> 16) & 0xFFFFFF) / 16777216.0f;
  w[i] = scale * sqrtf(-2.0f * logf(u1)) * cosf(6.283185307179586f * u2);
}

// Sample rows: row i of Xs = row floor(i * n / ns) of X (padded rows).
__global__ void k_gather_sample(const float* __restrict__ X, int64_t n, int dpad, int64_t ns,
                                float* __restrict__ Xs) {
  const int q = dpad / 4;
  const int64_t g = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (g >= ns * q) return;
  const int64_t i = g / q;
  const int c4 = (int)(g - i * q);
  const int64_t src = (int64_t)(((unsigned __int128)i * (unsigned __int128)n) / (unsigned __int128)ns);
  reinterpret_cast<float4*>(Xs)[g] = reinterpret_cast<const float4*>(X + src * dpad)[c4];
}

namespace {

inline unsigned blocks_for(int64_t count, int threads) { return (unsigned)((count + threads - 1) / threads); }

void gemm(cudaStream_t st, int M, int N, int K, const float* A, int64_t sai, int64_t sak, const float* B,
          int64_t sbj, int64_t sbk, const float* bias, float* C, int64_t ldc, float* P, int gelu) {
  dim3 grid((N + kGT - 1) / kGT, (M + kGT - 1) / kGT, 1);
  k_gemm<<<grid, 256, 0, st>>>(M, N, K, A, sai, sak, B, sbj, sbk, bias, C, ldc, P, gelu);
}

// Weight gradient C[M][N] (dense) reduced over a long K: kSplitK partial
// products, then a fixed-order sum.
void gemm_splitk(cudaStream_t st, int M, int N, int K, const float* A, int64_t sai, int64_t sak, const float* B,
                 int64_t sbj, int64_t sbk, float* C, float* part) {
  dim3 grid((N + kGT - 1) / kGT, (M + kGT - 1) / kGT, kSplitK);
  k_gemm<<<grid, 256, 0, st>>>(M, N, K, A, sai, sak, B, sbj, sbk, nullptr, part, N, nullptr, 0);
  const int64_t count = (int64_t)M * N;
  k_sum_splits<<<blocks_for(count, 256), 256, 0, st>>>(part, kSplitK, count, C);
}

struct MlpParams {
  float* W1;
  float* b1;
  float* W2;
  float* b2;
};

MlpParams param_view(float* p, int d) {
  MlpParams q;
  q.W1 = p;
  q.b1 = q.W1 + (size_t)kMlpHidden * d;
  q.W2 = q.b1 + kMlpHidden;
  q.b2 = q.W2 + (size_t)kMlpEmbed * kMlpHidden;
  return q;
}

// Workspace of one forward + backward over R rows: A1, G1, dG [R][H];
// Z, dZ [R][E]; split-K partials.
// Z, dZ [R][E]; hinge [B]; column-sum partials [kColSplits][H]; split-K
// partials.
struct FwdBwdWs {
  float *A1, *G1, *dG, *Z, *dZ, *hinge, *cpart, *part;
};
FwdBwdWs ws_view(float* ws, int R) {
  FwdBwdWs w;
  w.A1 = ws;
  w.G1 = w.A1 + (size_t)R * kMlpHidden;
  w.dG = w.G1 + (size_t)R * kMlpHidden;
  w.Z = w.dG + (size_t)R * kMlpHidden;
  w.dZ = w.Z + (size_t)R * kMlpEmbed;
  w.hinge = w.dZ + (size_t)R * kMlpEmbed;
  w.cpart = w.hinge + (size_t)R;
  w.part = w.cpart + (size_t)kColSplits * kMlpHidden;
  return w;
}

void colsum(cudaStream_t st, const float* G, int M, int N, float* out, float* cpart) {
  dim3 grid((N + 31) / 32, 1, kColSplits);
  k_colsum_part<<<grid, 256, 0, st>>>(G, M, N, N, cpart);
  k_sum_splits<<<blocks_for((int64_t)N, 256), 256, 0, st>>>(cpart, kColSplits, (int64_t)N, out);
}

void fwd_bwd(cudaStream_t st, const float* params, int d, const float* rows, int B, float margin, float* grad,
             float* ws, const int* step, float* loss, LaunchLog& log) {
  const int R = 3 * B, H = kMlpHidden, E = kMlpEmbed;
  const MlpParams p = param_view(const_cast<float*>(params), d);
  const MlpParams g = param_view(grad, d);
  const FwdBwdWs w = ws_view(ws, R);
  // forward: A1 = rows W1^T + b1, G1 = gelu(A1); Z = G1 W2^T + b2
  gemm(st, R, H, d, rows, d, 1, p.W1, d, 1, p.b1, w.G1, H, w.A1, 1);
  gemm(st, R, E, H, w.G1, H, 1, p.W2, H, 1, p.b2, w.Z, E, nullptr, 0);
  k_triplet<<<blocks_for(B, 8), 256, 0, st>>>(w.Z, B, E, margin, w.dZ, w.hinge);
  k_loss_mean<<<1, 256, 0, st>>>(w.hinge, B, step, loss);
  // dW2[e][h] = sum_r dZ[r][e] G1[r][h];  db2 = colsum dZ
  gemm_splitk(st, E, H, R, w.dZ, 1, E, w.G1, 1, H, g.W2, w.part);
  colsum(st, w.dZ, R, E, g.b2, w.cpart);
  // dA1 = (dZ W2) * gelu'(A1)
  gemm(st, R, H, E, w.dZ, E, 1, p.W2, 1, H, nullptr, w.dG, H, nullptr, 0);
  k_gelu_back<<<blocks_for((int64_t)R * H, 256), 256, 0, st>>>(w.A1, w.dG, (int64_t)R * H, w.dG);
  // dW1[h][c] = sum_r dA1[r][h] rows[r][c];  db1 = colsum dA1
  gemm_splitk(st, H, d, R, w.dG, 1, H, rows, 1, d, g.W1, w.part);
  colsum(st, w.dG, R, H, g.b1, w.cpart);
  log.add(14);
}

}  // namespace

size_t mlp_param_count(int d) {
  return (size_t)kMlpHidden * d + kMlpHidden + (size_t)kMlpEmbed * kMlpHidden + kMlpEmbed;
}

size_t mlp_fwd_bwd_ws_floats(int d, int B) {
  const size_t R = 3 * (size_t)B;
  const size_t part = (size_t)kSplitK * (size_t)kMlpHidden * (size_t)(d > kMlpEmbed ? d : kMlpEmbed);
  return R * kMlpHidden * 3 + R * kMlpEmbed * 2 + R + (size_t)kColSplits * kMlpHidden + part;
}

size_t mlp_train_ws_floats(int d, int B) {
  return mlp_fwd_bwd_ws_floats(d, B) + (size_t)3 * B * d + 3 * mlp_param_count(d) + 64;
}

int mlp_train(const MlpTrainArgs& a, LaunchLog& log) {
  cudaStream_t st = a.stream;
  const size_t np = mlp_param_count(a.d);
  const int B = a.batch;
  float* fb = a.ws;
  float* rows = fb + mlp_fwd_bwd_ws_floats(a.d, B);
  float* grad = rows + (size_t)3 * B * a.d;
  float* adam_m = grad + np;
  float* adam_v = adam_m + np;
  int* step = reinterpret_cast<int*>(adam_v + np);

  const MlpParams p = param_view(a.params, a.d);
  k_init_normal<<<blocks_for((int64_t)kMlpHidden * a.d, 256), 256, 0, st>>>(
      p.W1, (int64_t)kMlpHidden * a.d, 1.0f / sqrtf((float)a.d), a.seed);
  k_init_normal<<<blocks_for((int64_t)kMlpEmbed * kMlpHidden, 256), 256, 0, st>>>(
      p.W2, (int64_t)kMlpEmbed * kMlpHidden, 1.0f / sqrtf((float)kMlpHidden), a.seed ^ 0xA5A5A5A5ull);
  if (cudaMemsetAsync(p.b1, 0, sizeof(float) * kMlpHidden, st) != cudaSuccess ||
      cudaMemsetAsync(p.b2, 0, sizeof(float) * kMlpEmbed, st) != cudaSuccess ||
      cudaMemsetAsync(adam_m, 0, sizeof(float) * 2 * np + sizeof(int), st) != cudaSuccess ||
      cudaMemsetAsync(a.loss, 0, sizeof(float) * (size_t)(a.steps > 0 ? a.steps : 1), st) != cudaSuccess)
    return KNN_ERR_CUDA;
  k_standardise_stats<<<blocks_for(a.d, 8), 256, 0, st>>>(a.Xs, a.norms, a.dpad, a.d, a.ns, a.mean, a.inv_std);
  log.add(3);
  const int half = a.gk >= 2 ? a.gk / 2 : 1;
  // One Adam step: triplet rows, forward + backward, update, step counter.
  // The step index lives on the device, so the step is captured once as a
  // CUDA graph and replayed (direct launches when the stream is already
  // being captured by the caller).
  auto one_step = [&](LaunchLog& lg) {
    k_triplet_rows<<<3 * B, 128, 0, st>>>(a.Xs, a.norms, a.dpad, a.d, a.ns, a.graph, a.gk, half, B, a.seed, step,
                                           a.mean, a.inv_std, rows);
    fwd_bwd(st, a.params, a.d, rows, B, a.margin, grad, fb, step, a.loss, lg);
    k_adam<<<blocks_for((int64_t)np, 256), 256, 0, st>>>(a.params, grad, adam_m, adam_v, (int64_t)np, a.lr, step);
    k_step_advance<<<1, 1, 0, st>>>(step);
    lg.add(3);
  };
  cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
  if (cudaStreamIsCapturing(st, &cs) != cudaSuccess) return KNN_ERR_CUDA;
  if (cs != cudaStreamCaptureStatusNone || a.steps < 2) {
    for (int s = 0; s < a.steps; ++s) one_step(log);
    return cudaPeekAtLastError() == cudaSuccess ? KNN_OK : KNN_ERR_CUDA;
  }
  if (cudaPeekAtLastError() != cudaSuccess) return KNN_ERR_CUDA;
  LaunchLog step_log;
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t exec = nullptr;
  if (cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal) != cudaSuccess) return KNN_ERR_CUDA;
  one_step(step_log);
  cudaError_t e = cudaStreamEndCapture(st, &graph);
  if (e == cudaSuccess) e = cudaGraphInstantiate(&exec, graph, 0);
  for (int s = 0; e == cudaSuccess && s < a.steps; ++s) e = cudaGraphLaunch(exec, st);
  // the executable graph is released only after its launches have finished
  if (e == cudaSuccess) e = cudaStreamSynchronize(st);
  if (exec) cudaGraphExecDestroy(exec);
  if (graph) cudaGraphDestroy(graph);
  log.add(step_log.count * a.steps);
  return e == cudaSuccess ? KNN_OK : KNN_ERR_CUDA;
}

size_t mlp_embed_ws_floats(int d, int64_t chunk) { return (size_t)chunk * ((size_t)d + kMlpHidden); }

int mlp_embed(const float* X, const float* norms, int64_t n, int d, int dpad, const float* params,
              const float* mean, const float* inv_std, float* ws, int64_t chunk, float* Z, cudaStream_t st,
              LaunchLog& log) {
  const MlpParams p = param_view(const_cast<float*>(params), d);
  float* S = ws;                      // [chunk][d]
  float* G1 = S + (size_t)chunk * d;  // [chunk][H]
  for (int64_t r0 = 0; r0 < n; r0 += chunk) {
    const int m = (int)(n - r0 < chunk ? n - r0 : chunk);
    k_standardise_rows<<<blocks_for((int64_t)m * d, 256), 256, 0, st>>>(X, norms, dpad, d, r0, m, mean, inv_std,
                                                                          S);
    gemm(st, m, kMlpHidden, d, S, d, 1, p.W1, d, 1, p.b1, G1, kMlpHidden, nullptr, 1);
    gemm(st, m, kMlpEmbed, kMlpHidden, G1, kMlpHidden, 1, p.W2, kMlpHidden, 1, p.b2, Z + (size_t)r0 * kMlpEmbed,
         kMlpEmbed, nullptr, 0);
    log.add(3);
  }
  return cudaPeekAtLastError() == cudaSuccess ? KNN_OK : KNN_ERR_CUDA;
}

int mlp_loss_grad(const float* params, int d, const float* rows, int B, float margin, float* grad, float* ws,
                  float* loss, cudaStream_t st, LaunchLog& log) {
  fwd_bwd(st, params, d, rows, B, margin, grad, ws, nullptr, loss, log);
  return cudaPeekAtLastError() == cudaSuccess ? KNN_OK : KNN_ERR_CUDA;
}

void launch_gather_sample(const float* X, int64_t n, int dpad, int64_t ns, float* Xs, cudaStream_t st) {
  k_gather_sample<<<blocks_for(ns * (dpad / 4), 256), 256, 0, st>>>(X, n, dpad, ns, Xs);
}

}  // namespace knn
