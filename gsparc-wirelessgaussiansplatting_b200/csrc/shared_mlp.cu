// Shared emission MLP: one network for all Gaussians, evaluated per
// (receiver, Gaussian) pair.
//
// The reference's emission model is a per-Gaussian 3-32-2 MLP on the receiver
// position (forward.cu:17-75).  The benchmark's configurations instead name a
// shared MLP from per-pair features to amplitudes ("2x64 ReLU", "3x128 GELU",
// 1 or 64 outputs); this file is that model.  Features of pair (r, g), with
// mu the Gaussian centre, rx the receiver and d = |mu - rx|:
//   x[0:3]            mu
//   x[3 + 6k + 2j]    sin(2^k pi mu_j),  x[4 + 6k + 2j]  cos(2^k pi mu_j),
//                     k = 0..3, j = 0..2 (positional encoding, 24 values)
//   x[27:30]          (mu - rx) / d      (receiver-relative direction)
//   x[30]             1 / d^2            (distance attenuation)
//   x[31]             0                  (pad to 32)
// Layers: L hidden layers of width H with ReLU or GELU (erf form), then a
// linear layer to C outputs; the signal of output c is sigmoid(o_c) (the
// real channel of the blend; the imaginary channel is 0).  Parameters are
// flat fp32, layer by layer: W_l [out, in] row-major, then b_l [out].
// Culled pairs (radius 0) get zero features and no signal.
//
// This is the FP32 (SIMT) path: the layers are tiled SIMT GEMMs over the
// R*P pair rows with the activations kept in a workspace for the adjoint.
#include <algorithm>

#include "common.cuh"
#include "kernels.cuh"

namespace gsparc {

constexpr int kFeat = 32;
constexpr float kPi = 3.14159265358979323846f;

__device__ __forceinline__ float gelu_erf(float z) { return 0.5f * z * (1.0f + erff(z * 0.70710678118654752f)); }

__device__ __forceinline__ float gelu_erf_grad(float z) {
  const float cdf = 0.5f * (1.0f + erff(z * 0.70710678118654752f));
  const float pdf = 0.39894228040143268f * expf(-0.5f * z * z);
  return cdf + z * pdf;
}

// act: 0 identity, 1 ReLU, 2 GELU
__device__ __forceinline__ float act_fwd(int act, float z) {
  return act == 1 ? fmaxf(z, 0.0f) : (act == 2 ? gelu_erf(z) : z);
}
__device__ __forceinline__ float act_grad(int act, float z) {
  return act == 1 ? (z > 0.0f ? 1.0f : 0.0f) : (act == 2 ? gelu_erf_grad(z) : 1.0f);
}

// ---- features ---------------------------------------------------------------
// x = [mu, sin/cos(2^k pi mu_j) for k < 4, (mu - rx) / d, 1 / d^2, 0]
__device__ __forceinline__ void pair_features_fp32(const float* __restrict__ means3D, const float* __restrict__ rx_pos,
                                                   int g, int r, float* x) {
  const float m[3] = {means3D[3 * g], means3D[3 * g + 1], means3D[3 * g + 2]};
  const float v[3] = {m[0] - rx_pos[3 * r], m[1] - rx_pos[3 * r + 1], m[2] - rx_pos[3 * r + 2]};
  const float d2 = v[0] * v[0] + v[1] * v[1] + v[2] * v[2];
  const float d = sqrtf(d2);
  x[0] = m[0]; x[1] = m[1]; x[2] = m[2];
#pragma unroll
  for (int k = 0; k < 4; ++k)
#pragma unroll
    for (int j = 0; j < 3; ++j) {
      float s, c;
      sincosf((float)(1 << k) * kPi * m[j], &s, &c);
      x[3 + 6 * k + 2 * j] = s;
      x[4 + 6 * k + 2 * j] = c;
    }
  x[27] = v[0] / d; x[28] = v[1] / d; x[29] = v[2] / d;
  x[30] = 1.0f / d2;
  x[31] = 0.0f;
}

__global__ void __launch_bounds__(256)
mlp_features_kernel(int P, const float* __restrict__ means3D, const float* __restrict__ rx_pos,
                    const int* __restrict__ radii, float* __restrict__ X) {
  const int g = blockIdx.x * blockDim.x + threadIdx.x;
  const int r = blockIdx.y;
  if (g >= P) return;
  const size_t row = (size_t)r * P + g;
  float* x = X + row * kFeat;
  if (radii[row] <= 0) {
#pragma unroll
    for (int i = 0; i < kFeat; ++i) x[i] = 0.0f;
    return;
  }
  float f[kFeat];
  pair_features_fp32(means3D, rx_pos, g, r, f);
#pragma unroll
  for (int i = 0; i < kFeat; ++i) x[i] = f[i];
}

// dL/dmu from dL/dx.  The positional-encoding part does not depend on the
// receiver, so dX[0..26] is summed over receivers first (sum_pe); the
// direction and 1/d^2 parts are accumulated per receiver (acc).  dX rows are
// read as float4s, through L2 only when kL2 (written earlier in the same kernel).
template <bool kL2>
__device__ __forceinline__ void features_partial(int g, int P, int r_lo, int r_hi, const float (&m)[3],
                                                 const float* __restrict__ rx_pos, const int* __restrict__ radii,
                                                 const float* dX, float (&sum_pe)[27], float (&acc)[3]) {
  for (int r = r_lo; r < r_hi; ++r) {
    const size_t row = (size_t)r * P + g;
    if (radii[row] <= 0) continue;
    float dx[kFeat];
    const float4* src = reinterpret_cast<const float4*>(dX + row * kFeat);
#pragma unroll
    for (int q = 0; q < kFeat / 4; ++q) {
      const float4 v = kL2 ? __ldcg(src + q) : src[q];
      dx[4 * q] = v.x; dx[4 * q + 1] = v.y; dx[4 * q + 2] = v.z; dx[4 * q + 3] = v.w;
    }
#pragma unroll
    for (int i = 0; i < 27; ++i) sum_pe[i] += dx[i];
    const float v[3] = {m[0] - rx_pos[3 * r], m[1] - rx_pos[3 * r + 1], m[2] - rx_pos[3 * r + 2]};
    const float d2 = v[0] * v[0] + v[1] * v[1] + v[2] * v[2];
    const float d = sqrtf(d2);
    const float u[3] = {v[0] / d, v[1] / d, v[2] / d};
    // direction u = v / d: du_i/dv_j = (delta_ij - u_i u_j) / d
    const float gu = dx[27] * u[0] + dx[28] * u[1] + dx[29] * u[2];
    // attenuation 1/d^2: d/dv = -2 v / d^4
    const float ga = dx[30] * (-2.0f / (d2 * d2));
#pragma unroll
    for (int j = 0; j < 3; ++j) acc[j] += (dx[27 + j] - gu * u[j]) / d + ga * v[j];
  }
}

// the positional encoding's chain rule, added to dL/dmeans3D[g]
__device__ __forceinline__ void features_finish(int g, const float (&m)[3], const float (&sum_pe)[27],
                                                const float (&acc)[3], float* __restrict__ dL_dmeans3D) {
#pragma unroll
  for (int j = 0; j < 3; ++j) {
    float gj = sum_pe[j];
#pragma unroll
    for (int k = 0; k < 4; ++k) {
      const float w = (float)(1 << k) * kPi;
      float s, c;
      sincosf(w * m[j], &s, &c);
      gj += w * (c * sum_pe[3 + 6 * k + 2 * j] - s * sum_pe[4 + 6 * k + 2 * j]);
    }
    dL_dmeans3D[3 * g + j] += gj + acc[j];
  }
}

// Gaussian g over all R receivers in order (one thread)
template <bool kL2>
__device__ __forceinline__ void features_adjoint(int g, int P, int R, const float* __restrict__ means3D,
                                                 const float* __restrict__ rx_pos, const int* __restrict__ radii,
                                                 const float* dX, float* __restrict__ dL_dmeans3D) {
  const float m[3] = {means3D[3 * g], means3D[3 * g + 1], means3D[3 * g + 2]};
  float sum_pe[27] = {}, acc[3] = {};
  features_partial<kL2>(g, P, 0, R, m, rx_pos, radii, dX, sum_pe, acc);
  features_finish(g, m, sum_pe, acc, dL_dmeans3D);
}

// Several receivers: four lanes per Gaussian, lane q taking receivers
// [q R / 4, (q + 1) R / 4) in order; the four partial sums are combined as
// (q0 + q1) + (q2 + q3) (a fixed order: deterministic).
constexpr int kFeatLanes = 4;
__global__ void __launch_bounds__(256)
mlp_features_backward_kernel(int P, int R, const float* __restrict__ means3D, const float* __restrict__ rx_pos,
                             const int* __restrict__ radii, const float* __restrict__ dX,
                             float* __restrict__ dL_dmeans3D) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  const int g = t / kFeatLanes, q = t % kFeatLanes;
  const bool live = g < P;
  float m[3] = {0.0f, 0.0f, 0.0f};
  if (live) {
    m[0] = means3D[3 * g];
    m[1] = means3D[3 * g + 1];
    m[2] = means3D[3 * g + 2];
  }
  float sum_pe[27] = {}, acc[3] = {};
  if (live)
    features_partial<false>(g, P, (int)((long long)q * R / kFeatLanes), (int)((long long)(q + 1) * R / kFeatLanes),
                            m, rx_pos, radii, dX, sum_pe, acc);
#pragma unroll
  for (int o = 1; o < kFeatLanes; o <<= 1) {
#pragma unroll
    for (int i = 0; i < 27; ++i) sum_pe[i] += __shfl_down_sync(0xffffffffu, sum_pe[i], o, kFeatLanes);
#pragma unroll
    for (int j = 0; j < 3; ++j) acc[j] += __shfl_down_sync(0xffffffffu, acc[j], o, kFeatLanes);
  }
  if (live && q == 0) features_finish(g, m, sum_pe, acc, dL_dmeans3D);
}

// ---- tiled SIMT GEMM ----------------------------------------------------------
// C[i, j] = sum_k A(i, k) B(k, j), A(i, k) = A[i * sai + k * sak],
// B(k, j) = B[k * sbk + j * sbj]; rows i < M, cols j < N, k < K.  Tile 64x64,
// 256 threads with 4x4 outputs each.  Epilogues:
//   kEpiFwd:    Z = acc + bias[j] -> C; act(Z) -> C2
//   kEpiDx:     acc * act'(Zin[i, j]) -> C   (act 0: plain store)
//   kEpiAtomic: atomicAdd(C[i, j], acc), with k split over blockIdx.z in
//               chunks of kchunk
enum { kEpiFwd = 0, kEpiDx = 1, kEpiAtomic = 2 };
constexpr int kBM = 64, kBN = 64, kBK = 16;

template <int kEpi>
__global__ void __launch_bounds__(256)
mlp_gemm_kernel(int M, int N, int K, int kchunk, const float* __restrict__ A, long long sai, long long sak,
                const float* __restrict__ B, long long sbk, long long sbj, float* __restrict__ C, int ldc,
                const float* __restrict__ bias, int act, float* __restrict__ C2, const float* __restrict__ Zin) {
  __shared__ float As[kBK][kBM + 4];
  __shared__ float Bs[kBK][kBN + 4];
  const int tid = threadIdx.x, ty = tid >> 4, tx = tid & 15;
  const long long i0 = (long long)blockIdx.x * kBM;   // rows on x: the pair count exceeds grid.y's limit
  const int j0 = blockIdx.y * kBN;
  const int kbeg = kEpi == kEpiAtomic ? blockIdx.z * kchunk : 0;
  const int kend = kEpi == kEpiAtomic ? min(K, kbeg + kchunk) : K;
  float acc[4][4] = {};
  for (int k0 = kbeg; k0 < kend; k0 += kBK) {
#pragma unroll
    for (int q = 0; q < 4; ++q) {
      const int e = tid + q * 256;          // 0..1023: consecutive threads walk the unit-stride index
      const int ai = sak == 1 ? e / kBK : e % kBM, ak = sak == 1 ? e % kBK : e / kBM;
      const long long gi = i0 + ai, gk = k0 + ak;
      As[ak][ai] = (gi < M && gk < kend) ? A[gi * sai + gk * sak] : 0.0f;
      const int bj = sbj == 1 ? e % kBN : e / kBK, bk = sbj == 1 ? e / kBN : e % kBK;
      const long long gj = j0 + bj, gk2 = k0 + bk;
      Bs[bk][bj] = (gj < N && gk2 < kend) ? B[gk2 * sbk + gj * sbj] : 0.0f;
    }
    __syncthreads();
#pragma unroll
    for (int kk = 0; kk < kBK; ++kk) {
      float a[4], b[4];
#pragma unroll
      for (int u = 0; u < 4; ++u) { a[u] = As[kk][ty * 4 + u]; b[u] = Bs[kk][tx * 4 + u]; }
#pragma unroll
      for (int u = 0; u < 4; ++u)
#pragma unroll
        for (int w = 0; w < 4; ++w) acc[u][w] += a[u] * b[w];
    }
    __syncthreads();
  }
#pragma unroll
  for (int u = 0; u < 4; ++u)
#pragma unroll
    for (int w = 0; w < 4; ++w) {
      const long long i = i0 + ty * 4 + u;
      const int j = j0 + tx * 4 + w;
      if (i >= M || j >= N) continue;
      const size_t o = (size_t)i * ldc + j;
      if (kEpi == kEpiFwd) {
        const float z = acc[u][w] + bias[j];
        C[o] = z;
        C2[o] = act_fwd(act, z);
      } else if (kEpi == kEpiDx) {
        C[o] = act == 0 ? acc[u][w] : acc[u][w] * act_grad(act, Zin[o]);
      } else {
        atomicAdd(&C[o], acc[u][w]);
      }
    }
}

// column sums of an [M, N] matrix into out[N] (atomic over row chunks)
__global__ void __launch_bounds__(256)
mlp_colsum_kernel(int M, int N, const float* __restrict__ A, float* __restrict__ out) {
  const int j = blockIdx.x * 32 + (threadIdx.x & 31);
  const int i0 = blockIdx.y * 2048;
  if (j >= N) return;
  float s = 0.0f;
  for (int i = i0 + (threadIdx.x >> 5); i < min(M, i0 + 2048); i += 8) s += A[(size_t)i * N + j];
  __shared__ float red[8][32];
  red[threadIdx.x >> 5][threadIdx.x & 31] = s;
  __syncthreads();
  if (threadIdx.x < 32) {
    float t = 0.0f;
#pragma unroll
    for (int w = 0; w < 8; ++w) t += red[w][threadIdx.x];
    atomicAdd(&out[j], t);
  }
}

// S = sigmoid(O) per output; with one output the signal of visible pairs is
// (S, 0).  Backward: dO = dL/dS * S (1 - S), where dL/dS is the real part of
// dL/dsignal (stride 2) for one output and dL/dfeatures (stride Cout) otherwise.
__global__ void __launch_bounds__(256)
mlp_signal_kernel(size_t rows, int Cout, const float* __restrict__ O, const int* __restrict__ radii,
                  float* __restrict__ S, float2* __restrict__ signal) {
  const size_t row = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
  if (row >= rows) return;
  for (int c = 0; c < Cout; ++c) S[row * Cout + c] = 1.0f / (1.0f + expf(-O[row * Cout + c]));
  if (Cout == 1 && radii[row] > 0) signal[row] = make_float2(S[row], 0.0f);
}

__global__ void __launch_bounds__(256)
mlp_signal_backward_kernel(size_t rows, int Cout, const float* __restrict__ S, const int* __restrict__ radii,
                           const float* __restrict__ dL_dsignal, float* __restrict__ dO) {
  const size_t row = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
  if (row >= rows) return;
  const bool vis = radii[row] > 0;
  const int ld = Cout == 1 ? 2 : Cout;
  for (int c = 0; c < Cout; ++c) {
    const float s = S[row * Cout + c];
    dO[row * Cout + c] = vis ? dL_dsignal[row * ld + c] * s * (1.0f - s) : 0.0f;
  }
}

// ---- fused path: width 64, one output, one or two hidden layers --------------
// One row (receiver, Gaussian pair) per thread with the network evaluated in
// registers and the weights in shared memory (every thread reads the same
// weight at the same time: broadcast).  Each layer's sums run in the same
// order as the tiled GEMMs above (inputs ascending from zero, then + bias), so
// the forward matches them bit for bit.  The forward also writes each hidden
// layer's pre-activations Z (fp32, tile-transposed: [layer][tile][64][128], so a
// warp's float4 stores and loads are contiguous) next to the sigmoid outputs S;
// the adjoint reads them instead of recomputing the forward GEMMs, and reduces
// the weight gradients over each tile of 128 rows in shared memory,
// accumulating per thread across tiles.
constexpr int kW64 = 64;
constexpr int kFusedRows = 128;

bool shared_mlp_fused(int layers, int width, int out) { return width == kW64 && out == 1 && layers >= 1 && layers <= 2; }

// parameter block as in the global vector: W0 [64][32], b0, (W1 [64][64], b1), wo [64], bo
template <int kL>
struct FusedParams {
  static constexpr int kW0 = 0, kB0 = kW0 + kW64 * kFeat;
  static constexpr int kW1 = kB0 + kW64, kB1 = kW1 + (kL == 2 ? kW64 * kW64 : 0);
  static constexpr int kWo = kB1 + (kL == 2 ? kW64 : 0), kBo = kWo + kW64;
  static constexpr int kCount = kBo + 1;                 // floats in the global parameter vector
  static constexpr int kPadded = (kCount + 3) / 4 * 4;   // keeps what follows 16-byte aligned
};

template <int N>
__device__ __forceinline__ void store_row(float* dst, const float* v) {
#pragma unroll
  for (int q = 0; q < N / 4; ++q)
    reinterpret_cast<float4*>(dst)[q] = make_float4(v[4 * q], v[4 * q + 1], v[4 * q + 2], v[4 * q + 3]);
}

// W [64][K] (row-major, global) -> W^T [K][64] in shared memory.  Each thread
// takes four consecutive inputs of one output row, consecutive threads
// consecutive outputs, so the shared-memory writes of a warp are contiguous;
// every load is independent (all of them in flight at once).  blockDim.x must
// be kFusedRows.
template <int K>
__device__ __forceinline__ void stage_transposed(float* __restrict__ dst, const float* __restrict__ W) {
  constexpr int kItems = kW64 * (K / 4);
#pragma unroll
  for (int it = 0; it < (kItems + kFusedRows - 1) / kFusedRows; ++it) {
    const int i = it * kFusedRows + (int)threadIdx.x;
    if (i < kItems) {
      const int j = i % kW64, k = 4 * (i / kW64);
      const float w0 = W[j * K + k], w1 = W[j * K + k + 1], w2 = W[j * K + k + 2], w3 = W[j * K + k + 3];
      dst[k * kW64 + j] = w0;
      dst[(k + 1) * kW64 + j] = w1;
      dst[(k + 2) * kW64 + j] = w2;
      dst[(k + 3) * kW64 + j] = w3;
    }
  }
}

// Row strides of the per-thread shared-memory rows: float4-aligned, and eight
// consecutive rows' float4s fall on distinct banks.
constexpr int kXs = kFeat + 4, kHs = kW64 + 4;

// Column swizzle of the 64-wide row tiles (D, A0): row r keeps its float4
// groups but XORs their index with (r / 4) mod 8.  The 8x4 blocks' row-major
// stores put rows 4 apart in the lanes of one quarter-warp; without the XOR
// those rows land on two bank groups (4-way conflicts), with it on eight.
__device__ __forceinline__ int row_swz(int r) { return ((r >> 2) & 7) << 2; }

// C[8 rows][8 cols] += sum_k AT[k][rows] * BT[k][cols], k ascending from zero:
// a register-blocked SIMT GEMM step over operands in shared memory (AT rows
// contiguous, BT columns contiguous).  The thread's rows are r0..r0+3 and
// r0+64..r0+67, its columns c0..c0+3 and c0+32..c0+35.
template <int K>
__device__ __forceinline__ void gemm_8x8(const float* __restrict__ AT, int lda, const float* __restrict__ BT,
                                         int ldb, int r0, int c0, float (&acc)[8][8]) {
#pragma unroll 2
  for (int k = 0; k < K; ++k) {
    const float4 a0 = *reinterpret_cast<const float4*>(AT + k * lda + r0);
    const float4 a1 = *reinterpret_cast<const float4*>(AT + k * lda + r0 + 64);
    const float4 b0 = *reinterpret_cast<const float4*>(BT + k * ldb + c0);
    const float4 b1 = *reinterpret_cast<const float4*>(BT + k * ldb + c0 + 32);
    const float a[8] = {a0.x, a0.y, a0.z, a0.w, a1.x, a1.y, a1.z, a1.w};
    const float2 b[4] = {make_float2(b0.x, b0.y), make_float2(b0.z, b0.w), make_float2(b1.x, b1.y),
                         make_float2(b1.z, b1.w)};
#pragma unroll
    for (int i = 0; i < 8; ++i) {
      const float2 ai = make_float2(a[i], a[i]);
#pragma unroll
      for (int j = 0; j < 4; ++j) {   // two columns per FP32x2 FMA, each lane rounded as fmaf
        const float2 c = ffma2(ai, b[j], make_float2(acc[i][2 * j], acc[i][2 * j + 1]));
        acc[i][2 * j] = c.x;
        acc[i][2 * j + 1] = c.y;
      }
    }
  }
}

// forward: W0^T [32][64], W1^T [64][64] (two layers), b0, b1, wo, bo; then the
// transposed tiles X^T [32][128] and H^T [64][128] (hidden activations, then the
// last layer's)
template <int kL>
struct FusedFwdSmem {
  static constexpr int kWt0 = 0, kWt1 = kWt0 + kFeat * kW64;
  static constexpr int kB0 = kWt1 + (kL == 2 ? kW64 * kW64 : 0), kB1 = kB0 + kW64, kWo = kB1 + kW64;
  static constexpr int kBo = kWo + kW64, kXT = kBo + 4, kHT = kXT + kFeat * kFusedRows;
  static constexpr int kTotal = kHT + kW64 * kFusedRows;
};

template <int kL, int kAct>
__global__ void __launch_bounds__(kFusedRows)
mlp64_forward_kernel(int P, size_t rows, const float* __restrict__ means3D, const float* __restrict__ rx_pos,
                     const float* __restrict__ params, const int* __restrict__ radii, float* __restrict__ S,
                     float* __restrict__ Z, float2* __restrict__ signal) {
  using FP = FusedParams<kL>;
  using SM = FusedFwdSmem<kL>;
  extern __shared__ __align__(16) float sm[];
  const int t = threadIdx.x;
  stage_transposed<kFeat>(sm + SM::kWt0, params + FP::kW0);
  if (kL == 2) stage_transposed<kW64>(sm + SM::kWt1, params + FP::kW1);
  for (int i = t; i < kW64; i += blockDim.x) {
    sm[SM::kB0 + i] = params[FP::kB0 + i];
    if (kL == 2) sm[SM::kB1 + i] = params[FP::kB1 + i];
    sm[SM::kWo + i] = params[FP::kWo + i];
  }
  if (t == 0) sm[SM::kBo] = params[FP::kBo];
  float* XT = sm + SM::kXT;
  float* HT = sm + SM::kHT;
  // GEMM blocks: 16 row groups x 8 column groups; eight consecutive lanes share
  // a column group, so the transposed stores of a lane octet are contiguous
  const int r0 = (t & 15) * 4, c0 = (t >> 4) * 4;
  const size_t ntiles = (rows + kFusedRows - 1) / kFusedRows;
  const size_t zl = ntiles * (kFusedRows * kW64);   // floats of one layer's Z
  for (size_t tile = blockIdx.x; tile < ntiles; tile += gridDim.x) {
    const size_t row = tile * kFusedRows + t;
    const bool vis = row < rows && radii[row] > 0;
    float* Zt = Z + tile * (kFusedRows * kW64);
    __syncthreads();   // the previous tile's reads of XT / HT are done
    {
      float x[kFeat];
      if (vis) pair_features_fp32(means3D, rx_pos, (int)(row % P), (int)(row / P), x);
      else
#pragma unroll
        for (int f = 0; f < kFeat; ++f) x[f] = 0.0f;
#pragma unroll
      for (int f = 0; f < kFeat; ++f) XT[f * kFusedRows + t] = x[f];
    }
    __syncthreads();
    float acc[8][8];
#pragma unroll
    for (int i = 0; i < 8; ++i)
#pragma unroll
      for (int j = 0; j < 8; ++j) acc[i][j] = 0.0f;
    gemm_8x8<kFeat>(XT, kFusedRows, sm + SM::kWt0, kW64, r0, c0, acc);
    if (kL == 2) {
      // Z0 = X W0^T + b0 -> HBM, H^T = act(Z0), then the second layer over it
#pragma unroll
      for (int j = 0; j < 8; ++j) {
        const int c = c0 + (j & 3) + (j >> 2) * 32;
        const float b = sm[SM::kB0 + c];
        float z[8], h[8];
#pragma unroll
        for (int i = 0; i < 8; ++i) {
          z[i] = acc[i][j] + b;
          h[i] = act_fwd(kAct, z[i]);
        }
        *reinterpret_cast<float4*>(Zt + c * kFusedRows + r0) = make_float4(z[0], z[1], z[2], z[3]);
        *reinterpret_cast<float4*>(Zt + c * kFusedRows + r0 + 64) = make_float4(z[4], z[5], z[6], z[7]);
        *reinterpret_cast<float4*>(HT + c * kFusedRows + r0) = make_float4(h[0], h[1], h[2], h[3]);
        *reinterpret_cast<float4*>(HT + c * kFusedRows + r0 + 64) = make_float4(h[4], h[5], h[6], h[7]);
      }
      __syncthreads();
#pragma unroll
      for (int i = 0; i < 8; ++i)
#pragma unroll
        for (int j = 0; j < 8; ++j) acc[i][j] = 0.0f;
      gemm_8x8<kW64>(HT, kFusedRows, sm + SM::kWt1, kW64, r0, c0, acc);
      __syncthreads();   // every thread has read HT before it is overwritten
    }
    // the last hidden layer's activations -> H^T, then the output per row in the
    // GEMMs' order (hidden units ascending)
    const float* bl = sm + (kL == 2 ? SM::kB1 : SM::kB0);
    float* Zl = Zt + (kL - 1) * zl;
#pragma unroll
    for (int j = 0; j < 8; ++j) {
      const int c = c0 + (j & 3) + (j >> 2) * 32;
      const float b = bl[c];
      float z[8], h[8];
#pragma unroll
      for (int i = 0; i < 8; ++i) {
        z[i] = acc[i][j] + b;
        h[i] = act_fwd(kAct, z[i]);
      }
      *reinterpret_cast<float4*>(Zl + c * kFusedRows + r0) = make_float4(z[0], z[1], z[2], z[3]);
      *reinterpret_cast<float4*>(Zl + c * kFusedRows + r0 + 64) = make_float4(z[4], z[5], z[6], z[7]);
      *reinterpret_cast<float4*>(HT + c * kFusedRows + r0) = make_float4(h[0], h[1], h[2], h[3]);
      *reinterpret_cast<float4*>(HT + c * kFusedRows + r0 + 64) = make_float4(h[4], h[5], h[6], h[7]);
    }
    __syncthreads();
    if (vis) {
      float o = 0.0f;
#pragma unroll 8
      for (int j = 0; j < kW64; ++j) o = fmaf(HT[j * kFusedRows + t], sm[SM::kWo + j], o);
      const float sg = 1.0f / (1.0f + expf(-(o + sm[SM::kBo])));
      S[row] = sg;
      signal[row] = make_float2(sg, 0.0f);
    }
  }
}

// C[8 rows][4 cols] += sum_k AT[k][rows] * B[k][cols] (rows r0..r0+3, r0+64..r0+67;
// columns c0..c0+3), k ascending
template <int K>
__device__ __forceinline__ void gemm_8x4(const float* __restrict__ AT, int lda, const float* __restrict__ B, int ldb,
                                         int r0, int c0, float (&acc)[8][4]) {
#pragma unroll 2
  for (int k = 0; k < K; ++k) {
    const float4 a0 = *reinterpret_cast<const float4*>(AT + k * lda + r0);
    const float4 a1 = *reinterpret_cast<const float4*>(AT + k * lda + r0 + 64);
    const float4 b0 = *reinterpret_cast<const float4*>(B + k * ldb + c0);
    const float a[8] = {a0.x, a0.y, a0.z, a0.w, a1.x, a1.y, a1.z, a1.w};
    const float2 b[2] = {make_float2(b0.x, b0.y), make_float2(b0.z, b0.w)};
#pragma unroll
    for (int i = 0; i < 8; ++i) {
      const float2 ai = make_float2(a[i], a[i]);
#pragma unroll
      for (int j = 0; j < 2; ++j) {
        const float2 c = ffma2(ai, b[j], make_float2(acc[i][2 * j], acc[i][2 * j + 1]));
        acc[i][2 * j] = c.x;
        acc[i][2 * j + 1] = c.y;
      }
    }
  }
}

// adjoint shared memory (floats): weights W0 [64][32], W1 [64][64] (two layers),
// b0, b1, wo, bo; tiles X [128][36] (rows, for dW0), HT [64][128] (dZ1^T, then
// dZ0^T), A0 [128][68] (act(Z0) rows, for dW1), D [128][68] (dZ1, then dZ0, rows),
// dO [128], dwo [64 + 4]
template <int kL>
struct FusedTiles {
  static constexpr int kW0 = 0, kW1 = kW0 + kW64 * kFeat, kB0 = kW1 + (kL == 2 ? kW64 * kW64 : 0);
  static constexpr int kB1 = kB0 + kW64, kWo = kB1 + kW64, kBo = kWo + kW64;
  static constexpr int kX = kBo + 4, kHT = kX + kFusedRows * kXs;
  static constexpr int kA0 = kHT + kW64 * kFusedRows, kD = kA0 + (kL == 2 ? kFusedRows * kHs : 0);
  static constexpr int kDO = kD + kFusedRows * kHs, kDwo = kDO + kFusedRows, kTotal = kDwo + kW64 + 4;
};

// acc[4][NI] += sum over the tile's rows of D[r][j0..j0+3] (x) A[r][i0..i0+NI-1];
// bsum[4] += sum of D[r][j0..j0+3] when `bias`.  D is a swizzled row tile (row_swz),
// A one too when its stride is kHs (A0), else plain rows (X)
template <int NI, int kAs>
__device__ __forceinline__ void tile_outer(const float* __restrict__ D, const float* __restrict__ A, int j0, int i0,
                                           bool bias, float (&acc)[4][NI], float (&bsum)[4]) {
#pragma unroll 2
  for (int r = 0; r < kFusedRows; ++r) {
    const float4 d = *reinterpret_cast<const float4*>(D + r * kHs + (j0 ^ row_swz(r)));
    float a[NI];
#pragma unroll
    for (int q = 0; q < NI / 4; ++q) {
      const int ci = kAs == kHs ? ((i0 + 4 * q) ^ row_swz(r)) : i0 + 4 * q;
      const float4 v = *reinterpret_cast<const float4*>(A + r * kAs + ci);
      a[4 * q] = v.x; a[4 * q + 1] = v.y; a[4 * q + 2] = v.z; a[4 * q + 3] = v.w;
    }
    const float dd[4] = {d.x, d.y, d.z, d.w};
#pragma unroll
    for (int u = 0; u < 4; ++u) {
      const float2 du = make_float2(dd[u], dd[u]);
#pragma unroll
      for (int i = 0; i < NI; i += 2) {   // two inputs per FP32x2 FMA, each lane rounded as fmaf
        const float2 c = ffma2(du, make_float2(a[i], a[i + 1]), make_float2(acc[u][i], acc[u][i + 1]));
        acc[u][i] = c.x;
        acc[u][i + 1] = c.y;
      }
      if (bias) bsum[u] += dd[u];
    }
  }
}

// the thread's GEMM block row (i = 0..7) indices: r0..r0+3, r0+64..r0+67
__device__ __forceinline__ int blk_row(int r0, int i) { return r0 + (i & 3) + (i >> 2) * 64; }

// The adjoint runs 256 threads on each 128-row tile (8 warps per SM where the
// tile buffers allow one CTA): every GEMM over the tile's 64 columns uses 8x4
// register blocks (16 row groups x 16 column groups); the per-row phases
// (features, output layer) and the 32-wide ones (dW0, dX) run on the first
// 128 threads with the forward's mapping.  Each element's sum keeps its order
// (k ascending, rows ascending), so the results are those of 8x8 blocks.
constexpr int kAdjThreads = 256;

// v[8][4] of the thread's block (rows r0..r0+3, r0+64..r0+67; columns c0..c0+3)
// -> T [col][row] (transposed tile, 128 rows)
__device__ __forceinline__ void store_block4_T(float* T, int r0, int c0, const float (&v)[8][4]) {
#pragma unroll
  for (int j = 0; j < 4; ++j) {
    *reinterpret_cast<float4*>(T + (c0 + j) * kFusedRows + r0) = make_float4(v[0][j], v[1][j], v[2][j], v[3][j]);
    *reinterpret_cast<float4*>(T + (c0 + j) * kFusedRows + r0 + 64) = make_float4(v[4][j], v[5][j], v[6][j], v[7][j]);
  }
}
// T [col][row] (transposed tile, 128 rows, global) -> v[8][4] of the thread's block
__device__ __forceinline__ void load_block4_T(const float* __restrict__ T, int r0, int c0, float (&v)[8][4]) {
#pragma unroll
  for (int j = 0; j < 4; ++j) {
    const float4 a = *reinterpret_cast<const float4*>(T + (c0 + j) * kFusedRows + r0);
    const float4 b = *reinterpret_cast<const float4*>(T + (c0 + j) * kFusedRows + r0 + 64);
    v[0][j] = a.x; v[1][j] = a.y; v[2][j] = a.z; v[3][j] = a.w;
    v[4][j] = b.x; v[5][j] = b.y; v[6][j] = b.z; v[7][j] = b.w;
  }
}
// v[8][4] -> D [row][col] (swizzled row tiles, stride kHs)
__device__ __forceinline__ void store_block4_rows(float* D, int r0, int c0, const float (&v)[8][4]) {
#pragma unroll
  for (int i = 0; i < 8; ++i) {
    const int r = blk_row(r0, i);
    *reinterpret_cast<float4*>(D + r * kHs + (c0 ^ row_swz(r))) = make_float4(v[i][0], v[i][1], v[i][2], v[i][3]);
  }
}

template <int kL, int kAct, bool kFeatAdj>
__global__ void __launch_bounds__(kAdjThreads, 1)
mlp64_backward_kernel(int P, size_t rows, const float* __restrict__ means3D, const float* __restrict__ rx_pos,
                      const float* __restrict__ params, const int* __restrict__ radii, const float* __restrict__ S,
                      const float* __restrict__ Z, const float* __restrict__ dL_dsignal, float* dX,
                      float* __restrict__ dparams, float* __restrict__ dL_dmeans3D) {
  using FP = FusedParams<kL>;
  using TL = FusedTiles<kL>;
  extern __shared__ __align__(16) float sm[];
  const int t = threadIdx.x, lane = t & 31;
  const bool row_thread = t < kFusedRows;   // one tile row per thread in the per-row phases
  for (int i = t; i < kW64 * kFeat; i += kAdjThreads) sm[TL::kW0 + i] = params[FP::kW0 + i];
  if (kL == 2)
    for (int i = t; i < kW64 * kW64; i += kAdjThreads) sm[TL::kW1 + i] = params[FP::kW1 + i];
  for (int i = t; i < kW64; i += kAdjThreads) {
    sm[TL::kB0 + i] = params[FP::kB0 + i];
    if (kL == 2) sm[TL::kB1 + i] = params[FP::kB1 + i];
    sm[TL::kWo + i] = params[FP::kWo + i];
  }
  if (t == 0) sm[TL::kBo] = params[FP::kBo];
  for (int i = t; i < kW64 + 4; i += kAdjThreads) sm[TL::kDwo + i] = 0.0f;
  float* Xr = sm + TL::kX;
  float* HT = sm + TL::kHT;
  float* A0 = sm + TL::kA0;
  float* D = sm + TL::kD;
  float* sdO = sm + TL::kDO;
  float* dwo = sm + TL::kDwo;
  const float* wo = sm + TL::kWo;
  const int r0 = (t & 15) * 4, c0 = (t >> 4) * 4;    // 8x4 block over the 64 columns
  const int r0x = (t & 15) * 4, c0x = (t >> 4) * 4;  // dX (32 columns, first 128 threads)
  const int j1 = (t >> 4) * 4, i1 = (t & 15) * 4;    // dW1: outputs j1..j1+3 x inputs i1..i1+3
  const int j0 = (t >> 3) * 4, i0 = (t & 7) * 4;     // dW0: outputs j0..j0+3 x features i0..i0+3 (first 128)
  float g1[4][4] = {}, gb1[4] = {};   // accumulated over tiles
  float g0[4][4] = {}, gb0[4] = {};
  const size_t ntiles = (rows + kFusedRows - 1) / kFusedRows;
  const size_t zl = ntiles * (kFusedRows * kW64);   // floats of one layer's Z
  for (size_t tile = blockIdx.x; tile < ntiles; tile += gridDim.x) {
    const size_t row = tile * kFusedRows + t;
    const bool vis = row_thread && row < rows && radii[row] > 0;
    const float* Zt = Z + tile * (kFusedRows * kW64);
    __syncthreads();   // weights staged / the previous tile's reads done
    if (row_thread) {
      float x[kFeat];
      if (vis) pair_features_fp32(means3D, rx_pos, (int)(row % P), (int)(row / P), x);
      else
#pragma unroll
        for (int f = 0; f < kFeat; ++f) x[f] = 0.0f;
      store_row<kFeat>(Xr + t * kXs, x);
      // output layer: dL/do = dL/dsignal * S (1 - S), S from the forward
      const float sg = vis ? S[row] : 0.0f;
      const float dO = vis ? dL_dsignal[2 * row] * sg * (1.0f - sg) : 0.0f;
      sdO[t] = dO;
      float ds = dO;
#pragma unroll
      for (int q = 16; q > 0; q >>= 1) ds += __shfl_xor_sync(0xffffffffu, ds, q);
      if (lane == 0) atomicAdd(&dwo[kW64], ds);
    }
    // the forward's pre-activations of this thread's block: act(Z0) -> A0 rows
    // (two layers), the last hidden layer's Z -> acc
    float acc[8][4];
    if (kL == 2) {
      load_block4_T(Zt, r0, c0, acc);
#pragma unroll
      for (int i = 0; i < 8; ++i)
#pragma unroll
        for (int j = 0; j < 4; ++j) acc[i][j] = act_fwd(kAct, acc[i][j]);
      store_block4_rows(A0, r0, c0, acc);
    }
    load_block4_T(Zt + (kL - 1) * zl, r0, c0, acc);
    __syncthreads();   // dO and A0 ready
    {
      // output-layer weight gradient: this block's rows, then over the 16 row groups (lanes)
      float dOr[8];
#pragma unroll
      for (int i = 0; i < 8; ++i) dOr[i] = sdO[blk_row(r0, i)];
      float part[4];
#pragma unroll
      for (int j = 0; j < 4; ++j) {
        float p = 0.0f;
#pragma unroll
        for (int i = 0; i < 8; ++i) p = fmaf(dOr[i], act_fwd(kAct, acc[i][j]), p);
        part[j] = p;
      }
#pragma unroll
      for (int j = 0; j < 4; ++j)
#pragma unroll
        for (int q = 8; q > 0; q >>= 1) part[j] += __shfl_xor_sync(0xffffffffu, part[j], q);
      if ((t & 15) == 0)
#pragma unroll
        for (int j = 0; j < 4; ++j) atomicAdd(&dwo[c0 + j], part[j]);
      // dZ of the last hidden layer -> rows (D) and transposed (HT)
#pragma unroll
      for (int j = 0; j < 4; ++j) {
        const float w = wo[c0 + j];
#pragma unroll
        for (int i = 0; i < 8; ++i) acc[i][j] = dOr[i] * w * act_grad(kAct, acc[i][j]);
      }
      store_block4_rows(D, r0, c0, acc);
      store_block4_T(HT, r0, c0, acc);
    }
    __syncthreads();
    if (kL == 2) {
      // second layer: dW1 += dZ1^T A0, db1 += column sums of dZ1
      tile_outer<4, kHs>(D, A0, j1, i1, (t & 15) == 0, g1, gb1);
      // dZ0 = (dZ1 W1) * act'(Z0)
#pragma unroll
      for (int i = 0; i < 8; ++i)
#pragma unroll
        for (int j = 0; j < 4; ++j) acc[i][j] = 0.0f;
      gemm_8x4<kW64>(HT, kFusedRows, sm + TL::kW1, kW64, r0, c0, acc);
      {
        float z[8][4];   // Z0 again (this CTA read it a moment ago: L2)
        load_block4_T(Zt, r0, c0, z);
#pragma unroll
        for (int i = 0; i < 8; ++i)
#pragma unroll
          for (int j = 0; j < 4; ++j) acc[i][j] *= act_grad(kAct, z[i][j]);
      }
      __syncthreads();   // D (dZ1) and HT (dZ1^T) fully read
      store_block4_rows(D, r0, c0, acc);
      store_block4_T(HT, r0, c0, acc);
      __syncthreads();
    }
    if (row_thread) {
      // first layer: dW0 += dZ0^T X, db0 += column sums of dZ0
      tile_outer<4, kXs>(D, Xr, j0, i0, (t & 7) == 0, g0, gb0);
      // dX = dZ0 W0 (feature gradient, to HBM)
      float dx[8][4];
#pragma unroll
      for (int i = 0; i < 8; ++i)
#pragma unroll
        for (int j = 0; j < 4; ++j) dx[i][j] = 0.0f;
      gemm_8x4<kW64>(HT, kFusedRows, sm + TL::kW0, kFeat, r0x, c0x, dx);
#pragma unroll
      for (int i = 0; i < 8; ++i) {
        const size_t rr = tile * kFusedRows + blk_row(r0x, i);
        if (rr < rows)
          *reinterpret_cast<float4*>(dX + rr * kFeat + c0x) = make_float4(dx[i][0], dx[i][1], dx[i][2], dx[i][3]);
      }
    }
    if (kFeatAdj) {   // one receiver (row = Gaussian): the feature adjoint of the tile here
      __syncthreads();              // the tile's dL/dx rows are written
      if (row_thread && row < rows)
        features_adjoint<true>((int)row, P, 1, means3D, rx_pos, radii, dX, dL_dmeans3D);
    }
  }
  __syncthreads();
  // this CTA's share -> global
#pragma unroll
  for (int u = 0; u < 4; ++u) {
    if (row_thread) {
#pragma unroll
      for (int i = 0; i < 4; ++i) atomicAdd(&dparams[FP::kW0 + (size_t)(j0 + u) * kFeat + i0 + i], g0[u][i]);
      if ((t & 7) == 0) atomicAdd(&dparams[FP::kB0 + j0 + u], gb0[u]);
    }
    if (kL == 2) {
#pragma unroll
      for (int i = 0; i < 4; ++i) atomicAdd(&dparams[FP::kW1 + (size_t)(j1 + u) * kW64 + i1 + i], g1[u][i]);
      if ((t & 15) == 0) atomicAdd(&dparams[FP::kB1 + j1 + u], gb1[u]);
    }
  }
  for (int j = t; j <= kW64; j += kAdjThreads) atomicAdd(&dparams[FP::kWo + j], dwo[j]);   // kWo + 64 = kBo
}

template <int kL, int kAct>
static cudaError_t launch_fused(bool fwd, int P, size_t rows, const float* means3D, const float* rx_pos,
                                const float* params, const GeomView& geo, const SharedMlpLayout& L, float* work,
                                const float* dL_dsignal, float* dparams, float* dmeans, cudaStream_t s) {
  const size_t smem = (size_t)(fwd ? FusedFwdSmem<kL>::kTotal : FusedTiles<kL>::kTotal) * sizeof(float);
  static bool attr_done[3][64] = {};   // forward, adjoint, adjoint with the feature adjoint
  const int variant = fwd ? 0 : (dmeans ? 2 : 1);
  static int sm_count[64] = {};
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return e;
  int sms = dev >= 0 && dev < 64 ? sm_count[dev] : 0;
  if (sms == 0) {
    if ((e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev)) != cudaSuccess) return e;
    if (dev >= 0 && dev < 64) sm_count[dev] = sms;
  }
  if (dev < 0 || dev >= 64 || !attr_done[variant][dev]) {
    e = fwd ? cudaFuncSetAttribute(mlp64_forward_kernel<kL, kAct>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                   (int)smem)
            : (dmeans ? cudaFuncSetAttribute(mlp64_backward_kernel<kL, kAct, true>,
                                             cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem)
                      : cudaFuncSetAttribute(mlp64_backward_kernel<kL, kAct, false>,
                                             cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    if (e != cudaSuccess) return e;
    if (dev >= 0 && dev < 64) attr_done[variant][dev] = true;
  }
  const size_t ntiles = (rows + kFusedRows - 1) / kFusedRows;
  if (fwd) {
    // persistent: as many CTAs per SM as fit (74 KB of shared memory each: three)
    static int per_sm[64][2][3] = {};
    int occ = dev >= 0 && dev < 64 ? per_sm[dev][kL - 1][kAct] : 0;
    if (occ == 0) {
      e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, mlp64_forward_kernel<kL, kAct>, kFusedRows, smem);
      if (e != cudaSuccess) return e;
      if (occ < 1) occ = 1;
      if (dev >= 0 && dev < 64) per_sm[dev][kL - 1][kAct] = occ;
    }
    const size_t cap = (size_t)sms * occ;
    mlp64_forward_kernel<kL, kAct><<<(unsigned)(ntiles < cap ? ntiles : cap), kFusedRows, smem, s>>>(
        P, rows, means3D, rx_pos, params, geo.radii, work + L.s, work + L.z[1], geo.signal);
    return cudaGetLastError();
  }
  const unsigned grid = (unsigned)(ntiles < (size_t)sms ? ntiles : (size_t)sms);
  if (dmeans)
    mlp64_backward_kernel<kL, kAct, true><<<grid, kAdjThreads, smem, s>>>(
        P, rows, means3D, rx_pos, params, geo.radii, work + L.s, work + L.z[1], dL_dsignal, work + L.d0, dparams, dmeans);
  else
    mlp64_backward_kernel<kL, kAct, false><<<grid, kAdjThreads, smem, s>>>(
        P, rows, means3D, rx_pos, params, geo.radii, work + L.s, work + L.z[1], dL_dsignal, work + L.d0, dparams,
        nullptr);
  return cudaGetLastError();
}

// dmeans: dL/dmeans3D when the adjoint also runs the feature adjoint (one receiver), else nullptr
static cudaError_t launch_fused_dispatch(bool fwd, int layers, int act, int P, size_t rows, const float* means3D,
                                         const float* rx_pos, const float* params, const GeomView& geo,
                                         const SharedMlpLayout& L, float* work, const float* dL_dsignal,
                                         float* dparams, float* dmeans, cudaStream_t s) {
  if (layers == 1)
    return act == 1
               ? launch_fused<1, 1>(fwd, P, rows, means3D, rx_pos, params, geo, L, work, dL_dsignal, dparams, dmeans, s)
               : launch_fused<1, 2>(fwd, P, rows, means3D, rx_pos, params, geo, L, work, dL_dsignal, dparams, dmeans, s);
  return act == 1
             ? launch_fused<2, 1>(fwd, P, rows, means3D, rx_pos, params, geo, L, work, dL_dsignal, dparams, dmeans, s)
             : launch_fused<2, 2>(fwd, P, rows, means3D, rx_pos, params, geo, L, work, dL_dsignal, dparams, dmeans, s);
}

// ---- layout of parameters and workspace ----------------------------------------
SharedMlpLayout shared_mlp_layout(int layers, int width, int out, size_t rows) {
  SharedMlpLayout L{};
  L.layers = layers;
  L.width = width;
  L.out = out;
  size_t p = 0;
  for (int l = 0; l <= layers; ++l) {
    const int in = l == 0 ? kFeat : width;
    const int o = l == layers ? out : width;
    L.w[l] = p;
    p += (size_t)o * in;
    L.b[l] = p;
    p += o;
  }
  L.params = p;
  auto al = [](size_t x) { return (x + 63) / 64 * 64; };   // 256-byte aligned segments
  size_t w = 0;
  if (shared_mlp_fused(layers, width, out)) {   // the fused kernels keep S, the hidden Z (tiles) and dL/dx
    L.s = w;
    w += al(rows);
    L.z[1] = w;
    w += (size_t)layers * ((rows + kFusedRows - 1) / kFusedRows) * kFusedRows * kW64;
    L.d0 = L.d1 = w;
    w += al(rows * kFeat);
    L.work = w;
    return L;
  }
  L.s = w;   // first: the sigmoid outputs [rows][out] (the amplitudes for out > 1)
  w += al(rows * out);
  L.x0 = w;
  w += al(rows * kFeat);
  for (int l = 1; l <= layers; ++l) {
    L.z[l] = w;
    w += al(rows * width);
    L.a[l] = w;
    w += al(rows * width);
  }
  L.o = w;
  w += al(rows * out);
  size_t dw = width > kFeat ? width : kFeat;
  if ((size_t)out > dw) dw = out;
  L.d0 = w;
  w += al(rows * dw);
  L.d1 = w;
  w += al(rows * dw);
  L.work = w;
  return L;
}

SharedMlpLayout shared_mlp_layout_bf16(int layers, size_t rows, int out) {
  SharedMlpLayout L = shared_mlp_layout(layers, 128, out, 0);   // parameter offsets as the FP32 path
  auto a = [](size_t x) { return (x + 63) / 64 * 64; };           // 256-byte aligned segments (vector access)
  size_t w = 0;
  L.s = w;   // first: the sigmoid outputs [rows][out] (the amplitudes for out > 1)
  w += a(rows * (size_t)out);
  L.z[1] = w;
  // BF16 pre-activations, two per float, for whole 128-row tiles (tile-transposed)
  w += a((size_t)layers * ((rows + 127) / 128 * 128) * 128 / 2);
  L.d0 = w;   // no feature-gradient segment: the adjoint applies it in place
  L.work = w;
  return L;
}

cudaError_t launch_mlp_features_backward(int P, int R, const float* means3D, const float* rx_pos, const int* radii,
                                         const float* dX, float* dL_dmeans3D, cudaStream_t s) {
  const unsigned blocks = (unsigned)(((long long)P * kFeatLanes + 255) / 256);
  mlp_features_backward_kernel<<<blocks, 256, 0, s>>>(P, R, means3D, rx_pos, radii, dX, dL_dmeans3D);
  return cudaGetLastError();
}

static cudaError_t gemm_fwd(size_t M, int N, int K, const float* A, const float* W, const float* bias, float* Z,
                            float* Aout, int act, cudaStream_t s) {
  dim3 grid((unsigned)((M + kBM - 1) / kBM), (N + kBN - 1) / kBN);
  mlp_gemm_kernel<kEpiFwd><<<grid, 256, 0, s>>>((int)M, N, K, 0, A, K, 1, W, 1, K, Z, N, bias, act, Aout, nullptr);
  return cudaGetLastError();
}

cudaError_t launch_shared_mlp_forward(int P, int R, int layers, int width, int act, int out, const float* means3D,
                                      const float* rx_pos, const float* params, const GeomView& geo,
                                      float* work, cudaStream_t s) {
  const size_t rows = (size_t)P * R;
  const SharedMlpLayout L = shared_mlp_layout(layers, width, out, rows);
  if (shared_mlp_fused(layers, width, out))
    return launch_fused_dispatch(true, layers, act, P, rows, means3D, rx_pos, params, geo, L, work, nullptr, nullptr,
                                 nullptr, s);
  mlp_features_kernel<<<dim3((P + 255) / 256, R), 256, 0, s>>>(P, means3D, rx_pos, geo.radii, work + L.x0);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return e;
  const float* in = work + L.x0;
  int kin = kFeat;
  for (int l = 1; l <= layers; ++l) {
    e = gemm_fwd(rows, width, kin, in, params + L.w[l - 1], params + L.b[l - 1], work + L.z[l], work + L.a[l], act, s);
    if (e != cudaSuccess) return e;
    in = work + L.a[l];
    kin = width;
  }
  // output layer (identity) into O, then the signal
  e = gemm_fwd(rows, out, kin, in, params + L.w[layers], params + L.b[layers], work + L.o, work + L.o, 0, s);
  if (e != cudaSuccess) return e;
  mlp_signal_kernel<<<(unsigned)((rows + 255) / 256), 256, 0, s>>>(rows, out, work + L.o, geo.radii, work + L.s,
                                                                    geo.signal);
  return cudaGetLastError();
}

cudaError_t launch_shared_mlp_backward(int P, int R, int layers, int width, int act, int out, const float* means3D,
                                       const float* rx_pos, const float* params, const GeomView& geo, float* work,
                                       const float* dL_dsignal, float* dL_dparams, float* dL_dmeans3D,
                                       cudaStream_t s) {
  const size_t rows = (size_t)P * R;
  const SharedMlpLayout L = shared_mlp_layout(layers, width, out, rows);
  cudaError_t e = cudaMemsetAsync(dL_dparams, 0, L.params * sizeof(float), s);
  if (e != cudaSuccess) return e;
  if (shared_mlp_fused(layers, width, out)) {
    // one receiver: the adjoint finishes each tile's feature adjoint itself (row = Gaussian)
    e = launch_fused_dispatch(false, layers, act, P, rows, means3D, rx_pos, params, geo, L, work, dL_dsignal,
                              dL_dparams, R == 1 ? dL_dmeans3D : nullptr, s);
    if (e != cudaSuccess || R == 1) return e;
    return launch_mlp_features_backward(P, R, means3D, rx_pos, geo.radii, work + L.d0, dL_dmeans3D, s);
  }
  float* dcur = work + L.d1;   // dZ of the current layer
  float* dnext = work + L.d0;
  mlp_signal_backward_kernel<<<(unsigned)((rows + 255) / 256), 256, 0, s>>>(rows, out, work + L.s, geo.radii,
                                                                             dL_dsignal, dcur);
  if ((e = cudaGetLastError()) != cudaSuccess) return e;
  for (int l = layers; l >= 0; --l) {
    const int o = l == layers ? out : width;
    const int in = l == 0 ? kFeat : width;
    const float* xin = l == 0 ? work + L.x0 : work + L.a[l];
    // dW_l[o, in] += sum_rows dZ[row, o] * X[row, in]: the row sum is split
    // over grid.z so that about four CTAs per SM run, each folding its partial
    // tile into dW with one atomic per element; chunks stay >= 128 rows.
    {
      const unsigned gxy = (unsigned)(((o + kBM - 1) / kBM) * ((in + kBN - 1) / kBN));
      const long long want_z = std::max<long long>(1, (4LL * device_sm_count()) / gxy);
      long long kchunk = (rows + want_z - 1) / want_z;
      kchunk = std::max<long long>(128, (kchunk + kBK - 1) / kBK * kBK);
      const unsigned zsplit = (unsigned)((rows + kchunk - 1) / kchunk);
      dim3 grid((o + kBM - 1) / kBM, (in + kBN - 1) / kBN, zsplit);
      mlp_gemm_kernel<kEpiAtomic><<<grid, 256, 0, s>>>(o, in, (int)rows, (int)kchunk, dcur, 1, o, xin, in, 1,
                                                       dL_dparams + L.w[l], in, nullptr, 0, nullptr, nullptr);
      if ((e = cudaGetLastError()) != cudaSuccess) return e;
      mlp_colsum_kernel<<<dim3((o + 31) / 32, (unsigned)((rows + 2047) / 2048)), 256, 0, s>>>(
          (int)rows, o, dcur, dL_dparams + L.b[l]);
      if ((e = cudaGetLastError()) != cudaSuccess) return e;
    }
    // dX_{l}[row, in] = sum_o dZ[row, o] W_l[o, in], times act'(Z_l) below the output layer
    {
      dim3 grid((unsigned)((rows + kBM - 1) / kBM), (in + kBN - 1) / kBN);
      mlp_gemm_kernel<kEpiDx><<<grid, 256, 0, s>>>((int)rows, in, o, 0, dcur, o, 1, params + L.w[l], in, 1, dnext,
                                                    in, nullptr, l == 0 ? 0 : act, nullptr,
                                                    l == 0 ? nullptr : work + L.z[l]);
      if ((e = cudaGetLastError()) != cudaSuccess) return e;
    }
    float* t = dcur;
    dcur = dnext;
    dnext = t;
  }
  // dcur now holds dL/dx of the features
  return launch_mlp_features_backward(P, R, means3D, rx_pos, geo.radii, dcur, dL_dmeans3D, s);
}

}  // namespace gsparc
