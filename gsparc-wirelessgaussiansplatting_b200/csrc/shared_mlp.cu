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

// activation and its derivative together (one erf for GELU); same values as act_fwd / act_grad
__device__ __forceinline__ void act_both(int act, float z, float& a, float& d) {
  if (act == 2) {
    const float cdf = 0.5f * (1.0f + erff(z * 0.70710678118654752f));
    a = 0.5f * z * (1.0f + erff(z * 0.70710678118654752f));
    d = cdf + z * (0.39894228040143268f * expf(-0.5f * z * z));
  } else {
    a = act_fwd(act, z);
    d = act_grad(act, z);
  }
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

// dL/dmu from dL/dx, summed over receivers (thread per Gaussian).
__global__ void __launch_bounds__(256)
mlp_features_backward_kernel(int P, int R, const float* __restrict__ means3D, const float* __restrict__ rx_pos,
                             const int* __restrict__ radii, const float* __restrict__ dX,
                             float* __restrict__ dL_dmeans3D) {
  const int g = blockIdx.x * blockDim.x + threadIdx.x;
  if (g >= P) return;
  const float m[3] = {means3D[3 * g], means3D[3 * g + 1], means3D[3 * g + 2]};
  float acc[3] = {0.0f, 0.0f, 0.0f};
  // positional part does not depend on the receiver: sum dX over receivers first
  float sum_pe[kFeat];
#pragma unroll
  for (int i = 0; i < 27; ++i) sum_pe[i] = 0.0f;
  for (int r = 0; r < R; ++r) {
    const size_t row = (size_t)r * P + g;
    if (radii[row] <= 0) continue;
    const float* dx = dX + row * kFeat;
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

// signal = sigmoid(o_0) for visible pairs; dO = dL/dsignal_real * s (1 - s)
__global__ void __launch_bounds__(256)
mlp_signal_kernel(size_t rows, int Cout, const float* __restrict__ O, const int* __restrict__ radii,
                  float* __restrict__ S, float2* __restrict__ signal) {
  const size_t row = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
  if (row >= rows) return;
  const float s = 1.0f / (1.0f + expf(-O[row * Cout]));
  S[row] = s;
  if (radii[row] > 0) signal[row] = make_float2(s, 0.0f);
}

__global__ void __launch_bounds__(256)
mlp_signal_backward_kernel(size_t rows, int Cout, const float* __restrict__ S, const int* __restrict__ radii,
                           const float* __restrict__ dL_dsignal, float* __restrict__ dO) {
  const size_t row = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
  if (row >= rows) return;
  const float s = S[row];
  const float g = radii[row] > 0 ? dL_dsignal[2 * row] * s * (1.0f - s) : 0.0f;
  for (int c = 0; c < Cout; ++c) dO[row * Cout + c] = c == 0 ? g : 0.0f;
}

// ---- fused path: width 64, one output, one or two hidden layers --------------
// One row (receiver, Gaussian pair) per thread with the network evaluated in
// registers and the weights in shared memory (every thread reads the same
// weight at the same time: broadcast).  Each layer's sums run in the same
// order as the tiled GEMMs above (inputs ascending from zero, then + bias), so
// the forward matches them bit for bit.  The adjoint recomputes the forward (no
// activations go to HBM) and reduces the weight gradients over each tile of
// 128 rows in shared memory, accumulating per thread across tiles.
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

// acc[j] = sum_i v[i] * W[j][i] over i ascending, for one output j (W row-major)
template <int N>
__device__ __forceinline__ float dot_row(const float* __restrict__ v, const float* __restrict__ wrow) {
  const float4* w = reinterpret_cast<const float4*>(wrow);
  float acc = 0.0f;
#pragma unroll
  for (int q = 0; q < N / 4; ++q) {
    const float4 w4 = w[q];
    acc = fmaf(v[4 * q], w4.x, acc);
    acc = fmaf(v[4 * q + 1], w4.y, acc);
    acc = fmaf(v[4 * q + 2], w4.z, acc);
    acc = fmaf(v[4 * q + 3], w4.w, acc);
  }
  return acc;
}

template <int kL, int kAct>
__global__ void __launch_bounds__(kFusedRows)
mlp64_forward_kernel(int P, size_t rows, const float* __restrict__ means3D, const float* __restrict__ rx_pos,
                     const float* __restrict__ params, const int* __restrict__ radii, float* __restrict__ S,
                     float2* __restrict__ signal) {
  using FP = FusedParams<kL>;
  // W0 transposed ([32][64]: the first layer runs input-outer over 64 accumulators), then the rest as given
  constexpr int kWt0 = 0, kRest = kW64 * kFeat;
  __shared__ __align__(16) float sp[FP::kPadded];
  for (int i = threadIdx.x; i < kW64 * kFeat; i += blockDim.x) {
    const int k = i / kW64, j = i % kW64;
    sp[kWt0 + i] = params[FP::kW0 + j * kFeat + k];
  }
  for (int i = kRest + threadIdx.x; i < FP::kCount; i += blockDim.x) sp[i] = params[i];
  __syncthreads();
  for (size_t row = blockIdx.x * (size_t)blockDim.x + threadIdx.x; row < rows; row += (size_t)gridDim.x * blockDim.x) {
    if (radii[row] <= 0) continue;
    float x[kFeat];
    pair_features_fp32(means3D, rx_pos, (int)(row % P), (int)(row / P), x);
    float a0[kW64];
#pragma unroll
    for (int j = 0; j < kW64; ++j) a0[j] = 0.0f;
#pragma unroll
    for (int k = 0; k < kFeat; ++k) {
      const float4* w = reinterpret_cast<const float4*>(sp + kWt0 + k * kW64);
#pragma unroll
      for (int q = 0; q < kW64 / 4; ++q) {
        const float4 w4 = w[q];
        a0[4 * q] = fmaf(x[k], w4.x, a0[4 * q]);
        a0[4 * q + 1] = fmaf(x[k], w4.y, a0[4 * q + 1]);
        a0[4 * q + 2] = fmaf(x[k], w4.z, a0[4 * q + 2]);
        a0[4 * q + 3] = fmaf(x[k], w4.w, a0[4 * q + 3]);
      }
    }
#pragma unroll
    for (int j = 0; j < kW64; ++j) a0[j] = act_fwd(kAct, a0[j] + sp[FP::kB0 + j]);
    float o = 0.0f;
    if (kL == 1) {
#pragma unroll
      for (int j = 0; j < kW64; ++j) o = fmaf(a0[j], sp[FP::kWo + j], o);
    } else {
#pragma unroll 4
      for (int j = 0; j < kW64; ++j)
        o = fmaf(act_fwd(kAct, dot_row<kW64>(a0, sp + FP::kW1 + j * kW64) + sp[FP::kB1 + j]), sp[FP::kWo + j], o);
    }
    const float sg = 1.0f / (1.0f + expf(-(o + sp[FP::kBo])));
    S[row] = sg;
    signal[row] = make_float2(sg, 0.0f);
  }
}

// Sum of v[i] over the warp, returned in lane i (v is overwritten).
__device__ __forceinline__ float warp_sum_transpose32(float* v, int lane) {
#pragma unroll
  for (int half = 16; half >= 1; half >>= 1) {
    const bool upper = lane & half;
#pragma unroll
    for (int i = 0; i < half; ++i) {
      const float send = upper ? v[i] : v[i + half];
      const float keep = upper ? v[i + half] : v[i];
      v[i] = keep + __shfl_xor_sync(0xffffffffu, send, half);
    }
  }
  return v[0];
}

// Shared-memory tiles of the adjoint (floats; row strides keep float4 rows
// aligned and 8 consecutive rows on distinct banks).
constexpr int kXs = kFeat + 4, kHs = kW64 + 4;

template <int kL>
struct FusedTiles {
  using FP = FusedParams<kL>;
  static constexpr int kX = FP::kPadded;
  static constexpr int kA0 = kX + kFusedRows * kXs;        // act(Z0) rows (two layers)
  static constexpr int kZ0 = kA0 + (kL == 2 ? kFusedRows * kHs : 0);
  static constexpr int kD1 = kZ0 + (kL == 2 ? kFusedRows * kHs : 0);   // Z1, then dZ1, rows (two layers)
  static constexpr int kD0 = kD1 + (kL == 2 ? kFusedRows * kHs : 0);   // Z0 then dZ0 (one layer); dZ0
  static constexpr int kDwo = kD0 + kFusedRows * kHs;      // output-layer weight gradient, then its bias
  static constexpr int kTotal = kDwo + kW64 + 4;
};

// acc[4][NI] += sum over the tile's rows of D[r][j0..j0+3] (x) A[r][i0..i0+NI-1];
// bsum[4] += sum of D[r][j0..j0+3] when `bias`
template <int NI, int kAs>
__device__ __forceinline__ void tile_outer(const float* __restrict__ D, const float* __restrict__ A, int j0, int i0,
                                           bool bias, float (&acc)[4][NI], float (&bsum)[4]) {
#pragma unroll 4
  for (int r = 0; r < kFusedRows; ++r) {
    const float4 d = *reinterpret_cast<const float4*>(D + r * kHs + j0);
    float a[NI];
#pragma unroll
    for (int q = 0; q < NI / 4; ++q) {
      const float4 v = *reinterpret_cast<const float4*>(A + r * kAs + i0 + 4 * q);
      a[4 * q] = v.x; a[4 * q + 1] = v.y; a[4 * q + 2] = v.z; a[4 * q + 3] = v.w;
    }
    const float dd[4] = {d.x, d.y, d.z, d.w};
#pragma unroll
    for (int u = 0; u < 4; ++u) {
#pragma unroll
      for (int i = 0; i < NI; ++i) acc[u][i] = fmaf(dd[u], a[i], acc[u][i]);
      if (bias) bsum[u] += dd[u];
    }
  }
}

template <int N>
__device__ __forceinline__ void load_row(const float* __restrict__ src, float* v) {
#pragma unroll
  for (int q = 0; q < N / 4; ++q) {
    const float4 a = reinterpret_cast<const float4*>(src)[q];
    v[4 * q] = a.x; v[4 * q + 1] = a.y; v[4 * q + 2] = a.z; v[4 * q + 3] = a.w;
  }
}
template <int N>
__device__ __forceinline__ void store_row(float* dst, const float* v) {
#pragma unroll
  for (int q = 0; q < N / 4; ++q)
    reinterpret_cast<float4*>(dst)[q] = make_float4(v[4 * q], v[4 * q + 1], v[4 * q + 2], v[4 * q + 3]);
}

// One layer of the forward in dot form for this thread's row: z[j] (and
// act(z)) for j in 0..63, written four at a time to the row's tile slots.
template <int N, int kAct>
__device__ __forceinline__ void layer_rows(const float* v, const float* __restrict__ W, const float* __restrict__ b,
                                           float* zrow, float* arow) {
#pragma unroll 2
  for (int j = 0; j < kW64; j += 4) {
    float z[4];
#pragma unroll
    for (int u = 0; u < 4; ++u) z[u] = dot_row<N>(v, W + (j + u) * N) + b[j + u];
    reinterpret_cast<float4*>(zrow)[j / 4] = make_float4(z[0], z[1], z[2], z[3]);
    if (arow)
      reinterpret_cast<float4*>(arow)[j / 4] =
          make_float4(act_fwd(kAct, z[0]), act_fwd(kAct, z[1]), act_fwd(kAct, z[2]), act_fwd(kAct, z[3]));
  }
}

template <int kL, int kAct>
__global__ void __launch_bounds__(kFusedRows, 1)
mlp64_backward_kernel(int P, size_t rows, const float* __restrict__ means3D, const float* __restrict__ rx_pos,
                      const float* __restrict__ params, const int* __restrict__ radii,
                      const float* __restrict__ dL_dsignal, float* __restrict__ dX, float* __restrict__ dparams) {
  using FP = FusedParams<kL>;
  using TL = FusedTiles<kL>;
  extern __shared__ __align__(16) float sm[];
  const int t = threadIdx.x, lane = t & 31;
  for (int i = t; i < FP::kCount; i += blockDim.x) sm[i] = params[i];
  for (int i = t; i < kW64 + 4; i += blockDim.x) sm[TL::kDwo + i] = 0.0f;
  __syncthreads();
  const float* W0 = sm + FP::kW0;
  const float* W1 = sm + FP::kW1;
  const float* wo = sm + FP::kWo;
  float* Xs = sm + TL::kX;
  float* A0 = sm + TL::kA0;
  float* Z0 = sm + TL::kZ0;
  float* D1 = sm + TL::kD1;
  float* D0 = sm + TL::kD0;
  float* dwo = sm + TL::kDwo;
  // the last hidden layer's pre-activation / dZ rows
  float* DL = kL == 2 ? D1 : D0;

  // this thread's blocks of the weight gradients, accumulated over all tiles
  const int j0 = (t >> 3) * 4;
  const bool bias_owner = (t & 7) == 0;
  float g1[4][8] = {}, gb1[4] = {};   // second layer: outputs j0..j0+3 x inputs (t & 7) * 8 ..+7
  float g0[4][4] = {}, gb0[4] = {};   // first layer: outputs j0..j0+3 x features (t & 7) * 4 ..+3
  const size_t ntiles = (rows + kFusedRows - 1) / kFusedRows;
  for (size_t tile = blockIdx.x; tile < ntiles; tile += gridDim.x) {
    const size_t row = tile * kFusedRows + t;
    const bool vis = row < rows && radii[row] > 0;
    float* xr = Xs + t * kXs;
    float* dl = DL + t * kHs;
    float red[kW64];   // dO * act(z) of the last hidden layer: this row's output-layer gradient
    float dO = 0.0f;
    if (!vis) {   // zero rows: they add nothing to the reductions
#pragma unroll
      for (int j = 0; j < kW64; ++j) red[j] = 0.0f;
      store_row<kFeat>(xr, red);
      store_row<kW64>(dl, red);
      if (kL == 2) {
        store_row<kW64>(A0 + t * kHs, red);
        store_row<kW64>(Z0 + t * kHs, red);
      }
    } else {
      // ---- forward recompute (same sums as mlp64_forward_kernel), Z of the
      // last hidden layer into its dZ slots
      {
        float x[kFeat];
        pair_features_fp32(means3D, rx_pos, (int)(row % P), (int)(row / P), x);
        store_row<kFeat>(xr, x);
        if (kL == 1) layer_rows<kFeat, kAct>(x, W0, sm + FP::kB0, dl, nullptr);
        else layer_rows<kFeat, kAct>(x, W0, sm + FP::kB0, Z0 + t * kHs, A0 + t * kHs);
      }
      if (kL == 2) {
        float a0[kW64];
        load_row<kW64>(A0 + t * kHs, a0);
        layer_rows<kW64, kAct>(a0, W1, sm + FP::kB1, dl, nullptr);
      }
      float zl[kW64];
      load_row<kW64>(dl, zl);
      float o = 0.0f;
#pragma unroll
      for (int j = 0; j < kW64; ++j) o = fmaf(act_fwd(kAct, zl[j]), wo[j], o);
      const float sg = 1.0f / (1.0f + expf(-(o + sm[FP::kBo])));
      dO = dL_dsignal[2 * row] * sg * (1.0f - sg);
      // zl becomes dZ of the last hidden layer in place
#pragma unroll
      for (int j = 0; j < kW64; ++j) {
        float a, d;
        act_both(kAct, zl[j], a, d);
        red[j] = dO * a;
        zl[j] = dO * wo[j] * d;
      }
      store_row<kW64>(dl, zl);
    }
    {
      const float s0 = warp_sum_transpose32(red, lane);
      const float s1 = warp_sum_transpose32(red + 32, lane);
      atomicAdd(&dwo[lane], s0);
      atomicAdd(&dwo[32 + lane], s1);
      float ds = dO;
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) ds += __shfl_xor_sync(0xffffffffu, ds, o);
      if (lane == 0) atomicAdd(&dwo[kW64], ds);
    }
    __syncthreads();
    if (kL == 2) {
      // second layer: dW1 += D1^T A0, db1 += column sums of D1
      tile_outer<8, kHs>(D1, A0, j0, (t & 7) * 8, bias_owner, g1, gb1);
      // dZ0 = (W1^T dZ1) * act'(Z0) for this row: dZ1-outer over 64 accumulators
      float da[kW64];
#pragma unroll
      for (int k = 0; k < kW64; ++k) da[k] = 0.0f;
      if (vis) {
#pragma unroll 2
        for (int j = 0; j < kW64; ++j) {
          const float dj = D1[t * kHs + j];
          const float4* w = reinterpret_cast<const float4*>(W1 + j * kW64);
#pragma unroll
          for (int q = 0; q < kW64 / 4; ++q) {
            const float4 w4 = w[q];
            da[4 * q] = fmaf(dj, w4.x, da[4 * q]);
            da[4 * q + 1] = fmaf(dj, w4.y, da[4 * q + 1]);
            da[4 * q + 2] = fmaf(dj, w4.z, da[4 * q + 2]);
            da[4 * q + 3] = fmaf(dj, w4.w, da[4 * q + 3]);
          }
        }
        float z0[kW64];
        load_row<kW64>(Z0 + t * kHs, z0);
#pragma unroll
        for (int k = 0; k < kW64; ++k) da[k] *= act_grad(kAct, z0[k]);
      }
      store_row<kW64>(D0 + t * kHs, da);
    }
    // dX = W0^T dZ0 for this row (feature gradient, to HBM): dZ0-outer over 32 accumulators
    if (row < rows) {
      float dx[kFeat];
#pragma unroll
      for (int k = 0; k < kFeat; ++k) dx[k] = 0.0f;
#pragma unroll 2
      for (int j = 0; j < kW64; ++j) {
        const float dj = D0[t * kHs + j];
        const float4* w = reinterpret_cast<const float4*>(W0 + j * kFeat);
#pragma unroll
        for (int q = 0; q < kFeat / 4; ++q) {
          const float4 w4 = w[q];
          dx[4 * q] = fmaf(dj, w4.x, dx[4 * q]);
          dx[4 * q + 1] = fmaf(dj, w4.y, dx[4 * q + 1]);
          dx[4 * q + 2] = fmaf(dj, w4.z, dx[4 * q + 2]);
          dx[4 * q + 3] = fmaf(dj, w4.w, dx[4 * q + 3]);
        }
      }
      store_row<kFeat>(dX + row * kFeat, dx);
    }
    __syncthreads();
    // first layer: dW0 += D0^T X, db0 += column sums of D0
    tile_outer<4, kXs>(D0, Xs, j0, (t & 7) * 4, bias_owner, g0, gb0);
    __syncthreads();
  }
  // this CTA's share -> global
#pragma unroll
  for (int u = 0; u < 4; ++u) {
#pragma unroll
    for (int i = 0; i < 4; ++i) atomicAdd(&dparams[FP::kW0 + (size_t)(j0 + u) * kFeat + (t & 7) * 4 + i], g0[u][i]);
    if (bias_owner) atomicAdd(&dparams[FP::kB0 + j0 + u], gb0[u]);
    if (kL == 2) {
#pragma unroll
      for (int i = 0; i < 8; ++i) atomicAdd(&dparams[FP::kW1 + (size_t)(j0 + u) * kW64 + (t & 7) * 8 + i], g1[u][i]);
      if (bias_owner) atomicAdd(&dparams[FP::kB1 + j0 + u], gb1[u]);
    }
  }
  for (int j = t; j <= kW64; j += blockDim.x) atomicAdd(&dparams[FP::kWo + j], dwo[j]);   // kWo + 64 = kBo
}

template <int kL, int kAct>
static cudaError_t launch_fused(bool fwd, int P, size_t rows, const float* means3D, const float* rx_pos,
                                const float* params, const GeomView& geo, const SharedMlpLayout& L, float* work,
                                const float* dL_dsignal, float* dparams, cudaStream_t s) {
  if (fwd) {
    const size_t blocks = (rows + kFusedRows - 1) / kFusedRows;
    mlp64_forward_kernel<kL, kAct><<<(unsigned)(blocks < 148 * 16 ? blocks : 148 * 16), kFusedRows, 0, s>>>(
        P, rows, means3D, rx_pos, params, geo.radii, work + L.s, geo.signal);
    return cudaGetLastError();
  }
  const size_t smem = (size_t)FusedTiles<kL>::kTotal * sizeof(float);
  static bool attr_done[64] = {};
  static int sm_count[64] = {};
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return e;
  int sms = dev >= 0 && dev < 64 ? sm_count[dev] : 0;
  if (sms == 0) {
    if ((e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev)) != cudaSuccess) return e;
    if (dev >= 0 && dev < 64) sm_count[dev] = sms;
  }
  if (dev < 0 || dev >= 64 || !attr_done[dev]) {
    e = cudaFuncSetAttribute(mlp64_backward_kernel<kL, kAct>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
    if (dev >= 0 && dev < 64) attr_done[dev] = true;
  }
  const size_t ntiles = (rows + kFusedRows - 1) / kFusedRows;
  const unsigned grid = (unsigned)(ntiles < (size_t)sms ? ntiles : (size_t)sms);
  mlp64_backward_kernel<kL, kAct><<<grid, kFusedRows, smem, s>>>(P, rows, means3D, rx_pos, params, geo.radii,
                                                                 dL_dsignal, work + L.d0, dparams);
  return cudaGetLastError();
}

static cudaError_t launch_fused_dispatch(bool fwd, int layers, int act, int P, size_t rows, const float* means3D,
                                         const float* rx_pos, const float* params, const GeomView& geo,
                                         const SharedMlpLayout& L, float* work, const float* dL_dsignal,
                                         float* dparams, cudaStream_t s) {
  if (layers == 1)
    return act == 1 ? launch_fused<1, 1>(fwd, P, rows, means3D, rx_pos, params, geo, L, work, dL_dsignal, dparams, s)
                    : launch_fused<1, 2>(fwd, P, rows, means3D, rx_pos, params, geo, L, work, dL_dsignal, dparams, s);
  return act == 1 ? launch_fused<2, 1>(fwd, P, rows, means3D, rx_pos, params, geo, L, work, dL_dsignal, dparams, s)
                  : launch_fused<2, 2>(fwd, P, rows, means3D, rx_pos, params, geo, L, work, dL_dsignal, dparams, s);
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
  if (shared_mlp_fused(layers, width, out)) {   // the fused kernels keep only S and dL/dx
    L.s = w;
    w += al(rows);
    L.d0 = L.d1 = w;
    w += al(rows * kFeat);
    L.work = w;
    return L;
  }
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
  L.s = w;
  w += al(rows);
  size_t dw = width > kFeat ? width : kFeat;
  if ((size_t)out > dw) dw = out;
  L.d0 = w;
  w += al(rows * dw);
  L.d1 = w;
  w += al(rows * dw);
  L.work = w;
  return L;
}

SharedMlpLayout shared_mlp_layout_bf16(int layers, size_t rows) {
  SharedMlpLayout L = shared_mlp_layout(layers, 128, 1, 0);   // parameter offsets as the FP32 path
  auto a = [](size_t x) { return (x + 63) / 64 * 64; };         // 256-byte aligned segments (vector access)
  size_t w = 0;
  L.z[1] = w;
  w += a((size_t)layers * rows * 128 / 2);   // BF16 pre-activations, two per float
  L.s = w;
  w += a(rows);
  L.d0 = w;
  w += a(rows * kFeat);
  L.work = w;
  return L;
}

cudaError_t launch_mlp_features_backward(int P, int R, const float* means3D, const float* rx_pos, const int* radii,
                                         const float* dX, float* dL_dmeans3D, cudaStream_t s) {
  mlp_features_backward_kernel<<<(P + 255) / 256, 256, 0, s>>>(P, R, means3D, rx_pos, radii, dX, dL_dmeans3D);
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
                                 s);
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
    e = launch_fused_dispatch(false, layers, act, P, rows, means3D, rx_pos, params, geo, L, work, dL_dsignal,
                              dL_dparams, s);
    if (e != cudaSuccess) return e;
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
      const long long want_z = std::max<long long>(1, (4 * 148) / gxy);
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
  mlp_features_backward_kernel<<<(P + 255) / 256, 256, 0, s>>>(P, R, means3D, rx_pos, geo.radii, dcur,
                                                               dL_dmeans3D);
  return cudaGetLastError();
}

}  // namespace gsparc
