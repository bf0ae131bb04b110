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
