// Fused SSIM (11x11 Gaussian window, sigma 1.5, zero "same" padding).
//
// Same mathematics as fused-ssim/ssim.cu (forward 187-286, backward
// 288-366): separable convolution along x then y, SSIM map, and the three
// partial derivatives dm/dmu1, dm/dsigma1^2, dm/dsigma12 that the backward
// convolves.  Per-pixel accumulation order (taps 0..10, x pass then y pass)
// is the reference's, so the map matches it bit for bit.
//
// Layout: one CTA per 32x8 output tile per image plane (grid.z = B*CH), so a
// 90x360 spectrum spreads over 144 CTAs (the reference's 32x32 tiles give 36).
// Both images are staged once with their 5-pixel halo; all five moments are
// filtered from the same staged tile in one horizontal pass (the reference
// restages and rescans the tile five times).
#include "common.cuh"
#include "kernels.cuh"

namespace gsparc {

// The window of utils.py:116-124 (gaussian(11, 1.5) normalised in float32).
__constant__ float kSsimWin[11] = {
    0.001028380123898387f, 0.0075987582094967365f, 0.036000773310661316f, 0.10936068743467331f,
    0.21300552785396576f,  0.26601171493530273f,   0.21300552785396576f,  0.10936068743467331f,
    0.036000773310661316f, 0.0075987582094967365f, 0.001028380123898387f};

constexpr int kSW = 32, kSH = 8, kHalo = 5;
constexpr int kTW = kSW + 2 * kHalo;   // 42
constexpr int kTH = kSH + 2 * kHalo;   // 18

__device__ __forceinline__ void stage_tile(float (*dst)[kTW + 1], const float* __restrict__ src, int H, int W,
                                           int x0, int y0) {
  for (int i = threadIdx.x; i < kTH * kTW; i += blockDim.x) {
    const int ly = i / kTW, lx = i % kTW;
    const int gy = y0 + ly, gx = x0 + lx;
    dst[ly][lx] = (gx >= 0 && gy >= 0 && gx < W && gy < H) ? src[(size_t)gy * W + gx] : 0.0f;
  }
}

__global__ void __launch_bounds__(256)
ssim_forward_kernel(int H, int W, float C1, float C2, const float* __restrict__ img1,
                    const float* __restrict__ img2, float* __restrict__ ssim_map,
                    float* __restrict__ dm_dmu1, float* __restrict__ dm_dsigma1_sq,
                    float* __restrict__ dm_dsigma12) {
  __shared__ float s1[kTH][kTW + 1];
  __shared__ float s2[kTH][kTW + 1];
  __shared__ float hx[5][kTH][kSW];
  const size_t plane = (size_t)blockIdx.z * H * W;
  const int x0 = blockIdx.x * kSW - kHalo, y0 = blockIdx.y * kSH - kHalo;
  stage_tile(s1, img1 + plane, H, W, x0, y0);
  stage_tile(s2, img2 + plane, H, W, x0, y0);
  __syncthreads();
  for (int i = threadIdx.x; i < kTH * kSW; i += blockDim.x) {
    const int ly = i / kSW, lx = i % kSW;
    float a = 0.0f, b = 0.0f, c = 0.0f, d = 0.0f, e = 0.0f;
#pragma unroll
    for (int k = 0; k < 11; ++k) {
      const float p = s1[ly][lx + k], q = s2[ly][lx + k];
      const float w = kSsimWin[k];
      a += w * p;
      b += w * (p * p);
      c += w * q;
      d += w * (q * q);
      e += w * (p * q);
    }
    hx[0][ly][lx] = a; hx[1][ly][lx] = b; hx[2][ly][lx] = c; hx[3][ly][lx] = d; hx[4][ly][lx] = e;
  }
  __syncthreads();
  const int lx = threadIdx.x % kSW, ly = threadIdx.x / kSW;
  float v[5] = {0.f, 0.f, 0.f, 0.f, 0.f};
#pragma unroll
  for (int q = 0; q < 5; ++q)
#pragma unroll
    for (int k = 0; k < 11; ++k) v[q] += kSsimWin[k] * hx[q][ly + k][lx];
  const float mu1 = v[0];
  const float sigma1_sq = v[1] - mu1 * mu1;
  const float mu2 = v[2];
  const float sigma2_sq = v[3] - mu2 * mu2;
  const float sigma12 = v[4] - mu1 * mu2;
  const float mu1_sq = mu1 * mu1;
  const float mu2_sq = mu2 * mu2;
  const float mu1_mu2 = mu1 * mu2;
  const float C = (2.0f * mu1_mu2 + C1);
  const float D = (2.0f * sigma12 + C2);
  const float A = (mu1_sq + mu2_sq + C1);
  const float B = (sigma1_sq + sigma2_sq + C2);
  const float m = (C * D) / (A * B);
  const int px = blockIdx.x * kSW + lx, py = blockIdx.y * kSH + ly;
  if (px < W && py < H) {
    const size_t idx = plane + (size_t)py * W + px;
    ssim_map[idx] = m;
    if (dm_dmu1) {
      dm_dmu1[idx] = ((mu2 * 2.0f * D) / (A * B) - (mu2 * 2.0f * C) / (A * B) - (mu1 * 2.0f * C * D) / (A * A * B) +
                      (mu1 * 2.0f * C * D) / (A * B * B));
      dm_dsigma1_sq[idx] = ((-C * D) / (A * B * B));
      dm_dsigma12[idx] = ((2 * C) / (A * B));
    }
  }
}

__device__ __forceinline__ void stage_product(float (*dst)[kTW + 1], const float* __restrict__ a,
                                              const float* __restrict__ b, int H, int W, int x0, int y0) {
  for (int i = threadIdx.x; i < kTH * kTW; i += blockDim.x) {
    const int ly = i / kTW, lx = i % kTW;
    const int gy = y0 + ly, gx = x0 + lx;
    float v = 0.0f;
    if (gx >= 0 && gy >= 0 && gx < W && gy < H) {
      const size_t o = (size_t)gy * W + gx;
      v = a[o] * b[o];
    }
    dst[ly][lx] = v;
  }
}

__global__ void __launch_bounds__(256)
ssim_backward_kernel(int H, int W, const float* __restrict__ img1, const float* __restrict__ img2,
                     const float* __restrict__ dL_dmap, const float* __restrict__ dm_dmu1,
                     const float* __restrict__ dm_dsigma1_sq, const float* __restrict__ dm_dsigma12,
                     float* __restrict__ dL_dimg1) {
  __shared__ float sp[3][kTH][kTW + 1];
  __shared__ float hx[3][kTH][kSW];
  const size_t plane = (size_t)blockIdx.z * H * W;
  const int x0 = blockIdx.x * kSW - kHalo, y0 = blockIdx.y * kSH - kHalo;
  stage_product(sp[0], dm_dmu1 + plane, dL_dmap + plane, H, W, x0, y0);
  stage_product(sp[1], dm_dsigma1_sq + plane, dL_dmap + plane, H, W, x0, y0);
  stage_product(sp[2], dm_dsigma12 + plane, dL_dmap + plane, H, W, x0, y0);
  __syncthreads();
  for (int i = threadIdx.x; i < kTH * kSW; i += blockDim.x) {
    const int ly = i / kSW, lx = i % kSW;
    float a = 0.0f, b = 0.0f, c = 0.0f;
#pragma unroll
    for (int k = 0; k < 11; ++k) {
      const float w = kSsimWin[k];
      a += w * sp[0][ly][lx + k];
      b += w * sp[1][ly][lx + k];
      c += w * sp[2][ly][lx + k];
    }
    hx[0][ly][lx] = a; hx[1][ly][lx] = b; hx[2][ly][lx] = c;
  }
  __syncthreads();
  const int lx = threadIdx.x % kSW, ly = threadIdx.x / kSW;
  const int px = blockIdx.x * kSW + lx, py = blockIdx.y * kSH + ly;
  float v[3] = {0.f, 0.f, 0.f};
#pragma unroll
  for (int q = 0; q < 3; ++q)
#pragma unroll
    for (int k = 0; k < 11; ++k) v[q] += kSsimWin[k] * hx[q][ly + k][lx];
  if (px < W && py < H) {
    const size_t idx = plane + (size_t)py * W + px;
    const float pix1 = img1[idx], pix2 = img2[idx];
    float g = 0.0f;
    g += v[0];
    g += pix1 * 2.0f * v[1];
    g += pix2 * v[2];
    dL_dimg1[idx] = g;
  }
}

cudaError_t launch_ssim_forward(int planes, int H, int W, float C1, float C2, const float* img1, const float* img2,
                                float* map, float* dmu1, float* ds11, float* ds12, cudaStream_t stream) {
  if (planes == 0 || H == 0 || W == 0) return cudaSuccess;
  dim3 grid((W + kSW - 1) / kSW, (H + kSH - 1) / kSH, planes);
  ssim_forward_kernel<<<grid, 256, 0, stream>>>(H, W, C1, C2, img1, img2, map, dmu1, ds11, ds12);
  return cudaGetLastError();
}

cudaError_t launch_ssim_backward(int planes, int H, int W, const float* img1, const float* img2, const float* dL_dmap,
                                 const float* dmu1, const float* ds11, const float* ds12, float* dL_dimg1,
                                 cudaStream_t stream) {
  if (planes == 0 || H == 0 || W == 0) return cudaSuccess;
  dim3 grid((W + kSW - 1) / kSW, (H + kSH - 1) / kSH, planes);
  ssim_backward_kernel<<<grid, 256, 0, stream>>>(H, W, img1, img2, dL_dmap, dmu1, ds11, ds12, dL_dimg1);
  return cudaGetLastError();
}

}  // namespace gsparc
