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

// ---------------------------------------------------------------------------
// Training loss of one step over R spectra (train.py:420-436 per receiver,
// averaged over the receivers of a batch):
//   l1_r    = mean |pred - target|                       (utils.py:40-41)
//   ssim_r  = mean SSIM map                              (fused_ssim, "same")
//   recon_r = (1 - lambda1) l1_r + lambda1 (1 - ssim_r)
//   conf_r  = 1 + exp(fc2(relu(fc1(rx_r))))              (gaussian.py:575-609)
//   loss    = mean_r (conf_r recon_r - alpha log conf_r)
// and its adjoint with respect to pred and the confidence-MLP parameters,
// in two launches: tile moments + per-tile partial sums, whose last CTA runs
// the head (reductions, MLP forward/backward, per-receiver gradient scales),
// then the SSIM/L1 backward with the per-receiver scales applied while
// staging.
// Every reduction has a fixed order, so the loss is deterministic.
// ---------------------------------------------------------------------------

__device__ __forceinline__ float warp_sum_all(float v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

__device__ __forceinline__ void loss_head_body(int R, int nblk, int HW, int hidden, float lambda1, float alpha,
                                               const float* __restrict__ rx, const float* __restrict__ cp,
                                               const float2* __restrict__ partial, float* __restrict__ pre,
                                               float4* __restrict__ coef, float* __restrict__ terms,
                                               float* __restrict__ loss_out, float* __restrict__ dconf);

// Tile moments, SSIM partial derivatives and per-tile partial sums; the last
// CTA to finish (arrival counter in the scratch) runs the head.
__global__ void __launch_bounds__(256)
loss_forward_kernel(int H, int W, float C1, float C2, const float* __restrict__ pred,
                    const float* __restrict__ target, float* __restrict__ dm_dmu1,
                    float* __restrict__ dm_dsigma1_sq, float* __restrict__ dm_dsigma12,
                    float2* __restrict__ partial, int hidden, float lambda1, float alpha,
                    const float* __restrict__ rx, const float* __restrict__ cp, float* __restrict__ pre,
                    float4* __restrict__ coef, float* __restrict__ terms, float* __restrict__ loss_out,
                    float* __restrict__ dconf, unsigned* __restrict__ arrived) {
  __shared__ float s1[kTH][kTW + 1];
  __shared__ float s2[kTH][kTW + 1];
  __shared__ float hx[5][kTH][kSW];
  __shared__ float red[2][8];
  const size_t plane = (size_t)blockIdx.z * H * W;
  const int x0 = blockIdx.x * kSW - kHalo, y0 = blockIdx.y * kSH - kHalo;
  stage_tile(s1, pred + plane, H, W, x0, y0);
  stage_tile(s2, target + plane, H, W, x0, y0);
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
  const float C = (2.0f * (mu1 * mu2) + C1);
  const float D = (2.0f * sigma12 + C2);
  const float A = (mu1 * mu1 + mu2 * mu2 + C1);
  const float B = (sigma1_sq + sigma2_sq + C2);
  const int px = blockIdx.x * kSW + lx, py = blockIdx.y * kSH + ly;
  float l1 = 0.0f, sm = 0.0f;
  if (px < W && py < H) {
    const size_t idx = plane + (size_t)py * W + px;
    sm = (C * D) / (A * B);
    l1 = fabsf(s1[ly + kHalo][lx + kHalo] - s2[ly + kHalo][lx + kHalo]);
    dm_dmu1[idx] = ((mu2 * 2.0f * D) / (A * B) - (mu2 * 2.0f * C) / (A * B) - (mu1 * 2.0f * C * D) / (A * A * B) +
                    (mu1 * 2.0f * C * D) / (A * B * B));
    dm_dsigma1_sq[idx] = ((-C * D) / (A * B * B));
    dm_dsigma12[idx] = ((2 * C) / (A * B));
  }
  l1 = warp_sum_all(l1);
  sm = warp_sum_all(sm);
  if ((threadIdx.x & 31) == 0) {
    red[0][threadIdx.x >> 5] = l1;
    red[1][threadIdx.x >> 5] = sm;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    float a = 0.0f, b = 0.0f;
#pragma unroll
    for (int w = 0; w < 8; ++w) { a += red[0][w]; b += red[1][w]; }
    partial[((size_t)blockIdx.z * gridDim.y + blockIdx.y) * gridDim.x + blockIdx.x] = make_float2(a, b);
  }
  __shared__ bool s_last;
  if (threadIdx.x == 0) {
    __threadfence();
    s_last = atomicAdd(arrived, 1u) == gridDim.x * gridDim.y * gridDim.z - 1;
  }
  __syncthreads();
  if (s_last) {
    __threadfence();
    loss_head_body(gridDim.z, gridDim.x * gridDim.y, H * W, hidden, lambda1, alpha, rx, cp, partial, pre, coef,
                   terms, loss_out, dconf);
    if (threadIdx.x == 0) *arrived = 0u;
  }
}

// One CTA: warp per receiver for the reductions and the confidence MLP
// forward, then thread per MLP parameter for its gradient (sum over
// receivers in receiver order).  coef[r] = (dL/dpred scale of the L1 term,
// dL/dmap of the SSIM term, loss_r, dL/draw_r).
__device__ __forceinline__ void loss_head_body(int R, int nblk, int HW, int hidden, float lambda1, float alpha,
                                               const float* __restrict__ rx,
                 const float* __restrict__ cp, const float2* __restrict__ partial, float* __restrict__ pre,
                 float4* __restrict__ coef, float* __restrict__ terms, float* __restrict__ loss_out,
                 float* __restrict__ dconf) {
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const float* w1 = cp;
  const float* b1 = cp + 3 * hidden;
  const float* w2 = b1 + hidden;
  const float b2 = w2[hidden];
  const float n = (float)HW, fR = (float)R;
  for (int r = warp; r < R; r += 8) {
    float a = 0.0f, b = 0.0f;
    for (int i = lane; i < nblk; i += 32) {
      const float2 p = __ldcg(partial + (size_t)r * nblk + i);   // written by other CTAs
      a += p.x;
      b += p.y;
    }
    a = warp_sum_all(a);
    b = warp_sum_all(b);
    const float l1 = a / n, ssim = b / n;
    const float x0 = rx[3 * r], x1 = rx[3 * r + 1], x2 = rx[3 * r + 2];
    float acc = 0.0f;
    for (int j = lane; j < hidden; j += 32) {
      const float p = w1[3 * j] * x0 + w1[3 * j + 1] * x1 + w1[3 * j + 2] * x2 + b1[j];
      pre[(size_t)r * hidden + j] = p;
      acc += w2[j] * fmaxf(p, 0.0f);
    }
    acc = warp_sum_all(acc);
    const float e = expf(acc + b2);
    const float conf = 1.0f + e;
    const float recon = (1.0f - lambda1) * l1 + lambda1 * (1.0f - ssim);
    const float loss_r = conf * recon - alpha * logf(conf);
    const float g_rec = conf / fR;
    const float draw = ((recon - alpha / conf) / fR) * e;
    if (lane == 0) {
      coef[r] = make_float4((g_rec * (1.0f - lambda1)) / n, -(g_rec * lambda1) / n, loss_r, draw);
      if (terms) {
        terms[4 * r] = l1;
        terms[4 * r + 1] = ssim;
        terms[4 * r + 2] = conf;
        terms[4 * r + 3] = loss_r;
      }
    }
  }
  __syncthreads();
  const int np = 5 * hidden + 1;
  for (int p = threadIdx.x; p < np; p += blockDim.x) {
    float g = 0.0f;
    if (p < 3 * hidden) {            // fc1.weight [hidden, 3]
      const int j = p / 3, k = p % 3;
      for (int r = 0; r < R; ++r)
        if (pre[(size_t)r * hidden + j] > 0.0f) g += (coef[r].w * w2[j]) * rx[3 * r + k];
    } else if (p < 4 * hidden) {     // fc1.bias
      const int j = p - 3 * hidden;
      for (int r = 0; r < R; ++r)
        if (pre[(size_t)r * hidden + j] > 0.0f) g += coef[r].w * w2[j];
    } else if (p < 5 * hidden) {     // fc2.weight [1, hidden]
      const int j = p - 4 * hidden;
      for (int r = 0; r < R; ++r) g += coef[r].w * fmaxf(pre[(size_t)r * hidden + j], 0.0f);
    } else {                         // fc2.bias
      for (int r = 0; r < R; ++r) g += coef[r].w;
    }
    dconf[p] = g;
  }
  if (threadIdx.x == 0) {
    float s = 0.0f;
    for (int r = 0; r < R; ++r) s += coef[r].z;
    loss_out[0] = s / fR;
  }
}

__device__ __forceinline__ void stage_scaled(float (*dst)[kTW + 1], const float* __restrict__ a, float c, int H,
                                             int W, int x0, int y0) {
  for (int i = threadIdx.x; i < kTH * kTW; i += blockDim.x) {
    const int ly = i / kTW, lx = i % kTW;
    const int gy = y0 + ly, gx = x0 + lx;
    dst[ly][lx] = (gx >= 0 && gy >= 0 && gx < W && gy < H) ? a[(size_t)gy * W + gx] * c : 0.0f;
  }
}

// SSIM backward (as ssim_backward_kernel) with a map gradient that is the
// same for every pixel of a spectrum, plus the L1 term scale * sign(p - t).
__global__ void __launch_bounds__(256)
loss_backward_kernel(int H, int W, const float* __restrict__ pred, const float* __restrict__ target,
                     const float* __restrict__ dm_dmu1, const float* __restrict__ dm_dsigma1_sq,
                     const float* __restrict__ dm_dsigma12, const float4* __restrict__ coef,
                     float* __restrict__ dL_dpred) {
  __shared__ float sp[3][kTH][kTW + 1];
  __shared__ float hx[3][kTH][kSW];
  const size_t plane = (size_t)blockIdx.z * H * W;
  const float4 cf = coef[blockIdx.z];
  const int x0 = blockIdx.x * kSW - kHalo, y0 = blockIdx.y * kSH - kHalo;
  stage_scaled(sp[0], dm_dmu1 + plane, cf.y, H, W, x0, y0);
  stage_scaled(sp[1], dm_dsigma1_sq + plane, cf.y, H, W, x0, y0);
  stage_scaled(sp[2], dm_dsigma12 + plane, cf.y, H, W, x0, y0);
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
    const float pix1 = pred[idx], pix2 = target[idx];
    float g = 0.0f;
    g += v[0];
    g += pix1 * 2.0f * v[1];
    g += pix2 * v[2];
    const float d = pix1 - pix2;
    const float sgn = (d > 0.0f) ? 1.0f : ((d < 0.0f) ? -1.0f : 0.0f);
    dL_dpred[idx] = cf.x * sgn + g;
  }
}

LossLayout loss_layout(size_t R, size_t H, size_t W, size_t hidden) {
  auto a = [](size_t x) { return (x + 63) / 64 * 64; };
  LossLayout L;
  const size_t n = R * H * W;
  L.nblk = ((W + kSW - 1) / kSW) * ((H + kSH - 1) / kSH);
  L.dmu1 = 0;
  L.ds11 = a(n);
  L.ds12 = L.ds11 + a(n);
  L.partial = L.ds12 + a(n);
  L.pre = L.partial + a(2 * R * L.nblk);
  L.coef = L.pre + a(R * hidden);
  L.sync = L.coef + a(4 * R);
  L.total = L.sync + 64;
  return L;
}

cudaError_t launch_splat_loss(int R, int H, int W, int hidden, float lambda1, float alpha, float C1, float C2,
                              const float* pred, const float* target, const float* rx, const float* conf_params,
                              float* scratch, float* loss_out, float* terms, float* dL_dpred, float* dconf,
                              cudaStream_t stream) {
  const LossLayout L = loss_layout(R, H, W, hidden);
  dim3 grid((W + kSW - 1) / kSW, (H + kSH - 1) / kSH, R);
  float2* partial = reinterpret_cast<float2*>(scratch + L.partial);
  float4* coef = reinterpret_cast<float4*>(scratch + L.coef);
  loss_forward_kernel<<<grid, 256, 0, stream>>>(H, W, C1, C2, pred, target, scratch + L.dmu1, scratch + L.ds11,
                                                scratch + L.ds12, partial, hidden, lambda1, alpha, rx, conf_params,
                                                scratch + L.pre, coef, terms, loss_out, dconf,
                                                reinterpret_cast<unsigned*>(scratch + L.sync));
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return e;
  loss_backward_kernel<<<grid, 256, 0, stream>>>(H, W, pred, target, scratch + L.dmu1, scratch + L.ds11,
                                                 scratch + L.ds12, coef, dL_dpred);
  return cudaGetLastError();
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
