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
// in two launches:
//   1. SSIM moments, map derivatives and per-block partial sums of |p - t|
//      and the map.  The last block of each spectrum runs that spectrum's
//      head (its means, the confidence MLP forward, the per-spectrum
//      gradient scales and its share of every confidence-parameter
//      gradient); the last head sums the shares and the loss in spectrum
//      order.
//   2. The SSIM/L1 backward with the per-spectrum scales applied while
//      staging.
// Two block layouts run the same per-pixel arithmetic: 32x8 tiles with their
// halo (few spectra: 144 blocks per 90x360 spectrum), or 128-column strips
// that walk down a band of rows with the vertical window in registers (many
// spectra: each input row is filtered horizontally once instead of 2.25
// times, and no halo rows are staged twice).
// Every reduction has a fixed order, so the loss is deterministic.
// ---------------------------------------------------------------------------

__device__ __forceinline__ float warp_sum_all(float v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

// SSIM of one pixel from its five window moments (mu1, E[x^2], mu2, E[y^2],
// E[xy]), and the three partial derivatives the backward convolves
// (fused-ssim/ssim.cu:262-283): the same quantities, with the seven
// divisions by A B, A^2 B and A B^2 taken as products with the correctly
// rounded reciprocals of A and B (a few ulps from the quotient form).
__device__ __forceinline__ float ssim_pixel(const float (&v)[5], float C1, float C2, float& d_mu1, float& d_s11,
                                            float& d_s12) {
  const float mu1 = v[0];
  const float sigma1_sq = v[1] - mu1 * mu1;
  const float mu2 = v[2];
  const float sigma2_sq = v[3] - mu2 * mu2;
  const float sigma12 = v[4] - mu1 * mu2;
  const float C = (2.0f * (mu1 * mu2) + C1);
  const float D = (2.0f * sigma12 + C2);
  const float A = (mu1 * mu1 + mu2 * mu2 + C1);
  const float B = (sigma1_sq + sigma2_sq + C2);
  const float ia = __frcp_rn(A), ib = __frcp_rn(B);
  const float iab = ia * ib;
  const float m = (C * D) * iab;
  const float m2 = (mu1 * 2.0f) * m;
  d_mu1 = (mu2 * 2.0f) * (D - C) * iab - m2 * ia + m2 * ib;
  d_s11 = -m * ib;
  d_s12 = (2.0f * C) * iab;
  return m;
}

struct LossHead {
  int R, hidden;
  float lambda1, alpha;
  const float* rx;   // [R][3]
  const float* cp;   // confidence MLP: fc1.weight [hidden][3], fc1.bias, fc2.weight [hidden], fc2.bias
  float* pre;        // [R][hidden] fc1 pre-activations
  float4* coef;      // [R]
  float* terms;      // [R][4] or null
  float* loss_out;
  float* dconf;      // [5 hidden + 1]
  float* share;      // [R][5 hidden + 1] per-spectrum parameter-gradient terms
  unsigned* psync;   // [R] arrivals per spectrum
  unsigned* sync;    // heads done
};

// Spectrum r's head: mean L1 and SSIM (block partials in block order), the
// confidence MLP forward, coef[r] = (dL/dpred scale of the L1 term, dL/dmap
// of the SSIM term, loss_r, dL/draw_r), and r's term of every confidence
// parameter's gradient.
__device__ void loss_spectrum_head(int r, int nblk, int HW, const LossHead& h, const float2* __restrict__ partial) {
  __shared__ float s_draw;
  const int hidden = h.hidden;
  const float* w1 = h.cp;
  const float* b1 = h.cp + 3 * hidden;
  const float* w2 = b1 + hidden;
  const float b2 = w2[hidden];
  const float* x = h.rx + 3 * r;
  if (threadIdx.x < 32) {
    const int lane = threadIdx.x;
    float a = 0.0f, b = 0.0f;
    for (int i = lane; i < nblk; i += 32) {
      const float2 p = __ldcg(partial + (size_t)r * nblk + i);   // written by other blocks
      a += p.x;
      b += p.y;
    }
    a = warp_sum_all(a);
    b = warp_sum_all(b);
    const float n = (float)HW, fR = (float)h.R;
    const float l1 = a / n, ssim = b / n;
    float acc = 0.0f;
    for (int j = lane; j < hidden; j += 32) {
      const float p = w1[3 * j] * x[0] + w1[3 * j + 1] * x[1] + w1[3 * j + 2] * x[2] + b1[j];
      h.pre[(size_t)r * hidden + j] = p;
      acc += w2[j] * fmaxf(p, 0.0f);
    }
    acc = warp_sum_all(acc);
    const float e = expf(acc + b2);
    const float conf = 1.0f + e;
    const float recon = (1.0f - h.lambda1) * l1 + h.lambda1 * (1.0f - ssim);
    const float loss_r = conf * recon - h.alpha * logf(conf);
    const float g_rec = conf / fR;
    const float draw = ((recon - h.alpha / conf) / fR) * e;
    if (lane == 0) {
      h.coef[r] = make_float4((g_rec * (1.0f - h.lambda1)) / n, -(g_rec * h.lambda1) / n, loss_r, draw);
      if (h.terms) {
        h.terms[4 * r] = l1;
        h.terms[4 * r + 1] = ssim;
        h.terms[4 * r + 2] = conf;
        h.terms[4 * r + 3] = loss_r;
      }
      s_draw = draw;
    }
  }
  __syncthreads();
  const float cw = s_draw;
  const int np = 5 * hidden + 1;
  float* sh = h.share + (size_t)r * np;
  for (int p = threadIdx.x; p < np; p += blockDim.x) {
    float g;
    if (p < 3 * hidden) {            // fc1.weight [hidden, 3]
      const int j = p / 3, k = p % 3;
      g = __ldcg(h.pre + (size_t)r * hidden + j) > 0.0f ? (cw * w2[j]) * x[k] : 0.0f;
    } else if (p < 4 * hidden) {     // fc1.bias
      const int j = p - 3 * hidden;
      g = __ldcg(h.pre + (size_t)r * hidden + j) > 0.0f ? cw * w2[j] : 0.0f;
    } else if (p < 5 * hidden) {     // fc2.weight [1, hidden]
      const int j = p - 4 * hidden;
      g = cw * fmaxf(__ldcg(h.pre + (size_t)r * hidden + j), 0.0f);
    } else {                         // fc2.bias
      g = cw;
    }
    sh[p] = g;
  }
}

// The confidence-parameter gradients and the loss: sums over the spectra in
// spectrum order.
// The confidence-parameter gradients and the loss: sums over the spectra in a
// fixed order (eight interleaved partial sums per parameter, so that eight
// loads are in flight; lane-strided sums for the loss).
__device__ void loss_final(const LossHead& h) {
  const int np = 5 * h.hidden + 1;
  for (int p = threadIdx.x; p < np; p += blockDim.x) {
    float acc[8] = {0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f};
    int r = 0;
    for (; r + 8 <= h.R; r += 8)
#pragma unroll
      for (int i = 0; i < 8; ++i) acc[i] += __ldcg(h.share + (size_t)(r + i) * np + p);
#pragma unroll
    for (int i = 0; i < 7; ++i)
      if (r + i < h.R) acc[i] += __ldcg(h.share + (size_t)(r + i) * np + p);
    h.dconf[p] = ((acc[0] + acc[1]) + (acc[2] + acc[3])) + ((acc[4] + acc[5]) + (acc[6] + acc[7]));
  }
  if (threadIdx.x < 32) {
    float s = 0.0f;
    for (int r = threadIdx.x; r < h.R; r += 32) s += __ldcg(h.coef + r).z;
    s = warp_sum_all(s);
    if (threadIdx.x == 0) h.loss_out[0] = s / (float)h.R;
  }
}

// Called by every thread after thread 0 wrote the block's partial: the last
// block of spectrum blockIdx.z runs its head, the last head the final sums.
// Each counter is reset by its last user, so the scratch stays reusable.
__device__ void loss_arrive(int nblk, int HW, const LossHead& h, const float2* __restrict__ partial) {
  __shared__ int s_last;
  if (threadIdx.x == 0) {
    __threadfence();
    s_last = atomicAdd(h.psync + blockIdx.z, 1u) == (unsigned)nblk - 1u;
  }
  __syncthreads();
  if (!s_last) return;
  __threadfence();
  loss_spectrum_head((int)blockIdx.z, nblk, HW, h, partial);
  __threadfence();   // this block's coef / terms / share before the head count
  __syncthreads();
  if (threadIdx.x == 0) {
    h.psync[blockIdx.z] = 0u;
    s_last = atomicAdd(h.sync, 1u) == (unsigned)h.R - 1u;
  }
  __syncthreads();
  if (!s_last) return;
  __threadfence();
  loss_final(h);
  if (threadIdx.x == 0) *h.sync = 0u;
}

// Block partial (sum of |p - t|, sum of the map) from every thread's values,
// reduced in a fixed order; written by thread 0.
__device__ __forceinline__ void block_partial(float l1, float sm, float2* __restrict__ partial) {
  __shared__ float red[2][32];
  l1 = warp_sum_all(l1);
  sm = warp_sum_all(sm);
  if ((threadIdx.x & 31) == 0) {
    red[0][threadIdx.x >> 5] = l1;
    red[1][threadIdx.x >> 5] = sm;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    float a = 0.0f, b = 0.0f;
    for (int w = 0; w < (int)(blockDim.x >> 5); ++w) {
      a += red[0][w];
      b += red[1][w];
    }
    partial[((size_t)blockIdx.z * gridDim.y + blockIdx.y) * gridDim.x + blockIdx.x] = make_float2(a, b);
  }
}

// ---- evaluation metrics (train.py:76-102, 686-694) ---------------------------
// Per spectrum: PSNR = 20 log10(1 / sqrt(mse)) (infinite when mse = 0), the
// RSSI difference 10 log10(mean pred^2) - 10 log10(mean target^2) (the -30 dBm
// reference cancels), MAE, mean SSIM (the window SSIM of utils.py:81-114,
// the same map), the confidence 1 + exp(fc2(relu(fc1(rx)))) and the
// evaluation loss (1 - lambda1) MAE + lambda1 (1 - SSIM).  The SSIM pass of
// the loss runs without its map derivatives and sums five per-block values.
struct EvalOut {
  float* partial;     // [R][nblk][kEvalSums]
  unsigned* psync;    // [R] arrivals per spectrum
  const float* rx;    // [R][3]
  const float* cp;    // confidence MLP
  int hidden;
  float lambda1;
  float* metrics;     // [R][GSPARC_EVAL_METRICS]
};
constexpr int kEvalSums = 8;   // |p - t|, map, (p - t)^2, p^2, t^2, (three unused)

__device__ void eval_spectrum_head(int r, int nblk, int HW, const EvalOut& ev) {
  if (threadIdx.x >= 32) return;
  const int lane = threadIdx.x;
  float s[5] = {0.f, 0.f, 0.f, 0.f, 0.f};
  for (int i = lane; i < nblk; i += 32) {
    const float* q = ev.partial + ((size_t)r * nblk + i) * kEvalSums;
#pragma unroll
    for (int k = 0; k < 5; ++k) s[k] += __ldcg(q + k);   // written by other blocks
  }
#pragma unroll
  for (int k = 0; k < 5; ++k) s[k] = warp_sum_all(s[k]);
  const int hidden = ev.hidden;
  const float* w1 = ev.cp;
  const float* b1 = ev.cp + 3 * hidden;
  const float* w2 = b1 + hidden;
  const float* x = ev.rx + 3 * r;
  float acc = 0.0f;
  for (int j = lane; j < hidden; j += 32) {
    const float p = w1[3 * j] * x[0] + w1[3 * j + 1] * x[1] + w1[3 * j + 2] * x[2] + b1[j];
    acc += w2[j] * fmaxf(p, 0.0f);
  }
  acc = warp_sum_all(acc);
  if (lane == 0) {
    const float n = (float)HW;
    const float mae = s[0] / n, ssim = s[1] / n, mse = s[2] / n;
    const float psnr = mse == 0.0f ? __int_as_float(0x7f800000) : 20.0f * log10f(1.0f / sqrtf(mse));
    const float rssi_p = 10.0f * log10f(s[3] / n) - 30.0f, rssi_t = 10.0f * log10f(s[4] / n) - 30.0f;
    float* m = ev.metrics + (size_t)r * GSPARC_EVAL_METRICS;
    m[0] = psnr;
    m[1] = rssi_p - rssi_t;
    m[2] = mae;
    m[3] = ssim;
    m[4] = 1.0f + expf(acc + w2[hidden]);
    m[5] = (1.0f - ev.lambda1) * mae + ev.lambda1 * (1.0f - ssim);
  }
}

// Block sums (fixed order) written by thread 0, then the last block of the
// spectrum runs its head.
__device__ void eval_arrive(const float (&v)[5], int nblk, int HW, const EvalOut& ev) {
  __shared__ float red[5][32];
  __shared__ int s_last;
  float w[5];
#pragma unroll
  for (int k = 0; k < 5; ++k) w[k] = warp_sum_all(v[k]);
  if ((threadIdx.x & 31) == 0)
#pragma unroll
    for (int k = 0; k < 5; ++k) red[k][threadIdx.x >> 5] = w[k];
  __syncthreads();
  if (threadIdx.x == 0) {
    float* q = ev.partial + (((size_t)blockIdx.z * gridDim.y + blockIdx.y) * gridDim.x + blockIdx.x) * kEvalSums;
#pragma unroll
    for (int k = 0; k < 5; ++k) {
      float a = 0.0f;
      for (int i = 0; i < (int)(blockDim.x >> 5); ++i) a += red[k][i];
      q[k] = a;
    }
    __threadfence();
    s_last = atomicAdd(ev.psync + blockIdx.z, 1u) == (unsigned)nblk - 1u;
  }
  __syncthreads();
  if (!s_last) return;
  __threadfence();
  eval_spectrum_head((int)blockIdx.z, nblk, HW, ev);
  if (threadIdx.x == 0) ev.psync[blockIdx.z] = 0u;
}

// ---- tile layout: 32x8 outputs per block with the 5-pixel halo --------------

// kEval: the evaluation pass (no map derivatives; EvalOut sums and heads)
template <bool kEval>
__global__ void __launch_bounds__(256)
loss_forward_kernel(int H, int W, float C1, float C2, const float* __restrict__ pred,
                    const float* __restrict__ target, float* __restrict__ dm_dmu1,
                    float* __restrict__ dm_dsigma1_sq, float* __restrict__ dm_dsigma12,
                    float2* __restrict__ partial, LossHead head, EvalOut ev) {
  __shared__ float s1[kTH][kTW + 1];
  __shared__ float s2[kTH][kTW + 1];
  __shared__ float hx[5][kTH][kSW];
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
  const int px = blockIdx.x * kSW + lx, py = blockIdx.y * kSH + ly;
  float l1 = 0.0f, sm = 0.0f, sq = 0.0f, pp = 0.0f, tt = 0.0f;
  if (px < W && py < H) {
    const size_t idx = plane + (size_t)py * W + px;
    float d1, d2, d3;
    sm = ssim_pixel(v, C1, C2, d1, d2, d3);
    const float p = s1[ly + kHalo][lx + kHalo], q = s2[ly + kHalo][lx + kHalo];
    l1 = fabsf(p - q);
    if constexpr (kEval) {
      sq = (p - q) * (p - q);
      pp = p * p;
      tt = q * q;
    } else {
      dm_dmu1[idx] = d1;
      dm_dsigma1_sq[idx] = d2;
      dm_dsigma12[idx] = d3;
    }
  }
  if constexpr (kEval) {
    const float vals[5] = {l1, sm, sq, pp, tt};
    eval_arrive(vals, gridDim.x * gridDim.y, H * W, ev);
  } else {
    block_partial(l1, sm, partial);
    loss_arrive(gridDim.x * gridDim.y, H * W, head, partial);
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

// The L1 and SSIM terms of dL/dpred for one pixel: the map gradient is the
// same for every pixel of a spectrum, so the three convolved derivative maps
// arrive already scaled by it (fused-ssim/ssim.cu:288-366).
__device__ __forceinline__ float loss_pixel_grad(const float (&v)[3], float pix1, float pix2, float l1_scale) {
  float g = 0.0f;
  g += v[0];
  g += pix1 * 2.0f * v[1];
  g += pix2 * v[2];
  const float d = pix1 - pix2;
  const float sgn = (d > 0.0f) ? 1.0f : ((d < 0.0f) ? -1.0f : 0.0f);
  return l1_scale * sgn + g;
}

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
    dL_dpred[idx] = loss_pixel_grad(v, pred[idx], target[idx], cf.x);
  }
}

// ---- strip layout: 128 columns per block, walking down a band of rows ------
// Input rows are staged 11 at a time (one window height) by cp.async into a
// double buffer; each thread filters its column of every input row
// horizontally into a ring of 11 rows held in registers, and an output row is
// the vertical window over the ring once the 11 rows around it are in.
// Paired quantities (p and t, their squares, two of the three derivative
// maps) are staged interleaved and filtered with the FP32x2 instructions of
// sm_100, whose lanes round exactly as the scalar ones: the per-pixel
// arithmetic and its order are the tile layout's.

constexpr int kBandThreads = 128;                     // output columns per strip
constexpr int kBandCols = kBandThreads + 2 * kHalo;   // 138 staged columns
constexpr int kBandPitch = kBandCols + 2;
constexpr int kRing = 11;                             // window height = rows per staged chunk
constexpr int kBandMinPlanes = 16;                    // fewer spectra: tile layout
constexpr size_t kBandTargetBlocks = 592;             // four 4-warp blocks per SM

// {w_k, w_k}: the window as FP32x2 operands
__constant__ float2 kSsimWin2[11] = {
    {0.001028380123898387f, 0.001028380123898387f},   {0.0075987582094967365f, 0.0075987582094967365f},
    {0.036000773310661316f, 0.036000773310661316f},   {0.10936068743467331f, 0.10936068743467331f},
    {0.21300552785396576f, 0.21300552785396576f},     {0.26601171493530273f, 0.26601171493530273f},
    {0.21300552785396576f, 0.21300552785396576f},     {0.10936068743467331f, 0.10936068743467331f},
    {0.036000773310661316f, 0.036000773310661316f},   {0.0075987582094967365f, 0.0075987582094967365f},
    {0.001028380123898387f, 0.001028380123898387f}};

__device__ __forceinline__ void cp_async4(float* dst, const float* src, bool ok) {
  asm volatile("cp.async.ca.shared.global [%0], [%1], 4, %2;" ::"r"((uint32_t)__cvta_generic_to_shared(dst)),
               "l"(src), "r"(ok ? 4 : 0)
               : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
__device__ __forceinline__ void cp_async_wait_prev() { asm volatile("cp.async.wait_group 1;" ::: "memory"); }

// Staged chunk: rows yin0 .. yin0 + 10, columns x0 - 5 .. x0 + 132, zero
// outside the image (nothing is read there; the source address stays the
// plane's base).  Images 0 and 1 interleave as float2 [row][column]; image 2
// (if any) follows as float [row][column].  Thread i copies columns i and
// i + 128 of every row and image, and scales its own copies in the backward.
__device__ __forceinline__ int band_slot(int im, int j, int col) {
  return im < 2 ? (j * kBandPitch + col) * 2 + im : 2 * kRing * kBandPitch + j * kBandPitch + col;
}
template <int kImgs>
__device__ __forceinline__ void band_stage(float* dst, const float* const (&src)[kImgs], int H, int W, int x0,
                                           int yin0) {
#pragma unroll
  for (int half = 0; half < 2; ++half) {
    const int col = (int)threadIdx.x + half * kBandThreads;
    if (col < kBandCols) {
      const int gx = x0 - kHalo + col;
      const bool cok = gx >= 0 && gx < W;
#pragma unroll
      for (int j = 0; j < kRing; ++j) {
        const int gy = yin0 + j;
        const bool ok = cok && gy >= 0 && gy < H;
        const size_t o = ok ? (size_t)gy * W + gx : 0;
#pragma unroll
        for (int im = 0; im < kImgs; ++im) cp_async4(dst + band_slot(im, j, col), src[im] + o, ok);
      }
    }
  }
}

template <bool kEval>
__global__ void __launch_bounds__(kBandThreads)
loss_forward_band_kernel(int H, int W, int hb, float C1, float C2, const float* __restrict__ pred,
                         const float* __restrict__ target, float* __restrict__ dm_dmu1,
                         float* __restrict__ dm_dsigma1_sq, float* __restrict__ dm_dsigma12,
                         float2* __restrict__ partial, LossHead head, EvalOut ev) {
  __shared__ __align__(16) float s_in[2][2 * kRing * kBandPitch];
  const size_t plane = (size_t)blockIdx.z * H * W;
  const int x0 = blockIdx.x * kBandThreads, x = x0 + (int)threadIdx.x;
  const int y0 = blockIdx.y * hb, y1 = min(H, y0 + hb);
  const int n_in = y1 - y0 + 2 * kHalo;   // input rows y0 - 5 .. y1 + 4
  const int nchunks = (n_in + kRing - 1) / kRing;
  const float* const src[2] = {pred + plane, target + plane};
  float2 w2[11];
#pragma unroll
  for (int k = 0; k < 11; ++k) w2[k] = kSsimWin2[k];
  // ring of horizontal moments per input row: (a, c) = (mu1, mu2), (b, d) = (E x^2, E y^2), e = E xy
  float2 r_ac[kRing], r_bd[kRing];
  float r_e[kRing];
  float l1 = 0.0f, sm = 0.0f, sq = 0.0f, pp = 0.0f, tt = 0.0f;
  band_stage<2>(s_in[0], src, H, W, x0, y0 - kHalo);
  cp_async_commit();
  for (int ci = 0; ci < nchunks; ++ci) {
    if (ci + 1 < nchunks) band_stage<2>(s_in[(ci + 1) & 1], src, H, W, x0, y0 - kHalo + (ci + 1) * kRing);
    cp_async_commit();
    cp_async_wait_prev();
    __syncthreads();
    const float2* spq = reinterpret_cast<const float2*>(s_in[ci & 1]) + threadIdx.x;   // (p, t) pairs
#pragma unroll
    for (int j = 0; j < kRing; ++j) {
      const int g = ci * kRing + j;   // input row y0 - 5 + g; its ring slot is g % 11 = j
      if (g < n_in) {
        float2 ac = make_float2(0.0f, 0.0f), bd = make_float2(0.0f, 0.0f);
        float e = 0.0f;
#pragma unroll
        for (int k = 0; k < 11; ++k) {
          const float2 pq = spq[j * kBandPitch + k];
          ac = ffma2(w2[k], pq, ac);               // a += w p;      c += w q
          bd = ffma2(w2[k], fmul2(pq, pq), bd);    // b += w (p p);  d += w (q q)
          e = fmaf(w2[k].x, pq.x * pq.y, e);       // e += w (p q)
        }
        r_ac[j] = ac;
        r_bd[j] = bd;
        r_e[j] = e;
        if (g >= kHalo && g < n_in - kHalo && x < W) {
          const float2 c = spq[j * kBandPitch + kHalo];
          l1 += fabsf(c.x - c.y);
          if constexpr (kEval) {
            sq += (c.x - c.y) * (c.x - c.y);
            pp += c.x * c.x;
            tt += c.y * c.y;
          }
        }
        if (g >= 2 * kHalo) {   // output row y0 + g - 10: window rows g - 10 .. g
          float2 vac = make_float2(0.0f, 0.0f), vbd = make_float2(0.0f, 0.0f);
          float ve = 0.0f;
#pragma unroll
          for (int k = 0; k < 11; ++k) {
            const int s = (j + 1 + k) % kRing;
            vac = ffma2(w2[k], r_ac[s], vac);
            vbd = ffma2(w2[k], r_bd[s], vbd);
            ve = fmaf(w2[k].x, r_e[s], ve);
          }
          if (x < W) {
            const float v[5] = {vac.x, vbd.x, vac.y, vbd.y, ve};
            const size_t idx = plane + (size_t)(y0 + g - 2 * kHalo) * W + x;
            float d1, d2, d3;
            sm += ssim_pixel(v, C1, C2, d1, d2, d3);
            if constexpr (!kEval) {
              dm_dmu1[idx] = d1;
              dm_dsigma1_sq[idx] = d2;
              dm_dsigma12[idx] = d3;
            }
          }
        }
      }
    }
    __syncthreads();   // the buffer is restaged two chunks on
  }
  if constexpr (kEval) {
    const float vals[5] = {l1, sm, sq, pp, tt};
    eval_arrive(vals, gridDim.x * gridDim.y, H * W, ev);
  } else {
    block_partial(l1, sm, partial);
    loss_arrive(gridDim.x * gridDim.y, H * W, head, partial);
  }
}

__global__ void __launch_bounds__(kBandThreads)
loss_backward_band_kernel(int H, int W, int hb, const float* __restrict__ pred, const float* __restrict__ target,
                          const float* __restrict__ dm_dmu1, const float* __restrict__ dm_dsigma1_sq,
                          const float* __restrict__ dm_dsigma12, const float4* __restrict__ coef,
                          float* __restrict__ dL_dpred) {
  __shared__ __align__(16) float s_in[2][3 * kRing * kBandPitch];
  const size_t plane = (size_t)blockIdx.z * H * W;
  const float4 cf = coef[blockIdx.z];
  const int x0 = blockIdx.x * kBandThreads, x = x0 + (int)threadIdx.x;
  const int y0 = blockIdx.y * hb, y1 = min(H, y0 + hb);
  const int n_in = y1 - y0 + 2 * kHalo;
  const int nchunks = (n_in + kRing - 1) / kRing;
  const float* const src[3] = {dm_dmu1 + plane, dm_dsigma1_sq + plane, dm_dsigma12 + plane};
  float2 w2[11];
#pragma unroll
  for (int k = 0; k < 11; ++k) w2[k] = kSsimWin2[k];
  float2 r_ab[kRing];   // horizontal sums of the dm/dmu1 and dm/dsigma1^2 maps
  float r_c[kRing];     // and of dm/dsigma12
  band_stage<3>(s_in[0], src, H, W, x0, y0 - kHalo);
  cp_async_commit();
  for (int ci = 0; ci < nchunks; ++ci) {
    if (ci + 1 < nchunks) band_stage<3>(s_in[(ci + 1) & 1], src, H, W, x0, y0 - kHalo + (ci + 1) * kRing);
    cp_async_commit();
    // pred and target of this chunk's output rows, loaded while the chunk lands
    float pv[kRing], tv[kRing];
#pragma unroll
    for (int j = 0; j < kRing; ++j) {
      const int g = ci * kRing + j;
      const bool ok = g >= 2 * kHalo && g < n_in && x < W;
      const size_t idx = plane + (ok ? (size_t)(y0 + g - 2 * kHalo) * W + x : 0);
      pv[j] = ok ? pred[idx] : 0.0f;
      tv[j] = ok ? target[idx] : 0.0f;
    }
    cp_async_wait_prev();
    {   // the staged derivative maps times the spectrum's map gradient, as the tile layout stages them
      float* own = s_in[ci & 1];
#pragma unroll
      for (int half = 0; half < 2; ++half) {
        const int col = (int)threadIdx.x + half * kBandThreads;
        if (col < kBandCols)
#pragma unroll
          for (int j = 0; j < kRing; ++j)
#pragma unroll
            for (int im = 0; im < 3; ++im) own[band_slot(im, j, col)] *= cf.y;
      }
    }
    __syncthreads();
    const float2* s01 = reinterpret_cast<const float2*>(s_in[ci & 1]) + threadIdx.x;
    const float* s2 = s_in[ci & 1] + 2 * kRing * kBandPitch + threadIdx.x;
#pragma unroll
    for (int j = 0; j < kRing; ++j) {
      const int g = ci * kRing + j;
      if (g < n_in) {
        float2 ab = make_float2(0.0f, 0.0f);
        float c = 0.0f;
#pragma unroll
        for (int k = 0; k < 11; ++k) {
          ab = ffma2(w2[k], s01[j * kBandPitch + k], ab);
          c = fmaf(w2[k].x, s2[j * kBandPitch + k], c);
        }
        r_ab[j] = ab;
        r_c[j] = c;
        if (g >= 2 * kHalo && x < W) {
          float2 vab = make_float2(0.0f, 0.0f);
          float vc = 0.0f;
#pragma unroll
          for (int k = 0; k < 11; ++k) {
            const int s = (j + 1 + k) % kRing;
            vab = ffma2(w2[k], r_ab[s], vab);
            vc = fmaf(w2[k].x, r_c[s], vc);
          }
          const float v[3] = {vab.x, vab.y, vc};
          const size_t idx = plane + (size_t)(y0 + g - 2 * kHalo) * W + x;
          dL_dpred[idx] = loss_pixel_grad(v, pv[j], tv[j], cf.x);
        }
      }
    }
    __syncthreads();
  }
}

// Block layout of the loss for R spectra of H x W (the scratch layout and
// the launch both follow it).
struct LossGeom {
  bool band;
  int gx, gy, hb;
};
static LossGeom loss_geom(size_t R, size_t H, size_t W) {
  LossGeom g;
  g.band = R >= (size_t)kBandMinPlanes;
  if (g.band) {
    g.gx = (int)((W + kBandThreads - 1) / kBandThreads);
    const size_t per_band = R * (size_t)g.gx;
    size_t nb = (kBandTargetBlocks + per_band - 1) / per_band;
    const size_t max_bands = (H + 7) / 8;   // bands of at least 8 rows
    nb = nb < 1 ? 1 : (nb > max_bands ? max_bands : nb);
    g.hb = (int)((H + nb - 1) / nb);
    g.gy = (int)((H + g.hb - 1) / g.hb);
  } else {
    g.gx = (int)((W + kSW - 1) / kSW);
    g.gy = (int)((H + kSH - 1) / kSH);
    g.hb = kSH;
  }
  return g;
}

LossLayout loss_layout(size_t R, size_t H, size_t W, size_t hidden) {
  auto a = [](size_t x) { return (x + 63) / 64 * 64; };
  const LossGeom g = loss_geom(R, H, W);
  LossLayout L;
  const size_t n = R * H * W;
  L.nblk = (size_t)g.gx * g.gy;
  L.dmu1 = 0;
  L.ds11 = a(n);
  L.ds12 = L.ds11 + a(n);
  L.partial = L.ds12 + a(n);
  L.pre = L.partial + a(2 * R * L.nblk);
  L.coef = L.pre + a(R * hidden);
  L.share = L.coef + a(4 * R);
  L.psync = L.share + a(R * (5 * hidden + 1));
  L.sync = L.psync + a(R);
  L.total = L.sync + 64;
  return L;
}

cudaError_t launch_splat_loss(int R, int H, int W, int hidden, float lambda1, float alpha, float C1, float C2,
                              const float* pred, const float* target, const float* rx, const float* conf_params,
                              float* scratch, float* loss_out, float* terms, float* dL_dpred, float* dconf,
                              cudaStream_t stream) {
  const LossGeom G = loss_geom(R, H, W);
  const LossLayout L = loss_layout(R, H, W, hidden);
  float2* partial = reinterpret_cast<float2*>(scratch + L.partial);
  float4* coef = reinterpret_cast<float4*>(scratch + L.coef);
  LossHead head;
  head.R = R;
  head.hidden = hidden;
  head.lambda1 = lambda1;
  head.alpha = alpha;
  head.rx = rx;
  head.cp = conf_params;
  head.pre = scratch + L.pre;
  head.coef = coef;
  head.terms = terms;
  head.loss_out = loss_out;
  head.dconf = dconf;
  head.share = scratch + L.share;
  head.psync = reinterpret_cast<unsigned*>(scratch + L.psync);
  head.sync = reinterpret_cast<unsigned*>(scratch + L.sync);
  const dim3 grid((unsigned)G.gx, (unsigned)G.gy, (unsigned)R);
  const EvalOut ev{};
  if (G.band) {
    loss_forward_band_kernel<false><<<grid, kBandThreads, 0, stream>>>(
        H, W, G.hb, C1, C2, pred, target, scratch + L.dmu1, scratch + L.ds11, scratch + L.ds12, partial, head, ev);
  } else {
    loss_forward_kernel<false><<<grid, 256, 0, stream>>>(H, W, C1, C2, pred, target, scratch + L.dmu1,
                                                         scratch + L.ds11, scratch + L.ds12, partial, head, ev);
  }
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return e;
  if (G.band) {
    loss_backward_band_kernel<<<grid, kBandThreads, 0, stream>>>(H, W, G.hb, pred, target, scratch + L.dmu1,
                                                                 scratch + L.ds11, scratch + L.ds12, coef, dL_dpred);
  } else {
    loss_backward_kernel<<<grid, 256, 0, stream>>>(H, W, pred, target, scratch + L.dmu1, scratch + L.ds11,
                                                   scratch + L.ds12, coef, dL_dpred);
  }
  return cudaGetLastError();
}

size_t eval_scratch_floats(size_t R, size_t H, size_t W) {
  const LossGeom g = loss_geom(R, H, W);
  return (R * (size_t)g.gx * g.gy * kEvalSums + 63) / 64 * 64 + (R + 63) / 64 * 64;
}

cudaError_t launch_eval_metrics(int R, int H, int W, int hidden, float lambda1, float C1, float C2, const float* pred,
                                const float* target, const float* rx, const float* conf_params, float* scratch,
                                float* metrics, cudaStream_t stream) {
  const LossGeom G = loss_geom(R, H, W);
  const size_t np = ((size_t)R * G.gx * G.gy * kEvalSums + 63) / 64 * 64;
  EvalOut ev;
  ev.partial = scratch;
  ev.psync = reinterpret_cast<unsigned*>(scratch + np);
  ev.rx = rx;
  ev.cp = conf_params;
  ev.hidden = hidden;
  ev.lambda1 = lambda1;
  ev.metrics = metrics;
  const LossHead head{};
  const dim3 grid((unsigned)G.gx, (unsigned)G.gy, (unsigned)R);
  if (G.band)
    loss_forward_band_kernel<true><<<grid, kBandThreads, 0, stream>>>(H, W, G.hb, C1, C2, pred, target, nullptr,
                                                                      nullptr, nullptr, nullptr, head, ev);
  else
    loss_forward_kernel<true><<<grid, 256, 0, stream>>>(H, W, C1, C2, pred, target, nullptr, nullptr, nullptr, nullptr,
                                                        head, ev);
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
