// Adam over the per-Gaussian parameters, fused with the adjoints of their
// activations.
//
// The reference trains the Gaussians with torch.optim.Adam (eps 1e-15,
// gaussian.py:197) on the raw parameters, whose activations (gaussian.py:33-38,
// :82-96) are applied before every render; the rasterizer backward returns
// gradients with respect to the activated values.  Here one pass per
// Gaussian turns those into raw-parameter gradients and applies Adam:
//   centre        identity; NaN gradients zeroed (train.py:443-445); clamped to
//                 the scene box after the step (train.py:556-562)
//   log-scale     d/dx exp(x) = exp(x)
//   quaternion    F.normalize: d = (g - q^ (q^.g)) / max(|q|, 1e-12)
//   opacity logit d/dx sigmoid(x) = s (1 - s)
//   emission MLP  identity (elementwise kernel, float4 vectorised)
//   global block  identity, own learning rate (the confidence MLP,
//                 gaussian.py:186-195, whose torch Adam group it replaces)
// Adam follows torch's update: m = b1 m + (1-b1) g, v = b2 v + (1-b2) g^2,
// p -= (lr / bc1) * m / (sqrt(v) / sqrt(bc2) + eps), bc_i = 1 - b_i^t, with the
// step count t and the learning rates read from device memory so the whole
// update can be captured in a CUDA graph.
//
// Flat layout of parameters, gradients and both moments (floats), each
// segment starting on a 256-byte boundary (gaussian_layout):
//   [centre 3P | log_scale 3P | quaternion 4P | opacity_logit P | mlp 194P | conf]
// With activation outputs given, the per-Gaussian kernel also writes the
// activated values of the updated parameters (exp(log_scale),
// normalize(quaternion), sigmoid(logit)) -- the rasterizer inputs of the next
// step -- so no separate activation pass runs per step.
#include "common.cuh"
#include "kernels.cuh"

namespace gsparc {

struct AdamHyper {
  float lr, step_size, inv_sqrt_bc2, beta1, beta2, eps;
};

__device__ __forceinline__ AdamHyper adam_hyper(const float* lr6, int group, const float* step, float beta1,
                                                float beta2, float eps) {
  const float t = *step;
  AdamHyper h;
  h.lr = lr6[group];
  const float bc1 = 1.0f - powf(beta1, t);
  const float bc2 = 1.0f - powf(beta2, t);
  h.step_size = h.lr / bc1;
  h.inv_sqrt_bc2 = 1.0f / sqrtf(bc2);
  h.beta1 = beta1;
  h.beta2 = beta2;
  h.eps = eps;
  return h;
}

__device__ __forceinline__ float adam_update(float p, float g, float& m, float& v, const AdamHyper& h) {
  m = h.beta1 * m + (1.0f - h.beta1) * g;
  v = h.beta2 * v + (1.0f - h.beta2) * g * g;
  const float denom = sqrtf(v) * h.inv_sqrt_bc2 + h.eps;
  return p - h.step_size * (m / denom);
}

// F.normalize(q, dim=1): q / max(|q|, 1e-12)
__device__ __forceinline__ void store_normalized(float* dst, const float q[4]) {
  const float nrm = fmaxf(sqrtf(q[0] * q[0] + q[1] * q[1] + q[2] * q[2] + q[3] * q[3]), 1e-12f);
#pragma unroll
  for (int k = 0; k < 4; ++k) dst[k] = q[k] / nrm;
}

__global__ void adam_count_kernel(float* step) { *step += 1.0f; }

__global__ void __launch_bounds__(256)
gaussian_adam_kernel(int P, GaussianLayout L, float* __restrict__ params, const float* __restrict__ grads,
                     float* __restrict__ m, float* __restrict__ v, const float* __restrict__ step,
                     const float* __restrict__ lr6, float beta1, float beta2, float eps,
                     const float* __restrict__ lo3, const float* __restrict__ hi3, float* __restrict__ act_s,
                     float* __restrict__ act_q, float* __restrict__ act_o) {
  const int g = blockIdx.x * blockDim.x + threadIdx.x;
  if (g >= P) return;
  const size_t oC = L.centre, oS = L.scale, oQ = L.quat, oO = L.opacity;
  // centre: NaN-zeroed gradient, Adam, clamp
  {
    const AdamHyper h = adam_hyper(lr6, 0, step, beta1, beta2, eps);
#pragma unroll
    for (int k = 0; k < 3; ++k) {
      const size_t i = oC + 3 * (size_t)g + k;
      float gr = grads[i];
      if (isnan(gr)) gr = 0.0f;
      float mi = m[i], vi = v[i];
      float p = adam_update(params[i], gr, mi, vi, h);
      p = fminf(fmaxf(p, lo3[k]), hi3[k]);
      params[i] = p;
      m[i] = mi;
      v[i] = vi;
    }
  }
  // log-scale: d exp(x)/dx = exp(x)
  {
    const AdamHyper h = adam_hyper(lr6, 1, step, beta1, beta2, eps);
#pragma unroll
    for (int k = 0; k < 3; ++k) {
      const size_t i = oS + 3 * (size_t)g + k;
      const float x = params[i];
      const float gr = grads[i] * expf(x);
      float mi = m[i], vi = v[i];
      const float xn = adam_update(x, gr, mi, vi, h);
      params[i] = xn;
      m[i] = mi;
      v[i] = vi;
      if (act_s) act_s[3 * (size_t)g + k] = expf(xn);
    }
  }
  // quaternion through F.normalize (eps 1e-12)
  {
    const AdamHyper h = adam_hyper(lr6, 2, step, beta1, beta2, eps);
    float q[4], gq[4];
#pragma unroll
    for (int k = 0; k < 4; ++k) {
      q[k] = params[oQ + 4 * (size_t)g + k];
      gq[k] = grads[oQ + 4 * (size_t)g + k];
    }
    const float nrm = fmaxf(sqrtf(q[0] * q[0] + q[1] * q[1] + q[2] * q[2] + q[3] * q[3]), 1e-12f);
    const float inv = 1.0f / nrm;
    const float dot = (q[0] * gq[0] + q[1] * gq[1] + q[2] * gq[2] + q[3] * gq[3]) * inv;
#pragma unroll
    for (int k = 0; k < 4; ++k) {
      const size_t i = oQ + 4 * (size_t)g + k;
      const float gr = (gq[k] - q[k] * inv * dot) * inv;
      float mi = m[i], vi = v[i];
      q[k] = adam_update(q[k], gr, mi, vi, h);
      params[i] = q[k];
      m[i] = mi;
      v[i] = vi;
    }
    if (act_q) store_normalized(act_q + 4 * (size_t)g, q);
  }
  // opacity logit: d sigmoid(x)/dx = s (1 - s)
  {
    const AdamHyper h = adam_hyper(lr6, 3, step, beta1, beta2, eps);
    const size_t i = oO + g;
    const float x = params[i];
    const float s = 1.0f / (1.0f + expf(-x));
    const float gr = grads[i] * s * (1.0f - s);
    float mi = m[i], vi = v[i];
    const float xn = adam_update(x, gr, mi, vi, h);
    params[i] = xn;
    m[i] = mi;
    v[i] = vi;
    if (act_o) act_o[g] = 1.0f / (1.0f + expf(-xn));
  }
}

// Activations of the raw per-Gaussian parameters (gaussian.py:33-38, :82-96).
__global__ void __launch_bounds__(256)
gaussian_activate_kernel(int P, GaussianLayout L, const float* __restrict__ params, float* __restrict__ act_s,
                         float* __restrict__ act_q, float* __restrict__ act_o) {
  const int g = blockIdx.x * blockDim.x + threadIdx.x;
  if (g >= P) return;
#pragma unroll
  for (int k = 0; k < 3; ++k) act_s[3 * (size_t)g + k] = expf(params[L.scale + 3 * (size_t)g + k]);
  float q[4];
#pragma unroll
  for (int k = 0; k < 4; ++k) q[k] = params[L.quat + 4 * (size_t)g + k];
  store_normalized(act_q + 4 * (size_t)g, q);
  act_o[g] = 1.0f / (1.0f + expf(-params[L.opacity + g]));
}

// Emission-MLP weights and the global block: identity activation, float4
// vectorised.  Indices below n_mlp use learning rate 4, the rest rate 5; both
// segments start on a 256-byte boundary, so no float4 straddles them, and the
// padding between them holds zeros that Adam leaves at zero.
__global__ void __launch_bounds__(256)
mlp_adam_kernel(size_t n, size_t n_mlp, float* __restrict__ params, const float* __restrict__ grads,
                float* __restrict__ m, float* __restrict__ v, const float* __restrict__ step,
                const float* __restrict__ lr6, float beta1, float beta2, float eps) {
  const AdamHyper h4 = adam_hyper(lr6, 4, step, beta1, beta2, eps);
  const AdamHyper h5 = (n > n_mlp) ? adam_hyper(lr6, 5, step, beta1, beta2, eps) : h4;
  const size_t n4 = n / 4;
  const size_t stride = (size_t)gridDim.x * blockDim.x;
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n4; i += stride) {
    const AdamHyper& h = (4 * i < n_mlp) ? h4 : h5;
    float4 p = reinterpret_cast<float4*>(params)[i];
    const float4 g = reinterpret_cast<const float4*>(grads)[i];
    float4 mm = reinterpret_cast<float4*>(m)[i];
    float4 vv = reinterpret_cast<float4*>(v)[i];
    p.x = adam_update(p.x, g.x, mm.x, vv.x, h);
    p.y = adam_update(p.y, g.y, mm.y, vv.y, h);
    p.z = adam_update(p.z, g.z, mm.z, vv.z, h);
    p.w = adam_update(p.w, g.w, mm.w, vv.w, h);
    reinterpret_cast<float4*>(params)[i] = p;
    reinterpret_cast<float4*>(m)[i] = mm;
    reinterpret_cast<float4*>(v)[i] = vv;
  }
  for (size_t i = n4 * 4 + blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += stride) {
    const AdamHyper& h = (i < n_mlp) ? h4 : h5;
    float mi = m[i], vi = v[i];
    params[i] = adam_update(params[i], grads[i], mi, vi, h);
    m[i] = mi;
    v[i] = vi;
  }
}

cudaError_t launch_gaussian_adam(int P, int conf_floats, float* params, const float* grads, float* m, float* v,
                                 float* step, const float* lr6, float beta1, float beta2, float eps,
                                 const float* lo3, const float* hi3, float* act_scales, float* act_rots,
                                 float* act_opac, cudaStream_t stream) {
  adam_count_kernel<<<1, 1, 0, stream>>>(step);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return e;
  const GaussianLayout L = gaussian_layout((size_t)P, (size_t)conf_floats);
  if (P > 0) {
    gaussian_adam_kernel<<<(P + 255) / 256, 256, 0, stream>>>(P, L, params, grads, m, v, step, lr6, beta1, beta2,
                                                              eps, lo3, hi3, act_scales, act_rots, act_opac);
    e = cudaGetLastError();
    if (e != cudaSuccess) return e;
  }
  const size_t off = L.mlp;
  const size_t n_mlp = (size_t)kMlpFloats * P;
  const size_t n = conf_floats > 0 ? (L.conf - L.mlp) + (size_t)conf_floats : n_mlp;
  if (n == 0) return cudaSuccess;
  int blocks = (int)((n / 4 + 255) / 256);
  if (blocks > 148 * 8) blocks = 148 * 8;
  if (blocks < 1) blocks = 1;
  mlp_adam_kernel<<<blocks, 256, 0, stream>>>(n, n_mlp, params + off, grads + off, m + off, v + off, step, lr6,
                                              beta1, beta2, eps);
  return cudaGetLastError();
}

cudaError_t launch_gaussian_activate(int P, const float* params, float* act_scales, float* act_rots,
                                     float* act_opac, cudaStream_t stream) {
  if (P == 0) return cudaSuccess;
  const GaussianLayout L = gaussian_layout((size_t)P);
  gaussian_activate_kernel<<<(P + 255) / 256, 256, 0, stream>>>(P, L, params, act_scales, act_rots, act_opac);
  return cudaGetLastError();
}

}  // namespace gsparc
