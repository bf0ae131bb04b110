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
// update can be captured in a CUDA graph.  All groups are updated by one
// launch (train_adam_kernel).
//
// Flat layout of parameters, gradients and both moments (floats), each
// segment starting on a 256-byte boundary (gaussian_layout):
//   [centre 3P | log_scale 3P | quaternion 4P | opacity_logit P | mlp | conf]
// (mlp: the per-Gaussian MLPs, 194 P floats, or the shared MLP's parameters)
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

__device__ __forceinline__ AdamHyper adam_hyper(const float* lr6, int group, float t, float beta1, float beta2,
                                                float eps) {
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

__device__ __forceinline__ void gaussian_adam_body(int g, GaussianLayout L, float* __restrict__ params,
                                                   const float* __restrict__ grads, float* __restrict__ m,
                                                   float* __restrict__ v, float step, const float* __restrict__ lr6,
                                                   float beta1, float beta2, float eps, const float* __restrict__ lo3,
                                                   const float* __restrict__ hi3, float* __restrict__ act_s,
                                                   float* __restrict__ act_q, float* __restrict__ act_o) {
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
__device__ __forceinline__ void mlp_adam_body(int block, int nblocks, size_t n, size_t n_mlp,
                                              float* __restrict__ params, const float* __restrict__ grads,
                                              float* __restrict__ m, float* __restrict__ v, float step,
                                              const float* __restrict__ lr6, float beta1, float beta2, float eps) {
  const AdamHyper h4 = adam_hyper(lr6, 4, step, beta1, beta2, eps);
  const AdamHyper h5 = (n > n_mlp) ? adam_hyper(lr6, 5, step, beta1, beta2, eps) : h4;
  const size_t n4 = n / 4;
  const size_t stride = (size_t)nblocks * blockDim.x;
  for (size_t i = block * (size_t)blockDim.x + threadIdx.x; i < n4; i += stride) {
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
  for (size_t i = n4 * 4 + block * (size_t)blockDim.x + threadIdx.x; i < n; i += stride) {
    const AdamHyper& h = (i < n_mlp) ? h4 : h5;
    float mi = m[i], vi = v[i];
    params[i] = adam_update(params[i], grads[i], mi, vi, h);
    m[i] = mi;
    v[i] = vi;
  }
}

// One launch for the whole state: CTAs [0, nb_g) update the per-Gaussian
// groups, the rest stream the MLP / global segments, so the short latency-bound
// per-Gaussian work overlaps the bandwidth-bound MLP update.  Every CTA uses
// step t = stored count + 1; the last CTA to finish (arrival counter in the
// word after the count) stores t and clears the counter.
__global__ void __launch_bounds__(256)
train_adam_kernel(int P, GaussianLayout L, int nb_g, size_t n, size_t n_mlp, float* __restrict__ params,
                  const float* __restrict__ grads, float* __restrict__ m, float* __restrict__ v,
                  float* __restrict__ step, const float* __restrict__ lr6, float beta1, float beta2, float eps,
                  const float* __restrict__ lo3, const float* __restrict__ hi3, float* __restrict__ act_s,
                  float* __restrict__ act_q, float* __restrict__ act_o) {
  const float t = __ldcg(step) + 1.0f;
  if ((int)blockIdx.x < nb_g) {
    const int g = blockIdx.x * blockDim.x + threadIdx.x;
    if (g < P) gaussian_adam_body(g, L, params, grads, m, v, t, lr6, beta1, beta2, eps, lo3, hi3, act_s, act_q, act_o);
  } else {
    mlp_adam_body(blockIdx.x - nb_g, gridDim.x - nb_g, n, n_mlp, params + L.mlp, grads + L.mlp, m + L.mlp,
                  v + L.mlp, t, lr6, beta1, beta2, eps);
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    unsigned* arrived = reinterpret_cast<unsigned*>(step + 1);
    __threadfence();
    if (atomicAdd(arrived, 1u) == gridDim.x - 1) {
      step[0] = t;
      *arrived = 0u;
    }
  }
}

cudaError_t launch_gaussian_adam(int P, long long mlp_floats, int conf_floats, float* params, const float* grads,
                                 float* m, float* v,
                                 float* step, const float* lr6, float beta1, float beta2, float eps,
                                 const float* lo3, const float* hi3, float* act_scales, float* act_rots,
                                 float* act_opac, cudaStream_t stream) {
  const GaussianLayout L = gaussian_layout((size_t)P, (size_t)mlp_floats, (size_t)conf_floats);
  const size_t n_mlp = (size_t)mlp_floats;
  const size_t n = conf_floats > 0 ? (L.conf - L.mlp) + (size_t)conf_floats : n_mlp;
  const int nb_g = (P + 255) / 256;
  int nb_m = (int)((n / 4 + 255) / 256);
  if (nb_m > device_sm_count() * 8) nb_m = device_sm_count() * 8;
  if (nb_m < 1) nb_m = 1;
  train_adam_kernel<<<nb_g + nb_m, 256, 0, stream>>>(P, L, nb_g, n, n_mlp, params, grads, m, v, step, lr6, beta1,
                                                     beta2, eps, lo3, hi3, act_scales, act_rots, act_opac);
  return cudaGetLastError();
}

cudaError_t launch_gaussian_activate(int P, const float* params, float* act_scales, float* act_rots,
                                     float* act_opac, cudaStream_t stream) {
  if (P == 0) return cudaSuccess;
  const GaussianLayout L = gaussian_layout((size_t)P, 0);   // the segments before the MLP's
  gaussian_activate_kernel<<<(P + 255) / 256, 256, 0, stream>>>(P, L, params, act_scales, act_rots, act_opac);
  return cudaGetLastError();
}

}  // namespace gsparc
