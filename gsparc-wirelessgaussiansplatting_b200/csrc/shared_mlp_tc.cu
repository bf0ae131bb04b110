// Shared emission MLP in BF16 on the 5th-generation tensor cores (tcgen05).
//
// Same network as shared_mlp.cu (features, hidden layers of width 128,
// sigmoid of one output, or of 64 outputs whose layer is one more MMA) with
// BF16 operands and FP32 accumulation in tensor memory.  Two fused persistent kernels over tiles of 128 (receiver, Gaussian)
// rows, one row per thread of a 128-thread warpgroup:
//
//   forward:  four warpgroups per CTA, each with its own tile in flight and
//             its own 128 TMEM columns; per layer the group's leader issues
//             the MMA, the group runs the +bias/activation epilogue.  The
//             weights are staged in shared memory once per CTA; only the BF16
//             pre-activations (for the adjoint) and the signal go to HBM.
//   backward: two compute warpgroups, each with its own tile, and one MMA
//             warp that issues every MMA of the CTA (so all accumulation into
//             the shared weight-gradient columns is in issue order).  Per tile
//             and hidden layer l (last first):
//               dW_l | db_l += dZ_l^T [A_{l-1} | 1]   (M = 128 outputs, K = the
//                              128 rows; accumulated in TMEM over all tiles)
//               dA_{l-1}     = dZ_l W_l              (M = 128 rows; one
//                              shared scratch accumulator)
//             A_{l-1} = act(Z_{l-1}) and act'(Z_{l-1}) come from one pass over
//             the stored pre-activations (one CDF evaluation per element;
//             act' is held in registers as FP16 until dA arrives); the output
//             layer's gradient is reduced on the CUDA cores.  At the end the
//             CTA adds its TMEM accumulators to the global gradient.
//
// Operands use the no-swizzle core-matrix layouts of tcgen05.cuh.  A buffer
// written row-per-thread in the K-major layout of a [rows x cols] matrix is
// also the MN-major layout of its transpose (same core matrices, LBO and SBO
// exchanged), which is how dZ and A feed the weight-gradient MMA without a
// transposed copy.  Every wait is bounded: on give-up the error word gets
// kErrMlpWait and the CTA stops.
#include <cuda_bf16.h>
#include <cuda_fp16.h>

#include "common.cuh"
#include "kernels.cuh"
#include "tcgen05.cuh"

namespace gsparc {

namespace {

constexpr int kH = 128;        // hidden width of the BF16 path
constexpr int kFin = 32;       // features
constexpr int kRows = 128;     // rows per tile (= MMA M)
constexpr int kFwdGroups = 4;  // forward: warpgroups (tiles in flight) per CTA
constexpr int kBwdGroups = 2;  // backward: compute warpgroups per CTA (+ one MMA warp)
constexpr int kBwdThreads = kBwdGroups * 128 + 32;
constexpr uint32_t kLbo = 128; // core matrices along K are adjacent
constexpr uint32_t kSboX = (kFin / 8) * 128u;         // [rows x 32] K-major
constexpr uint32_t kSboH = (kH / 8) * 128u;           // [rows x 128] K-major
constexpr uint32_t kSboA = ((kH + 16) / 8) * 128u;    // [rows x 144] K-major (activations | ones)
constexpr uint32_t kPolls = 1u << 24;
constexpr float kPiF = 3.14159265358979323846f;

// GELU of two pre-activations at once (FP32x2) for the forward, where no
// density term is needed: Phi from Abramowitz & Stegun 7.1.28,
//   erf(x) = 1 - (1 + a1 x + a2 x^2 + ... + a6 x^6)^-16,  x >= 0, |error| <= 3e-7,
// one approximate reciprocal per element and four squarings, no exponential.
__device__ __forceinline__ float rcp_approx(float x) {
  float r;
  asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"(x));
  return r;
}
__device__ __forceinline__ float2 gelu2(float2 z) {
  const float2 x = make_float2(fabsf(z.x) * 0.70710678118654752f, fabsf(z.y) * 0.70710678118654752f);
  float2 p = ffma2(x, make_float2(4.30638e-5f, 4.30638e-5f), make_float2(2.765672e-4f, 2.765672e-4f));
  p = ffma2(p, x, make_float2(1.520143e-4f, 1.520143e-4f));
  p = ffma2(p, x, make_float2(9.2705272e-3f, 9.2705272e-3f));
  p = ffma2(p, x, make_float2(4.22820123e-2f, 4.22820123e-2f));
  p = ffma2(p, x, make_float2(7.05230784e-2f, 7.05230784e-2f));
  p = ffma2(p, x, make_float2(1.0f, 1.0f));
  float2 r = make_float2(rcp_approx(p.x), rcp_approx(p.y));
  r = fmul2(r, r);
  r = fmul2(r, r);
  r = fmul2(r, r);
  r = fmul2(r, r);   // 1 - erf(x)
  // Phi(z) = 1 - r / 2 (z >= 0) or r / 2 (z < 0) = 1/2 + h (r - 1), h = -+1/2
  const float2 h = make_float2(copysignf(0.5f, -z.x), copysignf(0.5f, -z.y));
  const float2 ph = ffma2(h, fadd2(r, make_float2(-1.0f, -1.0f)), make_float2(0.5f, 0.5f));
  return fmul2(z, ph);
}
__device__ __forceinline__ float ex2_approx(float x) {
  float r;
  asm("ex2.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"(x));
  return r;
}
// Activation and derivative of two elements from one evaluation (FP32x2), for
// the adjoint.  GELU's normal CDF Phi(z) = (1 + erf(z / sqrt 2)) / 2 by
// Abramowitz & Stegun 7.1.26 (Hastings' rational approximation, |error of
// erf| <= 1.5e-7, three orders below the BF16 rounding the results go through):
//   erf(x) = 1 - t (a1 + t (a2 + t (a3 + t (a4 + t a5)))) exp(-x^2),
//   t = 1 / (1 + p x), x >= 0, odd extension for x < 0,
// whose exponential is also the density term of GELU':
//   a = z Phi(z),  d = Phi(z) + z phi(z),  phi(z) = exp(-z^2 / 2) / sqrt(2 pi).
__device__ __forceinline__ void act_and_grad2(int act, float2 z, float2& a, float2& d) {
  if (act == 1) {
    a = make_float2(fmaxf(z.x, 0.0f), fmaxf(z.y, 0.0f));
    d = make_float2(z.x > 0.0f ? 1.0f : 0.0f, z.y > 0.0f ? 1.0f : 0.0f);
    return;
  }
  const float2 x = make_float2(fabsf(z.x) * 0.70710678118654752f, fabsf(z.y) * 0.70710678118654752f);
  const float2 arg = fmul2(fmul2(z, z), make_float2(-0.72134752044448170f, -0.72134752044448170f));  // -z^2/2 log2 e
  const float2 ez = make_float2(ex2_approx(arg.x), ex2_approx(arg.y));
  const float2 den = ffma2(make_float2(0.3275911f, 0.3275911f), x, make_float2(1.0f, 1.0f));
  const float2 tt = make_float2(rcp_approx(den.x), rcp_approx(den.y));
  // -(a1 + t (a2 + t (a3 + t (a4 + t a5)))): negated so erf = 1 + t p' e^{-x^2} is one FMA
  float2 p = ffma2(tt, make_float2(-1.061405429f, -1.061405429f), make_float2(1.453152027f, 1.453152027f));
  p = ffma2(tt, p, make_float2(-1.421413741f, -1.421413741f));
  p = ffma2(tt, p, make_float2(0.284496736f, 0.284496736f));
  p = ffma2(tt, p, make_float2(-0.254829592f, -0.254829592f));
  const float2 e = ffma2(fmul2(tt, p), ez, make_float2(1.0f, 1.0f));   // erf(|z| / sqrt 2)
  const float2 h = make_float2(copysignf(0.5f, z.x), copysignf(0.5f, z.y));
  const float2 ph = ffma2(h, e, make_float2(0.5f, 0.5f));
  a = fmul2(z, ph);
  d = ffma2(fmul2(z, make_float2(0.39894228040143268f, 0.39894228040143268f)), ez, ph);
}

__device__ __forceinline__ uint32_t pack2(float a, float b) {
  const __nv_bfloat162 h = __floats2bfloat162_rn(a, b);
  return *reinterpret_cast<const uint32_t*>(&h);
}
__device__ __forceinline__ uint4 pack8(const float* v) {
  return make_uint4(pack2(v[0], v[1]), pack2(v[2], v[3]), pack2(v[4], v[5]), pack2(v[6], v[7]));
}
__device__ __forceinline__ void unpack8(uint4 u, float* v) {
  const uint32_t w[4] = {u.x, u.y, u.z, u.w};
#pragma unroll
  for (int i = 0; i < 4; ++i) {
    const __nv_bfloat162 h = *reinterpret_cast<const __nv_bfloat162*>(&w[i]);
    const float2 f = __bfloat1622float2(h);
    v[2 * i] = f.x;
    v[2 * i + 1] = f.y;
  }
}

// (receiver, Gaussian) of row row0 + t, with one 64-bit division per tile.
__device__ __forceinline__ void row_pair(size_t row0, int t, int P, int& r, int& g) {
  const size_t rr = row0 / (size_t)P;
  int gg = (int)(row0 - rr * (size_t)P) + t;
  int ri = (int)rr;
  while (gg >= P) {   // at most 128 / P + 1 steps
    gg -= P;
    ++ri;
  }
  r = ri;
  g = gg;
}

// Stored pre-activations, tile-transposed so that a warp's 16-byte accesses to
// one 8-column chunk of its 32 rows cover 512 contiguous bytes: layer l, row
// tile, chunk k (columns 8k..8k+7), row t of the tile at element
//   l * zrows * 128 + tile * 128 * 128 + k * 128 * 8 + t * 8,
// zrows = the row count rounded up to whole tiles (the allocation's size).
__device__ __forceinline__ size_t z_row_base(size_t zrows, int l, size_t tile, int t) {
  return (size_t)l * zrows * kH + tile * (size_t)kRows * kH + (size_t)t * 8;
}
constexpr int kZChunk = kRows * 8;   // elements between a row's consecutive 8-column chunks

// Features of one pair (as mlp_features_kernel), zero for culled pairs.  The
// positional encoding's higher octaves come from the first by the double-angle
// identities: the arguments are exact power-of-two multiples of the first, so
// only a few FP32 ulps separate them from direct sin/cos, far below BF16.
__device__ __forceinline__ void pair_features(const float* __restrict__ means3D, const float* __restrict__ rx_pos,
                                              int g, int r, bool vis, float* x) {
  if (!vis) {
#pragma unroll
    for (int i = 0; i < kFin; ++i) x[i] = 0.0f;
    return;
  }
  const float m[3] = {means3D[3 * g], means3D[3 * g + 1], means3D[3 * g + 2]};
  const float v[3] = {m[0] - rx_pos[3 * r], m[1] - rx_pos[3 * r + 1], m[2] - rx_pos[3 * r + 2]};
  const float d2 = v[0] * v[0] + v[1] * v[1] + v[2] * v[2];
  const float d = sqrtf(d2);
  x[0] = m[0]; x[1] = m[1]; x[2] = m[2];
#pragma unroll
  for (int j = 0; j < 3; ++j) {
    float s, c;
    sincosf(kPiF * m[j], &s, &c);
#pragma unroll
    for (int k = 0; k < 4; ++k) {
      x[3 + 6 * k + 2 * j] = s;
      x[4 + 6 * k + 2 * j] = c;
      const float s2 = 2.0f * s * c, c2 = fmaf(c, c, -s * s);
      s = s2;
      c = c2;
    }
  }
  x[27] = v[0] / d; x[28] = v[1] / d; x[29] = v[2] / d;
  x[30] = 1.0f / d2;
  x[31] = 0.0f;
}

// Sum 32 per-lane values over the warp: returns, in lane j, the sum of value j.
__device__ __forceinline__ float warp_transpose_sum32(float (&v)[32], int lane) {
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

// Warpgroup-local ordering of generic shared-memory writes and TMEM reads
// before the group's leader issues MMAs that read / overwrite them.
__device__ __forceinline__ void group_publish(uint32_t bar_id) {
  tc::fence_async_smem();
  tc::fence_before_sync();
  tc::named_sync(bar_id, 128);
  tc::fence_after_sync();
}

}  // namespace

// ---- forward ------------------------------------------------------------------
// dynamic smem: W_l K-major [128 x in_l] bf16 (the B operand: n = output,
// k = input), then per warpgroup an activation tile H [128 x 128] K-major bf16
// whose first 8 KB also hold the feature tile X [128 x 32]; biases and the
// output row in fp32.
template <int kLayers, int act, int kOut>
__global__ void __launch_bounds__(128 * kFwdGroups, 1)
mlp_bf16_forward_kernel(int P, size_t rows, const float* __restrict__ means3D,
                        const float* __restrict__ rx_pos, const float* __restrict__ params,
                        const int* __restrict__ radii, __nv_bfloat16* __restrict__ zb, float* __restrict__ S,
                        float2* __restrict__ signal, ImageHeader* __restrict__ hdr, uint32_t polls) {
  extern __shared__ __align__(1024) unsigned char smem[];
  __shared__ __align__(8) uint64_t mbar[kFwdGroups];
  __shared__ uint32_t tbase;
  const int tid = threadIdx.x, t = tid & 127, grp = tid >> 7, warp = tid >> 5;
  unsigned char* Ws[kLayers];
  size_t off = 0;
  for (int l = 0; l < kLayers; ++l) {
    Ws[l] = smem + off;
    off += (size_t)kH * (l == 0 ? kFin : kH) * 2;
  }
  unsigned char* Hs = smem + off + (size_t)grp * kRows * kH * 2;
  off += (size_t)kFwdGroups * kRows * kH * 2;
  float* bias = reinterpret_cast<float*>(smem + off);   // [kLayers][128], then w_out[128] + b_out (one
  float* wout = bias + kLayers * kH;                    // output) or b_out[kOut] (kOut outputs)
  off += (size_t)(kLayers * kH + kH + 4) * sizeof(float);
  // kOut > 1: the output layer as an MMA, W_out K-major [kOut x 128] bf16
  unsigned char* Wo = smem + (off + 127) / 128 * 128;

  size_t poff = 0;
  for (int l = 0; l < kLayers; ++l) {
    const int in = l == 0 ? kFin : kH;
    const float* W = params + poff;
    const uint32_t sbo = (uint32_t)(in / 8) * 128u;
    for (int c = tid; c < kH * (in / 8); c += blockDim.x) {
      const int n = c / (in / 8), kc = c % (in / 8);
      float v[8];
#pragma unroll
      for (int i = 0; i < 8; ++i) v[i] = W[(size_t)n * in + kc * 8 + i];
      *reinterpret_cast<uint4*>(Ws[l] + tc::kmajor_off(n, kc * 8, kLbo, sbo)) = pack8(v);
    }
    poff += (size_t)kH * in;
    for (int j = tid; j < kH; j += blockDim.x) bias[l * kH + j] = params[poff + j];
    poff += kH;
  }
  float bout = 0.0f;
  if constexpr (kOut == 1) {
    for (int j = tid; j < kH; j += blockDim.x) wout[j] = params[poff + j];
    bout = params[poff + kH];
  } else {
    for (int c = tid; c < kOut * (kH / 8); c += blockDim.x) {
      const int n = c / (kH / 8), kc = c % (kH / 8);
      float v[8];
#pragma unroll
      for (int i = 0; i < 8; ++i) v[i] = params[poff + (size_t)n * kH + kc * 8 + i];
      *reinterpret_cast<uint4*>(Wo + tc::kmajor_off(n, kc * 8, kLbo, kSboH)) = pack8(v);
    }
    for (int j = tid; j < kOut; j += blockDim.x) wout[j] = params[poff + (size_t)kOut * kH + j];
  }
  if (tid == 0)
    for (int q = 0; q < kFwdGroups; ++q) tc::mbar_init(&mbar[q], 1);
  if (warp == 0) tc::tmem_alloc(&tbase, kFwdGroups * kH);
  tc::fence_async_smem();
  tc::fence_before_sync();
  __syncthreads();
  tc::fence_after_sync();
  const uint32_t tmem = tbase + (uint32_t)(grp * kH);
  const uint32_t lane_base = (uint32_t)((warp & 3) * 32) << 16;
  const uint32_t bar_id = 1u + (uint32_t)grp;
  uint32_t phase = 0;
  bool ok = true;
  const size_t ntiles = (rows + kRows - 1) / kRows;
  const size_t zrows = ntiles * kRows;   // pre-activation rows, whole tiles
  for (size_t tile = (size_t)blockIdx.x * kFwdGroups + grp; tile < ntiles; tile += (size_t)gridDim.x * kFwdGroups) {
    const size_t row0 = tile * kRows, row = row0 + t;
    const bool valid = row < rows;
    const bool vis = valid && radii[row] > 0;
    {
      int r, g;
      row_pair(row0, t, P, r, g);
      float x[kFin];
      pair_features(means3D, rx_pos, g, r, vis, x);
#pragma unroll
      for (int kc = 0; kc < kFin / 8; ++kc)
        *reinterpret_cast<uint4*>(Hs + tc::kmajor_off(t, kc * 8, kLbo, kSboX)) = pack8(x + kc * 8);
    }
    float o = bout;
    for (int l = 0; l < kLayers; ++l) {
      const int in = l == 0 ? kFin : kH;
      group_publish(bar_id);
      if (t == 0) {
        const uint32_t sbo = (uint32_t)(in / 8) * 128u;
        const uint32_t a0 = tc::smem_u32(Hs), b0 = tc::smem_u32(Ws[l]);
        const uint32_t idesc = tc::idesc_bf16(kRows, kH, false, false);
        for (int kk = 0; kk < in / 16; ++kk)
          tc::mma_bf16(tmem, tc::smem_desc(a0 + kk * 2 * kLbo, kLbo, sbo),
                       tc::smem_desc(b0 + kk * 2 * kLbo, kLbo, sbo), idesc, kk > 0 ? 1u : 0u);
        tc::commit(&mbar[grp]);
      }
      const bool got = tc::mbar_wait(&mbar[grp], phase, polls);
      phase ^= 1u;
      tc::fence_after_sync();
      if (!tc::named_all(bar_id, 128, got)) {
        ok = false;
        break;
      }
      __nv_bfloat16* z_out = zb + z_row_base(zrows, l, tile, t);
#pragma unroll 1
      for (int c0 = 0; c0 < kH; c0 += 32) {
        float v[32];
        tc::tmem_ld32(tmem + lane_base + c0, v);
        const float2* b2 = reinterpret_cast<const float2*>(bias + l * kH + c0);
#pragma unroll
        for (int q = 0; q < 4; ++q) {
          float2 z2[4];
#pragma unroll
          for (int i = 0; i < 4; ++i) z2[i] = fadd2(make_float2(v[q * 8 + 2 * i], v[q * 8 + 2 * i + 1]), b2[q * 4 + i]);
          const uint4 zp = make_uint4(pack2(z2[0].x, z2[0].y), pack2(z2[1].x, z2[1].y), pack2(z2[2].x, z2[2].y),
                                      pack2(z2[3].x, z2[3].y));
          if (valid) *reinterpret_cast<uint4*>(z_out + (size_t)((c0 + q * 8) / 8) * kZChunk) = zp;
          // the next layer (and the adjoint) see the BF16-rounded pre-activation
          float zr[8], a[8];
          unpack8(zp, zr);
          if (act == 1) {
#pragma unroll
            for (int i = 0; i < 8; ++i) a[i] = fmaxf(zr[i], 0.0f);
          } else {
#pragma unroll
            for (int i = 0; i < 4; ++i) {
              const float2 g = gelu2(make_float2(zr[2 * i], zr[2 * i + 1]));
              a[2 * i] = g.x;
              a[2 * i + 1] = g.y;
            }
          }
          if (l + 1 < kLayers || kOut > 1) {
            *reinterpret_cast<uint4*>(Hs + tc::kmajor_off(t, c0 + q * 8, kLbo, kSboH)) = pack8(a);
          } else {
#pragma unroll
            for (int i = 0; i < 8; ++i) o += wout[c0 + q * 8 + i] * a[i];
          }
        }
      }
    }
    if (!ok) break;
    if constexpr (kOut == 1) {
      if (valid) {
        const float s = 1.0f / (1.0f + expf(-o));
        S[row] = s;
        if (vis) signal[row] = make_float2(s, 0.0f);
      }
    } else {
      // output layer: [128 rows x kOut] = A_{L-1} W_out^T into the group's TMEM columns
      group_publish(bar_id);
      if (t == 0) {
        const uint32_t a0 = tc::smem_u32(Hs), b0 = tc::smem_u32(Wo);
        const uint32_t idesc = tc::idesc_bf16(kRows, kOut, false, false);
        for (int kk = 0; kk < kH / 16; ++kk)
          tc::mma_bf16(tmem, tc::smem_desc(a0 + kk * 2 * kLbo, kLbo, kSboH),
                       tc::smem_desc(b0 + kk * 2 * kLbo, kLbo, kSboH), idesc, kk > 0 ? 1u : 0u);
        tc::commit(&mbar[grp]);
      }
      const bool got = tc::mbar_wait(&mbar[grp], phase, polls);
      phase ^= 1u;
      tc::fence_after_sync();
      if (!tc::named_all(bar_id, 128, got)) {
        ok = false;
        break;
      }
#pragma unroll 1
      for (int c0 = 0; c0 < kOut; c0 += 32) {
        float v[32];
        tc::tmem_ld32(tmem + lane_base + c0, v);
#pragma unroll
        for (int i = 0; i < 32; ++i) v[i] = 1.0f / (1.0f + expf(-(v[i] + wout[c0 + i])));
        if (valid)
#pragma unroll
          for (int q = 0; q < 8; ++q)
            *reinterpret_cast<float4*>(S + row * kOut + c0 + 4 * q) =
                make_float4(v[4 * q], v[4 * q + 1], v[4 * q + 2], v[4 * q + 3]);
      }
    }
  }
  if (!ok && t == 0) {
    if (hdr) atomic_or_error(hdr, kErrMlpWait);
    // drain: the MMAs this group's leader committed last (the phase the group
    // gave up on) complete before the tensor memory is freed
    tc::mbar_wait(&mbar[grp], phase ^ 1u, kPolls);
  }
  tc::fence_before_sync();
  __syncthreads();
  if (warp == 0) tc::tmem_dealloc(tbase, kFwdGroups * kH);
}

// ---- backward -----------------------------------------------------------------
// dynamic smem: W_l as the MN-major B operand of dA = dZ W ([n = in_l] x
// [k = 128 outputs]) for every layer; per compute warpgroup dZ [128 rows x 128]
// and A [128 rows x 144] (activations, then a ones column and 15 zero columns),
// both K-major by row; the output row in fp32 (one output) or W_out as the
// MN-major B operand of dA = dO W_out ([n = 128] x [k = kOut]) (kOut outputs).
// TMEM columns: dW_l accumulators of (in_l + 16) columns each (last layer
// first; with kOut outputs the first layer's bias is summed on the CUDA cores
// and its accumulator is in_0 wide), then dW_out^T (kOut columns, lanes =
// hidden units; kOut outputs only), then one 128-column scratch accumulator
// for dA.  With kOut outputs every tile starts with an output step: dW_out^T +=
// A_{L-1}^T dO and dA_{L-1} = dO W_out on the tensor cores, dO staged as a
// K-major row tile in the dZ buffer.
template <int kLayers, int act, int kOut>
__global__ void __launch_bounds__(kBwdThreads, 1)
mlp_bf16_backward_kernel(int P, size_t rows, const float* __restrict__ means3D,
                         const float* __restrict__ rx_pos, const float* __restrict__ params,
                         const int* __restrict__ radii, const __nv_bfloat16* __restrict__ zb,
                         const float* __restrict__ S, const float* __restrict__ dL_dsignal,
                         float* __restrict__ dX0, float* __restrict__ dparams, ImageHeader* __restrict__ hdr,
                         uint32_t polls) {
  extern __shared__ __align__(1024) unsigned char smem[];
  __shared__ __align__(8) uint64_t bar_ready[kBwdGroups];
  __shared__ __align__(8) uint64_t bar_done[kBwdGroups];
  __shared__ __align__(8) uint64_t bar_free;
  __shared__ __align__(8) uint64_t bar_drain;
  __shared__ uint32_t tbase;
  __shared__ int s_fail;
  // one output: dw_out[128], db_out; kOut outputs: db_out[kOut], db_0[128]
  constexpr int kRed = kOut == 1 ? kH + 1 : kOut + kH;
  __shared__ float s_red[kRed];
  constexpr bool kMulti = kOut > 1;
  constexpr uint32_t kSboO = (uint32_t)(kOut / 8) * 128u;   // [rows x kOut] K-major / W_out MN-major
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int grp = tid >> 7;   // compute warpgroup 0..kBwdGroups-1; kBwdGroups = the MMA warp
  const int t = tid & 127;
  constexpr size_t kGroupBytes = (size_t)kRows * kH * 2 + (size_t)kRows * (kH + 16) * 2;
  unsigned char* Wb[kLayers];
  size_t off = 0;
  for (int l = 0; l < kLayers; ++l) {
    Wb[l] = smem + off;
    off += (size_t)(l == 0 ? kFin : kH) * kH * 2;
  }
  unsigned char* const groups = smem + off;
  off += kBwdGroups * kGroupBytes;
  float* wout = reinterpret_cast<float*>(smem + off);   // one output: w_out[128]
  off += (size_t)kH * sizeof(float);
  unsigned char* const Wo = smem + off;                 // kOut outputs: W_out MN-major

  // W_l [out][in] -> MN-major B operand (n = in, k = out), once per CTA
  size_t poff = 0;
  size_t woff[kLayers + 1], boff[kLayers + 1];
  for (int l = 0; l < kLayers; ++l) {
    const int in = l == 0 ? kFin : kH;
    woff[l] = poff;
    const float* W = params + poff;
    for (int c = tid; c < kH * (in / 8); c += blockDim.x) {
      const int k = c / (in / 8), nc = c % (in / 8);   // k = output row of W, nc = group of 8 inputs
      float v[8];
#pragma unroll
      for (int i = 0; i < 8; ++i) v[i] = W[(size_t)k * in + nc * 8 + i];
      *reinterpret_cast<uint4*>(Wb[l] + tc::mnmajor_off(nc * 8, k, kLbo, kSboH)) = pack8(v);
    }
    poff += (size_t)kH * in;
    boff[l] = poff;
    poff += kH;
  }
  woff[kLayers] = poff;
  boff[kLayers] = poff + (size_t)kOut * kH;
  if constexpr (kMulti) {
    for (int c = tid; c < kOut * (kH / 8); c += blockDim.x) {
      const int k = c / (kH / 8), nc = c % (kH / 8);   // k = output row of W_out, nc = group of 8 hidden units
      float v[8];
#pragma unroll
      for (int i = 0; i < 8; ++i) v[i] = params[poff + (size_t)k * kH + nc * 8 + i];
      *reinterpret_cast<uint4*>(Wo + tc::mnmajor_off(nc * 8, k, kLbo, kSboO)) = pack8(v);
    }
  } else {
    for (int j = tid; j < kH; j += blockDim.x) wout[j] = params[woff[kLayers] + j];
  }
  for (int j = tid; j < kRed; j += blockDim.x) s_red[j] = 0.0f;
  unsigned char* const dZ = groups + (size_t)(grp < kBwdGroups ? grp : 0) * kGroupBytes;
  unsigned char* const Ab = dZ + (size_t)kRows * kH * 2;
  if (grp < kBwdGroups) {   // the constant ones column (db) of the activation tile
    const uint4 one = make_uint4(pack2(1.0f, 0.0f), 0u, 0u, 0u);
    *reinterpret_cast<uint4*>(Ab + tc::kmajor_off(t, kH, kLbo, kSboA)) = one;
    *reinterpret_cast<uint4*>(Ab + tc::kmajor_off(t, kH + 8, kLbo, kSboA)) = make_uint4(0u, 0u, 0u, 0u);
  }
  if (tid == 0) {
    for (int q = 0; q < kBwdGroups; ++q) {
      tc::mbar_init(&bar_ready[q], 128);
      tc::mbar_init(&bar_done[q], 1);
    }
    tc::mbar_init(&bar_free, 128);
    tc::mbar_init(&bar_drain, 1);
    s_fail = 0;
  }
  if (warp == 0) tc::tmem_alloc(&tbase, 512);
  tc::fence_async_smem();
  tc::fence_before_sync();
  __syncthreads();
  tc::fence_after_sync();
  const uint32_t tmem = tbase;
  // the first layer's accumulator has the ones columns unless kOut outputs need the room
  auto dw_width = [](int l) { return (l == 0 ? kFin : kH) + ((l == 0 && kMulti) ? 0 : 16); };
  uint32_t dwcol[kLayers];
  uint32_t col = 0;
  for (int l = kLayers - 1; l >= 0; --l) {
    dwcol[l] = col;
    col += dw_width(l);
  }
  const uint32_t dwo_col = col;                       // kOut outputs: dW_out^T
  const uint32_t scratch = col + (kMulti ? kOut : 0);  // 3 layers: 336 (+ 0) or 320 + 64 = 384; + 128 <= 512
  const size_t ntiles = (rows + kRows - 1) / kRows;
  const size_t zrows = ntiles * kRows;   // pre-activation rows, whole tiles
  const size_t tile_stride = (size_t)gridDim.x * kBwdGroups;
  // steps per tile, from the top: the output step (kOut outputs), then hidden layers L-1 .. 0
  constexpr int kTop = kMulti ? kLayers : kLayers - 1;

  if (grp == kBwdGroups) {
    // ---- MMA warp: one thread issues every MMA of the CTA, in the order
    // (tile round, step, group), so both groups' weight gradients accumulate
    // into the same TMEM columns in issue order.
    if (lane == 0) {
      uint32_t ph_ready[kBwdGroups] = {};
      bool first[kLayers + 1];
      for (int l = 0; l <= kLayers; ++l) first[l] = true;
      uint32_t n_da = 0;
      bool ok = true;
      for (size_t base = (size_t)blockIdx.x * kBwdGroups; base < ntiles && ok; base += tile_stride) {
        for (int l = kTop; l >= 0 && ok; --l) {
          const bool out_step = kMulti && l == kLayers;
          const int in = l == 0 ? kFin : kH;
          for (int q = 0; q < kBwdGroups; ++q) {
            if (base + q >= ntiles) break;
            if (!tc::mbar_wait(&bar_ready[q], ph_ready[q], polls)) {
              ok = false;
              break;
            }
            ph_ready[q] ^= 1u;
            tc::fence_after_sync();
            const uint32_t zq = tc::smem_u32(groups + (size_t)q * kGroupBytes);
            const uint32_t aq = zq + (uint32_t)(kRows * kH * 2);
            if (out_step) {
              // dW_out^T += A_{L-1}^T dO: A operand A^T (M = hidden units, K = rows) and B operand
              // dO^T (N = outputs, K = rows), MN-major views of the row tiles
              const uint32_t id_o = tc::idesc_bf16(kH, kOut, true, true);
              for (int kk = 0; kk < kRows / 16; ++kk)
                tc::mma_bf16(tmem + dwo_col, tc::smem_desc(aq + kk * 2 * kSboA, kSboA, 128u),
                             tc::smem_desc(zq + kk * 2 * kSboO, kSboO, 128u), id_o,
                             (!first[kLayers] || kk > 0) ? 1u : 0u);
              first[kLayers] = false;
            } else {
              // dW_l | db_l += dZ^T [A | 1]: A operand dZ^T (M = outputs, K = rows) and
              // B operand [A | 1]^T (N = in (+ 16), K = rows), both MN-major views of the
              // row-major tiles (core-matrix stride 128 B along M/N, one row group along K)
              const uint32_t id_w = tc::idesc_bf16(kH, dw_width(l), true, true);
              for (int kk = 0; kk < kRows / 16; ++kk)
                tc::mma_bf16(tmem + dwcol[l], tc::smem_desc(zq + kk * 2 * kSboH, kSboH, 128u),
                             tc::smem_desc(aq + kk * 2 * kSboA, kSboA, 128u), id_w,
                             (!first[l] || kk > 0) ? 1u : 0u);
              first[l] = false;
            }
            // dA = dZ_l W_l (or dO W_out) into the scratch, once its previous reader has drained it
            if (n_da > 0) {
              if (!tc::mbar_wait(&bar_free, (n_da - 1) & 1u, polls)) {
                ok = false;
                break;
              }
              tc::fence_after_sync();
            }
            if (out_step) {
              const uint32_t id_x = tc::idesc_bf16(kRows, kH, false, true);
              const uint32_t wo = tc::smem_u32(Wo);
              for (int kk = 0; kk < kOut / 16; ++kk)
                tc::mma_bf16(tmem + scratch, tc::smem_desc(zq + kk * 2 * kLbo, kLbo, kSboO),
                             tc::smem_desc(wo + kk * 2 * kLbo, kLbo, kSboO), id_x, kk > 0 ? 1u : 0u);
            } else {
              const uint32_t id_x = tc::idesc_bf16(kRows, in, false, true);
              const uint32_t wb = tc::smem_u32(Wb[l]);
              for (int kk = 0; kk < kH / 16; ++kk)
                tc::mma_bf16(tmem + scratch, tc::smem_desc(zq + kk * 2 * kLbo, kLbo, kSboH),
                             tc::smem_desc(wb + kk * 2 * kLbo, kLbo, kSboH), id_x, kk > 0 ? 1u : 0u);
            }
            ++n_da;
            tc::commit(&bar_done[q]);
          }
        }
      }
      if (!ok) s_fail = 1;
    }
  } else {
    // ---- compute warpgroup
    const uint32_t lane_base = (uint32_t)((warp & 3) * 32) << 16;
    const uint32_t bar_id = 1u + (uint32_t)grp;
    uint32_t ph_done = 0;
    bool ok = true;
    for (size_t tile = (size_t)blockIdx.x * kBwdGroups + grp; tile < ntiles && ok; tile += tile_stride) {
      const size_t row0 = tile * kRows, row = row0 + t;
      const bool valid = row < rows;
      if (t == 0) {
        // into L2 ahead of use: this tile's remaining pre-activation slabs (one
        // contiguous 32 KB range per layer), then the next tile's first inputs
        for (int l = 0; l + 1 < kLayers; ++l) tc::prefetch_l2(zb + z_row_base(zrows, l, tile, 0), kRows * kH * 2);
        const size_t nt = tile + tile_stride;
        if (nt < ntiles) {
          const size_t r1 = nt * kRows;
          const uint32_t n1 = (uint32_t)(rows - r1 < (size_t)kRows ? rows - r1 : (size_t)kRows);
          tc::prefetch_l2(zb + z_row_base(zrows, kLayers - 1, nt, 0), kRows * kH * 2);
          tc::prefetch_l2(S + r1 * kOut, n1 * 4 * kOut);
          tc::prefetch_l2(radii + r1, n1 * 4);
          tc::prefetch_l2(dL_dsignal + (kMulti ? r1 * kOut : 2 * r1), n1 * (kMulti ? 4 * kOut : 8));
        }
      }
      const bool vis = valid && radii[row] > 0;
      if constexpr (kMulti) {
        // dO = dL/dfeatures * s (1 - s) -> the dO row tile (BF16) in the dZ buffer; db_out
#pragma unroll 1
        for (int c0 = 0; c0 < kOut; c0 += 32) {
          float d[32];
#pragma unroll
          for (int q = 0; q < 8; ++q) {
            float4 sv = make_float4(0.f, 0.f, 0.f, 0.f), gv = make_float4(0.f, 0.f, 0.f, 0.f);
            if (vis) {
              sv = *reinterpret_cast<const float4*>(S + row * kOut + c0 + 4 * q);
              gv = *reinterpret_cast<const float4*>(dL_dsignal + row * kOut + c0 + 4 * q);
            }
            d[4 * q] = gv.x * sv.x * (1.0f - sv.x);
            d[4 * q + 1] = gv.y * sv.y * (1.0f - sv.y);
            d[4 * q + 2] = gv.z * sv.z * (1.0f - sv.z);
            d[4 * q + 3] = gv.w * sv.w * (1.0f - sv.w);
          }
#pragma unroll
          for (int q = 0; q < 4; ++q)
            *reinterpret_cast<uint4*>(dZ + tc::kmajor_off(t, c0 + q * 8, kLbo, kSboO)) = pack8(d + q * 8);
          const float sum = warp_transpose_sum32(d, lane);
          atomicAdd(&s_red[c0 + lane], sum);
        }
      } else {
        // output layer: dO, its weight gradient (reduced over the warp's rows), dZ of the last hidden layer
        const float s = valid ? S[row] : 0.0f;
        const float dO = vis ? dL_dsignal[2 * row] * s * (1.0f - s) : 0.0f;
        const __nv_bfloat16* zl = zb + z_row_base(zrows, kLayers - 1, tile, t);
#pragma unroll 1
        for (int c0 = 0; c0 < kH; c0 += 32) {
          uint4 zq[4];   // a 32-column chunk of the row in flight at once
#pragma unroll
          for (int q = 0; q < 4; ++q)
            zq[q] = valid ? *reinterpret_cast<const uint4*>(zl + (size_t)(c0 / 8 + q) * kZChunk)
                          : make_uint4(0u, 0u, 0u, 0u);
          float red[32];
#pragma unroll
          for (int q = 0; q < 4; ++q) {
            float z[8], dz[8];
            unpack8(zq[q], z);
#pragma unroll
            for (int i = 0; i < 8; ++i) {
              if (i & 1) continue;
              float2 a, d;
              act_and_grad2(act, make_float2(z[i], z[i + 1]), a, d);
              red[q * 8 + i] = dO * a.x;
              red[q * 8 + i + 1] = dO * a.y;
              dz[i] = dO * wout[c0 + q * 8 + i] * d.x;
              dz[i + 1] = dO * wout[c0 + q * 8 + i + 1] * d.y;
            }
            *reinterpret_cast<uint4*>(dZ + tc::kmajor_off(t, c0 + q * 8, kLbo, kSboH)) = pack8(dz);
          }
          const float sum = warp_transpose_sum32(red, lane);
          atomicAdd(&s_red[c0 + lane], sum);
        }
        float dsum = dO;
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) dsum += __shfl_xor_sync(0xffffffffu, dsum, o);
        if (lane == 0) atomicAdd(&s_red[kH], dsum);
      }
      for (int l = kTop; l >= 0; --l) {
        // act'(Z_{l-1}) of this row, kept for dZ_{l-1} after the MMAs as FP16 pairs
        // (nine warps leave 168 registers a thread; the FP16 rounding, 2^-11
        // relative, sits below the BF16 rounding of dZ that follows)
        __half2 ad[kH / 2];
        // A_{l-1}: features (l == 0) or act(Z_{l-1}); the ones column sits at `in`
        if (l == 0) {
          int r, g;
          row_pair(row0, t, P, r, g);
          float x[kFin];
          pair_features(means3D, rx_pos, g, r, vis, x);
#pragma unroll
          for (int kc = 0; kc < kFin / 8; ++kc)
            *reinterpret_cast<uint4*>(Ab + tc::kmajor_off(t, kc * 8, kLbo, kSboA)) = pack8(x + kc * 8);
          if constexpr (!kMulti) {
            *reinterpret_cast<uint4*>(Ab + tc::kmajor_off(t, kFin, kLbo, kSboA)) =
                make_uint4(pack2(1.0f, 0.0f), 0u, 0u, 0u);
            *reinterpret_cast<uint4*>(Ab + tc::kmajor_off(t, kFin + 8, kLbo, kSboA)) = make_uint4(0u, 0u, 0u, 0u);
          }
        } else {
          const __nv_bfloat16* zp = zb + z_row_base(zrows, l - 1, tile, t);
#pragma unroll
          for (int c0 = 0; c0 < kH; c0 += 8) {
            float z[8], a[8];
            if (valid) unpack8(*reinterpret_cast<const uint4*>(zp + (size_t)(c0 / 8) * kZChunk), z);
            else
#pragma unroll
              for (int i = 0; i < 8; ++i) z[i] = 0.0f;
            float d[8];
#pragma unroll
            for (int i = 0; i < 4; ++i) {
              float2 a2, d2;
              act_and_grad2(act, make_float2(z[2 * i], z[2 * i + 1]), a2, d2);
              a[2 * i] = a2.x;
              a[2 * i + 1] = a2.y;
              d[2 * i] = d2.x;
              d[2 * i + 1] = d2.y;
            }
#pragma unroll
            for (int i = 0; i < 4; ++i) ad[c0 / 2 + i] = __floats2half2_rn(d[2 * i], d[2 * i + 1]);
            *reinterpret_cast<uint4*>(Ab + tc::kmajor_off(t, c0, kLbo, kSboA)) = pack8(a);
          }
        }
        // hand dZ_l (or dO) and A_{l-1} to the MMA warp
        tc::fence_async_smem();
        tc::mbar_arrive(&bar_ready[grp]);
        const bool got = tc::mbar_wait(&bar_done[grp], ph_done, polls);
        ph_done ^= 1u;
        tc::fence_after_sync();
        if (!tc::named_all(bar_id, 128, got)) {
          ok = false;
          break;
        }
        if (l == 0) {
          float v[32];
          tc::tmem_ld32(tmem + lane_base + scratch, v);
          tc::fence_before_sync();
          tc::mbar_arrive(&bar_free);
          if (valid)
#pragma unroll
            for (int q = 0; q < 8; ++q)
              *reinterpret_cast<float4*>(dX0 + row * kFin + q * 4) =
                  make_float4(v[4 * q], v[4 * q + 1], v[4 * q + 2], v[4 * q + 3]);
        } else {
          // dZ_{l-1} = dA_{l-1} * act'(Z_{l-1}); the MMAs that read dZ_l (or dO) are done
#pragma unroll
          for (int c0 = 0; c0 < kH; c0 += 32) {
            float v[32];
            tc::tmem_ld32(tmem + lane_base + scratch + c0, v);
            if (c0 + 32 == kH) {
              tc::fence_before_sync();
              tc::mbar_arrive(&bar_free);
            }
#pragma unroll
            for (int i = 0; i < 16; ++i) {
              const float2 d = __half22float2(ad[c0 / 2 + i]);
              v[2 * i] *= d.x;
              v[2 * i + 1] *= d.y;
            }
#pragma unroll
            for (int q = 0; q < 4; ++q) {
              const uint4 p = pack8(v + q * 8);
              *reinterpret_cast<uint4*>(dZ + tc::kmajor_off(t, c0 + q * 8, kLbo, kSboH)) = p;
              if (kMulti && l == 1) unpack8(p, v + q * 8);   // db_0 sums the BF16 dZ_0 the MMAs see
            }
            if (kMulti && l == 1) {
              const float sum = warp_transpose_sum32(v, lane);
              atomicAdd(&s_red[kOut + c0 + lane], sum);
            }
          }
        }
      }
    }
    if (!ok && t == 0) s_fail = 1;
  }
  __syncthreads();
  tc::fence_after_sync();
  // the CTA's weight and bias gradients -> global (rows of dW_l are TMEM lanes);
  // (layer, 32-column chunk) items are split over the compute warpgroups
  if (!s_fail && grp < kBwdGroups) {
    const uint32_t lane_base = (uint32_t)((warp & 3) * 32) << 16;
    int item = 0;
    for (int l = 0; l < kLayers; ++l) {
      const int in = l == 0 ? kFin : kH;
      const int ncols = (l == 0 && kMulti) ? in : in + 1;   // weights, then the bias column
#pragma unroll 1
      for (int c0 = 0; c0 < ncols; c0 += 32, ++item) {
        if (item % kBwdGroups != grp) continue;
        float v[32];
        tc::tmem_ld32(tmem + lane_base + dwcol[l] + c0, v);
#pragma unroll
        for (int i = 0; i < 32; ++i) {
          const int n = c0 + i;
          if (n < in) atomicAdd(&dparams[woff[l] + (size_t)t * in + n], v[i]);
          else if (n == in && n < ncols) atomicAdd(&dparams[boff[l] + t], v[i]);
        }
      }
    }
    if constexpr (kMulti) {
      // dW_out^T: lane = hidden unit t, column = output
#pragma unroll 1
      for (int c0 = 0; c0 < kOut; c0 += 32, ++item) {
        if (item % kBwdGroups != grp) continue;
        float v[32];
        tc::tmem_ld32(tmem + lane_base + dwo_col + c0, v);
#pragma unroll
        for (int i = 0; i < 32; ++i) atomicAdd(&dparams[woff[kLayers] + (size_t)(c0 + i) * kH + t], v[i]);
      }
      if (grp == 0) {
        for (int j = t; j < kOut; j += 128) atomicAdd(&dparams[boff[kLayers] + j], s_red[j]);
        for (int j = t; j < kH; j += 128) atomicAdd(&dparams[boff[0] + j], s_red[kOut + j]);
      }
    } else {
      if (grp == 0)
        for (int j = t; j <= kH; j += 128) atomicAdd(&dparams[j < kH ? woff[kLayers] + j : boff[kLayers]], s_red[j]);
    }
  }
  if (s_fail && tid == 0 && hdr) atomic_or_error(hdr, kErrMlpWait);
  if (s_fail && grp == kBwdGroups && lane == 0) {
    // drain: every MMA the issuing thread started completes before the
    // tensor memory is freed
    tc::commit(&bar_drain);
    tc::mbar_wait(&bar_drain, 0, kPolls);
  }
  tc::fence_before_sync();
  __syncthreads();
  if (warp == 0) tc::tmem_dealloc(tmem, 512);
}

// ---- launchers ------------------------------------------------------------------

size_t mlp_bf16_forward_smem(int layers, int out) {
  const size_t base = (size_t)kH * kFin * 2 + (size_t)(layers - 1) * kH * kH * 2 +
                      (size_t)kFwdGroups * kRows * kH * 2 + (size_t)(layers * kH + kH + 4) * sizeof(float);
  return out > 1 ? (base + 127) / 128 * 128 + (size_t)out * kH * 2 : base;
}
size_t mlp_bf16_backward_smem(int layers, int out) {
  return (size_t)kFin * kH * 2 + (size_t)(layers - 1) * kH * kH * 2 +
         (size_t)kBwdGroups * ((size_t)kRows * kH * 2 + (size_t)kRows * (kH + 16) * 2) + (size_t)kH * sizeof(float) +
         (out > 1 ? (size_t)out * kH * 2 : 0);
}

template <int L, int A, int O>
static cudaError_t launch_bf16_layers(bool fwd, int P, size_t rows, const float* means3D, const float* rx_pos,
                                      const float* params, const GeomView& geo, const SharedMlpLayout& Lt,
                                      float* work, const float* dL_dsignal, float* dparams, ImageHeader* hdr,
                                      cudaStream_t s) {
  const size_t smem = fwd ? mlp_bf16_forward_smem(L, O) : mlp_bf16_backward_smem(L, O);
  static bool attr_done[2][64] = {};   // per instantiation
  static int sm_count[64] = {};
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return e;
  int sms = dev >= 0 && dev < 64 ? sm_count[dev] : 0;
  if (sms == 0) {
    if ((e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev)) != cudaSuccess) return e;
    if (dev >= 0 && dev < 64) sm_count[dev] = sms;
  }
  if (dev < 0 || dev >= 64 || !attr_done[fwd][dev]) {
    e = fwd ? cudaFuncSetAttribute(mlp_bf16_forward_kernel<L, A, O>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                   (int)smem)
            : cudaFuncSetAttribute(mlp_bf16_backward_kernel<L, A, O>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                   (int)smem);
    if (e != cudaSuccess) return e;
    if (dev >= 0 && dev < 64) attr_done[fwd][dev] = true;
  }
  // persistent: at most one CTA per SM, and every CTA's first warpgroup owns a tile
  const size_t ntiles = (rows + kRows - 1) / kRows;
  const size_t per = fwd ? kFwdGroups : kBwdGroups;
  const size_t want = (ntiles + per - 1) / per;
  const unsigned grid = (unsigned)(want < (size_t)sms ? want : (size_t)sms);
  __nv_bfloat16* zb = reinterpret_cast<__nv_bfloat16*>(work + Lt.z[1]);
  if (fwd)
    mlp_bf16_forward_kernel<L, A, O><<<grid, 128 * kFwdGroups, smem, s>>>(P, rows, means3D, rx_pos, params,
                                                                          geo.radii, zb, work + Lt.s, geo.signal,
                                                                          hdr, wait_polls(kPolls));
  else
    mlp_bf16_backward_kernel<L, A, O><<<grid, kBwdThreads, smem, s>>>(P, rows, means3D, rx_pos, params, geo.radii,
                                                                      zb, work + Lt.s, dL_dsignal, work + Lt.d0,
                                                                      dparams, hdr, wait_polls(kPolls));
  return cudaGetLastError();
}

template <int L>
static cudaError_t launch_bf16_act(bool fwd, int P, size_t rows, int act, int out, const float* means3D,
                                   const float* rx_pos, const float* params, const GeomView& geo,
                                   const SharedMlpLayout& Lt, float* work, const float* dL_dsignal, float* dparams,
                                   ImageHeader* hdr, cudaStream_t s) {
  if (out == 64)
    return act == 1 ? launch_bf16_layers<L, 1, 64>(fwd, P, rows, means3D, rx_pos, params, geo, Lt, work,
                                                   dL_dsignal, dparams, hdr, s)
                    : launch_bf16_layers<L, 2, 64>(fwd, P, rows, means3D, rx_pos, params, geo, Lt, work,
                                                   dL_dsignal, dparams, hdr, s);
  if (out != 1) return cudaErrorInvalidValue;
  return act == 1 ? launch_bf16_layers<L, 1, 1>(fwd, P, rows, means3D, rx_pos, params, geo, Lt, work, dL_dsignal,
                                                dparams, hdr, s)
                  : launch_bf16_layers<L, 2, 1>(fwd, P, rows, means3D, rx_pos, params, geo, Lt, work, dL_dsignal,
                                                dparams, hdr, s);
}

cudaError_t launch_shared_mlp_bf16(bool fwd, int P, int R, int layers, int act, int out, const float* means3D,
                                   const float* rx_pos, const float* params, const GeomView& geo, float* work,
                                   const float* dL_dsignal, float* dparams, float* dL_dmeans3D, ImageHeader* hdr,
                                   cudaStream_t s) {
  const size_t rows = (size_t)P * R;
  const SharedMlpLayout Lt = shared_mlp_layout_bf16(layers, rows, out);
  cudaError_t e = cudaSuccess;
  if (!fwd) {
    e = cudaMemsetAsync(dparams, 0, Lt.params * sizeof(float), s);
    if (e != cudaSuccess) return e;
  }
  switch (layers) {
    case 1: e = launch_bf16_act<1>(fwd, P, rows, act, out, means3D, rx_pos, params, geo, Lt, work, dL_dsignal, dparams, hdr, s); break;
    case 2: e = launch_bf16_act<2>(fwd, P, rows, act, out, means3D, rx_pos, params, geo, Lt, work, dL_dsignal, dparams, hdr, s); break;
    case 3: e = launch_bf16_act<3>(fwd, P, rows, act, out, means3D, rx_pos, params, geo, Lt, work, dL_dsignal, dparams, hdr, s); break;
    default: return cudaErrorInvalidValue;
  }
  if (e != cudaSuccess || fwd || dL_dmeans3D == nullptr) return e;
  return launch_mlp_features_backward(P, R, means3D, rx_pos, geo.radii, work + Lt.d0, dL_dmeans3D, s);
}

}  // namespace gsparc
