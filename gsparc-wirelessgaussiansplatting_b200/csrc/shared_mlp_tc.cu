// Shared emission MLP in BF16 on the 5th-generation tensor cores (tcgen05).
//
// Same network as shared_mlp.cu (features, hidden layers of width 128,
// sigmoid of one output) with BF16 operands and FP32 accumulation in tensor
// memory.  Two fused kernels, each a persistent loop over tiles of 128
// (receiver, Gaussian) rows with one row per thread of a 128-thread CTA:
//
//   forward:  features -> [MMA -> +bias, act] x layers -> output dot on the
//             CUDA cores -> sigmoid.  The layer weights stay in shared memory
//             for the whole launch; only the BF16 pre-activations of each
//             hidden layer (for the adjoint) and the signal go to HBM.
//   backward: from dL/dsignal, per tile and layer l (last first):
//               dW_l (+ db_l)  += dZ_l^T [A_{l-1} | 1]   (M = 128 outputs,
//                                 K = 128 rows, accumulated in TMEM over all
//                                 of the CTA's tiles; the ones row yields db)
//               dA_{l-1}        = dZ_l W_l             (M = 128 rows)
//             with A_{l-1} = act(Z_{l-1}) recomputed from the stored
//             pre-activations and the features recomputed from the centres;
//             the output layer's gradient is reduced on the CUDA cores.  At
//             the end every CTA adds its TMEM accumulators to the global
//             gradient.
//
// Operands use the no-swizzle core-matrix layouts of tcgen05.cuh.  One thread
// issues the MMAs; completion is signalled through an mbarrier (bounded wait:
// on give-up the error word gets kErrMlpWait and the CTA stops).
#include <cuda_bf16.h>

#include "common.cuh"
#include "kernels.cuh"
#include "tcgen05.cuh"

namespace gsparc {

namespace {

constexpr int kH = 128;        // hidden width of the BF16 path
constexpr int kFin = 32;       // features
constexpr int kRows = 128;     // rows per tile (= MMA M)
constexpr uint32_t kLbo = 128; // core matrices along K are adjacent
constexpr uint32_t kPolls = 1u << 24;
constexpr float kPiF = 3.14159265358979323846f;

__device__ __forceinline__ float gelu(float z) { return 0.5f * z * (1.0f + erff(z * 0.70710678118654752f)); }
__device__ __forceinline__ float gelu_d(float z) {
  return 0.5f * (1.0f + erff(z * 0.70710678118654752f)) + z * 0.39894228040143268f * expf(-0.5f * z * z);
}
__device__ __forceinline__ float actf(int act, float z) { return act == 1 ? fmaxf(z, 0.0f) : gelu(z); }
__device__ __forceinline__ float actd(int act, float z) { return act == 1 ? (z > 0.0f ? 1.0f : 0.0f) : gelu_d(z); }

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

// Features of one pair (as mlp_features_kernel), zero for culled pairs.
__device__ __forceinline__ void pair_features(const float* __restrict__ means3D, const float* __restrict__ rx_pos,
                                              int P, size_t row, bool vis, float* x) {
  if (!vis) {
#pragma unroll
    for (int i = 0; i < kFin; ++i) x[i] = 0.0f;
    return;
  }
  const int g = (int)(row % P), r = (int)(row / P);
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
      sincosf((float)(1 << k) * kPiF * m[j], &s, &c);
      x[3 + 6 * k + 2 * j] = s;
      x[4 + 6 * k + 2 * j] = c;
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

struct TileSync {
  uint64_t* mbar;
  uint32_t phase;
  // all threads: make generic smem writes visible to the MMA and order TMEM use
  __device__ __forceinline__ void publish() {
    tc::fence_async_smem();
    tc::fence_before_sync();
    __syncthreads();
    tc::fence_after_sync();
  }
  __device__ __forceinline__ bool wait() {
    const bool ok = tc::mbar_wait(mbar, phase, kPolls);
    phase ^= 1u;
    tc::fence_after_sync();
    return ok;
  }
};

}  // namespace

// ---- forward ------------------------------------------------------------------
// dynamic smem: W_l K-major [128 x in_l] bf16 (l < layers), X [128 x 32],
// H [128 x 128] K-major bf16, biases and the output row in fp32.
template <int kLayers>
__global__ void __launch_bounds__(128)
mlp_bf16_forward_kernel(int P, size_t rows, int act, const float* __restrict__ means3D,
                        const float* __restrict__ rx_pos, const float* __restrict__ params,
                        const int* __restrict__ radii, __nv_bfloat16* __restrict__ zb, float* __restrict__ S,
                        float2* __restrict__ signal, ImageHeader* __restrict__ hdr) {
  extern __shared__ __align__(1024) unsigned char smem[];
  __shared__ __align__(8) uint64_t mbar;
  __shared__ uint32_t tbase;
  const int t = threadIdx.x, warp = t >> 5;
  unsigned char* Ws[kLayers];
  size_t off = 0;
  for (int l = 0; l < kLayers; ++l) {
    Ws[l] = smem + off;
    off += (size_t)kH * (l == 0 ? kFin : kH) * 2;
  }
  unsigned char* Xs = smem + off;
  off += (size_t)kRows * kFin * 2;
  unsigned char* Hs = smem + off;
  off += (size_t)kRows * kH * 2;
  float* bias = reinterpret_cast<float*>(smem + off);   // [kLayers][128], then w_out[128], b_out
  float* wout = bias + kLayers * kH;

  // weights -> bf16 K-major (B operand: n = output, k = input), once per CTA
  size_t poff = 0;
  for (int l = 0; l < kLayers; ++l) {
    const int in = l == 0 ? kFin : kH;
    const float* W = params + poff;
    const uint32_t sbo = (uint32_t)(in / 8) * 128u;
    for (int c = t; c < kH * (in / 8); c += blockDim.x) {
      const int n = c / (in / 8), kc = c % (in / 8);
      float v[8];
#pragma unroll
      for (int i = 0; i < 8; ++i) v[i] = W[(size_t)n * in + kc * 8 + i];
      *reinterpret_cast<uint4*>(Ws[l] + tc::kmajor_off(n, kc * 8, kLbo, sbo)) = pack8(v);
    }
    poff += (size_t)kH * in;
    for (int j = t; j < kH; j += blockDim.x) bias[l * kH + j] = params[poff + j];
    poff += kH;
  }
  for (int j = t; j < kH; j += blockDim.x) wout[j] = params[poff + j];
  const float bout = params[poff + kH];
  if (t == 0) tc::mbar_init(&mbar, 1);
  if (warp == 0) tc::tmem_alloc(&tbase, kH);
  TileSync sync{&mbar, 0u};
  sync.publish();
  const uint32_t tmem = tbase;
  const uint32_t lane_base = (uint32_t)(warp * 32) << 16;
  bool ok = true;
  const size_t ntiles = (rows + kRows - 1) / kRows;
  for (size_t tile = blockIdx.x; tile < ntiles && ok; tile += gridDim.x) {
    const size_t row = tile * kRows + t;
    const bool valid = row < rows;
    const bool vis = valid && radii[row] > 0;
    {
      float x[kFin];
      pair_features(means3D, rx_pos, P, row, vis, x);
#pragma unroll
      for (int kc = 0; kc < kFin / 8; ++kc)
        *reinterpret_cast<uint4*>(Xs + tc::kmajor_off(t, kc * 8, kLbo, (kFin / 8) * 128u)) = pack8(x + kc * 8);
    }
    sync.publish();
    float o = bout;
    for (int l = 0; l < kLayers && ok; ++l) {
      const int in = l == 0 ? kFin : kH;
      if (t == 0) {
        const uint32_t sbo = (uint32_t)(in / 8) * 128u;
        const uint32_t a0 = tc::smem_u32(l == 0 ? Xs : Hs), b0 = tc::smem_u32(Ws[l]);
        const uint32_t idesc = tc::idesc_bf16(kRows, kH, false, false);
        for (int kk = 0; kk < in / 16; ++kk)
          tc::mma_bf16(tmem, tc::smem_desc(a0 + kk * 2 * kLbo, kLbo, sbo),
                       tc::smem_desc(b0 + kk * 2 * kLbo, kLbo, sbo), idesc, kk > 0 ? 1u : 0u);
        tc::commit(&mbar);
      }
      if (!sync.wait()) {
        ok = false;
        break;
      }
      __nv_bfloat16* z_out = zb + (size_t)l * rows * kH;
#pragma unroll 1
      for (int c0 = 0; c0 < kH; c0 += 32) {
        float v[32];
        tc::tmem_ld32(tmem + lane_base + c0, v);
#pragma unroll
        for (int q = 0; q < 4; ++q) {
          float z[8], a[8];
#pragma unroll
          for (int i = 0; i < 8; ++i) z[i] = v[q * 8 + i] + bias[l * kH + c0 + q * 8 + i];
          const uint4 zp = pack8(z);
          if (valid) *reinterpret_cast<uint4*>(z_out + row * kH + c0 + q * 8) = zp;
          // the next layer (and the adjoint) see the BF16-rounded pre-activation
          float zr[8];
          unpack8(zp, zr);
#pragma unroll
          for (int i = 0; i < 8; ++i) a[i] = actf(act, zr[i]);
          if (l + 1 < kLayers) {
            *reinterpret_cast<uint4*>(Hs + tc::kmajor_off(t, c0 + q * 8, kLbo, (kH / 8) * 128u)) = pack8(a);
          } else {
#pragma unroll
            for (int i = 0; i < 8; ++i) o += wout[c0 + q * 8 + i] * a[i];
          }
        }
      }
      sync.publish();
    }
    if (ok && valid) {
      const float s = 1.0f / (1.0f + expf(-o));
      S[row] = s;
      if (vis) signal[row] = make_float2(s, 0.0f);
    }
  }
  if (!ok && t == 0 && hdr) atomic_or_error(hdr, kErrMlpWait);
  tc::fence_before_sync();
  __syncthreads();
  if (warp == 0) tc::tmem_dealloc(tmem, kH);
}

// ---- backward -----------------------------------------------------------------
// dynamic smem: W_l as the MN-major B operand of dA = dZ W ([n = in_l] x
// [k = 128 outputs]) for every layer; dZ K-major and MN-major [128 x 128];
// A_{l-1} MN-major [(in + 16) x 128 rows] (row `in` = ones, the rest of the
// 16 extra rows zero); the output row and its gradient in fp32.
// TMEM columns: dW_l accumulators of (in_l + 16) columns each, then a
// 144-column scratch accumulator.
template <int kLayers>
__global__ void __launch_bounds__(128)
mlp_bf16_backward_kernel(int P, size_t rows, int act, const float* __restrict__ means3D,
                         const float* __restrict__ rx_pos, const float* __restrict__ params,
                         const int* __restrict__ radii, const __nv_bfloat16* __restrict__ zb,
                         const float* __restrict__ S, const float* __restrict__ dL_dsignal,
                         float* __restrict__ dX0, float* __restrict__ dparams, ImageHeader* __restrict__ hdr) {
  extern __shared__ __align__(1024) unsigned char smem[];
  __shared__ __align__(8) uint64_t mbar;
  __shared__ uint32_t tbase;
  __shared__ float s_dwo[kH + 1];
  const int t = threadIdx.x, warp = t >> 5, lane = t & 31;
  unsigned char* Wb[kLayers];
  size_t off = 0;
  for (int l = 0; l < kLayers; ++l) {
    Wb[l] = smem + off;
    off += (size_t)(l == 0 ? kFin : kH) * kH * 2;
  }
  unsigned char* dZk = smem + off;
  off += (size_t)kRows * kH * 2;
  unsigned char* dZm = smem + off;
  off += (size_t)kH * kRows * 2;
  unsigned char* Am = smem + off;
  off += (size_t)(kH + 16) * kRows * 2;
  float* wout = reinterpret_cast<float*>(smem + off);
  constexpr uint32_t kSboRows = (kRows / 8) * 128u;   // MN-major, K = 128 rows
  constexpr uint32_t kSboH = (kH / 8) * 128u;         // K-major / MN-major with K = 128

  // W_l [out][in] -> MN-major B operand (n = in, k = out), once per CTA
  size_t poff = 0;
  size_t woff[kLayers + 1], boff[kLayers + 1];
  for (int l = 0; l < kLayers; ++l) {
    const int in = l == 0 ? kFin : kH;
    woff[l] = poff;
    const float* W = params + poff;
    for (int c = t; c < kH * (in / 8); c += blockDim.x) {
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
  boff[kLayers] = poff + kH;
  for (int j = t; j < kH; j += blockDim.x) wout[j] = params[woff[kLayers] + j];
  for (int j = t; j <= kH; j += blockDim.x) s_dwo[j] = 0.0f;
  if (t == 0) tc::mbar_init(&mbar, 1);
  if (warp == 0) tc::tmem_alloc(&tbase, 512);
  TileSync sync{&mbar, 0u};
  sync.publish();
  const uint32_t tmem = tbase;
  const uint32_t lane_base = (uint32_t)(warp * 32) << 16;
  uint32_t dwcol[kLayers];
  uint32_t col = 0;
  for (int l = kLayers - 1; l >= 0; --l) {
    dwcol[l] = col;
    col += (l == 0 ? kFin : kH) + 16;
  }
  const uint32_t scratch = col;   // <= 144 + 144 + 48 = 336; scratch needs 128 more
  bool ok = true;
  bool any_tile = false;
  const size_t ntiles = (rows + kRows - 1) / kRows;
  for (size_t tile = blockIdx.x; tile < ntiles && ok; tile += gridDim.x) {
    const size_t row = tile * kRows + t;
    const bool valid = row < rows;
    const bool vis = valid && radii[row] > 0;
    // output layer: dO, its weight gradient (reduced over the warp's rows), dZ of the last hidden layer
    const float s = valid ? S[row] : 0.0f;
    const float dO = vis ? dL_dsignal[2 * row] * s * (1.0f - s) : 0.0f;
    {
      const __nv_bfloat16* zl = zb + (size_t)(kLayers - 1) * rows * kH;
#pragma unroll 1
      for (int c0 = 0; c0 < kH; c0 += 32) {
        float z[32], red[32];
#pragma unroll
        for (int q = 0; q < 4; ++q) {
          if (valid) unpack8(*reinterpret_cast<const uint4*>(zl + row * kH + c0 + q * 8), z + q * 8);
          else
#pragma unroll
            for (int i = 0; i < 8; ++i) z[q * 8 + i] = 0.0f;
        }
#pragma unroll
        for (int i = 0; i < 32; ++i) red[i] = dO * actf(act, z[i]);
        const float sum = warp_transpose_sum32(red, lane);
        atomicAdd(&s_dwo[c0 + lane], sum);
        float dz[32];
#pragma unroll
        for (int i = 0; i < 32; ++i) dz[i] = dO * wout[c0 + i] * actd(act, z[i]);
#pragma unroll
        for (int q = 0; q < 4; ++q) {
          const uint4 p = pack8(dz + q * 8);
          *reinterpret_cast<uint4*>(dZk + tc::kmajor_off(t, c0 + q * 8, kLbo, kSboH)) = p;
        }
        // MN-major copy: element (m = output c0 + i, k = row t)
#pragma unroll
        for (int i = 0; i < 32; ++i)
          *reinterpret_cast<__nv_bfloat16*>(dZm + tc::mnmajor_off(c0 + i, t, kLbo, kSboRows)) =
              __float2bfloat16_rn(dz[i]);
      }
      float dsum = dO;
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) dsum += __shfl_xor_sync(0xffffffffu, dsum, o);
      if (lane == 0) atomicAdd(&s_dwo[kH], dsum);
    }
    for (int l = kLayers - 1; l >= 0 && ok; --l) {
      const int in = l == 0 ? kFin : kH;
      // A_{l-1}: features (l == 0) or act(Z_{l-1}), MN-major with the ones row at n = in
      if (l == 0) {
        float x[kFin];
        pair_features(means3D, rx_pos, P, row, vis, x);
#pragma unroll
        for (int i = 0; i < kFin; ++i)
          *reinterpret_cast<__nv_bfloat16*>(Am + tc::mnmajor_off(i, t, kLbo, kSboRows)) = __float2bfloat16_rn(x[i]);
      } else {
        const __nv_bfloat16* zp = zb + (size_t)(l - 1) * rows * kH;
#pragma unroll 1
        for (int c0 = 0; c0 < kH; c0 += 8) {
          float z[8];
          if (valid) unpack8(*reinterpret_cast<const uint4*>(zp + row * kH + c0), z);
          else
#pragma unroll
            for (int i = 0; i < 8; ++i) z[i] = 0.0f;
#pragma unroll
          for (int i = 0; i < 8; ++i)
            *reinterpret_cast<__nv_bfloat16*>(Am + tc::mnmajor_off(c0 + i, t, kLbo, kSboRows)) =
                __float2bfloat16_rn(actf(act, z[i]));
        }
      }
#pragma unroll
      for (int i = 0; i < 16; ++i)
        *reinterpret_cast<__nv_bfloat16*>(Am + tc::mnmajor_off(in + i, t, kLbo, kSboRows)) =
            __float2bfloat16_rn(i == 0 ? 1.0f : 0.0f);
      sync.publish();
      if (t == 0) {
        const uint32_t zm = tc::smem_u32(dZm), zk = tc::smem_u32(dZk), am = tc::smem_u32(Am), wb = tc::smem_u32(Wb[l]);
        // dW_l | db_l  (M = 128 outputs, N = in + 16, K = 128 rows; both operands MN-major)
        const uint32_t id_w = tc::idesc_bf16(kH, in + 16, true, true);
        for (int kk = 0; kk < kRows / 16; ++kk)
          tc::mma_bf16(tmem + dwcol[l], tc::smem_desc(zm + kk * 2 * kLbo, kLbo, kSboRows),
                       tc::smem_desc(am + kk * 2 * kLbo, kLbo, kSboRows), id_w, (any_tile || kk > 0) ? 1u : 0u);
        // dA_{l-1} = dZ_l W_l  (M = 128 rows, N = in, K = 128 outputs)
        const uint32_t id_x = tc::idesc_bf16(kRows, in, false, true);
        for (int kk = 0; kk < kH / 16; ++kk)
          tc::mma_bf16(tmem + scratch, tc::smem_desc(zk + kk * 2 * kLbo, kLbo, kSboH),
                       tc::smem_desc(wb + kk * 2 * kLbo, kLbo, kSboH), id_x, kk > 0 ? 1u : 0u);
        tc::commit(&mbar);
      }
      if (!sync.wait()) {
        ok = false;
        break;
      }
      if (l == 0) {
        float v[32];
        tc::tmem_ld32(tmem + lane_base + scratch, v);
        if (valid)
#pragma unroll
          for (int q = 0; q < 8; ++q)
            *reinterpret_cast<float4*>(dX0 + row * kFin + q * 4) =
                make_float4(v[4 * q], v[4 * q + 1], v[4 * q + 2], v[4 * q + 3]);
      } else {
        const __nv_bfloat16* zp = zb + (size_t)(l - 1) * rows * kH;
#pragma unroll 1
        for (int c0 = 0; c0 < kH; c0 += 32) {
          float v[32], z[32];
          tc::tmem_ld32(tmem + lane_base + scratch + c0, v);
#pragma unroll
          for (int q = 0; q < 4; ++q) {
            if (valid) unpack8(*reinterpret_cast<const uint4*>(zp + row * kH + c0 + q * 8), z + q * 8);
            else
#pragma unroll
              for (int i = 0; i < 8; ++i) z[q * 8 + i] = 0.0f;
          }
#pragma unroll
          for (int i = 0; i < 32; ++i) v[i] = valid ? v[i] * actd(act, z[i]) : 0.0f;
#pragma unroll
          for (int q = 0; q < 4; ++q)
            *reinterpret_cast<uint4*>(dZk + tc::kmajor_off(t, c0 + q * 8, kLbo, kSboH)) = pack8(v + q * 8);
#pragma unroll
          for (int i = 0; i < 32; ++i)
            *reinterpret_cast<__nv_bfloat16*>(dZm + tc::mnmajor_off(c0 + i, t, kLbo, kSboRows)) =
                __float2bfloat16_rn(v[i]);
        }
      }
      sync.publish();
    }
    any_tile = true;
  }
  // the CTA's weight and bias gradients -> global (rows of dW_l are TMEM lanes)
  if (ok && any_tile) {
    for (int l = 0; l < kLayers; ++l) {
      const int in = l == 0 ? kFin : kH;
      const int m = warp * 32 + lane;
#pragma unroll 1
      for (int c0 = 0; c0 <= in; c0 += 32) {
        float v[32];
        tc::tmem_ld32(tmem + lane_base + dwcol[l] + c0, v);
#pragma unroll
        for (int i = 0; i < 32; ++i) {
          const int n = c0 + i;
          if (n < in) atomicAdd(&dparams[woff[l] + (size_t)m * in + n], v[i]);
          else if (n == in) atomicAdd(&dparams[boff[l] + m], v[i]);
        }
      }
    }
    __syncthreads();
    for (int j = t; j <= kH; j += blockDim.x)
      atomicAdd(&dparams[j < kH ? woff[kLayers] + j : boff[kLayers]], s_dwo[j]);
  }
  if (!ok && t == 0 && hdr) atomic_or_error(hdr, kErrMlpWait);
  tc::fence_before_sync();
  __syncthreads();
  if (warp == 0) tc::tmem_dealloc(tmem, 512);
}

// ---- launchers ------------------------------------------------------------------

size_t mlp_bf16_forward_smem(int layers) {
  return (size_t)kH * kFin * 2 + (size_t)(layers - 1) * kH * kH * 2 + (size_t)kRows * kFin * 2 +
         (size_t)kRows * kH * 2 + (size_t)(layers * kH + kH + 4) * sizeof(float);
}
size_t mlp_bf16_backward_smem(int layers) {
  return (size_t)kFin * kH * 2 + (size_t)(layers - 1) * kH * kH * 2 + 2 * (size_t)kRows * kH * 2 +
         (size_t)(kH + 16) * kRows * 2 + (size_t)kH * sizeof(float);
}

template <int L>
static cudaError_t launch_bf16_layers(bool fwd, int P, size_t rows, int act, const float* means3D,
                                      const float* rx_pos, const float* params, const GeomView& geo,
                                      const SharedMlpLayout& Lt, float* work, const float* dL_dsignal,
                                      float* dparams, ImageHeader* hdr, cudaStream_t s) {
  const size_t smem = fwd ? mlp_bf16_forward_smem(L) : mlp_bf16_backward_smem(L);
  static bool attr_done[2][64] = {};
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return e;
  if (dev < 0 || dev >= 64 || !attr_done[fwd][dev]) {
    e = fwd ? cudaFuncSetAttribute(mlp_bf16_forward_kernel<L>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem)
            : cudaFuncSetAttribute(mlp_bf16_backward_kernel<L>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                   (int)smem);
    if (e != cudaSuccess) return e;
    if (dev >= 0 && dev < 64) attr_done[fwd][dev] = true;
  }
  const size_t ntiles = (rows + kRows - 1) / kRows;
  const unsigned grid = (unsigned)(ntiles < 148 ? ntiles : 148);
  __nv_bfloat16* zb = reinterpret_cast<__nv_bfloat16*>(work + Lt.z[1]);
  if (fwd)
    mlp_bf16_forward_kernel<L><<<grid, 128, smem, s>>>(P, rows, act, means3D, rx_pos, params, geo.radii, zb,
                                                       work + Lt.s, geo.signal, hdr);
  else
    mlp_bf16_backward_kernel<L><<<grid, 128, smem, s>>>(P, rows, act, means3D, rx_pos, params, geo.radii, zb,
                                                        work + Lt.s, dL_dsignal, work + Lt.d0, dparams, hdr);
  return cudaGetLastError();
}

cudaError_t launch_shared_mlp_bf16(bool fwd, int P, int R, int layers, int act, const float* means3D,
                                   const float* rx_pos, const float* params, const GeomView& geo, float* work,
                                   const float* dL_dsignal, float* dparams, float* dL_dmeans3D, ImageHeader* hdr,
                                   cudaStream_t s) {
  const size_t rows = (size_t)P * R;
  const SharedMlpLayout Lt = shared_mlp_layout_bf16(layers, rows);
  cudaError_t e = cudaSuccess;
  if (!fwd) {
    e = cudaMemsetAsync(dparams, 0, Lt.params * sizeof(float), s);
    if (e != cudaSuccess) return e;
  }
  switch (layers) {
    case 1: e = launch_bf16_layers<1>(fwd, P, rows, act, means3D, rx_pos, params, geo, Lt, work, dL_dsignal, dparams, hdr, s); break;
    case 2: e = launch_bf16_layers<2>(fwd, P, rows, act, means3D, rx_pos, params, geo, Lt, work, dL_dsignal, dparams, hdr, s); break;
    case 3: e = launch_bf16_layers<3>(fwd, P, rows, act, means3D, rx_pos, params, geo, Lt, work, dL_dsignal, dparams, hdr, s); break;
    default: return cudaErrorInvalidValue;
  }
  if (e != cudaSuccess || fwd) return e;
  return launch_mlp_features_backward(P, R, means3D, rx_pos, geo.radii, work + Lt.d0, dL_dmeans3D, s);
}

}  // namespace gsparc
