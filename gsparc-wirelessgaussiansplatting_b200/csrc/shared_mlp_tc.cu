// Shared emission MLP in BF16 on the 5th-generation tensor cores (tcgen05).
//
// Same network as shared_mlp.cu (features, hidden layers of width 128,
// sigmoid of one output, or of 64 outputs) with BF16 operands and FP32
// accumulation in tensor memory; every layer, the output layer included, is
// an MMA (one output is padded to an N = 16 MMA).  The epilogues between the
// MMAs -- activation, its derivative, the adjoint's product with it -- run in
// packed BF16 arithmetic (two elements per instruction, no conversions:
// the operands the next MMA reads and the stored pre-activations are BF16
// anyway).  Two fused persistent kernels over tiles of 128 (receiver,
// Gaussian) rows, one row per thread of a 128-thread warpgroup:
//
//   forward:  four warpgroups per CTA, each with its own tile in flight and
//             its own 128 TMEM columns; per layer the group's first warp
//             issues the MMAs (one elected lane), the group runs the
//             +bias/activation epilogue.  The
//             weights are staged in shared memory once per CTA; only the BF16
//             pre-activations (for the adjoint) and the signal go to HBM.
//   backward: two compute groups of 256 threads (two per row, 64 columns
//             each), each group with its own tile, and one MMA warp that issues
//             every MMA of the CTA (so all accumulation into the shared
//             weight-gradient columns is in issue order).  Per tile,
//             first the output step
//               dW_out^T += A_{L-1}^T dO,   dA_{L-1} = dO W_out
//             then per hidden layer l (last first):
//               dW_l | db_l += dZ_l^T [A_{l-1} | 1]   (M = 128 outputs, K = the
//                              128 rows; accumulated in TMEM over all tiles)
//               dA_{l-1}     = dZ_l W_l              (M = 128 rows; one
//                              shared scratch accumulator)
//             A_{l-1} = act(Z_{l-1}) and act'(Z_{l-1}) come from one pass over
//             the stored pre-activations (act' is held in registers as BF16
//             pairs until dA arrives).  At the end the CTA adds its TMEM
//             accumulators to the global gradient.
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
constexpr int kBwdGroups = 2;  // backward: compute groups (tiles in flight) per CTA (+ one MMA warp)
constexpr int kBwdHalves = 2;  // backward: threads per row, each with kH / kBwdHalves columns
constexpr int kBwdGroupThreads = 128 * kBwdHalves;
static_assert(kBwdGroupThreads * 64 == kRows * kH, "one 128-byte line of a tile's slab per thread");
constexpr int kBwdThreads = kBwdGroups * kBwdGroupThreads + 32;
constexpr uint32_t kLbo = 128; // core matrices along K are adjacent
constexpr uint32_t kSboX = (kFin / 8) * 128u;         // [rows x 32] K-major
constexpr uint32_t kSboH = (kH / 8) * 128u;           // [rows x 128] K-major
// The adjoint's activation tile [128 rows x 144] (activations | ones) is laid
// out like one stored pre-activation slab -- 8-column chunk k, row t at byte
// k * 2048 + t * 16 -- so a slab lands in it with one bulk copy and is
// activated in place.  As an MN-major operand (N = columns, K = rows) the core
// matrices step 128 bytes along K and 2048 along N.
constexpr uint32_t kChunkA = kRows * 16;   // bytes per 8-column chunk
__host__ __device__ constexpr uint32_t slab_off(int r, int c) {
  return (uint32_t)(c / 8) * kChunkA + (uint32_t)r * 16u + (uint32_t)(c % 8) * 2u;
}
constexpr uint32_t kPolls = 1u << 24;
// N of the output layer's MMA: one output is padded to the smallest N (16)
constexpr int out_mma_width(int out) { return out < 16 ? 16 : out; }
// The forward adds the hidden biases inside the MMAs (a K = 16 tile of ones
// times a hi/lo BF16 split of the bias) where shared memory has room: one
// output (the 64-output W_out takes the space).
constexpr bool fwd_bias_in_mma(int out) { return out == 1; }
// Adjoint TMEM plan: the weight-gradient accumulators with their ones (bias)
// columns, dW_out^T and the 128-column dA scratch must fit 512 columns; when
// they do not, the first layer's bias gradient is summed on the CUDA cores.
constexpr bool bwd_bias0_on_cuda_cores(int layers, int out) {
  return (kFin + 16) + (layers - 1) * (kH + 16) + out_mma_width(out) + kH > 512;
}
constexpr float kPiF = 3.14159265358979323846f;

__device__ __forceinline__ uint32_t pack2(float a, float b) {
  const __nv_bfloat162 h = __floats2bfloat162_rn(a, b);
  return *reinterpret_cast<const uint32_t*>(&h);
}
__device__ __forceinline__ uint4 pack8(const float* v) {
  return make_uint4(pack2(v[0], v[1]), pack2(v[2], v[3]), pack2(v[4], v[5]), pack2(v[6], v[7]));
}

// ---- packed BF16 epilogue arithmetic (two elements per 32-bit register) ----
__device__ __forceinline__ uint32_t bf2_mul(uint32_t a, uint32_t b) {
  uint32_t d;
  asm("mul.rn.bf16x2 %0, %1, %2;" : "=r"(d) : "r"(a), "r"(b));
  return d;
}
__device__ __forceinline__ uint32_t bf2_max(uint32_t a, uint32_t b) {
  uint32_t d;
  asm("max.bf16x2 %0, %1, %2;" : "=r"(d) : "r"(a), "r"(b));
  return d;
}
__device__ __forceinline__ float tanh_approx(float x) {
  float r;
  asm("tanh.approx.f32 %0, %1;" : "=f"(r) : "f"(x));
  return r;
}
// the two BF16 halves of a packed pair as floats (exact)
__device__ __forceinline__ float2 bf2_unpack(uint32_t z) {
  return make_float2(__uint_as_float(z << 16), __uint_as_float(z & 0xFFFF0000u));
}
constexpr uint32_t kBfOne = 0x3F803F80u;   // BF16 1.0 in both halves

// GELU of BF16 pre-activations in the tanh form
//   a = z g,  g = (1 + t) / 2,  t = tanh v,  v = z (c1 + c3 z^2),
// i.e. Phi(z) ~ g, evaluated in FP32 with the hardware tanh and rounded to
// BF16 once.  c1 = 0.80078125 and c3 = 0.034423828125 are fitted to the erf
// GELU z Phi(z): max |a - z Phi(z)| = 3.6e-4 over [-8, 8] (the classic
// sqrt(2/pi), 0.044715 sqrt(2/pi) give 4.7e-4), below the BF16 spacing of the
// activations it feeds.  The adjoint's derivative is the form's own:
//   a' = g + z (1 - t^2) (c1 + 3 c3 z^2) / 2,
// in FP32 (1 - t^2 needs FP32 where t is within a BF16 step of +-1).  One
// special-function evaluation (the tanh) per element in both kernels.
constexpr float kGeluC1 = 0.80078125f, kGeluC3 = 0.034423828125f;
__device__ __forceinline__ float2 gelu_tanh_term(float2 z, float2 zz) {
  const float2 v = fmul2(z, ffma2(zz, make_float2(kGeluC3, kGeluC3), make_float2(kGeluC1, kGeluC1)));
  return make_float2(tanh_approx(v.x), tanh_approx(v.y));
}
__device__ __forceinline__ uint32_t act_fwd2(int act, uint32_t zb) {
  if (act == 1) return bf2_max(zb, 0u);
  const float2 z = bf2_unpack(zb);
  const float2 t = gelu_tanh_term(z, fmul2(z, z));
  const float2 a = fmul2(z, ffma2(t, make_float2(0.5f, 0.5f), make_float2(0.5f, 0.5f)));
  return pack2(a.x, a.y);
}
// act (the forward's, bit for bit) and act' of a pair, both rounded to BF16
__device__ __forceinline__ void act_bwd2(int act, uint32_t zb, uint32_t& a2, uint32_t& d2) {
  if (act == 1) {
    a2 = bf2_max(zb, 0u);
    d2 = __vcmpgts2(zb, 0u) & kBfOne;   // 1 where the BF16 half is > 0 (as a signed 16-bit integer)
    return;
  }
  const float2 z = bf2_unpack(zb);
  const float2 zz = fmul2(z, z);
  const float2 t = gelu_tanh_term(z, zz);
  const float2 g = ffma2(t, make_float2(0.5f, 0.5f), make_float2(0.5f, 0.5f));
  const float2 a = fmul2(z, g);
  const float2 s = ffma2(make_float2(-t.x, -t.y), t, make_float2(1.0f, 1.0f));   // 1 - t^2
  const float2 w = ffma2(zz, make_float2(1.5f * kGeluC3, 1.5f * kGeluC3), make_float2(0.5f * kGeluC1, 0.5f * kGeluC1));
  // (z s) first: s is exactly 0 where t saturates, so w (~z^2) cannot make inf * 0
  const float2 d = ffma2(fmul2(z, s), w, g);
  a2 = pack2(a.x, a.y);
  d2 = pack2(d.x, d.y);
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

// pair_features rounded to BF16 pairs, produced in feature order (octave by
// octave, all three coordinates at once) so that each value is packed as soon
// as it exists; the values are those of pair_features.
__device__ __forceinline__ void pair_features_bf16(const float* __restrict__ means3D, const float* __restrict__ rx_pos,
                                                   int g, int r, bool vis, uint4 (&xp)[kFin / 8]) {
  if (!vis) {
#pragma unroll
    for (int q = 0; q < kFin / 8; ++q) xp[q] = make_uint4(0u, 0u, 0u, 0u);
    return;
  }
  const float m[3] = {means3D[3 * g], means3D[3 * g + 1], means3D[3 * g + 2]};
  float s[3], c[3];
#pragma unroll
  for (int j = 0; j < 3; ++j) sincosf(kPiF * m[j], &s[j], &c[j]);
  uint32_t w[16];
  w[0] = pack2(m[0], m[1]);
  // x[2] = m2, then per octave k: x[3 + 6k + 2j] = sin, x[4 + 6k + 2j] = cos
  float carry = m[2];
#pragma unroll
  for (int k = 0; k < 4; ++k) {
    // the octave's six values x[3 + 6k .. 8 + 6k]; x[2 + 6k] is `carry`
    w[1 + 3 * k] = pack2(carry, s[0]);
    w[2 + 3 * k] = pack2(c[0], s[1]);
    w[3 + 3 * k] = pack2(c[1], s[2]);
    carry = c[2];
#pragma unroll
    for (int j = 0; j < 3; ++j) {
      const float s2 = 2.0f * s[j] * c[j], c2 = fmaf(c[j], c[j], -s[j] * s[j]);
      s[j] = s2;
      c[j] = c2;
    }
  }
  const float v[3] = {m[0] - rx_pos[3 * r], m[1] - rx_pos[3 * r + 1], m[2] - rx_pos[3 * r + 2]};
  const float d2 = v[0] * v[0] + v[1] * v[1] + v[2] * v[2];
  const float d = sqrtf(d2);
  w[13] = pack2(carry, v[0] / d);       // x[26], x[27]
  w[14] = pack2(v[1] / d, v[2] / d);    // x[28], x[29]
  w[15] = pack2(1.0f / d2, 0.0f);       // x[30], x[31]
#pragma unroll
  for (int q = 0; q < kFin / 8; ++q) xp[q] = make_uint4(w[4 * q], w[4 * q + 1], w[4 * q + 2], w[4 * q + 3]);
}

// pair_features of one pair written as BF16 straight into row r of the
// adjoint's activation tile (the slab layout), split between the row's two
// threads: part 0 -- the first two coordinates (x[j] and the sines and
// cosines of their octaves), part 1 -- the third coordinate, the direction and
// the attenuation (x[27..31]).  Every value comes from the FP32 arithmetic of
// pair_features and is rounded to BF16 once; a culled pair's row is zero
// (written by part 0).
__device__ __forceinline__ void store_feature(unsigned char* Ab, int r, int c, float v) {
  *reinterpret_cast<__nv_bfloat16*>(Ab + slab_off(r, c)) = __float2bfloat16_rn(v);
}
// x[j], then per octave k: x[3 + 6k + 2j] = sin, x[4 + 6k + 2j] = cos
__device__ __forceinline__ void coord_features(unsigned char* Ab, int r, int j, float mj) {
  store_feature(Ab, r, j, mj);
  float s, c;
  sincosf(kPiF * mj, &s, &c);
#pragma unroll
  for (int k = 0; k < 4; ++k) {
    store_feature(Ab, r, 3 + 6 * k + 2 * j, s);
    store_feature(Ab, r, 4 + 6 * k + 2 * j, c);
    const float s2 = 2.0f * s * c, c2 = fmaf(c, c, -s * s);
    s = s2;
    c = c2;
  }
}
__device__ __forceinline__ void pair_features_tile(const float* __restrict__ means3D, const float* __restrict__ rx_pos,
                                                   int g, int rr, bool vis, int part, unsigned char* Ab, int r) {
  if (!vis) {
    if (part == 0)
#pragma unroll
      for (int kc = 0; kc < kFin / 8; ++kc) *reinterpret_cast<uint4*>(Ab + slab_off(r, kc * 8)) = make_uint4(0u, 0u, 0u, 0u);
    return;
  }
  const float m[3] = {means3D[3 * g], means3D[3 * g + 1], means3D[3 * g + 2]};
  if (part == 0) {
    coord_features(Ab, r, 0, m[0]);
    coord_features(Ab, r, 1, m[1]);
    return;
  }
  const float v[3] = {m[0] - rx_pos[3 * rr], m[1] - rx_pos[3 * rr + 1], m[2] - rx_pos[3 * rr + 2]};
  coord_features(Ab, r, 2, m[2]);
  const float d2 = v[0] * v[0] + v[1] * v[1] + v[2] * v[2];
  const float d = sqrtf(d2);
  store_feature(Ab, r, 27, v[0] / d);
  store_feature(Ab, r, 28, v[1] / d);
  store_feature(Ab, r, 29, v[2] / d);
  store_feature(Ab, r, 30, 1.0f / d2);
  store_feature(Ab, r, 31, 0.0f);
}

// The chain rule of pair_features for one visible pair: its feature gradient
// dx through the centre, added to dL_dmeans3D[g] by atomics (the rows of a
// tile are distinct Gaussians; a Gaussian's receivers meet in the atomics).
// The coordinates are split between the row's two threads as in
// pair_features_tile (part 0: x and y, part 1: z; part -1: all three, one
// thread); the octaves' sines and cosines come from the same double-angle
// steps as in pair_features.
__device__ __forceinline__ void pair_features_adjoint(const float* __restrict__ means3D,
                                                      const float* __restrict__ rx_pos, int g, int r,
                                                      const float (&dx)[kFin], int part,
                                                      float* __restrict__ dL_dmeans3D) {
  const float m[3] = {means3D[3 * g], means3D[3 * g + 1], means3D[3 * g + 2]};
  const float v[3] = {m[0] - rx_pos[3 * r], m[1] - rx_pos[3 * r + 1], m[2] - rx_pos[3 * r + 2]};
  const float d2 = v[0] * v[0] + v[1] * v[1] + v[2] * v[2];
  const float d = sqrtf(d2);
  const float u[3] = {v[0] / d, v[1] / d, v[2] / d};
  // direction u = v / d: du_i/dv_j = (delta_ij - u_i u_j) / d;  1 / d^2: d/dv = -2 v / d^4
  const float gu = dx[27] * u[0] + dx[28] * u[1] + dx[29] * u[2];
  const float ga = dx[30] * (-2.0f / (d2 * d2));
  auto coord = [&](int j) {
    float gj = dx[j] + (dx[27 + j] - gu * u[j]) / d + ga * v[j];
    float s, c;
    sincosf(kPiF * m[j], &s, &c);
    float w = kPiF;
#pragma unroll
    for (int k = 0; k < 4; ++k) {
      gj += w * (c * dx[3 + 6 * k + 2 * j] - s * dx[4 + 6 * k + 2 * j]);
      const float s2 = 2.0f * s * c, c2 = fmaf(c, c, -s * s);
      s = s2;
      c = c2;
      w *= 2.0f;
    }
    atomicAdd(&dL_dmeans3D[3 * g + j], gj);
  };
  if (part != 1) {   // part 0 (or -1: all three coordinates)
    coord(0);
    coord(1);
  }
  if (part != 0) coord(2);
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

// Sum 16 per-lane values over the warp: returns, in lane j < 16, the sum of value j.
__device__ __forceinline__ float warp_transpose_sum16(float (&v)[16], int lane) {
#pragma unroll
  for (int half = 8; half >= 1; half >>= 1) {
    const bool upper = lane & half;
#pragma unroll
    for (int i = 0; i < half; ++i) {
      const float send = upper ? v[i] : v[i + half];
      const float keep = upper ? v[i + half] : v[i];
      v[i] = keep + __shfl_xor_sync(0xffffffffu, send, half);
    }
  }
  return v[0] + __shfl_xor_sync(0xffffffffu, v[0], 16);
}

// Warpgroup-local ordering of generic shared-memory writes and TMEM reads
// before the group's first warp issues MMAs that read / overwrite them.
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
// whose first 8 KB also hold the feature tile X [128 x 32]; the hidden biases
// and the output biases in fp32; W_out K-major [kOutMma x 128] bf16 (rows past
// the real outputs zero).  With one output the hidden biases also enter the
// MMAs: a shared K = 16 tile of ones [128 x 16] (columns 0 and 1 one) times a
// bias tile per layer [128 x 16] (column 0 the bias rounded to BF16, column 1
// the BF16 remainder), so the epilogue adds nothing (64 outputs leave no
// room for the 16 KB).
template <int kLayers, int act, int kOut>
__global__ void __launch_bounds__(128 * kFwdGroups, 1)
mlp_bf16_forward_kernel(int P, size_t rows, const float* __restrict__ means3D,
                        const float* __restrict__ rx_pos, const float* __restrict__ params,
                        const int* __restrict__ radii, __nv_bfloat16* __restrict__ zb, float* __restrict__ S,
                        float2* __restrict__ signal, ImageHeader* __restrict__ hdr, uint32_t polls) {
  constexpr int kOutMma = out_mma_width(kOut);
  constexpr bool kBiasMma = fwd_bias_in_mma(kOut);
  constexpr uint32_t kSboK16 = 2u * 128u;   // [rows x 16] K-major
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
  unsigned char* ones = smem + off;                      // kBiasMma: [128 x 16], then the bias tiles
  unsigned char* Bt = ones + kRows * 16 * 2;
  if (kBiasMma) off += (size_t)kRows * 16 * 2 + (size_t)kLayers * kH * 16 * 2;
  float* bias = reinterpret_cast<float*>(smem + off);   // [kLayers][128], then b_out[kOut]
  float* bout = bias + kLayers * kH;
  off += (size_t)(kLayers * kH + kH + 4) * sizeof(float);
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
    for (int j = tid; j < kH; j += blockDim.x) {
      const float b = params[poff + j];
      bias[l * kH + j] = b;
      if (kBiasMma) {
        const __nv_bfloat16 hi = __float2bfloat16_rn(b);
        const __nv_bfloat16 lo = __float2bfloat16_rn(b - __bfloat162float(hi));
        unsigned char* bt = Bt + (size_t)l * kH * 16 * 2;
        const uint32_t row2 = (uint32_t)__bfloat16_as_ushort(hi) | ((uint32_t)__bfloat16_as_ushort(lo) << 16);
        *reinterpret_cast<uint4*>(bt + tc::kmajor_off(j, 0, kLbo, kSboK16)) = make_uint4(row2, 0u, 0u, 0u);
        *reinterpret_cast<uint4*>(bt + tc::kmajor_off(j, 8, kLbo, kSboK16)) = make_uint4(0u, 0u, 0u, 0u);
      }
    }
    poff += kH;
  }
  if (kBiasMma)
    for (int r = tid; r < kRows; r += blockDim.x) {
      *reinterpret_cast<uint4*>(ones + tc::kmajor_off(r, 0, kLbo, kSboK16)) = make_uint4(pack2(1.0f, 1.0f), 0u, 0u, 0u);
      *reinterpret_cast<uint4*>(ones + tc::kmajor_off(r, 8, kLbo, kSboK16)) = make_uint4(0u, 0u, 0u, 0u);
    }
  for (int c = tid; c < kOutMma * (kH / 8); c += blockDim.x) {
    const int n = c / (kH / 8), kc = c % (kH / 8);
    float v[8];
#pragma unroll
    for (int i = 0; i < 8; ++i) v[i] = n < kOut ? params[poff + (size_t)n * kH + kc * 8 + i] : 0.0f;
    *reinterpret_cast<uint4*>(Wo + tc::kmajor_off(n, kc * 8, kLbo, kSboH)) = pack8(v);
  }
  for (int j = tid; j < kOut; j += blockDim.x) bout[j] = params[poff + (size_t)kOut * kH + j];
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
  const size_t fwd_stride = (size_t)gridDim.x * kFwdGroups;
  for (size_t tile = (size_t)blockIdx.x * kFwdGroups + grp; tile < ntiles; tile += fwd_stride) {
    const size_t row0 = tile * kRows, row = row0 + t;
    const bool valid = row < rows;
    if (t == 0 && tile + fwd_stride < ntiles) {
      // the next tile's radii and Gaussian centres into L2 (its rows are
      // consecutive Gaussians of at most two receivers)
      const size_t r1 = (tile + fwd_stride) * kRows;
      const uint32_t n1 = (uint32_t)(rows - r1 < (size_t)kRows ? rows - r1 : (size_t)kRows);
      tc::prefetch_l2(radii + r1, n1 * 4);
      // centres [gs, ge) of the tile's first receiver, gs rounded down to a
      // 16-byte boundary, ge <= P (the range stays inside the buffer)
      const size_t g1 = r1 % (size_t)P, gs = g1 & ~(size_t)3;
      const size_t ge = (size_t)P - g1 < (size_t)n1 ? (size_t)P : g1 + n1;
      tc::prefetch_l2(means3D + 3 * gs, (uint32_t)((ge - gs) * 12));
    }
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
    // hidden layers, then the output layer (l == kLayers)
    for (int l = 0; l <= kLayers; ++l) {
      const bool out_layer = l == kLayers;
      group_publish(bar_id);
      if (t < 32) {
        // the group's first warp issues the layer's MMAs (one elected lane, unrolled)
        const uint32_t a0 = tc::smem_u32(Hs), b0 = tc::smem_u32(out_layer ? Wo : Ws[l]);
        const uint32_t idesc = tc::idesc_bf16(kRows, out_layer ? kOutMma : kH, false, false);
        if (l == 0) {
          constexpr uint32_t sbo = (uint32_t)(kFin / 8) * 128u;
#pragma unroll
          for (int kk = 0; kk < kFin / 16; ++kk)
            tc::mma_bf16_warp(tmem, tc::smem_desc(a0 + kk * 2 * kLbo, kLbo, sbo),
                              tc::smem_desc(b0 + kk * 2 * kLbo, kLbo, sbo), idesc, kk > 0 ? 1u : 0u);
        } else {
          constexpr uint32_t sbo = (uint32_t)(kH / 8) * 128u;
#pragma unroll
          for (int kk = 0; kk < kH / 16; ++kk)
            tc::mma_bf16_warp(tmem, tc::smem_desc(a0 + kk * 2 * kLbo, kLbo, sbo),
                              tc::smem_desc(b0 + kk * 2 * kLbo, kLbo, sbo), idesc, kk > 0 ? 1u : 0u);
        }
        if (kBiasMma && !out_layer)   // + 1 * b_hi + 1 * b_lo
          tc::mma_bf16_warp(tmem, tc::smem_desc(tc::smem_u32(ones), kLbo, kSboK16),
                            tc::smem_desc(tc::smem_u32(Bt) + (uint32_t)(l * kH * 16 * 2), kLbo, kSboK16), idesc, 1u);
        tc::commit_warp(&mbar[grp]);
      }
      const bool got = tc::mbar_wait(&mbar[grp], phase, polls);
      phase ^= 1u;
      tc::fence_after_sync();
      if (!tc::named_all(bar_id, 128, got)) {
        ok = false;
        break;
      }
      if (out_layer) break;
      // z = acc + b rounded to BF16 (stored for the adjoint), a = act(z) in BF16
      // -> the next layer's operand tile
      __nv_bfloat16* z_out = zb + z_row_base(zrows, l, tile, t);
      const float* bl = bias + l * kH;
#pragma unroll 1
      for (int c0 = 0; c0 < kH; c0 += 32) {
        float v[32];
        tc::tmem_ld32(tmem + lane_base + c0, v);
#pragma unroll
        for (int q = 0; q < 4; ++q) {
          float2 z0 = make_float2(v[q * 8 + 0], v[q * 8 + 1]), z1 = make_float2(v[q * 8 + 2], v[q * 8 + 3]);
          float2 z2 = make_float2(v[q * 8 + 4], v[q * 8 + 5]), z3 = make_float2(v[q * 8 + 6], v[q * 8 + 7]);
          if constexpr (!kBiasMma) {
            const float4 b0 = *reinterpret_cast<const float4*>(bl + c0 + q * 8);
            const float4 b1 = *reinterpret_cast<const float4*>(bl + c0 + q * 8 + 4);
            z0 = fadd2(z0, make_float2(b0.x, b0.y));
            z1 = fadd2(z1, make_float2(b0.z, b0.w));
            z2 = fadd2(z2, make_float2(b1.x, b1.y));
            z3 = fadd2(z3, make_float2(b1.z, b1.w));
          }
          const uint4 zp = make_uint4(pack2(z0.x, z0.y), pack2(z1.x, z1.y), pack2(z2.x, z2.y), pack2(z3.x, z3.y));
          if (valid) *reinterpret_cast<uint4*>(z_out + (size_t)((c0 + q * 8) / 8) * kZChunk) = zp;
          const uint4 ap = make_uint4(act_fwd2(act, zp.x), act_fwd2(act, zp.y), act_fwd2(act, zp.z),
                                      act_fwd2(act, zp.w));
          *reinterpret_cast<uint4*>(Hs + tc::kmajor_off(t, c0 + q * 8, kLbo, kSboH)) = ap;
        }
      }
    }
    if (!ok) break;
    // output layer [128 rows x kOutMma] in the group's TMEM columns: sigmoid(acc + b_out)
    if constexpr (kOut == 1) {
      const float o = tc::tmem_ld1(tmem + lane_base);
      if (valid) {
        const float s = 1.0f / (1.0f + expf(-(o + bout[0])));
        S[row] = s;
        if (vis) signal[row] = make_float2(s, 0.0f);
      }
    } else {
#pragma unroll 1
      for (int c0 = 0; c0 < kOut; c0 += 32) {
        float v[32];
        tc::tmem_ld32(tmem + lane_base + c0, v);
#pragma unroll
        for (int i = 0; i < 32; ++i) v[i] = 1.0f / (1.0f + expf(-(v[i] + bout[c0 + i])));
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
    // drain: the MMAs the group's issuing lane committed last (the phase the
    // group gave up on) complete before the tensor memory is freed
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
// both K-major by row; W_out as the MN-major B operand of dA = dO W_out
// ([n = 128] x [k = kOutMma]; rows past the real outputs zero).
// TMEM columns: dW_l accumulators of in_l (+ 16) columns each (last layer
// first; the ones columns give db_l, except for the first layer when the
// columns run short -- 3 hidden layers and 64 outputs -- whose bias is then
// summed on the CUDA cores), then dW_out^T (kOutMma columns, lanes = hidden
// units), then one 128-column scratch accumulator for dA.  Every tile starts
// with the output step: dW_out^T += A_{L-1}^T dO and dA_{L-1} = dO W_out,
// dO staged as a K-major row tile in the dZ buffer.
template <int kLayers, int act, int kOut>
__global__ void __launch_bounds__(kBwdThreads, 1)
mlp_bf16_backward_kernel(int P, size_t rows, const float* __restrict__ means3D,
                         const float* __restrict__ rx_pos, const float* __restrict__ params,
                         const int* __restrict__ radii, const __nv_bfloat16* __restrict__ zb,
                         const float* __restrict__ S, const float* __restrict__ dL_dsignal,
                         float* __restrict__ dL_dmeans3D, float* __restrict__ dparams, ImageHeader* __restrict__ hdr,
                         uint32_t polls) {
  constexpr int kOutMma = out_mma_width(kOut);
  constexpr bool kBias0Cuda = bwd_bias0_on_cuda_cores(kLayers, kOut);
  // the last step's features and feature adjoint split between a row's two
  // threads (one output: 2.84 -> 2.66 ms at 6.4 M rows); with 64 outputs one
  // thread per row measured faster (1.20 against 1.28 ms at 1.6 M rows)
  constexpr bool kSplitFeatures = kOut == 1;
  extern __shared__ __align__(1024) unsigned char smem[];
  __shared__ __align__(8) uint64_t bar_ready[kBwdGroups];
  __shared__ __align__(8) uint64_t bar_done[kBwdGroups];
  __shared__ __align__(8) uint64_t bar_free;
  __shared__ __align__(8) uint64_t bar_drain;
  __shared__ __align__(8) uint64_t bar_z[kBwdGroups];   // a pre-activation slab has landed
  __shared__ __align__(8) uint64_t bar_afree[kBwdGroups];  // a step's MMAs reading the activation tile are done
  __shared__ uint32_t tbase;
  __shared__ int s_fail;
  // db_out[kOut], then (kBias0Cuda) db_0[128]
  constexpr int kRed = kOut + (kBias0Cuda ? kH : 0);
  __shared__ float s_red[kRed];
  constexpr uint32_t kSboO = (uint32_t)(kOutMma / 8) * 128u;   // [rows x kOutMma] K-major / W_out MN-major
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int grp = tid / kBwdGroupThreads;   // compute group 0..kBwdGroups-1; kBwdGroups = the MMA warp
  const int t = tid % kBwdGroupThreads;
  const int r = t & 127;                    // the thread's row of the tile (its TMEM lane)
  const int hf = t >> 7;                    // which half of the row's columns (uniform per warp)
  constexpr int kHc = kH / kBwdHalves;      // columns per thread
  constexpr size_t kGroupBytes = (size_t)kRows * kH * 2 + (size_t)kRows * (kH + 16) * 2;
  unsigned char* Wb[kLayers];
  size_t off = 0;
  for (int l = 0; l < kLayers; ++l) {
    Wb[l] = smem + off;
    off += (size_t)(l == 0 ? kFin : kH) * kH * 2;
  }
  unsigned char* const groups = smem + off;
  off += kBwdGroups * kGroupBytes;
  unsigned char* const Wo = smem + off;

  // offsets in the flat parameters of W_l and b_l (l == kLayers: the output
  // layer), recomputed where needed rather than held in registers
  auto woff = [](int l) -> size_t {
    return l == 0 ? 0 : (size_t)(kFin * kH + kH) + (size_t)(l - 1) * (kH * kH + kH);
  };
  auto boff = [&](int l) -> size_t { return woff(l) + (size_t)kH * (l == kLayers ? kOut : (l == 0 ? kFin : kH)); };
  // W_l [out][in] -> MN-major B operand (n = in, k = out), once per CTA
  for (int l = 0; l < kLayers; ++l) {
    const int in = l == 0 ? kFin : kH;
    const float* W = params + woff(l);
    for (int c = tid; c < kH * (in / 8); c += blockDim.x) {
      const int k = c / (in / 8), nc = c % (in / 8);   // k = output row of W, nc = group of 8 inputs
      float v[8];
#pragma unroll
      for (int i = 0; i < 8; ++i) v[i] = W[(size_t)k * in + nc * 8 + i];
      *reinterpret_cast<uint4*>(Wb[l] + tc::mnmajor_off(nc * 8, k, kLbo, kSboH)) = pack8(v);
    }
  }
  const size_t poff = woff(kLayers);
  for (int c = tid; c < kOutMma * (kH / 8); c += blockDim.x) {
    const int k = c / (kH / 8), nc = c % (kH / 8);   // k = output row of W_out, nc = group of 8 hidden units
    float v[8];
#pragma unroll
    for (int i = 0; i < 8; ++i) v[i] = k < kOut ? params[poff + (size_t)k * kH + nc * 8 + i] : 0.0f;
    *reinterpret_cast<uint4*>(Wo + tc::mnmajor_off(nc * 8, k, kLbo, kSboO)) = pack8(v);
  }
  for (int j = tid; j < kRed; j += blockDim.x) s_red[j] = 0.0f;
  unsigned char* const dZ = groups + (size_t)(grp < kBwdGroups ? grp : 0) * kGroupBytes;
  unsigned char* const Ab = dZ + (size_t)kRows * kH * 2;
  if (grp < kBwdGroups && hf == 0) {   // the constant ones column (db) of the activation tile
    const uint4 one = make_uint4(pack2(1.0f, 0.0f), 0u, 0u, 0u);
    *reinterpret_cast<uint4*>(Ab + slab_off(r, kH)) = one;
    *reinterpret_cast<uint4*>(Ab + slab_off(r, kH + 8)) = make_uint4(0u, 0u, 0u, 0u);
  }
  if (tid == 0) {
    for (int q = 0; q < kBwdGroups; ++q) {
      tc::mbar_init(&bar_ready[q], kBwdGroupThreads);
      tc::mbar_init(&bar_done[q], 1);
      tc::mbar_init(&bar_z[q], 1);
      tc::mbar_init(&bar_afree[q], 1);
    }
    tc::mbar_init(&bar_free, kBwdGroupThreads);
    tc::mbar_init(&bar_drain, 1);
    s_fail = 0;
  }
  if (warp == 0) tc::tmem_alloc(&tbase, 512);
  tc::fence_async_smem();
  tc::fence_before_sync();
  __syncthreads();
  tc::fence_after_sync();
  const uint32_t tmem = tbase;
  // TMEM columns: dW_l (last layer first), dW_out^T, the dA scratch
  auto dw_width = [](int l) { return (l == 0 ? kFin : kH) + ((l == 0 && kBias0Cuda) ? 0 : 16); };
  auto dwcol = [](int l) -> uint32_t { return (uint32_t)(kLayers - 1 - l) * (kH + 16); };
  constexpr uint32_t dwo_col = (uint32_t)(kLayers - 1) * (kH + 16) + kFin + (kBias0Cuda ? 0 : 16);
  constexpr uint32_t scratch = dwo_col + kOutMma;   // + 128 <= 512 (bwd_bias0_on_cuda_cores)
  const size_t ntiles = (rows + kRows - 1) / kRows;
  const size_t zrows = ntiles * kRows;   // pre-activation rows, whole tiles
  const size_t tile_stride = (size_t)gridDim.x * kBwdGroups;

  if (grp == kBwdGroups) {
    // ---- MMA warp: the whole warp walks the schedule and one elected lane
    // issues every MMA and commit of the CTA, in the order (tile round, step,
    // group), so both groups' weight gradients accumulate into the same TMEM
    // columns in issue order.  The K loops are unrolled (uniform descriptors).
    constexpr uint32_t kAll = 0xffffffffu;
    uint32_t ph_ready[kBwdGroups] = {};
    bool first[kLayers + 1];
    for (int l = 0; l <= kLayers; ++l) first[l] = true;
    uint32_t n_da = 0;
    bool ok = true;
    for (size_t base = (size_t)blockIdx.x * kBwdGroups; base < ntiles && ok; base += tile_stride) {
#pragma unroll 1
      for (int l = kLayers; l >= 0 && ok; --l) {
        const bool out_step = l == kLayers;
        const int in = l == 0 ? kFin : kH;
#pragma unroll 1
        for (int q = 0; q < kBwdGroups; ++q) {
          if (base + q >= ntiles) break;
          if (!__all_sync(kAll, tc::mbar_wait(&bar_ready[q], ph_ready[q], polls))) {
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
            const uint32_t id_o = tc::idesc_bf16(kH, kOutMma, true, true);
#pragma unroll
            for (int kk = 0; kk < kRows / 16; ++kk)
              tc::mma_bf16_warp(tmem + dwo_col, tc::smem_desc(aq + kk * 256u, 128u, kChunkA),
                                tc::smem_desc(zq + kk * 2 * kSboO, kSboO, 128u), id_o,
                                (!first[kLayers] || kk > 0) ? 1u : 0u);
            first[kLayers] = false;
          } else {
            // dW_l | db_l += dZ^T [A | 1]: A operand dZ^T (M = outputs, K = rows) and
            // B operand [A | 1]^T (N = in (+ 16), K = rows), both MN-major views of the
            // row tiles
            const uint32_t id_w = tc::idesc_bf16(kH, dw_width(l), true, true);
            const uint32_t dcol = tmem + dwcol(l);
            const uint32_t acc0 = first[l] ? 0u : 1u;
#pragma unroll
            for (int kk = 0; kk < kRows / 16; ++kk)
              tc::mma_bf16_warp(dcol, tc::smem_desc(zq + kk * 2 * kSboH, kSboH, 128u),
                                tc::smem_desc(aq + kk * 256u, 128u, kChunkA), id_w, kk > 0 ? 1u : acc0);
            first[l] = false;
          }
          // the activation tile is read: the group may stage the next slab into it
          tc::commit_warp(&bar_afree[q]);
          // dA = dZ_l W_l (or dO W_out) into the scratch, once its previous reader has drained it
          if (n_da > 0) {
            if (!__all_sync(kAll, tc::mbar_wait(&bar_free, (n_da - 1) & 1u, polls))) {
              ok = false;
              break;
            }
            tc::fence_after_sync();
          }
          if (out_step) {
            const uint32_t id_x = tc::idesc_bf16(kRows, kH, false, true);
            const uint32_t wo = tc::smem_u32(Wo);
#pragma unroll
            for (int kk = 0; kk < kOutMma / 16; ++kk)
              tc::mma_bf16_warp(tmem + scratch, tc::smem_desc(zq + kk * 2 * kLbo, kLbo, kSboO),
                                tc::smem_desc(wo + kk * 2 * kLbo, kLbo, kSboO), id_x, kk > 0 ? 1u : 0u);
          } else {
            const uint32_t id_x = tc::idesc_bf16(kRows, in, false, true);
            const uint32_t wb = tc::smem_u32(Wb[l]);
#pragma unroll
            for (int kk = 0; kk < kH / 16; ++kk)
              tc::mma_bf16_warp(tmem + scratch, tc::smem_desc(zq + kk * 2 * kLbo, kLbo, kSboH),
                                tc::smem_desc(wb + kk * 2 * kLbo, kLbo, kSboH), id_x, kk > 0 ? 1u : 0u);
          }
          ++n_da;
          tc::commit_warp(&bar_done[q]);
        }
      }
    }
    if (!ok && lane == 0) s_fail = 1;
  } else {
    // ---- compute group: thread (r, hf) handles row r, columns [hf kHc, hf kHc + kHc)
    const uint32_t lane_base = (uint32_t)((warp & 3) * 32) << 16;
    const uint32_t bar_id = 1u + (uint32_t)grp;
    const int cb = hf * kHc;
    uint32_t ph_done = 0, ph_z = 0;
    bool ok = true, z_pending = false;
    // one pre-activation slab (layer l of a tile, 32 KB) -> the activation
    // tile, by the group's first thread once the MMAs reading the tile are done
    auto stage_slab = [&](int l, size_t tl) {
      if (t == 0) {
        tc::mbar_arrive_expect_tx(&bar_z[grp], kRows * kH * 2);
        tc::bulk_load(Ab, zb + z_row_base(zrows, l, tl, 0), kRows * kH * 2, &bar_z[grp]);
        z_pending = true;
      }
    };
    // a row's visibility and (one output) its dO = dL/dsignal s (1 - s), loaded
    // a step ahead (the next tile's during this tile's last MMAs)
    auto load_row = [&](size_t rw, bool& vis_out) -> float {
      vis_out = rw < rows && radii[rw] > 0;
      if (kOut != 1 || hf != 0 || !vis_out) return 0.0f;
      const float sg = S[rw];
      return dL_dsignal[2 * rw] * sg * (1.0f - sg);
    };
    const size_t tile0 = (size_t)blockIdx.x * kBwdGroups + grp;
    bool vis_n = false;
    float dO_n = 0.0f;
    if (tile0 < ntiles) {
      stage_slab(kLayers - 1, tile0);
      dO_n = load_row(tile0 * kRows + r, vis_n);
    }
    for (size_t tile = tile0; tile < ntiles && ok; tile += tile_stride) {
      const size_t row0 = tile * kRows, row = row0 + r;
      const bool valid = row < rows;
      const bool vis = vis_n;
      if (t == 0 && tile + tile_stride < ntiles) {
        // the next tile's pre-activation slabs, outputs, radii and incoming gradients into L2
        for (int l = kLayers - 1; l >= 0; --l)
          tc::prefetch_l2(zb + z_row_base(zrows, l, tile + tile_stride, 0), kRows * kH * 2);
        const size_t r1 = (tile + tile_stride) * kRows;
        const uint32_t n1 = (uint32_t)(rows - r1 < (size_t)kRows ? rows - r1 : (size_t)kRows);
        tc::prefetch_l2(S + r1 * kOut, n1 * 4 * kOut);
        tc::prefetch_l2(radii + r1, n1 * 4);
        tc::prefetch_l2(dL_dsignal + (kOut > 1 ? r1 * kOut : 2 * r1), n1 * (kOut > 1 ? 4 * kOut : 8));
      }
      // dO -> the dO row tile (BF16) in the dZ buffer; db_out sums it in FP32
      if constexpr (kOut == 1) {
        if (hf == 0) {
          const float dO = dO_n;
          *reinterpret_cast<uint4*>(dZ + tc::kmajor_off(r, 0, kLbo, kSboO)) =
              make_uint4(pack2(dO, 0.0f), 0u, 0u, 0u);
          *reinterpret_cast<uint4*>(dZ + tc::kmajor_off(r, 8, kLbo, kSboO)) = make_uint4(0u, 0u, 0u, 0u);
          float dsum = dO;
#pragma unroll
          for (int o = 16; o > 0; o >>= 1) dsum += __shfl_xor_sync(0xffffffffu, dsum, o);
          if (lane == 0) atomicAdd(&s_red[0], dsum);
        }
      } else {
        constexpr int kOc = kOut / kBwdHalves;   // outputs per thread (a multiple of 32)
#pragma unroll 1
        for (int c0 = hf * kOc; c0 < hf * kOc + kOc; c0 += 32) {
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
            *reinterpret_cast<uint4*>(dZ + tc::kmajor_off(r, c0 + q * 8, kLbo, kSboO)) = pack8(d + q * 8);
          const float sum = warp_transpose_sum32(d, lane);
          atomicAdd(&s_red[c0 + lane], sum);
        }
      }
#pragma unroll 1
      for (int l = kLayers; l >= 0; --l) {
        // act'(Z_{l-1}) of this row's columns as BF16 pairs, kept for dZ_{l-1}
        // after the MMAs
        uint32_t ad[kHc / 2];
        if (l == 0) {
          // A_{-1}: the row's features (BF16; the row's two threads split them),
          // then the ones column (not for the layer whose bias is summed on the
          // CUDA cores).  Forming them while
          // step 1's MMAs ran was slower (3.20 -> 3.72 ms at 6.4 M rows): the
          // features' registers beside act' spilled in the per-step code.
          if constexpr (kSplitFeatures) {
            int rr, g;
            row_pair(row0, r, P, rr, g);
            pair_features_tile(means3D, rx_pos, g, rr, vis, hf, Ab, r);
          } else if (hf == 0) {
            int rr, g;
            row_pair(row0, r, P, rr, g);
            uint4 xp[kFin / 8];
            pair_features_bf16(means3D, rx_pos, g, rr, vis, xp);
#pragma unroll
            for (int kc = 0; kc < kFin / 8; ++kc) *reinterpret_cast<uint4*>(Ab + slab_off(r, kc * 8)) = xp[kc];
          }
          if constexpr (!kBias0Cuda) {
            if (hf == 1) {
              *reinterpret_cast<uint4*>(Ab + slab_off(r, kFin)) = make_uint4(pack2(1.0f, 0.0f), 0u, 0u, 0u);
              *reinterpret_cast<uint4*>(Ab + slab_off(r, kFin + 8)) = make_uint4(0u, 0u, 0u, 0u);
            }
          }
        }
        if (l > 0) {
          // Z_{l-1} of the tile, staged in the activation tile by a bulk copy:
          // activate it in place (rows past the end read as zero)
          const bool zgot = tc::mbar_wait(&bar_z[grp], ph_z, polls);
          if (zgot) {
            ph_z ^= 1u;
            z_pending = false;
          }
          if (!tc::named_all(bar_id, kBwdGroupThreads, zgot)) {
            ok = false;
            break;
          }
#pragma unroll
          for (int k = 0; k < kHc / 8; ++k) {
            uint4* cell = reinterpret_cast<uint4*>(Ab + slab_off(r, cb + 8 * k));
            const uint4 zq = valid ? *cell : make_uint4(0u, 0u, 0u, 0u);
            const uint32_t zk[4] = {zq.x, zq.y, zq.z, zq.w};
            uint32_t a[4];
#pragma unroll
            for (int j = 0; j < 4; ++j) act_bwd2(act, zk[j], a[j], ad[4 * k + j]);
            *cell = make_uint4(a[0], a[1], a[2], a[3]);
          }
        }
        // hand dZ_l (or dO) and A_{l-1} to the MMA warp
        tc::fence_async_smem();
        tc::mbar_arrive(&bar_ready[grp]);
        bool afree = true;
        if (t == 0 && (l >= 2 || (l == 0 && tile + tile_stride < ntiles))) {
          // once the weight-gradient MMA has read the activation tile (before dA
          // is computed), stage the slab the next step activates into it
          afree = tc::mbar_wait(&bar_afree[grp], ph_done, polls);
          if (afree) {
            if (l >= 2) stage_slab(l - 2, tile);
            else stage_slab(kLayers - 1, tile + tile_stride);
          }
        }
        if (l == 0 && tile + tile_stride < ntiles) dO_n = load_row((tile + tile_stride) * kRows + r, vis_n);
        const bool got = tc::mbar_wait(&bar_done[grp], ph_done, polls);
        ph_done ^= 1u;
        tc::fence_after_sync();
        if (!tc::named_all(bar_id, kBwdGroupThreads, got && afree)) {
          ok = false;
          break;
        }
        if (l == 0) {
          // dL/dx of the row, then through the features into dL/dmeans3D
          // (with kSplitFeatures the coordinates are split between the row's
          // two threads, else the first takes all three)
          if (kSplitFeatures || hf == 0) {
            float v[32];
            tc::tmem_ld32(tmem + lane_base + scratch, v);
            tc::fence_before_sync();
            tc::mbar_arrive(&bar_free);
            if (vis && dL_dmeans3D != nullptr) {
              int rr, g;
              row_pair(row0, r, P, rr, g);
              pair_features_adjoint(means3D, rx_pos, g, rr, v, kSplitFeatures ? hf : -1, dL_dmeans3D);
            }
          } else {
            tc::fence_before_sync();
            tc::mbar_arrive(&bar_free);
          }
        } else {
          // dZ_{l-1} = BF16(dA_{l-1}) * act'(Z_{l-1}) in BF16, 32 columns (two TMEM loads, one
          // wait) at a time; the MMAs that read dZ_l (or dO) are done
          auto form_dz = [&](float (&v)[16], int c) {
            const int c0 = cb + 16 * c;
            uint32_t p[8];
#pragma unroll
            for (int i = 0; i < 8; ++i) p[i] = bf2_mul(pack2(v[2 * i], v[2 * i + 1]), ad[8 * c + i]);
            *reinterpret_cast<uint4*>(dZ + tc::kmajor_off(r, c0, kLbo, kSboH)) = make_uint4(p[0], p[1], p[2], p[3]);
            *reinterpret_cast<uint4*>(dZ + tc::kmajor_off(r, c0 + 8, kLbo, kSboH)) =
                make_uint4(p[4], p[5], p[6], p[7]);
            if (kBias0Cuda && l == 1) {
              // db_0 sums the BF16 dZ_0 the MMAs see (16 columns: half a warp transpose)
#pragma unroll
              for (int i = 0; i < 8; ++i) {
                const float2 f = bf2_unpack(p[i]);
                v[2 * i] = f.x;
                v[2 * i + 1] = f.y;
              }
              const float sum = warp_transpose_sum16(v, lane);
              if (lane < 16) atomicAdd(&s_red[kOut + c0 + lane], sum);
            }
          };
#pragma unroll
          for (int c = 0; c < kHc / 16; c += 2) {
            float v0[16], v1[16];
            tc::tmem_ld16x2(tmem + lane_base + scratch + cb + 16 * c, tmem + lane_base + scratch + cb + 16 * c + 16,
                            v0, v1);
            if (c + 2 == kHc / 16) {
              tc::fence_before_sync();
              tc::mbar_arrive(&bar_free);
            }
            form_dz(v0, c);
            form_dz(v1, c + 1);
          }
        }
      }
    }
    if (!ok && t == 0) {
      s_fail = 1;
      // a slab copy still in flight lands before the CTA's shared memory goes away
      if (z_pending) tc::mbar_wait(&bar_z[grp], ph_z, kPolls);
    }
  }
  __syncthreads();
  tc::fence_after_sync();
  // the CTA's weight and bias gradients -> global (rows of dW_l are TMEM lanes);
  // (layer, 32-column chunk) items are split over the compute warpgroups
  if (!s_fail && grp < kBwdGroups) {
    const uint32_t lane_base = (uint32_t)((warp & 3) * 32) << 16;
    const int part = grp * kBwdHalves + hf, nparts = kBwdGroups * kBwdHalves;
    int item = 0;
    for (int l = 0; l < kLayers; ++l) {
      const int in = l == 0 ? kFin : kH;
      const int ncols = (l == 0 && kBias0Cuda) ? in : in + 1;   // weights, then the bias column
#pragma unroll 1
      for (int c0 = 0; c0 < ncols; c0 += 32, ++item) {
        if (item % nparts != part) continue;
        float v[32];
        tc::tmem_ld32(tmem + lane_base + dwcol(l) + c0, v);
#pragma unroll
        for (int i = 0; i < 32; ++i) {
          const int n = c0 + i;
          if (n < in) atomicAdd(&dparams[woff(l) + (size_t)r * in + n], v[i]);
          else if (n == in && n < ncols) atomicAdd(&dparams[boff(l) + r], v[i]);
        }
      }
    }
    // dW_out^T: lane = hidden unit t, column = output
    if constexpr (kOut == 1) {
      if (item % nparts == part) atomicAdd(&dparams[woff(kLayers) + r], tc::tmem_ld1(tmem + lane_base + dwo_col));
      ++item;
    } else {
#pragma unroll 1
      for (int c0 = 0; c0 < kOut; c0 += 32, ++item) {
        if (item % nparts != part) continue;
        float v[32];
        tc::tmem_ld32(tmem + lane_base + dwo_col + c0, v);
#pragma unroll
        for (int i = 0; i < 32; ++i) atomicAdd(&dparams[woff(kLayers) + (size_t)(c0 + i) * kH + r], v[i]);
      }
    }
    if (grp == 0) {
      for (int j = t; j < kOut; j += kBwdGroupThreads) atomicAdd(&dparams[boff(kLayers) + j], s_red[j]);
      if constexpr (kBias0Cuda)
        for (int j = t; j < kH; j += kBwdGroupThreads) atomicAdd(&dparams[boff(0) + j], s_red[kOut + j]);
    }
  }
  if (s_fail && tid == 0 && hdr) atomic_or_error(hdr, kErrMlpWait);
  if (s_fail && grp == kBwdGroups) {
    // drain: every MMA the MMA warp's issuing lane started completes before
    // the tensor memory is freed
    tc::commit_warp(&bar_drain);
    tc::mbar_wait(&bar_drain, 0, kPolls);
  }
  tc::fence_before_sync();
  __syncthreads();
  if (warp == 0) tc::tmem_dealloc(tmem, 512);
}

// ---- the epilogue's activation as a table ----------------------------------
// Every BF16 input z (bit pattern i), through the kernels' own packed
// arithmetic: out [3][2][65536] = {act (forward), act (adjoint), act'} x
// {low lane, high lane}; thread i puts z = i in the low lane and z = 65535 - i
// in the high lane of the same register, so both lanes of every input are
// produced and can be compared.
__global__ void bf16_act_table_kernel(int act, uint16_t* __restrict__ out) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= 65536u) return;
  const uint32_t j = 65535u - i;
  const uint32_t z = i | (j << 16);
  // the forward's call and the adjoint's
  const uint32_t af = act == 1 ? act_fwd2(1, z) : act_fwd2(2, z);
  uint32_t a, d;
  if (act == 1) act_bwd2(1, z, a, d);
  else act_bwd2(2, z, a, d);
  const uint32_t v[3] = {af, a, d};
#pragma unroll
  for (int k = 0; k < 3; ++k) {
    out[(size_t)(2 * k) * 65536 + i] = (uint16_t)(v[k] & 0xFFFFu);
    out[(size_t)(2 * k + 1) * 65536 + j] = (uint16_t)(v[k] >> 16);
  }
}

cudaError_t launch_bf16_act_table(int act, uint16_t* out, cudaStream_t s) {
  bf16_act_table_kernel<<<256, 256, 0, s>>>(act, out);
  return cudaGetLastError();
}

// ---- launchers ------------------------------------------------------------------

size_t mlp_bf16_forward_smem(int layers, int out) {
  const size_t base = (size_t)kH * kFin * 2 + (size_t)(layers - 1) * kH * kH * 2 +
                      (size_t)kFwdGroups * kRows * kH * 2 + (size_t)(layers * kH + kH + 4) * sizeof(float) +
                      (fwd_bias_in_mma(out) ? (size_t)kRows * 16 * 2 + (size_t)layers * kH * 16 * 2 : 0);
  return (base + 127) / 128 * 128 + (size_t)out_mma_width(out) * kH * 2;
}
size_t mlp_bf16_backward_smem(int layers, int out) {
  return (size_t)kFin * kH * 2 + (size_t)(layers - 1) * kH * kH * 2 +
         (size_t)kBwdGroups * ((size_t)kRows * kH * 2 + (size_t)kRows * (kH + 16) * 2) +
         (size_t)out_mma_width(out) * kH * 2;
}

template <int L, int A, int O>
static cudaError_t launch_bf16_layers(bool fwd, int P, size_t rows, const float* means3D, const float* rx_pos,
                                      const float* params, const GeomView& geo, const SharedMlpLayout& Lt,
                                      float* work, const float* dL_dsignal, float* dparams, float* dL_dmeans3D,
                                      ImageHeader* hdr, cudaStream_t s) {
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
                                                                      zb, work + Lt.s, dL_dsignal, dL_dmeans3D,
                                                                      dparams, hdr, wait_polls(kPolls));
  return cudaGetLastError();
}

template <int L>
static cudaError_t launch_bf16_act(bool fwd, int P, size_t rows, int act, int out, const float* means3D,
                                   const float* rx_pos, const float* params, const GeomView& geo,
                                   const SharedMlpLayout& Lt, float* work, const float* dL_dsignal, float* dparams,
                                   float* dL_dmeans3D, ImageHeader* hdr, cudaStream_t s) {
  if (out == 64)
    return act == 1 ? launch_bf16_layers<L, 1, 64>(fwd, P, rows, means3D, rx_pos, params, geo, Lt, work,
                                                   dL_dsignal, dparams, dL_dmeans3D, hdr, s)
                    : launch_bf16_layers<L, 2, 64>(fwd, P, rows, means3D, rx_pos, params, geo, Lt, work,
                                                   dL_dsignal, dparams, dL_dmeans3D, hdr, s);
  if (out != 1) return cudaErrorInvalidValue;
  return act == 1 ? launch_bf16_layers<L, 1, 1>(fwd, P, rows, means3D, rx_pos, params, geo, Lt, work, dL_dsignal,
                                                dparams, dL_dmeans3D, hdr, s)
                  : launch_bf16_layers<L, 2, 1>(fwd, P, rows, means3D, rx_pos, params, geo, Lt, work, dL_dsignal,
                                                dparams, dL_dmeans3D, hdr, s);
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
    case 1: e = launch_bf16_act<1>(fwd, P, rows, act, out, means3D, rx_pos, params, geo, Lt, work, dL_dsignal, dparams, dL_dmeans3D, hdr, s); break;
    case 2: e = launch_bf16_act<2>(fwd, P, rows, act, out, means3D, rx_pos, params, geo, Lt, work, dL_dsignal, dparams, dL_dmeans3D, hdr, s); break;
    case 3: e = launch_bf16_act<3>(fwd, P, rows, act, out, means3D, rx_pos, params, geo, Lt, work, dL_dsignal, dparams, dL_dmeans3D, hdr, s); break;
    default: return cudaErrorInvalidValue;
  }
  return e;
}

}  // namespace gsparc
