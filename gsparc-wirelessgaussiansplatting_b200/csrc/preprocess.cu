// Forward preprocess: one thread per (Gaussian, receiver), 64-thread CTAs.
//
// Follows preprocessCUDA (cuda_wireless_rasterizer/forward.cu:252-327) and the
// per-Gaussian emission MLP computeSignalFromMLP (forward.cu:17-75).  The
// float expressions keep the reference's operation order so radii, tile
// rectangles and depth bits match it bit for bit.  Differences in structure:
//   * receivers are batched on grid.y, outputs are receiver-major SoA;
//   * the per-tile instance histogram the binning needs is accumulated here
//     in shared memory (one global atomic per touched tile per block) instead
//     of a separate scan over tiles_touched (rasterizer_impl.cu:270), and the
//     last CTA to finish scans it into the tile ranges (no separate launch);
//   * the depth key of every (receiver, Gaussian) and its digit histograms
//     for the depth order (binning.cu) are produced here too.
#include "common.cuh"
#include "kernels.cuh"

namespace gsparc {

// ---- per-Gaussian emission MLP ---------------------------------------------
// computeSignalFromMLP (forward.cu:17-75): h = leaky(b1 + W1 rx),
// o = sigmoid(b2 + W2 h - log(|tx - mean| + 1e-6)).
//
// The parameters of a warp's 32 consecutive Gaussians are contiguous in each
// of the four blocks of the flat buffer (W1 [P,32,3], b1 [P,32], W2 [P,2,32],
// b2 [P,2]), so the warp stages them into shared memory with coalesced
// loads, one padded row per Gaussian (row strides 97, 33, 65 are odd, so the
// 32 threads reading their own rows hit 32 different banks).  Each thread
// then evaluates its Gaussian's MLP in the reference's operation order.
constexpr int kPreThreads = 64;
constexpr int kW1S = 97, kB1S = 33, kW2S = 65, kB2S = 2;
constexpr int kMlpSmemPerWarp = 32 * (kW1S + kB1S + kW2S + kB2S);   // floats

template <bool kVec>
__device__ __forceinline__ void stage_mlp(float* __restrict__ sm, const float* __restrict__ mlp, int P, int g0,
                                          int lane) {
  const int nv = min(32, P - g0);
  float* w1 = sm;
  float* b1 = w1 + 32 * kW1S;
  float* w2 = b1 + 32 * kB1S;
  float* b2 = w2 + 32 * kW2S;
  const float* gw1 = mlp + (size_t)g0 * (kMlpIn * kMlpHidden);
  const float* gb1 = mlp + (size_t)P * (kMlpIn * kMlpHidden) + (size_t)g0 * kMlpHidden;
  const float* gw2 = mlp + (size_t)P * (kMlpIn * kMlpHidden + kMlpHidden) + (size_t)g0 * (kMlpOut * kMlpHidden);
  const float* gb2 = mlp + (size_t)P * (kMlpIn * kMlpHidden + kMlpHidden + kMlpOut * kMlpHidden) + (size_t)g0 * kMlpOut;
  if (kVec) {   // 16-byte aligned buffer: rows of 96, 32 and 64 floats split into whole float4s
    for (int e = lane; e < nv * 24; e += 32) {
      const float4 v = __ldg(reinterpret_cast<const float4*>(gw1) + e);
      float* d = w1 + (e / 24) * kW1S + (e % 24) * 4;
      d[0] = v.x; d[1] = v.y; d[2] = v.z; d[3] = v.w;
    }
    for (int e = lane; e < nv * 8; e += 32) {
      const float4 v = __ldg(reinterpret_cast<const float4*>(gb1) + e);
      float* d = b1 + (e / 8) * kB1S + (e % 8) * 4;
      d[0] = v.x; d[1] = v.y; d[2] = v.z; d[3] = v.w;
    }
    for (int e = lane; e < nv * 16; e += 32) {
      const float4 v = __ldg(reinterpret_cast<const float4*>(gw2) + e);
      float* d = w2 + (e / 16) * kW2S + (e % 16) * 4;
      d[0] = v.x; d[1] = v.y; d[2] = v.z; d[3] = v.w;
    }
    if (lane < nv) {
      const float2 v = __ldg(reinterpret_cast<const float2*>(gb2) + lane);
      b2[lane * kB2S] = v.x;
      b2[lane * kB2S + 1] = v.y;
    }
  } else {
    for (int e = lane; e < nv * 96; e += 32) w1[(e / 96) * kW1S + e % 96] = __ldg(gw1 + e);
    for (int e = lane; e < nv * 32; e += 32) b1[(e / 32) * kB1S + e % 32] = __ldg(gb1 + e);
    for (int e = lane; e < nv * 64; e += 32) w2[(e / 64) * kW2S + e % 64] = __ldg(gw2 + e);
    for (int e = lane; e < nv * 2; e += 32) b2[(e / 2) * kB2S + e % 2] = __ldg(gb2 + e);
  }
}

__device__ __forceinline__ float2 emission_mlp_row(const float* __restrict__ sm, int lane, const float3 mean,
                                                   const float3 rx, const float3 tx) {
  const float* w1 = sm + lane * kW1S;
  const float* b1 = sm + 32 * kW1S + lane * kB1S;
  const float* w2 = sm + 32 * (kW1S + kB1S) + lane * kW2S;
  const float* b2 = sm + 32 * (kW1S + kB1S + kW2S) + lane * kB2S;
  const float in[3] = {rx.x, rx.y, rx.z};
  const float3 diff = make_float3(tx.x - mean.x, tx.y - mean.y, tx.z - mean.z);
  const float d = sqrtf(diff.x * diff.x + diff.y * diff.y + diff.z * diff.z);
  const float log_d = logf(d + 1e-6f);
  float hidden[kMlpHidden];
#pragma unroll
  for (int i = 0; i < kMlpHidden; ++i) {
    float s = b1[i];
#pragma unroll
    for (int j = 0; j < kMlpIn; ++j) s += w1[i * kMlpIn + j] * in[j];
    hidden[i] = (s > 0.0f) ? s : (0.01f * s);
  }
  float o[kMlpOut];
#pragma unroll
  for (int k = 0; k < kMlpOut; ++k) {
    float s = b2[k];
#pragma unroll
    for (int j = 0; j < kMlpHidden; ++j) s += w2[k * kMlpHidden + j] * hidden[j];
    const float att = s - log_d;
    o[k] = 1.0f / (1.0f + expf(-att));
  }
  return make_float2(o[0], o[1]);
}

// Dynamic shared memory: the warps' MLP staging areas (per-Gaussian MLP
// only), the 4 x 256 digit counters of the depth keys (the radix sort's
// histograms), then (kSharedHist) one counter per tile.  kMlp: 0 no
// per-Gaussian MLP (the shared MLP writes the signal later; without the
// 50 KB staging area four times as many CTAs fit on an SM), 1 staged with
// float4 loads, 2 staged with scalar loads.
template <bool kSharedHist, int kMlp>
__global__ void __launch_bounds__(kPreThreads)
preprocess_kernel(int P, int H, int W, TileGrid grid, float mod,
                  const float* __restrict__ means3D, const float* __restrict__ mlp,
                  const float* __restrict__ opacities, const float* __restrict__ scales,
                  const float* __restrict__ rotations, const float* __restrict__ views,
                  const float* __restrict__ tx_pos, const float* __restrict__ rx_pos,
                  GeomView geo, int* __restrict__ radii_out, ImageView img, int per_cta) {
  uint32_t* __restrict__ counts = img.counts;
  extern __shared__ float smem[];
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  float* sm_mlp = smem + wid * kMlpSmemPerWarp;
  uint32_t* dhist = reinterpret_cast<uint32_t*>(smem + (kMlp ? (kPreThreads / 32) * kMlpSmemPerWarp : 0));
  uint32_t* hist = dhist + 1024;
  const int r = blockIdx.y;
  for (int t = threadIdx.x; t < 1024; t += blockDim.x) dhist[t] = 0;
  if (kSharedHist)
    for (int t = threadIdx.x; t < grid.T; t += blockDim.x) hist[t] = 0;
  __syncthreads();

  // per_cta consecutive groups of kPreThreads Gaussians, the histograms
  // flushed once for all of them
  for (int grp = 0; grp < per_cta; ++grp) {
  const int g0 = (blockIdx.x * per_cta + grp) * kPreThreads;
  const int g = g0 + (int)threadIdx.x;
  bool vis = false;
  int x0 = 0, y0 = 0, x1 = 0, y1 = 0;
  TileSpan span{0, 0, 0, 0, grid.gx, 0};
  const size_t rg = (size_t)r * P + g;
  float3 p = make_float3(0.f, 0.f, 0.f);
  if (g < P) {
    const float* m = views + 16 * r;
    float mv[16];
#pragma unroll
    for (int i = 0; i < 16; ++i) mv[i] = __ldg(m + i);
    p = make_float3(__ldg(means3D + 3 * g), __ldg(means3D + 3 * g + 1), __ldg(means3D + 3 * g + 2));
    int radius_i = 0;
    uint32_t dkey = 0xffffffffu;   // depth key of the per-receiver depth order: culled Gaussians sort last
    // computeCov3D (forward.cu:124-149).  Receiver independent: written by the
    // receiver-0 thread for every Gaussian, including ones receiver 0 culls,
    // because other receivers of the batch (and the backward) read it.
    const float3 s = make_float3(mod * __ldg(scales + 3 * g), mod * __ldg(scales + 3 * g + 1),
                                 mod * __ldg(scales + 3 * g + 2));
    const float4 q = make_float4(__ldg(rotations + 4 * g), __ldg(rotations + 4 * g + 1),
                                 __ldg(rotations + 4 * g + 2), __ldg(rotations + 4 * g + 3));
    const Mat3 M = scale_rot(s, quat_to_rot(q));
    const Mat3 Sigma = mat_mul(mat_T(M), M);
    float cov3[6] = {Sigma.c[0][0], Sigma.c[0][1], Sigma.c[0][2], Sigma.c[1][1], Sigma.c[1][2], Sigma.c[2][2]};
    if (r == 0) {
#pragma unroll
      for (int i = 0; i < 6; ++i) geo.cov3D[(size_t)g * 6 + i] = cov3[i];
    }
    // range cull (too_close, auxiliary.h:133-155)
    const float3 t = view_point(p, mv);
    const float rr = range_sq(t);
    if (rr > 0.04f) {
      const float rdist = sqrtf(rr);
      // transformProj (auxiliary.h:101-113)
      const float inv_r = 1.0f / (rdist + 0.0000001f);
      const float lon = atan2f(t.x, t.z);
      const float lat = asinf(t.y * inv_r);
      const float ndc_x = lon * kInvPi;
      const float ndc_y = lat * (kTwoInvPi);
      // computeCov2D (forward.cu:78-122)
      const ProjJac pj = proj_jacobian(t, W, H);
      const Mat3 J = jac_mat(pj.J00, pj.J02, pj.J10, pj.J11, pj.J12);
      const Mat3 Wr = view_rot(mv);
      const Mat3 T = mat_mul(Wr, J);
      const Mat3 Vrk = sym_from6(cov3);
      Mat3 cov = mat_mul(mat_mul(mat_T(T), mat_T(Vrk)), T);
      cov.c[0][0] += 0.3f;
      cov.c[1][1] += 0.3f;
      const float ca = cov.c[0][0], cb = cov.c[0][1], cc = cov.c[1][1];
      const float det = (ca * cc - cb * cb);
      if (det != 0.0f) {
        const float det_inv = 1.f / det;
        const float3 conic = make_float3(cc * det_inv, -cb * det_inv, ca * det_inv);
        const float mid = 0.5f * (ca + cc);
        const float lambda1 = mid + sqrtf(fmaxf(0.1f, mid * mid - det));
        const float lambda2 = mid - sqrtf(fmaxf(0.1f, mid * mid - det));
        const float my_radius = ceilf(3.f * sqrtf(fmaxf(lambda1, lambda2)));
        const float px = ndc_to_pixel(ndc_x, W);
        const float py = ndc_to_pixel(ndc_y, H);
        radius_i = (int)my_radius;
        span = tile_span(px, py, radius_i, grid);
        x0 = span.x0; y0 = span.y0; x1 = span.x1; y1 = span.y1;
        // radius_i > 0 keeps the histogram consistent with the scatter, which
        // keys on radii > 0, even for non-finite inputs (ceil(NaN) -> 0)
        if (radius_i > 0 && (x1 - x0) * (y1 - y0) != 0) {
          vis = true;
          dkey = __float_as_uint(rdist);
          geo.depth[rg] = rdist;
          geo.means2D[rg] = make_float2(px, py);
          const float4 co = make_float4(conic.x, conic.y, conic.z, __ldg(opacities + g));
          geo.conic_opacity[rg] = co;
          geo.box[rg] = footprint_box(make_float2(px, py), co);
        }
      }
    }
    if (!vis) radius_i = 0;
    geo.radii[rg] = radius_i;
    if (radii_out) radii_out[rg] = radius_i;
    geo.sort_key[0][rg] = dkey;
#pragma unroll
    for (int pass = 0; pass < 4; ++pass) atomicAdd(&dhist[pass * 256 + ((dkey >> (8 * pass)) & 255u)], 1u);
  }
  // emission MLP of the visible Gaussians, from the warp's staged parameters
  // (no per-Gaussian MLP: the signal is written later by the shared MLP)
  if (kMlp != 0 && __any_sync(0xffffffffu, vis)) {
    stage_mlp<kMlp == 1>(sm_mlp, mlp, P, g0 + wid * 32, lane);
    __syncwarp();
    if (vis) {
      const float3 rx = make_float3(__ldg(rx_pos + 3 * r), __ldg(rx_pos + 3 * r + 1), __ldg(rx_pos + 3 * r + 2));
      const float3 tx = make_float3(__ldg(tx_pos), __ldg(tx_pos + 1), __ldg(tx_pos + 2));
      geo.signal[rg] = emission_mlp_row(sm_mlp, lane, p, rx, tx);
    }
  }

  if (vis) {
    for_each_tile(span, grid.gx, [&](int tile) {
      if (kSharedHist) atomicAdd(&hist[tile], 1u);
      else atomicAdd(&counts[(size_t)r * grid.T + tile], 1u);
    });
  }
  __syncwarp();   // the warp's staged MLP rows are read before the next group restages them
  }
  __syncthreads();
  if (kSharedHist) {
    for (int t = threadIdx.x; t < grid.T; t += blockDim.x) {
      const uint32_t c = hist[t];
      if (c) atomicAdd(&counts[(size_t)r * grid.T + t], c);
    }
  }
  for (int t = threadIdx.x; t < 1024; t += blockDim.x) {
    const uint32_t c = dhist[t];
    if (c) atomicAdd(&geo.sort_state[(size_t)r * 1024 + t], c);
  }
  // the last CTA to finish scans the tile counts into segment ranges
  __shared__ bool s_last;
  __syncthreads();
  if (threadIdx.x == 0) {
    __threadfence();
    s_last = atomicAdd(&img.hdr->arrived, 1u) == gridDim.x * gridDim.y - 1;
  }
  __syncthreads();
  if (s_last) {
    __threadfence();
    scan_segments_cta((int)gridDim.y * grid.T, counts, img.ranges, img.cursor, img.chunk_base, img.hdr);
  }
}

// Range cull only (checkFrustum, rasterizer_impl.cu:173-185).
__global__ void mark_visible_kernel(int P, const float* __restrict__ means3D,
                                    const float* __restrict__ view, uint8_t* __restrict__ present) {
  const int g = blockIdx.x * blockDim.x + threadIdx.x;
  if (g >= P) return;
  float mv[16];
#pragma unroll
  for (int i = 0; i < 16; ++i) mv[i] = __ldg(view + i);
  const float3 p = make_float3(means3D[3 * g], means3D[3 * g + 1], means3D[3 * g + 2]);
  const float3 t = view_point(p, mv);
  const float rr = range_sq(t);
  present[g] = rr <= 0.04f ? 0 : 1;
}

// MLP staging (50,432 B), digit counters (4 KB)
constexpr size_t kMlpStageBytes = (kPreThreads / 32) * kMlpSmemPerWarp * sizeof(float);
constexpr size_t kDigitSmemBytes = 1024 * sizeof(uint32_t);
// dynamic shared memory ceiling: 227 KB per CTA less 1 KB kept for the
// kernel's static shared memory (the last CTA's scan)
constexpr int kPreDynSmemMax = 226 * 1024;

template <bool kSharedHist, int kMlp>
static cudaError_t set_preprocess_smem() {
  return cudaFuncSetAttribute(preprocess_kernel<kSharedHist, kMlp>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                              kPreDynSmemMax);
}

template <int kMlp>
static void preprocess_launch(bool shared_hist, dim3 gridd, size_t smem, cudaStream_t stream, int P, int H, int W,
                              const TileGrid& grid, float mod, const float* means3D, const float* mlp,
                              const float* opacities, const float* scales, const float* rotations,
                              const float* views, const float* tx_pos, const float* rx_pos, const GeomView& geo,
                              int* radii_out, const ImageView& img, int per_cta) {
  if (shared_hist)
    preprocess_kernel<true, kMlp><<<gridd, kPreThreads, smem, stream>>>(
        P, H, W, grid, mod, means3D, mlp, opacities, scales, rotations, views, tx_pos, rx_pos, geo, radii_out, img,
        per_cta);
  else
    preprocess_kernel<false, kMlp><<<gridd, kPreThreads, smem, stream>>>(
        P, H, W, grid, mod, means3D, mlp, opacities, scales, rotations, views, tx_pos, rx_pos, geo, radii_out, img,
        per_cta);
}

cudaError_t launch_preprocess(int P, int R, int H, int W, const TileGrid& grid, float mod,
                              const float* means3D, const float* mlp, const float* opacities,
                              const float* scales, const float* rotations, const float* views,
                              const float* tx_pos, const float* rx_pos, const GeomView& geo,
                              int* radii_out, const ImageView& img, cudaStream_t stream) {
  if (P == 0 || R == 0) return cudaSuccess;
  // the shared-memory opt-in is set once per device, so later calls (including
  // ones made while a CUDA graph is being captured) only enqueue the launch
  static bool attr_done[64] = {false};
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return e;
  if (dev < 0 || dev >= 64 || !attr_done[dev]) {
    if ((e = set_preprocess_smem<true, 0>()) != cudaSuccess) return e;
    if ((e = set_preprocess_smem<true, 1>()) != cudaSuccess) return e;
    if ((e = set_preprocess_smem<true, 2>()) != cudaSuccess) return e;
    if ((e = set_preprocess_smem<false, 0>()) != cudaSuccess) return e;
    if ((e = set_preprocess_smem<false, 1>()) != cudaSuccess) return e;
    if ((e = set_preprocess_smem<false, 2>()) != cudaSuccess) return e;
    if (dev >= 0 && dev < 64) attr_done[dev] = true;
  }
  const int mode = mlp == nullptr ? 0 : ((((uintptr_t)mlp) & 15u) == 0 ? 1 : 2);
  // groups of kPreThreads Gaussians per CTA: one while the launch is small
  // (latency), up to 16 when it fills many waves, so that each CTA's
  // histogram initialisation and flush serve up to 1,024 Gaussians
  int per_cta = 1;
  while (per_cta < 16 && (long long)P * R >= 2LL * per_cta * device_sm_count() * kPreThreads * 16) per_cta *= 2;
  const dim3 gridd((P + kPreThreads * per_cta - 1) / (kPreThreads * per_cta), R);
  const size_t base = (mode ? kMlpStageBytes : 0) + kDigitSmemBytes;
  const bool shared_hist = base + (size_t)grid.T * sizeof(uint32_t) <= (size_t)kPreDynSmemMax;
  const size_t smem = base + (shared_hist ? (size_t)grid.T * sizeof(uint32_t) : 0);
  if (mode == 0)
    preprocess_launch<0>(shared_hist, gridd, smem, stream, P, H, W, grid, mod, means3D, mlp, opacities, scales,
                         rotations, views, tx_pos, rx_pos, geo, radii_out, img, per_cta);
  else if (mode == 1)
    preprocess_launch<1>(shared_hist, gridd, smem, stream, P, H, W, grid, mod, means3D, mlp, opacities, scales,
                         rotations, views, tx_pos, rx_pos, geo, radii_out, img, per_cta);
  else
    preprocess_launch<2>(shared_hist, gridd, smem, stream, P, H, W, grid, mod, means3D, mlp, opacities, scales,
                         rotations, views, tx_pos, rx_pos, geo, radii_out, img, per_cta);
  return cudaGetLastError();
}

cudaError_t launch_mark_visible(int P, const float* means3D, const float* view, uint8_t* present,
                                cudaStream_t stream) {
  if (P == 0) return cudaSuccess;
  mark_visible_kernel<<<(P + 255) / 256, 256, 0, stream>>>(P, means3D, view, present);
  return cudaGetLastError();
}

}  // namespace gsparc
