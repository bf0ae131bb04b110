// Forward preprocess: one thread per (Gaussian, receiver).
//
// Follows preprocessCUDA (cuda_wireless_rasterizer/forward.cu:252-327) and the
// per-Gaussian emission MLP computeSignalFromMLP (forward.cu:17-75).  The
// float expressions keep the reference's operation order so radii, tile
// rectangles and depth bits match it bit for bit.  Differences in structure:
//   * receivers are batched on grid.y, outputs are receiver-major SoA;
//   * the per-tile instance histogram the binning needs is accumulated here
//     in shared memory (one global atomic per touched tile per block) instead
//     of a separate scan over tiles_touched (rasterizer_impl.cu:270).
#include "common.cuh"
#include "kernels.cuh"

namespace gsparc {

// computeSignalFromMLP (forward.cu:17-75): h = leaky(b1 + W1 rx),
// o = sigmoid(b2 + W2 h - log(|tx - mean| + 1e-6)).
__device__ __forceinline__ float2 emission_mlp_ref(int g, int P, const float* __restrict__ mlp,
                                                   const float3 mean, const float3 rx, const float3 tx) {
  const float* w1 = mlp + (size_t)g * (kMlpIn * kMlpHidden);
  const float* b1 = mlp + (size_t)P * (kMlpIn * kMlpHidden) + (size_t)g * kMlpHidden;
  const float* w2 = mlp + (size_t)P * (kMlpIn * kMlpHidden + kMlpHidden) + (size_t)g * (kMlpOut * kMlpHidden);
  const float* b2 = mlp + (size_t)P * (kMlpIn * kMlpHidden + kMlpHidden + kMlpOut * kMlpHidden) + (size_t)g * kMlpOut;
  const float in[3] = {rx.x, rx.y, rx.z};
  const float3 diff = make_float3(tx.x - mean.x, tx.y - mean.y, tx.z - mean.z);
  const float d = sqrtf(diff.x * diff.x + diff.y * diff.y + diff.z * diff.z);
  const float log_d = logf(d + 1e-6f);
  float hidden[kMlpHidden];
#pragma unroll
  for (int i = 0; i < kMlpHidden; ++i) {
    float s = __ldg(b1 + i);
#pragma unroll
    for (int j = 0; j < kMlpIn; ++j) s += __ldg(w1 + i * kMlpIn + j) * in[j];
    hidden[i] = (s > 0.0f) ? s : (0.01f * s);
  }
  float o[kMlpOut];
#pragma unroll
  for (int k = 0; k < kMlpOut; ++k) {
    float s = __ldg(b2 + k);
#pragma unroll
    for (int j = 0; j < kMlpHidden; ++j) s += __ldg(w2 + k * kMlpHidden + j) * hidden[j];
    const float att = s - log_d;
    o[k] = 1.0f / (1.0f + expf(-att));
  }
  return make_float2(o[0], o[1]);
}

template <bool kSharedHist>
__global__ void __launch_bounds__(256)
preprocess_kernel(int P, int H, int W, TileGrid grid, float mod,
                  const float* __restrict__ means3D, const float* __restrict__ mlp,
                  const float* __restrict__ opacities, const float* __restrict__ scales,
                  const float* __restrict__ rotations, const float* __restrict__ views,
                  const float* __restrict__ tx_pos, const float* __restrict__ rx_pos,
                  GeomView geo, int* __restrict__ radii_out, uint32_t* __restrict__ counts) {
  extern __shared__ uint32_t hist[];
  const int r = blockIdx.y;
  const int g = blockIdx.x * blockDim.x + threadIdx.x;
  if (kSharedHist) {
    for (int t = threadIdx.x; t < grid.T; t += blockDim.x) hist[t] = 0;
    __syncthreads();
  }

  bool vis = false;
  int x0 = 0, y0 = 0, x1 = 0, y1 = 0;
  if (g < P) {
    const size_t rg = (size_t)r * P + g;
    const float* m = views + 16 * r;
    float mv[16];
#pragma unroll
    for (int i = 0; i < 16; ++i) mv[i] = __ldg(m + i);
    const float3 p = make_float3(__ldg(means3D + 3 * g), __ldg(means3D + 3 * g + 1), __ldg(means3D + 3 * g + 2));
    int radius_i = 0;
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
        tile_rect(px, py, radius_i, grid, x0, y0, x1, y1);
        // radius_i > 0 keeps the histogram consistent with the scatter, which
        // keys on radii > 0, even for non-finite inputs (ceil(NaN) -> 0)
        if (radius_i > 0 && (x1 - x0) * (y1 - y0) != 0) {
          vis = true;
          const float3 rx = make_float3(__ldg(rx_pos + 3 * r), __ldg(rx_pos + 3 * r + 1), __ldg(rx_pos + 3 * r + 2));
          const float3 tx = make_float3(__ldg(tx_pos), __ldg(tx_pos + 1), __ldg(tx_pos + 2));
          geo.signal[rg] = emission_mlp_ref(g, P, mlp, p, rx, tx);
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
  }

  if (vis) {
    for (int ty = y0; ty < y1; ++ty)
      for (int tx = x0; tx < x1; ++tx) {
        const int tile = ty * grid.gx + tx;
        if (kSharedHist) atomicAdd(&hist[tile], 1u);
        else atomicAdd(&counts[(size_t)r * grid.T + tile], 1u);
      }
  }
  if (kSharedHist) {
    __syncthreads();
    for (int t = threadIdx.x; t < grid.T; t += blockDim.x) {
      const uint32_t c = hist[t];
      if (c) atomicAdd(&counts[(size_t)r * grid.T + t], c);
    }
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

constexpr int kMaxSharedHistTiles = 40960;   // 160 KB of shared counters

cudaError_t launch_preprocess(int P, int R, int H, int W, const TileGrid& grid, float mod,
                              const float* means3D, const float* mlp, const float* opacities,
                              const float* scales, const float* rotations, const float* views,
                              const float* tx_pos, const float* rx_pos, const GeomView& geo,
                              int* radii_out, uint32_t* counts, cudaStream_t stream) {
  if (P == 0 || R == 0) return cudaSuccess;
  dim3 block(256), gridd((P + 255) / 256, R);
  if (grid.T <= kMaxSharedHistTiles) {
    const size_t smem = (size_t)grid.T * sizeof(uint32_t);
    if (smem > 48 * 1024) {
      cudaError_t e = cudaFuncSetAttribute(preprocess_kernel<true>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
      if (e != cudaSuccess) return e;
    }
    preprocess_kernel<true><<<gridd, block, smem, stream>>>(P, H, W, grid, mod, means3D, mlp, opacities, scales,
                                                            rotations, views, tx_pos, rx_pos, geo, radii_out, counts);
  } else {
    preprocess_kernel<false><<<gridd, block, 0, stream>>>(P, H, W, grid, mod, means3D, mlp, opacities, scales,
                                                          rotations, views, tx_pos, rx_pos, geo, radii_out, counts);
  }
  return cudaGetLastError();
}

cudaError_t launch_mark_visible(int P, const float* means3D, const float* view, uint8_t* present,
                                cudaStream_t stream) {
  if (P == 0) return cudaSuccess;
  mark_visible_kernel<<<(P + 255) / 256, 256, 0, stream>>>(P, means3D, view, present);
  return cudaGetLastError();
}

}  // namespace gsparc
