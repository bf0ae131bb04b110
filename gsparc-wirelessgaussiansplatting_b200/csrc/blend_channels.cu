// Multi-channel per-tile blend: C amplitude channels per Gaussian (features
// [R][P][C], C <= 64, e.g. one per frequency bin), rendering C spectra per
// receiver with one set of transmittance / contributor decisions.  This
// extends renderCUDA (forward.cu:151-249), which blends NUM_CHANNELS = 1
// (config.h:15); the per-entry power / alpha / termination arithmetic is the
// single-channel kernels' (blend.cu), so final T and contributor counts equal
// a single-channel render of the same geometry.
//
// The channels are split into groups of up to 16, one CTA per (tile,
// receiver, channel group): every group walks the tile's list with the same
// transmittance decisions, so a long list is walked by C / 16 CTAs at once,
// each with a quarter of the per-entry work.
//
// Forward: one 256-thread CTA per (tile, receiver, group), one pixel per
// thread; the tile's list is staged 32 entries at a time (position, conic, the
// group's features), each pixel keeps the group's accumulators in registers:
// out[c] += f_c * (alpha * T).  Group 0 writes final T and contributor counts.
//
// Adjoint (the true derivative; the 0.99 alpha clamp blocks the gradient):
// back to front from each pixel's contributor count, T recomputed by division
// from final T.  The colour behind entry j enters dL/dalpha only through its
// dot product with dL/dout, so one scalar per pixel carries it:
//   B_j = sum_{k>j} alpha_k T_k (f_k . g),  dL/dalpha_j = T_j (f_j . g - B_j / T_{j+1}).
// dL/dalpha, and through it the position, conic and opacity gradients, is
// linear in the per-channel products, so each channel group adds its share.
// dL/df_j,c = sum over pixels of alpha_j T_j g_c is a small GEMM per staged
// batch: the batch's (entry, pixel) weights alpha T go to shared memory and
// every thread sums one entry's two channels over the pixel blocks the entry
// reached, against the tile's dL/dout of the group, held in shared memory for
// the whole walk.  Position, conic and opacity gradients are reduced per warp
// (warp_reduce8) and summed per batch in shared memory before one global
// atomic per (CTA, entry, term).
#include "common.cuh"
#include "kernels.cuh"

namespace gsparc {

namespace {
constexpr int kMcThreads = 256;   // one thread per pixel: every tile shape holds 256 pixels
constexpr int kMcBatch = 32;      // list entries staged per round
constexpr int kMcWs = kMcThreads + 1;   // row stride of the (entry, pixel) weights
constexpr int kMcGroupFwd = 32;          // channels per forward CTA
constexpr int kMcGroupBwd = 64;          // channels per adjoint CTA
}  // namespace

// Pixel of thread li in its tile: every warp covers an 8x4 block, and skips
// the staged entries whose footprint box (alpha < 1/255 outside it, from the
// preprocess) misses its block -- no result changes.
__device__ __forceinline__ int2 mc_pixel(int li, int tile_w) {
  const int w = li >> 5, ln = li & 31, bx = tile_w >> 3;
  return make_int2((w % bx) * 8 + (ln & 7), (w / bx) * 4 + (ln >> 3));
}
struct McRect {
  float x0, x1, y0, y1;
};
__device__ __forceinline__ McRect mc_warp_rect(int px, int py) {
  McRect w;
  w.x0 = (float)__reduce_min_sync(0xffffffffu, px);
  w.x1 = (float)__reduce_max_sync(0xffffffffu, px);
  w.y0 = (float)__reduce_min_sync(0xffffffffu, py);
  w.y1 = (float)__reduce_max_sync(0xffffffffu, py);
  return w;
}

template <int kMcGroup>
__global__ void __launch_bounds__(kMcThreads)
blend_channels_forward_kernel(int P, int H, int W, int C, TileGrid grid, const uint2* __restrict__ ranges,
                              const uint32_t* __restrict__ point_list, GeomView geo, ImageHeader* __restrict__ hdr,
                              const float* __restrict__ features, float* __restrict__ final_T,
                              uint32_t* __restrict__ n_contrib, float* __restrict__ out) {
  if (hdr->error) return;
  __shared__ float2 s_xy[kMcBatch];
  __shared__ float4 s_co[kMcBatch];
  __shared__ float4 s_bb[kMcBatch];
  __shared__ __align__(16) float s_f[kMcBatch][kMcGroup];
  const int r = blockIdx.y, tile = blockIdx.x;
  const int c_lo = blockIdx.z * kMcGroup, Cg = min(kMcGroup, C - c_lo);   // this CTA's channels
  const int tx = tile % grid.gx, ty = tile / grid.gx;
  const int li = threadIdx.x;
  const int2 lp = mc_pixel(li, grid.tile_w);
  const int px = tx * grid.tile_w + lp.x, py = ty * grid.tile_h + lp.y;
  const bool inside = px < W && py < H;
  const float2 pixf = make_float2((float)px, (float)py);
  const McRect wr = mc_warp_rect(px, py);
  const uint2 range = ranges[(size_t)r * grid.T + tile];
  const int n = (int)(range.y - range.x);
  const size_t roff = (size_t)r * P;
  const int C4 = (Cg + 3) & ~3;
  float T = 1.0f;
  float acc[kMcGroup];
#pragma unroll
  for (int c = 0; c < kMcGroup; ++c) acc[c] = 0.0f;
  uint32_t last = 0;
  bool done = !inside;
  for (int b0 = 0; b0 < n; b0 += kMcBatch) {
    if (__syncthreads_count(done) == kMcThreads) break;   // also: the previous batch is consumed
    const int cnt = min(kMcBatch, n - b0);
    if (li < cnt) {
      const uint32_t id = checked_id(point_list[range.x + b0 + li], P, hdr);
      float2 xy = geo.means2D[roff + id];
      float4 bb = geo.box[roff + id];
      const float sh = wrap_shift(xy.x, tx, grid);
      xy.x += sh;
      bb.x += sh;
      bb.y += sh;
      s_xy[li] = xy;
      s_bb[li] = bb;
      s_co[li] = geo.conic_opacity[roff + id];
    }
    for (int i = li; i < cnt * C4; i += kMcThreads) {   // channels padded with zeros to a multiple of 4
      const int e = i / C4, c = i - e * C4;
      const uint32_t id = checked_id(point_list[range.x + b0 + e], P, hdr);
      s_f[e][c] = c < Cg ? features[(roff + id) * C + c_lo + c] : 0.0f;
    }
    __syncthreads();
    if (done) continue;
    for (int e = 0; e < cnt; ++e) {
      if (box_outside(s_bb[e], wr.x0, wr.x1, wr.y0, wr.y1)) continue;   // warp-uniform
      const float2 xy = s_xy[e];
      const float4 con_o = s_co[e];
      const float2 d = make_float2(xy.x - pixf.x, xy.y - pixf.y);
      const float power = -0.5f * (con_o.x * d.x * d.x + con_o.z * d.y * d.y) - con_o.y * d.x * d.y;
      if (power > 0.0f) continue;
      const float alpha = fminf(0.99f, con_o.w * expf(power));
      if (alpha < 1.0f / 255.0f) continue;
      const float test_T = T * (1 - alpha);
      if (test_T < 0.0001f) {
        done = true;
        break;
      }
      const float w = alpha * T;
#pragma unroll
      for (int q = 0; q < kMcGroup / 4; ++q)
        if (4 * q < Cg) {
          const float4 f = *reinterpret_cast<const float4*>(&s_f[e][4 * q]);
          acc[4 * q] = fmaf(f.x, w, acc[4 * q]);
          acc[4 * q + 1] = fmaf(f.y, w, acc[4 * q + 1]);
          acc[4 * q + 2] = fmaf(f.z, w, acc[4 * q + 2]);
          acc[4 * q + 3] = fmaf(f.w, w, acc[4 * q + 3]);
        }
      T = test_T;
      last = (uint32_t)(b0 + e + 1);
    }
  }
  if (inside) {
    const size_t pix = (size_t)r * H * W + (size_t)py * W + px;
    if (blockIdx.z == 0) {
      final_T[pix] = T;
      n_contrib[pix] = last;
    }
    const size_t plane = (size_t)H * W;
    float* o = out + ((size_t)r * C + c_lo) * plane + (size_t)py * W + px;
#pragma unroll
    for (int c = 0; c < kMcGroup; ++c)
      if (c < Cg) o[c * plane] = acc[c];
  }
}

template <int kMcGroup>
__global__ void __launch_bounds__(kMcThreads)
blend_channels_backward_kernel(int P, int H, int W, int C, TileGrid grid, const uint2* __restrict__ ranges,
                               const uint32_t* __restrict__ point_list, GeomView geo, ImageHeader* __restrict__ hdr,
                               const float* __restrict__ features, const float* __restrict__ final_T,
                               const uint32_t* __restrict__ n_contrib, const float* __restrict__ dL_dout,
                               float* __restrict__ dL_dfeatures, float* __restrict__ dmean2D,
                               float* __restrict__ dconic, float* __restrict__ dopacity) {
  if (hdr->error) return;
  constexpr int kMcGs = kMcGroup + 4;      // row stride of the tile's dL/dout: float4 rows on distinct banks
  constexpr int kCpt = kMcGroup / 8;       // channels per thread in the dL/df GEMM
  static_assert(kCpt % 4 == 0, "the dL/df GEMM reads float4 channel quads");
  extern __shared__ __align__(16) float mc_sm[];
  float* s_g = mc_sm;                                   // [256 pixels][kMcGs] dL/dout of the tile (group)
  float* s_w = s_g + kMcThreads * kMcGs;                // [kMcBatch][257] alpha T of (entry, pixel)
  __shared__ float2 s_xy[kMcBatch];
  __shared__ float4 s_co[kMcBatch];
  __shared__ float4 s_bb[kMcBatch];
  __shared__ uint32_t s_id[kMcBatch];
  __shared__ __align__(16) float s_f[kMcBatch][kMcGroup];
  __shared__ float s_grad[kMcBatch][8];
  __shared__ uint32_t s_hit[kMcBatch];   // per entry: the warps with a contributing pixel
  __shared__ int s_top;
  const int r = blockIdx.y, tile = blockIdx.x;
  const int c_lo = blockIdx.z * kMcGroup, Cg = min(kMcGroup, C - c_lo);   // this CTA's channels
  const int tx = tile % grid.gx, ty = tile / grid.gx;
  const int li = threadIdx.x, lane = li & 31;
  const int2 lp = mc_pixel(li, grid.tile_w);
  const int px = tx * grid.tile_w + lp.x, py = ty * grid.tile_h + lp.y;
  const bool inside = px < W && py < H;
  const float2 pixf = make_float2((float)px, (float)py);
  const McRect wr = mc_warp_rect(px, py);
  const uint2 range = ranges[(size_t)r * grid.T + tile];
  const size_t roff = (size_t)r * P;
  const size_t plane = (size_t)H * W;
  const size_t pix = (size_t)r * H * W + (size_t)py * W + px;
  float T = inside ? final_T[pix] : 1.0f;
  const int last = inside ? (int)n_contrib[pix] : 0;
  const int C4 = (Cg + 3) & ~3;
  float g[kMcGroup];
#pragma unroll
  for (int c = 0; c < kMcGroup; ++c)
    g[c] = (inside && c < Cg) ? dL_dout[((size_t)r * C + c_lo + c) * plane + (size_t)py * W + px] : 0.0f;
#pragma unroll
  for (int q = 0; q < kMcGroup / 4; ++q)
    *reinterpret_cast<float4*>(s_g + li * kMcGs + 4 * q) = make_float4(g[4 * q], g[4 * q + 1], g[4 * q + 2], g[4 * q + 3]);
  if (li == 0) s_top = 0;
  for (int i = li; i < kMcBatch * 8; i += kMcThreads) (&s_grad[0][0])[i] = 0.0f;
  if (li < kMcBatch) s_hit[li] = 0u;
  __syncthreads();
  atomicMax(&s_top, last);
  __syncthreads();
  // entries at list positions >= every pixel's contributor count are skipped by all pixels
  const int top = s_top;
  const float ddelx_dx = 0.5f * W, ddely_dy = 0.5f * H;
  float B = 0.0f;
  for (int hi = top; hi > 0; hi -= kMcBatch) {
    const int cnt = min(kMcBatch, hi);
    const int lo = hi - cnt;   // this batch holds list positions [lo, hi), walked from hi - 1 down
    if (li < cnt) {
      const uint32_t id = checked_id(point_list[range.x + lo + li], P, hdr);
      s_id[li] = id;
      float2 xy = geo.means2D[roff + id];
      float4 bb = geo.box[roff + id];
      const float sh = wrap_shift(xy.x, tx, grid);
      xy.x += sh;
      bb.x += sh;
      bb.y += sh;
      s_xy[li] = xy;
      s_bb[li] = bb;
      s_co[li] = geo.conic_opacity[roff + id];
    }
    for (int i = li; i < cnt * C4; i += kMcThreads) {   // channels padded with zeros to a multiple of 4
      const int e = i / C4, c = i - e * C4;
      const uint32_t id = checked_id(point_list[range.x + lo + e], P, hdr);
      s_f[e][c] = c < Cg ? features[(roff + id) * C + c_lo + c] : 0.0f;
    }
    __syncthreads();
    for (int e = cnt - 1; e >= 0; --e) {
      // warp-uniform: no pixel of the warp takes the entry, so its weights stay unread (s_hit)
      if (box_outside(s_bb[e], wr.x0, wr.x1, wr.y0, wr.y1)) continue;
      const int pos = lo + e;
      const float2 xy = s_xy[e];
      const float4 con_o = s_co[e];
      const float2 d = make_float2(xy.x - pixf.x, xy.y - pixf.y);
      const float power = -0.5f * (con_o.x * d.x * d.x + con_o.z * d.y * d.y) - con_o.y * d.x * d.y;
      const float G = expf(power);
      const float a_raw = con_o.w * G;
      const float alpha = fminf(0.99f, a_raw);
      const bool c_ok = inside && pos < last && !(power > 0.0f) && !(alpha < 1.0f / 255.0f);
      float v[8];
      float wgt = 0.0f;
      if (c_ok) {
        const float Tn = T * __frcp_rn(1.f - alpha);
        float fg = 0.0f;
#pragma unroll
        for (int q = 0; q < kMcGroup / 4; ++q)
          if (4 * q < Cg) {
            const float4 f = *reinterpret_cast<const float4*>(&s_f[e][4 * q]);
            fg = fmaf(f.x, g[4 * q], fg);
            fg = fmaf(f.y, g[4 * q + 1], fg);
            fg = fmaf(f.z, g[4 * q + 2], fg);
            fg = fmaf(f.w, g[4 * q + 3], fg);
          }
        float dL_dalpha = (fg - B / T) * Tn;
        if (a_raw > 0.99f) dL_dalpha = 0.0f;   // clamp blocks the gradient
        const float dL_dG = con_o.w * dL_dalpha;
        const float gdx = G * d.x;
        const float gdy = G * d.y;
        const float dG_ddelx = -gdx * con_o.x - gdy * con_o.y;
        const float dG_ddely = -gdy * con_o.z - gdx * con_o.y;
        v[0] = dL_dG * dG_ddelx * ddelx_dx;
        v[1] = dL_dG * dG_ddely * ddely_dy;
        v[2] = -0.5f * gdx * d.x * dL_dG;
        v[3] = -0.5f * gdx * d.y * dL_dG;
        v[4] = -0.5f * gdy * d.y * dL_dG;
        v[5] = G * dL_dalpha;
        wgt = alpha * Tn;
        B = fmaf(wgt, fg, B);
        T = Tn;
      } else {
#pragma unroll
        for (int k = 0; k < 6; ++k) v[k] = 0.0f;
      }
      v[6] = 0.0f;
      v[7] = 0.0f;
      s_w[e * kMcWs + li] = wgt;
      if (__any_sync(0xffffffffu, c_ok)) {
        if (lane == 0) atomicOr(&s_hit[e], 1u << (li >> 5));
        const float z = warp_reduce8(v, lane);
        if ((lane & 3) == 0) {
          const int vidx = ((lane >> 4) & 1) * 4 + ((lane >> 3) & 1) * 2 + ((lane >> 2) & 1);
          if (vidx < 6) atomicAdd(&s_grad[e][vidx], z);
        }
      }
    }
    __syncthreads();
    // dL/df for the batch: thread = (entry e, kCpt channels from c0), summed over the tile's pixels
    {
      const int e = li >> 3, c0 = (li & 7) * kCpt;
      if (e < cnt && c0 < Cg) {
        float y[kCpt];
#pragma unroll
        for (int k = 0; k < kCpt; ++k) y[k] = 0.0f;
        const float* wrow = s_w + e * kMcWs;
        // only the warps (32-pixel blocks) where the entry contributed have nonzero weights
        for (uint32_t m = s_hit[e]; m; m &= m - 1) {
          const int p0 = (__ffs(m) - 1) * 32;
#pragma unroll 4
          for (int p = p0; p < p0 + 32; ++p) {
            const float wv = wrow[p];
#pragma unroll
            for (int k = 0; k < kCpt; k += 4) {
              const float4 gv = *reinterpret_cast<const float4*>(s_g + p * kMcGs + c0 + k);
              y[k] = fmaf(wv, gv.x, y[k]);
              y[k + 1] = fmaf(wv, gv.y, y[k + 1]);
              y[k + 2] = fmaf(wv, gv.z, y[k + 2]);
              y[k + 3] = fmaf(wv, gv.w, y[k + 3]);
            }
          }
        }
        float* dst = dL_dfeatures + (roff + s_id[e]) * C + c_lo;
#pragma unroll
        for (int k = 0; k < kCpt; ++k)
          if (c0 + k < Cg && y[k] != 0.0f) atomicAdd(dst + c0 + k, y[k]);
      }
      if (li < cnt) {
        const size_t rg = roff + s_id[li];
        float gv[6];
#pragma unroll
        for (int k = 0; k < 6; ++k) {
          gv[k] = s_grad[li][k];
          s_grad[li][k] = 0.0f;
        }
        if (gv[0] != 0.0f) atomicAdd(dmean2D + rg * 3 + 0, gv[0]);
        if (gv[1] != 0.0f) atomicAdd(dmean2D + rg * 3 + 1, gv[1]);
        if (gv[2] != 0.0f) atomicAdd(dconic + rg * 4 + 0, gv[2]);
        if (gv[3] != 0.0f) atomicAdd(dconic + rg * 4 + 1, gv[3]);
        if (gv[4] != 0.0f) atomicAdd(dconic + rg * 4 + 3, gv[4]);
        if (gv[5] != 0.0f) atomicAdd(dopacity + s_id[li], gv[5]);
      }
    }
    __syncthreads();
    if (li < kMcBatch) s_hit[li] = 0u;   // read above by every thread; the next batch sets it after a barrier
  }
}

static size_t blend_channels_backward_smem() {
  return ((size_t)kMcThreads * (kMcGroupBwd + 4) + (size_t)kMcBatch * kMcWs) * sizeof(float);
}

cudaError_t launch_blend_channels_forward(int P, int R, int H, int W, int C, const TileGrid& grid,
                                          const GeomView& geo, const ImageView& img, const BinningView& bin,
                                          const float* features, float* out, cudaStream_t s) {
  dim3 g((unsigned)grid.T, (unsigned)R, (unsigned)((C + kMcGroupFwd - 1) / kMcGroupFwd));
  blend_channels_forward_kernel<kMcGroupFwd><<<g, kMcThreads, 0, s>>>(P, H, W, C, grid, img.ranges, bin.point_list, geo, img.hdr,
                                                         features, img.final_T, img.n_contrib, out);
  return cudaGetLastError();
}

cudaError_t launch_blend_channels_backward(int P, int R, int H, int W, int C, const TileGrid& grid,
                                           const GeomView& geo, const ImageView& img, const BinningView& bin,
                                           const float* features, const float* dL_dout, float* dL_dfeatures,
                                           float* dmean2D, float* dconic, float* dopacity, cudaStream_t s) {
  const size_t smem = blend_channels_backward_smem();
  static bool attr_done[64] = {};
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return e;
  if (dev < 0 || dev >= 64 || !attr_done[dev]) {
    e = cudaFuncSetAttribute(blend_channels_backward_kernel<kMcGroupBwd>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)smem);
    if (e != cudaSuccess) return e;
    if (dev >= 0 && dev < 64) attr_done[dev] = true;
  }
  dim3 g((unsigned)grid.T, (unsigned)R, (unsigned)((C + kMcGroupBwd - 1) / kMcGroupBwd));
  blend_channels_backward_kernel<kMcGroupBwd><<<g, kMcThreads, smem, s>>>(P, H, W, C, grid, img.ranges, bin.point_list, geo,
                                                             img.hdr, features, img.final_T, img.n_contrib, dL_dout,
                                                             dL_dfeatures, dmean2D, dconic, dopacity);
  return cudaGetLastError();
}

}  // namespace gsparc
