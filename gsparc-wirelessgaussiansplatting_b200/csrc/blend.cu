// Per-tile alpha blending, forward and adjoint.
//
// One CTA per (tile, receiver); 256 threads = one pixel each (16x16, 8x32 or
// 32x8 tiles).  Gaussian attributes for the next batch of 256 list entries
// are prefetched into registers while the current batch, staged in shared
// memory, is being blended (double buffer, one barrier per batch).
//
// Forward: renderCUDA (cuda_wireless_rasterizer/forward.cu:151-249).  The
// per-pixel arithmetic keeps the reference's operation order so final T,
// contributor counts and the spectra match it bit for bit.  Early exit is the
// same block-wide count of finished pixels.
//
// Adjoint: renderCUDA backward (backward.cu:442-616).  Two changes of
// method: (1) only list positions below the largest contributor count of the
// tile are visited; (2) the eight per-(pixel, Gaussian) gradient terms are
// reduced across the warp with a transposing shuffle tree (9 shuffles), then
// accumulated per batch in shared memory and flushed with one global atomic
// per (tile, Gaussian, term), instead of 8 global atomics per pixel.
#include "common.cuh"
#include "kernels.cuh"

namespace gsparc {

__global__ void __launch_bounds__(kBlendThreads)
blend_forward_kernel(int P, int H, int W, TileGrid grid, const uint2* __restrict__ ranges,
                     const uint32_t* __restrict__ point_list, GeomView geo,
                     ImageHeader* __restrict__ hdr, float* __restrict__ final_T,
                     uint32_t* __restrict__ n_contrib, float* __restrict__ out_real,
                     float* __restrict__ out_imag) {
  if (hdr->error) return;
  __shared__ float2 s_xy[2][kBlendThreads];
  __shared__ float4 s_co[2][kBlendThreads];
  __shared__ float2 s_sg[2][kBlendThreads];

  const int r = blockIdx.z;
  const int tile = blockIdx.y * grid.gx + blockIdx.x;
  const int tid = threadIdx.x;
  const int px = blockIdx.x * grid.tile_w + tid % grid.tile_w;
  const int py = blockIdx.y * grid.tile_h + tid / grid.tile_w;
  const bool inside = px < W && py < H;
  const size_t pix = (size_t)r * H * W + (size_t)py * W + px;
  const float2 pixf = make_float2((float)px, (float)py);
  const uint2 range = ranges[(size_t)r * grid.T + tile];
  const int n = (int)(range.y - range.x);
  const size_t roff = (size_t)r * P;

  float T = 1.0f;
  uint32_t last_contributor = 0;
  float acc_r = 0.0f, acc_i = 0.0f;
  bool done = !inside;

  float2 pf_xy = make_float2(0.f, 0.f), pf_sg = make_float2(0.f, 0.f);
  float4 pf_co = make_float4(0.f, 0.f, 0.f, 0.f);
  if (tid < n) {
    const uint32_t id = checked_id(point_list[range.x + tid], P, hdr);
    pf_xy = geo.means2D[roff + id];
    pf_co = geo.conic_opacity[roff + id];
    pf_sg = geo.signal[roff + id];
  }
  const int rounds = (n + kBlendThreads - 1) / kBlendThreads;
  for (int i = 0; i < rounds; ++i) {
    const int buf = i & 1;
    s_xy[buf][tid] = pf_xy;
    s_co[buf][tid] = pf_co;
    s_sg[buf][tid] = pf_sg;
    if (__syncthreads_count(done) == kBlendThreads) break;
    const int nxt = (i + 1) * kBlendThreads + tid;
    if (nxt < n) {
      const uint32_t id = checked_id(point_list[range.x + nxt], P, hdr);
      pf_xy = geo.means2D[roff + id];
      pf_co = geo.conic_opacity[roff + id];
      pf_sg = geo.signal[roff + id];
    }
    const int cnt = min(kBlendThreads, n - i * kBlendThreads);
    const uint32_t list_base = (uint32_t)(i * kBlendThreads);
    // Predicated, 4-way unrolled walk: the per-entry math of consecutive
    // entries is independent (only T and the sums carry over), so unrolling
    // lets the scheduler overlap it.  Decisions are written as the negations
    // the reference tests (`power > 0`, `alpha < 1/255`) so NaNs take the same
    // path; the contributor count is the entry's position + 1.
    for (int j0 = 0; j0 < cnt; j0 += 4) {
      if (__all_sync(0xffffffffu, done)) break;
#pragma unroll
      for (int u = 0; u < 4; ++u) {
        const int j = j0 + u;
        if (j < cnt) {
          const float2 xy = s_xy[buf][j];
          const float4 con_o = s_co[buf][j];
          const float2 sg = s_sg[buf][j];
          const float2 d = make_float2(xy.x - pixf.x, xy.y - pixf.y);
          const float power = -0.5f * (con_o.x * d.x * d.x + con_o.z * d.y * d.y) - con_o.y * d.x * d.y;
          const float alpha = fminf(0.99f, con_o.w * expf(power));
          const float test_T = T * (1 - alpha);
          const bool take = !done && !(power > 0.0f) && !(alpha < 1.0f / 255.0f);
          const bool stop = take && (test_T < 0.0001f);
          done = done || stop;
          if (take && !stop) {
            acc_r += sg.x * alpha * T;
            acc_i += sg.y * alpha * T;
            T = test_T;
            last_contributor = list_base + (uint32_t)j + 1u;
          }
        }
      }
    }
  }
  if (inside) {
    final_T[pix] = T;
    n_contrib[pix] = last_contributor;
    out_real[pix] = acc_r;   // background 0 (forward.cu:187, :244)
    out_imag[pix] = acc_i;
  }
}

// Sum eight per-lane values over the warp.  Returns the full sum of value
// `vidx` in lanes with (lane & 3) == 0, where vidx = bits 4,3,2 of the lane.
__device__ __forceinline__ float warp_reduce8(const float v[8], int lane) {
  const bool b16 = lane & 16, b8 = lane & 8, b4 = lane & 4;
  float u[4];
#pragma unroll
  for (int k = 0; k < 4; ++k) {
    const float send = b16 ? v[k] : v[k + 4];
    const float keep = b16 ? v[k + 4] : v[k];
    u[k] = keep + __shfl_xor_sync(0xffffffffu, send, 16);
  }
  float w[2];
#pragma unroll
  for (int k = 0; k < 2; ++k) {
    const float send = b8 ? u[k] : u[k + 2];
    const float keep = b8 ? u[k + 2] : u[k];
    w[k] = keep + __shfl_xor_sync(0xffffffffu, send, 8);
  }
  float z;
  {
    const float send = b4 ? w[0] : w[1];
    const float keep = b4 ? w[1] : w[0];
    z = keep + __shfl_xor_sync(0xffffffffu, send, 4);
  }
  z += __shfl_xor_sync(0xffffffffu, z, 2);
  z += __shfl_xor_sync(0xffffffffu, z, 1);
  return z;
}

__global__ void __launch_bounds__(kBlendThreads)
blend_backward_kernel(int P, int H, int W, TileGrid grid, unsigned grad_mode,
                      const uint2* __restrict__ ranges, const uint32_t* __restrict__ point_list,
                      GeomView geo, ImageHeader* __restrict__ hdr,
                      const float* __restrict__ final_Ts, const uint32_t* __restrict__ n_contrib,
                      const float* __restrict__ dL_dout_real, const float* __restrict__ dL_dout_imag,
                      float* __restrict__ dmean2D, float* __restrict__ dconic,
                      float* __restrict__ dsig, float* __restrict__ dopac) {
  if (hdr->error) return;
  __shared__ uint32_t s_id[2][kBlendThreads];
  __shared__ float2 s_xy[2][kBlendThreads];
  __shared__ float4 s_co[2][kBlendThreads];
  __shared__ float2 s_sg[2][kBlendThreads];
  __shared__ float s_grad[2][kBlendThreads][8];
  __shared__ int s_maxlast;

  const bool ref = grad_mode == GSPARC_GRAD_REFERENCE;
  const int r = blockIdx.z;
  const int tile = blockIdx.y * grid.gx + blockIdx.x;
  const int tid = threadIdx.x, lane = tid & 31;
  const int px = blockIdx.x * grid.tile_w + tid % grid.tile_w;
  const int py = blockIdx.y * grid.tile_h + tid / grid.tile_w;
  const bool inside = px < W && py < H;
  const size_t pix = (size_t)r * H * W + (size_t)py * W + px;
  const float2 pixf = make_float2((float)px, (float)py);
  const uint2 range = ranges[(size_t)r * grid.T + tile];
  const size_t roff = (size_t)r * P;

  float T = inside ? final_Ts[pix] : 0.0f;
  const int last_contributor = inside ? (int)n_contrib[pix] : 0;
  const float dLr = inside ? dL_dout_real[pix] : 0.0f;
  const float dLi = inside ? dL_dout_imag[pix] : 0.0f;

  if (tid == 0) s_maxlast = 0;
#pragma unroll
  for (int k = 0; k < 8; ++k) { s_grad[0][tid][k] = 0.0f; s_grad[1][tid][k] = 0.0f; }
  __syncthreads();
  const int wmax = __reduce_max_sync(0xffffffffu, last_contributor);
  if (lane == 0) atomicMax(&s_maxlast, wmax);
  __syncthreads();
  // entries at list positions >= every pixel's contributor count are skipped
  // by all pixels (backward.cu:548-550), so the walk starts below the maximum
  const int nproc = s_maxlast;

  float acc_r = 0.0f, acc_i = 0.0f, last_alpha = 0.0f, last_sr = 0.0f, last_si = 0.0f;
  const float ddelx_dx = 0.5f * W;
  const float ddely_dy = 0.5f * H;
  int contributor = nproc;

  uint32_t pf_id = 0;
  float2 pf_xy = make_float2(0.f, 0.f), pf_sg = make_float2(0.f, 0.f);
  float4 pf_co = make_float4(0.f, 0.f, 0.f, 0.f);
  if (tid < nproc) {
    pf_id = checked_id(point_list[range.x + nproc - 1 - tid], P, hdr);
    pf_xy = geo.means2D[roff + pf_id];
    pf_co = geo.conic_opacity[roff + pf_id];
    pf_sg = geo.signal[roff + pf_id];
  }
  const int rounds = (nproc + kBlendThreads - 1) / kBlendThreads;
  for (int i = 0; i < rounds; ++i) {
    const int buf = i & 1;
    s_id[buf][tid] = pf_id;
    s_xy[buf][tid] = pf_xy;
    s_co[buf][tid] = pf_co;
    s_sg[buf][tid] = pf_sg;
    __syncthreads();
    const int nxt = (i + 1) * kBlendThreads + tid;
    if (nxt < nproc) {
      pf_id = checked_id(point_list[range.x + nproc - 1 - nxt], P, hdr);
      pf_xy = geo.means2D[roff + pf_id];
      pf_co = geo.conic_opacity[roff + pf_id];
      pf_sg = geo.signal[roff + pf_id];
    }
    const int cnt = min(kBlendThreads, nproc - i * kBlendThreads);
    for (int j = 0; j < cnt; ++j) {
      contributor--;
      float v[8] = {0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f};
      bool contrib = false;
      if (contributor < last_contributor) {
        const float2 xy = s_xy[buf][j];
        const float2 d = make_float2(xy.x - pixf.x, xy.y - pixf.y);
        const float4 con_o = s_co[buf][j];
        const float power = -0.5f * (con_o.x * d.x * d.x + con_o.z * d.y * d.y) - con_o.y * d.x * d.y;
        const float G = expf(power);
        const float a_raw = con_o.w * G;
        const float alpha = fminf(0.99f, a_raw);
        if (power <= 0.0f && alpha >= 1.0f / 255.0f) {
          contrib = true;
          T = T / (1.f - alpha);
          const float dchannel_dsignal = alpha * T;
          const float2 sg = s_sg[buf][j];
          const float sig_r = sg.x;
          const float sig_i = ref ? sg.x : sg.y;
          acc_r = last_alpha * last_sr + (1.f - last_alpha) * acc_r;
          acc_i = last_alpha * last_si + (1.f - last_alpha) * acc_i;
          last_sr = sig_r;
          last_si = sig_i;
          float dL_dalpha = (sig_r - acc_r) * dLr;
          if (!ref) dL_dalpha += (sig_i - acc_i) * dLi;
          dL_dalpha *= T;
          if (!ref && a_raw > 0.99f) dL_dalpha = 0.0f;   // clamp blocks the gradient
          last_alpha = alpha;
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
          v[6] = dchannel_dsignal * dLr;
          v[7] = dchannel_dsignal * dLi;
        }
      }
      if (__any_sync(0xffffffffu, contrib)) {
        const float z = warp_reduce8(v, lane);
        if ((lane & 3) == 0) {
          const int vidx = ((lane >> 4) & 1) * 4 + ((lane >> 3) & 1) * 2 + ((lane >> 2) & 1);
          atomicAdd(&s_grad[buf][j][vidx], z);
        }
      }
    }
    __syncthreads();
    if (i * kBlendThreads + tid < nproc) {
      const uint32_t g = s_id[buf][tid];
      const size_t rg = roff + g;
      float gv[8];
#pragma unroll
      for (int k = 0; k < 8; ++k) { gv[k] = s_grad[buf][tid][k]; s_grad[buf][tid][k] = 0.0f; }
      if (gv[0] != 0.0f) atomicAdd(dmean2D + rg * 3 + 0, gv[0]);
      if (gv[1] != 0.0f) atomicAdd(dmean2D + rg * 3 + 1, gv[1]);
      if (gv[2] != 0.0f) atomicAdd(dconic + rg * 4 + 0, gv[2]);
      if (gv[3] != 0.0f) atomicAdd(dconic + rg * 4 + 1, gv[3]);
      if (gv[4] != 0.0f) atomicAdd(dconic + rg * 4 + 3, gv[4]);
      if (gv[5] != 0.0f) atomicAdd(dopac + g, gv[5]);
      if (gv[6] != 0.0f) atomicAdd(dsig + rg * 2 + 0, gv[6]);
      if (gv[7] != 0.0f) atomicAdd(dsig + rg * 2 + 1, gv[7]);
    }
  }
}

cudaError_t launch_blend_forward(int P, int R, int H, int W, const TileGrid& grid, const GeomView& geo,
                                 const ImageView& img, const BinningView& bin, float* out_real,
                                 float* out_imag, cudaStream_t stream) {
  if (R == 0 || grid.T == 0) return cudaSuccess;
  dim3 g(grid.gx, grid.gy, R);
  blend_forward_kernel<<<g, kBlendThreads, 0, stream>>>(P, H, W, grid, img.ranges, bin.point_list, geo, img.hdr,
                                                        img.final_T, img.n_contrib, out_real, out_imag);
  return cudaGetLastError();
}

cudaError_t launch_blend_backward(int P, int R, int H, int W, const TileGrid& grid, unsigned grad_mode,
                                  const GeomView& geo, const ImageView& img, const BinningView& bin,
                                  const float* dL_dout_real, const float* dL_dout_imag, float* dmean2D,
                                  float* dconic, float* dsig, float* dopac, cudaStream_t stream) {
  if (R == 0 || grid.T == 0) return cudaSuccess;
  dim3 g(grid.gx, grid.gy, R);
  blend_backward_kernel<<<g, kBlendThreads, 0, stream>>>(P, H, W, grid, grad_mode, img.ranges, bin.point_list, geo,
                                                         img.hdr, img.final_T, img.n_contrib, dL_dout_real,
                                                         dL_dout_imag, dmean2D, dconic, dsig, dopac);
  return cudaGetLastError();
}

}  // namespace gsparc
