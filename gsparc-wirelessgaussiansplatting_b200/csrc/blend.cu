// Per-tile alpha blending, forward and adjoint.
//
// Forward: a tile of 256 pixels (16x16, 8x32 or 32x8) is covered by
// 256/kThreads CTAs of kThreads threads, one pixel each: kThreads = 256 when
// there are enough tiles to fill the GPU (batched receivers), kThreads = 64
// for a single receiver, where the kernel's time is the longest tile list
// walked by one warp -- four CTAs per tile put that tile's warps on four SMs.
//
// Every CTA stages its tile's sorted list in batches of 256 entries (position,
// conic, signal, footprint box) in shared memory, prefetching the next batch
// into registers while the current one is blended (double buffer, one
// barrier per batch).  A warp skips an entry when the splat's footprint box
// (footprint_box, computed in the preprocess) lies entirely outside the
// warp's pixels: alpha < 1/255 there, so the reference would skip the entry
// for every one of those pixels and no result changes.
//
// Forward: renderCUDA (cuda_wireless_rasterizer/forward.cu:151-249).  The
// per-pixel arithmetic keeps the reference's operation order so final T,
// contributor counts and the spectra match it bit for bit.  Each warp walks
// only the compacted list of entries whose footprint touches its pixels,
// eight entries per predicated pass; block-wide early exit as in the
// reference.
//
// The forward also records, at every kBwdChunk-th list position of a tile,
// each pixel's (T, accumulated real, accumulated imag) before that position.
//
// Adjoint: renderCUDA backward (backward.cu:442-616).  Each tile's list is cut
// into chunks of kBwdChunk entries and every (tile, chunk) is an independent
// work item: it walks its entries back to front from the forward's
// checkpoint at the chunk's end (or, for pixels whose last contributor lies
// in the chunk, from final T as the reference does), so a long list no
// longer serialises on one CTA.  The eight per-(pixel, Gaussian) gradient
// terms are reduced across the warp with a transposing shuffle tree (9
// shuffles), summed per batch in shared memory and flushed with one global
// atomic per (CTA, Gaussian, term).
#include "common.cuh"
#include "kernels.cuh"

namespace gsparc {

constexpr int kBatch = 256;   // list entries staged per round

struct WarpRect {
  float x0, x1, y0, y1;
};

__device__ __forceinline__ WarpRect warp_rect(int px, int py) {
  WarpRect w;
  w.x0 = (float)__reduce_min_sync(0xffffffffu, px);
  w.x1 = (float)__reduce_max_sync(0xffffffffu, px);
  w.y0 = (float)__reduce_min_sync(0xffffffffu, py);
  w.y1 = (float)__reduce_max_sync(0xffffffffu, py);
  return w;
}

// Pixel of thread li within its tile: every warp covers an 8x4 block (the
// blocks tile the 256 pixels row-major), whose short perimeter lets the
// footprint test drop more list entries than a 16x2 or 32x1 strip would.
__device__ __forceinline__ int2 tile_pixel(int li, int tile_w) {
  const int w = li >> 5, ln = li & 31, bx = tile_w >> 3;
  return make_int2((w % bx) * 8 + (ln & 7), (w / bx) * 4 + (ln >> 3));
}

// 256-thread CTAs capped at 80 registers (three per SM instead of two, no
// spills): 427 -> 409 us at 200k x 32 receivers, 734 -> 675 us at 50k x 64.
template <int kThreads, bool kWrap>
__global__ void __launch_bounds__(kThreads, kThreads == 256 ? 3 : 1)
blend_forward_kernel(int P, int H, int W, TileGrid grid, const uint2* __restrict__ ranges,
                     const uint32_t* __restrict__ chunk_base, const uint32_t* __restrict__ point_list,
                     float4* __restrict__ ckpt, GeomView geo, ImageHeader* __restrict__ hdr,
                     float* __restrict__ final_T, uint32_t* __restrict__ n_contrib,
                     float2* __restrict__ accum, float* __restrict__ out_real, float* __restrict__ out_imag) {
  constexpr int kParts = kBlendThreads / kThreads;
  constexpr int kPer = kBatch / kThreads;
  if (hdr->error) return;
  __shared__ float2 s_xy[2][kBatch];
  __shared__ float4 s_co[2][kBatch];
  __shared__ float2 s_sg[2][kBatch];
  __shared__ float4 s_bb[2][kBatch];
  __shared__ uint8_t s_hits[kThreads / 32][kBatch];

  const int r = blockIdx.z;
  const int tile_x = blockIdx.x / kParts, part = blockIdx.x % kParts;
  const int tile = blockIdx.y * grid.gx + tile_x;
  const int tid = threadIdx.x;
  const int wid = tid >> 5, lane = tid & 31;
  const int li = part * kThreads + tid;
  const int2 lxy = tile_pixel(li, grid.tile_w);
  const int px = tile_x * grid.tile_w + lxy.x;
  const int py = blockIdx.y * grid.tile_h + lxy.y;
  const bool inside = px < W && py < H;
  const size_t pix = (size_t)r * H * W + (size_t)py * W + px;
  const float2 pixf = make_float2((float)px, (float)py);
  const WarpRect wr = warp_rect(px, py);
  const uint2 range = ranges[(size_t)r * grid.T + tile];
  const int n = (int)(range.y - range.x);
  const size_t roff = (size_t)r * P;

  float T = 1.0f;
  uint32_t last_contributor = 0;
  float acc_r = 0.0f, acc_i = 0.0f;
  bool done = !inside;
  // checkpoint slots: interior chunk boundary b (a multiple of kBwdChunk) of
  // this tile's list holds every pixel's state before position b, at slot
  // ck_base + b / kBwdChunk - 1; the adjoint chunk that ends at b starts there
  const size_t ck_base = chunk_base[(size_t)r * grid.T + tile];
  uint32_t next_ck = kBwdChunk;

  float2 pf_xy[kPer], pf_sg[kPer];
  float4 pf_co[kPer], pf_bb[kPer];
  auto prefetch = [&](int base) {
#pragma unroll
    for (int k = 0; k < kPer; ++k) {
      const int e = base + k * kThreads + tid;
      if (e < n) {
        const uint32_t id = checked_id(point_list[range.x + e], P, hdr);
        pf_xy[k] = geo.means2D[roff + id];
        pf_co[k] = geo.conic_opacity[roff + id];
        pf_sg[k] = geo.signal[roff + id];
        pf_bb[k] = geo.box[roff + id];
        if constexpr (kWrap) {   // the copy across the seam, if nearer
          const float sh = wrap_shift(pf_xy[k].x, tile_x, grid);
          pf_xy[k].x += sh;
          pf_bb[k].x += sh;
          pf_bb[k].y += sh;
        }
      }
    }
  };
  prefetch(0);
  const int rounds = (n + kBatch - 1) / kBatch;
  for (int i = 0; i < rounds; ++i) {
    const int buf = i & 1;
#pragma unroll
    for (int k = 0; k < kPer; ++k) {
      const int s = k * kThreads + tid;
      s_xy[buf][s] = pf_xy[k];
      s_co[buf][s] = pf_co[k];
      s_sg[buf][s] = pf_sg[k];
      s_bb[buf][s] = pf_bb[k];
    }
    if (__syncthreads_count(done) == kThreads) break;
    if (i + 1 < rounds) prefetch((i + 1) * kBatch);
    const int cnt = min(kBatch, n - i * kBatch);
    const uint32_t list_base = (uint32_t)(i * kBatch);
    // The warp's hit list for this batch: every lane tests the footprint
    // boxes of eight entries against the warp's pixels and the ballots
    // compact the entries that can touch them, in list order.  Only those
    // are walked, eight per pass, with branch-free predicated math: the
    // eight alphas do not depend on T, so they are all evaluated before the
    // short sequential update of T and the sums.  Decisions are the
    // negations of the reference's tests (`power > 0`, `alpha < 1/255`) so
    // NaNs take the same path; the contributor count is the entry's list
    // position + 1.
    int nh = 0;
#pragma unroll
    for (int q = 0; q < kBatch / 32; ++q) {
      const int e = q * 32 + lane;
      const bool hit = e < cnt && !box_outside(s_bb[buf][e], wr.x0, wr.x1, wr.y0, wr.y1);
      const unsigned m = __ballot_sync(0xffffffffu, hit);
      if (hit) s_hits[wid][nh + __popc(m & ((1u << lane) - 1u))] = (uint8_t)e;
      nh += __popc(m);
    }
    __syncwarp();
    for (int h0 = 0; h0 < nh; h0 += 8) {
      if (__all_sync(0xffffffffu, done)) break;
      int js[8];
      bool vs[8];
#pragma unroll
      for (int u = 0; u < 8; ++u) {
        vs[u] = h0 + u < nh;
        js[u] = vs[u] ? s_hits[wid][h0 + u] : 0;
      }
      float al[8];
      bool ok[8];
      float2 sgv[8];
#pragma unroll
      for (int u = 0; u < 8; ++u) {
        const int j = js[u];
        const float2 xy = s_xy[buf][j];
        const float4 con_o = s_co[buf][j];
        sgv[u] = s_sg[buf][j];
        const float2 d = make_float2(xy.x - pixf.x, xy.y - pixf.y);
        const float power = -0.5f * (con_o.x * d.x * d.x + con_o.z * d.y * d.y) - con_o.y * d.x * d.y;
        al[u] = fminf(0.99f, con_o.w * expf(power));
        ok[u] = vs[u] && !(power > 0.0f) && !(al[u] < 1.0f / 255.0f);
      }
#pragma unroll
      for (int u = 0; u < 8; ++u) {
        // checkpoints of the boundaries this entry passes (warp-uniform)
        const uint32_t pos = list_base + (uint32_t)js[u];
        while (vs[u] && next_ck <= pos) {
          ckpt[(ck_base + next_ck / kBwdChunk - 1) * kBlendThreads + li] = make_float4(T, acc_r, acc_i, 0.0f);
          next_ck += kBwdChunk;
        }
        const float alpha = al[u];
        const float test_T = T * (1 - alpha);
        const bool take = ok[u] && !done;
        const bool stop = take && (test_T < 0.0001f);
        done = done || stop;
        if (take && !stop) {
          acc_r += sgv[u].x * alpha * T;
          acc_i += sgv[u].y * alpha * T;
          T = test_T;
          last_contributor = pos + 1u;
        }
      }
    }
    // boundaries inside the batch after its last hit (a warp whose pixels
    // have all stopped leaves them unwritten: none of its pixels reads them)
    if (!__all_sync(0xffffffffu, done)) {
      while (next_ck < list_base + (uint32_t)cnt) {
        ckpt[(ck_base + next_ck / kBwdChunk - 1) * kBlendThreads + li] = make_float4(T, acc_r, acc_i, 0.0f);
        next_ck += kBwdChunk;
      }
    }
    __syncwarp();
  }
  if (inside) {
    final_T[pix] = T;
    n_contrib[pix] = last_contributor;
    out_real[pix] = acc_r;   // background 0 (forward.cu:187, :244)
    out_imag[pix] = acc_i;
    accum[pix] = make_float2(acc_r, acc_i);
  }
}

// Capped at 64 registers (four CTAs per SM instead of three; 36 bytes of
// spills): 730 -> 686 us at 200k x 32 receivers, 1398 -> 1291 us at 50k x 64.
template <int kThreads, bool kWrap>
__global__ void __launch_bounds__(kThreads, 4)
blend_backward_kernel(int P, int H, int W, TileGrid grid, int RT, int span, unsigned grad_mode,
                      const uint2* __restrict__ ranges, const uint32_t* __restrict__ chunk_base,
                      const uint32_t* __restrict__ item_base,
                      const uint32_t* __restrict__ point_list, const float4* __restrict__ ckpt,
                      const float2* __restrict__ accum, GeomView geo, ImageHeader* __restrict__ hdr,
                      const float* __restrict__ final_Ts, const uint32_t* __restrict__ n_contrib,
                      const float* __restrict__ dL_dout_real, const float* __restrict__ dL_dout_imag,
                      float* __restrict__ dmean2D, float* __restrict__ dconic,
                      float* __restrict__ dsig, float* __restrict__ dopac) {
  constexpr int kParts = kBlendThreads / kThreads;
  constexpr int kPer = kBatch / kThreads;
  if (hdr->error) return;
  __shared__ uint32_t s_id[2][kBatch];
  __shared__ float2 s_xy[2][kBatch];
  __shared__ float4 s_co[2][kBatch];
  __shared__ float2 s_sg[2][kBatch];
  __shared__ float4 s_bb[2][kBatch];
  __shared__ float s_grad[2][kBatch][8];
  __shared__ int s_maxlast;

  // work item -> (segment t, chunk): with span 1 segment t owns items
  // [chunk_base[t] + t, chunk_base[t + 1] + t + 1), one per chunk; with a
  // larger span, items [item_base[t], item_base[t + 1]), one per `span` chunks
  const int item = blockIdx.x / kParts, part = blockIdx.x % kParts;
  int t, chunk;
  if (span == 1) {
    if (item >= (int)chunk_base[RT] + RT) return;
    int lo = 0, hi = RT - 1;
    while (lo < hi) {
      const int mid = (lo + hi + 1) >> 1;
      if ((int)chunk_base[mid] + mid <= item) lo = mid;
      else hi = mid - 1;
    }
    t = lo;
    chunk = item - ((int)chunk_base[t] + t);
  } else {
    if (item >= (int)item_base[RT]) return;
    int lo = 0, hi = RT - 1;
    while (lo < hi) {
      const int mid = (lo + hi + 1) >> 1;
      if ((int)item_base[mid] <= item) lo = mid;
      else hi = mid - 1;
    }
    t = lo;
    chunk = (item - (int)item_base[t]) * span;
  }
  const uint2 range = ranges[t];
  const int jlo = chunk * kBwdChunk;
  const int jhi = min((int)(range.y - range.x), jlo + span * kBwdChunk);
  if (jlo >= jhi) return;   // empty segment

  const bool ref = grad_mode == GSPARC_GRAD_REFERENCE;
  const int r = t / grid.T, tile = t % grid.T;
  const int tile_x = tile % grid.gx, tile_y = tile / grid.gx;
  const int tid = threadIdx.x, lane = tid & 31;
  const int li = part * kThreads + tid;
  const int2 lxy = tile_pixel(li, grid.tile_w);
  const int px = tile_x * grid.tile_w + lxy.x;
  const int py = tile_y * grid.tile_h + lxy.y;
  const bool inside = px < W && py < H;
  const size_t pix = (size_t)r * H * W + (size_t)py * W + px;
  const float2 pixf = make_float2((float)px, (float)py);
  const WarpRect wr = warp_rect(px, py);
  const size_t roff = (size_t)r * P;

  const int last_contributor = inside ? (int)n_contrib[pix] : 0;
  const float dLr = inside ? dL_dout_real[pix] : 0.0f;
  const float dLi = inside ? dL_dout_imag[pix] : 0.0f;
  // State at the top of the chunk.  A pixel whose last contributor lies in
  // this chunk starts as the reference does (final T, nothing accumulated
  // behind it); one that contributes past the chunk starts from the
  // forward's checkpoint at position jhi: T there, and the colour blended
  // behind it, (total - accumulated before jhi) / T, as the accumulator the
  // reference's recurrence would hold at that point.
  float T = inside ? final_Ts[pix] : 0.0f;
  float acc_r = 0.0f, acc_i = 0.0f;
  if (last_contributor > jhi) {
    const float4 c = ckpt[((size_t)chunk_base[t] + chunk + span - 1) * kBlendThreads + li];
    const float2 tot = accum[pix];
    T = c.x;
    acc_r = (tot.x - c.y) / c.x;
    acc_i = ref ? acc_r : (tot.y - c.z) / c.x;
  }

  if (tid == 0) s_maxlast = 0;
  for (int e = tid; e < 2 * kBatch * 8; e += kThreads) (&s_grad[0][0][0])[e] = 0.0f;
  __syncthreads();
  const int wmax = __reduce_max_sync(0xffffffffu, last_contributor);
  if (lane == 0) atomicMax(&s_maxlast, wmax);
  __syncthreads();
  // entries at list positions >= every pixel's contributor count are skipped
  // by all pixels (backward.cu:548-550), so the walk starts below the maximum
  const int top = min(jhi, s_maxlast);
  const int nproc = top - jlo;
  if (nproc <= 0) return;

  float last_alpha = 0.0f, last_sr = 0.0f, last_si = 0.0f;
  const float ddelx_dx = 0.5f * W;
  const float ddely_dy = 0.5f * H;

  uint32_t pf_id[kPer];
  float2 pf_xy[kPer], pf_sg[kPer];
  float4 pf_co[kPer], pf_bb[kPer];
  // batch i holds list positions top-1-i*kBatch down to top-(i+1)*kBatch
  auto prefetch = [&](int base) {
#pragma unroll
    for (int q = 0; q < kPer; ++q) {
      const int e = base + q * kThreads + tid;
      if (e < nproc) {
        const uint32_t id = checked_id(point_list[range.x + top - 1 - e], P, hdr);
        pf_id[q] = id;
        pf_xy[q] = geo.means2D[roff + id];
        pf_co[q] = geo.conic_opacity[roff + id];
        pf_sg[q] = geo.signal[roff + id];
        pf_bb[q] = geo.box[roff + id];
        if constexpr (kWrap) {   // as the forward: the nearer copy
          const float sh = wrap_shift(pf_xy[q].x, tile_x, grid);
          pf_xy[q].x += sh;
          pf_bb[q].x += sh;
          pf_bb[q].y += sh;
        }
      }
    }
  };
  prefetch(0);

  const int rounds = (nproc + kBatch - 1) / kBatch;
  for (int i = 0; i < rounds; ++i) {
    const int buf = i & 1;
#pragma unroll
    for (int k = 0; k < kPer; ++k) {
      const int s = k * kThreads + tid;
      s_id[buf][s] = pf_id[k];
      s_xy[buf][s] = pf_xy[k];
      s_co[buf][s] = pf_co[k];
      s_sg[buf][s] = pf_sg[k];
      s_bb[buf][s] = pf_bb[k];
    }
    __syncthreads();
    if (i + 1 < rounds) prefetch((i + 1) * kBatch);
    const int cnt = min(kBatch, nproc - i * kBatch);
    const int pos_base = top - 1 - i * kBatch;   // list position of batch entry 0
    // Chunks of 32 entries: a ballot keeps the entries whose footprint box
    // touches the warp's pixels and whose position is below the warp's
    // largest contributor count; they are processed four per pass with
    // predicated math.  T is recovered with a reciprocal taken off the
    // dependency chain (the reference divides, backward.cu:565; the results
    // differ by at most one rounding).
    for (int c0 = 0; c0 < cnt; c0 += 32) {
      const int jl = c0 + lane;
      unsigned mask = __ballot_sync(0xffffffffu, jl < cnt && pos_base - jl < wmax &&
                                                     !box_outside(s_bb[buf][min(jl, kBatch - 1)], wr.x0, wr.x1,
                                                                  wr.y0, wr.y1));
      while (mask) {
        int js[4];
        bool vs[4];
#pragma unroll
        for (int u = 0; u < 4; ++u) {
          vs[u] = mask != 0u;
          js[u] = c0 + (vs[u] ? __ffs(mask) - 1 : 0);
          mask &= mask - 1u;
        }
        float v[4][8];
        bool contrib[4];
#pragma unroll
        for (int u = 0; u < 4; ++u) {
          const int j = js[u];
          const float2 xy = s_xy[buf][j];
          const float2 d = make_float2(xy.x - pixf.x, xy.y - pixf.y);
          const float4 con_o = s_co[buf][j];
          const float2 sg = s_sg[buf][j];
          const float power = -0.5f * (con_o.x * d.x * d.x + con_o.z * d.y * d.y) - con_o.y * d.x * d.y;
          const float G = expf(power);
          const float a_raw = con_o.w * G;
          const float alpha = fminf(0.99f, a_raw);
          const bool c = vs[u] && (pos_base - j < last_contributor) && !(power > 0.0f) &&
                         !(alpha < 1.0f / 255.0f);
          contrib[u] = c;
          const float inv_one_minus = __frcp_rn(1.f - alpha);
          const float Tn = c ? T * inv_one_minus : T;
          const float dchannel_dsignal = alpha * Tn;
          const float sig_r = sg.x;
          const float sig_i = ref ? sg.x : sg.y;
          const float acc_rn = last_alpha * last_sr + (1.f - last_alpha) * acc_r;
          const float acc_in = last_alpha * last_si + (1.f - last_alpha) * acc_i;
          float dL_dalpha = (sig_r - acc_rn) * dLr;
          if (!ref) dL_dalpha += (sig_i - acc_in) * dLi;
          dL_dalpha *= Tn;
          if (!ref && a_raw > 0.99f) dL_dalpha = 0.0f;   // clamp blocks the gradient
          const float dL_dG = con_o.w * dL_dalpha;
          const float gdx = G * d.x;
          const float gdy = G * d.y;
          const float dG_ddelx = -gdx * con_o.x - gdy * con_o.y;
          const float dG_ddely = -gdy * con_o.z - gdx * con_o.y;
          v[u][0] = c ? dL_dG * dG_ddelx * ddelx_dx : 0.0f;
          v[u][1] = c ? dL_dG * dG_ddely * ddely_dy : 0.0f;
          v[u][2] = c ? -0.5f * gdx * d.x * dL_dG : 0.0f;
          v[u][3] = c ? -0.5f * gdx * d.y * dL_dG : 0.0f;
          v[u][4] = c ? -0.5f * gdy * d.y * dL_dG : 0.0f;
          v[u][5] = c ? G * dL_dalpha : 0.0f;
          v[u][6] = c ? dchannel_dsignal * dLr : 0.0f;
          v[u][7] = c ? dchannel_dsignal * dLi : 0.0f;
          if (c) {
            T = Tn;
            acc_r = acc_rn;
            acc_i = acc_in;
            last_sr = sig_r;
            last_si = sig_i;
            last_alpha = alpha;
          }
        }
#pragma unroll
        for (int u = 0; u < 4; ++u) {
          if (__any_sync(0xffffffffu, contrib[u])) {
            const float z = warp_reduce8(v[u], lane);
            if ((lane & 3) == 0) {
              const int vidx = ((lane >> 4) & 1) * 4 + ((lane >> 3) & 1) * 2 + ((lane >> 2) & 1);
              atomicAdd(&s_grad[buf][js[u]][vidx], z);
            }
          }
        }
      }
    }
    __syncthreads();
    for (int s = tid; s < cnt; s += kThreads) {
      const uint32_t g = s_id[buf][s];
      const size_t rg = roff + g;
      float gv[8];
#pragma unroll
      for (int k = 0; k < 8; ++k) { gv[k] = s_grad[buf][s][k]; s_grad[buf][s][k] = 0.0f; }
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

// 64-thread CTAs (four per tile) while the launch has fewer tiles than two
// per SM; full-tile CTAs otherwise.
static bool use_split_tiles(int R, const TileGrid& grid) { return (long long)R * grid.T < 2LL * device_sm_count(); }

cudaError_t launch_blend_forward(int P, int R, int H, int W, const TileGrid& grid, const GeomView& geo,
                                 const ImageView& img, const BinningView& bin, float* out_real,
                                 float* out_imag, cudaStream_t stream) {
  if (R == 0 || grid.T == 0) return cudaSuccess;
  // the seam wrap is a separate instantiation: without it the kernels are the clamped ones, register for register
  if (use_split_tiles(R, grid)) {
    dim3 g(grid.gx * (kBlendThreads / 64), grid.gy, R);
    auto k = grid.wrap ? blend_forward_kernel<64, true> : blend_forward_kernel<64, false>;
    k<<<g, 64, 0, stream>>>(P, H, W, grid, img.ranges, img.chunk_base, bin.point_list, bin.ckpt, geo, img.hdr,
                            img.final_T, img.n_contrib, img.accum, out_real, out_imag);
  } else {
    dim3 g(grid.gx, grid.gy, R);
    auto k = grid.wrap ? blend_forward_kernel<kBlendThreads, true> : blend_forward_kernel<kBlendThreads, false>;
    k<<<g, kBlendThreads, 0, stream>>>(P, H, W, grid, img.ranges, img.chunk_base, bin.point_list, bin.ckpt, geo,
                                       img.hdr, img.final_T, img.n_contrib, img.accum, out_real, out_imag);
  }
  return cudaGetLastError();
}

// One full-tile CTA per (segment, chunk) work item: the chunks already give
// a single receiver's launch hundreds of CTAs, so the tile is not split (a
// split would stage every entry and flush its gradients four times).  The
// number of items is only known on the device (chunk_base[R*T] + R*T); the
// grid covers its bound capacity / kBwdChunk + R*T and surplus CTAs exit.
// A work item spans `span` checkpoint intervals (its CTA starts from the
// checkpoint at its end; a one-CTA scan first numbers each tile's items): 1 while the
// launch has few items (the chunk length is the critical path of a single
// receiver), up to 32 when there are many waves of them (each CTA's fixed
// cost -- pixel state, checkpoint, list staging, gradient flush -- is then
// spread over more entries: 3.43 -> 0.73 ms at 200k x 32 receivers).

// item_base[t] = sum over tiles t' < t of ceil(chunks(t') / span), chunks(t)
// = chunk_base[t + 1] - chunk_base[t] + 1; item_base[RT] = the item count
__global__ void __launch_bounds__(1024)
blend_item_scan_kernel(int RT, int span, const uint32_t* __restrict__ chunk_base, uint32_t* __restrict__ item_base) {
  __shared__ uint32_t s_part[1024];
  uint32_t carry = 0;
  for (int t0 = 0; t0 < RT; t0 += 1024) {
    const int t = t0 + (int)threadIdx.x;
    const uint32_t v = t < RT ? (chunk_base[t + 1] - chunk_base[t] + 1u + (uint32_t)span - 1u) / (uint32_t)span : 0u;
    s_part[threadIdx.x] = v;
    __syncthreads();
    for (int off = 1; off < 1024; off <<= 1) {   // inclusive Hillis-Steele scan
      const uint32_t x = (int)threadIdx.x >= off ? s_part[threadIdx.x - off] : 0u;
      __syncthreads();
      s_part[threadIdx.x] += x;
      __syncthreads();
    }
    if (t < RT) item_base[t] = carry + s_part[threadIdx.x] - v;
    carry += s_part[1023];
    __syncthreads();
  }
  if (threadIdx.x == 0) item_base[RT] = carry;
}

cudaError_t launch_blend_backward(int P, int R, int H, int W, const TileGrid& grid, unsigned grad_mode,
                                  long long capacity, const GeomView& geo, const ImageView& img,
                                  const BinningView& bin, const float* dL_dout_real, const float* dL_dout_imag,
                                  float* dmean2D, float* dconic, float* dsig, float* dopac, cudaStream_t stream) {
  if (R == 0 || grid.T == 0) return cudaSuccess;
  const int RT = R * grid.T;
  const long long items = capacity / kBwdChunk + RT;
  if (items > 0x7fffffffLL) return cudaErrorInvalidValue;
  int span = 1;   // the largest power of two up to 32 that leaves about 64 items per SM
  while (span < 32 && items >= 2LL * span * device_sm_count() * 64) span *= 2;
  long long grid_items = items;
  if (span > 1) {
    blend_item_scan_kernel<<<1, 1024, 0, stream>>>(RT, span, img.chunk_base, img.item_base);
    grid_items = capacity / (kBwdChunk * span) + 2LL * RT;   // bounds sum ceil(chunks / span)
  }
  auto k = grid.wrap ? blend_backward_kernel<kBlendThreads, true> : blend_backward_kernel<kBlendThreads, false>;
  k<<<(unsigned)grid_items, kBlendThreads, 0, stream>>>(
      P, H, W, grid, RT, span, grad_mode, img.ranges, img.chunk_base, img.item_base, bin.point_list, bin.ckpt, img.accum, geo, img.hdr,
      img.final_T, img.n_contrib, dL_dout_real, dL_dout_imag, dmean2D, dconic, dsig, dopac);
  return cudaGetLastError();
}

}  // namespace gsparc
