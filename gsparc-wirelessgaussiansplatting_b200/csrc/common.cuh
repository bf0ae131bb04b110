// Shared device helpers and state layouts for the sm_100a splatting kernels.
//
// Layout in HBM (all receiver-major, structure-of-arrays, 256-byte aligned):
//   geometry state  [R][P]  means2D float2 | depth f32 | radii i32 |
//                           conic_opacity float4 | signal float2 (real, imag)
//                   [P]     cov3D 6 x f32 (receiver independent)
//                   [R][P]  footprint box float4 (blend skipping, see below)
//   image state     header (K, error word) | ranges uint2[R*T] |
//                   counts u32[R*T] | cursor u32[R*T] |
//                   final_T f32[R*H*W] | n_contrib u32[R*H*W]
//   binning state   keys u64[Kcap] | keys_alt u64[Kcap] | point_list u32[Kcap]
// R = receivers per launch, P = Gaussians, T = tiles per receiver.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include "../../include/gsparc_b200.h"

namespace gsparc {

// 1/pi and 2/pi: the same decimal constants as glibc's M_1_PIf32 / M_2_PIf32
// (which the reference uses, auxiliary.h:109-110), rounded to float.
constexpr float kInvPi = 0.318309886183790671537767526745028724f;
constexpr float kTwoInvPi = 0.636619772367581343075535053490057448f;

constexpr int kBlendThreads = 256;       // pixels per tile (16x16, 8x32 or 32x8)
constexpr int kMlpIn = 3;                // emission MLP input: receiver position
constexpr int kMlpHidden = 32;
constexpr int kMlpOut = 2;               // (real, imag)
constexpr int kMlpFloats = kMlpIn * kMlpHidden + kMlpHidden + kMlpOut * kMlpHidden + kMlpOut;

// Streaming multiprocessors of the current device (148 on a B200), looked up
// once per device; grid-size heuristics scale with it.
inline int device_sm_count() {
  static int cache[64] = {};
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) return 148;
  if (cache[dev] == 0) {
    int n = 0;
    if (cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess || n <= 0) return 148;
    cache[dev] = n;
  }
  return cache[dev];
}

// error word bits (image state header)
constexpr uint32_t kErrCapacity = 1u << 0;   // K exceeded the binning capacity
constexpr uint32_t kErrSegment = 1u << 1;    // a tile segment exceeded the sort limit
constexpr uint32_t kErrBadIndex = 1u << 2;   // a point list held an id >= P (arena mismatch)
constexpr uint32_t kErrSortWait = 1u << 3;   // a depth-sort look-back wait gave up (bounded spin)
constexpr uint32_t kErrMlpWait = 1u << 4;    // a tensor-core MLP wait on its MMAs gave up (bounded)

struct ImageHeader {
  unsigned long long num_rendered;   // K, written by the preprocess's last CTA (segment scan)
  unsigned int error;                // error bits, OR-ed by kernels
  unsigned int arrived;              // preprocess CTAs done (the last one scans the tile counts)
  unsigned long long capacity;       // binning capacity the render was given
  unsigned long long reserved[29];   // pad to 256 bytes
};
static_assert(sizeof(ImageHeader) == 256, "header is one 256-byte block");

__host__ __device__ inline size_t align_up(size_t v, size_t a) { return (v + a - 1) / a * a; }

// Tile grid of an H x W spectrum.  `wrap` (GSPARC_FLAG_WRAP_AZIMUTH): pixel
// columns x and x +- W are the same azimuth, so footprints continue across the
// 0/2pi seam; off, footprints are clamped at the image edges as the reference
// does (auxiliary.h:14-24).
struct TileGrid {
  int tile_h, tile_w, gx, gy, T, W, wrap;
  __host__ __device__ TileGrid(int H, int W_, int th, int tw, int wrap_ = 0)
      : tile_h(th), tile_w(tw), gx((W_ + tw - 1) / tw), gy((H + th - 1) / th), T(gx * gy), W(W_), wrap(wrap_) {}
};

// Per-receiver depth order (binning.cu): an LSD radix sort of one 32-bit key
// per (receiver, Gaussian) -- the depth bits of visible Gaussians, ~0 for the
// rest -- in tiles of kSortTileKeys keys with decoupled look-back.
constexpr int kSortTileKeys = 2048;   // 256 threads x 8 keys
// Multi-channel blend (blend_channels.cu): at most this many amplitude channels.
constexpr int kMaxChannels = 64;
__host__ __device__ inline size_t sort_tiles(size_t P) { return (P + kSortTileKeys - 1) / kSortTileKeys; }
// words of the sort state: digit histograms [R][4][256], tile tickets [R][4],
// look-back words [R][4][tiles][256]; zeroed before every preprocess
__host__ __device__ inline size_t sort_state_words(size_t P, size_t R) {
  return R * 1024 + R * 4 + R * 4 * sort_tiles(P) * 256;
}

struct GeomView {
  float2* means2D;
  float* depth;
  int* radii;
  float4* conic_opacity;
  float2* signal;
  float* cov3D;
  float4* box;            // [R][P] pixel box (x_lo, x_hi, y_lo, y_hi) outside which alpha < 1/255
  uint32_t* sort_key[2];  // [R][P] radix ping-pong; sort_key[0] starts as the depth keys
  uint32_t* sort_val[2];  // [R][P]; sort_val[0] ends as the Gaussian ids in depth order
  uint32_t* rank;         // [R][P] position of each Gaussian in its receiver's depth order
  uint32_t* sort_state;   // sort_state_words(P, R) words
};

struct ImageView {
  ImageHeader* hdr;
  uint2* ranges;
  uint32_t* counts;
  uint32_t* cursor;
  float* final_T;
  uint32_t* n_contrib;
  uint32_t* chunk_base;   // [R*T + 1]: exclusive scan of interior chunk boundaries per tile
  float2* accum;          // [R, H, W]: accumulated (real, imag) of the forward
  uint32_t* item_base;    // [R*T + 1]: first adjoint work item of each tile (written by the adjoint launch)
};

// The adjoint walks each tile's list in chunks of kBwdChunk entries, one CTA
// per (tile, chunk); the forward checkpoints every pixel's (T, accumulated
// real, imag) at each interior chunk boundary so a chunk can start without
// the entries behind it.
constexpr int kBwdChunk = 64;

struct BinningView {
  uint32_t* seg_rank;     // [K] depth rank of each instance, grouped by segment (unordered within)
  uint32_t* point_list;   // [K] Gaussian ids, segments in depth order
  float4* ckpt;           // [K / kBwdChunk][256 pixels]
};

// Host/device carving of the three caller-provided arenas.  The sizes are the
// exact byte counts the gsparc_*_state_bytes() entry points report.
__host__ __device__ inline size_t carve_geom(char* base, size_t P, size_t R, GeomView* v) {
  size_t off = 0;
  auto take = [&](size_t bytes) { char* p = base ? base + off : nullptr; off = align_up(off + bytes, 256); return p; };
  size_t n = P * R;
  char* a = take(n * sizeof(float2));
  char* b = take(n * sizeof(float));
  char* c = take(n * sizeof(int));
  char* d = take(n * sizeof(float4));
  char* e = take(n * sizeof(float2));
  char* f = take(P * 6 * sizeof(float));
  char* g = take(n * sizeof(float4));
  char* k0 = take(n * sizeof(uint32_t));
  char* k1 = take(n * sizeof(uint32_t));
  char* v0 = take(n * sizeof(uint32_t));
  char* v1 = take(n * sizeof(uint32_t));
  char* rk = take(n * sizeof(uint32_t));
  char* ss = take(sort_state_words(P, R) * sizeof(uint32_t));
  if (v) {
    v->means2D = (float2*)a; v->depth = (float*)b; v->radii = (int*)c;
    v->conic_opacity = (float4*)d; v->signal = (float2*)e; v->cov3D = (float*)f; v->box = (float4*)g;
    v->sort_key[0] = (uint32_t*)k0; v->sort_key[1] = (uint32_t*)k1;
    v->sort_val[0] = (uint32_t*)v0; v->sort_val[1] = (uint32_t*)v1;
    v->rank = (uint32_t*)rk; v->sort_state = (uint32_t*)ss;
  }
  return off;
}

__host__ __device__ inline size_t carve_image(char* base, size_t R, size_t T, size_t npix, ImageView* v) {
  size_t off = 0;
  auto take = [&](size_t bytes) { char* p = base ? base + off : nullptr; off = align_up(off + bytes, 256); return p; };
  char* h = take(sizeof(ImageHeader));
  char* a = take(R * T * sizeof(uint2));
  char* b = take(R * T * sizeof(uint32_t));
  char* c = take(R * T * sizeof(uint32_t));
  char* d = take(R * npix * sizeof(float));
  char* e = take(R * npix * sizeof(uint32_t));
  char* f = take((R * T + 1) * sizeof(uint32_t));
  char* g = take(R * npix * sizeof(float2));
  char* i = take((R * T + 1) * sizeof(uint32_t));
  if (v) {
    v->hdr = (ImageHeader*)h; v->ranges = (uint2*)a; v->counts = (uint32_t*)b;
    v->cursor = (uint32_t*)c; v->final_T = (float*)d; v->n_contrib = (uint32_t*)e;
    v->chunk_base = (uint32_t*)f; v->accum = (float2*)g; v->item_base = (uint32_t*)i;
  }
  return off;
}

__host__ __device__ inline size_t carve_binning(char* base, size_t K, BinningView* v) {
  size_t off = 0;
  auto take = [&](size_t bytes) { char* p = base ? base + off : nullptr; off = align_up(off + bytes, 256); return p; };
  char* a = take(K * sizeof(uint32_t));
  char* c = take(K * sizeof(uint32_t));
  char* d = take((K / kBwdChunk) * kBlendThreads * sizeof(float4));
  if (v) {
    v->seg_rank = (uint32_t*)a; v->point_list = (uint32_t*)c; v->ckpt = (float4*)d;
  }
  return off;
}

// Flat per-Gaussian training state (parameters, gradients, Adam moments):
// segments in float units, each starting on a 256-byte boundary.
struct GaussianLayout {
  size_t centre, scale, quat, opacity, mlp, conf, total;
};

// mlp_floats: size of the emission-MLP segment (194 P for the per-Gaussian
// MLP, the shared MLP's parameter count otherwise); conf_floats: size of the
// trailing segment for a global parameter block such as the confidence MLP.
__host__ __device__ inline GaussianLayout gaussian_layout(size_t P, size_t mlp_floats, size_t conf_floats = 0) {
  auto a = [](size_t x) { return (x + 63) / 64 * 64; };
  GaussianLayout L;
  L.centre = 0;
  L.scale = a(3 * P);
  L.quat = L.scale + a(3 * P);
  L.opacity = L.quat + a(4 * P);
  L.mlp = L.opacity + a(P);
  L.conf = L.mlp + a(mlp_floats);
  L.total = L.conf + a(conf_floats);
  return L;
}

// Exclusive scan of one value per thread over the CTA (any multiple of 32
// threads up to 1024); every thread also receives the total.  warp_tot: 32
// words of shared memory.
template <typename V>
__device__ __forceinline__ V cta_exclusive_scan(V local, V* warp_tot, V& total) {
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5, nw = blockDim.x >> 5;
  V incl = local;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const V v = __shfl_up_sync(0xffffffffu, incl, o);
    if (lane >= o) incl += v;
  }
  if (lane == 31) warp_tot[wid] = incl;
  __syncthreads();
  if (wid == 0) {
    V w = lane < nw ? warp_tot[lane] : V(0);
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const V v = __shfl_up_sync(0xffffffffu, w, o);
      if (lane >= o) w += v;
    }
    if (lane < nw) warp_tot[lane] = w;
  }
  __syncthreads();
  const V excl = (wid ? warp_tot[wid - 1] : V(0)) + (incl - local);
  total = warp_tot[nw - 1];
  __syncthreads();
  return excl;
}

// ---- scan of per-segment counts -> ranges, cursors, K, chunk bases ---------
// Run by the preprocess's last CTA (preprocess.cu) (any block size) once every CTA's tile
// counts have landed: n = R*T segments, each thread owns 8 consecutive
// segments of every chunk of 8 * blockDim.x.
__device__ __forceinline__ void scan_segments_cta(int n, const uint32_t* __restrict__ counts, uint2* __restrict__ ranges,
                                  uint32_t* __restrict__ cursor, uint32_t* __restrict__ chunk_base,
                                  ImageHeader* __restrict__ hdr) {
  __shared__ unsigned long long warp_tot[32];
  const int tid = threadIdx.x;
  unsigned long long carry = 0, carry_b = 0;
  for (int base = 0; base < n; base += (int)blockDim.x * 8) {
    uint32_t c[8], nb[8];
    unsigned long long local = 0, local_b = 0;
#pragma unroll
    for (int k = 0; k < 8; ++k) {
      const int i = base + tid * 8 + k;
      c[k] = i < n ? __ldcg(counts + i) : 0u;
      nb[k] = c[k] ? (c[k] - 1u) / kBwdChunk : 0u;   // interior chunk boundaries of the segment
      local += c[k];
      local_b += nb[k];
    }
    unsigned long long tot, tot_b;
    unsigned long long start = carry + cta_exclusive_scan<unsigned long long>(local, warp_tot, tot);
    unsigned long long start_b = carry_b + cta_exclusive_scan<unsigned long long>(local_b, warp_tot, tot_b);
#pragma unroll
    for (int k = 0; k < 8; ++k) {
      const int i = base + tid * 8 + k;
      if (i < n) {
        // empty tiles keep the reference's zeroed range (rasterizer_impl.cu:303)
        ranges[i] = c[k] ? make_uint2((uint32_t)start, (uint32_t)(start + c[k])) : make_uint2(0u, 0u);
        cursor[i] = (uint32_t)start;
        chunk_base[i] = (uint32_t)start_b;
        start += c[k];
        start_b += nb[k];
      }
    }
    carry += tot;
    carry_b += tot_b;
  }
  if (tid == 0) {
    hdr->num_rendered = carry;
    chunk_base[n] = (uint32_t)carry_b;
  }
}

// Scratch of the fused training loss (ssim.cu), in floats.
struct LossLayout {
  size_t nblk, dmu1, ds11, ds12, partial, pre, coef, share, psync, sync, total;
};

// ---------------------------------------------------------------------------
// Projection math.  The float expression order of every helper below is kept
// identical to the reference kernels (cited per function) so the integer
// outputs that depend on it -- radii, tile rectangles, depth key bits -- come
// out bit-identical under the same compiler and default -fmad.
// ---------------------------------------------------------------------------

// world -> receiver frame, matrix stored transposed (auxiliary.h:38-46)
__device__ __forceinline__ float3 view_point(const float3& p, const float* m) {
  float3 t = {
      m[0] * p.x + m[4] * p.y + m[8] * p.z + m[12],
      m[1] * p.x + m[5] * p.y + m[9] * p.z + m[13],
      m[2] * p.x + m[6] * p.y + m[10] * p.z + m[14],
  };
  return t;
}

// squared range |t|^2 with the reference's rounding pinned: the reference
// expression x*x + y*y + z*z (auxiliary.h:141) compiles to
// fma(z, z, fma(x, x, y*y)), established against the depth bits recorded from
// the reference extension (tests/golden/raster_ref_golden.npz); written with
// explicit intrinsics so the depth key bits do not depend on contraction
// choices made around this expression
__device__ __forceinline__ float range_sq(const float3& t) {
  return __fmaf_rn(t.z, t.z, __fmaf_rn(t.x, t.x, __fmul_rn(t.y, t.y)));
}

// transpose of the rotation part applied to a vector (auxiliary.h:117-125)
__device__ __forceinline__ float3 view_vec_T(const float3& v, const float* m) {
  float3 t = {
      m[0] * v.x + m[1] * v.y + m[2] * v.z,
      m[4] * v.x + m[5] * v.y + m[6] * v.z,
      m[8] * v.x + m[9] * v.y + m[10] * v.z,
  };
  return t;
}

// pixel coordinate of a normalised hemisphere coordinate; evaluated in double
// because the reference's literals are doubles (auxiliary.h:10-13)
__device__ __forceinline__ float ndc_to_pixel(float v, int S) {
  return (float)((((double)v + 1.0) * S - 1.0) * 0.5);
}

// tile rectangle touched by a footprint of the given radius, clamped to the
// grid (no azimuth wrap), (auxiliary.h:14-24)
__device__ __forceinline__ void tile_rect(float px, float py, int radius, const TileGrid& g,
                                          int& x0, int& y0, int& x1, int& y1) {
  const float bx = (float)g.tile_w, by = (float)g.tile_h;
  x0 = min(g.gx, max(0, (int)((px - radius) / bx)));
  y0 = min(g.gy, max(0, (int)((py - radius) / by)));
  x1 = min(g.gx, max(0, (int)((px + radius + bx - 1) / bx)));
  y1 = min(g.gy, max(0, (int)((py + radius + by - 1) / by)));
}

// Tile columns a footprint covers: the clamped rectangle [x0, x1) x [y0, y1)
// above and, with the azimuth wrap, the columns of the part beyond the left
// edge, [xl, gx), and beyond the right edge, [0, xr) (xl = gx / xr = 0 when
// there is none; they never overlap [x0, x1)).  The wrapped edges use the
// rectangle's own rounding: xl = (int)(((px - r) + W) / bx),
// xr = (int)((((px + r) - W) + bx) - 1) / bx).
struct TileSpan {
  int x0, y0, x1, y1, xl, xr;
};
__device__ __forceinline__ TileSpan tile_span(float px, float py, int radius, const TileGrid& g) {
  TileSpan s;
  tile_rect(px, py, radius, g, s.x0, s.y0, s.x1, s.y1);
  s.xl = g.gx;
  s.xr = 0;
  if (g.wrap) {
    const float bx = (float)g.tile_w, Wf = (float)g.W, rf = (float)radius;
    const float ql = (px - rf) + Wf;
    if (px - rf < 0.0f) s.xl = max(s.x1, min(g.gx, max(0, (int)(ql / bx))));
    const float qr = (px + rf) - Wf;
    if (qr > 0.0f) s.xr = min(s.x0, max(0, (int)(((qr + bx) - 1.0f) / bx)));
  }
  return s;
}
__device__ __forceinline__ int span_tiles(const TileSpan& s, int gx) {
  return ((s.x1 - s.x0) + (gx - s.xl) + s.xr) * (s.y1 - s.y0);
}
template <class F>
__device__ __forceinline__ void for_each_tile(const TileSpan& s, int gx, F&& f) {
  for (int ty = s.y0; ty < s.y1; ++ty) {
    for (int tx = s.x0; tx < s.x1; ++tx) f(ty * gx + tx);
    for (int tx = s.xl; tx < gx; ++tx) f(ty * gx + tx);
    for (int tx = 0; tx < s.xr; ++tx) f(ty * gx + tx);
  }
}
// With the azimuth wrap, the copy of a Gaussian (x of its mean) nearest to
// tile column tx: shifted by -W or +W when it lies more than W/2 from the
// tile's centre; 0 otherwise (and always 0 without the wrap).
__device__ __forceinline__ float wrap_shift(float x, int tx, const TileGrid& g) {
  if (!g.wrap) return 0.0f;
  const float half = 0.5f * (float)g.W;
  const float cx = (float)(tx * g.tile_w) + 0.5f * (float)g.tile_w;
  const float d = x - cx;
  return d > half ? -(float)g.W : (d < -half ? (float)g.W : 0.0f);
}

// small column-major 3x3 matrix with GLM's element convention: c[col][row]
struct Mat3 {
  float c[3][3];
};

// GLM-convention product: (A*B)[j][i] = sum_k A[k][i] * B[j][k], k ascending
__device__ __forceinline__ Mat3 mat_mul(const Mat3& A, const Mat3& B) {
  Mat3 o;
#pragma unroll
  for (int j = 0; j < 3; ++j)
#pragma unroll
    for (int i = 0; i < 3; ++i)
      o.c[j][i] = A.c[0][i] * B.c[j][0] + A.c[1][i] * B.c[j][1] + A.c[2][i] * B.c[j][2];
  return o;
}

__device__ __forceinline__ Mat3 mat_T(const Mat3& A) {
  Mat3 o;
#pragma unroll
  for (int j = 0; j < 3; ++j)
#pragma unroll
    for (int i = 0; i < 3; ++i) o.c[j][i] = A.c[i][j];
  return o;
}

// rotation matrix of a (normalised) quaternion q = (r, x, y, z), columns as
// the reference's mat3 constructor (forward.cu:131-138)
__device__ __forceinline__ Mat3 quat_to_rot(const float4 q) {
  const float r = q.x, x = q.y, y = q.z, z = q.w;
  Mat3 R;
  R.c[0][0] = 1.f - 2.f * (y * y + z * z); R.c[0][1] = 2.f * (x * y - r * z); R.c[0][2] = 2.f * (x * z + r * y);
  R.c[1][0] = 2.f * (x * y + r * z); R.c[1][1] = 1.f - 2.f * (x * x + z * z); R.c[1][2] = 2.f * (y * z - r * x);
  R.c[2][0] = 2.f * (x * z - r * y); R.c[2][1] = 2.f * (y * z + r * x); R.c[2][2] = 1.f - 2.f * (x * x + y * y);
  return R;
}

// M = S * R with S = diag(s) (forward.cu:126-140)
__device__ __forceinline__ Mat3 scale_rot(const float3 s, const Mat3& R) {
  Mat3 S;
#pragma unroll
  for (int j = 0; j < 3; ++j)
#pragma unroll
    for (int i = 0; i < 3; ++i) S.c[j][i] = 0.0f;
  S.c[0][0] = s.x; S.c[1][1] = s.y; S.c[2][2] = s.z;
  return mat_mul(S, R);
}

// view rotation as the reference builds it from the flat matrix (forward.cu:104-107)
__device__ __forceinline__ Mat3 view_rot(const float* m) {
  Mat3 W;
  W.c[0][0] = m[0]; W.c[0][1] = m[4]; W.c[0][2] = m[8];
  W.c[1][0] = m[1]; W.c[1][1] = m[5]; W.c[1][2] = m[9];
  W.c[2][0] = m[2]; W.c[2][1] = m[6]; W.c[2][2] = m[10];
  return W;
}

__device__ __forceinline__ Mat3 sym_from6(const float* v) {
  Mat3 V;
  V.c[0][0] = v[0]; V.c[0][1] = v[1]; V.c[0][2] = v[2];
  V.c[1][0] = v[1]; V.c[1][1] = v[3]; V.c[1][2] = v[4];
  V.c[2][0] = v[2]; V.c[2][1] = v[4]; V.c[2][2] = v[5];
  return V;
}

// Equirectangular projection Jacobian rows (forward.cu:82-102).  x_scale is
// 1 in the forward; the reference backward multiplies the azimuth row by 0.5
// (backward.cu:172-173), reproduced when the reference-compatible gradient
// mode is selected.
struct ProjJac {
  float J00, J02, J10, J11, J12;
  float trxztrxz, trxztrxz_inv, trxz, trxz_inv, trtr, trtr_inv, W_div_2pi, H_div_pi;
};

__device__ __forceinline__ ProjJac proj_jacobian(const float3 t, int width, int height) {
  ProjJac j;
  j.trxztrxz = t.x * t.x + t.z * t.z;
  j.trxztrxz_inv = 1.0f / (j.trxztrxz + 1e-7f);
  j.trxz = sqrtf(j.trxztrxz);
  j.trxz_inv = 1.0f / (j.trxz + 1e-7f);
  j.trtr = j.trxztrxz + t.y * t.y;
  j.trtr_inv = 1.0f / (j.trtr + 1e-7f);
  j.W_div_2pi = width * 0.5f * kInvPi;
  j.H_div_pi = height * kInvPi;
  j.J00 = j.W_div_2pi * t.z * j.trxztrxz_inv;
  j.J02 = -j.W_div_2pi * t.x * j.trxztrxz_inv;
  j.J10 = -j.H_div_pi * t.x * t.y * j.trxz_inv * j.trtr_inv;
  j.J11 = j.H_div_pi * j.trxz * j.trtr_inv;
  j.J12 = -j.H_div_pi * t.z * t.y * j.trxz_inv * j.trtr_inv;
  return j;
}

__device__ __forceinline__ Mat3 jac_mat(float J00, float J02, float J10, float J11, float J12) {
  Mat3 J;
  J.c[0][0] = J00; J.c[0][1] = 0.0f; J.c[0][2] = J02;
  J.c[1][0] = J10; J.c[1][1] = J11; J.c[1][2] = J12;
  J.c[2][0] = 0.0f; J.c[2][1] = 0.0f; J.c[2][2] = 0.0f;
  return J;
}

// Conservative pixel box (x_lo, x_hi, y_lo, y_hi) of a splat: outside it
// the blend's alpha = min(0.99, o * exp(power)) stays below 1/255, so a warp
// whose pixels all lie outside may skip the entry without changing any result.
//  * alpha <= o, so o < 0.99/255 never reaches 1/255: empty box;
//  * otherwise contributing pixels satisfy Q = a dx^2 + 2 b dx dy + c dy^2 <=
//    2 ln(255 o); the box bounds that ellipse with a 2 % + 2e-3 margin on the
//    level and 1 % + 0.01 px on the half-widths, which covers the FP32
//    rounding of `power` whenever the conic is not near-degenerate;
//  * near-degenerate conics (b^2 > 0.99 ac), a non-positive determinant and
//    non-finite values give an unbounded box (never skipped); NaN positions
//    give NaN bounds, which every comparison treats as "do not skip".
__device__ __forceinline__ float4 footprint_box(const float2 xy, const float4 co) {
  const float inf = __int_as_float(0x7f800000);
  const float l = logf(255.0f * co.w);
  if (l < -0.01f) return make_float4(inf, -inf, inf, -inf);
  const float q0 = fmaxf(l, 0.0f) * 2.04f + 2e-3f;
  const float ac = co.x * co.z;
  const float det = ac - co.y * co.y;
  const float ex = sqrtf(q0 * co.z / det) * 1.01f + 0.01f;
  const float ey = sqrtf(q0 * co.x / det) * 1.01f + 0.01f;
  if (!(det > 0.0f) || !(co.y * co.y <= 0.99f * ac) || !(ex < 1e30f) || !(ey < 1e30f))
    return make_float4(-inf, inf, -inf, inf);
  return make_float4(xy.x - ex, xy.x + ex, xy.y - ey, xy.y + ey);
}

// True when the box lies entirely outside the pixel rectangle [x0,x1]x[y0,y1]
// (false for NaN boxes).
__device__ __forceinline__ bool box_outside(const float4 b, float x0, float x1, float y0, float y1) {
  return b.y < x0 || b.x > x1 || b.w < y0 || b.z > y1;
}

// Two FP32 lanes per instruction (add / mul / fma .rn.f32x2, sm_100): each
// lane rounds exactly as the scalar instruction.
__device__ __forceinline__ unsigned long long f2_bits(float2 v) {
  return ((unsigned long long)__float_as_uint(v.y) << 32) | __float_as_uint(v.x);
}
__device__ __forceinline__ float2 bits_f2(unsigned long long b) {
  return make_float2(__uint_as_float((unsigned)b), __uint_as_float((unsigned)(b >> 32)));
}
__device__ __forceinline__ float2 ffma2(float2 a, float2 b, float2 c) {
  unsigned long long d;
  asm("fma.rn.f32x2 %0, %1, %2, %3;" : "=l"(d) : "l"(f2_bits(a)), "l"(f2_bits(b)), "l"(f2_bits(c)));
  return bits_f2(d);
}
__device__ __forceinline__ float2 fmul2(float2 a, float2 b) {
  unsigned long long d;
  asm("mul.rn.f32x2 %0, %1, %2;" : "=l"(d) : "l"(f2_bits(a)), "l"(f2_bits(b)));
  return bits_f2(d);
}
__device__ __forceinline__ float2 fadd2(float2 a, float2 b) {
  unsigned long long d;
  asm("add.rn.f32x2 %0, %1, %2;" : "=l"(d) : "l"(f2_bits(a)), "l"(f2_bits(b)));
  return bits_f2(d);
}

__device__ __forceinline__ void atomic_or_error(ImageHeader* hdr, uint32_t bits) {
  atomicOr(&hdr->error, bits);
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

// Gaussian id read from a point list, clamped into [0, P) so a mismatched or
// corrupt arena can never index out of bounds; the error word records it.
__device__ __forceinline__ uint32_t checked_id(uint32_t id, int P, ImageHeader* hdr) {
  if (id >= (uint32_t)P) {
    atomic_or_error(hdr, kErrBadIndex);
    return 0u;
  }
  return id;
}

}  // namespace gsparc
