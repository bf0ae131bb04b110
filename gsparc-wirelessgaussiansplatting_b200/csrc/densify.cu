// Densification on the device (gaussian.py:223-551, train.py:508-553).
//
// Statistics (train.py:508-516): per step, for every receiver and visible
// Gaussian, accum += |dL/dmeans2D[0:2]|, denom += 1, max_radii2D = max(., radius).
//
// densify_and_prune (gaussian.py:515-542) on the flat training state, as the
// reference sequences it: clone (grad >= threshold, largest scale <=
// percent_dense * extent; raw parameters copied, appended), then split
// (grad >= threshold, largest scale > percent_dense * extent; two copies
// appended with centre R(q) (s * z) + centre, z ~ N(0, 1), log-scale
// log(s / 1.2), the originals removed), then prune (opacity < min_opacity,
// largest scale > 0.1 extent when a screen-size limit is given -- the
// screen-radius test itself never fires there, the statistics having been
// reset by the appends -- and centres outside the scene box).  The new
// Gaussians start with zero Adam moments; the statistics restart at zero.
//
// Survivors keep the reference's order: kept originals, kept clones, kept
// first split copies, kept second split copies, each in index order.  The
// decision of every copy is known from its original (a clone is identical;
// a split copy has the original's opacity, scale / 1.2 and its sampled
// centre), so one classification pass gives four flags per Gaussian; their
// block counts are scanned and a gather pass writes the new state.
//
// The normal samples come from a counter-based generator (SplitMix64 of
// (seed, Gaussian, copy, axis), Box-Muller), so a run is reproducible; the
// reference draws them with torch.normal, so split centres agree with it in
// distribution, not value.
#include "common.cuh"
#include "kernels.cuh"

namespace gsparc {

namespace {
constexpr int kDensifyThreads = 256;

__device__ __forceinline__ unsigned long long splitmix64(unsigned long long x) {
  x += 0x9E3779B97F4A7C15ull;
  x = (x ^ (x >> 30)) * 0xBF58476D1CE4E5B9ull;
  x = (x ^ (x >> 27)) * 0x94D049BB133111EBull;
  return x ^ (x >> 31);
}
}  // namespace

// Standard normal sample for (seed, Gaussian g, copy k, axis d): two 24-bit
// uniforms in (0, 1] from one SplitMix64 draw, Box-Muller (cosine branch).
__device__ __forceinline__ float densify_normal(unsigned long long seed, int g, int k, int d) {
  const unsigned long long h = splitmix64(seed ^ splitmix64(((unsigned long long)g << 8) | (unsigned)(k * 4 + d)));
  const float u1 = (float)((h >> 40) + 1) * (1.0f / 16777216.0f);
  const float u2 = (float)(((h >> 16) & 0xFFFFFFull) + 1) * (1.0f / 16777216.0f);
  return sqrtf(-2.0f * logf(u1)) * cosf(6.283185307179586f * u2);
}

__global__ void densify_stats_kernel(int P, int R, const int* __restrict__ radii, const float* __restrict__ dmeans2D,
                                     float* __restrict__ accum, float* __restrict__ denom,
                                     float* __restrict__ max_radii) {
  const int g = blockIdx.x * blockDim.x + threadIdx.x;
  if (g >= P) return;
  float a = accum[g], n = denom[g], m = max_radii[g];
  for (int r = 0; r < R; ++r) {
    const size_t rg = (size_t)r * P + g;
    const int rad = radii[rg];
    if (rad > 0) {
      const float dx = dmeans2D[rg * 3], dy = dmeans2D[rg * 3 + 1];
      a += sqrtf(dx * dx + dy * dy);
      n += 1.0f;
      m = fmaxf(m, (float)rad);
    }
  }
  accum[g] = a;
  denom[g] = n;
  max_radii[g] = m;
}

struct DensifyArgs {
  int P;
  const float* centre;     // [P,3] raw (flat state segments)
  const float* log_scale;  // [P,3]
  const float* rotation;   // [P,4] (w, x, y, z), not normalised
  const float* opacity;    // [P] logits
  const float* accum;
  const float* denom;
  float grad_threshold, percent_dense, extent, min_opacity, max_screen_size;
  float lo[3], hi[3];      // scene box
  unsigned long long seed;
};

// rotation of the normalised quaternion (w, x, y, z) times v (utils.py build_rotation)
__device__ __forceinline__ float3 rotate(const float* q4, float3 v) {
  const float n = sqrtf(q4[0] * q4[0] + q4[1] * q4[1] + q4[2] * q4[2] + q4[3] * q4[3]);
  const float r = q4[0] / n, x = q4[1] / n, y = q4[2] / n, z = q4[3] / n;
  return make_float3((1 - 2 * (y * y + z * z)) * v.x + 2 * (x * y - r * z) * v.y + 2 * (x * z + r * y) * v.z,
                     2 * (x * y + r * z) * v.x + (1 - 2 * (x * x + z * z)) * v.y + 2 * (y * z - r * x) * v.z,
                     2 * (x * z - r * y) * v.x + 2 * (y * z + r * x) * v.y + (1 - 2 * (x * x + y * y)) * v.z);
}

__device__ __forceinline__ float3 split_centre(const DensifyArgs& a, int g, int k, float3 s) {
  const float3 z = make_float3(densify_normal(a.seed, g, k, 0), densify_normal(a.seed, g, k, 1),
                               densify_normal(a.seed, g, k, 2));
  const float3 d = rotate(a.rotation + 4 * (size_t)g, make_float3(s.x * z.x, s.y * z.y, s.z * z.z));
  const float* c = a.centre + 3 * (size_t)g;
  return make_float3(d.x + c[0], d.y + c[1], d.z + c[2]);
}

// the prune test of gaussian.py:522-534 for one Gaussian of the post-split state
__device__ __forceinline__ bool pruned(const DensifyArgs& a, float logit, float maxs, float3 c) {
  bool p = 1.0f / (1.0f + expf(-logit)) < a.min_opacity;
  if (a.max_screen_size > 0.0f) p = p || maxs > 0.1f * a.extent;
  p = p || c.x < a.lo[0] || c.y < a.lo[1] || c.z < a.lo[2] || c.x > a.hi[0] || c.y > a.hi[1] || c.z > a.hi[2];
  return p;
}

// Flags of Gaussian g: bit 0 keep the original, 1 keep its clone, 2 / 3 keep
// its first / second split copy.
__device__ __forceinline__ unsigned densify_flags(const DensifyArgs& a, int g) {
  const float n = a.denom[g];
  float grad = a.accum[g] / n;
  if (grad != grad) grad = 0.0f;   // 0/0 (never visible): NaN -> 0 as gaussian.py:517
  const float* ls = a.log_scale + 3 * (size_t)g;
  const float3 s = make_float3(expf(ls[0]), expf(ls[1]), expf(ls[2]));
  const float maxs = fmaxf(s.x, fmaxf(s.y, s.z));
  const bool sel = grad >= a.grad_threshold;
  const bool clone = sel && maxs <= a.percent_dense * a.extent;
  const bool split = sel && maxs > a.percent_dense * a.extent;
  const float logit = a.opacity[g];
  const float* c = a.centre + 3 * (size_t)g;
  const bool pr = pruned(a, logit, maxs, make_float3(c[0], c[1], c[2]));
  unsigned f = 0;
  if (!split && !pr) f |= 1u;
  if (clone && !pr) f |= 2u;
  if (split) {
    const float3 sc = make_float3(s.x / 1.2f, s.y / 1.2f, s.z / 1.2f);
    const float maxc = fmaxf(sc.x, fmaxf(sc.y, sc.z));
#pragma unroll
    for (int k = 0; k < 2; ++k)
      if (!pruned(a, logit, maxc, split_centre(a, g, k, s))) f |= 4u << k;
  }
  return f;
}

// Per block: counts of the four categories; work: flags [P], counts [4][nblk]
__global__ void __launch_bounds__(kDensifyThreads)
densify_classify_kernel(DensifyArgs a, unsigned* __restrict__ flags, int* __restrict__ counts, int nblk) {
  __shared__ int s_cnt[4];
  if (threadIdx.x < 4) s_cnt[threadIdx.x] = 0;
  __syncthreads();
  const int g = blockIdx.x * kDensifyThreads + threadIdx.x;
  const unsigned f = g < a.P ? densify_flags(a, g) : 0u;
  if (g < a.P) flags[g] = f;
#pragma unroll
  for (int c = 0; c < 4; ++c) {
    const int w = __popc(__ballot_sync(0xffffffffu, (f >> c) & 1u));
    if ((threadIdx.x & 31) == 0 && w) atomicAdd(&s_cnt[c], w);
  }
  __syncthreads();
  if (threadIdx.x < 4) counts[threadIdx.x * nblk + blockIdx.x] = s_cnt[threadIdx.x];
}

// One CTA: exclusive scan of each category's block counts into block bases
// (category c starts after all survivors of categories < c); totals[0] = P_new.
__global__ void __launch_bounds__(1024)
densify_scan_kernel(const int* __restrict__ counts, int* __restrict__ bases, int nblk, int* __restrict__ P_new) {
  __shared__ int s_part[1024];
  int carry_all = 0;
  for (int c = 0; c < 4; ++c) {
    int carry = 0;
    for (int b0 = 0; b0 < nblk; b0 += 1024) {
      const int b = b0 + threadIdx.x;
      const int v = b < nblk ? counts[c * nblk + b] : 0;
      s_part[threadIdx.x] = v;
      __syncthreads();
      for (int off = 1; off < 1024; off <<= 1) {   // inclusive Hillis-Steele scan
        const int t = threadIdx.x >= off ? s_part[threadIdx.x - off] : 0;
        __syncthreads();
        s_part[threadIdx.x] += t;
        __syncthreads();
      }
      if (b < nblk) bases[c * nblk + b] = carry_all + carry + s_part[threadIdx.x] - v;
      carry += s_part[1023];
      __syncthreads();
    }
    carry_all += carry;
  }
  if (threadIdx.x == 0) *P_new = carry_all;
}

struct DensifyOut {
  int P_new;
  float* params;        // new flat state (raw parameters)
  float* exp_avg;
  float* exp_avg_sq;
  size_t off[6];        // new segment offsets (centre, log-scale, rotation, opacity, MLP, confidence)
};
struct DensifyIn {
  const float* params;
  const float* exp_avg;
  const float* exp_avg_sq;
  size_t off[6];        // old segment offsets
  long long mlp_floats; // old MLP segment floats
  int per_gaussian_mlp; // 194 floats per Gaussian in four per-kind blocks, else one global segment
  int conf_floats;
};

// The per-Gaussian MLP blocks of gaussian.py's EmissionMLPs flat layout: fc1
// weights [P][96], fc1 bias [P][32], fc2 weights [P][64], fc2 bias [P][2].
__device__ __constant__ int kMlpBlock[4] = {96, 32, 64, 2};

__device__ void densify_write(const DensifyArgs& a, const DensifyIn& in, const DensifyOut& o, int g, int dst,
                              int kind /* 0 original, 1 clone, 2 / 3 split copy */) {
  const int Pn = o.P_new, P = a.P;
  const bool keep_moments = kind == 0;
  auto put = [&](int seg, int width, int j, float v, float m1, float m2) {
    const size_t oi = o.off[seg] + (size_t)dst * width + j;
    o.params[oi] = v;
    o.exp_avg[oi] = keep_moments ? m1 : 0.0f;
    o.exp_avg_sq[oi] = keep_moments ? m2 : 0.0f;
  };
  auto src = [&](int seg, int width, int j) { return in.off[seg] + (size_t)g * width + j; };
  float3 c = make_float3(in.params[src(0, 3, 0)], in.params[src(0, 3, 1)], in.params[src(0, 3, 2)]);
  if (kind >= 2) {
    const float* ls = in.params + src(1, 3, 0);
    c = split_centre(a, g, kind - 2, make_float3(expf(ls[0]), expf(ls[1]), expf(ls[2])));
  }
  const float cc[3] = {c.x, c.y, c.z};
  for (int j = 0; j < 3; ++j) put(0, 3, j, cc[j], in.exp_avg[src(0, 3, j)], in.exp_avg_sq[src(0, 3, j)]);
  for (int j = 0; j < 3; ++j) {
    float v = in.params[src(1, 3, j)];
    if (kind >= 2) v = logf(expf(v) / 1.2f);   // scaling_inverse_activation(s / (0.6 N)), N = 2
    put(1, 3, j, v, in.exp_avg[src(1, 3, j)], in.exp_avg_sq[src(1, 3, j)]);
  }
  for (int j = 0; j < 4; ++j) put(2, 4, j, in.params[src(2, 4, j)], in.exp_avg[src(2, 4, j)], in.exp_avg_sq[src(2, 4, j)]);
  put(3, 1, 0, in.params[src(3, 1, 0)], in.exp_avg[src(3, 1, 0)], in.exp_avg_sq[src(3, 1, 0)]);
  if (in.per_gaussian_mlp) {
    size_t ob = 0, nb = 0;
    for (int b = 0; b < 4; ++b) {
      const int w = kMlpBlock[b];
      for (int j = 0; j < w; ++j) {
        const size_t si = in.off[4] + ob + (size_t)g * w + j;
        const size_t oi = o.off[4] + nb + (size_t)dst * w + j;
        o.params[oi] = in.params[si];
        o.exp_avg[oi] = keep_moments ? in.exp_avg[si] : 0.0f;
        o.exp_avg_sq[oi] = keep_moments ? in.exp_avg_sq[si] : 0.0f;
      }
      ob += (size_t)P * w;
      nb += (size_t)Pn * w;
    }
  }
}

__global__ void __launch_bounds__(kDensifyThreads)
densify_apply_kernel(DensifyArgs a, DensifyIn in, DensifyOut o, const unsigned* __restrict__ flags,
                     const int* __restrict__ bases, int nblk) {
  __shared__ int s_warp[4][kDensifyThreads / 32];
  const int g = blockIdx.x * kDensifyThreads + threadIdx.x;
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  const unsigned f = g < a.P ? flags[g] : 0u;
  int rank[4];
#pragma unroll
  for (int c = 0; c < 4; ++c) {
    const unsigned m = __ballot_sync(0xffffffffu, (f >> c) & 1u);
    rank[c] = __popc(m & ((1u << lane) - 1u));
    if (lane == 0) s_warp[c][wid] = __popc(m);
  }
  __syncthreads();
#pragma unroll
  for (int c = 0; c < 4; ++c) {
    int before = 0;
    for (int w = 0; w < wid; ++w) before += s_warp[c][w];
    if ((f >> c) & 1u) densify_write(a, in, o, g, bases[c * nblk + blockIdx.x] + before + rank[c], c);
  }
  // the global segments (shared MLP, confidence MLP) are copied with their moments
  const size_t nthreads = (size_t)gridDim.x * kDensifyThreads, tid = (size_t)blockIdx.x * kDensifyThreads + threadIdx.x;
  if (!in.per_gaussian_mlp)
    for (size_t i = tid; i < (size_t)in.mlp_floats; i += nthreads) {
      o.params[o.off[4] + i] = in.params[in.off[4] + i];
      o.exp_avg[o.off[4] + i] = in.exp_avg[in.off[4] + i];
      o.exp_avg_sq[o.off[4] + i] = in.exp_avg_sq[in.off[4] + i];
    }
  for (size_t i = tid; i < (size_t)in.conf_floats; i += nthreads) {
    o.params[o.off[5] + i] = in.params[in.off[5] + i];
    o.exp_avg[o.off[5] + i] = in.exp_avg[in.off[5] + i];
    o.exp_avg_sq[o.off[5] + i] = in.exp_avg_sq[in.off[5] + i];
  }
}

// reset_opacity (gaussian.py:223-230): logit(min(sigmoid(x), 0.01)), its moments zeroed
__global__ void reset_opacity_kernel(int P, float* __restrict__ logit, float* __restrict__ m1, float* __restrict__ m2) {
  const int g = blockIdx.x * blockDim.x + threadIdx.x;
  if (g >= P) return;
  const float o = fminf(1.0f / (1.0f + expf(-logit[g])), 0.01f);
  float v = logf(o / (1.0f - o));
  if (v != v) v = 0.0f;
  logit[g] = fminf(fmaxf(v, -3.402823466e38f), 3.402823466e38f);
  m1[g] = 0.0f;
  m2[g] = 0.0f;
}

size_t densify_work_ints(int P) {
  const int nblk = (P + kDensifyThreads - 1) / kDensifyThreads;
  return (size_t)P + 8 * (size_t)nblk + 16;
}

cudaError_t launch_densify_stats(int P, int R, const int* radii, const float* dmeans2D, float* accum, float* denom,
                                 float* max_radii, cudaStream_t s) {
  if (P == 0) return cudaSuccess;
  densify_stats_kernel<<<(P + 255) / 256, 256, 0, s>>>(P, R, radii, dmeans2D, accum, denom, max_radii);
  return cudaGetLastError();
}

// box6: lo[3], hi[3] in host memory, passed to the kernels by value
static DensifyArgs make_args(int P, const float* params, const size_t* off, const float* accum, const float* denom,
                             float grad_threshold, float percent_dense, float extent, float min_opacity,
                             float max_screen_size, const float* box6, unsigned long long seed) {
  DensifyArgs a;
  a.P = P;
  a.centre = params + off[0];
  a.log_scale = params + off[1];
  a.rotation = params + off[2];
  a.opacity = params + off[3];
  a.accum = accum;
  a.denom = denom;
  a.grad_threshold = grad_threshold;
  a.percent_dense = percent_dense;
  a.extent = extent;
  a.min_opacity = min_opacity;
  a.max_screen_size = max_screen_size;
  for (int i = 0; i < 3; ++i) {
    a.lo[i] = box6[i];
    a.hi[i] = box6[3 + i];
  }
  a.seed = seed;
  return a;
}

cudaError_t launch_densify_count(int P, const float* params, const size_t* off, const float* accum,
                                 const float* denom, float grad_threshold, float percent_dense, float extent,
                                 float min_opacity, float max_screen_size, const float* box6,
                                 unsigned long long seed, int* work, int* P_new, cudaStream_t s) {
  const int nblk = (P + kDensifyThreads - 1) / kDensifyThreads;
  const DensifyArgs a = make_args(P, params, off, accum, denom, grad_threshold, percent_dense, extent, min_opacity,
                                  max_screen_size, box6, seed);
  unsigned* flags = reinterpret_cast<unsigned*>(work);
  int* counts = work + P;
  int* bases = counts + 4 * nblk;
  if (nblk > 0) densify_classify_kernel<<<nblk, kDensifyThreads, 0, s>>>(a, flags, counts, nblk);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return e;
  densify_scan_kernel<<<1, 1024, 0, s>>>(counts, bases, nblk, P_new);
  return cudaGetLastError();
}

cudaError_t launch_densify_apply(int P, int P_new, const float* params, const float* exp_avg, const float* exp_avg_sq,
                                 const size_t* off, long long mlp_floats, int per_gaussian_mlp, int conf_floats,
                                 float grad_threshold, float percent_dense, float extent, float min_opacity,
                                 float max_screen_size, const float* box6, unsigned long long seed, const int* work,
                                 float* new_params, float* new_exp_avg, float* new_exp_avg_sq, const size_t* new_off,
                                 cudaStream_t s) {
  const int nblk = (P + kDensifyThreads - 1) / kDensifyThreads;
  const DensifyArgs a = make_args(P, params, off, nullptr, nullptr, grad_threshold, percent_dense, extent,
                                  min_opacity, max_screen_size, box6, seed);
  DensifyIn in;
  in.params = params;
  in.exp_avg = exp_avg;
  in.exp_avg_sq = exp_avg_sq;
  for (int i = 0; i < 6; ++i) in.off[i] = off[i];
  in.mlp_floats = mlp_floats;
  in.per_gaussian_mlp = per_gaussian_mlp;
  in.conf_floats = conf_floats;
  DensifyOut o;
  o.P_new = P_new;
  o.params = new_params;
  o.exp_avg = new_exp_avg;
  o.exp_avg_sq = new_exp_avg_sq;
  for (int i = 0; i < 6; ++i) o.off[i] = new_off[i];
  const unsigned* flags = reinterpret_cast<const unsigned*>(work);
  const int* bases = work + P + 4 * nblk;
  densify_apply_kernel<<<nblk > 0 ? nblk : 1, kDensifyThreads, 0, s>>>(a, in, o, flags, bases, nblk);
  return cudaGetLastError();
}

cudaError_t launch_reset_opacity(int P, float* logit, float* m1, float* m2, cudaStream_t s) {
  if (P == 0) return cudaSuccess;
  reset_opacity_kernel<<<(P + 255) / 256, 256, 0, s>>>(P, logit, m1, m2);
  return cudaGetLastError();
}

}  // namespace gsparc
