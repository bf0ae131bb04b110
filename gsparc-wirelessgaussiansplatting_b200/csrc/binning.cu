// Binning: per-(receiver, tile) segments sorted by depth.
//
// The reference duplicates one (tile << 32 | depth bits, gaussian id) pair per
// touched tile in Gaussian order and stable-radix-sorts all of them with CUB
// (rasterizer_impl.cu:102-143, :293-300), then finds tile boundaries
// (:149-171).  The sorted order it produces is: by tile, then by depth bits,
// then by Gaussian id (stability over an id-ordered input).
//
// Here the tile counts come from the preprocess histogram, so the segment
// boundaries (= the reference's tile ranges) are known after one scan.  Each
// instance is scattered straight into its segment as a 64-bit key
// (depth bits << 32 | gaussian id); the keys are unique, so sorting each
// segment by that key reproduces the reference order exactly without any
// stability requirement.  Segments are sorted independently, one CTA each,
// in shared memory (bitonic network) with a merge-path fallback for segments
// larger than shared memory.  Traffic is one scatter write plus one read and
// one write per instance, instead of 5 radix passes over the whole list.
#include "common.cuh"
#include "kernels.cuh"

namespace gsparc {

// ---- scan of per-segment counts -> ranges, cursors, K, chunk bases ---------
// One block; n = R*T segments (a few thousand at most for a spectrum batch).

// Exclusive scan of one value per thread over the 1024-thread block; every
// thread also receives the block total.
__device__ __forceinline__ unsigned long long block_exclusive_scan(unsigned long long local,
                                                                   unsigned long long* warp_tot,
                                                                   unsigned long long& total) {
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  unsigned long long incl = local;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const unsigned long long v = __shfl_up_sync(0xffffffffu, incl, o);
    if (lane >= o) incl += v;
  }
  if (lane == 31) warp_tot[wid] = incl;
  __syncthreads();
  if (wid == 0) {
    unsigned long long w = warp_tot[lane];
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const unsigned long long v = __shfl_up_sync(0xffffffffu, w, o);
      if (lane >= o) w += v;
    }
    warp_tot[lane] = w;   // inclusive over warps
  }
  __syncthreads();
  const unsigned long long excl = (wid ? warp_tot[wid - 1] : 0ull) + (incl - local);
  total = warp_tot[31];
  __syncthreads();
  return excl;
}

__global__ void __launch_bounds__(1024)
scan_segments_kernel(int n, const uint32_t* __restrict__ counts, uint2* __restrict__ ranges,
                     uint32_t* __restrict__ cursor, uint32_t* __restrict__ chunk_base,
                     ImageHeader* __restrict__ hdr) {
  __shared__ unsigned long long warp_tot[32];
  const int tid = threadIdx.x;
  unsigned long long carry = 0, carry_b = 0;
  for (int base = 0; base < n; base += 1024 * 4) {
    // each thread owns 4 consecutive segments of this chunk
    uint32_t c[4], nb[4];
    unsigned long long local = 0, local_b = 0;
#pragma unroll
    for (int k = 0; k < 4; ++k) {
      const int i = base + tid * 4 + k;
      c[k] = i < n ? counts[i] : 0u;
      nb[k] = c[k] ? (c[k] - 1u) / kBwdChunk : 0u;   // interior chunk boundaries of the segment
      local += c[k];
      local_b += nb[k];
    }
    unsigned long long tot, tot_b;
    unsigned long long start = carry + block_exclusive_scan(local, warp_tot, tot);
    unsigned long long start_b = carry_b + block_exclusive_scan(local_b, warp_tot, tot_b);
#pragma unroll
    for (int k = 0; k < 4; ++k) {
      const int i = base + tid * 4 + k;
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

// Flags a capacity overflow before any kernel writes into the binning arena.
__global__ void check_capacity_kernel(ImageHeader* hdr, unsigned long long capacity) {
  hdr->capacity = capacity;
  if (hdr->num_rendered > capacity) atomic_or_error(hdr, kErrCapacity);
}

// ---- scatter instances into their segments ---------------------------------
// grid (ceil(P/256), R).  Block-aggregated reservation: shared counters per
// tile, one global atomic per (block, tile), then shared-atomic slots.
__global__ void __launch_bounds__(256)
scatter_kernel(int P, TileGrid grid, GeomView geo, uint32_t* __restrict__ cursor,
               const ImageHeader* __restrict__ hdr, unsigned long long* __restrict__ keys) {
  if (hdr->error) return;
  extern __shared__ uint32_t sh[];
  uint32_t* cnt = sh;
  uint32_t* base = sh + grid.T;
  const int r = blockIdx.y;
  const int g = blockIdx.x * blockDim.x + threadIdx.x;
  for (int t = threadIdx.x; t < grid.T; t += blockDim.x) cnt[t] = 0;
  __syncthreads();
  int x0 = 0, y0 = 0, x1 = 0, y1 = 0;
  bool vis = false;
  unsigned long long lowkey = 0;
  if (g < P) {
    const size_t rg = (size_t)r * P + g;
    const int rad = geo.radii[rg];
    if (rad > 0) {
      vis = true;
      const float2 xy = geo.means2D[rg];
      tile_rect(xy.x, xy.y, rad, grid, x0, y0, x1, y1);
      lowkey = ((unsigned long long)__float_as_uint(geo.depth[rg]) << 32) | (unsigned long long)(uint32_t)g;
      for (int ty = y0; ty < y1; ++ty)
        for (int tx = x0; tx < x1; ++tx) atomicAdd(&cnt[ty * grid.gx + tx], 1u);
    }
  }
  __syncthreads();
  for (int t = threadIdx.x; t < grid.T; t += blockDim.x) {
    const uint32_t c = cnt[t];
    base[t] = c ? atomicAdd(&cursor[(size_t)r * grid.T + t], c) : 0u;
  }
  __syncthreads();
  if (vis) {
    for (int ty = y0; ty < y1; ++ty)
      for (int tx = x0; tx < x1; ++tx) {
        const uint32_t pos = atomicAdd(&base[ty * grid.gx + tx], 1u);
        keys[pos] = lowkey;
      }
  }
}

// ---- per-segment sort -------------------------------------------------------
// Two launches over all segments; each CTA returns at once unless its segment
// belongs to its size class:
//  * small (n <= kSmallCap): bitonic network in shared memory, 256 threads,
//    many CTAs per SM;
//  * large: each of 512 threads sorts 16 keys in registers, then merge-path
//    merges in shared memory (9 levels for 8192 keys -- far less shared-memory
//    traffic than a bitonic network's 91 passes); segments above kSortCap are
//    sorted in kSortCap chunks and merged through global memory.
constexpr int kSmallThreads = 256;
constexpr int kSmallCap = 2048;
constexpr int kSortThreads = 512;
constexpr int kPerThread = 16;
constexpr int kSortCap = kSortThreads * kPerThread;   // 8192 keys
// Shared-memory index with one pad slot per 16 keys: thread t's run
// [16t, 16t+16) then starts at 17t, so a warp's strided accesses spread over
// the banks (2-way) instead of all landing on one (32-way).
__device__ __forceinline__ int pidx(int i) { return i + (i >> 4); }
constexpr int kPadded = kSortCap + kSortCap / 16;    // 8704 keys per buffer, 2 x 68 KB

__device__ __forceinline__ void bitonic_sort_shared(unsigned long long* s, int npad) {
  for (int k = 2; k <= npad; k <<= 1) {
    for (int j = k >> 1; j > 0; j >>= 1) {
      for (int i = threadIdx.x; i < (npad >> 1); i += blockDim.x) {
        const int lo = ((i & ~(j - 1)) << 1) | (i & (j - 1));   // j is a power of two
        const int hi = lo + j;
        const bool up = (lo & k) == 0;
        const unsigned long long a = s[lo], b = s[hi];
        if ((a > b) == up) { s[lo] = b; s[hi] = a; }
      }
      __syncthreads();
    }
  }
}

__device__ __forceinline__ int next_pow2(int n) {
  int p = 1;
  while (p < n) p <<= 1;
  return p;
}

// Sorting network over a register array (all indices compile-time).
template <int N>
__device__ __forceinline__ void register_bitonic(unsigned long long (&a)[N]) {
#pragma unroll
  for (int k = 2; k <= N; k <<= 1)
#pragma unroll
    for (int j = k >> 1; j > 0; j >>= 1)
#pragma unroll
      for (int i = 0; i < N; ++i) {
        const int l = i ^ j;
        if (l > i) {
          const bool up = (i & k) == 0;
          const unsigned long long x = a[i], y = a[l];
          const bool sw = (x > y) == up;
          a[i] = sw ? y : x;
          a[l] = sw ? x : y;
        }
      }
}

// Sort kSortCap keys held in `a` (shared memory, pidx layout, padded with ~0)
// using `b` as the second buffer; returns the buffer holding the result.
__device__ unsigned long long* merge_sort_shared(unsigned long long* a, unsigned long long* b) {
  const int t = threadIdx.x;
  {
    unsigned long long r[kPerThread];
#pragma unroll
    for (int k = 0; k < kPerThread; ++k) r[k] = a[pidx(t * kPerThread + k)];
    register_bitonic<kPerThread>(r);
#pragma unroll
    for (int k = 0; k < kPerThread; ++k) a[pidx(t * kPerThread + k)] = r[k];
  }
  __syncthreads();
  unsigned long long* src = a;
  unsigned long long* dst = b;
  for (int width = kPerThread; width < kSortCap; width <<= 1) {
    const int out0 = t * kPerThread;
    const int base = (out0 / (2 * width)) * (2 * width);
    const int a0 = base, b0 = base + width;   // run starts (logical indices)
    const int d = out0 - base;
    // merge path: number of A elements among the first d outputs (A wins ties)
    int lo = max(0, d - width), hi = min(d, width);
    while (lo < hi) {
      const int mid = (lo + hi) >> 1;
      if (src[pidx(a0 + mid)] <= src[pidx(b0 + d - 1 - mid)]) lo = mid + 1;
      else hi = mid;
    }
    int i = lo, j = d - lo;
#pragma unroll
    for (int k = 0; k < kPerThread; ++k) {
      const unsigned long long x = i < width ? src[pidx(a0 + i)] : ~0ull;
      const unsigned long long y = j < width ? src[pidx(b0 + j)] : ~0ull;
      const bool take_a = (j >= width) || (i < width && x <= y);
      dst[pidx(out0 + k)] = take_a ? x : y;
      i += take_a ? 1 : 0;
      j += take_a ? 0 : 1;
    }
    __syncthreads();
    unsigned long long* tmp = src;
    src = dst;
    dst = tmp;
  }
  return src;
}

// Merge two sorted runs a[0:na), b[0:nb) into out[0:na+nb) with one CTA
// (merge path partitioning; keys are unique).
__device__ void merge_runs_cta(const unsigned long long* __restrict__ a, int na,
                               const unsigned long long* __restrict__ b, int nb,
                               unsigned long long* __restrict__ out) {
  const int total = na + nb;
  const int per = (total + blockDim.x - 1) / blockDim.x;
  const int d = min(total, (int)threadIdx.x * per);
  const int dend = min(total, d + per);
  int lo = max(0, d - nb), hi = min(d, na);
  while (lo < hi) {
    const int mid = (lo + hi) >> 1;
    if (a[mid] < b[d - mid - 1]) lo = mid + 1;
    else hi = mid;
  }
  int i = lo, j = d - lo;
  for (int o = d; o < dend; ++o) {
    const bool take_a = (j >= nb) || (i < na && a[i] < b[j]);
    out[o] = take_a ? a[i++] : b[j++];
  }
}

__global__ void __launch_bounds__(kSmallThreads)
segment_sort_small_kernel(const uint2* __restrict__ ranges, const ImageHeader* __restrict__ hdr,
                          const unsigned long long* __restrict__ keys, uint32_t* __restrict__ point_list) {
  if (hdr->error) return;
  __shared__ unsigned long long skeys[kSmallCap];
  const uint2 rg = ranges[blockIdx.x];
  const int n = (int)(rg.y - rg.x);
  if (n <= 0 || n > kSmallCap) return;
  const unsigned long long* seg = keys + rg.x;
  if (n == 1) {
    if (threadIdx.x == 0) point_list[rg.x] = (uint32_t)seg[0];
    return;
  }
  const int npad = next_pow2(n);
  for (int i = threadIdx.x; i < npad; i += blockDim.x) skeys[i] = i < n ? seg[i] : ~0ull;
  __syncthreads();
  bitonic_sort_shared(skeys, npad);
  for (int i = threadIdx.x; i < n; i += blockDim.x) point_list[rg.x + i] = (uint32_t)skeys[i];
}

__global__ void __launch_bounds__(kSortThreads)
segment_sort_large_kernel(const uint2* __restrict__ ranges, const ImageHeader* __restrict__ hdr,
                          unsigned long long* __restrict__ keys, unsigned long long* __restrict__ keys_alt,
                          uint32_t* __restrict__ point_list) {
  if (hdr->error) return;
  extern __shared__ unsigned long long smem[];
  unsigned long long* sa = smem;
  unsigned long long* sb = smem + kPadded;
  const uint2 rg = ranges[blockIdx.x];
  const int n = (int)(rg.y - rg.x);
  if (n <= kSmallCap) return;
  unsigned long long* seg = keys + rg.x;
  if (n <= kSortCap) {
    for (int i = threadIdx.x; i < kSortCap; i += blockDim.x) sa[pidx(i)] = i < n ? seg[i] : ~0ull;
    __syncthreads();
    const unsigned long long* res = merge_sort_shared(sa, sb);
    for (int i = threadIdx.x; i < n; i += blockDim.x) point_list[rg.x + i] = (uint32_t)res[pidx(i)];
    return;
  }
  // above kSortCap: sort chunks in shared memory, then merge runs through
  // global memory, ping-ponging keys <-> keys_alt
  for (int c0 = 0; c0 < n; c0 += kSortCap) {
    const int cn = min(kSortCap, n - c0);
    for (int i = threadIdx.x; i < kSortCap; i += blockDim.x) sa[pidx(i)] = i < cn ? seg[c0 + i] : ~0ull;
    __syncthreads();
    const unsigned long long* res = merge_sort_shared(sa, sb);
    for (int i = threadIdx.x; i < cn; i += blockDim.x) seg[c0 + i] = res[pidx(i)];
    __syncthreads();
  }
  unsigned long long* src = seg;
  unsigned long long* dst = keys_alt + rg.x;
  for (int width = kSortCap; width < n; width <<= 1) {
    for (int lo = 0; lo < n; lo += 2 * width) {
      const int na = min(width, n - lo);
      const int nb = max(0, min(width, n - lo - width));
      merge_runs_cta(src + lo, na, src + lo + na, nb, dst + lo);
    }
    __syncthreads();
    unsigned long long* t = src;
    src = dst;
    dst = t;
  }
  for (int i = threadIdx.x; i < n; i += blockDim.x) point_list[rg.x + i] = (uint32_t)src[i];
}

cudaError_t launch_scan_segments(int n, const uint32_t* counts, uint2* ranges, uint32_t* cursor,
                                 uint32_t* chunk_base, ImageHeader* hdr, cudaStream_t stream) {
  scan_segments_kernel<<<1, 1024, 0, stream>>>(n, counts, ranges, cursor, chunk_base, hdr);
  return cudaGetLastError();
}

cudaError_t launch_check_capacity(ImageView img, unsigned long long capacity, cudaStream_t stream) {
  check_capacity_kernel<<<1, 1, 0, stream>>>(img.hdr, capacity);
  return cudaGetLastError();
}

cudaError_t launch_scatter(int P, int R, const TileGrid& grid, const GeomView& geo, ImageView img, BinningView bin,
                           cudaStream_t stream) {
  if (P == 0 || R == 0) return cudaSuccess;
  const size_t smem = 2 * (size_t)grid.T * sizeof(uint32_t);
  if (smem > 48 * 1024) {
    cudaError_t e = cudaFuncSetAttribute(scatter_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
  }
  scatter_kernel<<<dim3((P + 255) / 256, R), 256, smem, stream>>>(P, grid, geo, img.cursor, img.hdr, bin.keys);
  return cudaGetLastError();
}

cudaError_t launch_segment_sort(int R, const TileGrid& grid, ImageView img, BinningView bin, cudaStream_t stream) {
  const size_t sort_smem = 2 * (size_t)kPadded * sizeof(unsigned long long);
  // set the shared-memory opt-in once per device, so later calls (including
  // ones made while a CUDA graph is being captured) only enqueue the launches
  static bool attr_done[64] = {false};
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return e;
  if (dev < 0 || dev >= 64 || !attr_done[dev]) {
    e = cudaFuncSetAttribute(segment_sort_large_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)sort_smem);
    if (e != cudaSuccess) return e;
    if (dev >= 0 && dev < 64) attr_done[dev] = true;
  }
  const int nseg = R * grid.T;
  if (nseg == 0) return cudaSuccess;
  segment_sort_small_kernel<<<nseg, kSmallThreads, 0, stream>>>(img.ranges, img.hdr, bin.keys, bin.point_list);
  e = cudaGetLastError();
  if (e != cudaSuccess) return e;
  segment_sort_large_kernel<<<nseg, kSortThreads, sort_smem, stream>>>(img.ranges, img.hdr, bin.keys, bin.keys_alt,
                                                                      bin.point_list);
  return cudaGetLastError();
}

}  // namespace gsparc
