// Binning: per-(receiver, tile) segments in depth order.
//
// The reference duplicates one (tile << 32 | depth bits, gaussian id) pair per
// touched tile in Gaussian order and stable-radix-sorts all of them with CUB
// (rasterizer_impl.cu:102-143, :293-300), then finds tile boundaries
// (:149-171).  The sorted order it produces is: by tile, then by depth bits,
// then by Gaussian id (stability over an id-ordered input).
//
// Here the order is built in two independent halves:
//  * the tile counts come from the preprocess histogram, so the segment
//    boundaries (= the reference's tile ranges) are known after one scan;
//  * each receiver's Gaussians are put in depth order once -- an LSD radix
//    sort (4 passes of 8 bits, decoupled look-back, stable) of one 32-bit
//    key per Gaussian, P keys instead of K instances -- which gives every
//    Gaussian its rank in (depth bits, id) order.
// Each instance is then scattered into its segment as that rank, and a
// segment in rank order is the reference's segment: ranks are unique, so a
// segment is placed by one CTA with a bitmap over the ranks (prefix
// popcounts give each rank's position) or, for short segments, a bitonic
// network in shared memory.
#include "common.cuh"
#include "kernels.cuh"

namespace gsparc {

// Flags a capacity overflow before any kernel writes into the binning arena.
__global__ void check_capacity_kernel(ImageHeader* hdr, unsigned long long capacity) {
  hdr->capacity = capacity;
  if (hdr->num_rendered > capacity) atomic_or_error(hdr, kErrCapacity);
}

// ---- per-receiver depth order: radix passes ---------------------------------
// grid (tiles, R), 256 threads, kSortTileKeys keys per CTA in striped order
// (key k*256 + t of the tile belongs to thread t), so the rank of a key among
// equal digits follows (slice k, warp, lane) = input order: stable.  Tiles
// are taken in ticket order; each CTA publishes its per-digit counts and
// looks back over earlier tiles' published counts (bounded spin; on give-up
// the error word gets kErrSortWait and the pass finishes with wrong offsets
// rather than waiting).
constexpr int kRadixThreads = 256;
constexpr int kRadixItems = kSortTileKeys / kRadixThreads;   // 8
constexpr uint32_t kLookbackSpins = 1u << 22;

__device__ __forceinline__ uint32_t ld_volatile_u32(const uint32_t* p) {
  return *reinterpret_cast<const volatile uint32_t*>(p);
}

// One pass over one tile.  ticketed: take the tile index from the pass's
// ticket counter (separate launches per pass, CTAs not all resident);
// otherwise tile = blockIdx.x (one cooperative launch, all CTAs resident).
// Keys and values are read with L1-bypassing loads: in the cooperative
// kernel the buffer a pass reads was written by other CTAs since this CTA
// last read it.
// Lanes of the warp whose valid 8-bit digit equals this lane's (0 for an
// invalid lane): eight ballots, one per digit bit (match.any serialises on
// the SM and is far slower here).
__device__ __forceinline__ unsigned match_digit(uint32_t d, bool ok) {
  unsigned m = __ballot_sync(0xffffffffu, ok);
#pragma unroll
  for (int b = 0; b < 8; ++b) {
    const bool bit = (d >> b) & 1u;
    const unsigned v = __ballot_sync(0xffffffffu, bit);
    m &= bit ? v : ~v;
  }
  return ok ? m : 0u;
}

struct RadixShared {
  uint32_t w[kRadixThreads / 32][256];   // per-warp digit counters, then per-warp digit offsets
  uint32_t run[256];
  uint32_t off[256];
  uint32_t wsum[kRadixThreads / 32];
  uint32_t tile;
};

// Ranking: warp w owns keys [256 w, 256 w + 256) of the tile, slice k of it
// being 32 consecutive keys (one per lane), so (warp, slice, lane) is input
// order.  Within a warp the slices are ranked against warp-private digit
// counters without block barriers (the lowest lane of each equal-digit group
// bumps the counter and broadcasts the old value); one column scan over the
// warps then gives each warp's offset per digit: a stable rank in the tile.
__device__ __forceinline__ void radix_pass_body(RadixShared& sh, int P, int pass, bool ticketed, GeomView geo,
                                                ImageHeader* __restrict__ hdr, uint32_t spin_limit) {
  auto& s_run = sh.run;
  auto& s_off = sh.off;
  auto& s_wsum = sh.wsum;
  const int R = gridDim.y, r = blockIdx.y;
  const int t = threadIdx.x, lane = t & 31, wid = t >> 5;
  const size_t ntiles = sort_tiles((size_t)P);
  const uint32_t* hist = geo.sort_state + (size_t)r * 1024 + pass * 256;
  uint32_t* ticket = geo.sort_state + (size_t)R * 1024 + (size_t)r * 4 + pass;
  uint32_t* flags = geo.sort_state + (size_t)R * 1028 + ((size_t)r * 4 + pass) * ntiles * 256;
  if (t == 0) sh.tile = ticketed ? atomicAdd(ticket, 1u) : blockIdx.x;
  uint32_t* cw = sh.w[wid];
#pragma unroll
  for (int d = lane; d < 256; d += 32) cw[d] = 0;
  __syncthreads();
  const uint32_t tile = sh.tile;
  const size_t base = (size_t)tile * kSortTileKeys + (size_t)wid * (32 * kRadixItems);
  const size_t roff = (size_t)r * P;
  const uint32_t* kin = ((pass & 1) ? geo.sort_key[1] : geo.sort_key[0]) + roff;
  const uint32_t* vin = ((pass & 1) ? geo.sort_val[1] : geo.sort_val[0]) + roff;
  const int shift = 8 * pass;

  const uint32_t h = __ldcg(hist + t);   // issued with the key loads
  uint32_t key[kRadixItems], val[kRadixItems], lr[kRadixItems];
  bool ok[kRadixItems];
#pragma unroll
  for (int k = 0; k < kRadixItems; ++k) {
    const size_t idx = base + (size_t)k * 32 + lane;
    ok[k] = idx < (size_t)P;
    key[k] = ok[k] ? __ldcg(kin + idx) : 0xffffffffu;
    val[k] = ok[k] ? (pass == 0 ? (uint32_t)idx : __ldcg(vin + idx)) : 0u;
  }
  const unsigned lt = (1u << lane) - 1u;
#pragma unroll
  for (int k = 0; k < kRadixItems; ++k) {
    const uint32_t d = (key[k] >> shift) & 255u;
    const unsigned peers = match_digit(d, ok[k]);
    const int leader = __ffs(peers) - 1;
    uint32_t old = 0;
    if (ok[k] && lane == leader) {
      old = cw[d];
      cw[d] = old + __popc(peers);
    }
    old = __shfl_sync(0xffffffffu, old, leader);
    lr[k] = old + __popc(peers & lt);
    __syncwarp();
  }
  __syncthreads();
  {   // thread t owns digit t: exclusive scan over the warps, tile total
    uint32_t c[kRadixThreads / 32];
#pragma unroll
    for (int w = 0; w < kRadixThreads / 32; ++w) c[w] = sh.w[w][t];
    uint32_t run = 0;
#pragma unroll
    for (int w = 0; w < kRadixThreads / 32; ++w) {
      sh.w[w][t] = run;
      run += c[w];
    }
    s_run[t] = run;
  }
  __syncthreads();
#pragma unroll
  for (int k = 0; k < kRadixItems; ++k)
    if (ok[k]) lr[k] += cw[(key[k] >> shift) & 255u];
  // global offset of each digit for this tile: digits below it over all keys
  // (exclusive scan of the histogram) + this digit in earlier tiles (look-back)
  uint32_t incl = h;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const uint32_t v = __shfl_up_sync(0xffffffffu, incl, o);
    if (lane >= o) incl += v;
  }
  if (lane == 31) s_wsum[wid] = incl;
  const uint32_t cnt = s_run[t];
  uint32_t* mine = flags + (size_t)tile * 256 + t;
  uint32_t excl = 0;
  if (tile == 0) {
    atomicExch(mine, (2u << 30) | cnt);
  } else {
    atomicExch(mine, (1u << 30) | cnt);
    // read the predecessors eight at a time (independent loads), then add
    // them in order until an inclusive prefix; re-read from the first one
    // not yet published
    long long j = (long long)tile - 1;
    uint32_t spins = 0;
    bool finished = false;
    while (!finished) {
      uint32_t f[8];
#pragma unroll
      for (int u = 0; u < 8; ++u) f[u] = j - u >= 0 ? ld_volatile_u32(flags + (size_t)(j - u) * 256 + t) : 0u;
      int used = 0;
      bool stalled = false;
#pragma unroll
      for (int u = 0; u < 8; ++u) {
        if (finished || stalled) continue;
        const uint32_t st = f[u] >> 30;
        if (st == 0) { stalled = true; continue; }   // j - u >= 0 here: tile 0 is always inclusive
        excl += f[u] & 0x3fffffffu;
        ++used;
        if (st == 2) finished = true;
      }
      j -= used;
      if (stalled && ++spins > spin_limit) {
        atomic_or_error(hdr, kErrSortWait);
        break;
      }
    }
    atomicExch(mine, (2u << 30) | (excl + cnt));
  }
  __syncthreads();
  uint32_t wbase = 0;
  for (int w = 0; w < wid; ++w) wbase += s_wsum[w];
  s_off[t] = wbase + incl - h + excl;
  __syncthreads();
  if (pass < 3) {
    uint32_t* kout = ((pass & 1) ? geo.sort_key[0] : geo.sort_key[1]) + roff;
    uint32_t* vout = ((pass & 1) ? geo.sort_val[0] : geo.sort_val[1]) + roff;
#pragma unroll
    for (int k = 0; k < kRadixItems; ++k)
      if (ok[k]) {
        const uint32_t dest = s_off[(key[k] >> shift) & 255u] + lr[k];
        if (dest < (uint32_t)P) {
          kout[dest] = key[k];
          vout[dest] = val[k];
        }
      }
  } else {
    uint32_t* sorted = geo.sort_val[0] + roff;
    uint32_t* rank = geo.rank + roff;
#pragma unroll
    for (int k = 0; k < kRadixItems; ++k)
      if (ok[k]) {
        const uint32_t dest = s_off[(key[k] >> shift) & 255u] + lr[k];
        if (dest < (uint32_t)P && val[k] < (uint32_t)P) {
          sorted[dest] = val[k];
          rank[val[k]] = dest;
        }
      }
  }
  __syncthreads();   // shared memory is reused by the next pass
}

// The binning capacity is recorded and K checked against it by the first CTA
// of the first pass, before any kernel that writes the binning arena runs.
__device__ __forceinline__ void capacity_check(ImageHeader* hdr, unsigned long long capacity) {
  if (blockIdx.x == 0 && blockIdx.y == 0 && threadIdx.x == 0) {
    hdr->capacity = capacity;
    if (hdr->num_rendered > capacity) atomic_or_error(hdr, kErrCapacity);
  }
}

__global__ void __launch_bounds__(kRadixThreads)
radix_pass_kernel(int P, int pass, GeomView geo, ImageHeader* __restrict__ hdr, unsigned long long capacity,
                  uint32_t spin_limit) {
  __shared__ RadixShared sh;
  if (pass == 0) capacity_check(hdr, capacity);
  radix_pass_body(sh, P, pass, true, geo, hdr, spin_limit);
}

// All four passes in one cooperative launch (every CTA resident), with a
// per-receiver barrier between passes: an arrival counter per (receiver,
// barrier) in the sort state, spun on with a bound (kErrSortWait on give-up).
__device__ __forceinline__ void receiver_barrier(uint32_t* counter, uint32_t expected, ImageHeader* hdr,
                                                 uint32_t spin_limit) {
  __syncthreads();
  if (threadIdx.x == 0) {
    __threadfence();
    atomicAdd(counter, 1u);
    uint32_t spins = 0;
    while (ld_volatile_u32(counter) < expected) {
      if (++spins > spin_limit) {
        atomic_or_error(hdr, kErrSortWait);
        break;
      }
    }
    __threadfence();
  }
  __syncthreads();
}

__global__ void __launch_bounds__(kRadixThreads)
radix_sort_coop_kernel(int P, GeomView geo, ImageHeader* __restrict__ hdr, unsigned long long capacity,
                       uint32_t spin_limit) {
  __shared__ RadixShared sh;
  capacity_check(hdr, capacity);
  // barrier counters share the (unused) ticket words of passes 1..3
  uint32_t* bars = geo.sort_state + (size_t)gridDim.y * 1024 + (size_t)blockIdx.y * 4;
  for (int pass = 0; pass < 4; ++pass) {
    radix_pass_body(sh, P, pass, false, geo, hdr, spin_limit);
    if (pass < 3) receiver_barrier(bars + pass + 1, gridDim.x, hdr, spin_limit);
  }
}

// ---- scatter instances (as depth ranks) into their segments ------------------
// grid (ceil(P/256), R).  Block-aggregated reservation: shared counters per
// tile, one global atomic per (block, tile), then shared-atomic slots.
__global__ void __launch_bounds__(256)
scatter_kernel(int P, TileGrid grid, GeomView geo, uint32_t* __restrict__ cursor,
               const ImageHeader* __restrict__ hdr, uint32_t* __restrict__ seg_rank) {
  if (hdr->error) return;
  extern __shared__ uint32_t sh[];
  uint32_t* cnt = sh;
  uint32_t* base = sh + grid.T;
  const int r = blockIdx.y;
  const int g = blockIdx.x * blockDim.x + threadIdx.x;
  for (int t = threadIdx.x; t < grid.T; t += blockDim.x) cnt[t] = 0;
  __syncthreads();
  TileSpan span{0, 0, 0, 0, grid.gx, 0};
  bool vis = false;
  uint32_t rk = 0;
  if (g < P) {
    const size_t rg = (size_t)r * P + g;
    const int rad = geo.radii[rg];
    if (rad > 0) {
      vis = true;
      const float2 xy = geo.means2D[rg];
      span = tile_span(xy.x, xy.y, rad, grid);
      rk = geo.rank[rg];
      for_each_tile(span, grid.gx, [&](int tile) { atomicAdd(&cnt[tile], 1u); });
    }
  }
  __syncthreads();
  for (int t = threadIdx.x; t < grid.T; t += blockDim.x) {
    const uint32_t c = cnt[t];
    base[t] = c ? atomicAdd(&cursor[(size_t)r * grid.T + t], c) : 0u;
  }
  __syncthreads();
  if (vis) {
    for_each_tile(span, grid.gx, [&](int tile) {
      const uint32_t pos = atomicAdd(&base[tile], 1u);
      seg_rank[pos] = rk;
    });
  }
}

// ---- segment placement ------------------------------------------------------
// One CTA per segment.  A segment's ranks are unique values below P, so:
//  * bitmap (P <= kBitmapMaxP, and the segment is not tiny next to P): set
//    one bit per rank, prefix-popcount the words per group of 8, then walk
//    the words in order, each set bit writing its id at the next position;
//  * short segments (n <= kPlaceSmall) otherwise: bitonic network over the
//    32-bit ranks in shared memory.
// The Gaussian id of rank q is the depth order's entry q.
constexpr int kPlaceThreads = 512;
constexpr int kPlaceSmall = 2048;
constexpr int kBitmapMaxP = kMaxBinningP;

__device__ __forceinline__ int next_pow2(int n) {
  int p = 1;
  while (p < n) p <<= 1;
  return p;
}

__global__ void __launch_bounds__(kPlaceThreads)
segment_place_kernel(int P, int T, const uint2* __restrict__ ranges, const ImageHeader* __restrict__ hdr,
                     const uint32_t* __restrict__ seg_rank, GeomView geo, uint32_t* __restrict__ point_list) {
  if (hdr->error) return;
  extern __shared__ uint32_t sm[];
  __shared__ uint32_t warp_tot[32];
  const int seg = blockIdx.x, r = seg / T;
  const uint2 rg = ranges[seg];
  const int n = (int)(rg.y - rg.x);
  if (n <= 0) return;
  const uint32_t* ids = geo.sort_val[0] + (size_t)r * P;
  const uint32_t* sr = seg_rank + rg.x;
  uint32_t* out = point_list + rg.x;
  auto id_of = [&](uint32_t q) { return q < (uint32_t)P ? ids[q] : 0xffffffffu; };
  const bool bitmap = P <= kBitmapMaxP && (n > kPlaceSmall || (size_t)n * 256 >= (size_t)P);
  if (!bitmap) {
    const int npad = next_pow2(n);
    for (int i = threadIdx.x; i < npad; i += blockDim.x) sm[i] = i < n ? sr[i] : 0xffffffffu;
    __syncthreads();
    for (int k = 2; k <= npad; k <<= 1)
      for (int j = k >> 1; j > 0; j >>= 1) {
        for (int i = threadIdx.x; i < (npad >> 1); i += blockDim.x) {
          const int lo = ((i & ~(j - 1)) << 1) | (i & (j - 1));
          const int hi = lo + j;
          const bool up = (lo & k) == 0;
          const uint32_t a = sm[lo], b = sm[hi];
          if ((a > b) == up) { sm[lo] = b; sm[hi] = a; }
        }
        __syncthreads();
      }
    for (int i = threadIdx.x; i < n; i += blockDim.x) out[i] = id_of(sm[i]);
    return;
  }
  const int words = (P + 31) >> 5, groups = (words + 7) >> 3;
  uint32_t* bm = sm;
  uint32_t* pre = sm + words;
  for (int w = threadIdx.x; w < words; w += blockDim.x) bm[w] = 0u;
  __syncthreads();
  // eight independent rank loads in flight per thread
  for (int i0 = threadIdx.x; i0 < n; i0 += 8 * kPlaceThreads) {
    uint32_t q[8];
#pragma unroll
    for (int u = 0; u < 8; ++u) {
      const int i = i0 + u * kPlaceThreads;
      q[u] = i < n ? sr[i] : 0xffffffffu;
    }
#pragma unroll
    for (int u = 0; u < 8; ++u)
      if (q[u] < (uint32_t)P) atomicOr(&bm[q[u] >> 5], 1u << (q[u] & 31u));
  }
  __syncthreads();
  const int per = (groups + blockDim.x - 1) / blockDim.x;
  const int g0 = min(groups, (int)threadIdx.x * per), g1 = min(groups, g0 + per);
  uint32_t tsum = 0;
  for (int gi = g0; gi < g1; ++gi) {
    uint32_t c = 0;
    for (int w = gi * 8; w < min(words, gi * 8 + 8); ++w) c += __popc(bm[w]);
    pre[gi] = c;
    tsum += c;
  }
  uint32_t total;
  uint32_t off = cta_exclusive_scan<uint32_t>(tsum, warp_tot, total);
  for (int gi = g0; gi < g1; ++gi) {
    const uint32_t c = pre[gi];
    pre[gi] = off;
    off += c;
  }
  __syncthreads();
  // walk the bitmap in rank order: thread i of a round takes word w = round
  // base + i, so the 8 lanes of a group hold its 8 words; a word's first
  // position is its group's prefix plus the popcounts of the lanes before it
  // (a shuffle scan within the 8 lanes), and its set bits take the positions
  // after it in bit order.  A warp writes one contiguous run of the segment.
  const int lane = threadIdx.x & 31;
  for (int base = 0; base < words; base += kPlaceThreads) {
    const int w = base + (int)threadIdx.x;
    uint32_t bits = w < words ? bm[w] : 0u;
    const uint32_t c = __popc(bits);
    uint32_t incl = c;
#pragma unroll
    for (int d = 1; d < 8; d <<= 1) {
      const uint32_t o = __shfl_up_sync(0xffffffffu, incl, d, 8);
      if ((lane & 7) >= d) incl += o;
    }
    if (w < words) {
      uint32_t pos = pre[w >> 3] + incl - c;
      const uint32_t* idw = ids + ((size_t)w << 5);
      // up to eight set bits at a time: their id loads are issued together,
      // then stored in bit order (one load latency per eight bits, not per bit)
      while (bits) {
        uint32_t v[8];
        int m = 0;
#pragma unroll
        for (int u = 0; u < 8; ++u)
          if (bits) {
            const int b = __ffs(bits) - 1;
            bits &= bits - 1u;
            v[u] = idw[b];
            m = u + 1;
          }
#pragma unroll
        for (int u = 0; u < 8; ++u)
          if (u < m && pos + u < (uint32_t)n) out[pos + u] = v[u];
        pos += m;
      }
    }
  }
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
  scatter_kernel<<<dim3((P + 255) / 256, R), 256, smem, stream>>>(P, grid, geo, img.cursor, img.hdr, bin.seg_rank);
  return cudaGetLastError();
}

// One cooperative launch when every CTA of the sort fits on the GPU at once
// (the launch itself guarantees co-residency), else one launch per pass.
namespace {
// CTAs of the cooperative sort that fit on the current device at once (-1:
// no cooperative launch), looked up once per device.
cudaError_t coop_sort_capacity(int* dev_out, long long* cap) {
  static long long coop_capacity[64] = {0};
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return e;
  *dev_out = dev;
  *cap = -1;
  if (dev < 0 || dev >= 64) return cudaSuccess;
  if (coop_capacity[dev] == 0) {
    int per_sm = 0, sms = 0, coop = 0;
    if ((e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, radix_sort_coop_kernel, kRadixThreads, 0)) !=
        cudaSuccess)
      return e;
    if ((e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev)) != cudaSuccess) return e;
    if ((e = cudaDeviceGetAttribute(&coop, cudaDevAttrCooperativeLaunch, dev)) != cudaSuccess) return e;
    coop_capacity[dev] = coop ? (long long)per_sm * sms : -1;
  }
  *cap = coop_capacity[dev];
  return cudaSuccess;
}
}  // namespace

int depth_sort_launches(int P, int R) {
  if (P <= 0 || R <= 0) return 0;
  int dev = 0;
  long long cap = -1;
  if (coop_sort_capacity(&dev, &cap) != cudaSuccess) return -1;
  const long long ctas = (long long)sort_tiles((size_t)P) * R;
  return (cap > 0 && ctas <= cap) ? 1 : 4;
}

cudaError_t launch_depth_sort(int P, int R, const GeomView& geo, ImageView img, unsigned long long capacity,
                              cudaStream_t stream) {
  if (P == 0 || R == 0) return cudaSuccess;
  int dev = 0;
  long long cap = -1;
  cudaError_t e = coop_sort_capacity(&dev, &cap);
  if (e != cudaSuccess) return e;
  const dim3 grid((unsigned)sort_tiles((size_t)P), R);
  const long long ctas = (long long)grid.x * grid.y;
  const uint32_t spin_limit = wait_polls(kLookbackSpins);
  if (cap > 0 && ctas <= cap) {
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = grid;
    cfg.blockDim = dim3(kRadixThreads);
    cfg.dynamicSmemBytes = 0;
    cfg.stream = stream;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeCooperative;
    attr[0].val.cooperative = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    ImageHeader* hdr = img.hdr;
    return cudaLaunchKernelEx(&cfg, radix_sort_coop_kernel, P, geo, hdr, capacity, spin_limit);
  }
  for (int pass = 0; pass < 4; ++pass) {
    radix_pass_kernel<<<grid, kRadixThreads, 0, stream>>>(P, pass, geo, img.hdr, capacity, spin_limit);
    e = cudaGetLastError();
    if (e != cudaSuccess) return e;
  }
  return cudaSuccess;
}

size_t place_smem_bytes(int P) {
  const size_t words = ((size_t)P + 31) / 32, groups = (words + 7) / 8;
  const size_t bitmap = (words + groups) * sizeof(uint32_t);
  const size_t small = kPlaceSmall * sizeof(uint32_t);
  return P <= kBitmapMaxP ? (bitmap > small ? bitmap : small) : small;
}

cudaError_t launch_segment_place(int P, int R, const TileGrid& grid, const GeomView& geo, ImageView img,
                                 BinningView bin, cudaStream_t stream) {
  // the shared-memory opt-in is set once per device, so later calls (including
  // ones made while a CUDA graph is being captured) only enqueue the launch
  static bool attr_done[64] = {false};
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return e;
  if (dev < 0 || dev >= 64 || !attr_done[dev]) {
    e = cudaFuncSetAttribute(segment_place_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)place_smem_bytes(kBitmapMaxP));
    if (e != cudaSuccess) return e;
    if (dev >= 0 && dev < 64) attr_done[dev] = true;
  }
  const int nseg = R * grid.T;
  if (nseg == 0 || P == 0) return cudaSuccess;
  segment_place_kernel<<<nseg, kPlaceThreads, place_smem_bytes(P), stream>>>(P, grid.T, img.ranges, img.hdr,
                                                                             bin.seg_rank, geo, bin.point_list);
  return cudaGetLastError();
}

}  // namespace gsparc
