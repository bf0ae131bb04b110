// extern "C" entry points: argument checks, arena carving and launch order.
//
// Launch sequence of one forward (all on the caller's stream):
//   memset(header, counts, sort state) -> preprocess (+ tile and digit
//   histograms; its last CTA scans the tile counts)               [prepare]
//   depth sort (+ capacity check) -> scatter -> segment placement -> blend
//                                                                  [render]
// and of one backward:
//   memset(accumulated grads) -> blend adjoint -> geometry adjoint
//   -> emission-MLP adjoint.
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <atomic>
#include <mutex>
#include <vector>

#include <nvtx3/nvToolsExt.h>

#include "common.cuh"
#include "kernels.cuh"

using namespace gsparc;

namespace {

thread_local char g_detail[256] = "";

int cuda_fail(cudaError_t e, const char* where) {
  std::snprintf(g_detail, sizeof(g_detail), "%s: %s", where, cudaGetErrorString(e));
  return GSPARC_ERR_CUDA;
}

int invalid(const char* what) {
  std::snprintf(g_detail, sizeof(g_detail), "invalid argument: %s", what);
  return GSPARC_ERR_INVALID;
}

bool valid_tile(int th, int tw) {
  return th * tw == kBlendThreads && (th == 8 || th == 16 || th == 32) && (tw == 8 || tw == 16 || tw == 32);
}

#define GS_CHECK(call, where)                 \
  do {                                        \
    cudaError_t e_ = (call);                  \
    if (e_ != cudaSuccess) return cuda_fail(e_, where); \
  } while (0)

// ---- optional per-kernel timing (CUDA events around each launch) ----------
enum KernelId {
  KID_PREPROCESS, KID_CHECK, KID_SCATTER, KID_DEPTH_SORT, KID_PLACE, KID_BLEND_FWD, KID_BLEND_BWD,
  KID_GEOM_BWD, KID_MLP_BWD, KID_SSIM_FWD, KID_SSIM_BWD, KID_MARK_VISIBLE, KID_ADAM, KID_LOSS, KID_ACTIVATE, KID_SHARED_MLP, KID_SHARED_MLP_BWD,
  KID_BLEND_MC_FWD, KID_BLEND_MC_BWD, KID_EVAL, KID_DENSIFY, KID_MLP_FEAT_BWD,
  KID_COUNT
};
const char* const kKernelNames[KID_COUNT] = {
    "preprocess_kernel", "check_capacity_kernel", "scatter_kernel",
    "depth_sort_kernels", "segment_place_kernel", "blend_forward_kernel", "blend_backward_kernel", "geometry_backward_kernel",
    "emission_backward_kernel", "ssim_forward_kernel", "ssim_backward_kernel", "mark_visible_kernel",
    "gaussian_adam_kernels", "splat_loss_kernels", "gaussian_activate_kernel", "shared_mlp_forward_kernels",
    "shared_mlp_backward_kernels", "blend_channels_forward_kernel", "blend_channels_backward_kernel",
    "eval_metrics_kernel", "densify_kernels", "mlp_features_backward_kernel"};

struct PendingTiming {
  int id;
  cudaEvent_t a, b;
};
std::mutex g_tmu;
bool g_timing = false;
std::vector<PendingTiming> g_pending;
std::vector<cudaEvent_t> g_event_pool;
double g_ms[KID_COUNT] = {0};
long long g_launches[KID_COUNT] = {0};

cudaEvent_t pool_event() {
  if (!g_event_pool.empty()) {
    cudaEvent_t e = g_event_pool.back();
    g_event_pool.pop_back();
    return e;
  }
  cudaEvent_t e = nullptr;
  cudaEventCreate(&e);
  return e;
}

// Marks one pipeline stage: an NVTX range named after its kernels around the
// host-side launch (seen by profilers that record NVTX: stage names on the
// timeline, `ncu --nvtx --nvtx-include <stage>/` to capture one stage), and,
// when timing is enabled, an event pair around the launch.
struct Timed {
  int id;
  cudaStream_t s;
  cudaEvent_t a = nullptr;
  Timed(int id_, cudaStream_t s_) : id(id_), s(s_) {
    nvtxRangePushA(kKernelNames[id]);
    if (!g_timing) return;
    std::lock_guard<std::mutex> lk(g_tmu);
    a = pool_event();
    cudaEventRecord(a, s);
  }
  ~Timed() {
    nvtxRangePop();
    if (!a) return;
    std::lock_guard<std::mutex> lk(g_tmu);
    cudaEvent_t b = pool_event();
    cudaEventRecord(b, s);
    g_pending.push_back({id, a, b});
  }
};

}  // namespace

namespace {
std::atomic<long long> g_wait_limit{-1};   // < 0: every wait uses its own default bound
}  // namespace

namespace gsparc {
uint32_t wait_polls(uint32_t dflt) {
  const long long lim = g_wait_limit.load(std::memory_order_relaxed);
  return (lim < 0 || lim >= (long long)dflt) ? dflt : (uint32_t)lim;
}
// error reporting shared with entry points defined in other files
int report_invalid(const char* what) { return invalid(what); }
int report_cuda(cudaError_t e, const char* where) { return cuda_fail(e, where); }
}  // namespace gsparc

extern "C" {

int gsparc_abi_version(void) { return 7; }

const char* gsparc_status_string(int status) {
  switch (status) {
    case GSPARC_OK: return "ok";
    case GSPARC_ERR_INVALID: return "invalid argument";
    case GSPARC_ERR_CUDA: return "CUDA error";
    case GSPARC_ERR_CAPACITY: return "binning capacity exceeded";
    case GSPARC_ERR_DEVICE: return "device error word set";
    default: return "unknown status";
  }
}

const char* gsparc_last_error_detail(void) { return g_detail; }

size_t gsparc_geom_state_bytes(int P, int R) {
  if (P < 0 || R < 0) return 0;
  return carve_geom(nullptr, (size_t)P, (size_t)R, nullptr);
}

size_t gsparc_image_state_bytes(int R, int H, int W, int tile_h, int tile_w) {
  if (R < 0 || H <= 0 || W <= 0 || !valid_tile(tile_h, tile_w)) return 0;
  TileGrid g(H, W, tile_h, tile_w);
  return carve_image(nullptr, (size_t)R, (size_t)g.T, (size_t)H * W, nullptr);
}

size_t gsparc_binning_state_bytes(long long capacity) {
  if (capacity < 0) return 0;
  return carve_binning(nullptr, (size_t)capacity, nullptr);
}

int gsparc_geom_state_layout(int P, int R, size_t* o) {
  if (P < 0 || R < 0 || !o) return invalid("geom layout");
  GeomView v;
  char* base = (char*)(uintptr_t)4096;   // any non-null base; offsets are relative
  carve_geom(base, (size_t)P, (size_t)R, &v);
  o[0] = (char*)v.means2D - base; o[1] = (char*)v.depth - base; o[2] = (char*)v.radii - base;
  o[3] = (char*)v.conic_opacity - base; o[4] = (char*)v.signal - base; o[5] = (char*)v.cov3D - base;
  return GSPARC_OK;
}

int gsparc_image_state_layout(int R, int H, int W, int tile_h, int tile_w, size_t* o) {
  if (R < 0 || H <= 0 || W <= 0 || !valid_tile(tile_h, tile_w) || !o) return invalid("image layout");
  TileGrid g(H, W, tile_h, tile_w);
  ImageView v;
  char* base = (char*)(uintptr_t)4096;
  carve_image(base, (size_t)R, (size_t)g.T, (size_t)H * W, &v);
  o[0] = (char*)v.hdr - base; o[1] = (char*)v.ranges - base; o[2] = (char*)v.counts - base;
  o[3] = (char*)v.cursor - base; o[4] = (char*)v.final_T - base; o[5] = (char*)v.n_contrib - base;
  return GSPARC_OK;
}

int gsparc_binning_state_layout(long long capacity, size_t* o) {
  if (capacity < 0 || !o) return invalid("binning layout");
  BinningView v;
  char* base = (char*)(uintptr_t)4096;
  carve_binning(base, (size_t)capacity, &v);
  o[0] = (char*)v.seg_rank - base; o[1] = (char*)v.point_list - base; o[2] = (char*)v.ckpt - base;
  return GSPARC_OK;
}

int gsparc_rasterize_prepare(int P, int R, int H, int W, int tile_h, int tile_w, unsigned int flags,
                             float scale_modifier,
                             const float* means3D, const float* emission_mlps, const float* opacities,
                             const float* scales, const float* rotations, const float* viewmatrices,
                             const float* tx_pos, const float* rx_pos, int* radii_out, void* geom_state,
                             void* image_state, long long* num_rendered, void* stream) {
  if (P < 0 || R < 1 || H <= 0 || W <= 0) return invalid("sizes (need P >= 0, R >= 1, H, W > 0)");
  if (P > kMaxBinningP) return invalid("P above 1048576 Gaussians per call (the binning's rank bitmap limit)");
  if (R > 65535) return invalid("R above 65535 receivers per call");
  if (!valid_tile(tile_h, tile_w)) return invalid("tile shape must be 16x16, 8x32 or 32x8");
  if (!image_state || !viewmatrices || !tx_pos || !rx_pos) return invalid("null state or receiver pointer");
  if (P > 0 && (!geom_state || !means3D || !opacities || !scales || !rotations))
    return invalid("null Gaussian pointer");
  cudaStream_t s = (cudaStream_t)stream;
  if (flags & ~GSPARC_FLAG_WRAP_AZIMUTH) return invalid("unknown flags");
  TileGrid grid(H, W, tile_h, tile_w, (flags & GSPARC_FLAG_WRAP_AZIMUTH) ? 1 : 0);
  GeomView geo{};
  if (geom_state) carve_geom((char*)geom_state, (size_t)P, (size_t)R, &geo);
  ImageView img;
  carve_image((char*)image_state, (size_t)R, (size_t)grid.T, (size_t)H * W, &img);
  GS_CHECK(cudaMemsetAsync(img.hdr, 0, sizeof(ImageHeader), s), "memset header");
  GS_CHECK(cudaMemsetAsync(img.counts, 0, (size_t)R * grid.T * sizeof(uint32_t), s), "memset counts");
  if (P > 0)
    GS_CHECK(cudaMemsetAsync(geo.sort_state, 0, sort_state_words((size_t)P, (size_t)R) * sizeof(uint32_t), s),
             "memset sort state");
  {
    Timed t(KID_PREPROCESS, s);
    GS_CHECK(launch_preprocess(P, R, H, W, grid, scale_modifier, means3D, emission_mlps, opacities, scales,
                               rotations, viewmatrices, tx_pos, rx_pos, geo, radii_out, img, s),
             "preprocess");
  }
  if (P == 0) {   // no preprocess CTA to scan: empty segments
    GS_CHECK(cudaMemsetAsync(img.ranges, 0, (size_t)R * grid.T * sizeof(uint2), s), "memset ranges");
    GS_CHECK(cudaMemsetAsync(img.chunk_base, 0, ((size_t)R * grid.T + 1) * sizeof(uint32_t), s), "memset chunks");
  }
  if (num_rendered) {
    unsigned long long k = 0;
    GS_CHECK(cudaMemcpyAsync(&k, &img.hdr->num_rendered, sizeof(k), cudaMemcpyDeviceToHost, s), "read K");
    GS_CHECK(cudaStreamSynchronize(s), "sync K");
    *num_rendered = (long long)k;
  }
  return GSPARC_OK;
}

namespace {
// The binning stages shared by the single- and multi-channel renders: depth
// order, instance scatter, segment placement.
int render_binning(int P, int R, const TileGrid& grid, GeomView& geo, ImageView& img, BinningView& bin,
                   long long capacity, cudaStream_t s) {
  if (P == 0) {
    Timed t(KID_CHECK, s);
    GS_CHECK(launch_check_capacity(img, (unsigned long long)capacity, s), "capacity check");
  } else {
    Timed t(KID_DEPTH_SORT, s);   // also records the capacity and flags K > capacity
    GS_CHECK(launch_depth_sort(P, R, geo, img, (unsigned long long)capacity, s), "depth sort");
  }
  {
    Timed t(KID_SCATTER, s);
    GS_CHECK(launch_scatter(P, R, grid, geo, img, bin, s), "scatter");
  }
  {
    Timed t(KID_PLACE, s);
    GS_CHECK(launch_segment_place(P, R, grid, geo, img, bin, s), "segment place");
  }
  return GSPARC_OK;
}
}  // namespace

int gsparc_rasterize_render(int P, int R, int H, int W, int tile_h, int tile_w, unsigned int flags,
                            const void* geom_state,
                            void* image_state, void* binning_state, long long capacity, float* out_real,
                            float* out_imag, void* stream) {
  if (P < 0 || R < 1 || H <= 0 || W <= 0 || capacity < 0) return invalid("sizes");
  if (!valid_tile(tile_h, tile_w)) return invalid("tile shape must be 16x16, 8x32 or 32x8");
  if (!image_state || !out_real || !out_imag) return invalid("null image state or output");
  if (capacity > 0 && !binning_state) return invalid("null binning state");
  if (P > 0 && !geom_state) return invalid("null geometry state");
  cudaStream_t s = (cudaStream_t)stream;
  if (flags & ~GSPARC_FLAG_WRAP_AZIMUTH) return invalid("unknown flags");
  TileGrid grid(H, W, tile_h, tile_w, (flags & GSPARC_FLAG_WRAP_AZIMUTH) ? 1 : 0);
  GeomView geo{};
  if (geom_state) carve_geom((char*)geom_state, (size_t)P, (size_t)R, &geo);
  ImageView img;
  carve_image((char*)image_state, (size_t)R, (size_t)grid.T, (size_t)H * W, &img);
  BinningView bin{};
  carve_binning((char*)binning_state, (size_t)capacity, &bin);
  int st = render_binning(P, R, grid, geo, img, bin, capacity, s);
  if (st != GSPARC_OK) return st;
  {
    Timed t(KID_BLEND_FWD, s);
    GS_CHECK(launch_blend_forward(P, R, H, W, grid, geo, img, bin, out_real, out_imag, s), "blend forward");
  }
  return GSPARC_OK;
}

int gsparc_rasterize_render_channels(int P, int R, int H, int W, int tile_h, int tile_w, unsigned int flags, int C,
                                     const void* geom_state, void* image_state, void* binning_state,
                                     long long capacity, const float* features, float* out, void* stream) {
  if (P < 0 || R < 1 || H <= 0 || W <= 0 || capacity < 0) return invalid("sizes");
  if (C < 1 || C > kMaxChannels) return invalid("channels must be in [1, 64]");
  if (!valid_tile(tile_h, tile_w)) return invalid("tile shape must be 16x16, 8x32 or 32x8");
  if (!image_state || !out) return invalid("null image state or output");
  if (capacity > 0 && !binning_state) return invalid("null binning state");
  if (P > 0 && (!geom_state || !features)) return invalid("null geometry state or features");
  cudaStream_t s = (cudaStream_t)stream;
  if (flags & ~GSPARC_FLAG_WRAP_AZIMUTH) return invalid("unknown flags");
  TileGrid grid(H, W, tile_h, tile_w, (flags & GSPARC_FLAG_WRAP_AZIMUTH) ? 1 : 0);
  GeomView geo{};
  if (geom_state) carve_geom((char*)geom_state, (size_t)P, (size_t)R, &geo);
  ImageView img;
  carve_image((char*)image_state, (size_t)R, (size_t)grid.T, (size_t)H * W, &img);
  BinningView bin{};
  carve_binning((char*)binning_state, (size_t)capacity, &bin);
  int st = render_binning(P, R, grid, geo, img, bin, capacity, s);
  if (st != GSPARC_OK) return st;
  {
    Timed t(KID_BLEND_MC_FWD, s);
    GS_CHECK(launch_blend_channels_forward(P, R, H, W, C, grid, geo, img, bin, features, out, s),
             "blend forward (channels)");
  }
  return GSPARC_OK;
}

int gsparc_read_status(const void* image_state, long long* num_rendered, unsigned int* error_word, void* stream) {
  if (!image_state) return invalid("null image state");
  cudaStream_t s = (cudaStream_t)stream;
  ImageHeader h;
  GS_CHECK(cudaMemcpyAsync(&h, image_state, 16, cudaMemcpyDeviceToHost, s), "read header");
  GS_CHECK(cudaStreamSynchronize(s), "sync header");
  if (num_rendered) *num_rendered = (long long)h.num_rendered;
  if (error_word) *error_word = h.error;
  if (h.error & kErrCapacity) return GSPARC_ERR_CAPACITY;
  if (h.error) return GSPARC_ERR_DEVICE;
  return GSPARC_OK;
}

int gsparc_rasterize_backward(int P, int R, int H, int W, int tile_h, int tile_w, unsigned int flags,
                              float scale_modifier,
                              unsigned int grad_mode, const float* means3D, const float* emission_mlps,
                              const float* scales, const float* rotations, const float* viewmatrices,
                              const float* tx_pos, const float* rx_pos, const void* geom_state,
                              const void* image_state, const void* binning_state, long long binning_capacity,
                              const float* dL_dout_real, const float* dL_dout_imag, float* dL_dmeans2D,
                              float* dL_dconic, float* dL_dsignal, float* dL_dopacity, float* dL_dmeans3D,
                              float* dL_dcov3D, float* dL_dscales, float* dL_drotations, float* dL_demission_mlps,
                              void* stream) {
  if (P < 0 || R < 1 || H <= 0 || W <= 0 || binning_capacity < 0) return invalid("sizes");
  if (!valid_tile(tile_h, tile_w)) return invalid("tile shape must be 16x16, 8x32 or 32x8");
  if (grad_mode != GSPARC_GRAD_REFERENCE && grad_mode != GSPARC_GRAD_EXACT) return invalid("grad_mode");
  if (!image_state || !dL_dout_real || !dL_dout_imag || !viewmatrices || !tx_pos || !rx_pos)
    return invalid("null image state, upstream gradient or receiver pointer");
  if (P == 0) return GSPARC_OK;
  if (!geom_state || !means3D || !scales || !rotations || !dL_dmeans2D || !dL_dconic || !dL_dsignal ||
      !dL_dopacity || !dL_dmeans3D || !dL_dcov3D || !dL_dscales || !dL_drotations)
    return invalid("null Gaussian input or gradient output");
  if ((emission_mlps == nullptr) != (dL_demission_mlps == nullptr))
    return invalid("emission_mlps and dL_demission_mlps: give both (per-Gaussian MLP) or neither (shared MLP)");
  if (binning_capacity > 0 && !binning_state) return invalid("null binning state");
  cudaStream_t s = (cudaStream_t)stream;
  if (flags & ~GSPARC_FLAG_WRAP_AZIMUTH) return invalid("unknown flags");
  TileGrid grid(H, W, tile_h, tile_w, (flags & GSPARC_FLAG_WRAP_AZIMUTH) ? 1 : 0);
  GeomView geo;
  carve_geom((char*)geom_state, (size_t)P, (size_t)R, &geo);
  ImageView img;
  carve_image((char*)image_state, (size_t)R, (size_t)grid.T, (size_t)H * W, &img);
  BinningView bin{};
  carve_binning((char*)binning_state, (size_t)binning_capacity, &bin);
  const size_t rp = (size_t)R * P;
  GS_CHECK(cudaMemsetAsync(dL_dmeans2D, 0, rp * 3 * sizeof(float), s), "memset dmeans2D");
  GS_CHECK(cudaMemsetAsync(dL_dconic, 0, rp * 4 * sizeof(float), s), "memset dconic");
  GS_CHECK(cudaMemsetAsync(dL_dsignal, 0, rp * 2 * sizeof(float), s), "memset dsignal");
  GS_CHECK(cudaMemsetAsync(dL_dopacity, 0, (size_t)P * sizeof(float), s), "memset dopacity");
  {
    Timed t(KID_BLEND_BWD, s);
    GS_CHECK(launch_blend_backward(P, R, H, W, grid, grad_mode, binning_capacity, geo, img, bin, dL_dout_real,
                                   dL_dout_imag, dL_dmeans2D, dL_dconic, dL_dsignal, dL_dopacity, s),
             "blend backward");
  }
  {
    Timed t(KID_GEOM_BWD, s);
    GS_CHECK(launch_geometry_backward(P, R, H, W, scale_modifier, grad_mode, means3D, scales, rotations,
                                      viewmatrices, geo, dL_dmeans2D, dL_dconic, dL_dmeans3D, dL_dcov3D, dL_dscales,
                                      dL_drotations, s),
             "geometry backward");
  }
  if (emission_mlps) {
    Timed t(KID_MLP_BWD, s);
    GS_CHECK(launch_emission_backward(P, R, means3D, emission_mlps, tx_pos, rx_pos, geo.radii, dL_dsignal,
                                      dL_demission_mlps, dL_dmeans3D, s),
             "emission backward");
  }
  return GSPARC_OK;
}

int gsparc_rasterize_backward_channels(int P, int R, int H, int W, int tile_h, int tile_w, unsigned int flags,
                                       int C, float scale_modifier, const float* means3D, const float* scales,
                                       const float* rotations, const float* viewmatrices, const void* geom_state,
                                       const void* image_state, const void* binning_state,
                                       long long binning_capacity, const float* features, const float* dL_dout,
                                       float* dL_dfeatures, float* dL_dmeans2D, float* dL_dconic,
                                       float* dL_dopacity, float* dL_dmeans3D, float* dL_dcov3D, float* dL_dscales,
                                       float* dL_drotations, void* stream) {
  if (P < 0 || R < 1 || H <= 0 || W <= 0 || binning_capacity < 0) return invalid("sizes");
  if (C < 1 || C > kMaxChannels) return invalid("channels must be in [1, 64]");
  if (!valid_tile(tile_h, tile_w)) return invalid("tile shape must be 16x16, 8x32 or 32x8");
  if (!image_state || !dL_dout || !viewmatrices) return invalid("null image state, upstream gradient or view");
  if (P == 0) return GSPARC_OK;
  if (!geom_state || !means3D || !scales || !rotations || !features || !dL_dfeatures || !dL_dmeans2D ||
      !dL_dconic || !dL_dopacity || !dL_dmeans3D || !dL_dcov3D || !dL_dscales || !dL_drotations)
    return invalid("null Gaussian input or gradient output");
  if (binning_capacity > 0 && !binning_state) return invalid("null binning state");
  cudaStream_t s = (cudaStream_t)stream;
  if (flags & ~GSPARC_FLAG_WRAP_AZIMUTH) return invalid("unknown flags");
  TileGrid grid(H, W, tile_h, tile_w, (flags & GSPARC_FLAG_WRAP_AZIMUTH) ? 1 : 0);
  GeomView geo;
  carve_geom((char*)geom_state, (size_t)P, (size_t)R, &geo);
  ImageView img;
  carve_image((char*)image_state, (size_t)R, (size_t)grid.T, (size_t)H * W, &img);
  BinningView bin{};
  carve_binning((char*)binning_state, (size_t)binning_capacity, &bin);
  const size_t rp = (size_t)R * P;
  GS_CHECK(cudaMemsetAsync(dL_dmeans2D, 0, rp * 3 * sizeof(float), s), "memset dmeans2D");
  GS_CHECK(cudaMemsetAsync(dL_dconic, 0, rp * 4 * sizeof(float), s), "memset dconic");
  GS_CHECK(cudaMemsetAsync(dL_dfeatures, 0, rp * (size_t)C * sizeof(float), s), "memset dfeatures");
  GS_CHECK(cudaMemsetAsync(dL_dopacity, 0, (size_t)P * sizeof(float), s), "memset dopacity");
  {
    Timed t(KID_BLEND_MC_BWD, s);
    GS_CHECK(launch_blend_channels_backward(P, R, H, W, C, grid, geo, img, bin, features, dL_dout, dL_dfeatures,
                                            dL_dmeans2D, dL_dconic, dL_dopacity, s),
             "blend backward (channels)");
  }
  {
    Timed t(KID_GEOM_BWD, s);
    GS_CHECK(launch_geometry_backward(P, R, H, W, scale_modifier, GSPARC_GRAD_EXACT, means3D, scales, rotations,
                                      viewmatrices, geo, dL_dmeans2D, dL_dconic, dL_dmeans3D, dL_dcov3D, dL_dscales,
                                      dL_drotations, s),
             "geometry backward");
  }
  return GSPARC_OK;
}

// ---- shared emission MLP -------------------------------------------------------

namespace {
int check_mlp_spec(int layers, int width, int act, int out, int precision) {
  if (layers < 1 || layers > kMaxMlpLayers) return invalid("layers must be in [1, 6]");
  if (width < 8 || width > 256) return invalid("width must be in [8, 256]");
  if (act != GSPARC_ACT_RELU && act != GSPARC_ACT_GELU) return invalid("act must be GSPARC_ACT_RELU or _GELU");
  if (out < 1 || out > kMaxChannels) return invalid("out must be in [1, 64]");
  if (precision != GSPARC_MLP_FP32 && precision != GSPARC_MLP_BF16) return invalid("precision");
  if (precision == GSPARC_MLP_BF16 && (width != 128 || layers > 3 || (out != 1 && out != 64)))
    return invalid("the BF16 tensor-core path needs width 128, at most 3 hidden layers and 1 or 64 outputs");
  return GSPARC_OK;
}
}  // namespace

size_t gsparc_shared_mlp_param_floats(int layers, int width, int out) {
  if (layers < 1 || layers > kMaxMlpLayers || width < 1 || out < 1) return 0;
  return shared_mlp_layout(layers, width, out, 0).params;
}

size_t gsparc_shared_mlp_workspace_floats(int P, int R, int layers, int width, int out, int precision) {
  if (P < 0 || R < 0 || layers < 1 || layers > kMaxMlpLayers || width < 1 || out < 1) return 0;
  if (precision == GSPARC_MLP_BF16) return shared_mlp_layout_bf16(layers, (size_t)P * R, out).work;
  return shared_mlp_layout(layers, width, out, (size_t)P * R).work;
}

int gsparc_shared_mlp_forward(int P, int R, int layers, int width, int act, int out, int precision,
                              const float* means3D, const float* rx_pos, const float* params, void* geom_state,
                              void* image_state, float* workspace, void* stream) {
  if (P < 0 || R < 1) return invalid("sizes");
  int st = check_mlp_spec(layers, width, act, out, precision);
  if (st != GSPARC_OK) return st;
  if (P == 0) return GSPARC_OK;
  if (!means3D || !rx_pos || !params || !geom_state || !workspace) return invalid("null pointer");
  if (precision == GSPARC_MLP_BF16 && ((uintptr_t)workspace & 255u) != 0)
    return invalid("the BF16 path needs a 256-byte aligned workspace");
  cudaStream_t s = (cudaStream_t)stream;
  GeomView geo;
  carve_geom((char*)geom_state, (size_t)P, (size_t)R, &geo);
  Timed t(KID_SHARED_MLP, s);
  if (precision == GSPARC_MLP_BF16) {
    GS_CHECK(launch_shared_mlp_bf16(true, P, R, layers, act, out, means3D, rx_pos, params, geo, workspace, nullptr,
                                    nullptr, nullptr, (ImageHeader*)image_state, s),
             "shared mlp forward (bf16)");
  } else {
    GS_CHECK(launch_shared_mlp_forward(P, R, layers, width, act, out, means3D, rx_pos, params, geo, workspace, s),
             "shared mlp forward");
  }
  return GSPARC_OK;
}

int gsparc_shared_mlp_backward(int P, int R, int layers, int width, int act, int out, int precision,
                               const float* means3D, const float* rx_pos, const float* params,
                               const void* geom_state, void* image_state, float* workspace,
                               const float* dL_dsignal, float* dL_dparams, float* dL_dmeans3D, void* stream) {
  if (P < 0 || R < 1) return invalid("sizes");
  int st = check_mlp_spec(layers, width, act, out, precision);
  if (st != GSPARC_OK) return st;
  if (!dL_dparams) return invalid("null dL_dparams");
  cudaStream_t s = (cudaStream_t)stream;
  if (P == 0) {
    GS_CHECK(cudaMemsetAsync(dL_dparams, 0, shared_mlp_layout(layers, width, out, 0).params * sizeof(float), s),
             "memset dL_dparams");
    return GSPARC_OK;
  }
  if (!means3D || !rx_pos || !params || !geom_state || !workspace || !dL_dsignal || !dL_dmeans3D)
    return invalid("null pointer");
  if (precision == GSPARC_MLP_BF16 && ((uintptr_t)workspace & 255u) != 0)
    return invalid("the BF16 path needs a 256-byte aligned workspace");
  GeomView geo;
  carve_geom((char*)geom_state, (size_t)P, (size_t)R, &geo);
  if (precision == GSPARC_MLP_BF16) {
    // the tensor-core adjoint, with the feature adjoint in its last step
    Timed t(KID_SHARED_MLP_BWD, s);
    GS_CHECK(launch_shared_mlp_bf16(false, P, R, layers, act, out, means3D, rx_pos, params, geo, workspace,
                                    dL_dsignal, dL_dparams, dL_dmeans3D, (ImageHeader*)image_state, s),
             "shared mlp backward (bf16)");
  } else {
    Timed t(KID_SHARED_MLP_BWD, s);
    GS_CHECK(launch_shared_mlp_backward(P, R, layers, width, act, out, means3D, rx_pos, params, geo, workspace,
                                        dL_dsignal, dL_dparams, dL_dmeans3D, s),
             "shared mlp backward");
  }
  return GSPARC_OK;
}

int gsparc_shared_mlp_bf16_act_table(int act, uint16_t* out, void* stream) {
  if (act != GSPARC_ACT_RELU && act != GSPARC_ACT_GELU) return invalid("act");
  if (!out) return invalid("null pointer");
  GS_CHECK(launch_bf16_act_table(act, out, (cudaStream_t)stream), "bf16 activation table");
  return GSPARC_OK;
}

int gsparc_mark_visible(int P, const float* means3D, const float* viewmatrix, uint8_t* present, void* stream) {
  if (P < 0) return invalid("P");
  if (P == 0) return GSPARC_OK;
  if (!means3D || !viewmatrix || !present) return invalid("null pointer");
  Timed t(KID_MARK_VISIBLE, (cudaStream_t)stream);
  GS_CHECK(launch_mark_visible(P, means3D, viewmatrix, present, (cudaStream_t)stream), "mark visible");
  return GSPARC_OK;
}

int gsparc_ssim_forward(int B, int CH, int H, int W, float C1, float C2, const float* img1, const float* img2,
                        float* ssim_map, float* dm_dmu1, float* dm_dsigma1_sq, float* dm_dsigma12, void* stream) {
  if (B < 0 || CH < 0 || H < 0 || W < 0) return invalid("sizes");
  if ((size_t)B * CH * H * W == 0) return GSPARC_OK;
  if (!img1 || !img2 || !ssim_map) return invalid("null image or map");
  const bool any_d = dm_dmu1 || dm_dsigma1_sq || dm_dsigma12;
  const bool all_d = dm_dmu1 && dm_dsigma1_sq && dm_dsigma12;
  if (any_d && !all_d) return invalid("derivative maps must be all NULL or all non-NULL");
  Timed t(KID_SSIM_FWD, (cudaStream_t)stream);
  GS_CHECK(launch_ssim_forward(B * CH, H, W, C1, C2, img1, img2, ssim_map, dm_dmu1, dm_dsigma1_sq, dm_dsigma12,
                               (cudaStream_t)stream),
           "ssim forward");
  return GSPARC_OK;
}

int gsparc_ssim_backward(int B, int CH, int H, int W, float C1, float C2, const float* img1, const float* img2,
                         const float* dL_dmap, const float* dm_dmu1, const float* dm_dsigma1_sq,
                         const float* dm_dsigma12, float* dL_dimg1, void* stream) {
  (void)C1;
  (void)C2;
  if (B < 0 || CH < 0 || H < 0 || W < 0) return invalid("sizes");
  if ((size_t)B * CH * H * W == 0) return GSPARC_OK;
  if (!img1 || !img2 || !dL_dmap || !dm_dmu1 || !dm_dsigma1_sq || !dm_dsigma12 || !dL_dimg1)
    return invalid("null pointer");
  Timed t(KID_SSIM_BWD, (cudaStream_t)stream);
  GS_CHECK(launch_ssim_backward(B * CH, H, W, img1, img2, dL_dmap, dm_dmu1, dm_dsigma1_sq, dm_dsigma12, dL_dimg1,
                                (cudaStream_t)stream),
           "ssim backward");
  return GSPARC_OK;
}

// ---- training loss -------------------------------------------------------------

size_t gsparc_splat_loss_scratch_floats(int R, int H, int W, int hidden) {
  if (R < 0 || H < 0 || W < 0 || hidden < 0) return 0;
  return loss_layout((size_t)R, (size_t)H, (size_t)W, (size_t)hidden).total;
}

int gsparc_splat_loss(int R, int H, int W, int hidden, float lambda1, float alpha, float C1, float C2,
                      const float* pred, const float* target, const float* rx_pos, const float* conf_params,
                      float* scratch, float* loss_out, float* terms, float* dL_dpred, float* dL_dconf_params,
                      void* stream) {
  if (R < 1 || H < 1 || W < 1) return invalid("R, H and W must be positive");
  if (R > 65535 || (H + 7) / 8 > 65535) return invalid("R or H too large for the tile grid");
  if ((size_t)H * W > (size_t)INT32_MAX) return invalid("H*W too large");
  if (hidden < 1 || hidden > 4096) return invalid("hidden must be in [1, 4096]");
  if (!pred || !target || !rx_pos || !conf_params || !scratch || !loss_out || !dL_dpred || !dL_dconf_params)
    return invalid("null pointer");
  if (((uintptr_t)scratch) & 15u) return invalid("scratch must be 16-byte aligned");
  cudaStream_t s = (cudaStream_t)stream;
  Timed t(KID_LOSS, s);
  GS_CHECK(launch_splat_loss(R, H, W, hidden, lambda1, alpha, C1, C2, pred, target, rx_pos, conf_params, scratch,
                             loss_out, terms, dL_dpred, dL_dconf_params, s),
           "splat loss");
  return GSPARC_OK;
}

// ---- evaluation metrics --------------------------------------------------------

size_t gsparc_eval_scratch_floats(int R, int H, int W) {
  if (R < 0 || H < 0 || W < 0) return 0;
  return eval_scratch_floats((size_t)R, (size_t)H, (size_t)W);
}

int gsparc_eval_metrics(int R, int H, int W, int hidden, float lambda1, float C1, float C2, const float* pred,
                        const float* target, const float* rx_pos, const float* conf_params, float* scratch,
                        float* metrics, void* stream) {
  if (R < 1 || H < 1 || W < 1) return invalid("R, H and W must be positive");
  if (R > 65535 || (H + 7) / 8 > 65535) return invalid("R or H too large for the block grid");
  if ((size_t)H * W > (size_t)INT32_MAX) return invalid("H*W too large");
  if (hidden < 1 || hidden > 4096) return invalid("hidden must be in [1, 4096]");
  if (!pred || !target || !rx_pos || !conf_params || !scratch || !metrics) return invalid("null pointer");
  if (((uintptr_t)scratch) & 15u) return invalid("scratch must be 16-byte aligned");
  cudaStream_t s = (cudaStream_t)stream;
  Timed t(KID_EVAL, s);
  GS_CHECK(launch_eval_metrics(R, H, W, hidden, lambda1, C1, C2, pred, target, rx_pos, conf_params, scratch, metrics,
                               s),
           "eval metrics");
  return GSPARC_OK;
}

// ---- densification ---------------------------------------------------------------

int gsparc_densify_stats(int P, int R, const int* radii, const float* dL_dmeans2D, float* accum, float* denom,
                         float* max_radii2D, void* stream) {
  if (P < 0 || R < 1) return invalid("sizes");
  if (P == 0) return GSPARC_OK;
  if (!radii || !dL_dmeans2D || !accum || !denom || !max_radii2D) return invalid("null pointer");
  cudaStream_t s = (cudaStream_t)stream;
  Timed t(KID_DENSIFY, s);
  GS_CHECK(launch_densify_stats(P, R, radii, dL_dmeans2D, accum, denom, max_radii2D, s), "densify stats");
  return GSPARC_OK;
}

size_t gsparc_densify_work_ints(int P) { return P < 0 ? 0 : densify_work_ints(P); }

namespace {
int densify_check(int P, long long mlp_floats, int per_gaussian_mlp, int conf_floats, const float* box6) {
  if (P < 0 || mlp_floats < 0 || conf_floats < 0) return invalid("sizes");
  if (per_gaussian_mlp && mlp_floats != 194LL * P) return invalid("a per-Gaussian MLP segment holds 194*P floats");
  if (!box6) return invalid("null scene box");
  return GSPARC_OK;
}
}  // namespace

int gsparc_densify_count(int P, long long mlp_floats, int per_gaussian_mlp, int conf_floats, const float* params,
                         const float* accum, const float* denom, float grad_threshold, float percent_dense,
                         float extent, float min_opacity, float max_screen_size, const float* scene_box6,
                         unsigned long long seed, int* work, int* P_new, void* stream) {
  const int st = densify_check(P, mlp_floats, per_gaussian_mlp, conf_floats, scene_box6);
  if (st != GSPARC_OK) return st;
  if (!params || !accum || !denom || !work || !P_new) return invalid("null pointer");
  const GaussianLayout L = gaussian_layout((size_t)P, (size_t)mlp_floats, (size_t)conf_floats);
  const size_t off[6] = {L.centre, L.scale, L.quat, L.opacity, L.mlp, L.conf};
  cudaStream_t s = (cudaStream_t)stream;
  Timed t(KID_DENSIFY, s);
  GS_CHECK(launch_densify_count(P, params, off, accum, denom, grad_threshold, percent_dense, extent, min_opacity,
                                max_screen_size, scene_box6, seed, work, P_new, s),
           "densify count");
  return GSPARC_OK;
}

int gsparc_densify_apply(int P, int P_new, long long mlp_floats, int per_gaussian_mlp, int conf_floats,
                         const float* params, const float* exp_avg, const float* exp_avg_sq, float grad_threshold,
                         float percent_dense, float extent, float min_opacity, float max_screen_size,
                         const float* scene_box6, unsigned long long seed, const int* work, float* new_params,
                         float* new_exp_avg, float* new_exp_avg_sq, void* stream) {
  const int st = densify_check(P, mlp_floats, per_gaussian_mlp, conf_floats, scene_box6);
  if (st != GSPARC_OK) return st;
  if (P_new < 0) return invalid("P_new");
  if (!params || !exp_avg || !exp_avg_sq || !work || !new_params || !new_exp_avg || !new_exp_avg_sq)
    return invalid("null pointer");
  const GaussianLayout L = gaussian_layout((size_t)P, (size_t)mlp_floats, (size_t)conf_floats);
  const size_t off[6] = {L.centre, L.scale, L.quat, L.opacity, L.mlp, L.conf};
  const long long new_mlp = per_gaussian_mlp ? 194LL * P_new : mlp_floats;
  const GaussianLayout N = gaussian_layout((size_t)P_new, (size_t)new_mlp, (size_t)conf_floats);
  const size_t noff[6] = {N.centre, N.scale, N.quat, N.opacity, N.mlp, N.conf};
  cudaStream_t s = (cudaStream_t)stream;
  Timed t(KID_DENSIFY, s);
  GS_CHECK(launch_densify_apply(P, P_new, params, exp_avg, exp_avg_sq, off, mlp_floats, per_gaussian_mlp, conf_floats,
                                grad_threshold, percent_dense, extent, min_opacity, max_screen_size, scene_box6, seed,
                                work, new_params, new_exp_avg, new_exp_avg_sq, noff, s),
           "densify apply");
  return GSPARC_OK;
}

int gsparc_reset_opacity(int P, long long mlp_floats, int conf_floats, float* params, float* exp_avg,
                         float* exp_avg_sq, void* stream) {
  if (P < 0 || mlp_floats < 0 || conf_floats < 0) return invalid("sizes");
  if (P == 0) return GSPARC_OK;
  if (!params || !exp_avg || !exp_avg_sq) return invalid("null pointer");
  const GaussianLayout L = gaussian_layout((size_t)P, (size_t)mlp_floats, (size_t)conf_floats);
  cudaStream_t s = (cudaStream_t)stream;
  Timed t(KID_DENSIFY, s);
  GS_CHECK(launch_reset_opacity(P, params + L.opacity, exp_avg + L.opacity, exp_avg_sq + L.opacity, s),
           "reset opacity");
  return GSPARC_OK;
}

// ---- fused optimizer ---------------------------------------------------------

size_t gsparc_gaussian_state_floats(int P, long long mlp_floats, int conf_floats) {
  if (P < 0 || mlp_floats < 0 || conf_floats < 0) return 0;
  return gaussian_layout((size_t)P, (size_t)mlp_floats, (size_t)conf_floats).total;
}

int gsparc_gaussian_state_layout(int P, long long mlp_floats, int conf_floats, size_t* offsets6) {
  if (P < 0 || mlp_floats < 0 || conf_floats < 0 || !offsets6) return invalid("gaussian state layout");
  const GaussianLayout L = gaussian_layout((size_t)P, (size_t)mlp_floats, (size_t)conf_floats);
  offsets6[0] = L.centre; offsets6[1] = L.scale; offsets6[2] = L.quat; offsets6[3] = L.opacity;
  offsets6[4] = L.mlp; offsets6[5] = L.conf;
  return GSPARC_OK;
}

int gsparc_gaussian_activate(int P, const float* params, float* scales, float* rotations, float* opacities,
                             void* stream) {
  if (P < 0) return invalid("P");
  if (P == 0) return GSPARC_OK;
  if (!params || !scales || !rotations || !opacities) return invalid("null pointer");
  cudaStream_t s = (cudaStream_t)stream;
  Timed t(KID_ACTIVATE, s);
  GS_CHECK(launch_gaussian_activate(P, params, scales, rotations, opacities, s), "gaussian activate");
  return GSPARC_OK;
}

int gsparc_gaussian_adam_step(int P, long long mlp_floats, int conf_floats, float* params, const float* grads,
                              float* exp_avg,
                              float* exp_avg_sq, float* step_count, const float* lr6, float beta1, float beta2,
                              float eps, const float* centre_lo3, const float* centre_hi3, float* scales,
                              float* rotations, float* opacities, void* stream) {
  if (P < 0 || mlp_floats < 0 || conf_floats < 0) return invalid("P, mlp_floats or conf_floats");
  if (!step_count || !lr6 || !centre_lo3 || !centre_hi3) return invalid("null step, learning-rate or clamp pointer");
  if ((P > 0 || mlp_floats > 0 || conf_floats > 0) && (!params || !grads || !exp_avg || !exp_avg_sq))
    return invalid("null state pointer");
  if ((((uintptr_t)params) | ((uintptr_t)grads) | ((uintptr_t)exp_avg) | ((uintptr_t)exp_avg_sq)) & 15u)
    return invalid("state buffers must be 16-byte aligned");
  const int n_act = (scales != nullptr) + (rotations != nullptr) + (opacities != nullptr);
  if (n_act != 0 && n_act != 3) return invalid("activation outputs: give all three or none");
  if (!(beta1 >= 0.f && beta1 < 1.f && beta2 >= 0.f && beta2 < 1.f && eps >= 0.f)) return invalid("Adam betas/eps");
  cudaStream_t s = (cudaStream_t)stream;
  Timed t(KID_ADAM, s);
  GS_CHECK(launch_gaussian_adam(P, mlp_floats, conf_floats, params, grads, exp_avg, exp_avg_sq, step_count, lr6, beta1, beta2,
                                eps, centre_lo3, centre_hi3, scales, rotations, opacities, s),
           "gaussian adam");
  return GSPARC_OK;
}

// ---- per-kernel timing ------------------------------------------------------

int gsparc_timing_enable(int on) {
  std::lock_guard<std::mutex> lk(g_tmu);
  g_timing = on != 0;
  return GSPARC_OK;
}

int gsparc_timing_kernel_count(void) { return KID_COUNT; }

int gsparc_depth_sort_launches(int P, int R) { return depth_sort_launches(P, R); }

int gsparc_set_wait_limit(long long polls) {
  g_wait_limit.store(polls < 0 ? -1 : polls, std::memory_order_relaxed);
  return GSPARC_OK;
}

const char* gsparc_timing_kernel_name(int id) { return (id >= 0 && id < KID_COUNT) ? kKernelNames[id] : ""; }

int gsparc_timing_read(double* total_ms, long long* launches, int n, int reset) {
  std::lock_guard<std::mutex> lk(g_tmu);
  for (auto& p : g_pending) {
    GS_CHECK(cudaEventSynchronize(p.b), "timing sync");
    float ms = 0.f;
    GS_CHECK(cudaEventElapsedTime(&ms, p.a, p.b), "timing elapsed");
    g_ms[p.id] += ms;
    g_launches[p.id] += 1;
    g_event_pool.push_back(p.a);
    g_event_pool.push_back(p.b);
  }
  g_pending.clear();
  for (int i = 0; i < n && i < KID_COUNT; ++i) {
    if (total_ms) total_ms[i] = g_ms[i];
    if (launches) launches[i] = g_launches[i];
  }
  if (reset) {
    for (int i = 0; i < KID_COUNT; ++i) { g_ms[i] = 0.0; g_launches[i] = 0; }
  }
  return GSPARC_OK;
}

}  // extern "C"
