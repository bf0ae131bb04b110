// Host-side launch wrappers shared between the kernel files and the C ABI.
#pragma once

#include "common.cuh"

namespace gsparc {

// Record the detail text of a failed call and return its status (capi.cu).
int report_invalid(const char* what);
// Poll bound of the library's device-side waits: `dflt` unless the host set a
// limit with gsparc_set_wait_limit (the smaller of the two; 0 = give up at the
// first wait that is not already satisfied).
uint32_t wait_polls(uint32_t dflt);
int report_cuda(cudaError_t e, const char* where);

// Preprocess, tile counts and (last CTA) the segment scan: ranges, cursors,
// chunk bases and K in the image header.
cudaError_t launch_preprocess(int P, int R, int H, int W, const TileGrid& grid, float mod, const float* means3D,
                              const float* mlp, const float* opacities, const float* scales,
                              const float* rotations, const float* views, const float* tx_pos,
                              const float* rx_pos, const GeomView& geo, int* radii_out, const ImageView& img,
                              cudaStream_t stream);

cudaError_t launch_mark_visible(int P, const float* means3D, const float* view, uint8_t* present,
                                cudaStream_t stream);


cudaError_t launch_check_capacity(ImageView img, unsigned long long capacity, cudaStream_t stream);

cudaError_t launch_scatter(int P, int R, const TileGrid& grid, const GeomView& geo, ImageView img, BinningView bin,
                           cudaStream_t stream);

// Largest P the binning supports (the placement's rank bitmap lives in shared memory).
constexpr int kMaxBinningP = 1 << 20;

// Depth order of every receiver's Gaussians; also records the binning
// capacity in the header and flags K > capacity.
int depth_sort_launches(int P, int R);
cudaError_t launch_depth_sort(int P, int R, const GeomView& geo, ImageView img, unsigned long long capacity,
                              cudaStream_t stream);

cudaError_t launch_segment_place(int P, int R, const TileGrid& grid, const GeomView& geo, ImageView img,
                                 BinningView bin, cudaStream_t stream);

cudaError_t launch_blend_forward(int P, int R, int H, int W, const TileGrid& grid, const GeomView& geo,
                                 const ImageView& img, const BinningView& bin, float* out_real, float* out_imag,
                                 cudaStream_t stream);

cudaError_t launch_blend_backward(int P, int R, int H, int W, const TileGrid& grid, unsigned grad_mode,
                                  long long capacity, const GeomView& geo, const ImageView& img,
                                  const BinningView& bin,
                                  const float* dL_dout_real, const float* dL_dout_imag, float* dmean2D,
                                  float* dconic, float* dsig, float* dopac, cudaStream_t stream);

cudaError_t launch_geometry_backward(int P, int R, int H, int W, float mod, unsigned grad_mode,
                                     const float* means3D, const float* scales, const float* rotations,
                                     const float* views, const GeomView& geo, const float* dmean2D,
                                     const float* dconic, float* dL_dmeans3D, float* dL_dcov3D, float* dL_dscales,
                                     float* dL_drot, cudaStream_t stream);

cudaError_t launch_emission_backward(int P, int R, const float* means3D, const float* mlp, const float* tx_pos,
                                     const float* rx_pos, const int* radii, const float* dsig, float* dL_dmlp,
                                     float* dL_dmeans3D, cudaStream_t stream);

cudaError_t launch_gaussian_adam(int P, long long mlp_floats, int conf_floats, float* params, const float* grads,
                                 float* m, float* v,
                                 float* step, const float* lr6, float beta1, float beta2, float eps,
                                 const float* lo3, const float* hi3, float* act_scales, float* act_rots,
                                 float* act_opac, cudaStream_t stream);

cudaError_t launch_gaussian_activate(int P, const float* params, float* act_scales, float* act_rots,
                                     float* act_opac, cudaStream_t stream);

LossLayout loss_layout(size_t R, size_t H, size_t W, size_t hidden);
size_t eval_scratch_floats(size_t R, size_t H, size_t W);
size_t densify_work_ints(int P);
cudaError_t launch_densify_stats(int P, int R, const int* radii, const float* dmeans2D, float* accum, float* denom,
                                 float* max_radii, cudaStream_t s);
cudaError_t launch_densify_count(int P, const float* params, const size_t* off, const float* accum,
                                 const float* denom, float grad_threshold, float percent_dense, float extent,
                                 float min_opacity, float max_screen_size, const float* box6,
                                 unsigned long long seed, int* work, int* P_new, cudaStream_t s);
cudaError_t launch_densify_apply(int P, int P_new, const float* params, const float* exp_avg, const float* exp_avg_sq,
                                 const size_t* off, long long mlp_floats, int per_gaussian_mlp, int conf_floats,
                                 float grad_threshold, float percent_dense, float extent, float min_opacity,
                                 float max_screen_size, const float* box6, unsigned long long seed, const int* work,
                                 float* new_params, float* new_exp_avg, float* new_exp_avg_sq, const size_t* new_off,
                                 cudaStream_t s);
cudaError_t launch_reset_opacity(int P, float* logit, float* m1, float* m2, cudaStream_t s);
cudaError_t launch_eval_metrics(int R, int H, int W, int hidden, float lambda1, float C1, float C2, const float* pred,
                                const float* target, const float* rx, const float* conf_params, float* scratch,
                                float* metrics, cudaStream_t stream);

cudaError_t launch_splat_loss(int R, int H, int W, int hidden, float lambda1, float alpha, float C1, float C2,
                              const float* pred, const float* target, const float* rx, const float* conf_params,
                              float* scratch, float* loss_out, float* terms, float* dL_dpred, float* dconf,
                              cudaStream_t stream);

cudaError_t launch_ssim_forward(int planes, int H, int W, float C1, float C2, const float* img1, const float* img2,
                                float* map, float* dmu1, float* ds11, float* ds12, cudaStream_t stream);

cudaError_t launch_ssim_backward(int planes, int H, int W, const float* img1, const float* img2, const float* dL_dmap,
                                 const float* dmu1, const float* ds11, const float* ds12, float* dL_dimg1,
                                 cudaStream_t stream);

// Shared emission MLP (shared_mlp.cu): parameter and workspace offsets in
// floats; layers = hidden layers (at most kMaxMlpLayers).
constexpr int kMaxMlpLayers = 6;
struct SharedMlpLayout {
  int layers, width, out;
  size_t w[kMaxMlpLayers + 1], b[kMaxMlpLayers + 1], params;
  size_t x0, z[kMaxMlpLayers + 1], a[kMaxMlpLayers + 1], o, s, d0, d1, work;
};
SharedMlpLayout shared_mlp_layout(int layers, int width, int out, size_t rows);

// Multi-channel blend (blend_channels.cu): features [R][P][C], out [R][C][H][W].
cudaError_t launch_blend_channels_forward(int P, int R, int H, int W, int C, const TileGrid& grid,
                                          const GeomView& geo, const ImageView& img, const BinningView& bin,
                                          const float* features, float* out, cudaStream_t s);
cudaError_t launch_blend_channels_backward(int P, int R, int H, int W, int C, const TileGrid& grid,
                                           const GeomView& geo, const ImageView& img, const BinningView& bin,
                                           const float* features, const float* dL_dout, float* dL_dfeatures,
                                           float* dmean2D, float* dconic, float* dopacity, cudaStream_t s);

// BF16 / tcgen05 path (shared_mlp_tc.cu): width 128, 1 or 64 outputs, 1-3 layers;
// workspace: sigmoid outputs [rows][out] at s (offset 0), BF16 pre-activations
// [layers][rows][128] at z[1] (whole 128-row tiles, tile-transposed); the
// adjoint adds dL/dmeans3D through the features itself.
SharedMlpLayout shared_mlp_layout_bf16(int layers, size_t rows, int out);
cudaError_t launch_shared_mlp_bf16(bool fwd, int P, int R, int layers, int act, int out, const float* means3D,
                                   const float* rx_pos, const float* params, const GeomView& geo, float* work,
                                   const float* dL_dsignal, float* dparams, float* dL_dmeans3D, ImageHeader* hdr,
                                   cudaStream_t s);
cudaError_t launch_mlp_features_backward(int P, int R, const float* means3D, const float* rx_pos, const int* radii,
                                         const float* dX, float* dL_dmeans3D, cudaStream_t s);
// the BF16 path's activation (forward and adjoint) and derivative for every BF16 input
cudaError_t launch_bf16_act_table(int act, uint16_t* out, cudaStream_t s);

cudaError_t launch_shared_mlp_forward(int P, int R, int layers, int width, int act, int out, const float* means3D,
                                      const float* rx_pos, const float* params, const GeomView& geo, float* work,
                                      cudaStream_t s);

cudaError_t launch_shared_mlp_backward(int P, int R, int layers, int width, int act, int out, const float* means3D,
                                       const float* rx_pos, const float* params, const GeomView& geo, float* work,
                                       const float* dL_dsignal, float* dL_dparams, float* dL_dmeans3D,
                                       cudaStream_t s);

}  // namespace gsparc
