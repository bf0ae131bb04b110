/*
 * gsparc_b200.h -- C ABI of the sm_100a equirectangular RF splatting path.
 *
 * Plain device pointers, sizes and a CUDA stream (passed as void*, i.e. a
 * cudaStream_t; NULL = the legacy default stream).  No allocation happens
 * inside any entry point: the caller owns every buffer, including the three
 * opaque state arenas sized by the *_state_bytes() queries, exactly as the
 * reference's torch extension owns its geometry / binning / image byte
 * buffers (cuda_kernel_rasterize/rasterize_points.cu:24-30, :69-74).
 *
 * Every entry point returns a gsparc_status code; kernel launches are
 * asynchronous on the given stream unless stated otherwise.
 *
 * Batching: R receivers are rendered per call.  Per-receiver tensors are laid
 * out receiver-major ([R,3] positions, [R,16] view matrices, [R,H,W] spectra,
 * [R,P] radii).  R = 1 is the reference's per-receiver call.
 */
#ifndef GSPARC_B200_H_
#define GSPARC_B200_H_

#include <stddef.h>
#include <stdint.h>

#if defined(__GNUC__)
#define GSPARC_API __attribute__((visibility("default")))
#else
#define GSPARC_API
#endif

#ifdef __cplusplus
extern "C" {
#endif

typedef enum gsparc_status {
  GSPARC_OK = 0,
  GSPARC_ERR_INVALID = 1,   /* bad size, tile shape or null pointer */
  GSPARC_ERR_CUDA = 2,      /* a CUDA runtime call or launch failed */
  GSPARC_ERR_CAPACITY = 3,  /* duplicated instances exceeded the binning capacity */
  GSPARC_ERR_DEVICE = 4     /* a kernel raised a bit in the device error word */
} gsparc_status;

/* Gradient modes for gsparc_rasterize_backward. */
#define GSPARC_GRAD_REFERENCE 0u /* reproduce the reference backward bit-for-bit in
                                    structure: halved azimuth Jacobian row
                                    (backward.cu:172-173), real-only alpha
                                    gradient (backward.cu:577,587) */
#define GSPARC_GRAD_EXACT 1u     /* true derivative of the forward */

/* `flags` of gsparc_rasterize_prepare / _render / _backward (pass the same
 * value to all three for one forward).  0: footprints are clamped at the
 * image's left and right edges, as the reference's getRect does
 * (auxiliary.h:14-24) -- bit-exact parity.  GSPARC_FLAG_WRAP_AZIMUTH: pixel
 * columns x and x +- W are the same azimuth, so a footprint that crosses the
 * 0/2pi seam also covers the tiles on the other side (the columns beyond the
 * left edge: [(int)(((px - r) + W) / tile_w), gx); beyond the right edge:
 * [0, (int)((((px + r) - W) + tile_w) - 1) / tile_w)), and every tile blends
 * the copy of a Gaussian (mean x or x -+ W) nearest to its centre column.
 * Footprints that do not cross the seam give the same result either way. */
#define GSPARC_FLAG_WRAP_AZIMUTH 1u

/* Version of this ABI (bumped on any signature change). */
GSPARC_API int gsparc_abi_version(void);

/* Human-readable text for a status code. */
GSPARC_API const char* gsparc_status_string(int status);

/* Detail of the last failure on the calling host thread (CUDA error text or
 * the argument that was rejected).  Not part of the reference interface. */
GSPARC_API const char* gsparc_last_error_detail(void);

/* ---- arena sizing ------------------------------------------------------- */

/* Geometry arena: per-(receiver, Gaussian) preprocess results and cov3D.
 * Replaces GeometryState / required<GeometryState> (rasterizer_impl.cu:60-76,
 * rasterizer_impl.h:44-74). */
GSPARC_API size_t gsparc_geom_state_bytes(int P, int R);

/* Image arena: K, error word, tile ranges/counts, final T and contributor
 * counts.  Replaces ImageState (rasterizer_impl.cu:78-85). */
GSPARC_API size_t gsparc_image_state_bytes(int R, int H, int W, int tile_h, int tile_w);

/* Binning arena for `capacity` duplicated (Gaussian, tile) instances.
 * Replaces BinningState (rasterizer_impl.cu:87-100). */
GSPARC_API size_t gsparc_binning_state_bytes(long long capacity);

/* Byte offsets of the sub-arrays inside each arena (for inspection / tests).
 * geom:    means2D, depth, radii, conic_opacity, signal, cov3D   (6 entries)
 * image:   header, ranges, counts, cursor, final_T, n_contrib    (6 entries)
 * binning: seg_rank (per-instance depth rank, grouped by segment),
 *          point_list, adjoint checkpoints                       (3 entries) */
GSPARC_API int gsparc_geom_state_layout(int P, int R, size_t* offsets6);
GSPARC_API int gsparc_image_state_layout(int R, int H, int W, int tile_h, int tile_w, size_t* offsets6);
GSPARC_API int gsparc_binning_state_layout(long long capacity, size_t* offsets3);

/* ---- forward ------------------------------------------------------------ */

/* Stage 1 of the forward: per-(receiver, Gaussian) preprocess (range cull,
 * equirectangular projection, cov3D, 2D conic, radius, tile rectangle,
 * per-Gaussian emission MLP, depth), per-tile instance counts, prefix scan and
 * tile ranges.  Replaces FORWARD::preprocess + cub::DeviceScan::InclusiveSum
 * + the num_rendered readback of Rasterizer::forward
 * (rasterizer_impl.cu:227-274; forward.cu:252-327).
 *
 * means3D [P,3], emission_mlps [194*P] (layout of EmissionMLPs.get_all_params,
 * gaussian.py:565-572), opacities [P] (activated), scales [P,3] (activated),
 * rotations [P,4] (normalised, (w,x,y,z)), viewmatrices [R,16] (transposed
 * world->receiver, as built by preprocess_data.py:177-202), tx_pos [3],
 * rx_pos [R,3].  radii_out [R,P] may be NULL.  Limits: P <= 1048576 (the
 * binning places each tile's instances with a bitmap over the P depth
 * ranks, held in shared memory), R <= 65535.
 *
 * When num_rendered is non-NULL, K is copied to the host and the stream is
 * synchronised (the reference's blocking readback, rasterizer_impl.cu:274);
 * pass NULL to stay asynchronous (CUDA-graph capture). */
GSPARC_API int gsparc_rasterize_prepare(int P, int R, int H, int W, int tile_h, int tile_w,
                             unsigned int flags, float scale_modifier, const float* means3D,
                             const float* emission_mlps, const float* opacities,
                             const float* scales, const float* rotations,
                             const float* viewmatrices, const float* tx_pos,
                             const float* rx_pos, int* radii_out, void* geom_state,
                             void* image_state, long long* num_rendered, void* stream);

/* Stage 2 of the forward: put each receiver's Gaussians in (depth bits,
 * Gaussian id) order, duplicate instances into per-(receiver, tile) segments
 * and place every segment in that order -- the order the reference's stable
 * radix sort on (tile | depth) produces -- then blend each tile front to
 * back.  Replaces duplicateWithKeys, cub::DeviceRadixSort,
 * identifyTileRanges and FORWARD::render (rasterizer_impl.cu:276-331,
 * forward.cu:151-249).  out_real / out_imag are [R,H,W] (one channel).
 * If K exceeds `capacity` the device error word gets the capacity bit and the
 * outputs are left unwritten; gsparc_read_status reports it. */
GSPARC_API int gsparc_rasterize_render(int P, int R, int H, int W, int tile_h, int tile_w,
                            unsigned int flags, const void* geom_state, void* image_state, void* binning_state,
                            long long capacity, float* out_real, float* out_imag,
                            void* stream);

/* Synchronises the stream and reads K and the device error word of the last
 * forward that used `image_state`.  Returns GSPARC_ERR_CAPACITY or
 * GSPARC_ERR_DEVICE when the error word is set. */
GSPARC_API int gsparc_read_status(const void* image_state, long long* num_rendered,
                       unsigned int* error_word, void* stream);

/* ---- backward ----------------------------------------------------------- */

/* Full adjoint of the forward.  Replaces Rasterizer::backward
 * (rasterizer_impl.cu:339-442): reverse-order blend adjoint recomputing T
 * from the saved final T and contributor count (backward.cu:442-616), conic /
 * projection / cov3D adjoint (backward.cu:124-371) and the emission-MLP
 * backward (backward.cu:9-118).
 *
 * Inputs as for the forward, plus the arenas of that forward, the binning
 * capacity the render was given (the reference passes num_rendered,
 * rasterize_points.cu:124) and dL_dout_real / dL_dout_imag [R,H,W].  Outputs (all overwritten):
 *   dL_dmeans2D [R,P,3], dL_dconic [R,P,4] (slots x,y,-,w), dL_dsignal [R,P,2],
 *   dL_dopacity [P] (summed over receivers), dL_dmeans3D [P,3],
 *   dL_dcov3D [P,6], dL_dscales [P,3], dL_drotations [P,4],
 *   dL_demission_mlps [194*P].
 * grad_mode is GSPARC_GRAD_REFERENCE or GSPARC_GRAD_EXACT. */
GSPARC_API int gsparc_rasterize_backward(int P, int R, int H, int W, int tile_h, int tile_w,
                              unsigned int flags, float scale_modifier, unsigned int grad_mode,
                              const float* means3D, const float* emission_mlps,
                              const float* scales, const float* rotations,
                              const float* viewmatrices, const float* tx_pos,
                              const float* rx_pos, const void* geom_state,
                              const void* image_state, const void* binning_state,
                              long long binning_capacity, const float* dL_dout_real, const float* dL_dout_imag,
                              float* dL_dmeans2D, float* dL_dconic, float* dL_dsignal,
                              float* dL_dopacity, float* dL_dmeans3D, float* dL_dcov3D,
                              float* dL_dscales, float* dL_drotations,
                              float* dL_demission_mlps, void* stream);

/* ---- multi-channel render (C amplitude channels per Gaussian) ------------ */

/* Stage 2 of the forward for C channels (1 <= C <= 64, e.g. one per frequency
 * bin): the binning of gsparc_rasterize_render, then one blend of all C
 * channels with the same transmittance and contributor decisions (final T and
 * contributor counts equal a single-channel render of the same geometry).
 * The reference blends NUM_CHANNELS = 1 (config.h:15, forward.cu:151-249).
 * features [R,P,C] are per-(receiver, Gaussian) amplitudes (from
 * gsparc_shared_mlp_forward with out = C); out [R,C,H,W] is overwritten:
 * out[r,c] = sum_i features[r,i,c] * alpha_i * T_i. */
GSPARC_API int gsparc_rasterize_render_channels(int P, int R, int H, int W, int tile_h, int tile_w,
                                     unsigned int flags, int C, const void* geom_state, void* image_state,
                                     void* binning_state, long long capacity, const float* features,
                                     float* out, void* stream);

/* Adjoint of gsparc_rasterize_render_channels (the true derivative; the 0.99
 * alpha clamp blocks the gradient) followed by the conic / projection / cov3D
 * adjoint of gsparc_rasterize_backward in GSPARC_GRAD_EXACT mode.  dL_dout
 * [R,C,H,W].  Outputs (all overwritten): dL_dfeatures [R,P,C], dL_dmeans2D
 * [R,P,3], dL_dconic [R,P,4], dL_dopacity [P], dL_dmeans3D [P,3] (geometry
 * part), dL_dcov3D [P,6], dL_dscales [P,3], dL_drotations [P,4]. */
GSPARC_API int gsparc_rasterize_backward_channels(int P, int R, int H, int W, int tile_h, int tile_w,
                                       unsigned int flags, int C, float scale_modifier,
                                       const float* means3D, const float* scales, const float* rotations,
                                       const float* viewmatrices, const void* geom_state,
                                       const void* image_state, const void* binning_state,
                                       long long binning_capacity, const float* features,
                                       const float* dL_dout, float* dL_dfeatures, float* dL_dmeans2D,
                                       float* dL_dconic, float* dL_dopacity, float* dL_dmeans3D,
                                       float* dL_dcov3D, float* dL_dscales, float* dL_drotations, void* stream);

/* Range cull only: present[i] = |view * means3D[i]|^2 > 0.04.  Replaces
 * markVisible / checkFrustum (rasterize_points.cu:203-221,
 * rasterizer_impl.cu:173-202).  present is [P] bytes (0/1). */
GSPARC_API int gsparc_mark_visible(int P, const float* means3D, const float* viewmatrix,
                        uint8_t* present, void* stream);

/* ---- fused SSIM --------------------------------------------------------- */

/* SSIM map with an 11x11 Gaussian window (sigma 1.5), zero "same" padding, and
 * -- when the three derivative pointers are non-NULL -- the partial
 * derivatives the backward needs.  Replaces fusedssim / fusedssimCUDA
 * (fused-ssim/ssim.cu:187-286, :368-404).  Images are [B,CH,H,W] float32. */
GSPARC_API int gsparc_ssim_forward(int B, int CH, int H, int W, float C1, float C2,
                        const float* img1, const float* img2, float* ssim_map,
                        float* dm_dmu1, float* dm_dsigma1_sq, float* dm_dsigma12,
                        void* stream);

/* dL/dimg1 from dL/dmap and the forward's partial derivatives.  Replaces
 * fusedssim_backward / fusedssim_backwardCUDA (fused-ssim/ssim.cu:288-366,
 * :406-444). */
GSPARC_API int gsparc_ssim_backward(int B, int CH, int H, int W, float C1, float C2,
                         const float* img1, const float* img2, const float* dL_dmap,
                         const float* dm_dmu1, const float* dm_dsigma1_sq,
                         const float* dm_dsigma12, float* dL_dimg1, void* stream);

/* ---- shared emission MLP ------------------------------------------------ */

/* The benchmark configurations' emission model: one MLP shared by all
 * Gaussians, evaluated per (receiver, Gaussian) pair on 32 features (centre,
 * 4-frequency positional encoding of the centre, receiver-relative
 * direction, 1/d^2, one zero pad), `layers` hidden layers of `width` with
 * ReLU or GELU, a linear output; the pair's signal is sigmoid(output), real
 * channel (imaginary 0).  No counterpart in the reference, whose emission
 * model is the per-Gaussian 3-32-2 MLP (forward.cu:17-75); to use it, call
 * gsparc_rasterize_prepare with emission_mlps = NULL (signal left unset),
 * then gsparc_shared_mlp_forward, then gsparc_rasterize_render; in the
 * backward pass emission_mlps = dL_demission_mlps = NULL and follow
 * gsparc_rasterize_backward with gsparc_shared_mlp_backward.
 * params: flat fp32, per layer W [out, in] row-major then b [out].
 * workspace: gsparc_shared_mlp_workspace_floats floats (256-byte aligned for
 * GSPARC_MLP_BF16); the forward keeps what the backward needs there.
 * out: 1 (the signal of gsparc_rasterize_render), or up to 64 amplitude
 * channels for gsparc_rasterize_render_channels: then the first R*P*out floats
 * of the workspace hold features [R,P,out] = sigmoid(outputs) after the forward
 * and the geometry arena's signal is not written (FP32 only).
 * precision GSPARC_MLP_FP32: SIMT FP32 layers (any width 8..256, 1-6
 * layers; width 64 with one output and 1-2 layers runs fused kernels).
 * GSPARC_MLP_BF16: BF16 operands on the tcgen05 tensor cores with FP32
 * accumulation (width 128, 1-3 layers, 1 or 64 outputs); the forward and the
 * backward are one fused kernel each, their epilogues in packed BF16
 * arithmetic (GELU in the tanh form with BF16 coefficients fitted to the erf
 * GELU; gsparc_shared_mlp_bf16_act_table lists it).  image_state (optional)
 * receives the error bit of a bounded tensor-core wait that gave up. */
#define GSPARC_ACT_RELU 1
#define GSPARC_ACT_GELU 2
#define GSPARC_MLP_FP32 0
#define GSPARC_MLP_BF16 1
GSPARC_API size_t gsparc_shared_mlp_param_floats(int layers, int width, int out);
GSPARC_API size_t gsparc_shared_mlp_workspace_floats(int P, int R, int layers, int width, int out,
                                                     int precision);
/* Writes the signal of every visible pair into the geometry arena of a
 * prepared forward. */
GSPARC_API int gsparc_shared_mlp_forward(int P, int R, int layers, int width, int act, int out,
                                         int precision, const float* means3D, const float* rx_pos,
                                         const float* params, void* geom_state, void* image_state,
                                         float* workspace, void* stream);
/* dL_dsignal [R,P,2] as gsparc_rasterize_backward returns it (out = 1), or
 * dL_dfeatures [R,P,out] from gsparc_rasterize_backward_channels (out > 1);
 * dL_dparams is overwritten; dL/dmeans3D through the features is ADDED to
 * dL_dmeans3D. */
GSPARC_API int gsparc_shared_mlp_backward(int P, int R, int layers, int width, int act, int out,
                                          int precision, const float* means3D, const float* rx_pos,
                                          const float* params, const void* geom_state, void* image_state,
                                          float* workspace, const float* dL_dsignal, float* dL_dparams,
                                          float* dL_dmeans3D, void* stream);

/* The BF16 path's activation as its kernels evaluate it, for every BF16
 * input: out (device, 6 x 65536 uint16) = {act as the forward computes it,
 * act as the adjoint computes it, act'} x {input in the low lane of a packed
 * pair, in the high lane}, entry i of each table for the input whose BF16
 * bit pattern is i. */
GSPARC_API int gsparc_shared_mlp_bf16_act_table(int act, uint16_t* out, void* stream);

/* ---- training loss ------------------------------------------------------ */

/* Scratch floats gsparc_splat_loss needs for R spectra of H x W and a
 * confidence MLP with `hidden` units. */
GSPARC_API size_t gsparc_splat_loss_scratch_floats(int R, int H, int W, int hidden);

/* The training loss of train.py:420-436 and its adjoint in one call, for R
 * spectra at once (the loss of a batch is the mean over its receivers):
 *   l1_r   = mean |pred_r - target_r|                 (utils.py:40-41)
 *   ssim_r = mean fused-SSIM map, "same" padding      (train.py:423)
 *   recon_r = (1 - lambda1) l1_r + lambda1 (1 - ssim_r)
 *   conf_r = 1 + exp(fc2(relu(fc1(rx_pos_r))))        (ConfidenceMLP,
 *                                                      gaussian.py:575-609)
 *   loss   = mean_r (conf_r recon_r - alpha log conf_r)
 * Replaces l1_loss + fused_ssim + the confidence head and their autograd.
 * pred, target, dL_dpred: [R,H,W]; rx_pos: [R,3]; conf_params: the MLP's
 * parameters flat in nn.Module order (fc1.weight [hidden,3], fc1.bias
 * [hidden], fc2.weight [1,hidden], fc2.bias [1]: 5*hidden+1 floats);
 * dL_dconf_params: same layout, overwritten; loss_out: 1 float; terms:
 * optional [R,4] (l1, ssim, conf, loss_r); scratch: 16-byte aligned,
 * gsparc_splat_loss_scratch_floats floats, zero-filled before its first use
 * (it holds an arrival counter that every call leaves at zero).  All device
 * memory. */
GSPARC_API int gsparc_splat_loss(int R, int H, int W, int hidden, float lambda1, float alpha,
                                 float C1, float C2, const float* pred, const float* target,
                                 const float* rx_pos, const float* conf_params, float* scratch,
                                 float* loss_out, float* terms, float* dL_dpred,
                                 float* dL_dconf_params, void* stream);

/* ---- evaluation metrics --------------------------------------------------- */

/* Metrics per spectrum written by gsparc_eval_metrics, in this order. */
#define GSPARC_EVAL_METRICS 6
enum {
  GSPARC_EVAL_PSNR = 0,       /* 20 log10(1 / sqrt(mse)); +inf when mse = 0 (train.py:76-83) */
  GSPARC_EVAL_RSSI_DIFF = 1,  /* rssi(pred) - rssi(target), rssi = 10 log10(mean x^2) - 30 (train.py:86-91) */
  GSPARC_EVAL_MAE = 2,        /* mean |pred - target| (train.py:99-101) */
  GSPARC_EVAL_SSIM = 3,       /* mean SSIM map, 11x11 window, "same" padding (utils.py:81-114) */
  GSPARC_EVAL_CONFIDENCE = 4, /* 1 + exp(fc2(relu(fc1(rx_pos)))) (gaussian.py:575-609) */
  GSPARC_EVAL_LOSS = 5        /* (1 - lambda1) MAE + lambda1 (1 - SSIM) (train.py:696-697) */
};

/* Scratch floats gsparc_eval_metrics needs for R spectra of H x W. */
GSPARC_API size_t gsparc_eval_scratch_floats(int R, int H, int W);

/* The per-spectrum evaluation of train.py:672-701 (calculate_psnr,
 * calculate_rssi difference, calculate_mae, ssim, the confidence and the
 * evaluation loss), batched over R test spectra in one pass that shares the
 * SSIM moments of the training loss.  pred, target: [R,H,W]; rx_pos: [R,3];
 * conf_params: as gsparc_splat_loss; metrics: [R, GSPARC_EVAL_METRICS];
 * scratch: gsparc_eval_scratch_floats floats, zero-filled before its first
 * use (per-spectrum arrival counters that every call leaves at zero).  All
 * device memory. */
GSPARC_API int gsparc_eval_metrics(int R, int H, int W, int hidden, float lambda1, float C1, float C2,
                                   const float* pred, const float* target, const float* rx_pos,
                                   const float* conf_params, float* scratch, float* metrics, void* stream);

/* ---- densification (gaussian.py:223-551, train.py:508-553) --------------- */

/* Statistics of one step (train.py:508-516): for every receiver r and
 * Gaussian g with radii[r][g] > 0: accum[g] += |dL/dmeans2D[r][g][0:2]|,
 * denom[g] += 1, max_radii2D[g] = max(max_radii2D[g], radii[r][g]).
 * radii [R,P] int32 and dL_dmeans2D [R,P,3] as gsparc_rasterize_backward
 * leaves them; accum, denom, max_radii2D [P]. */
GSPARC_API int gsparc_densify_stats(int P, int R, const int* radii, const float* dL_dmeans2D, float* accum,
                                    float* denom, float* max_radii2D, void* stream);

/* Ints of the work buffer gsparc_densify_count / _apply share for P Gaussians. */
GSPARC_API size_t gsparc_densify_work_ints(int P);

/* densify_and_prune (gaussian.py:515-542) on a flat training state
 * (gsparc_gaussian_state_layout; a per-Gaussian MLP segment of 194*P floats
 * when per_gaussian_mlp, else a global one): clone (grad >= grad_threshold,
 * largest scale <= percent_dense * extent), split into two (grad >=
 * grad_threshold, largest scale > percent_dense * extent; centre R(q) (s z) +
 * centre with z ~ N(0,1) from a counter-based generator seeded by `seed`,
 * log-scale log(s / 1.2)), prune (opacity < min_opacity; largest scale >
 * 0.1 extent when max_screen_size > 0; centre outside scene_box6 = lo[3],
 * hi[3], 6 floats in HOST memory), grad = accum / denom (0 where 0/0).  Step 1 classifies and writes
 * the new count to *P_new (device int; read it, allocate the new state for
 * P_new, then call step 2, which gathers the survivors in the reference's
 * order -- kept originals, clones, first and second split copies -- with
 * zero Adam moments for the new Gaussians).  work: gsparc_densify_work_ints
 * ints.  Device memory except scene_box6. */
GSPARC_API int gsparc_densify_count(int P, long long mlp_floats, int per_gaussian_mlp, int conf_floats,
                                    const float* params, const float* accum, const float* denom,
                                    float grad_threshold, float percent_dense, float extent, float min_opacity,
                                    float max_screen_size, const float* scene_box6, unsigned long long seed,
                                    int* work, int* P_new, void* stream);
GSPARC_API int gsparc_densify_apply(int P, int P_new, long long mlp_floats, int per_gaussian_mlp, int conf_floats,
                                    const float* params, const float* exp_avg, const float* exp_avg_sq,
                                    float grad_threshold, float percent_dense, float extent, float min_opacity,
                                    float max_screen_size, const float* scene_box6, unsigned long long seed,
                                    const int* work, float* new_params, float* new_exp_avg,
                                    float* new_exp_avg_sq, void* stream);

/* reset_opacity (gaussian.py:223-230): opacity logits set to
 * logit(min(sigmoid(x), 0.01)), their Adam moments zeroed. */
GSPARC_API int gsparc_reset_opacity(int P, long long mlp_floats, int conf_floats, float* params, float* exp_avg,
                                    float* exp_avg_sq, void* stream);

/* ---- fused optimizer over the per-Gaussian parameters ------------------- */

/* Floats in a flat training-state buffer for P Gaussians, an emission-MLP
 * segment of mlp_floats floats (194*P: the per-Gaussian MLPs in the layout
 * of EmissionMLPs.get_all_params; or the shared MLP's parameter count) and a
 * global block of conf_floats floats (the confidence MLP; 0 for none), and
 * the float offsets of its six segments: centre [P,3], log-scale [P,3],
 * quaternion [P,4], opacity logit [P], emission MLP, global block.  Each
 * segment starts on a 256-byte boundary; the padding between segments must
 * stay zero in the gradient buffer. */
GSPARC_API size_t gsparc_gaussian_state_floats(int P, long long mlp_floats, int conf_floats);
GSPARC_API int gsparc_gaussian_state_layout(int P, long long mlp_floats, int conf_floats, size_t* offsets6);

/* Activated per-Gaussian values of a flat state buffer (gaussian.py:33-38):
 * scales [P,3] = exp(log-scale), rotations [P,4] = normalize(quaternion),
 * opacities [P] = sigmoid(logit). */
GSPARC_API int gsparc_gaussian_activate(int P, const float* params, float* scales, float* rotations,
                                        float* opacities, void* stream);

/* One Adam step (torch's update rule) over the whole flat state, fused with
 * the adjoints of the activations.  Replaces the torch.optim.Adam step over
 * GaussianModel's parameter groups and the confidence MLP's
 * (gaussian.py:176-197) together with the autograd of the activations
 * exp / normalize / sigmoid (gaussian.py:33-38), the NaN-zeroing of the
 * centre gradient (train.py:443-445) and the centre clamp (train.py:556-562).
 * params, exp_avg, exp_avg_sq: flat state buffers (raw parameters), updated in
 * place; grads: same layout, gradients with respect to the ACTIVATED values
 * (as gsparc_rasterize_backward returns them) and, in the global block, with
 * respect to its parameters; step_count: two device words, the step count
 * (float, incremented by this call) and a 32-bit arrival counter that must be
 * 0 before the first call (every call leaves it at 0); lr6: device floats (centre, scale, rotation, opacity, emission MLP,
 * global block); centre_lo3 / centre_hi3: device clamp box.  scales,
 * rotations, opacities: optional (all or none) outputs of the activated
 * updated parameters, as gsparc_gaussian_activate writes them.  State buffers
 * 16-byte aligned. */
GSPARC_API int gsparc_gaussian_adam_step(int P, long long mlp_floats, int conf_floats, float* params,
                                         const float* grads,
                                         float* exp_avg, float* exp_avg_sq, float* step_count,
                                         const float* lr6, float beta1, float beta2, float eps,
                                         const float* centre_lo3, const float* centre_hi3,
                                         float* scales, float* rotations, float* opacities,
                                         void* stream);

/* SSIM map and dL/dimg1 in one call that allocates nothing.  No counterpart
 * in the reference.  For callers that cannot call cudaMalloc (for example a
 * real-time receiver loop that cannot absorb cudaMalloc's implicit device
 * synchronisation, or a host handed fixed device buffers by another runtime):
 * the three partial-derivative maps the gradient needs live in a file-scope
 * device array of GSPARC_SSIM_STATIC_MAX_PIXELS * 3 floats (12 MiB, held by
 * every GPU that loads the library until exit).  Inputs img1, img2, dL_dmap
 * and outputs ssim_map, dL_dimg1 are [B,CH,H,W]; B*CH*H*W must not exceed
 * GSPARC_SSIM_STATIC_MAX_PIXELS (else GSPARC_ERR_INVALID).  All calls on a
 * device share the array and leave the last call's maps in it; nothing in it
 * needs clearing, but calls that overlap on the GPU race on it.  The first
 * call on a device looks up the array's device address and should be made
 * before any stream capture. */
#define GSPARC_SSIM_STATIC_MAX_PIXELS 1048576
GSPARC_API int gsparc_ssim_static_scratch(int B, int CH, int H, int W, float C1, float C2,
                                          const float* img1, const float* img2,
                                          const float* dL_dmap, float* ssim_map, float* dL_dimg1,
                                          void* stream);

/* ---- per-kernel timing (tracing; no counterpart in the reference, which
 * only times whole renders with time.time(), train.py:673-677) ------------ */

/* Enable/disable CUDA-event timing around every kernel launch of this
 * library (off by default; adds two event records per launch). */
GSPARC_API int gsparc_timing_enable(int on);

/* Number of timed kernel kinds, and the name of kind `id`. */
GSPARC_API int gsparc_timing_kernel_count(void);
GSPARC_API const char* gsparc_timing_kernel_name(int id);

/* Waits for the recorded events and returns, per kernel kind, the summed
 * device milliseconds and the launch count since the last reset (arrays of
 * n entries, either may be NULL).  reset != 0 clears the totals. */
GSPARC_API int gsparc_timing_read(double* total_ms, long long* launches, int n, int reset);

/* Kernel launches one depth sort of P Gaussians for R receivers makes on the
 * current device: 1 when all its CTAs fit at once (one cooperative launch),
 * else 4 (one per 8-bit pass); 0 for an empty sort, -1 on a CUDA error.  For
 * counting launches (the timing above counts calls). */
GSPARC_API int gsparc_depth_sort_launches(int P, int R);

/* ---- bounded device waits (failure detection; no counterpart in the
 * reference, which has no inter-CTA waits) ------------------------------- */

/* Every wait of one CTA on another CTA or on the tensor cores inside this
 * library is bounded: the depth sort's look-back and per-receiver barrier,
 * and the tensor-core MLP kernels' mbarrier waits.  A wait that runs out sets
 * kErrSortWait (bit 3) or kErrMlpWait (bit 4) in the image state's error word
 * (gsparc_read_status), the kernel drains its own tensor-core work in flight,
 * frees its tensor memory and returns; later stages skip their work.
 * polls >= 0 caps every such wait at `polls` polls (0: give up at the first
 * wait that is not already satisfied) for the launches that follow; polls < 0
 * restores each wait's default bound.  Process-wide; for tests of the give-up
 * path. */
GSPARC_API int gsparc_set_wait_limit(long long polls);

#ifdef __cplusplus
}
#endif

#endif /* GSPARC_B200_H_ */
