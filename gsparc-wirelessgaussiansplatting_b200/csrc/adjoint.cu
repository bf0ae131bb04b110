// Per-Gaussian adjoints: conic/projection/covariance and the emission MLP.
//
// geometry_backward_kernel: one thread per Gaussian, looping over receivers.
//   computeCov2DCUDA (cuda_wireless_rasterizer/backward.cu:124-303), the
//   screen-space-mean part of preprocessCUDA (backward.cu:412-430) and
//   computeCov3D backward (backward.cu:308-371).  dL/dcov3D and dL/dmean3D are
//   summed over receivers in registers, so the cov3D -> (scale, rotation)
//   adjoint runs once per Gaussian.
// emission_backward_kernel: one warp per Gaussian, lane = hidden unit.
//   computeSignalFromMLP backward (backward.cu:9-118).  Weight loads and
//   gradient stores are coalesced (the reference reads and writes 194 floats
//   per thread with a 776-byte stride), and gradients are summed over
//   receivers in registers.
#include "common.cuh"
#include "kernels.cuh"

namespace gsparc {

__global__ void __launch_bounds__(128)
geometry_backward_kernel(int P, int R, int H, int W, float mod, unsigned grad_mode,
                         const float* __restrict__ means3D, const float* __restrict__ scales,
                         const float* __restrict__ rotations, const float* __restrict__ views,
                         GeomView geo, const float* __restrict__ dmean2D, const float* __restrict__ dconic,
                         float* __restrict__ dL_dmeans3D, float* __restrict__ dL_dcov3D,
                         float* __restrict__ dL_dscales, float* __restrict__ dL_drot) {
  const int g = blockIdx.x * blockDim.x + threadIdx.x;
  if (g >= P) return;
  const bool ref = grad_mode == GSPARC_GRAD_REFERENCE;
  const float xscale = ref ? 0.5f : 1.0f;
  const float3 mean = make_float3(__ldg(means3D + 3 * g), __ldg(means3D + 3 * g + 1), __ldg(means3D + 3 * g + 2));
  float cov3[6];
  float acc_mean[3] = {0.f, 0.f, 0.f};
  float acc_cov[6] = {0.f, 0.f, 0.f, 0.f, 0.f, 0.f};
  bool any = false;
  for (int r = 0; r < R; ++r) {
    const size_t rg = (size_t)r * P + g;
    if (!(geo.radii[rg] > 0)) continue;
    if (!any) {
#pragma unroll
      for (int i = 0; i < 6; ++i) cov3[i] = geo.cov3D[(size_t)g * 6 + i];
    }
    any = true;
    float mv[16];
#pragma unroll
    for (int i = 0; i < 16; ++i) mv[i] = __ldg(views + 16 * r + i);
    const float gcx = dconic[rg * 4 + 0], gcy = dconic[rg * 4 + 1], gcz = dconic[rg * 4 + 3];
    const float3 t = view_point(mean, mv);
    const float txtx = t.x * t.x;
    const float tyty = t.y * t.y;
    const float tztz = t.z * t.z;
    const float txtytz = t.x * t.y * t.z;
    const float trxztrxz = txtx + tztz;
    const float trxztrxz_inv = 1.0f / (trxztrxz + 0.0000001f);
    const float trxztrxztrxztrxz_inv = trxztrxz_inv * trxztrxz_inv;
    const float trxz = sqrtf(trxztrxz);
    const float trxz_inv = 1.0f / (trxz + 0.0000001f);
    const float trtr = trxztrxz + tyty;
    const float trtr_inv = 1.0f / (trtr + 0.0000001f);
    const float trtrtrtr_inv = trtr_inv * trtr_inv;
    const float trxz_trtrtrtr_inv = trxz_inv * trtrtrtr_inv;
    const float trxztrxztrxz_trtrtrtr_inv = trxztrxz_inv * trxz_trtrtrtr_inv;
    const float tyty_minus_trxztrxz = tyty - trxztrxz;
    const float W_div_2pi = W * 0.5f * kInvPi;
    const float H_div_pi = H * kInvPi;
    const float dpx_dtx = W_div_2pi * t.z * trxztrxz_inv * xscale;
    const float dpx_dtz = -W_div_2pi * t.x * trxztrxz_inv * xscale;
    const float dpy_dtx = -H_div_pi * t.x * t.y * trxz_inv * trtr_inv;
    const float dpy_dty = H_div_pi * trxz * trtr_inv;
    const float dpy_dtz = -H_div_pi * t.z * t.y * trxz_inv * trtr_inv;

    const Mat3 J = jac_mat(dpx_dtx, dpx_dtz, dpy_dtx, dpy_dty, dpy_dtz);
    const Mat3 Wr = view_rot(mv);
    const Mat3 Vrk = sym_from6(cov3);
    const Mat3 T = mat_mul(Wr, J);
    const Mat3 cov2D = mat_mul(mat_mul(mat_T(T), mat_T(Vrk)), T);
    const float a = cov2D.c[0][0] + 0.3f;
    const float b = cov2D.c[0][1];
    const float c = cov2D.c[1][1] + 0.3f;
    const float denom = a * c - b * b;
    float dL_da = 0.f, dL_db = 0.f, dL_dc = 0.f;
    const float denom2inv = 1.0f / ((denom * denom) + 0.0000001f);
    float dcov[6] = {0.f, 0.f, 0.f, 0.f, 0.f, 0.f};
    if (denom2inv != 0) {
      dL_da = denom2inv * (-c * c * gcx + 2 * b * c * gcy + (denom - a * c) * gcz);
      dL_dc = denom2inv * (-a * a * gcz + 2 * a * b * gcy + (denom - a * c) * gcx);
      dL_db = denom2inv * 2 * (b * c * gcx - (denom + 2 * b * b) * gcy + a * b * gcz);
      const auto& Tc = T.c;
      dcov[0] = (Tc[0][0] * Tc[0][0] * dL_da + Tc[0][0] * Tc[1][0] * dL_db + Tc[1][0] * Tc[1][0] * dL_dc);
      dcov[3] = (Tc[0][1] * Tc[0][1] * dL_da + Tc[0][1] * Tc[1][1] * dL_db + Tc[1][1] * Tc[1][1] * dL_dc);
      dcov[5] = (Tc[0][2] * Tc[0][2] * dL_da + Tc[0][2] * Tc[1][2] * dL_db + Tc[1][2] * Tc[1][2] * dL_dc);
      dcov[1] = 2 * Tc[0][0] * Tc[0][1] * dL_da + (Tc[0][0] * Tc[1][1] + Tc[0][1] * Tc[1][0]) * dL_db + 2 * Tc[1][0] * Tc[1][1] * dL_dc;
      dcov[2] = 2 * Tc[0][0] * Tc[0][2] * dL_da + (Tc[0][0] * Tc[1][2] + Tc[0][2] * Tc[1][0]) * dL_db + 2 * Tc[1][0] * Tc[1][2] * dL_dc;
      dcov[4] = 2 * Tc[0][2] * Tc[0][1] * dL_da + (Tc[0][1] * Tc[1][2] + Tc[0][2] * Tc[1][1]) * dL_db + 2 * Tc[1][1] * Tc[1][2] * dL_dc;
    }
    const auto& Tc = T.c;
    const auto& V = Vrk.c;
    const float dL_dT00 = 2 * (Tc[0][0] * V[0][0] + Tc[0][1] * V[0][1] + Tc[0][2] * V[0][2]) * dL_da +
                          (Tc[1][0] * V[0][0] + Tc[1][1] * V[0][1] + Tc[1][2] * V[0][2]) * dL_db;
    const float dL_dT01 = 2 * (Tc[0][0] * V[1][0] + Tc[0][1] * V[1][1] + Tc[0][2] * V[1][2]) * dL_da +
                          (Tc[1][0] * V[1][0] + Tc[1][1] * V[1][1] + Tc[1][2] * V[1][2]) * dL_db;
    const float dL_dT02 = 2 * (Tc[0][0] * V[2][0] + Tc[0][1] * V[2][1] + Tc[0][2] * V[2][2]) * dL_da +
                          (Tc[1][0] * V[2][0] + Tc[1][1] * V[2][1] + Tc[1][2] * V[2][2]) * dL_db;
    const float dL_dT10 = 2 * (Tc[1][0] * V[0][0] + Tc[1][1] * V[0][1] + Tc[1][2] * V[0][2]) * dL_dc +
                          (Tc[0][0] * V[0][0] + Tc[0][1] * V[0][1] + Tc[0][2] * V[0][2]) * dL_db;
    const float dL_dT11 = 2 * (Tc[1][0] * V[1][0] + Tc[1][1] * V[1][1] + Tc[1][2] * V[1][2]) * dL_dc +
                          (Tc[0][0] * V[1][0] + Tc[0][1] * V[1][1] + Tc[0][2] * V[1][2]) * dL_db;
    const float dL_dT12 = 2 * (Tc[1][0] * V[2][0] + Tc[1][1] * V[2][1] + Tc[1][2] * V[2][2]) * dL_dc +
                          (Tc[0][0] * V[2][0] + Tc[0][1] * V[2][1] + Tc[0][2] * V[2][2]) * dL_db;
    const auto& Wc = Wr.c;
    const float dL_dJ00 = Wc[0][0] * dL_dT00 + Wc[0][1] * dL_dT01 + Wc[0][2] * dL_dT02;
    const float dL_dJ02 = Wc[2][0] * dL_dT00 + Wc[2][1] * dL_dT01 + Wc[2][2] * dL_dT02;
    const float dL_dJ10 = Wc[0][0] * dL_dT10 + Wc[0][1] * dL_dT11 + Wc[0][2] * dL_dT12;
    const float dL_dJ11 = Wc[1][0] * dL_dT10 + Wc[1][1] * dL_dT11 + Wc[1][2] * dL_dT12;
    const float dL_dJ12 = Wc[2][0] * dL_dT10 + Wc[2][1] * dL_dT11 + Wc[2][2] * dL_dT12;
    // second derivatives of the projection (unhalved in both modes, as in
    // backward.cu:272-292)
    const float temp1 = H_div_pi * tyty_minus_trxztrxz * trxz_trtrtrtr_inv;
    const float temp2 = H_div_pi * txtytz * (trtr + 2.0f * trxztrxz) * trxztrxztrxz_trtrtrtr_inv;
    const float temp3 = W_div_2pi * (txtx - tztz) * trxztrxztrxztrxz_inv;
    const float temp4 = W_div_2pi * 2.0f * t.x * t.z * trxztrxztrxztrxz_inv;
    const float temp5 = H_div_pi * t.y * trxztrxztrxz_trtrtrtr_inv;
    const float dL_dtx = -dL_dJ00 * temp4 + dL_dJ02 * temp3 + dL_dJ10 * temp5 * (2.0f * txtx * trxztrxz - tztz * trtr) +
                         dL_dJ11 * t.x * temp1 + dL_dJ12 * temp2;
    const float dL_dty = dL_dJ10 * t.x * temp1 - dL_dJ11 * H_div_pi * 2.0f * trxz * t.y * trtrtrtr_inv +
                         dL_dJ12 * t.z * temp1;
    const float dL_dtz = dL_dJ00 * temp3 + dL_dJ02 * temp4 + dL_dJ10 * temp2 + dL_dJ11 * t.z * temp1 +
                         dL_dJ12 * temp5 * (2.0f * tztz * trxztrxz - txtx * trtr);
    const float3 dmean_cov = view_vec_T(make_float3(dL_dtx, dL_dty, dL_dtz), mv);
    // screen-space mean (backward.cu:413-430)
    const float dL_dpx = dmean2D[rg * 3 + 0] * (2.0f / (float)W);
    const float dL_dpy = dmean2D[rg * 3 + 1] * (2.0f / (float)H);
    const float d2x = dL_dpx * dpx_dtx + dL_dpy * dpy_dtx;
    const float d2y = dL_dpx * 0.0f + dL_dpy * dpy_dty;
    const float d2z = dL_dpx * dpx_dtz + dL_dpy * dpy_dtz;
    const float3 dmean_2d = view_vec_T(make_float3(d2x, d2y, d2z), mv);
    acc_mean[0] += dmean_cov.x; acc_mean[1] += dmean_cov.y; acc_mean[2] += dmean_cov.z;
    acc_mean[0] += dmean_2d.x; acc_mean[1] += dmean_2d.y; acc_mean[2] += dmean_2d.z;
#pragma unroll
    for (int i = 0; i < 6; ++i) acc_cov[i] += dcov[i];
  }
  float dscale[3] = {0.f, 0.f, 0.f};
  float dq[4] = {0.f, 0.f, 0.f, 0.f};
  if (any) {
    // computeCov3D backward (backward.cu:308-371)
    const float4 q = make_float4(__ldg(rotations + 4 * g), __ldg(rotations + 4 * g + 1),
                                 __ldg(rotations + 4 * g + 2), __ldg(rotations + 4 * g + 3));
    const float rq = q.x, x = q.y, y = q.z, z = q.w;
    const Mat3 Rm = quat_to_rot(q);
    const float3 s = make_float3(mod * __ldg(scales + 3 * g), mod * __ldg(scales + 3 * g + 1),
                                 mod * __ldg(scales + 3 * g + 2));
    const Mat3 M = scale_rot(s, Rm);
    const float* dc = acc_cov;
    Mat3 dS;
    dS.c[0][0] = dc[0]; dS.c[0][1] = 0.5f * dc[1]; dS.c[0][2] = 0.5f * dc[2];
    dS.c[1][0] = 0.5f * dc[1]; dS.c[1][1] = dc[3]; dS.c[1][2] = 0.5f * dc[4];
    dS.c[2][0] = 0.5f * dc[2]; dS.c[2][1] = 0.5f * dc[4]; dS.c[2][2] = dc[5];
    Mat3 M2;
#pragma unroll
    for (int j = 0; j < 3; ++j)
#pragma unroll
      for (int i = 0; i < 3; ++i) M2.c[j][i] = 2.0f * M.c[j][i];
    const Mat3 dM = mat_mul(M2, dS);
    const Mat3 Rt = mat_T(Rm);
    Mat3 dMt = mat_T(dM);
    dscale[0] = Rt.c[0][0] * dMt.c[0][0] + Rt.c[0][1] * dMt.c[0][1] + Rt.c[0][2] * dMt.c[0][2];
    dscale[1] = Rt.c[1][0] * dMt.c[1][0] + Rt.c[1][1] * dMt.c[1][1] + Rt.c[1][2] * dMt.c[1][2];
    dscale[2] = Rt.c[2][0] * dMt.c[2][0] + Rt.c[2][1] * dMt.c[2][1] + Rt.c[2][2] * dMt.c[2][2];
    if (!ref) { dscale[0] *= mod; dscale[1] *= mod; dscale[2] *= mod; }
#pragma unroll
    for (int i = 0; i < 3; ++i) { dMt.c[0][i] *= s.x; dMt.c[1][i] *= s.y; dMt.c[2][i] *= s.z; }
    const auto& D = dMt.c;
    dq[0] = 2 * z * (D[0][1] - D[1][0]) + 2 * y * (D[2][0] - D[0][2]) + 2 * x * (D[1][2] - D[2][1]);
    dq[1] = 2 * y * (D[1][0] + D[0][1]) + 2 * z * (D[2][0] + D[0][2]) + 2 * rq * (D[1][2] - D[2][1]) - 4 * x * (D[2][2] + D[1][1]);
    dq[2] = 2 * x * (D[1][0] + D[0][1]) + 2 * rq * (D[2][0] - D[0][2]) + 2 * z * (D[1][2] + D[2][1]) - 4 * y * (D[2][2] + D[0][0]);
    dq[3] = 2 * rq * (D[0][1] - D[1][0]) + 2 * x * (D[2][0] + D[0][2]) + 2 * y * (D[1][2] + D[2][1]) - 4 * z * (D[1][1] + D[0][0]);
  }
#pragma unroll
  for (int i = 0; i < 3; ++i) dL_dmeans3D[(size_t)g * 3 + i] = acc_mean[i];
#pragma unroll
  for (int i = 0; i < 6; ++i) dL_dcov3D[(size_t)g * 6 + i] = acc_cov[i];
#pragma unroll
  for (int i = 0; i < 3; ++i) dL_dscales[(size_t)g * 3 + i] = dscale[i];
#pragma unroll
  for (int i = 0; i < 4; ++i) dL_drot[(size_t)g * 4 + i] = dq[i];
}

__device__ __forceinline__ float warp_sum(float v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

// Must run after geometry_backward_kernel on the same stream: it adds the
// log-distance term of the MLP input to dL_dmeans3D.
__global__ void __launch_bounds__(256)
emission_backward_kernel(int P, int R, const float* __restrict__ means3D, const float* __restrict__ mlp,
                         const float* __restrict__ tx_pos, const float* __restrict__ rx_pos,
                         const int* __restrict__ radii, const float* __restrict__ dsig,
                         float* __restrict__ dL_dmlp, float* __restrict__ dL_dmeans3D) {
  const int lane = threadIdx.x & 31;
  const int warps_total = gridDim.x * (blockDim.x >> 5);
  const size_t o1 = (size_t)P * (kMlpIn * kMlpHidden);
  const size_t o2 = o1 + (size_t)P * kMlpHidden;
  const size_t o3 = o2 + (size_t)P * (kMlpOut * kMlpHidden);
  const float3 tx = make_float3(__ldg(tx_pos), __ldg(tx_pos + 1), __ldg(tx_pos + 2));
  for (int g = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5); g < P; g += warps_total) {
    const float* w1 = mlp + (size_t)g * (kMlpIn * kMlpHidden) + lane * kMlpIn;
    const float w1_0 = __ldg(w1), w1_1 = __ldg(w1 + 1), w1_2 = __ldg(w1 + 2);
    const float b1 = __ldg(mlp + o1 + (size_t)g * kMlpHidden + lane);
    const float w2_0 = __ldg(mlp + o2 + (size_t)g * (kMlpOut * kMlpHidden) + lane);
    const float w2_1 = __ldg(mlp + o2 + (size_t)g * (kMlpOut * kMlpHidden) + kMlpHidden + lane);
    const float b2_0 = __ldg(mlp + o3 + (size_t)g * kMlpOut);
    const float b2_1 = __ldg(mlp + o3 + (size_t)g * kMlpOut + 1);
    const float3 mean = make_float3(__ldg(means3D + 3 * g), __ldg(means3D + 3 * g + 1), __ldg(means3D + 3 * g + 2));
    const float3 diff = make_float3(tx.x - mean.x, tx.y - mean.y, tx.z - mean.z);
    const float d = sqrtf(diff.x * diff.x + diff.y * diff.y + diff.z * diff.z);
    const float log_d = logf(d + 1e-6f);
    const float inv_de = 1.0f / (d + 1e-6f);
    const float3 unit = make_float3(diff.x * inv_de, diff.y * inv_de, diff.z * inv_de);
    float gw1_0 = 0.f, gw1_1 = 0.f, gw1_2 = 0.f, gb1 = 0.f, gw2_0 = 0.f, gw2_1 = 0.f, gb2_0 = 0.f, gb2_1 = 0.f;
    float gm_x = 0.f, gm_y = 0.f, gm_z = 0.f;
    for (int r = 0; r < R; ++r) {
      const size_t rg = (size_t)r * P + g;
      if (!(radii[rg] > 0)) continue;   // warp-uniform
      const float in0 = __ldg(rx_pos + 3 * r), in1 = __ldg(rx_pos + 3 * r + 1), in2 = __ldg(rx_pos + 3 * r + 2);
      float pre = 0.0f;
      pre += w1_0 * in0;
      pre += w1_1 * in1;
      pre += w1_2 * in2;
      pre += b1;
      const float h = (pre > 0.0f) ? pre : (0.01f * pre);
      const float o0 = warp_sum(w2_0 * h) + b2_0;
      const float o1v = warp_sum(w2_1 * h) + b2_1;
      const float s0 = 1.0f / (1.0f + expf(-(o0 - log_d)));
      const float s1 = 1.0f / (1.0f + expf(-(o1v - log_d)));
      const float2 ds = reinterpret_cast<const float2*>(dsig)[rg];
      const float d0 = ds.x * s0 * (1.0f - s0);
      const float d1 = ds.y * s1 * (1.0f - s1);
      float dlogd = 0.0f;
      dlogd -= d0;
      dlogd -= d1;
      const float dd = dlogd / (d + 1e-6f);
      gm_x += -dd * unit.x;
      gm_y += -dd * unit.y;
      gm_z += -dd * unit.z;
      gw2_0 += d0 * h;
      gw2_1 += d1 * h;
      gb2_0 += d0;
      gb2_1 += d1;
      float dh = 0.0f;
      dh += d0 * w2_0;
      dh += d1 * w2_1;
      const float dpre = (pre > 0.0f) ? dh : (0.01f * dh);
      gw1_0 += dpre * in0;
      gw1_1 += dpre * in1;
      gw1_2 += dpre * in2;
      gb1 += dpre;
    }
    float* gw1 = dL_dmlp + (size_t)g * (kMlpIn * kMlpHidden) + lane * kMlpIn;
    gw1[0] = gw1_0; gw1[1] = gw1_1; gw1[2] = gw1_2;
    dL_dmlp[o1 + (size_t)g * kMlpHidden + lane] = gb1;
    dL_dmlp[o2 + (size_t)g * (kMlpOut * kMlpHidden) + lane] = gw2_0;
    dL_dmlp[o2 + (size_t)g * (kMlpOut * kMlpHidden) + kMlpHidden + lane] = gw2_1;
    if (lane == 0) {
      dL_dmlp[o3 + (size_t)g * kMlpOut] = gb2_0;
      dL_dmlp[o3 + (size_t)g * kMlpOut + 1] = gb2_1;
      dL_dmeans3D[(size_t)g * 3 + 0] += gm_x;
      dL_dmeans3D[(size_t)g * 3 + 1] += gm_y;
      dL_dmeans3D[(size_t)g * 3 + 2] += gm_z;
    }
  }
}

cudaError_t launch_geometry_backward(int P, int R, int H, int W, float mod, unsigned grad_mode,
                                     const float* means3D, const float* scales, const float* rotations,
                                     const float* views, const GeomView& geo, const float* dmean2D,
                                     const float* dconic, float* dL_dmeans3D, float* dL_dcov3D,
                                     float* dL_dscales, float* dL_drot, cudaStream_t stream) {
  if (P == 0) return cudaSuccess;
  geometry_backward_kernel<<<(P + 127) / 128, 128, 0, stream>>>(P, R, H, W, mod, grad_mode, means3D, scales,
                                                               rotations, views, geo, dmean2D, dconic, dL_dmeans3D,
                                                               dL_dcov3D, dL_dscales, dL_drot);
  return cudaGetLastError();
}

cudaError_t launch_emission_backward(int P, int R, const float* means3D, const float* mlp, const float* tx_pos,
                                     const float* rx_pos, const int* radii, const float* dsig, float* dL_dmlp,
                                     float* dL_dmeans3D, cudaStream_t stream) {
  if (P == 0) return cudaSuccess;
  const int warps_per_block = 8;
  int blocks = (P + warps_per_block - 1) / warps_per_block;
  const int cap = device_sm_count() * 16;   // persistent-style grid: 16 CTAs per SM
  if (blocks > cap) blocks = cap;
  emission_backward_kernel<<<blocks, 32 * warps_per_block, 0, stream>>>(P, R, means3D, mlp, tx_pos, rx_pos, radii,
                                                                        dsig, dL_dmlp, dL_dmeans3D);
  return cudaGetLastError();
}

}  // namespace gsparc
