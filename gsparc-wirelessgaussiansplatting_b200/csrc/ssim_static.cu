// Fused SSIM map + gradient with no allocation anywhere: the three
// partial-derivative maps the gradient needs live in a fixed, file-scope
// device array instead of caller- or library-allocated memory.
//
// For callers that cannot call cudaMalloc: e.g. a real-time receiver loop
// whose latency budget cannot absorb cudaMalloc's implicit device
// synchronisation, or a host process that was handed a fixed set of device
// buffers by another runtime and owns no allocator of its own.  They pass the
// two images, dL/dmap and the two outputs; nothing else is needed.
//
// Limits and sharing:
//  * at most kStaticSsimMaxPixels = 1,048,576 pixels per call (B*CH*H*W),
//    e.g. 32 spectra of 90x360; every GPU that loads the library holds the
//    12 MiB array until the process exits;
//  * every call on a device uses the same array and leaves the last call's
//    maps in it; nothing in it has to start at zero (each call writes every
//    element it later reads), but two calls whose work overlaps on the GPU
//    (different streams without ordering) race on it;
//  * the first call on a device looks up the array's device address with
//    cudaGetSymbolAddress (with that device current) and caches it; make that
//    first call before any stream capture.
#include <initializer_list>
#include <mutex>

#include "common.cuh"
#include "kernels.cuh"

namespace {

constexpr size_t kStaticSsimMaxPixels = size_t(1) << 20;
static_assert(kStaticSsimMaxPixels == GSPARC_SSIM_STATIC_MAX_PIXELS,
              "the header's GSPARC_SSIM_STATIC_MAX_PIXELS must equal the scratch array's pixel limit");

// file-scope device scratch: dm/dmu1 | dm/dsigma1^2 | dm/dsigma12
static __device__ __align__(256) float g_ssim_static_scratch[3 * kStaticSsimMaxPixels];

std::mutex g_static_mu;
float* g_static_ptr[64] = {nullptr};

// Device address of the scratch array on the current device (the symbol name
// in host code is only a host-side stand-in, never a device address).
cudaError_t static_scratch(float** out) {
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return e;
  if (dev < 0 || dev >= 64) return cudaErrorInvalidDevice;
  std::lock_guard<std::mutex> lk(g_static_mu);
  if (!g_static_ptr[dev]) {
    void* p = nullptr;
    e = cudaGetSymbolAddress(&p, g_ssim_static_scratch);
    if (e != cudaSuccess) return e;
    g_static_ptr[dev] = static_cast<float*>(p);
  }
  *out = g_static_ptr[dev];
  return cudaSuccess;
}

}  // namespace

extern "C" int gsparc_ssim_static_scratch(int B, int CH, int H, int W, float C1, float C2, const float* img1,
                                          const float* img2, const float* dL_dmap, float* ssim_map,
                                          float* dL_dimg1, void* stream) {
  using namespace gsparc;
  if (B < 0 || CH < 0 || H < 0 || W < 0) return report_invalid("sizes");
  if (B == 0 || CH == 0 || H == 0 || W == 0) return GSPARC_OK;
  // the running product is checked after every factor, so it never exceeds
  // 2^20 * 2^31 and cannot wrap
  size_t n = 1;
  for (int f : {B, CH, H, W}) {
    n *= (size_t)f;
    if (n > kStaticSsimMaxPixels)
      return report_invalid("B*CH*H*W exceeds the 1048576 pixels of gsparc_ssim_static_scratch's static scratch");
  }
  if (!img1 || !img2 || !dL_dmap || !ssim_map || !dL_dimg1) return report_invalid("null pointer");
  float* scratch = nullptr;
  cudaError_t e = static_scratch(&scratch);
  if (e != cudaSuccess) return report_cuda(e, "static scratch address");
  cudaStream_t s = (cudaStream_t)stream;
  float* dmu1 = scratch;
  float* ds11 = scratch + n;
  float* ds12 = scratch + 2 * n;
  e = launch_ssim_forward(B * CH, H, W, C1, C2, img1, img2, ssim_map, dmu1, ds11, ds12, s);
  if (e != cudaSuccess) return report_cuda(e, "ssim forward (static scratch)");
  e = launch_ssim_backward(B * CH, H, W, img1, img2, dL_dmap, dmu1, ds11, ds12, dL_dimg1, s);
  if (e != cudaSuccess) return report_cuda(e, "ssim backward (static scratch)");
  return GSPARC_OK;
}
