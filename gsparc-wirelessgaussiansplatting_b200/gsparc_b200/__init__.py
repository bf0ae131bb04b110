"""sm_100a implementation of GSpaRC's differentiable equirectangular RF
splatting path.  The drop-in modules ``wireless_rasterizer``,
``cuda_kernel_rasterize.cuda_rasterizer``, ``fused_ssim_cuda`` and
``fused_ssim`` live next to this package; this package holds the C-ABI
binding, the batched API and the synthetic scenes."""
from . import _lib, raster, scenes  # noqa: F401
from .raster import set_grad_mode, get_grad_mode, set_tile_shape, get_tile_shape  # noqa: F401
