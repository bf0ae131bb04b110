"""ctypes binding of the C ABI in include/gsparc_b200.h.

The shared library is built in-tree (``make -C gsparc-wirelessgaussiansplatting_b200``
or ``__graft_entry__.build()``).  There is no fallback: if the library is
missing or fails to load, every entry point raises.
"""
from __future__ import annotations

import ctypes
import os

import torch

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libgsparc_b200.so")

GRAD_REFERENCE = 0
GRAD_EXACT = 1
FLAG_WRAP_AZIMUTH = 1   # GSPARC_FLAG_WRAP_AZIMUTH

_c_int, _c_ll, _c_size, _c_float, _c_uint = ctypes.c_int, ctypes.c_longlong, ctypes.c_size_t, ctypes.c_float, ctypes.c_uint
_vp = ctypes.c_void_p


class GsparcError(RuntimeError):
    """A C-ABI entry point returned a non-zero status."""

    def __init__(self, where: str, status: int, text: str, detail: str):
        super().__init__(f"{where} failed: {text} ({detail})" if detail else f"{where} failed: {text}")
        self.status = status


_SIGS = {
    "gsparc_abi_version": (_c_int, []),
    "gsparc_status_string": (ctypes.c_char_p, [_c_int]),
    "gsparc_last_error_detail": (ctypes.c_char_p, []),
    "gsparc_geom_state_bytes": (_c_size, [_c_int, _c_int]),
    "gsparc_image_state_bytes": (_c_size, [_c_int, _c_int, _c_int, _c_int, _c_int]),
    "gsparc_binning_state_bytes": (_c_size, [_c_ll]),
    "gsparc_geom_state_layout": (_c_int, [_c_int, _c_int, ctypes.POINTER(_c_size)]),
    "gsparc_image_state_layout": (_c_int, [_c_int, _c_int, _c_int, _c_int, _c_int, ctypes.POINTER(_c_size)]),
    "gsparc_binning_state_layout": (_c_int, [_c_ll, ctypes.POINTER(_c_size)]),
    "gsparc_rasterize_prepare": (_c_int, [_c_int, _c_int, _c_int, _c_int, _c_int, _c_int, _c_uint, _c_float,
                                          _vp, _vp, _vp, _vp, _vp, _vp, _vp, _vp, _vp, _vp, _vp,
                                          ctypes.POINTER(_c_ll), _vp]),
    "gsparc_rasterize_render": (_c_int, [_c_int, _c_int, _c_int, _c_int, _c_int, _c_int, _c_uint,
                                         _vp, _vp, _vp, _c_ll, _vp, _vp, _vp]),
    "gsparc_read_status": (_c_int, [_vp, ctypes.POINTER(_c_ll), ctypes.POINTER(_c_uint), _vp]),
    "gsparc_rasterize_backward": (_c_int, [_c_int, _c_int, _c_int, _c_int, _c_int, _c_int, _c_uint, _c_float,
                                           _c_uint,
                                           _vp, _vp, _vp, _vp, _vp, _vp, _vp, _vp, _vp, _vp, _c_ll,
                                           _vp, _vp, _vp, _vp, _vp, _vp, _vp, _vp, _vp, _vp, _vp, _vp]),
    "gsparc_rasterize_render_channels": (_c_int, [_c_int, _c_int, _c_int, _c_int, _c_int, _c_int, _c_uint, _c_int,
                                                  _vp, _vp, _vp, _c_ll, _vp, _vp, _vp]),
    "gsparc_rasterize_backward_channels": (_c_int, [_c_int, _c_int, _c_int, _c_int, _c_int, _c_int, _c_uint, _c_int,
                                                    _c_float, _vp, _vp, _vp, _vp, _vp, _vp, _vp, _c_ll, _vp, _vp,
                                                    _vp, _vp, _vp, _vp, _vp, _vp, _vp, _vp, _vp]),
    "gsparc_mark_visible": (_c_int, [_c_int, _vp, _vp, _vp, _vp]),
    "gsparc_ssim_forward": (_c_int, [_c_int, _c_int, _c_int, _c_int, _c_float, _c_float,
                                     _vp, _vp, _vp, _vp, _vp, _vp, _vp]),
    "gsparc_ssim_backward": (_c_int, [_c_int, _c_int, _c_int, _c_int, _c_float, _c_float,
                                      _vp, _vp, _vp, _vp, _vp, _vp, _vp, _vp]),
    "gsparc_ssim_static_scratch": (_c_int, [_c_int, _c_int, _c_int, _c_int, _c_float, _c_float,
                                            _vp, _vp, _vp, _vp, _vp, _vp]),
    "gsparc_shared_mlp_param_floats": (_c_size, [_c_int, _c_int, _c_int]),
    "gsparc_shared_mlp_workspace_floats": (_c_size, [_c_int] * 6),
    "gsparc_shared_mlp_forward": (_c_int, [_c_int] * 7 + [_vp] * 7),
    "gsparc_shared_mlp_backward": (_c_int, [_c_int] * 7 + [_vp] * 10),
    "gsparc_shared_mlp_bf16_act_table": (_c_int, [_c_int, _vp, _vp]),
    "gsparc_splat_loss_scratch_floats": (_c_size, [_c_int, _c_int, _c_int, _c_int]),
    "gsparc_splat_loss": (_c_int, [_c_int, _c_int, _c_int, _c_int, _c_float, _c_float, _c_float, _c_float,
                                   _vp, _vp, _vp, _vp, _vp, _vp, _vp, _vp, _vp, _vp]),
    "gsparc_eval_scratch_floats": (_c_size, [_c_int, _c_int, _c_int]),
    "gsparc_eval_metrics": (_c_int, [_c_int, _c_int, _c_int, _c_int, _c_float, _c_float, _c_float,
                                     _vp, _vp, _vp, _vp, _vp, _vp, _vp]),
    "gsparc_densify_stats": (_c_int, [_c_int, _c_int, _vp, _vp, _vp, _vp, _vp, _vp]),
    "gsparc_densify_work_ints": (_c_size, [_c_int]),
    "gsparc_densify_count": (_c_int, [_c_int, _c_ll, _c_int, _c_int, _vp, _vp, _vp, _c_float, _c_float, _c_float,
                                      _c_float, _c_float, _vp, ctypes.c_ulonglong, _vp, _vp, _vp]),
    "gsparc_densify_apply": (_c_int, [_c_int, _c_int, _c_ll, _c_int, _c_int, _vp, _vp, _vp, _c_float, _c_float,
                                      _c_float, _c_float, _c_float, _vp, ctypes.c_ulonglong, _vp, _vp, _vp, _vp, _vp]),
    "gsparc_reset_opacity": (_c_int, [_c_int, _c_ll, _c_int, _vp, _vp, _vp, _vp]),
    "gsparc_gaussian_state_floats": (_c_size, [_c_int, _c_ll, _c_int]),
    "gsparc_gaussian_state_layout": (_c_int, [_c_int, _c_ll, _c_int, ctypes.POINTER(_c_size)]),
    "gsparc_gaussian_activate": (_c_int, [_c_int, _vp, _vp, _vp, _vp, _vp]),
    "gsparc_gaussian_adam_step": (_c_int, [_c_int, _c_ll, _c_int, _vp, _vp, _vp, _vp, _vp, _vp, _c_float,
                                           _c_float, _c_float, _vp, _vp, _vp, _vp, _vp, _vp]),
    "gsparc_timing_enable": (_c_int, [_c_int]),
    "gsparc_timing_kernel_count": (_c_int, []),
    "gsparc_timing_kernel_name": (ctypes.c_char_p, [_c_int]),
    "gsparc_timing_read": (_c_int, [ctypes.POINTER(ctypes.c_double), ctypes.POINTER(_c_ll), _c_int, _c_int]),
    "gsparc_depth_sort_launches": (_c_int, [_c_int, _c_int]),
    "gsparc_set_wait_limit": (_c_int, [_c_ll]),
}

_lib = None


def lib() -> ctypes.CDLL:
    """Load libgsparc_b200.so (once) and declare every exported signature."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise RuntimeError(
                f"{LIB_PATH} is not built: run `make -C {os.path.dirname(_HERE)}` "
                "(or __graft_entry__.build()); there is no CPU fallback")
        handle = ctypes.CDLL(LIB_PATH)
        for name, (res, args) in _SIGS.items():
            fn = getattr(handle, name)
            fn.restype = res
            fn.argtypes = args
        _lib = handle
    return _lib


def exported_symbols():
    """Names of every entry point this binding declares."""
    return list(_SIGS)


def check(where: str, status: int) -> None:
    if status != 0:
        L = lib()
        raise GsparcError(where, status, L.gsparc_status_string(status).decode(),
                          L.gsparc_last_error_detail().decode())


def ptr(t):
    """Raw device pointer of a tensor (None -> NULL)."""
    return None if t is None else ctypes.c_void_p(t.data_ptr())


def stream_of(device) -> ctypes.c_void_p:
    """The current torch stream on ``device`` as a cudaStream_t."""
    return ctypes.c_void_p(torch.cuda.current_stream(device).cuda_stream)


def geom_state_bytes(P, R):
    return int(lib().gsparc_geom_state_bytes(P, R))


def image_state_bytes(R, H, W, tile_h, tile_w):
    n = int(lib().gsparc_image_state_bytes(R, H, W, tile_h, tile_w))
    if n == 0:
        raise ValueError(f"invalid image state request R={R} H={H} W={W} tile={tile_h}x{tile_w}")
    return n


def binning_state_bytes(K):
    return int(lib().gsparc_binning_state_bytes(int(K)))


def layout(kind: str, *args):
    """Byte offsets of the sub-arrays of an arena ('geom', 'image', 'binning')."""
    L = lib()
    if kind == "geom":
        out = (_c_size * 6)()
        check("geom layout", L.gsparc_geom_state_layout(*args, out))
    elif kind == "image":
        out = (_c_size * 6)()
        check("image layout", L.gsparc_image_state_layout(*args, out))
    else:
        out = (_c_size * 3)()
        check("binning layout", L.gsparc_binning_state_layout(*args, out))
    return [int(v) for v in out]


class KernelTimer:
    """Per-kernel device time of this library's launches (CUDA events around
    each launch).  Use as a context manager around the region to measure;
    ``results()`` gives {kernel name: (total ms, launches)}."""

    def __enter__(self):
        L = lib()
        n = L.gsparc_timing_kernel_count()
        L.gsparc_timing_read(None, None, n, 1)     # drop anything pending
        L.gsparc_timing_enable(1)
        return self

    def __exit__(self, *exc):
        L = lib()
        L.gsparc_timing_enable(0)
        n = L.gsparc_timing_kernel_count()
        ms = (ctypes.c_double * n)()
        cnt = (_c_ll * n)()
        check("timing_read", L.gsparc_timing_read(ms, cnt, n, 1))
        self._res = {L.gsparc_timing_kernel_name(i).decode(): (float(ms[i]), int(cnt[i])) for i in range(n)}
        return False

    def results(self):
        return dict(self._res)
