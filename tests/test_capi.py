"""CPU tests of the C ABI and the host layer: the library loads, exports every
symbol include/gsparc_b200.h declares, sizes its arenas consistently and
rejects bad arguments before any CUDA call; the Python layer refuses CPU
tensors (there is no CPU fallback)."""
import ctypes
import os
import re

import pytest
import torch

from gsparc_b200 import _lib, raster

HEADER = os.path.join(os.path.dirname(__file__), "..", "include", "gsparc_b200.h")


def _declared():
    src = open(HEADER).read()
    return sorted(set(re.findall(r"GSPARC_API\s+[\w\s\*]+?\b(gsparc_\w+)\s*\(", src)))


def test_library_exports_every_declared_symbol():
    L = _lib.lib()
    names = _declared()
    assert len(names) >= 16
    for n in names:
        assert hasattr(L, n), n
    # the Python binding declares exactly the header's entry points
    assert sorted(_lib.exported_symbols()) == names


def test_abi_version_and_status_strings():
    L = _lib.lib()
    assert L.gsparc_abi_version() == 7
    for code, text in [(0, b"ok"), (1, b"invalid argument"), (2, b"CUDA error"), (3, b"binning capacity exceeded")]:
        assert L.gsparc_status_string(code) == text


def test_arena_sizes_and_layouts():
    for P, R in [(0, 1), (1, 1), (4096, 1), (50000, 64)]:
        n = _lib.geom_state_bytes(P, R)
        off = _lib.layout("geom", P, R)
        assert all(o % 256 == 0 for o in off) and off == sorted(off) and off[-1] + P * 6 * 4 <= n
    for (th, tw) in [(16, 16), (8, 32), (32, 8)]:
        n = _lib.image_state_bytes(3, 90, 360, th, tw)
        off = _lib.layout("image", 3, 90, 360, th, tw)
        assert off[0] == 0 and off[-1] + 3 * 90 * 360 * 4 <= n
    assert _lib.lib().gsparc_image_state_bytes(1, 90, 360, 16, 8) == 0     # invalid tile
    k = _lib.binning_state_bytes(1000)
    assert k >= 1000 * 8
    off = _lib.layout("binning", 1000)
    assert off[1] + 1000 * 4 <= off[2] <= k


def _call_prepare(**kw):
    a = dict(P=10, R=1, H=90, W=360, th=16, tw=16, flags=0, mod=1.0)
    a.update(kw)
    dummy = ctypes.c_void_p(16)   # never dereferenced: validation fails first
    return _lib.lib().gsparc_rasterize_prepare(a["P"], a["R"], a["H"], a["W"], a["th"], a["tw"], a["flags"],
                                               a["mod"], *([dummy] * 11), None, None)


@pytest.mark.parametrize("kw", [dict(th=16, tw=8), dict(th=4, tw=64), dict(R=0), dict(H=0), dict(P=-1),
                                dict(flags=2), dict(flags=0x101)])
def test_prepare_rejects_bad_arguments_without_cuda(kw):
    assert _call_prepare(**kw) == 1
    assert b"invalid argument" in _lib.lib().gsparc_last_error_detail()


def test_prepare_rejects_null_state():
    L = _lib.lib()
    d = ctypes.c_void_p(16)
    st = L.gsparc_rasterize_prepare(10, 1, 90, 360, 16, 16, 0, 1.0, d, d, d, d, d, d, d, d, None, None, d, None,
                                    None)
    assert st == 1


def test_backward_rejects_bad_grad_mode():
    L = _lib.lib()
    d = ctypes.c_void_p(16)
    st = L.gsparc_rasterize_backward(10, 1, 90, 360, 16, 16, 0, 1.0, 7, *([d] * 10), 10, *([d] * 11), None)
    assert st == 1
    assert b"grad_mode" in L.gsparc_last_error_detail()


def test_ssim_rejects_partial_derivative_maps():
    L = _lib.lib()
    d = ctypes.c_void_p(16)
    st = L.gsparc_ssim_forward(1, 1, 8, 8, 1e-4, 9e-4, d, d, d, d, None, None, None)
    assert st == 1


def test_python_layer_refuses_cpu_tensors():
    P = 4
    with pytest.raises(ValueError, match="CUDA"):
        raster.forward(torch.zeros(P, 3), torch.zeros(194 * P), torch.zeros(P), torch.zeros(P, 3),
                       torch.zeros(P, 4), 90, 360, 1.0, torch.eye(4), torch.zeros(3), torch.zeros(3))
    import wireless_rasterizer as wr
    with pytest.raises(RuntimeError, match="num_points, 3"):
        wr.rasterize_gaussians(torch.zeros(P, 2), None, None, None, None, 90, 360, 1.0, None, None, None, None)


def test_grad_mode_and_tile_switches():
    assert raster.get_grad_mode() == "reference"
    raster.set_grad_mode("exact")
    assert raster.get_grad_mode() == "exact"
    raster.set_grad_mode("reference")
    with pytest.raises(ValueError):
        raster.set_tile_shape(16, 8)
    raster.set_tile_shape(8, 32)
    assert raster.get_tile_shape() == (8, 32)
    raster.set_tile_shape(16, 16)


def test_training_state_layout_with_global_block():
    L = _lib.lib()
    for P, nm, nc in [(0, 0, 0), (1, 194, 161), (20000, 194 * 20000, 161), (3, 0, 0), (20000, 6337, 161)]:
        out = (ctypes.c_size_t * 6)()
        assert L.gsparc_gaussian_state_layout(P, nm, nc, out) == 0
        off = list(out)
        total = L.gsparc_gaussian_state_floats(P, nm, nc)
        sizes = [3 * P, 3 * P, 4 * P, P, nm, nc]
        assert off[0] == 0 and all(o % 64 == 0 for o in off)          # 256-byte aligned segments
        for i in range(5):
            assert off[i] + sizes[i] <= off[i + 1]
        assert off[5] + nc <= total and total % 64 == 0
    assert L.gsparc_gaussian_state_layout(-1, 0, 0, (ctypes.c_size_t * 6)()) == 1


def test_splat_loss_rejects_bad_arguments_without_cuda():
    L = _lib.lib()
    d = ctypes.c_void_p(16)
    args = lambda R, H, W, hid, scratch=d: (R, H, W, hid, 0.2, 0.3, 1e-4, 9e-4, d, d, d, d, scratch, d, None, d, d,
                                            None)
    assert L.gsparc_splat_loss(*args(0, 90, 360, 32)) == 1
    assert L.gsparc_splat_loss(*args(1, 90, 360, 0)) == 1
    assert L.gsparc_splat_loss(*args(70000, 90, 360, 32)) == 1
    assert L.gsparc_splat_loss(*args(1, 90, 360, 32, scratch=ctypes.c_void_p(20))) == 1   # misaligned
    assert b"aligned" in L.gsparc_last_error_detail()
    assert L.gsparc_splat_loss(*args(1, 90, 360, 32, scratch=None)) == 1
    n1 = L.gsparc_splat_loss_scratch_floats(1, 90, 360, 32)
    n4 = L.gsparc_splat_loss_scratch_floats(4, 90, 360, 32)
    assert n1 >= 3 * 90 * 360 and n4 >= 4 * 3 * 90 * 360 and n4 > n1


def test_adam_step_rejects_partial_activation_outputs():
    L = _lib.lib()
    d = ctypes.c_void_p(256)
    st = L.gsparc_gaussian_adam_step(10, 1940, 161, d, d, d, d, d, d, 0.9, 0.999, 1e-15, d, d, d, None, None, None)
    assert st == 1
    assert b"all three" in L.gsparc_last_error_detail()


def test_bf16_shared_mlp_workspace_layout():
    """The BF16 shared MLP's workspace: the sigmoid outputs [rows][out], then
    the BF16 pre-activations of every hidden layer for whole 128-row tiles,
    each segment rounded up to 64 floats (256 bytes); no feature-gradient
    segment (the adjoint applies it in place)."""
    L = _lib.lib()
    a = lambda x: (x + 63) // 64 * 64
    for P, R, layers, out in [(1, 1, 1, 1), (20000, 1, 3, 1), (4097, 3, 2, 1), (100000, 16, 3, 64),
                              (200000, 32, 3, 1)]:
        rows = P * R
        zrows = (rows + 127) // 128 * 128
        want = a(rows * out) + a(layers * zrows * 128 // 2)
        assert L.gsparc_shared_mlp_workspace_floats(P, R, layers, 128, out, 1) == want, (P, R, layers, out)


def test_static_ssim_rejects_sizes_whose_product_wraps():
    """B = CH = H = W = 65536 multiplies to 2^64, i.e. 0 in 64 bits; the
    allocation-free SSIM entry point must reject it (each factor is checked
    against the limit as the product grows) rather than report success."""
    L = _lib.lib()
    d = ctypes.c_void_p(16)     # never dereferenced: the size check fails first
    for dims in ((65536, 65536, 65536, 65536), (1 << 20, 1 << 20, 1 << 20, 16), (1, 1, 1 << 20, 2)):
        assert L.gsparc_ssim_static_scratch(*dims, 1e-4, 9e-4, d, d, d, d, d, None) == 1, dims
        assert b"1048576" in L.gsparc_last_error_detail()
    assert L.gsparc_ssim_static_scratch(0, 65536, 65536, 65536, 1e-4, 9e-4, d, d, d, d, d, None) == 0
