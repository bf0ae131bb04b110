"""Host-side driver of the C ABI: arena allocation, argument checks, batching.

Everything here allocates through the torch caching allocator and launches
on the current torch stream; the arithmetic all happens in the sm_100a
kernels behind ``libgsparc_b200.so``.

Shapes (R receivers, P Gaussians, spectra H x W):
  means3D [P,3], emission_mlps [194*P], opacities [P] or [P,1], scales [P,3],
  rotations [P,4], viewmatrices [R,4,4] or [4,4], tx_pos [3], rx_pos [R,3] or [3].
"""
from __future__ import annotations

import ctypes
from dataclasses import dataclass

import torch

from . import _lib
from ._lib import check, ptr, stream_of

MLP_FLOATS = 194

_tile = (16, 16)
_grad_mode = _lib.GRAD_REFERENCE


def set_tile_shape(tile_h: int, tile_w: int) -> None:
    """Tile shape used by the drop-in path (16x16 like the reference, or 8x32 /
    32x8).  Only 16x16 reproduces the reference's binning bit for bit."""
    if (tile_h, tile_w) not in ((16, 16), (8, 32), (32, 8)):
        raise ValueError("tile shape must be 16x16, 8x32 or 32x8")
    global _tile
    _tile = (tile_h, tile_w)


def get_tile_shape():
    return _tile


def set_grad_mode(mode: str) -> None:
    """'reference' reproduces the reference backward (halved azimuth Jacobian
    row, real-only alpha gradient); 'exact' is the true derivative."""
    global _grad_mode
    _grad_mode = {"reference": _lib.GRAD_REFERENCE, "exact": _lib.GRAD_EXACT}[mode]


def get_grad_mode() -> str:
    return "reference" if _grad_mode == _lib.GRAD_REFERENCE else "exact"


def _dev_f32(t: torch.Tensor, name: str, device=None) -> torch.Tensor:
    if not isinstance(t, torch.Tensor):
        raise TypeError(f"{name} must be a torch.Tensor")
    if not t.is_cuda:
        raise ValueError(f"{name} must be a CUDA tensor")
    if device is not None and t.device != device:
        raise ValueError(f"{name} is on {t.device}, expected {device}")
    if t.dtype != torch.float32:
        raise TypeError(f"{name} must be float32, got {t.dtype}")
    return t.contiguous()


@dataclass
class ForwardState:
    """Arenas and sizes of one forward; handed to the backward."""
    P: int
    R: int
    H: int
    W: int
    tile: tuple
    capacity: int
    num_rendered: int
    geom: torch.Tensor
    image: torch.Tensor
    binning: torch.Tensor
    flags: int = 0


def _receivers(viewmatrices, rx_pos, device):
    v = _dev_f32(viewmatrices, "viewmatrix", device)
    rx = _dev_f32(rx_pos, "rx_pos", device)
    if v.dim() == 2:
        v = v.unsqueeze(0)
    if rx.dim() == 1:
        rx = rx.unsqueeze(0)
    if v.shape[1:] != (4, 4):
        raise ValueError("viewmatrix must be [4,4] or [R,4,4]")
    if rx.shape[1] != 3 or rx.shape[0] != v.shape[0]:
        raise ValueError("rx_pos must be [3] or [R,3] matching the view matrices")
    return v.contiguous(), rx.contiguous()


def forward(means3D, emission_mlps, opacities, scales, rotations, H, W, scale_modifier,
            viewmatrices, tx_pos, rx_pos, tile=None, capacity=None, binning=None,
            out_real=None, out_imag=None, radii=None, geom=None, image=None, shared=None, shared_params=None,
            wrap=False):
    """Render R spectra.  Returns (out_real [R,H,W], out_imag [R,H,W], radii [R,P] int32, ForwardState).

    With ``capacity=None`` the instance count K is read back (one host sync,
    as the reference does) and the binning arena is sized exactly.  With a
    capacity the call stays asynchronous (graph-capturable); an overflow is
    reported by ``read_status``.  Preallocated arenas/outputs may be passed.
    With ``shared`` (a ``SharedMLP``) and its flat ``shared_params`` the
    signals come from the shared emission MLP and ``emission_mlps`` must be
    None.  ``wrap=True`` continues footprints across the 0/2pi azimuth seam
    (GSPARC_FLAG_WRAP_AZIMUTH); the default clamps them at the image edges as
    the reference does."""
    if means3D.dim() != 2 or means3D.shape[1] != 3:
        raise RuntimeError("means3D must have dimensions (num_points, 3)")
    device = means3D.device
    m = _dev_f32(means3D, "means3D")
    P = m.shape[0]
    tile = tuple(tile or _tile)
    H, W = int(H), int(W)
    v, rx = _receivers(viewmatrices, rx_pos, device)
    R = v.shape[0]
    tx = _dev_f32(tx_pos, "tx_pos", device).reshape(-1)
    if tx.numel() != 3:
        raise ValueError("tx_pos must have 3 elements")
    if shared is not None and emission_mlps is not None:
        raise ValueError("pass either emission_mlps (per-Gaussian MLP) or shared (shared MLP), not both")
    if P > 0:
        if shared is None:
            mlp = _dev_f32(emission_mlps, "emission_mlps", device).reshape(-1)
            if mlp.numel() != MLP_FLOATS * P:
                raise ValueError(f"emission_mlps must hold {MLP_FLOATS}*P = {MLP_FLOATS * P} floats, "
                                 f"got {mlp.numel()}")
        else:
            mlp = None
            shared_params = _dev_f32(shared_params, "shared_params", device).reshape(-1)
            if shared_params.numel() != shared.n_params:
                raise ValueError(f"shared_params must hold {shared.n_params} floats")
        op = _dev_f32(opacities, "opacities", device).reshape(-1)
        sc = _dev_f32(scales, "scales", device).reshape(P, 3)
        rot = _dev_f32(rotations, "rotations", device).reshape(P, 4)
        if op.numel() != P:
            raise ValueError("opacities must have P elements")
    else:
        mlp = op = sc = rot = None
    L = _lib.lib()
    if out_real is None:
        out_real = torch.zeros((R, H, W), dtype=torch.float32, device=device)
    if out_imag is None:
        out_imag = torch.zeros((R, H, W), dtype=torch.float32, device=device)
    if radii is None:
        radii = torch.zeros((R, P), dtype=torch.int32, device=device)
    if geom is None:
        geom = torch.empty(_lib.geom_state_bytes(P, R), dtype=torch.uint8, device=device)
    if image is None:
        image = torch.empty(_lib.image_state_bytes(R, H, W, *tile), dtype=torch.uint8, device=device)
    stream = stream_of(device)
    K = ctypes.c_longlong(0)
    flags = _lib.FLAG_WRAP_AZIMUTH if wrap else 0
    check("rasterize_prepare", L.gsparc_rasterize_prepare(
        P, R, H, W, tile[0], tile[1], flags, float(scale_modifier), ptr(m), ptr(mlp), ptr(op), ptr(sc), ptr(rot),
        ptr(v), ptr(tx), ptr(rx), ptr(radii), ptr(geom), ptr(image),
        ctypes.byref(K) if capacity is None else None, stream))
    if shared is not None:
        shared.forward(P, R, m, rx, shared_params, geom, image)
    if capacity is None:
        capacity = int(K.value)
        num_rendered = capacity
    else:
        num_rendered = -1
    if binning is None:
        binning = torch.empty(max(_lib.binning_state_bytes(capacity), 1), dtype=torch.uint8, device=device)
    check("rasterize_render", L.gsparc_rasterize_render(
        P, R, H, W, tile[0], tile[1], flags, ptr(geom), ptr(image), ptr(binning), int(capacity),
        ptr(out_real), ptr(out_imag), stream))
    st = ForwardState(P, R, H, W, tile, int(capacity), num_rendered, geom, image, binning, flags)
    return out_real, out_imag, radii, st


def read_status(st: ForwardState):
    """Synchronise and return (K, error_word); raises on capacity overflow."""
    L = _lib.lib()
    K = ctypes.c_longlong(0)
    err = ctypes.c_uint(0)
    status = L.gsparc_read_status(ptr(st.image), ctypes.byref(K), ctypes.byref(err), stream_of(st.image.device))
    check("read_status", status)
    return int(K.value), int(err.value)


def backward(st: ForwardState, means3D, emission_mlps, scales, rotations, scale_modifier,
             viewmatrices, tx_pos, rx_pos, dL_dout_real, dL_dout_imag, grad_mode=None, out=None,
             shared=None, shared_params=None):
    """Adjoint of ``forward``.  Returns a dict of gradient tensors:
    dmeans2D [R,P,3], dconic [R,P,4], dsignal [R,P,2], dopacity [P],
    dmeans3D [P,3], dcov3D [P,6], dscales [P,3], drotations [P,4], dmlp [194*P]
    (per-Gaussian MLP) or dshared [n_params] (``shared``)."""
    device = means3D.device
    P, R, H, W = st.P, st.R, st.H, st.W
    mode = _grad_mode if grad_mode is None else {"reference": _lib.GRAD_REFERENCE, "exact": _lib.GRAD_EXACT}.get(grad_mode, grad_mode)
    m = _dev_f32(means3D, "means3D")
    v, rx = _receivers(viewmatrices, rx_pos, device)
    tx = _dev_f32(tx_pos, "tx_pos", device).reshape(-1)
    g_r = _dev_f32(dL_dout_real, "dL_dout_real", device).reshape(R, H, W)
    g_i = _dev_f32(dL_dout_imag, "dL_dout_imag", device).reshape(R, H, W)
    if out is None:
        z = lambda *s: torch.empty(s, dtype=torch.float32, device=device)
        out = dict(dmeans2D=z(R, P, 3), dconic=z(R, P, 4), dsignal=z(R, P, 2), dopacity=z(P),
                   dmeans3D=z(P, 3), dcov3D=z(P, 6), dscales=z(P, 3), drotations=z(P, 4))
        if shared is None:
            out["dmlp"] = z(MLP_FLOATS * P)
        else:
            out["dshared"] = z(shared.n_params)
    if P == 0:
        for t in out.values():
            t.zero_()
        return out
    mlp = _dev_f32(emission_mlps, "emission_mlps", device).reshape(-1) if shared is None else None
    sc = _dev_f32(scales, "scales", device).reshape(P, 3)
    rot = _dev_f32(rotations, "rotations", device).reshape(P, 4)
    L = _lib.lib()
    check("rasterize_backward", L.gsparc_rasterize_backward(
        P, R, H, W, st.tile[0], st.tile[1], st.flags, float(scale_modifier), int(mode),
        ptr(m), ptr(mlp), ptr(sc), ptr(rot), ptr(v), ptr(tx), ptr(rx),
        ptr(st.geom), ptr(st.image), ptr(st.binning), int(st.capacity), ptr(g_r), ptr(g_i),
        ptr(out["dmeans2D"]), ptr(out["dconic"]), ptr(out["dsignal"]), ptr(out["dopacity"]),
        ptr(out["dmeans3D"]), ptr(out["dcov3D"]), ptr(out["dscales"]), ptr(out["drotations"]),
        ptr(out["dmlp"]) if shared is None else None, stream_of(device)))
    if shared is not None:
        sp = _dev_f32(shared_params, "shared_params", device).reshape(-1)
        shared.backward(P, R, m, rx, sp, st.geom, out["dsignal"], out["dshared"], out["dmeans3D"], st.image)
    return out


def forward_channels(means3D, opacities, scales, rotations, H, W, scale_modifier, viewmatrices, tx_pos, rx_pos,
                     shared, shared_params, tile=None, capacity=None, binning=None, out=None, radii=None, geom=None,
                     image=None, wrap=False):
    """Render R x C spectra: the shared emission MLP with ``shared.out = C``
    outputs gives every (receiver, Gaussian) pair C amplitudes (one per
    frequency bin), blended with one set of transmittance decisions
    (gsparc_rasterize_render_channels).  Returns (out [R,C,H,W], radii [R,P],
    ForwardState); the amplitudes are ``shared.features(P, R)``."""
    if means3D.dim() != 2 or means3D.shape[1] != 3:
        raise RuntimeError("means3D must have dimensions (num_points, 3)")
    if shared is None or not (shared.precision == "fp32" or shared.out == 64):
        raise ValueError("forward_channels needs a SharedMLP with out = channels (BF16: out = 64)")
    device = means3D.device
    tile = tuple(_tile if tile is None else tile)
    P = means3D.shape[0]
    v, rx = _receivers(viewmatrices, rx_pos, device)
    R, C = v.shape[0], shared.out
    m = _dev_f32(means3D, "means3D")
    tx = _dev_f32(tx_pos, "tx_pos", device).reshape(-1)
    op = _dev_f32(opacities, "opacities", device).reshape(-1)
    sc = _dev_f32(scales, "scales", device).reshape(P, 3)
    rot = _dev_f32(rotations, "rotations", device).reshape(P, 4)
    sp = _dev_f32(shared_params, "shared_params", device).reshape(-1)
    if sp.numel() != shared.n_params:
        raise ValueError(f"shared_params must hold {shared.n_params} floats")
    L = _lib.lib()
    if out is None:
        out = torch.zeros((R, C, H, W), dtype=torch.float32, device=device)
    if radii is None:
        radii = torch.zeros((R, P), dtype=torch.int32, device=device)
    if geom is None:
        geom = torch.empty(_lib.geom_state_bytes(P, R), dtype=torch.uint8, device=device)
    if image is None:
        image = torch.empty(_lib.image_state_bytes(R, H, W, *tile), dtype=torch.uint8, device=device)
    stream = stream_of(device)
    flags = _lib.FLAG_WRAP_AZIMUTH if wrap else 0
    K = ctypes.c_longlong(0)
    check("rasterize_prepare", L.gsparc_rasterize_prepare(
        P, R, H, W, tile[0], tile[1], flags, float(scale_modifier), ptr(m), None, ptr(op), ptr(sc), ptr(rot),
        ptr(v), ptr(tx), ptr(rx), ptr(radii), ptr(geom), ptr(image),
        ctypes.byref(K) if capacity is None else None, stream))
    shared.forward(P, R, m, rx, sp, geom, image)
    feats = shared.features(P, R)
    if capacity is None:
        capacity = int(K.value)
        num_rendered = capacity
    else:
        num_rendered = -1
    if binning is None:
        binning = torch.empty(max(_lib.binning_state_bytes(capacity), 1), dtype=torch.uint8, device=device)
    check("rasterize_render_channels", L.gsparc_rasterize_render_channels(
        P, R, H, W, tile[0], tile[1], flags, C, ptr(geom), ptr(image), ptr(binning), int(capacity), ptr(feats),
        ptr(out), stream))
    st = ForwardState(P, R, H, W, tile, int(capacity), num_rendered, geom, image, binning, flags)
    return out, radii, st


def backward_channels(st: ForwardState, means3D, scales, rotations, scale_modifier, viewmatrices, tx_pos, rx_pos,
                      dL_dout, shared, shared_params, out=None):
    """Adjoint of ``forward_channels`` (true derivative).  Returns a dict:
    dmeans2D [R,P,3], dconic [R,P,4], dfeatures [R,P,C], dopacity [P],
    dmeans3D [P,3], dcov3D [P,6], dscales [P,3], drotations [P,4],
    dshared [n_params]."""
    device = means3D.device
    P, R, H, W = st.P, st.R, st.H, st.W
    C = shared.out
    m = _dev_f32(means3D, "means3D")
    v, rx = _receivers(viewmatrices, rx_pos, device)
    g = _dev_f32(dL_dout, "dL_dout", device).reshape(R, C, H, W)
    if out is None:
        z = lambda *s: torch.empty(s, dtype=torch.float32, device=device)
        out = dict(dmeans2D=z(R, P, 3), dconic=z(R, P, 4), dfeatures=z(R, P, C), dopacity=z(P), dmeans3D=z(P, 3),
                   dcov3D=z(P, 6), dscales=z(P, 3), drotations=z(P, 4), dshared=z(shared.n_params))
    if P == 0:
        for t in out.values():
            t.zero_()
        return out
    sc = _dev_f32(scales, "scales", device).reshape(P, 3)
    rot = _dev_f32(rotations, "rotations", device).reshape(P, 4)
    sp = _dev_f32(shared_params, "shared_params", device).reshape(-1)
    feats = shared.features(P, R)
    check("rasterize_backward_channels", _lib.lib().gsparc_rasterize_backward_channels(
        P, R, H, W, st.tile[0], st.tile[1], st.flags, C, float(scale_modifier), ptr(m), ptr(sc), ptr(rot), ptr(v),
        ptr(st.geom), ptr(st.image), ptr(st.binning), int(st.capacity), ptr(feats), ptr(g), ptr(out["dfeatures"]),
        ptr(out["dmeans2D"]), ptr(out["dconic"]), ptr(out["dopacity"]), ptr(out["dmeans3D"]), ptr(out["dcov3D"]),
        ptr(out["dscales"]), ptr(out["drotations"]), stream_of(device)))
    shared.backward(P, R, m, rx, sp, st.geom, out["dfeatures"], out["dshared"], out["dmeans3D"], st.image)
    return out


def mark_visible(means3D, viewmatrix):
    m = _dev_f32(means3D, "means3D")
    v = _dev_f32(viewmatrix, "viewmatrix", m.device).reshape(16)
    P = m.shape[0]
    present = torch.zeros(P, dtype=torch.uint8, device=m.device)
    check("mark_visible", _lib.lib().gsparc_mark_visible(P, ptr(m), ptr(v), ptr(present), stream_of(m.device)))
    return present.bool()


def state_views(st: ForwardState):
    """Typed views into the arenas of a forward (for inspection and tests):
    means2D [R,P,2], depth [R,P], radii [R,P], conic_opacity [R,P,4],
    signal [R,P,2], cov3D [P,6], num_rendered, ranges [R,T,2] (uint32 as int32),
    final_T [R,H,W], n_contrib [R,H,W] (int32), point_list [K] (int32)."""
    P, R, H, W = st.P, st.R, st.H, st.W
    th, tw = st.tile
    T = ((W + tw - 1) // tw) * ((H + th - 1) // th)
    go = _lib.layout("geom", P, R)
    io = _lib.layout("image", R, H, W, th, tw)
    bo = _lib.layout("binning", st.capacity)

    def view(buf, off, n, dtype, shape):
        nbytes = n * torch.empty((), dtype=dtype).element_size()
        return buf[off:off + nbytes].view(dtype).reshape(shape)

    out = {}
    if P > 0:
        out["means2D"] = view(st.geom, go[0], R * P * 2, torch.float32, (R, P, 2))
        out["depth"] = view(st.geom, go[1], R * P, torch.float32, (R, P))
        out["radii"] = view(st.geom, go[2], R * P, torch.int32, (R, P))
        out["conic_opacity"] = view(st.geom, go[3], R * P * 4, torch.float32, (R, P, 4))
        out["signal"] = view(st.geom, go[4], R * P * 2, torch.float32, (R, P, 2))
        out["cov3D"] = view(st.geom, go[5], P * 6, torch.float32, (P, 6))
    out["num_rendered"] = view(st.image, io[0], 1, torch.int64, (1,))
    out["ranges"] = view(st.image, io[1], R * T * 2, torch.int32, (R, T, 2))
    out["final_T"] = view(st.image, io[4], R * H * W, torch.float32, (R, H, W))
    out["n_contrib"] = view(st.image, io[5], R * H * W, torch.int32, (R, H, W))
    if st.capacity > 0:
        out["point_list"] = view(st.binning, bo[1], st.capacity, torch.int32, (st.capacity,))
    return out


def ssim_forward(img1, img2, C1, C2, train=True):
    """fusedssim: returns (map, dm_dmu1, dm_dsigma1_sq, dm_dsigma12); the last
    three are empty tensors when ``train`` is False."""
    a = _dev_f32(img1, "img1")
    b = _dev_f32(img2, "img2", a.device)
    if a.dim() != 4 or a.shape != b.shape:
        raise ValueError("img1 and img2 must both be [B,CH,H,W] with the same shape")
    B, CH, H, W = a.shape
    mp = torch.empty_like(a)          # the kernel writes every pixel of each output
    if train:
        d1, d2, d3 = torch.empty_like(a), torch.empty_like(a), torch.empty_like(a)
    else:
        d1 = d2 = d3 = torch.empty(0, device=a.device)
    check("ssim_forward", _lib.lib().gsparc_ssim_forward(
        B, CH, H, W, float(C1), float(C2), ptr(a), ptr(b), ptr(mp),
        ptr(d1) if train else None, ptr(d2) if train else None, ptr(d3) if train else None, stream_of(a.device)))
    return mp, d1, d2, d3


def ssim_backward(img1, img2, dL_dmap, dm_dmu1, dm_dsigma1_sq, dm_dsigma12, C1, C2):
    a = _dev_f32(img1, "img1")
    b = _dev_f32(img2, "img2", a.device)
    g = _dev_f32(dL_dmap, "dL_dmap", a.device)
    d1 = _dev_f32(dm_dmu1, "dm_dmu1", a.device)
    d2 = _dev_f32(dm_dsigma1_sq, "dm_dsigma1_sq", a.device)
    d3 = _dev_f32(dm_dsigma12, "dm_dsigma12", a.device)
    B, CH, H, W = a.shape
    out = torch.empty_like(a)         # written at every pixel
    check("ssim_backward", _lib.lib().gsparc_ssim_backward(
        B, CH, H, W, float(C1), float(C2), ptr(a), ptr(b), ptr(g), ptr(d1), ptr(d2), ptr(d3), ptr(out),
        stream_of(a.device)))
    return out
