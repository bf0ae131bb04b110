"""CPU oracle for the equirectangular RF splatting path (numpy, FP32 or FP64).

TEST INFRASTRUCTURE ONLY. Nothing in the product imports this module; only the
tests, ``__graft_entry__.smoke()`` and the ``cpu_baseline`` / ``--impl reference``
legs of ``bench.py`` may call it, and only as the checker or the timed CPU
restatement -- never as a fallback for the CUDA path.

Every function restates one piece of the reference rasterizer
(``cuda_kernel_rasterize/``) and cites the file:line it follows.  Arithmetic
is done in the dtype passed in (``np.float32`` reproduces the reference's
single-precision expression order operation by operation, without the fused
multiply-adds the GPU compiler forms; ``np.float64`` is the FP64 oracle).

Parity status: the reference ships no tests or golden vectors for the
rasterizer, so this restatement is pinned on the GPU against the reference
extension built from its own sources (``oracle/build_ref.py``, which supplies a
project-written stand-in for the absent GLM headers).  Where that build is not
available the rasterizer half of this oracle is "parity unpinned".

Conventions (all follow the reference):
  * ``view`` is the 4x4 world->receiver matrix stored transposed, read as a
    flat 16-vector exactly like ``transformPoint4x3`` (auxiliary.h:38-46).
  * ``mlp`` is the flat per-Gaussian emission MLP buffer in the layout of
    ``EmissionMLPs.get_all_params`` (gaussian.py:565-572):
    [W1 (P*32*3) | b1 (P*32) | W2 (P*2*32) | b2 (P*2)].
  * tiles are ``tile_h`` x ``tile_w`` pixels (reference: 16x16, config.h:15-17).
"""
from __future__ import annotations

import numpy as np

HID = 32          # emission MLP hidden width (forward.cu:25)
IN = 3            # emission MLP input = receiver position (forward.cu:24,29)
OUT = 2           # (real, imag) (forward.cu:26)
MLP_FLOATS = IN * HID + HID + OUT * HID + OUT   # 194 per Gaussian
LEAKY = 0.01      # forward.cu:27

M_1_PI32 = np.float32(1.0 / np.pi)
M_2_PI32 = np.float32(2.0 / np.pi)


def _c(dt, v):
    return dt.type(v)


def mlp_views(mlp, P):
    """Split the flat MLP buffer into (W1[P,32,3], b1[P,32], W2[P,2,32], b2[P,2]).

    Offsets follow forward.cu:36-44 / gaussian.py:565-572.
    """
    o1 = P * IN * HID
    o2 = o1 + P * HID
    o3 = o2 + P * OUT * HID
    W1 = mlp[:o1].reshape(P, HID, IN)
    b1 = mlp[o1:o2].reshape(P, HID)
    W2 = mlp[o2:o3].reshape(P, OUT, HID)
    b2 = mlp[o3:o3 + P * OUT].reshape(P, OUT)
    return W1, b1, W2, b2


def transform_point(p, m):
    """transformPoint4x3 (auxiliary.h:38-46)."""
    x = m[0] * p[:, 0] + m[4] * p[:, 1] + m[8] * p[:, 2] + m[12]
    y = m[1] * p[:, 0] + m[5] * p[:, 1] + m[9] * p[:, 2] + m[13]
    z = m[2] * p[:, 0] + m[6] * p[:, 1] + m[10] * p[:, 2] + m[14]
    return x, y, z


def cov3d(scales, rots, mod, dt):
    """computeCov3D (forward.cu:124-149): Sigma = (S R)^T (S R) in GLM's
    column-major convention.  Returns [P,6] = (S00,S01,S02,S11,S12,S22) and the
    intermediate R (GLM columns) for the backward."""
    s = _c(dt, mod) * scales.astype(dt)
    r, x, y, z = (rots[:, i].astype(dt) for i in range(4))
    one, two = _c(dt, 1), _c(dt, 2)
    # Rc[c][k]: GLM column c, row k (mat3 ctor takes columns, forward.cu:134-138)
    Rc = np.empty((rots.shape[0], 3, 3), dtype=dt)
    Rc[:, 0, 0] = one - two * (y * y + z * z)
    Rc[:, 0, 1] = two * (x * y - r * z)
    Rc[:, 0, 2] = two * (x * z + r * y)
    Rc[:, 1, 0] = two * (x * y + r * z)
    Rc[:, 1, 1] = one - two * (x * x + z * z)
    Rc[:, 1, 2] = two * (y * z - r * x)
    Rc[:, 2, 0] = two * (x * z - r * y)
    Rc[:, 2, 1] = two * (y * z + r * x)
    Rc[:, 2, 2] = one - two * (x * x + y * y)
    # M = S * R with S diagonal: M[c][k] = s_k * R[c][k]
    M = Rc * s[:, None, :]
    # Sigma[c][k] = sum_j M[k][j] * M[c][j]
    def sig(c, k):
        return M[:, k, 0] * M[:, c, 0] + M[:, k, 1] * M[:, c, 1] + M[:, k, 2] * M[:, c, 2]
    cov = np.stack([sig(0, 0), sig(0, 1), sig(0, 2), sig(1, 1), sig(1, 2), sig(2, 2)], axis=1)
    return cov, Rc, M, s


def _glm_mul(A, B):
    """GLM mat3 product on [P,3,3] arrays indexed [col][row]:
    (A*B)[c][r] = sum_k A[k][r] * B[c][k]."""
    out = np.empty_like(A)
    for c in range(3):
        for r_ in range(3):
            out[:, c, r_] = A[:, 0, r_] * B[:, c, 0] + A[:, 1, r_] * B[:, c, 1] + A[:, 2, r_] * B[:, c, 2]
    return out


def _glm_T(A):
    return np.swapaxes(A, 1, 2)


def _view_W(m, P, dt):
    """glm::mat3 W built from the view matrix (forward.cu:104-107)."""
    Wm = np.empty((P, 3, 3), dtype=dt)
    for c in range(3):
        for r_ in range(3):
            Wm[:, c, r_] = m[c + 4 * r_]
    return Wm


def jacobian(t, H, W, dt, x_scale=1.0):
    """Equirectangular projection Jacobian (forward.cu:82-97).  ``x_scale``
    multiplies the azimuth row: 1.0 in the forward, 0.5 reproduces
    backward.cu:172-173."""
    tx, ty, tz = t
    eps = _c(dt, 1e-7)
    trxztrxz = tx * tx + tz * tz
    trxztrxz_inv = _c(dt, 1) / (trxztrxz + eps)
    trxz = np.sqrt(trxztrxz)
    trxz_inv = _c(dt, 1) / (trxz + eps)
    trtr = trxztrxz + ty * ty
    trtr_inv = _c(dt, 1) / (trtr + eps)
    if dt == np.float32:
        W_div_2pi = np.float32(W) * np.float32(0.5) * M_1_PI32
        H_div_pi = np.float32(H) * M_1_PI32
    else:
        W_div_2pi = W * 0.5 / np.pi
        H_div_pi = H / np.pi
    xs = _c(dt, x_scale)
    J00 = W_div_2pi * tz * trxztrxz_inv
    J02 = -W_div_2pi * tx * trxztrxz_inv
    if x_scale != 1.0:
        J00 = J00 * xs
        J02 = J02 * xs
    J10 = -H_div_pi * tx * ty * trxz_inv * trtr_inv
    J11 = H_div_pi * trxz * trtr_inv
    J12 = -H_div_pi * tz * ty * trxz_inv * trtr_inv
    aux = dict(trxztrxz=trxztrxz, trxztrxz_inv=trxztrxz_inv, trxz=trxz, trxz_inv=trxz_inv,
               trtr=trtr, trtr_inv=trtr_inv, W_div_2pi=W_div_2pi, H_div_pi=H_div_pi)
    return (J00, J02, J10, J11, J12), aux


def _glm_J(Js, P, dt):
    J00, J02, J10, J11, J12 = Js
    J = np.zeros((P, 3, 3), dtype=dt)
    J[:, 0, 0] = J00
    J[:, 0, 2] = J02
    J[:, 1, 0] = J10
    J[:, 1, 1] = J11
    J[:, 1, 2] = J12
    return J


def _vrk(cov, dt):
    V = np.empty((cov.shape[0], 3, 3), dtype=dt)
    V[:, 0, 0] = cov[:, 0]; V[:, 0, 1] = cov[:, 1]; V[:, 0, 2] = cov[:, 2]
    V[:, 1, 0] = cov[:, 1]; V[:, 1, 1] = cov[:, 3]; V[:, 1, 2] = cov[:, 4]
    V[:, 2, 0] = cov[:, 2]; V[:, 2, 1] = cov[:, 4]; V[:, 2, 2] = cov[:, 5]
    return V


def get_rect(px, py, radius, grid_x, grid_y, tile_h, tile_w, dt):
    """getRect (auxiliary.h:14-24): clamp only, no azimuth wrap.  The float
    expression order matches the macro expansion ((p + r) + B) - 1."""
    rad = radius.astype(dt)
    bx, by = _c(dt, tile_w), _c(dt, tile_h)
    one = _c(dt, 1)
    with np.errstate(invalid="ignore"):
        x0 = np.trunc((px - rad) / bx)
        y0 = np.trunc((py - rad) / by)
        x1 = np.trunc(((px + rad) + bx - one) / bx)
        y1 = np.trunc(((py + rad) + by - one) / by)
    def clampi(v, hi):
        v = np.where(np.isfinite(v), v, 0.0)
        v = np.clip(v, -2 ** 31, 2 ** 31 - 1).astype(np.int64)
        return np.minimum(hi, np.maximum(0, v))
    return clampi(x0, grid_x), clampi(y0, grid_y), clampi(x1, grid_x), clampi(y1, grid_y)


def get_span(px, py, radius, grid_x, grid_y, tile_h, tile_w, W, dt, wrap):
    """Tile columns of a footprint: get_rect's clamped rectangle plus, with the
    azimuth seam wrap (this implementation's GSPARC_FLAG_WRAP_AZIMUTH; the
    reference has none), the columns beyond the left edge [xl, gx) and beyond
    the right edge [0, xr), with the rectangle's own rounding:
    xl = trunc(((px - r) + W) / bx), xr = trunc((((px + r) - W) + bx - 1) / bx),
    clamped so they never overlap [x0, x1)."""
    x0, y0, x1, y1 = get_rect(px, py, radius, grid_x, grid_y, tile_h, tile_w, dt)
    xl = np.full_like(x0, grid_x)
    xr = np.zeros_like(x0)
    if wrap:
        rad = radius.astype(dt)
        bx, Wf, one = _c(dt, tile_w), _c(dt, W), _c(dt, 1)
        with np.errstate(invalid="ignore"):
            left = (px - rad) < 0
            ql = np.trunc(((px - rad) + Wf) / bx)
            qr = (px + rad) - Wf
            right = qr > 0
            qrt = np.trunc(((qr + bx) - one) / bx)
        ql = np.clip(np.where(np.isfinite(ql), ql, 0.0), 0, grid_x).astype(np.int64)
        qrt = np.clip(np.where(np.isfinite(qrt), qrt, 0.0), 0, grid_x).astype(np.int64)
        xl = np.where(left, np.maximum(x1, ql), grid_x)
        xr = np.where(right, np.minimum(x0, qrt), 0)
    return x0, y0, x1, y1, xl, xr


def wrap_shift(x, tx, tile_w, W, dt):
    """With the seam wrap, the shift (-W, +W or 0) that moves a mean's x to its
    copy nearest tile column tx's centre (more than W/2 away: the other copy)."""
    half = _c(dt, 0.5) * _c(dt, W)
    cx = _c(dt, tx * tile_w) + _c(dt, 0.5) * _c(dt, tile_w)
    d = x - cx
    return np.where(d > half, -_c(dt, W), np.where(d < -half, _c(dt, W), _c(dt, 0)))


def preprocess(means, scales, rots, opac, mlp, view, tx, rx, H, W,
               mod=1.0, tile_h=16, tile_w=16, dtype=np.float32):
    """preprocessCUDA (forward.cu:252-327) for one receiver.

    Returns a dict with radii (int32), means2D [P,2], depth [P], conic_opacity
    [P,4], signal [P,2] (real, imag), cov3D [P,6], tiles_touched, rect."""
    dt = np.dtype(dtype)
    P = means.shape[0]
    m = view.reshape(16).astype(dt)
    p = means.astype(dt)
    out = {}
    with np.errstate(all="ignore"):
        x, y, z = transform_point(p, m)
        rr = x * x + y * y + z * z
        keep = rr > _c(dt, 0.04)                           # too_close, auxiliary.h:133-155
        r = np.sqrt(rr)
        inv_r = _c(dt, 1) / (r + _c(dt, 1e-7))             # transformProj, auxiliary.h:101-113
        lon = np.arctan2(x, z)
        lat = np.arcsin(y * inv_r)
        if dt == np.float32:
            ndc_x, ndc_y = lon * M_1_PI32, lat * M_2_PI32
        else:
            ndc_x, ndc_y = lon / np.pi, lat * 2.0 / np.pi
        cov, _, _, _ = cov3d(scales, rots, mod, dt)
        Js, _ = jacobian((x, y, z), H, W, dt)
        J = _glm_J(Js, P, dt)
        Wm = _view_W(m, P, dt)
        T = _glm_mul(Wm, J)                                  # forward.cu:109
        V = _vrk(cov, dt)
        C2 = _glm_mul(_glm_mul(_glm_T(T), _glm_T(V)), T)     # forward.cu:116
        ca = C2[:, 0, 0] + _c(dt, 0.3)
        cb = C2[:, 0, 1]
        cc = C2[:, 1, 1] + _c(dt, 0.3)
        det = ca * cc - cb * cb
        keep &= det != 0
        det_inv = _c(dt, 1) / det
        conic = np.stack([cc * det_inv, -cb * det_inv, ca * det_inv], axis=1)
        mid = _c(dt, 0.5) * (ca + cc)
        disc = np.maximum(_c(dt, 0.1), mid * mid - det)
        lam1 = mid + np.sqrt(disc)
        lam2 = mid - np.sqrt(disc)
        radius_f = np.ceil(_c(dt, 3) * np.sqrt(np.maximum(lam1, lam2)))
        # ndc2Pix is evaluated in double (auxiliary.h:10-13: 1.0 is a double literal)
        px = (((ndc_x.astype(np.float64) + 1.0) * W - 1.0) * 0.5).astype(dt)
        py = (((ndc_y.astype(np.float64) + 1.0) * H - 1.0) * 0.5).astype(dt)
        radius_i = np.where(np.isfinite(radius_f), radius_f, 0).clip(-2 ** 31, 2 ** 31 - 1).astype(np.int64)
        gx = (W + tile_w - 1) // tile_w
        gy = (H + tile_h - 1) // tile_h
        x0, y0, x1, y1 = get_rect(px, py, radius_i, gx, gy, tile_h, tile_w, dt)
        area = (x1 - x0) * (y1 - y0)
        keep &= area != 0
        sig = emission_forward(p, mlp, tx, rx, dt)
    radii = np.where(keep, radius_i, 0).astype(np.int32)
    out["radii"] = radii
    out["means2D"] = np.stack([px, py], axis=1)
    out["depth"] = r
    out["conic_opacity"] = np.concatenate([conic, opac.reshape(P, 1).astype(dt)], axis=1)
    out["signal"] = sig
    out["cov3D"] = cov
    out["tiles_touched"] = np.where(keep, area, 0).astype(np.int64)
    out["rect"] = (x0, y0, x1, y1)
    out["visible"] = keep
    out["view_xyz"] = (x, y, z)
    return out


def emission_forward(means, mlp, tx, rx, dt):
    """computeSignalFromMLP (forward.cu:17-75): h = leaky(b1 + W1 rx);
    o = sigmoid(b2 + W2 h - log(|tx - mean| + 1e-6)).  Sums start from the
    bias and accumulate inputs in index order, as the reference does."""
    P = means.shape[0]
    W1, b1, W2, b2 = (a.astype(dt) for a in mlp_views(mlp, P))
    inp = rx.astype(dt)
    diff = tx.astype(dt)[None, :] - means.astype(dt)
    d = np.sqrt(diff[:, 0] * diff[:, 0] + diff[:, 1] * diff[:, 1] + diff[:, 2] * diff[:, 2])
    log_d = np.log(d + _c(dt, 1e-6))
    pre = b1.copy()
    for j in range(IN):
        pre = pre + W1[:, :, j] * inp[j]
    h = np.where(pre > 0, pre, _c(dt, LEAKY) * pre)
    o = b2.copy()
    for j in range(HID):
        o = o + W2[:, :, j] * h[:, j:j + 1]
    att = o - log_d[:, None]
    return _c(dt, 1) / (_c(dt, 1) + np.exp(-att))


def bin_and_sort(means2D, depth, radii, H, W, tile_h=16, tile_w=16, wrap=False):
    """duplicateWithKeys + stable radix sort + identifyTileRanges
    (rasterizer_impl.cu:102-171, :270-310).

    Inputs are the FP32 preprocess outputs (means2D float32 [P,2], depth
    float32 [P], radii int32 [P]).  Returns (keys uint64 [K], values uint32 [K],
    ranges uint32 [tiles,2]).  The reference sorts with a stable LSD radix sort
    over (tile << 32 | depth bits); a stable sort on the same 64-bit key gives
    the identical order."""
    means2D = np.asarray(means2D, dtype=np.float32)
    depth = np.asarray(depth, dtype=np.float32)
    radii = np.asarray(radii, dtype=np.int32)
    gx = (W + tile_w - 1) // tile_w
    gy = (H + tile_h - 1) // tile_h
    ntiles = gx * gy
    P = radii.shape[0]
    x0, y0, x1, y1, xl, xr = get_span(means2D[:, 0], means2D[:, 1], radii.astype(np.int64), gx, gy,
                                      tile_h, tile_w, W, np.dtype(np.float32), wrap)
    dbits = depth.view(np.uint32).astype(np.uint64)
    keys, vals = [], []
    for g in np.nonzero(radii > 0)[0]:
        cols = list(range(x0[g], x1[g])) + list(range(xl[g], gx)) + list(range(0, xr[g]))
        for ty in range(y0[g], y1[g]):
            for tx in cols:
                keys.append((np.uint64(ty * gx + tx) << np.uint64(32)) | dbits[g])
                vals.append(g)
    keys = np.array(keys, dtype=np.uint64)
    vals = np.array(vals, dtype=np.uint32)
    order = np.argsort(keys, kind="stable")
    keys, vals = keys[order], vals[order]
    ranges = np.zeros((ntiles, 2), dtype=np.uint32)
    if keys.size:
        tiles = (keys >> np.uint64(32)).astype(np.int64)
        starts = np.searchsorted(tiles, np.arange(ntiles), side="left")
        ends = np.searchsorted(tiles, np.arange(ntiles), side="right")
        ranges[:, 0] = np.where(ends > starts, starts, 0)
        ranges[:, 1] = np.where(ends > starts, ends, 0)
    return keys, vals, ranges


def _tile_pixels(tile, gx, H, W, tile_h, tile_w):
    ty, tx = divmod(tile, gx)
    yy, xx = np.meshgrid(np.arange(ty * tile_h, ty * tile_h + tile_h),
                         np.arange(tx * tile_w, tx * tile_w + tile_w), indexing="ij")
    yy, xx = yy.reshape(-1), xx.reshape(-1)
    inside = (yy < H) & (xx < W)
    return yy[inside], xx[inside]


def blend_forward(ranges, point_list, means2D, conic_opacity, signal, H, W,
                  tile_h=16, tile_w=16, dtype=np.float32, record=False, wrap=False):
    """renderCUDA forward (forward.cu:151-249): per pixel, walk the tile's
    sorted list front to back; skip power>0 and alpha<1/255; stop before the
    first Gaussian that would take T below 1e-4.

    Returns out [2,H,W] (real, imag), final_T [H,W], n_contrib [H,W] (uint32).
    With ``record`` the per-pixel list of (list index, alpha, T-before) for
    contributing entries is also returned (used by the FP64 finite-difference
    oracle to freeze decisions)."""
    dt = np.dtype(dtype)
    gx = (W + tile_w - 1) // tile_w
    out = np.zeros((2, H, W), dtype=dt)
    final_T = np.ones((H, W), dtype=dt)
    n_contrib = np.zeros((H, W), dtype=np.uint32)
    xy = means2D.astype(dt)
    co = conic_opacity.astype(dt)
    sg = signal.astype(dt)
    thr = _c(dt, 1.0) / _c(dt, 255.0)
    rec = {} if record else None
    for tile in range(ranges.shape[0]):
        s, e = int(ranges[tile, 0]), int(ranges[tile, 1])
        yy, xx = _tile_pixels(tile, gx, H, W, tile_h, tile_w)
        if yy.size == 0:
            continue
        pxf, pyf = xx.astype(dt), yy.astype(dt)
        tcol = tile % gx
        T = np.ones(yy.size, dtype=dt)
        Cr = np.zeros(yy.size, dtype=dt)
        Ci = np.zeros(yy.size, dtype=dt)
        last = np.zeros(yy.size, dtype=np.int64)
        done = np.zeros(yy.size, dtype=bool)
        if record:
            trace = [[] for _ in range(yy.size)]
        with np.errstate(all="ignore"):
            for j in range(s, e):
                if done.all():
                    break
                g = int(point_list[j])
                xg = xy[g, 0] + wrap_shift(xy[g, 0], tcol, tile_w, W, dt) if wrap else xy[g, 0]
                dx = xg - pxf
                dy = xy[g, 1] - pyf
                c = co[g]
                power = _c(dt, -0.5) * (c[0] * dx * dx + c[2] * dy * dy) - c[1] * dx * dy
                alpha = np.minimum(_c(dt, 0.99), c[3] * np.exp(power))
                ok = (~done) & (power <= 0) & (alpha >= thr)
                test_T = T * (_c(dt, 1) - alpha)
                stop = ok & (test_T < _c(dt, 1e-4))
                done |= stop
                ok &= ~stop
                if record:
                    for k in np.nonzero(ok)[0]:
                        trace[k].append((j - s, g))
                w = alpha * T
                Cr = np.where(ok, Cr + sg[g, 0] * alpha * T, Cr)
                Ci = np.where(ok, Ci + sg[g, 1] * alpha * T, Ci)
                T = np.where(ok, test_T, T)
                last = np.where(ok, j - s + 1, last)
        out[0, yy, xx] = Cr
        out[1, yy, xx] = Ci
        final_T[yy, xx] = T
        n_contrib[yy, xx] = last
        if record:
            for k in range(yy.size):
                rec[(int(yy[k]), int(xx[k]))] = trace[k]
    if record:
        return out, final_T, n_contrib, rec
    return out, final_T, n_contrib


def blend_backward(ranges, point_list, means2D, conic_opacity, signal, final_T, n_contrib,
                   dL_dout, H, W, tile_h=16, tile_w=16, dtype=np.float32, ref_compat=True, wrap=False):
    """renderCUDA backward (backward.cu:442-616): reverse walk recomputing T
    from the saved final T by division.

    ``ref_compat`` reproduces the reference exactly: the imaginary signal is
    read from the real buffer (backward.cu:577) and only the real channel's
    gradient drives alpha (backward.cu:587-597).  With ``ref_compat=False`` both
    channels drive alpha and the 0.99 clamp blocks the gradient, i.e. the true
    derivative of the forward.

    Returns per-Gaussian (dL_dmeans2D [P,3], dL_dconic [P,4] with slots
    (x, y, -, w), dL_dopacity [P], dL_dsignal [P,2])."""
    dt = np.dtype(dtype)
    P = means2D.shape[0]
    gx = (W + tile_w - 1) // tile_w
    xy = means2D.astype(dt)
    co = conic_opacity.astype(dt)
    sg = signal.astype(dt)
    dmean = np.zeros((P, 3), dtype=dt)
    dconic = np.zeros((P, 4), dtype=dt)
    dopac = np.zeros(P, dtype=dt)
    dsig = np.zeros((P, 2), dtype=dt)
    thr = _c(dt, 1.0) / _c(dt, 255.0)
    hw, hh = _c(dt, 0.5 * W), _c(dt, 0.5 * H)
    one = _c(dt, 1)
    for tile in range(ranges.shape[0]):
        s, e = int(ranges[tile, 0]), int(ranges[tile, 1])
        yy, xx = _tile_pixels(tile, gx, H, W, tile_h, tile_w)
        if yy.size == 0 or e <= s:
            continue
        pxf, pyf = xx.astype(dt), yy.astype(dt)
        tcol = tile % gx
        T = final_T[yy, xx].astype(dt)
        last_c = n_contrib[yy, xx].astype(np.int64)
        gr = dL_dout[0, yy, xx].astype(dt)
        gi = dL_dout[1, yy, xx].astype(dt)
        acc_r = np.zeros(yy.size, dtype=dt)
        acc_i = np.zeros(yy.size, dtype=dt)
        last_a = np.zeros(yy.size, dtype=dt)
        last_sr = np.zeros(yy.size, dtype=dt)
        last_si = np.zeros(yy.size, dtype=dt)
        with np.errstate(all="ignore"):
            for j in range(e - 1, s - 1, -1):
                pos = j - s                      # contributor index after decrement
                act = pos < last_c
                if not act.any():
                    continue
                g = int(point_list[j])
                xg = xy[g, 0] + wrap_shift(xy[g, 0], tcol, tile_w, W, dt) if wrap else xy[g, 0]
                dx = xg - pxf
                dy = xy[g, 1] - pyf
                c = co[g]
                power = _c(dt, -0.5) * (c[0] * dx * dx + c[2] * dy * dy) - c[1] * dx * dy
                G = np.exp(power)
                a_raw = c[3] * G
                alpha = np.minimum(_c(dt, 0.99), a_raw)
                ok = act & (power <= 0) & (alpha >= thr)
                if not ok.any():
                    continue
                Tn = np.where(ok, T / (one - alpha), T)
                dch = alpha * Tn
                sr = sg[g, 0]
                si = sg[g, 0] if ref_compat else sg[g, 1]
                acc_r_n = last_a * last_sr + (one - last_a) * acc_r
                acc_i_n = last_a * last_si + (one - last_a) * acc_i
                dar = (sr - acc_r_n) * gr
                if ref_compat:
                    da = dar * Tn
                else:
                    dai = (si - acc_i_n) * gi
                    da = (dar + dai) * Tn
                    da = np.where(a_raw > _c(dt, 0.99), _c(dt, 0), da)
                dsig[g, 0] += np.sum(np.where(ok, dch * gr, 0), dtype=dt)
                dsig[g, 1] += np.sum(np.where(ok, dch * gi, 0), dtype=dt)
                dG = c[3] * da
                gdx = G * dx
                gdy = G * dy
                dGdx = -gdx * c[0] - gdy * c[1]
                dGdy = -gdy * c[2] - gdx * c[1]
                dmean[g, 0] += np.sum(np.where(ok, dG * dGdx * hw, 0), dtype=dt)
                dmean[g, 1] += np.sum(np.where(ok, dG * dGdy * hh, 0), dtype=dt)
                dconic[g, 0] += np.sum(np.where(ok, _c(dt, -0.5) * gdx * dx * dG, 0), dtype=dt)
                dconic[g, 1] += np.sum(np.where(ok, _c(dt, -0.5) * gdx * dy * dG, 0), dtype=dt)
                dconic[g, 3] += np.sum(np.where(ok, _c(dt, -0.5) * gdy * dy * dG, 0), dtype=dt)
                dopac[g] += np.sum(np.where(ok, G * da, 0), dtype=dt)
                acc_r = np.where(ok, acc_r_n, acc_r)
                acc_i = np.where(ok, acc_i_n, acc_i)
                last_sr = np.where(ok, sr, last_sr)
                last_si = np.where(ok, si, last_si)
                last_a = np.where(ok, alpha, last_a)
                T = Tn
    return dmean, dconic, dopac, dsig


def geometry_backward(means, scales, rots, view, radii, cov3D, dL_dmeans2D, dL_dconic,
                      H, W, mod=1.0, dtype=np.float32, ref_compat=True):
    """computeCov2DCUDA (backward.cu:124-303) + the 2D-mean part of
    preprocessCUDA (backward.cu:412-430) + computeCov3D backward
    (backward.cu:308-371).

    ``ref_compat`` reproduces the reference's halved azimuth Jacobian row in
    the backward (backward.cu:172-173); ``False`` uses the forward's Jacobian
    (forward.cu:92-93), i.e. the true derivative.

    Returns (dL_dmeans3D [P,3] geometry part, dL_dcov3D [P,6], dL_dscale [P,3],
    dL_drot [P,4]); rows with radii <= 0 are zero."""
    dt = np.dtype(dtype)
    P = means.shape[0]
    m = view.reshape(16).astype(dt)
    p = means.astype(dt)
    vis = radii > 0
    two = _c(dt, 2)
    with np.errstate(all="ignore"):
        tx, ty, tz = transform_point(p, m)
        Js, aux = jacobian((tx, ty, tz), H, W, dt, x_scale=0.5 if ref_compat else 1.0)
        J = _glm_J(Js, P, dt)
        Wm = _view_W(m, P, dt)
        V = _vrk(cov3D.astype(dt), dt)
        T = _glm_mul(Wm, J)
        C2 = _glm_mul(_glm_mul(_glm_T(T), _glm_T(V)), T)
        a = C2[:, 0, 0] + _c(dt, 0.3)
        b = C2[:, 0, 1]
        c = C2[:, 1, 1] + _c(dt, 0.3)
        gx_, gy_, gz_ = (dL_dconic[:, i].astype(dt) for i in (0, 1, 3))
        denom = a * c - b * b
        d2i = _c(dt, 1) / (denom * denom + _c(dt, 1e-7))
        nz = d2i != 0
        dL_da = np.where(nz, d2i * (-c * c * gx_ + two * b * c * gy_ + (denom - a * c) * gz_), 0)
        dL_dc = np.where(nz, d2i * (-a * a * gz_ + two * a * b * gy_ + (denom - a * c) * gx_), 0)
        dL_db = np.where(nz, d2i * two * (b * c * gx_ - (denom + two * b * b) * gy_ + a * b * gz_), 0)
        Tm = lambda i, j: T[:, i, j]
        Vm = lambda i, j: V[:, i, j]
        dcov = np.stack([
            Tm(0, 0) * Tm(0, 0) * dL_da + Tm(0, 0) * Tm(1, 0) * dL_db + Tm(1, 0) * Tm(1, 0) * dL_dc,
            two * Tm(0, 0) * Tm(0, 1) * dL_da + (Tm(0, 0) * Tm(1, 1) + Tm(0, 1) * Tm(1, 0)) * dL_db + two * Tm(1, 0) * Tm(1, 1) * dL_dc,
            two * Tm(0, 0) * Tm(0, 2) * dL_da + (Tm(0, 0) * Tm(1, 2) + Tm(0, 2) * Tm(1, 0)) * dL_db + two * Tm(1, 0) * Tm(1, 2) * dL_dc,
            Tm(0, 1) * Tm(0, 1) * dL_da + Tm(0, 1) * Tm(1, 1) * dL_db + Tm(1, 1) * Tm(1, 1) * dL_dc,
            two * Tm(0, 2) * Tm(0, 1) * dL_da + (Tm(0, 1) * Tm(1, 2) + Tm(0, 2) * Tm(1, 1)) * dL_db + two * Tm(1, 1) * Tm(1, 2) * dL_dc,
            Tm(0, 2) * Tm(0, 2) * dL_da + Tm(0, 2) * Tm(1, 2) * dL_db + Tm(1, 2) * Tm(1, 2) * dL_dc,
        ], axis=1)
        def rowdot(i, k):   # sum_j T[i][j] * V[k][j]
            return Tm(i, 0) * Vm(k, 0) + Tm(i, 1) * Vm(k, 1) + Tm(i, 2) * Vm(k, 2)
        dT00 = two * rowdot(0, 0) * dL_da + rowdot(1, 0) * dL_db
        dT01 = two * rowdot(0, 1) * dL_da + rowdot(1, 1) * dL_db
        dT02 = two * rowdot(0, 2) * dL_da + rowdot(1, 2) * dL_db
        dT10 = two * rowdot(1, 0) * dL_dc + rowdot(0, 0) * dL_db
        dT11 = two * rowdot(1, 1) * dL_dc + rowdot(0, 1) * dL_db
        dT12 = two * rowdot(1, 2) * dL_dc + rowdot(0, 2) * dL_db
        Wmm = lambda i, j: Wm[:, i, j]
        dJ00 = Wmm(0, 0) * dT00 + Wmm(0, 1) * dT01 + Wmm(0, 2) * dT02
        dJ02 = Wmm(2, 0) * dT00 + Wmm(2, 1) * dT01 + Wmm(2, 2) * dT02
        dJ10 = Wmm(0, 0) * dT10 + Wmm(0, 1) * dT11 + Wmm(0, 2) * dT12
        dJ11 = Wmm(1, 0) * dT10 + Wmm(1, 1) * dT11 + Wmm(1, 2) * dT12
        dJ12 = Wmm(2, 0) * dT10 + Wmm(2, 1) * dT11 + Wmm(2, 2) * dT12
        txtx, tyty, tztz = tx * tx, ty * ty, tz * tz
        txtytz = tx * ty * tz
        rho2, rho2_inv = aux["trxztrxz"], aux["trxztrxz_inv"]
        rho, rho_inv = aux["trxz"], aux["trxz_inv"]
        r2, r2_inv = aux["trtr"], aux["trtr_inv"]
        rho4_inv = rho2_inv * rho2_inv
        r4_inv = r2_inv * r2_inv
        rho_r4_inv = rho_inv * r4_inv
        rho3_r4_inv = rho2_inv * rho_r4_inv
        Hp, Wp = aux["H_div_pi"], aux["W_div_2pi"]
        t1 = Hp * (tyty - rho2) * rho_r4_inv
        t2 = Hp * txtytz * (r2 + two * rho2) * rho3_r4_inv
        t3 = Wp * (txtx - tztz) * rho4_inv
        t4 = Wp * two * tx * tz * rho4_inv
        t5 = Hp * ty * rho3_r4_inv
        dtx = -dJ00 * t4 + dJ02 * t3 + dJ10 * t5 * (two * txtx * rho2 - tztz * r2) + dJ11 * tx * t1 + dJ12 * t2
        dty = dJ10 * tx * t1 - dJ11 * Hp * two * rho * ty * r4_inv + dJ12 * tz * t1
        dtz = dJ00 * t3 + dJ02 * t4 + dJ10 * t2 + dJ11 * tz * t1 + dJ12 * t5 * (two * tztz * rho2 - txtx * r2)
        # screen-space mean part (backward.cu:413-430); dpx_dt/dpy_dt use the
        # same (possibly halved) Jacobian as stored by computeCov2DCUDA
        J00, J02, J10, J11, J12 = Js
        dpx = dL_dmeans2D[:, 0].astype(dt) * (_c(dt, 2) / _c(dt, W))
        dpy = dL_dmeans2D[:, 1].astype(dt) * (_c(dt, 2) / _c(dt, H))
        dtx2 = dpx * J00 + dpy * J10
        dty2 = dpx * _c(dt, 0) + dpy * J11
        dtz2 = dpx * J02 + dpy * J12
        def vT(vx, vy, vz):   # transformVec4x3Transpose (auxiliary.h:117-125)
            return np.stack([m[0] * vx + m[1] * vy + m[2] * vz,
                             m[4] * vx + m[5] * vy + m[6] * vz,
                             m[8] * vx + m[9] * vy + m[10] * vz], axis=1)
        dmean3 = vT(dtx, dty, dtz) + vT(dtx2, dty2, dtz2)
        dscale, drot = cov3d_backward(scales, rots, mod, dcov, dt, ref_compat)
    z = lambda a_: np.where(vis.reshape((-1,) + (1,) * (a_.ndim - 1)), a_, 0).astype(dt)
    return z(dmean3), z(dcov), z(dscale), z(drot)


def cov3d_backward(scales, rots, mod, dcov, dt, ref_compat=True):
    """computeCov3D backward (backward.cu:308-371).  The reference returns the
    gradient w.r.t. s = mod*scale; ``ref_compat=False`` multiplies by mod to
    give d/d(scale)."""
    _, Rc, M, s = cov3d(scales, rots, mod, dt)
    half = _c(dt, 0.5)
    dS = np.empty_like(M)
    dS[:, 0, 0] = dcov[:, 0]; dS[:, 0, 1] = half * dcov[:, 1]; dS[:, 0, 2] = half * dcov[:, 2]
    dS[:, 1, 0] = half * dcov[:, 1]; dS[:, 1, 1] = dcov[:, 3]; dS[:, 1, 2] = half * dcov[:, 4]
    dS[:, 2, 0] = half * dcov[:, 2]; dS[:, 2, 1] = half * dcov[:, 4]; dS[:, 2, 2] = dcov[:, 5]
    dM = _glm_mul(_c(dt, 2) * M, dS)
    Rt = _glm_T(Rc)
    dMt = _glm_T(dM).copy()
    dscale = np.stack([np.sum(Rt[:, i, :] * dMt[:, i, :], axis=1) for i in range(3)], axis=1)
    if not ref_compat:
        dscale = dscale * _c(dt, mod)
    dMt = dMt * s[:, :, None]
    r, x, y, z = (rots[:, i].astype(dt) for i in range(4))
    two, four = _c(dt, 2), _c(dt, 4)
    D = lambda i, j: dMt[:, i, j]
    dq = np.stack([
        two * z * (D(0, 1) - D(1, 0)) + two * y * (D(2, 0) - D(0, 2)) + two * x * (D(1, 2) - D(2, 1)),
        two * y * (D(1, 0) + D(0, 1)) + two * z * (D(2, 0) + D(0, 2)) + two * r * (D(1, 2) - D(2, 1)) - four * x * (D(2, 2) + D(1, 1)),
        two * x * (D(1, 0) + D(0, 1)) + two * r * (D(2, 0) - D(0, 2)) + two * z * (D(1, 2) + D(2, 1)) - four * y * (D(2, 2) + D(0, 0)),
        two * r * (D(0, 1) - D(1, 0)) + two * x * (D(2, 0) + D(0, 2)) + two * y * (D(1, 2) + D(2, 1)) - four * z * (D(1, 1) + D(0, 0)),
    ], axis=1)
    return dscale, dq


def emission_backward(means, mlp, tx, rx, radii, dsig, dtype=np.float32):
    """computeSignalFromMLP backward (backward.cu:9-118).

    Returns (dL_dmlp flat [194*P], dL_dmeans3D [P,3] from the log-distance
    term); rows with radii <= 0 are zero."""
    dt = np.dtype(dtype)
    P = means.shape[0]
    W1, b1, W2, b2 = (a.astype(dt) for a in mlp_views(mlp, P))
    inp = rx.astype(dt)
    diff = tx.astype(dt)[None, :] - means.astype(dt)
    with np.errstate(all="ignore"):
        d = np.sqrt(diff[:, 0] * diff[:, 0] + diff[:, 1] * diff[:, 1] + diff[:, 2] * diff[:, 2])
        log_d = np.log(d + _c(dt, 1e-6))
        unit = diff / (d + _c(dt, 1e-6))[:, None]
        pre = np.zeros((P, HID), dtype=dt)
        for j in range(IN):
            pre = pre + W1[:, :, j] * inp[j]
        pre = pre + b1
        h = np.where(pre > 0, pre, _c(dt, LEAKY) * pre)
        o = np.zeros((P, OUT), dtype=dt)
        for j in range(HID):
            o = o + W2[:, :, j] * h[:, j:j + 1]
        o = o + b2
        s = _c(dt, 1) / (_c(dt, 1) + np.exp(-(o - log_d[:, None])))
        dout = dsig.astype(dt) * s * (_c(dt, 1) - s)
        dlogd = -(dout[:, 0] + dout[:, 1])
        dd = dlogd / (d + _c(dt, 1e-6))
        dmean = -dd[:, None] * unit
        dW2 = dout[:, :, None] * h[:, None, :]
        db2 = dout
        dh = dout[:, 0:1] * W2[:, 0, :] + dout[:, 1:2] * W2[:, 1, :]
        dpre = np.where(pre > 0, dh, _c(dt, LEAKY) * dh)
        dW1 = dpre[:, :, None] * inp[None, None, :]
        db1 = dpre
    vis = radii > 0
    zero = lambda a_: np.where(vis.reshape((-1,) + (1,) * (a_.ndim - 1)), a_, 0).astype(dt)
    flat = np.concatenate([zero(dW1).reshape(-1), zero(db1).reshape(-1),
                           zero(dW2).reshape(-1), zero(db2).reshape(-1)])
    return flat, zero(dmean)


def mark_visible(means, view):
    """checkFrustum / in_frustum (rasterizer_impl.cu:173-185, auxiliary.h:75-99)."""
    m = view.reshape(16).astype(np.float32)
    x, y, z = transform_point(means.astype(np.float32), m)
    return (x * x + y * y + z * z) > np.float32(0.04)


def render(means, scales, rots, opac, mlp, view, tx, rx, H, W, mod=1.0,
           tile_h=16, tile_w=16, dtype=np.float32, signal_fn=None, wrap=False):
    """Whole forward for one receiver: preprocess -> bin/sort -> blend.
    ``signal_fn(radii) -> [P,2]`` replaces the per-Gaussian MLP's signals
    (the shared emission MLP); ``mlp`` may then be None.  ``wrap``: the
    azimuth seam wrap (get_span / wrap_shift)."""
    if mlp is None:
        mlp = np.zeros(194 * means.shape[0], np.float32)
    pre = preprocess(means, scales, rots, opac, mlp, view, tx, rx, H, W, mod, tile_h, tile_w, dtype)
    if signal_fn is not None:
        pre["signal"] = signal_fn(pre["radii"]).astype(pre["signal"].dtype)
    keys, vals, ranges = bin_and_sort(pre["means2D"].astype(np.float32), pre["depth"].astype(np.float32),
                                      pre["radii"], H, W, tile_h, tile_w, wrap)
    out, fT, nc = blend_forward(ranges, vals, pre["means2D"], pre["conic_opacity"], pre["signal"],
                                H, W, tile_h, tile_w, dtype, wrap=wrap)
    return dict(pre=pre, keys=keys, values=vals, ranges=ranges, out=out, final_T=fT, n_contrib=nc, wrap=wrap)


def render_backward(fwd, means, scales, rots, opac, mlp, view, tx, rx, dL_dout, H, W, mod=1.0,
                    tile_h=16, tile_w=16, dtype=np.float32, ref_compat=True):
    """Whole backward for one receiver; mirrors Rasterizer::backward
    (rasterizer_impl.cu:339-442).  Returns the seven tensors of
    rasterize_gaussians_backward (rasterize_points.cu:190-198) as a dict."""
    pre = fwd["pre"]
    dmean2, dconic, dopac, dsig = blend_backward(
        fwd["ranges"], fwd["values"], pre["means2D"], pre["conic_opacity"], pre["signal"],
        fwd["final_T"], fwd["n_contrib"], dL_dout, H, W, tile_h, tile_w, dtype, ref_compat,
        wrap=fwd.get("wrap", False))
    dmean3_geo, dcov, dscale, drot = geometry_backward(
        means, scales, rots, view, pre["radii"], pre["cov3D"], dmean2, dconic, H, W, mod, dtype, ref_compat)
    if mlp is None:   # shared emission MLP: its adjoint is the caller's (dL_dsignal)
        dmlp, dmean3_mlp = None, np.zeros_like(dmean3_geo)
    else:
        dmlp, dmean3_mlp = emission_backward(means, mlp, tx, rx, pre["radii"], dsig, dtype)
    return dict(dL_dmeans2D=dmean2, dL_dmeans3D=dmean3_geo + dmean3_mlp, dL_dmlp=dmlp,
                dL_dopacity=dopac.reshape(-1, 1), dL_dcov3D=dcov, dL_dscales=dscale,
                dL_drotations=drot, dL_dconic=dconic, dL_dsignal=dsig)


# ---- multi-channel blend (this implementation's C-channel extension; the
# reference renders one channel, NUM_CHANNELS 1 in config.h) ----------------
def blend_forward_channels(ranges, point_list, means2D, conic_opacity, features, H, W,
                           tile_h=16, tile_w=16, dtype=np.float32, wrap=False):
    """renderCUDA's front-to-back walk (forward.cu:151-249) with C amplitude
    channels per Gaussian (features [P,C]): the same skip / termination
    decisions as blend_forward, and out[c] += features[g,c] * (alpha * T).

    Returns out [C,H,W], final_T [H,W], n_contrib [H,W] (uint32)."""
    dt = np.dtype(dtype)
    gx = (W + tile_w - 1) // tile_w
    C = features.shape[1]
    out = np.zeros((C, H, W), dtype=dt)
    final_T = np.ones((H, W), dtype=dt)
    n_contrib = np.zeros((H, W), dtype=np.uint32)
    xy = means2D.astype(dt)
    co = conic_opacity.astype(dt)
    ft = features.astype(dt)
    thr = _c(dt, 1.0) / _c(dt, 255.0)
    for tile in range(ranges.shape[0]):
        s, e = int(ranges[tile, 0]), int(ranges[tile, 1])
        yy, xx = _tile_pixels(tile, gx, H, W, tile_h, tile_w)
        if yy.size == 0:
            continue
        pxf, pyf = xx.astype(dt), yy.astype(dt)
        tcol = tile % gx
        T = np.ones(yy.size, dtype=dt)
        acc = np.zeros((C, yy.size), dtype=dt)
        last = np.zeros(yy.size, dtype=np.int64)
        done = np.zeros(yy.size, dtype=bool)
        with np.errstate(all="ignore"):
            for j in range(s, e):
                if done.all():
                    break
                g = int(point_list[j])
                xg = xy[g, 0] + wrap_shift(xy[g, 0], tcol, tile_w, W, dt) if wrap else xy[g, 0]
                dx = xg - pxf
                dy = xy[g, 1] - pyf
                c = co[g]
                power = _c(dt, -0.5) * (c[0] * dx * dx + c[2] * dy * dy) - c[1] * dx * dy
                alpha = np.minimum(_c(dt, 0.99), c[3] * np.exp(power))
                ok = (~done) & (power <= 0) & (alpha >= thr)
                test_T = T * (_c(dt, 1) - alpha)
                stop = ok & (test_T < _c(dt, 1e-4))
                done |= stop
                ok &= ~stop
                w = alpha * T
                acc = np.where(ok[None], acc + ft[g][:, None] * w[None], acc)
                T = np.where(ok, test_T, T)
                last = np.where(ok, j - s + 1, last)
        out[:, yy, xx] = acc
        final_T[yy, xx] = T
        n_contrib[yy, xx] = last
    return out, final_T, n_contrib


def blend_backward_channels(ranges, point_list, means2D, conic_opacity, features, final_T, n_contrib,
                            dL_dout, H, W, tile_h=16, tile_w=16, dtype=np.float32, wrap=False):
    """Adjoint of blend_forward_channels (the true derivative: the 0.99 alpha
    clamp blocks the gradient).  Back to front from each pixel's contributor
    count, recomputing T by division from the saved final T.  The colour
    behind entry j, sum_{k>j} f_k alpha_k T_k / T_{j+1}, enters only through
    its dot product with dL/dout, so one scalar per pixel carries it:
    B += alpha_j T_j (f_j . g), and dL/dalpha_j = T_j (f_j . g - B / T_{j+1}).

    dL_dout [C,H,W].  Returns (dL_dmeans2D [P,3], dL_dconic [P,4] (slots x, y,
    -, w), dL_dopacity [P], dL_dfeatures [P,C])."""
    dt = np.dtype(dtype)
    P, C = features.shape
    gx = (W + tile_w - 1) // tile_w
    xy = means2D.astype(dt)
    co = conic_opacity.astype(dt)
    ft = features.astype(dt)
    dmean = np.zeros((P, 3), dtype=dt)
    dconic = np.zeros((P, 4), dtype=dt)
    dopac = np.zeros(P, dtype=dt)
    dfeat = np.zeros((P, C), dtype=dt)
    thr = _c(dt, 1.0) / _c(dt, 255.0)
    hw, hh = _c(dt, 0.5 * W), _c(dt, 0.5 * H)
    one = _c(dt, 1)
    for tile in range(ranges.shape[0]):
        s, e = int(ranges[tile, 0]), int(ranges[tile, 1])
        yy, xx = _tile_pixels(tile, gx, H, W, tile_h, tile_w)
        if yy.size == 0 or e <= s:
            continue
        pxf, pyf = xx.astype(dt), yy.astype(dt)
        tcol = tile % gx
        T = final_T[yy, xx].astype(dt)
        last_c = n_contrib[yy, xx].astype(np.int64)
        g = dL_dout[:, yy, xx].astype(dt)            # [C, px]
        B = np.zeros(yy.size, dtype=dt)
        with np.errstate(all="ignore"):
            for j in range(e - 1, s - 1, -1):
                pos = j - s
                act = pos < last_c
                if not act.any():
                    continue
                gi = int(point_list[j])
                xg = xy[gi, 0] + wrap_shift(xy[gi, 0], tcol, tile_w, W, dt) if wrap else xy[gi, 0]
                dx = xg - pxf
                dy = xy[gi, 1] - pyf
                c = co[gi]
                power = _c(dt, -0.5) * (c[0] * dx * dx + c[2] * dy * dy) - c[1] * dx * dy
                G = np.exp(power)
                a_raw = c[3] * G
                alpha = np.minimum(_c(dt, 0.99), a_raw)
                ok = act & (power <= 0) & (alpha >= thr)
                if not ok.any():
                    continue
                Tn = np.where(ok, T / (one - alpha), T)
                fg = (ft[gi][:, None] * g).sum(0, dtype=dt)
                da = (fg - B / T) * Tn
                da = np.where(a_raw > _c(dt, 0.99), _c(dt, 0), da)
                w = np.where(ok, alpha * Tn, _c(dt, 0))
                dfeat[gi] += (g * w[None]).sum(1, dtype=dt)
                dG = c[3] * da
                gdx = G * dx
                gdy = G * dy
                dGdx = -gdx * c[0] - gdy * c[1]
                dGdy = -gdy * c[2] - gdx * c[1]
                dmean[gi, 0] += np.sum(np.where(ok, dG * dGdx * hw, 0), dtype=dt)
                dmean[gi, 1] += np.sum(np.where(ok, dG * dGdy * hh, 0), dtype=dt)
                dconic[gi, 0] += np.sum(np.where(ok, _c(dt, -0.5) * gdx * dx * dG, 0), dtype=dt)
                dconic[gi, 1] += np.sum(np.where(ok, _c(dt, -0.5) * gdx * dy * dG, 0), dtype=dt)
                dconic[gi, 3] += np.sum(np.where(ok, _c(dt, -0.5) * gdy * dy * dG, 0), dtype=dt)
                dopac[gi] += np.sum(np.where(ok, G * da, 0), dtype=dt)
                B = np.where(ok, B + w * fg, B)
                T = Tn
    return dmean, dconic, dopac, dfeat
