"""CPU PyTorch rendition of the GSpaRC training step (multi-threaded torch on
the host cores).

CPU-BASELINE INFRASTRUCTURE ONLY: timed by bench.py's ``cpu_baseline`` leg and
its ``--impl reference`` arm as the CPU implementation of the path; never used
by the product, and not the checker (the numpy restatements next to it are).

The same step as train.py:364-566 with the benchmark's shared emission MLP,
written the way a PyTorch user would vectorise it on the CPU:

  * preprocess (forward.cu:252-327, auxiliary.h:10-155): receiver-frame
    transform, equirectangular projection, cov3D = (S R)^T (S R), the 2D
    covariance through the projection Jacobian + 0.3 I, conic, radius
    ceil(3 sqrt(lambda_max)), tile rectangle (getRect, auxiliary.h:14-24),
    culling r^2 <= 0.04;
  * the shared emission MLP on [position encoding, receiver-relative
    direction, 1/d^2] -> sigmoid amplitude;
  * the blend of renderCUDA (forward.cu:151-249) as (pixel, Gaussian) pairs:
    each visible Gaussian is paired with the pixels of its tile rectangle
    where its alpha can reach 1/255 (the ellipse's bounding box), pairs are
    put in (pixel, depth, id) order by one stable sort, alpha =
    min(0.99, o exp(power)) with the power > 0 and alpha < 1/255 skips,
    transmittance as an exclusive segmented cumulative product per pixel
    (log space, float64 prefix sums), the T * (1 - alpha) < 1e-4 stop as a
    prefix mask, and colour = sum alpha T signal per pixel;
  * L1 + (1 - SSIM) with SSIM as conv2d with the 11x11 Gaussian window,
    sigma 1.5 (utils.py:81-124), confidence weighting C recon - 0.3 log C
    with C = 1 + exp(ConfidenceMLP(rx)) (gaussian.py:575-609, train.py:420-436);
  * torch autograd for the whole adjoint (the true derivative; the reference
    extension's halved azimuth Jacobian row is not reproduced), the NaN/Inf
    zeroing of the centre gradient (train.py:443-445), torch.optim.Adam with
    the reference's per-group learning rates and eps 1e-15, and the centre
    clamp to the scene box (train.py:556-562).

Decisions (which pairs contribute) equal the reference's up to FP32 rounding;
colour sums run in a different order.  ``torch.set_num_threads`` is left to
the caller.
"""
from __future__ import annotations

import math

import torch
import torch.nn.functional as F

LR = dict(centre=0.00016, log_scale=0.005, rotation=0.001, opacity_logit=0.0055, mlp=0.002, conf=0.001)
LAMBDA1, CONF_ALPHA = 0.2, 0.3
C1, C2 = 0.01 ** 2, 0.03 ** 2


def _window(dtype=torch.float32):
    """11x11 Gaussian window, sigma 1.5 (utils.py:116-124)."""
    g = torch.tensor([math.exp(-(x - 5) ** 2 / (2 * 1.5 ** 2)) for x in range(11)], dtype=torch.float64)
    g = g / g.sum()
    return (g[:, None] @ g[None, :]).to(dtype)[None, None]


def ssim(img1, img2, win):
    """Mean SSIM of two [1,1,H,W] maps, "same" padding (utils.py:94-114)."""
    mu1 = F.conv2d(img1, win, padding=5)
    mu2 = F.conv2d(img2, win, padding=5)
    mu1_sq, mu2_sq, mu12 = mu1 * mu1, mu2 * mu2, mu1 * mu2
    s1 = F.conv2d(img1 * img1, win, padding=5) - mu1_sq
    s2 = F.conv2d(img2 * img2, win, padding=5) - mu2_sq
    s12 = F.conv2d(img1 * img2, win, padding=5) - mu12
    m = ((2 * mu12 + C1) * (2 * s12 + C2)) / ((mu1_sq + mu2_sq + C1) * (s1 + s2 + C2))
    return m.mean()


def features(means, rx, vis):
    """Input of the shared emission MLP: centre, sin/cos(2^k pi mu_j) for
    k = 0..3, (mu - rx)/d, 1/d^2, 0; zero rows for culled Gaussians."""
    v = means - rx[None, :]
    d2 = (v * v).sum(1, keepdim=True)
    d = d2.sqrt()
    pe = []
    for k in range(4):
        w = (2 ** k) * math.pi
        for j in range(3):
            pe += [torch.sin(w * means[:, j]), torch.cos(w * means[:, j])]
    x = torch.cat([means, torch.stack(pe, 1), v / d, 1.0 / d2, torch.zeros_like(d)], 1)
    return torch.where(vis[:, None], x, torch.zeros_like(x))


def shared_mlp(params, layers, width, act, x):
    """Hidden layers act(W h + b) (ReLU or erf-GELU), then sigmoid of the one
    output; params flat, per layer W [out, in] then b [out]."""
    dims = [32] + [width] * layers + [1]
    off, h = 0, x
    for i in range(len(dims) - 1):
        o, n = dims[i + 1], dims[i]
        w = params[off:off + o * n].view(o, n)
        off += o * n
        b = params[off:off + o]
        off += o
        h = h @ w.T + b
        if i + 1 < len(dims) - 1:
            h = F.relu(h) if act == "relu" else F.gelu(h)
    return torch.sigmoid(h[:, 0])


def preprocess(means, scales, rots, view, H, W, tile=16):
    """preprocessCUDA's geometry for one receiver (forward.cu:252-327).
    Returns px, py, depth, (a, b, c) conic, radius (int64), tile rectangle
    (x0, y0, x1, y1) and the visibility mask."""
    m = view.reshape(16)
    x = m[0] * means[:, 0] + m[4] * means[:, 1] + m[8] * means[:, 2] + m[12]
    y = m[1] * means[:, 0] + m[5] * means[:, 1] + m[9] * means[:, 2] + m[13]
    z = m[2] * means[:, 0] + m[6] * means[:, 1] + m[10] * means[:, 2] + m[14]
    rr = x * x + y * y + z * z
    vis = rr > 0.04
    r = rr.sqrt()
    lon = torch.atan2(x, z)
    lat = torch.asin((y / (r + 1e-7)).clamp(-1.0, 1.0))
    px = ((lon / math.pi + 1.0) * W - 1.0) * 0.5
    py = ((2.0 * lat / math.pi + 1.0) * H - 1.0) * 0.5
    # rotation of the normalised quaternion (w, x, y, z), Sigma = R diag(s^2) R^T
    qw, qx, qy, qz = rots.unbind(1)
    R = torch.stack([
        torch.stack([1 - 2 * (qy * qy + qz * qz), 2 * (qx * qy - qw * qz), 2 * (qx * qz + qw * qy)], 1),
        torch.stack([2 * (qx * qy + qw * qz), 1 - 2 * (qx * qx + qz * qz), 2 * (qy * qz - qw * qx)], 1),
        torch.stack([2 * (qx * qz - qw * qy), 2 * (qy * qz + qw * qx), 1 - 2 * (qx * qx + qy * qy)], 1)], 1)
    Sig = (R * (scales * scales)[:, None, :]) @ R.transpose(1, 2)
    # projection Jacobian (forward.cu:82-97) in the receiver frame, composed with the view rotation
    eps = 1e-7
    trxz2 = x * x + z * z
    trxz = trxz2.sqrt()
    trtr = trxz2 + y * y
    w2pi, hpi = W * 0.5 / math.pi, H / math.pi
    zero = torch.zeros_like(x)
    J = torch.stack([torch.stack([w2pi * z / (trxz2 + eps), zero, -w2pi * x / (trxz2 + eps)], 1),
                     torch.stack([-hpi * x * y / (trxz + eps) / (trtr + eps), hpi * trxz / (trtr + eps),
                                  -hpi * z * y / (trxz + eps) / (trtr + eps)], 1)], 1)
    Wr = torch.stack([torch.stack([m[0], m[4], m[8]]), torch.stack([m[1], m[5], m[9]]),
                      torch.stack([m[2], m[6], m[10]])])
    T = J @ Wr
    C2d = T @ Sig @ T.transpose(1, 2)
    a = C2d[:, 0, 0] + 0.3
    b = C2d[:, 0, 1]
    c = C2d[:, 1, 1] + 0.3
    det = a * c - b * b
    vis = vis & (det != 0)
    det = torch.where(det != 0, det, torch.ones_like(det))
    conic = (c / det, -b / det, a / det)
    with torch.no_grad():
        mid = 0.5 * (a + c)
        disc = torch.clamp(mid * mid - det, min=0.1)
        lam = torch.maximum(mid + disc.sqrt(), mid - disc.sqrt())
        radius = torch.ceil(3.0 * lam.sqrt()).nan_to_num(0.0).to(torch.int64)
        gx, gy = (W + tile - 1) // tile, (H + tile - 1) // tile
        rf = radius.to(px.dtype)
        x0 = torch.trunc((px - rf) / tile).nan_to_num(0.0).to(torch.int64).clamp(0, gx)
        y0 = torch.trunc((py - rf) / tile).nan_to_num(0.0).to(torch.int64).clamp(0, gy)
        x1 = torch.trunc((px + rf + tile - 1) / tile).nan_to_num(0.0).to(torch.int64).clamp(0, gx)
        y1 = torch.trunc((py + rf + tile - 1) / tile).nan_to_num(0.0).to(torch.int64).clamp(0, gy)
        vis = vis & ((x1 - x0) * (y1 - y0) != 0)
    return px, py, r, conic, radius, (x0, y0, x1, y1), vis


def blend(px, py, depth, conic, opac, signal, rect, vis, H, W, tile=16):
    """renderCUDA's forward (forward.cu:151-249) over (pixel, Gaussian) pairs;
    differentiable in px, py, conic, opacity and signal.  Which pairs
    contribute is decided without autograd over all candidate pairs; the
    colour is then recomputed with autograd over the contributing pairs only
    (a skipped pair leaves T unchanged and every pair after a pixel's stop is
    dropped, so T before a contributing pair is the product over the
    contributing pairs in front of it).  Returns the [H, W] spectrum and the
    number of contributing pairs."""
    ca, cb, cc = conic
    with torch.no_grad():
        idx = vis.nonzero()[:, 0]
        # depth order (ties by id), as the reference's stable sort on depth bits within a tile
        order = torch.argsort(depth[idx], stable=True)
        idx = idx[order]
        attr = torch.stack([px, py, ca, cb, cc, opac], 1)[idx]
        gxp, gyp, a, b, c, o = attr.unbind(1)
        # the ellipse alpha >= 1/255 covers: a dx^2 + 2 b dx dy + c dy^2 <= 2 ln(255 o)
        tau = (2.0 * torch.log(255.0 * o)).clamp(min=0.0)
        dc = a * c - b * b
        ok = (dc > 0) & (tau > 0)
        hx = torch.where(ok, (tau * c / dc.clamp(min=1e-30)).sqrt(), torch.zeros_like(a)) + 1.0
        hy = torch.where(ok, (tau * a / dc.clamp(min=1e-30)).sqrt(), torch.zeros_like(a)) + 1.0
        x0, y0, x1, y1 = (t[idx] for t in rect)
        xlo = torch.maximum(x0 * tile, torch.ceil(gxp - hx).to(torch.int64)).clamp(0, W - 1)
        xhi = torch.minimum(x1 * tile - 1, torch.floor(gxp + hx).to(torch.int64)).clamp(max=W - 1)
        ylo = torch.maximum(y0 * tile, torch.ceil(gyp - hy).to(torch.int64)).clamp(0, H - 1)
        yhi = torch.minimum(y1 * tile - 1, torch.floor(gyp + hy).to(torch.int64)).clamp(max=H - 1)
        nx = (xhi - xlo + 1).clamp(min=0) * ok
        ny = (yhi - ylo + 1).clamp(min=0) * ok
        cnt = nx * ny
        g = torch.repeat_interleave(torch.arange(idx.numel(), dtype=torch.int32), cnt)
        start = torch.cumsum(cnt, 0) - cnt
        loc = torch.arange(g.numel()) - start[g]
        nxg = nx[g]
        pix = (ylo[g] + loc // nxg) * W + xlo[g] + loc % nxg
        del loc, nxg, start
        srt = torch.argsort(pix.to(torch.int32), stable=True)   # (pixel, depth, id) order
        g, pix = g[srt], pix[srt]
        del srt
        ga = attr[g]
        dx = ga[:, 0] - (pix % W).to(ga.dtype)
        dy = ga[:, 1] - (pix // W).to(ga.dtype)
        power = -0.5 * (ga[:, 2] * dx * dx + ga[:, 4] * dy * dy) - ga[:, 3] * dx * dy
        alpha = torch.clamp(ga[:, 5] * torch.exp(power), max=0.99)
        keep = ((power <= 0) & (alpha >= 1.0 / 255.0)).nonzero()[:, 0]
        g, pix, alpha = g[keep], pix[keep], alpha[keep]
        del ga, dx, dy, power, keep
        # exclusive transmittance per pixel from prefix sums of log(1 - alpha) (float64)
        l = torch.log1p(-alpha).double()
        cs = torch.cumsum(l, 0)
        first = torch.ones_like(pix, dtype=torch.bool)
        first[1:] = pix[1:] != pix[:-1]
        seg = torch.cumsum(first.to(torch.int64), 0) - 1
        base = (cs - l)[first][seg]
        T_incl = torch.exp(cs - base).float()
        ci = (T_incl >= 1e-4).nonzero()[:, 0]            # the stop is a prefix: T only falls
        gid, pix = idx[g[ci].long()], pix[ci]
        del l, cs, first, seg, base, T_incl, g, alpha
        first = torch.ones_like(pix, dtype=torch.bool)
        first[1:] = pix[1:] != pix[:-1]
        seg = torch.cumsum(first.to(torch.int64), 0) - 1
        heads = first.nonzero()[:, 0]
        pxf = (pix % W).to(px.dtype)
        pyf = (pix // W).to(py.dtype)
    # with autograd, over the contributing pairs only
    dx = px[gid] - pxf
    dy = py[gid] - pyf
    power = -0.5 * (ca[gid] * dx * dx + cc[gid] * dy * dy) - cb[gid] * dx * dy
    alpha = torch.clamp(opac[gid] * torch.exp(power), max=0.99)
    lg = torch.log1p(-alpha).double()
    cs = torch.cumsum(lg, 0)
    excl = cs - lg
    T_excl = torch.exp(excl - excl[heads][seg]).float()
    w = alpha * T_excl * signal[gid]
    out = torch.zeros(H * W, dtype=w.dtype).index_add(0, pix, w)
    return out.view(H, W), int(gid.numel())


class TorchCPUTrainer:
    """Per-receiver training step on the CPU in PyTorch (fp32)."""

    def __init__(self, scene, layers, width, act, mlp_params, H=90, W=360, seed=0, room=None):
        self.H, self.W = H, W
        self.layers, self.width, self.act = layers, width, act
        t = lambda a: torch.tensor(a, dtype=torch.float32)
        self.centre = torch.nn.Parameter(t(scene.means))
        self.log_scale = torch.nn.Parameter(t(scene.log_scales))
        self.rotation = torch.nn.Parameter(t(scene.quats))
        self.opacity_logit = torch.nn.Parameter(t(scene.opacity_logits).reshape(-1))
        self.mlp = torch.nn.Parameter(t(mlp_params))
        g = torch.Generator().manual_seed(seed)
        lim1, lim2 = math.sqrt(6.0 / 35), math.sqrt(6.0 / 33)
        self.conf = [torch.nn.Parameter((torch.rand((32, 3), generator=g) * 2 - 1) * lim1),
                     torch.nn.Parameter(torch.zeros(32)),
                     torch.nn.Parameter((torch.rand((1, 32), generator=g) * 2 - 1) * lim2),
                     torch.nn.Parameter(torch.zeros(1))]
        self.opt = torch.optim.Adam(
            [{"params": [self.centre], "lr": LR["centre"]}, {"params": [self.log_scale], "lr": LR["log_scale"]},
             {"params": [self.rotation], "lr": LR["rotation"]},
             {"params": [self.opacity_logit], "lr": LR["opacity_logit"]},
             {"params": [self.mlp], "lr": LR["mlp"]}, {"params": self.conf, "lr": LR["conf"]}], eps=1e-15)
        self.room = room
        self.win = _window()
        self.last_pairs = 0

    def render(self, view, rx):
        scales = torch.exp(self.log_scale)
        rots = F.normalize(self.rotation, dim=1)
        opac = torch.sigmoid(self.opacity_logit)
        px, py, depth, conic, radius, rect, vis = preprocess(self.centre, scales, rots, view, self.H, self.W)
        sig = shared_mlp(self.mlp, self.layers, self.width, self.act, features(self.centre, rx, vis))
        out, n = blend(px, py, depth.detach(), conic, opac, sig, rect, vis, self.H, self.W)
        self.last_pairs = n
        return out

    def step(self, view, rx, target):
        """One training step for one receiver; returns the loss."""
        view = torch.as_tensor(view, dtype=torch.float32)
        rx = torch.as_tensor(rx, dtype=torch.float32)
        target = torch.as_tensor(target, dtype=torch.float32)
        self.opt.zero_grad(set_to_none=True)
        pred = self.render(view, rx)
        l1 = (pred - target).abs().mean()
        s = ssim(pred[None, None], target[None, None], self.win)
        recon = (1 - LAMBDA1) * l1 + LAMBDA1 * (1 - s)
        w1, b1, w2, b2 = self.conf
        C = 1.0 + torch.exp(F.relu(rx @ w1.T + b1) @ w2.T + b2)[0]
        loss = C * recon - CONF_ALPHA * torch.log(C)
        loss.backward()
        with torch.no_grad():
            gc = self.centre.grad
            if gc is not None:
                gc[~torch.isfinite(gc)] = 0.0
        self.opt.step()
        if self.room is not None:
            with torch.no_grad():
                self.centre.data.clamp_(min=self.room[0], max=self.room[1])
        return float(loss.detach())
