"""The training loss of one step and its adjoint, over the C ABI.

Per receiver (train.py:420-436):

    l1      = l1_loss(pred, target)                       (utils.py:40-41)
    ssim    = fused_ssim(pred, target)                    ("same" padding)
    recon   = (1 - lambda1) * l1 + lambda1 * (1 - ssim)
    conf    = ConfidenceMLP(rx_pos) = 1 + exp(fc2(relu(fc1(rx_pos))))
    loss    = conf * recon - alpha * log(conf)

and for a batch of R receivers the mean of the per-receiver losses.
``gsparc_splat_loss`` evaluates all of it and its gradients with respect to
the rendered spectra and the confidence-MLP parameters in two launches,
replacing the ~45 small torch kernels of the autograd formulation.
"""
from __future__ import annotations

import torch

from . import _lib
from ._lib import check, ptr, stream_of

LAMBDA1 = 0.2            # optimizer.py:8
CONFIDENCE_ALPHA = 0.3   # optimizer.py:33
C1, C2 = 0.01 ** 2, 0.03 ** 2


def conf_floats(hidden: int) -> int:
    """Parameters of ConfidenceMLP(hidden): fc1 (3 -> hidden) and fc2 (hidden -> 1)."""
    return 5 * int(hidden) + 1


class SplatLoss:
    """Static scratch and outputs for R spectra of H x W; call it with device
    tensors pred/target [R,H,W], rx_pos [R,3] and the confidence MLP's flat
    parameters (nn.Module order).  Writes the loss (1 float), per-receiver
    terms [R,4] = (l1, ssim, conf, loss_r), dL/dpred [R,H,W] and dL/dparams
    (into ``dconf``, overwritten)."""

    def __init__(self, R, H, W, hidden=32, device="cuda", lambda1=LAMBDA1, alpha=CONFIDENCE_ALPHA):
        self.R, self.H, self.W, self.hidden = int(R), int(H), int(W), int(hidden)
        self.lambda1, self.alpha = float(lambda1), float(alpha)
        dev = torch.device(device)
        n = int(_lib.lib().gsparc_splat_loss_scratch_floats(self.R, self.H, self.W, self.hidden))
        self.scratch = torch.zeros(max(n, 1), dtype=torch.float32, device=dev)   # zero once: arrival counter
        self.loss = torch.zeros((), dtype=torch.float32, device=dev)
        self.terms = torch.zeros((self.R, 4), dtype=torch.float32, device=dev)
        self.dpred = torch.empty((self.R, self.H, self.W), dtype=torch.float32, device=dev)

    def __call__(self, pred, target, rx_pos, conf_params, dconf, with_terms=True):
        for name, t, shape in (("pred", pred, (self.R, self.H, self.W)), ("target", target, (self.R, self.H, self.W)),
                               ("rx_pos", rx_pos, (self.R, 3))):
            if t.dtype != torch.float32 or not t.is_cuda or not t.is_contiguous() or t.numel() != _numel(shape):
                raise ValueError(f"{name} must be a contiguous float32 CUDA tensor of shape {shape}")
        nc = conf_floats(self.hidden)
        for name, t in (("conf_params", conf_params), ("dconf", dconf)):
            if t.dtype != torch.float32 or not t.is_cuda or not t.is_contiguous() or t.numel() != nc:
                raise ValueError(f"{name} must be a contiguous float32 CUDA tensor of {nc} floats")
        check("splat_loss", _lib.lib().gsparc_splat_loss(
            self.R, self.H, self.W, self.hidden, self.lambda1, self.alpha, C1, C2, ptr(pred), ptr(target),
            ptr(rx_pos), ptr(conf_params), ptr(self.scratch), ptr(self.loss),
            ptr(self.terms) if with_terms else None, ptr(self.dpred), ptr(dconf), stream_of(pred.device)))
        return self.loss, self.dpred


METRICS = ("psnr", "rssi_diff", "mae", "ssim", "confidence", "loss")


class Evaluator:
    """Batched evaluation of R test spectra (train.py:672-701): per spectrum
    the PSNR (train.py:76-83), the RSSI difference rssi(pred) - rssi(target)
    (train.py:86-91), the MAE (train.py:99-101), the mean SSIM (utils.py:81-114),
    the confidence 1 + exp(fc2(relu(fc1(rx)))) and the evaluation loss
    (1 - lambda1) MAE + lambda1 (1 - SSIM), in one launch over the C ABI.
    ``__call__`` returns a [R, 6] tensor in the order of ``METRICS``."""

    def __init__(self, R, H, W, hidden=32, device="cuda", lambda1=LAMBDA1):
        self.R, self.H, self.W, self.hidden = int(R), int(H), int(W), int(hidden)
        self.lambda1 = float(lambda1)
        dev = torch.device(device)
        n = int(_lib.lib().gsparc_eval_scratch_floats(self.R, self.H, self.W))
        self.scratch = torch.zeros(max(n, 1), dtype=torch.float32, device=dev)   # zero once: arrival counters
        self.metrics = torch.zeros((self.R, len(METRICS)), dtype=torch.float32, device=dev)

    def __call__(self, pred, target, rx_pos, conf_params):
        for name, t, shape in (("pred", pred, (self.R, self.H, self.W)), ("target", target, (self.R, self.H, self.W)),
                               ("rx_pos", rx_pos, (self.R, 3)), ("conf_params", conf_params, (conf_floats(self.hidden),))):
            if t.dtype != torch.float32 or not t.is_cuda or not t.is_contiguous() or t.numel() != _numel(shape):
                raise ValueError(f"{name} must be a contiguous float32 CUDA tensor of shape {shape}")
        check("eval_metrics", _lib.lib().gsparc_eval_metrics(
            self.R, self.H, self.W, self.hidden, self.lambda1, C1, C2, ptr(pred), ptr(target), ptr(rx_pos),
            ptr(conf_params), ptr(self.scratch), ptr(self.metrics), stream_of(pred.device)))
        return self.metrics


def _numel(shape):
    n = 1
    for s in shape:
        n *= s
    return n
