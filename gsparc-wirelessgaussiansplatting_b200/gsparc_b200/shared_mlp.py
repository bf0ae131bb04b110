"""Shared emission MLP (one network for all Gaussians) over the C ABI.

The benchmark configurations name this model: per (receiver, Gaussian) pair,
32 features -- the centre, a 4-frequency positional encoding of it, the
receiver-relative direction and 1/d^2 -- through ``layers`` hidden layers of
``width`` (ReLU or GELU) to one amplitude, whose sigmoid is the pair's signal
(real channel).  The reference's own emission model is the per-Gaussian
3-32-2 MLP (``EmissionMLPs``, gaussian.py:554-572), which stays the drop-in
default; this one is selected with ``shared=`` in ``raster.forward`` /
``raster.backward`` and in ``FusedTrainer``.

Parameters are one flat fp32 tensor, layer by layer: W [out, in] row-major,
then b [out].
"""
from __future__ import annotations

import math

import torch

from . import _lib
from ._lib import check, ptr, stream_of

FEATURES = 32
ACTS = {"relu": 1, "gelu": 2}
PRECISIONS = {"fp32": 0, "bf16": 1}


def _shapes(layers, width, out):
    dims = [FEATURES] + [width] * layers + [out]
    return [(dims[i + 1], dims[i]) for i in range(len(dims) - 1)]


def init_params_host(layers, width, out=1, seed=0):
    """nn.Linear's default initialisation (uniform +-1/sqrt(fan_in)) per
    layer, flat fp32 on the host (torch CPU generator, seeded)."""
    g = torch.Generator().manual_seed(seed)
    parts = []
    for o, i in _shapes(layers, width, out):
        bound = 1.0 / math.sqrt(i)
        parts.append(((torch.rand((o, i), generator=g) * 2 - 1) * bound).reshape(-1))
        parts.append((torch.rand((o,), generator=g) * 2 - 1) * bound)
    return torch.cat(parts).numpy()


class SharedMLP:
    """Spec of the shared MLP plus the workspace its forward keeps for the
    backward (sized per (P, R) on first use)."""

    def __init__(self, layers=2, width=64, act="relu", out=1, precision="fp32"):
        if act not in ACTS:
            raise ValueError(f"act must be one of {sorted(ACTS)}")
        if precision not in PRECISIONS:
            raise ValueError(f"precision must be one of {sorted(PRECISIONS)}")
        self.layers, self.width, self.act, self.out, self.precision = int(layers), int(width), act, int(out), precision
        self._work = None
        self._work_key = None

    @property
    def n_params(self):
        return int(_lib.lib().gsparc_shared_mlp_param_floats(self.layers, self.width, self.out))

    def shapes(self):
        """[(out, in)] per layer, input layer first."""
        return _shapes(self.layers, self.width, self.out)

    def init_params(self, seed=0, device="cuda"):
        """nn.Linear's default initialisation (uniform +-1/sqrt(fan_in)) per layer."""
        flat = torch.from_numpy(init_params_host(self.layers, self.width, self.out, seed)).to(device)
        assert flat.numel() == self.n_params
        return flat

    def unflatten(self, flat):
        """[(W, b)] views of a flat parameter tensor."""
        out, off = [], 0
        for o, i in self.shapes():
            w = flat[off:off + o * i].view(o, i)
            off += o * i
            b = flat[off:off + o]
            off += o
            out.append((w, b))
        return out

    def workspace(self, P, R, device):
        key = (int(P), int(R), str(device))
        if self._work_key != key:
            n = int(_lib.lib().gsparc_shared_mlp_workspace_floats(int(P), int(R), self.layers, self.width, self.out,
                                                                  PRECISIONS[self.precision]))
            self._work = torch.empty(max(n, 1), dtype=torch.float32, device=device)
            self._work_key = key
        return self._work

    def features(self, P, R):
        """[R, P, out] amplitudes (sigmoid outputs) of the last forward: the
        first R*P*out floats of the workspace."""
        return self._work[:int(R) * int(P) * self.out].view(int(R), int(P), self.out)

    def _spec(self):
        return (self.layers, self.width, ACTS[self.act], self.out, PRECISIONS[self.precision])

    def forward(self, P, R, means3D, rx_pos, params, geom, image=None):
        """Write the signal of every visible pair into a prepared forward's
        geometry arena (``image``: its image arena, for the error word)."""
        dev = means3D.device
        work = self.workspace(P, R, dev)
        check("shared_mlp_forward", _lib.lib().gsparc_shared_mlp_forward(
            int(P), int(R), *self._spec(), ptr(means3D), ptr(rx_pos), ptr(params), ptr(geom),
            ptr(image) if image is not None else None, ptr(work), stream_of(dev)))

    def backward(self, P, R, means3D, rx_pos, params, geom, dsignal, dparams, dmeans3D, image=None):
        """dparams is overwritten; dL/dmeans3D through the features is added to dmeans3D."""
        dev = means3D.device
        work = self.workspace(P, R, dev)
        check("shared_mlp_backward", _lib.lib().gsparc_shared_mlp_backward(
            int(P), int(R), *self._spec(), ptr(means3D), ptr(rx_pos), ptr(params), ptr(geom),
            ptr(image) if image is not None else None, ptr(work), ptr(dsignal), ptr(dparams), ptr(dmeans3D),
            stream_of(dev)))


def bf16_act_table(act, device="cuda"):
    """The BF16 path's activation for every BF16 input, as its kernels
    evaluate it: (a_forward, a_adjoint, a') float32 tensors of 65,536 entries,
    entry i for the input whose BF16 bit pattern is i, each from the low lane
    of a packed pair; raises if the high lane ever differs."""
    out = torch.empty(6 * 65536, dtype=torch.int16, device=device)
    check("shared_mlp_bf16_act_table",
          _lib.lib().gsparc_shared_mlp_bf16_act_table(ACTS[act], ptr(out), stream_of(torch.device(device))))
    t = out.view(3, 2, 65536)
    if not torch.equal(t[:, 0], t[:, 1]):
        raise RuntimeError("packed BF16 activation: the two lanes disagree")
    bits = t[:, 0].to(torch.int32) << 16
    f = bits.view(torch.float32)
    return f[0].clone(), f[1].clone(), f[2].clone()
