"""Spectrum dataset pipeline: the reference's Spectrum_dataset
(preprocess_data.py:116-202) as batched host tensors, and a prefetcher that
streams R-receiver batches into device buffers for the training step.

Dataset directory layout (as the reference's "rfid" spectrum datasets):
  spectrum/<idx>.npy   one [n_elevation, n_azimuth] float spectrum per sample
  rx_pos.csv           receiver positions, one row per sample (header row)
  gateway_info.yml     gateway1: position, orientation (quaternion x, y, z, w)
  train_index.txt / test_index.txt   sample names, one per line

Per sample (preprocess_data.py:157-172): the spectrum, rx_pos[int(idx) - 1],
the fixed transmitter (0, 0.5, 3) and the view matrix of build_view_matrix
(preprocess_data.py:180-202): R_w2c = R(q)^T, t = -R_w2c rx, stored
transposed (column-major, as the rasterizer reads it).
"""
from __future__ import annotations

import os

import numpy as np
import torch

TX_FIXED = (0.0, 0.5, 3.0)   # preprocess_data.py:156


def quat_to_matrix(q) -> np.ndarray:
    """Rotation matrix of a scalar-last quaternion (x, y, z, w), normalised
    first (the convention of scipy's Rotation.from_quat), in float64."""
    x, y, z, w = np.asarray(q, dtype=np.float64) / np.linalg.norm(np.asarray(q, dtype=np.float64))
    return np.array([[1 - 2 * (y * y + z * z), 2 * (x * y - z * w), 2 * (x * z + y * w)],
                     [2 * (x * y + z * w), 1 - 2 * (x * x + z * z), 2 * (y * z - x * w)],
                     [2 * (x * z - y * w), 2 * (y * z + x * w), 1 - 2 * (x * x + y * y)]])


def view_matrices(rx_pos, quat) -> np.ndarray:
    """[N,3] receiver positions -> [N,4,4] float32 view matrices
    (build_view_matrix: rotation cast to float32, then t = -R_w2c rx in float32)."""
    rx = np.asarray(rx_pos, dtype=np.float32).reshape(-1, 3)
    r_w2c = quat_to_matrix(quat).astype(np.float32).T
    out = np.zeros((rx.shape[0], 4, 4), dtype=np.float32)
    out[:, :3, :3] = r_w2c
    out[:, :3, 3] = -(rx @ r_w2c.T)
    out[:, 3, 3] = 1.0
    return np.ascontiguousarray(out.transpose(0, 2, 1))


class SpectrumDataset:
    """All samples of one split in host memory (pinned when CUDA is present):
    ``spectra`` [N,H,W], ``rx`` [N,3], ``tx`` [N,3], ``views`` [N,4,4], float32."""

    def __init__(self, datadir, index_file, pin=True):
        import pandas as pd
        import yaml
        self.datadir = datadir
        self.names = [str(s) for s in np.atleast_1d(np.loadtxt(index_file, dtype=str))]
        rx_all = pd.read_csv(os.path.join(datadir, "rx_pos.csv")).values.astype(np.float32)
        with open(os.path.join(datadir, "gateway_info.yml")) as f:
            self.quat = yaml.safe_load(f)["gateway1"]["orientation"]
        spectra = [np.load(os.path.join(datadir, "spectrum", n + ".npy")).astype(np.float32) for n in self.names]
        rx = np.stack([rx_all[int(n) - 1] for n in self.names]).astype(np.float32)
        pin = pin and torch.cuda.is_available()
        t = lambda a: (torch.from_numpy(np.ascontiguousarray(a)).pin_memory() if pin
                       else torch.from_numpy(np.ascontiguousarray(a)))
        self.spectra = t(np.stack(spectra))
        self.rx = t(rx)
        self.tx = t(np.tile(np.array(TX_FIXED, dtype=np.float32), (len(self.names), 1)))
        self.views = t(view_matrices(rx, self.quat))

    def __len__(self):
        return len(self.names)

    def batch_indices(self, R, shuffle=True, seed=0):
        """Index batches of R samples covering one epoch (the last partial batch dropped)."""
        order = np.random.default_rng(seed).permutation(len(self)) if shuffle else np.arange(len(self))
        for b in range(len(self) // R):
            yield torch.from_numpy(order[b * R:(b + 1) * R].astype(np.int64))


class DevicePrefetcher:
    """Streams R-sample batches of a SpectrumDataset to the device: batch i+1
    is gathered into pinned staging memory and copied on a side stream while
    batch i is consumed, into alternating device buffers.  Iterating yields
    (views [R,4,4], rx [R,3], spectra [R,H,W]) device tensors, valid until
    the next item is requested."""

    def __init__(self, ds: SpectrumDataset, R, device="cuda", shuffle=True, seed=0):
        self.ds, self.R, self.dev = ds, int(R), torch.device(device)
        self.shuffle, self.seed = shuffle, seed
        H, W = ds.spectra.shape[1:]
        pin = torch.cuda.is_available()
        host = lambda *s: torch.empty(s, dtype=torch.float32).pin_memory() if pin else torch.empty(s)
        self._stage = [(host(R, 4, 4), host(R, 3), host(R, H, W)) for _ in range(2)]
        dev = lambda *s: torch.empty(s, dtype=torch.float32, device=self.dev)
        self._bufs = [(dev(R, 4, 4), dev(R, 3), dev(R, H, W)) for _ in range(2)]
        self._stream = torch.cuda.Stream(self.dev)
        self._ready = [torch.cuda.Event() for _ in range(2)]
        self._free = [torch.cuda.Event() for _ in range(2)]

    def _issue(self, k, idx):
        sv, sr, ss = self._stage[k]
        self._free[k].synchronize()   # the staging copy of two batches ago has left the host buffer
        torch.index_select(self.ds.views, 0, idx, out=sv)
        torch.index_select(self.ds.rx, 0, idx, out=sr)
        torch.index_select(self.ds.spectra, 0, idx, out=ss)
        with torch.cuda.stream(self._stream):
            self._stream.wait_event(self._free[k])   # the device buffer is no longer read by the step
            for d, h in zip(self._bufs[k], self._stage[k]):
                d.copy_(h, non_blocking=True)
            self._ready[k].record(self._stream)

    def __iter__(self):
        batches = list(self.ds.batch_indices(self.R, self.shuffle, self.seed))
        cur = torch.cuda.current_stream(self.dev)
        for k in range(2):
            self._free[k].record(cur)
        if not batches:
            return
        self._issue(0, batches[0])
        for i in range(len(batches)):
            k = i & 1
            if i + 1 < len(batches):
                self._issue(k ^ 1, batches[i + 1])
            cur.wait_event(self._ready[k])
            yield self._bufs[k]
            self._free[k].record(cur)   # the step that used buffer k is queued before this point
