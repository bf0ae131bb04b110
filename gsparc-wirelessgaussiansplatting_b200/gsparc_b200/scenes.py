"""Seeded synthetic RF Gaussian scenes standing in for the measured spectra.

The real dataset (Sionna conference-room spectra, 90x360 per receiver, one
transmitter at (0, 0.5, 3), preprocess_data.py:154) is not available, so scenes
are drawn with the shapes and distributions of the benchmark configurations:

  * Gaussian means uniform in a 10 x 3 x 8 m room: x in [-5, 5], y (up, the
    elevation axis of the projection) in [0, 3], z in [-4, 4];
  * log-scales ~ N(-2, 0.5) per axis; quaternions = normalise(N(0, I4));
    opacity logits ~ N(0, 1);
  * per-Gaussian emission MLP weights ~ N(0, 1), as EmissionMLPs initialises
    them (gaussian.py:556-563);
  * optional clustering: a fraction of the means drawn from isotropic
    N(c_k, 0.3 m) clusters with centres uniform in the room;
  * receivers uniform in the room; view matrices follow build_view_matrix
    (preprocess_data.py:177-202) with an identity gateway orientation:
    R_w2c = I, t = -rx, stored transposed.

Seeds: scene 0, target scene 1, receivers 2, finite-difference picks 3.
"""
from __future__ import annotations

from dataclasses import dataclass

import numpy as np

ROOM_LO = np.array([-5.0, 0.0, -4.0])
ROOM_HI = np.array([5.0, 3.0, 4.0])
TX_POS = np.array([0.0, 0.5, 3.0], dtype=np.float32)
H, W = 90, 360

SEED_SCENE, SEED_TARGET, SEED_RX, SEED_FD = 0, 1, 2, 3


@dataclass
class Scene:
    means: np.ndarray          # [P,3] float32
    log_scales: np.ndarray     # [P,3]
    quats: np.ndarray          # [P,4] raw (unnormalised) quaternions (w, x, y, z)
    opacity_logits: np.ndarray # [P,1]
    mlp: np.ndarray            # [194*P] flat EmissionMLPs layout

    @property
    def P(self):
        return self.means.shape[0]

    def activated(self):
        """(means, scales, rotations, opacities) after the GaussianModel
        activations exp / normalize / sigmoid (gaussian.py:33-38)."""
        s = np.exp(self.log_scales).astype(np.float32)
        q = self.quats / np.linalg.norm(self.quats, axis=1, keepdims=True)
        o = (1.0 / (1.0 + np.exp(-self.opacity_logits))).astype(np.float32)
        return self.means, s, q.astype(np.float32), o


def make_scene(P: int, seed: int = SEED_SCENE, cluster_frac: float = 0.0, n_clusters: int = 5,
               cluster_sigma: float = 0.3) -> Scene:
    rng = np.random.default_rng(seed)
    means = rng.uniform(ROOM_LO, ROOM_HI, size=(P, 3))
    if cluster_frac > 0:
        nc = int(round(cluster_frac * P))
        centres = rng.uniform(ROOM_LO, ROOM_HI, size=(n_clusters, 3))
        which = rng.integers(0, n_clusters, size=nc)
        means[:nc] = centres[which] + rng.normal(0.0, cluster_sigma, size=(nc, 3))
        means[:nc] = np.clip(means[:nc], ROOM_LO, ROOM_HI)
    log_scales = rng.normal(-2.0, 0.5, size=(P, 3))
    quats = rng.normal(size=(P, 4))
    opac = rng.normal(size=(P, 1))
    mlp = rng.normal(size=(194 * P,))
    f = lambda a: np.ascontiguousarray(a, dtype=np.float32)
    return Scene(f(means), f(log_scales), f(quats), f(opac), f(mlp))


def make_receivers(R: int, seed: int = SEED_RX) -> np.ndarray:
    rng = np.random.default_rng(seed)
    return rng.uniform(ROOM_LO, ROOM_HI, size=(R, 3)).astype(np.float32)


def view_matrix(rx: np.ndarray) -> np.ndarray:
    """Transposed world->receiver matrix with identity orientation
    (preprocess_data.py:177-202): rows 0-2 identity, row 3 = (-rx, 1)."""
    v = np.eye(4, dtype=np.float32)
    v[3, :3] = -np.asarray(rx, dtype=np.float32)
    return v


def view_matrices(rxs: np.ndarray) -> np.ndarray:
    return np.stack([view_matrix(r) for r in rxs]).astype(np.float32)


CONFIGS = {
    # name: (P, R, cluster_frac)
    "cfg0_forward_4k": (4096, 1, 0.0),
    "cfg1_train_20k": (20000, 1, 0.0),
    "cfg2_batched_50k_r64": (50000, 64, 0.3),
    "cfg3_mixed_200k_r32": (200000, 32, 0.0),
    "cfg4_multifreq_100k_r16": (100000, 16, 0.0),
}
