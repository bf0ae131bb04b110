"""Golden view matrices from the reference's own dataset code.

Calls Spectrum_dataset.build_view_matrix (preprocess_data.py:180-202) of the
reference checkout on a few receiver positions and gateway orientations and
saves the results to dataset_views_golden.npz.  Run from the repository
root in a container with the reference checked out:

    python tests/golden/make_dataset_golden.py [REFERENCE_ROOT]

preprocess_data imports imageio (for the PNG spectra of another dataset
type) at module level; the method used here does not touch it, so an empty
stand-in module satisfies the import when imageio is not installed.
"""
import os
import sys
import tempfile
import types

import numpy as np
import torch
import yaml


def main(ref_dir):
    sys.path.insert(0, ref_dir)
    if "imageio" not in sys.modules:
        try:
            import imageio  # noqa: F401
        except ImportError:
            sys.modules["imageio"] = types.ModuleType("imageio")
    import preprocess_data as pdm

    rng = np.random.default_rng(2024)
    rx = (rng.random((6, 3)) * np.array([10.0, 8.0, 3.0]) - np.array([5.0, 4.0, 0.0])).astype(np.float32)
    quats = np.array([[0.0, 0.0, 0.0, 1.0], [0.5, -0.5, 0.5, 0.5], [0.1, 0.2, -0.3, 0.927]], dtype=np.float64)
    quats /= np.linalg.norm(quats, axis=1, keepdims=True)
    views = np.zeros((len(quats), len(rx), 4, 4), dtype=np.float32)
    with tempfile.TemporaryDirectory() as d:
        for qi, q in enumerate(quats):
            path = os.path.join(d, "gateway_info.yml")
            with open(path, "w") as f:
                yaml.safe_dump({"gateway1": {"position": [0.0, 0.0, 1.0], "orientation": [float(v) for v in q]}}, f)
            fake = types.SimpleNamespace(gateway_pos_dir=path)
            for ri in range(len(rx)):
                views[qi, ri] = pdm.Spectrum_dataset.build_view_matrix(fake, torch.tensor(rx[ri])).numpy()
    out = os.path.join(os.path.dirname(os.path.abspath(__file__)), "dataset_views_golden.npz")
    np.savez(out, rx=rx, quats=quats, views=views)
    print("wrote", out)


if __name__ == "__main__":
    sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
    from oracle.build_ref import REF_ROOT
    main(sys.argv[1] if len(sys.argv) > 1 else REF_ROOT)
