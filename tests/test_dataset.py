"""The spectrum dataset pipeline (preprocess_data.py:116-202): view matrices
against golden values produced by the reference's own build_view_matrix
(tests/golden/make_dataset_golden.py), and the loader on a synthetic dataset
directory in the reference's layout."""
import os

import numpy as np
import pytest
import torch
import yaml

from gsparc_b200 import dataset

GOLDEN = os.path.join(os.path.dirname(__file__), "golden", "dataset_views_golden.npz")


def test_view_matrices_match_reference_golden():
    g = np.load(GOLDEN)
    for qi, q in enumerate(g["quats"]):
        v = dataset.view_matrices(g["rx"], q)
        np.testing.assert_allclose(v, g["views"][qi], rtol=0, atol=2e-6)


def _write_dataset(d, n=7, H=9, W=12, seed=0):
    rng = np.random.default_rng(seed)
    os.makedirs(os.path.join(d, "spectrum"))
    spectra = rng.random((n, H, W)).astype(np.float32)
    for i in range(n):
        np.save(os.path.join(d, "spectrum", f"{i + 1}.npy"), spectra[i])
    rx = rng.random((n, 3)).astype(np.float32) * 4
    with open(os.path.join(d, "rx_pos.csv"), "w") as f:
        f.write("x,y,z\n")
        for r in rx:
            f.write(",".join(repr(float(v)) for v in r) + "\n")
    quat = [0.1, 0.2, -0.3, 0.927]
    with open(os.path.join(d, "gateway_info.yml"), "w") as f:
        yaml.safe_dump({"gateway1": {"position": [0.0, 0.0, 1.0], "orientation": quat}}, f)
    names = ["5", "2", "7", "1"]
    np.savetxt(os.path.join(d, "train_index.txt"), np.array(names), fmt="%s")
    return spectra, rx, quat, names


def test_loader_reads_the_reference_layout(tmp_path):
    spectra, rx, quat, names = _write_dataset(str(tmp_path))
    ds = dataset.SpectrumDataset(str(tmp_path), str(tmp_path / "train_index.txt"), pin=False)
    assert len(ds) == 4 and ds.names == names
    idx = [int(n) - 1 for n in names]                      # rx_pos[int(idx) - 1]
    np.testing.assert_array_equal(ds.spectra.numpy(), spectra[idx])
    np.testing.assert_allclose(ds.rx.numpy(), rx[idx], rtol=0, atol=1e-6)
    np.testing.assert_array_equal(ds.tx.numpy(), np.tile(np.float32(dataset.TX_FIXED), (4, 1)))
    np.testing.assert_allclose(ds.views.numpy(), dataset.view_matrices(rx[idx], quat), rtol=0, atol=0)
    b = list(ds.batch_indices(2, shuffle=True, seed=1))
    assert len(b) == 2 and sorted(torch.cat(b).tolist()) == [0, 1, 2, 3]
    assert [x.tolist() for x in ds.batch_indices(3, shuffle=False)] == [[0, 1, 2]]


@pytest.mark.gpu
def test_device_prefetcher_streams_batches_into_the_training_step(tmp_path):
    from gsparc_b200 import scenes
    from gsparc_b200.fused import FusedTrainer
    from gsparc_b200.shared_mlp import SharedMLP
    dev = torch.device("cuda")
    spectra, rx, quat, names = _write_dataset(str(tmp_path), n=7, H=90, W=360)
    ds = dataset.SpectrumDataset(str(tmp_path), str(tmp_path / "train_index.txt"))
    pf = dataset.DevicePrefetcher(ds, 2, dev, shuffle=True, seed=3)
    order = [b.tolist() for b in ds.batch_indices(2, shuffle=True, seed=3)]
    seen = []
    for views, rxs, targets in pf:
        seen.append((views.cpu().clone(), rxs.cpu().clone(), targets.cpu().clone()))
    assert len(seen) == len(order) == 2
    for (v, r, s), idx in zip(seen, order):
        assert torch.equal(v, ds.views[idx]) and torch.equal(r, ds.rx[idx]) and torch.equal(s, ds.spectra[idx])
    tr = FusedTrainer(scenes.make_scene(2000, seed=0), device=dev, shared=SharedMLP(2, 64, "relu"))
    tx = torch.tensor(dataset.TX_FIXED, device=dev)
    first = next(iter(pf))
    cap = tr.probe_capacity(first[0], first[1], tx)
    tr.capture(2, 2 * cap, tx, *first)
    losses = [float(tr.step(v, r, s)) for v, r, s in pf]
    tr.plan.check()
    assert len(losses) == 2 and all(np.isfinite(losses))
