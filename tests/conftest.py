"""Test configuration: import paths and the ``gpu`` marker.

GPU tests are marked ``@pytest.mark.gpu``; ``-m "not gpu"`` runs the CPU
suite (oracle vs golden vectors, host logic, C-ABI loading and argument
checks, multi-process gloo tests)."""
import os
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
PKG = os.path.join(ROOT, "gsparc-wirelessgaussiansplatting_b200")
for p in (PKG, ROOT):
    if p not in sys.path:
        sys.path.insert(0, p)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200, sm_100a)")
