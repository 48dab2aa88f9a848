import os
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200); runs the CUDA path")
    # the oracle restatement (plain C, and its FMA and dual-number builds) is
    # rebuilt here when missing
    for name in ("liboracle.so", "liboracle_fma.so", "liboracle_dual.so"):
        if not os.path.exists(os.path.join(ROOT, "oracle", name)):
            subprocess.run(["make", "-C", os.path.join(ROOT, "oracle"), name], check=True,
                           stdout=subprocess.DEVNULL)


def pytest_collection_modifyitems(config, items):
    try:
        import torch
        have_gpu = torch.cuda.is_available()
    except Exception:  # pragma: no cover
        have_gpu = False
    if have_gpu:
        return
    skip = pytest.mark.skip(reason="no CUDA device")
    for it in items:
        if "gpu" in it.keywords:
            it.add_marker(skip)
