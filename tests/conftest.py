import json
import os
import sys
from pathlib import Path

import numpy as np
import pytest

ROOT = Path(__file__).resolve().parents[1]
GOLDEN = ROOT / "tests" / "golden"
sys.path.insert(0, str(ROOT))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200, sm_100a)")


def _cuda_available() -> bool:
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False


HAS_GPU = _cuda_available()


def pytest_collection_modifyitems(config, items):
    if HAS_GPU:
        return
    skip = pytest.mark.skip(reason="no CUDA device")
    for item in items:
        if "gpu" in item.keywords:
            item.add_marker(skip)


def load_triangle_csr(path, prefix=""):
    from oracle import oracle as O
    z = np.load(path)
    n = int(z["n"])
    g = (lambda k: z[prefix + k])
    return O.csr_from_triplets(n, g("row"), g("col"), g("val"), True)


@pytest.fixture(scope="session")
def sio():
    return load_triangle_csr(GOLDEN / "SiO.npz")


@pytest.fixture(scope="session")
def kuumuu():
    from oracle import oracle as O
    z = np.load(GOLDEN / "KuuMuu.npz")
    n = int(z["n"])
    K = O.csr_from_triplets(n, z["k_row"], z["k_col"], z["k_val"], True)
    M = O.csr_from_triplets(n, z["m_row"], z["m_col"], z["m_val"], True)
    return K, M


@pytest.fixture(scope="session")
def spectra():
    return json.loads((GOLDEN / "spectra.json").read_text())
