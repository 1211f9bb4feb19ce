import os
import sys
from pathlib import Path

import numpy as np
import pytest

ROOT = Path(__file__).resolve().parents[1]
sys.path.insert(0, str(ROOT / "sie-gstc-2026_b200"))
sys.path.insert(0, str(ROOT))

GOLDEN = ROOT / "tests" / "golden" / "golden.npz"


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200); run with -m gpu")


def has_gpu() -> bool:
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False


@pytest.fixture(scope="session")
def golden():
    return dict(np.load(GOLDEN))


@pytest.fixture(scope="session")
def oracle_lib():
    from oracle import oracle as O
    return O.oracle()


@pytest.fixture(scope="session")
def ref_lib():
    from oracle import oracle as O
    lib = O.reference()
    if lib is None:
        pytest.skip("reference harness oracle/_ref/libsieref.so not built")
    return lib


@pytest.fixture(scope="session")
def gpu_ctx():
    if not has_gpu():
        pytest.skip("no CUDA device")
    import sieb200
    return sieb200.Context(0)


class GoldenMesh:
    def __init__(self, g, name):
        self.vertices = g[f"ico_{name}_V"]
        self.faces = g[f"ico_{name}_F"].astype(np.int32)
        self.edges = g[f"ico_{name}_E"].astype(np.int32)
        self.faces_edges = g[f"ico_{name}_FE"].astype(np.int32)


@pytest.fixture(scope="session")
def mesh_l0(golden):
    return GoldenMesh(golden, "L0")


def rel_err(a, b):
    a = np.asarray(a)
    b = np.asarray(b)
    den = max(np.abs(b).max(), 1e-300)
    return float(np.abs(a - b).max() / den)
