import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
for p in (os.path.join(ROOT, "dopamine-fdm_b200"), os.path.join(ROOT, "oracle")):
    if p not in sys.path:
        sys.path.insert(0, p)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200); parity tests through the C ABI")
    config.addinivalue_line("markers", "slow: long-running case")


def has_gpu() -> bool:
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False


def pytest_collection_modifyitems(config, items):
    if has_gpu():
        return
    skip = pytest.mark.skip(reason="no CUDA GPU in this environment")
    for it in items:
        if "gpu" in it.keywords:
            it.add_marker(skip)


def rel_l2(a, b) -> float:
    a = np.asarray(a, dtype=np.float64)
    b = np.asarray(b, dtype=np.float64)
    den = np.linalg.norm(b.ravel())
    num = np.linalg.norm((a - b).ravel())
    return float(num / den) if den > 0 else float(num)


def interior(case, key, a):
    """Independent cells of a ghosted reference array (periodic duplicates and ghosts removed)."""
    Nx, Ny, Nz = case.cells
    if key == "V":
        nyv = Ny if case.y_bc_type == 0 else Ny - 1
        return a[1:1 + Nx, 1:1 + nyv, 1:1 + Nz]
    return a[1:1 + Nx, 1:1 + Ny, 1:1 + Nz]


@pytest.fixture(scope="session")
def oracle_mod():
    import oracle as O
    O.build()
    return O
