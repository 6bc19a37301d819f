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


def cfl_reference(c, U, V, W, nu_t, dt=None):
    """compute_cfl (src/monitor.f90:304-424) on the ghosted 1-based arrays: i = 2..nxg-1, j = 2..nyg-1,
    k = 2..nzg-1, written out in numpy (0-based slices)."""
    from dfdm import cases
    x, y, z = cases.faces(c)
    dx = np.diff(cases.centres(x)).min()
    idx = 1.0 / dx
    idy = 1.0 / np.maximum(y[1:] - y[:-1], 1e-14)      # index j-2 holds 1/(y(j) - y(j-1)) for j = 2..ny
    idz = 1.0 / np.maximum(z[1:] - z[:-1], 1e-14)
    nxg, nyg, nzg = c.nxg, c.nyg, c.nzg
    I, J, K = slice(1, nxg - 1), slice(1, nyg - 1), slice(1, nzg - 1)
    uc = 0.5 * (U[1:nxg - 1, J, K] + U[0:nxg - 2, J, K])
    vc = 0.5 * (V[I, 1:nyg - 1, K] + V[I, 0:nyg - 2, K])
    wc = 0.5 * (W[I, J, 1:nzg - 1] + W[I, J, 0:nzg - 2])
    iy = idy[0:nyg - 2][None, :, None]
    iz = idz[0:nzg - 2][None, None, :]
    conv = (np.abs(uc) * idx + np.abs(vc) * iy + np.abs(wc) * iz).max()
    visc = ((c.nu + nu_t[I, J, K]) * 2.0 * (idx * idx + iy * iy + iz * iz)).max()
    dt = c.dt if dt is None else dt
    return conv * dt, visc * dt
