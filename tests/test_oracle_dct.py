"""The oracle's DCT-IV Poisson path (inflow/outflow x, src/projection.f90:124-130,334-343), pinned without the reference:
the DCT-IV against its definition and its self-inverse property, and the solution against the discrete operator it
inverts.  The DCT-IV basis cos(pi (2n+1)(2k+1) / (4N)) is even about the inflow face (ghost phi_-1 = phi_0, Neumann) and
odd about the outflow face (ghost phi_N = -phi_(N-1), Dirichlet), with eigenvalues 2 (cos(pi (2k+1) / (2N)) - 1) / dx^2;
with walls in y (Dyy) and periodic z the solved field must reproduce the right-hand side under that operator."""
import os
import sys

import numpy as np
import pytest

from dfdm.cases import inflow_outflow

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, os.path.join(ROOT, "oracle"))


def dct_case(nx=18, ny=17, nz=18, grid_type=2):
    return inflow_outflow(nx, ny, nz, grid_type)


@pytest.fixture(scope="module")
def oracle_mod():
    import oracle
    oracle.build()
    return oracle


@pytest.mark.parametrize("nx", [18, 34])
def test_dct4_matches_its_definition_and_is_its_own_inverse(oracle_mod, nx):
    o = oracle_mod.Oracle(dct_case(nx=nx))
    N = nx - 1
    rng = np.random.default_rng(nx)
    x = rng.standard_normal(N)
    n = np.arange(N)
    want = 2.0 * np.array([np.sum(x * np.cos(np.pi * (2 * n + 1) * (2 * k + 1) / (4 * N))) for k in range(N)])
    got = o.dct4(x)
    assert np.max(np.abs(got - want)) <= 1e-12 * np.max(np.abs(want))
    back = o.dct4(got) / (2 * N)
    assert np.max(np.abs(back - x)) <= 1e-13 * np.max(np.abs(x))
    o.close()


def _operator(o, phi, N, nym, nzp):
    """The discrete Laplacian the DCT-IV solve inverts, on the interior (x: N cells, y: nym rows, z: nzp planes)."""
    dx, dz = o.grid_array(7)
    d, lo, up = o.grid_array(5), o.grid_array(8), o.grid_array(9)
    p = phi[:N, :nym, :nzp]
    px = np.concatenate([p[:1], p, -p[-1:]], axis=0)                    # Neumann inflow, Dirichlet outflow
    lap = (px[2:] - 2.0 * px[1:-1] + px[:-2]) / dx**2
    ly = d[None, :, None] * p
    ly[:, 1:, :] += lo[None, 1:, None] * p[:, :-1, :]
    ly[:, :-1, :] += up[None, :-1, None] * p[:, 1:, :]
    lz = (np.roll(p, -1, axis=2) - 2.0 * p + np.roll(p, 1, axis=2)) / dz**2
    return lap + ly + lz


@pytest.mark.parametrize("nx,ny,nz,grid_type", [(18, 17, 18, 2), (34, 21, 16, 1)])
def test_dct_poisson_solution_satisfies_the_discrete_problem(oracle_mod, nx, ny, nz, grid_type):
    c = dct_case(nx, ny, nz, grid_type)
    o = oracle_mod.Oracle(c)
    N, nym, nzp = nx - 1, ny - 1, nz - 2
    rng = np.random.default_rng(7)
    rhs = np.asfortranarray(rng.standard_normal((nx, ny - 1, nz)))
    phi = o.solve_poisson(rhs)
    res = _operator(o, phi, N, nym, nzp) - rhs[:N, :nym, :nzp]
    assert np.max(np.abs(res)) <= 1e-10 * np.max(np.abs(rhs)), np.max(np.abs(res))
    # the planes the reference leaves alone keep their input; the periodic z copy is made
    assert np.array_equal(phi[N], rhs[N])
    assert np.array_equal(phi[:N, :, nzp], phi[:N, :, 0])
    o.close()
