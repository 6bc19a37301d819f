"""The oracle's 4-wall duct pressure solve (z walls with y walls, periodic x; src/projection.f90:172-217,
src/initialization.f90:543-618), pinned without the reference: the eigenvalues of the symmetrised z operator against
their closed form on uniform z faces, and the solved field against the discrete operator it inverts (periodic x
differences, Dyy and Dzz with their Neumann end rows).  Periodic x with Neumann y and z leaves the constant field in
the operator's null space; the right-hand side is the operator applied to a random field, so it lies in the range
and the pinned null mode (D(2) * 3/2 for kx = 0 and the zero eigenvalue) changes nothing."""
import os
import sys

import numpy as np
import pytest

from dfdm.cases import duct, inflow_duct, spanwise_wall

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, os.path.join(ROOT, "oracle"))


@pytest.fixture(scope="module")
def oracle_mod():
    import oracle
    oracle.build()
    return oracle


@pytest.mark.parametrize("nz", [10, 18, 34])
def test_duct_eigenvalues_match_the_neumann_spectrum(oracle_mod, nz):
    c = duct(18, 17, nz)
    o = oracle_mod.Oracle(c)
    lam = o.grid_array(13)
    N = nz - 1
    dz = c.Lz_i / (nz - 1)
    want = np.sort(2.0 * (np.cos(np.pi * np.arange(N) / N) - 1.0) / dz**2)
    assert lam.size == N
    assert np.max(np.abs(lam - want)) <= 1e-12 * np.max(np.abs(want))
    assert np.all(np.diff(lam) >= 0.0)
    o.close()


def operator(o, p, dx):
    """The discrete Laplacian of the duct solve on the interior (x: Nx periodic cells, y: Ny rows, z: Nz planes)."""
    dy, ly, uy = o.grid_array(5), o.grid_array(8), o.grid_array(9)
    dzz, lz, uz = o.grid_array(10), o.grid_array(11), o.grid_array(12)
    out = (np.roll(p, -1, axis=0) - 2.0 * p + np.roll(p, 1, axis=0)) / dx**2
    out += dy[None, :, None] * p
    out[:, 1:, :] += ly[None, 1:, None] * p[:, :-1, :]
    out[:, :-1, :] += uy[None, :-1, None] * p[:, 1:, :]
    out += dzz[None, None, :] * p
    out[:, :, 1:] += lz[None, None, 1:] * p[:, :, :-1]
    out[:, :, :-1] += uz[None, None, :-1] * p[:, :, 1:]
    return out


def duct_rhs(o, c, seed):
    """rhs_p in the reference's shape whose solved part is the operator applied to a random field."""
    Nx, Ny, Nz = c.nx - 2, c.ny - 1, c.nz - 1
    rng = np.random.default_rng(seed)
    rhs = np.asfortranarray(rng.standard_normal((c.nx, c.ny - 1, c.nz)))
    q = rng.standard_normal((Nx, Ny, Nz))
    rhs[:Nx, :Ny, :Nz] = operator(o, q, o.grid_array(7)[0])
    return rhs


@pytest.mark.parametrize("nx,ny,nz,grid_type", [(18, 17, 18, 2), (34, 21, 26, 1), (20, 33, 40, 2)])
def test_duct_solution_satisfies_the_discrete_problem(oracle_mod, nx, ny, nz, grid_type):
    c = duct(nx, ny, nz, grid_type)
    o = oracle_mod.Oracle(c)
    Nx, Ny, Nz = nx - 2, ny - 1, nz - 1
    rhs = duct_rhs(o, c, 7)
    phi = o.solve_poisson(rhs)
    res = operator(o, phi[:Nx, :Ny, :Nz], o.grid_array(7)[0]) - rhs[:Nx, :Ny, :Nz]
    assert np.max(np.abs(res)) <= 1e-10 * np.max(np.abs(rhs[:Nx, :Ny, :Nz])), np.max(np.abs(res))
    assert np.array_equal(phi[Nx], phi[0])           # apply_periodic_xz_pressure's x copy
    # no z copy with a z wall: the plane nzg keeps its input, except for the x copy, which covers every z plane
    assert np.array_equal(phi[:Nx, :, Nz], rhs[:Nx, :, Nz])
    assert np.array_equal(phi[Nx + 1, :, Nz], rhs[Nx + 1, :, Nz])
    o.close()


def spanwise_operator(o, p, dx, dy):
    """The discrete Laplacian of the spanwise-wall solve (x: Nx periodic cells, y: nyp periodic rows, z: Nz planes)."""
    dzz, lz, uz = o.grid_array(10), o.grid_array(11), o.grid_array(12)
    out = (np.roll(p, -1, axis=0) - 2.0 * p + np.roll(p, 1, axis=0)) / dx**2
    out += (np.roll(p, -1, axis=1) - 2.0 * p + np.roll(p, 1, axis=1)) / dy**2
    out += dzz[None, None, :] * p
    out[:, :, 1:] += lz[None, None, 1:] * p[:, :, :-1]
    out[:, :, :-1] += uz[None, None, :-1] * p[:, :, 1:]
    return out


def spanwise_rhs(o, c, seed):
    """rhs_p in the reference's shape whose solved part is the spanwise-wall operator applied to a random field."""
    Nx, nyp, Nz = c.nx - 2, c.ny - 2, c.nz - 1
    rng = np.random.default_rng(seed)
    rhs = np.asfortranarray(rng.standard_normal((c.nx, c.ny - 1, c.nz)))
    q = rng.standard_normal((Nx, nyp, Nz))
    rhs[:Nx, :nyp, :Nz] = spanwise_operator(o, q, o.grid_array(7)[0], c.Ly_i / (c.ny - 1))
    return rhs, q


@pytest.mark.parametrize("nx,ny,nz", [(18, 18, 18), (34, 26, 40)])
def test_spanwise_wall_solution_satisfies_the_discrete_problem(oracle_mod, nx, ny, nz):
    """Spanwise walls with periodic x and y (src/projection.f90:219-250): FFT in x and y, a z-tridiagonal solve per
    (kx, ky); the solution satisfies the operator, and the periodic copies and the untouched z-wall plane are as the
    reference leaves them (x copy, then y copy, both over every plane)."""
    c = spanwise_wall(nx, ny, nz)
    o = oracle_mod.Oracle(c)
    Nx, nyp, Nz = nx - 2, ny - 2, nz - 1
    rhs, q = spanwise_rhs(o, c, 11)
    phi = o.solve_poisson(rhs)
    res = spanwise_operator(o, phi[:Nx, :nyp, :Nz], o.grid_array(7)[0], c.Ly_i / (ny - 1)) - rhs[:Nx, :nyp, :Nz]
    assert np.max(np.abs(res)) <= 1e-10 * np.max(np.abs(rhs[:Nx, :nyp, :Nz])), np.max(np.abs(res))
    e = phi[:Nx, :nyp, :Nz] - q
    assert np.max(np.abs(e - e.mean())) <= 1e-10 * np.max(np.abs(q))
    assert np.array_equal(phi[Nx], phi[0])               # x copy
    assert np.array_equal(phi[:, nyp, :], phi[:, 0, :])   # y copy
    assert np.array_equal(phi[:Nx, :nyp, Nz], rhs[:Nx, :nyp, Nz])   # the z-wall plane keeps its input
    o.close()


def inflow_duct_operator(o, p, dx):
    """The discrete Laplacian of the inflow/outflow duct: x with the Neumann inflow (ghost p_-1 = p_0) and Dirichlet
    outflow (ghost p_N = -p_(N-1)) of the DCT-IV basis, Dyy and Dzz with their wall rows."""
    dy, ly, uy = o.grid_array(5), o.grid_array(8), o.grid_array(9)
    dzz, lz, uz = o.grid_array(10), o.grid_array(11), o.grid_array(12)
    px = np.concatenate([p[:1], p, -p[-1:]], axis=0)
    out = (px[2:] - 2.0 * px[1:-1] + px[:-2]) / dx**2
    out += dy[None, :, None] * p
    out[:, 1:, :] += ly[None, 1:, None] * p[:, :-1, :]
    out[:, :-1, :] += uy[None, :-1, None] * p[:, 1:, :]
    out += dzz[None, None, :] * p
    out[:, :, 1:] += lz[None, None, 1:] * p[:, :, :-1]
    out[:, :, :-1] += uz[None, None, :-1] * p[:, :, 1:]
    return out


@pytest.mark.parametrize("nx,ny,nz,grid_type", [(18, 17, 18, 2), (34, 21, 26, 1)])
def test_inflow_duct_solution_satisfies_the_discrete_problem(oracle_mod, nx, ny, nz, grid_type):
    """The duct with inflow/outflow x (the reference's CPU build): DCT-IV in x, z eigenmodes, one y solve per
    (kx, mode), no null mode (the outflow is Dirichlet), x normalised by 2 nxp; the planes i = nxg and k = nzg keep
    their input."""
    c = inflow_duct(nx, ny, nz, grid_type)
    o = oracle_mod.Oracle(c)
    N, Ny, Nz = nx - 1, ny - 1, nz - 1
    rhs = np.asfortranarray(np.random.default_rng(3).standard_normal((nx, ny - 1, nz)))
    phi = o.solve_poisson(rhs)
    res = inflow_duct_operator(o, phi[:N, :Ny, :Nz], o.grid_array(7)[0]) - rhs[:N, :Ny, :Nz]
    assert np.max(np.abs(res)) <= 1e-10 * np.max(np.abs(rhs)), np.max(np.abs(res))
    assert np.array_equal(phi[N], rhs[N])
    assert np.array_equal(phi[:, :, Nz], rhs[:, :, Nz])
    o.close()
