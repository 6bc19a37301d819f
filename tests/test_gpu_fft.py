"""Poisson-solve parity at every transform length the kernels specialise, through the C ABI.

The two-level register transforms handle lengths 8 ... 256 with a split N1 x N2 (x half-lengths, z lengths and
periodic y lengths); other lengths (here 10, 36 and 80) go through the Stockham path.  Each case solves the
Poisson equation of a random divergence field on the GPU and in the FP64 oracle: FP64 within 1e-12 relative L2,
FP32-mixed within 1e-5.
"""
import math

import numpy as np
import pytest

from conftest import rel_l2
from dfdm import cases
from dfdm.native import Solver

pytestmark = pytest.mark.gpu

TWO_LEVEL = [8, 16, 24, 32, 48, 64, 96, 128, 192, 256]
STOCKHAM = [10, 36, 80]


def _case(Nx, Ny, Nz, yper):
    nx, Lx = cases._periodic(Nx, 2.0 * math.pi)
    nz, Lz = cases._periodic(Nz, math.pi)
    if yper:
        ny, Ly = cases._periodic(Ny, 2.0 * math.pi)
        return cases.Case(name=f"p{Nx}x{Ny}x{Nz}", nx=nx, ny=ny, nz=nz, Lx_i=Lx, Ly_i=Ly, Lz_i=Lz, grid_type=1,
                          y_bc_type=0, ic="zero")
    return cases.Case(name=f"w{Nx}x{Ny}x{Nz}", nx=nx, ny=Ny + 1, nz=nz, Lx_i=Lx, Ly_i=2.0, Lz_i=Lz, grid_type=2,
                      alpha_grid=1.5, y_bc_type=1, ic="zero")


def _random_state(c, seed):
    g = np.random.Generator(np.random.PCG64(seed))
    sh = c.shapes()
    U = np.asfortranarray(g.uniform(-1.0, 1.0, sh["U"]))
    V = np.asfortranarray(g.uniform(-1.0, 1.0, sh["V"]))
    W = np.asfortranarray(g.uniform(-1.0, 1.0, sh["W"]))
    cases.fill_ghosts(c, U, V, W)
    P = np.zeros(sh["P"], order="F")
    return U, V, W, P


def _check(oracle_mod, c, seed):
    state = _random_state(c, seed)
    o = oracle_mod.Oracle(c)
    o.set_state(*state)
    rhs = o.divergence_rhs()
    want = o.solve_poisson(rhs)
    Nx, Ny, Nz = c.cells
    for prec, tol in (("fp64", 1e-12), ("fp32", 1e-5)):
        s = Solver(c, prec)
        s.set_state(*state)
        got = s.solve_poisson_equation(rhs)
        err = rel_l2(got[:Nx, :Ny, :Nz], want[:Nx, :Ny, :Nz])
        assert err <= tol, (c.name, prec, err)


@pytest.mark.parametrize("n", TWO_LEVEL + STOCKHAM)
def test_poisson_x_and_z_lengths(oracle_mod, n):
    """x half-length n (Nx = 2n) and z length n, walls in y."""
    _check(oracle_mod, _case(2 * n, 8, n, yper=False), 100 + n)


@pytest.mark.parametrize("n", TWO_LEVEL + STOCKHAM)
def test_poisson_periodic_y_lengths(oracle_mod, n):
    """Periodic y of length n (the y transform, the k^2 division and the (0,0,0) pin)."""
    _check(oracle_mod, _case(16, n, 8, yper=True), 200 + n)


@pytest.mark.parametrize("n", TWO_LEVEL + STOCKHAM)
def test_projection_x_lengths(oracle_mod, n):
    """The projection (divergence fused with the forward x transform, the solve and the correction) at x
    half-length n, FP64 against the oracle."""
    c = _case(2 * n, 8, 16, yper=False)
    state = _random_state(c, 300 + n)
    o = oracle_mod.Oracle(c)
    o.set_state(*state)
    o.compute_projection_step(save_p=True)
    o.apply_boundary_conditions()
    s = Solver(c, "fp64")
    s.set_state(*state)
    s.compute_projection_step(save_p=True)
    for key, a, b in zip("UVW", s.get_state()[:3], o.get_state()[:3]):
        assert rel_l2(a, b) <= 1e-12, (n, key, rel_l2(a, b))
