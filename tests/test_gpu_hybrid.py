"""advection_scheme = 2 (upwind-biased dissipation, src/adv_hybrid.f90) on the device against the oracle.

The dissipative terms are computed by k_adv_hybrid_faces and added to the stage kernels' right-hand sides.  FP64 within
1e-12 relative L2 of the oracle (one RHS evaluation and three full steps); FP32-mixed within 1e-5 (both stage
kernels).  Orders 3 and 5, walls (with and without the LES wall model) and a fully periodic box.
"""
import numpy as np
import pytest

from conftest import rel_l2
from dfdm import cases
from dfdm.native import Solver

pytestmark = pytest.mark.gpu

NAMES = ["tgv_small", "chan_small", "chan_les_amd_small"]


def _case(name, order, beta=0.3):
    return cases.get(name).with_(advection_scheme=2, adv_order=order, adv_beta0=beta)


@pytest.mark.parametrize("order", [3, 5])
@pytest.mark.parametrize("name", NAMES)
def test_hybrid_rhs_matches_the_oracle(oracle_mod, name, order):
    c = _case(name, order)
    U, V, W, P = cases.initial_condition(c)
    o = oracle_mod.Oracle(c)
    o.set_state(U, V, W, P)
    s = Solver(c, "fp64")
    s.set_state(U, V, W, P)
    if c.sgs_model:
        o.compute_sgs_model()
        s.compute_sgs_model()
    if c.flat_wall_model_flag:
        o.compute_wall_model(True)
        s.compute_wall_model(True)
    Nx, Ny, Nz = c.cells
    nyv = Ny if c.y_bc_type == 0 else Ny - 1
    for a, b, (n1, n2, n3) in zip(s.compute_rhs(), o.compute_rhs(), [(Nx, Ny, Nz), (Nx, nyv, Nz), (Nx, Ny, Nz)]):
        assert rel_l2(a[:n1, :n2, :n3], b[:n1, :n2, :n3]) <= 1e-12
    s.close()


@pytest.mark.parametrize("prec,tol,variants", [("fp64", 1e-12, [None]), ("fp32", 1e-5, [0, 1])])
@pytest.mark.parametrize("order", [3, 5])
@pytest.mark.parametrize("name", NAMES)
def test_hybrid_steps_match_the_oracle(oracle_mod, name, order, prec, tol, variants):
    c = _case(name, order)
    U, V, W, P = cases.initial_condition(c)
    o = oracle_mod.Oracle(c)
    o.set_state(U, V, W, P)
    o.step(3)
    want = o.get_state()
    for v in variants:
        s = Solver(c, prec)
        if v is not None:
            s.set_stage_variant(v)
        s.set_state(U, V, W, P)
        s.compute_time_step_RK3(3)
        for key, a, b in zip("UVWP", s.get_state(), want):
            assert rel_l2(a, b) <= tol, (key, v, rel_l2(a, b))
        s.close()


def test_hybrid_dissipation_changes_the_solution(oracle_mod):
    """The scheme is not a no-op: three steps with beta = 0.3 differ from scheme 0 well above the parity bound."""
    c0 = cases.get("chan_small")
    st = cases.initial_condition(c0)
    out = []
    for c in (c0, _case("chan_small", 3)):
        s = Solver(c, "fp64")
        s.set_state(*st)
        s.compute_time_step_RK3(3)
        out.append(s.get_state()[0])
        s.close()
    assert rel_l2(out[1], out[0]) > 1e-8


def _odd(order):
    # two 32-cell x tiles and a partial y tile (72 x 9 x 12 cells), and a partial x and y tile with the wall model
    wide = cases.channel(72, 9, 12, 6.0, 1.5, 1.5, 180.0, 1.0, 2e-3, 32, 3, "chan_72x9x12")
    les = cases.Case(name="les_20x11x12", nx=22, ny=12, nz=14, Lx_i=3.0, Ly_i=2.0, Lz_i=1.5, grid_type=2,
                     alpha_grid=2.0, y_bc_type=1, nu=0.002531645569620253, dt=0.002, dPdx=1.0, sgs_model=2,
                     flat_wall_model_flag=1, ic="reichardt_gauss", ic_amplitude=1.0, noise=0.25, seed=33, nsteps=3)
    tgv = cases.tgv(12, Re=400.0, dt=2e-3, nsteps=3, name="tgv12")
    # Nx = 18 (not a multiple of 4: the FP32 loader copies x pairs instead of quads)
    ch = cases.channel(18, 13, 10, 3.0, 1.5, 2.0, 180.0, 1.0, 2e-3, 31, 3, "chan_18x13x10")
    return [c.with_(advection_scheme=2, adv_order=order, adv_beta0=0.3) for c in (wide, les, tgv, ch)]


@pytest.mark.parametrize("order", [3, 5])
def test_hybrid_odd_shapes_match_the_oracle(oracle_mod, order):
    """Partial x and y tiles, several x tiles, a periodic y of 12 rows and an Nx that is not a multiple of 4: the
    faces at tile edges (evaluated by the edge warps), the clamped rows next to the walls and both loader widths,
    3 steps in FP64 (1e-12) and FP32-mixed (1e-5)."""
    for c in _odd(order):
        U, V, W, P = cases.initial_condition(c)
        o = oracle_mod.Oracle(c)
        o.set_state(U, V, W, P)
        o.step(3)
        want = o.get_state()
        for prec, tol in (("fp64", 1e-12), ("fp32", 1e-5)):
            s = Solver(c, prec)
            s.set_state(U, V, W, P)
            s.compute_time_step_RK3(3)
            for key, a, b in zip("UVWP", s.get_state(), want):
                assert rel_l2(a, b) <= tol, (c.name, prec, key, rel_l2(a, b))
            s.close()
