"""advection_scheme = 2 (upwind-biased dissipation, src/adv_hybrid.f90) on the device against the oracle.

The dissipative terms are computed by k_adv_hybrid and added to the stage kernels' right-hand sides.  FP64 within
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
