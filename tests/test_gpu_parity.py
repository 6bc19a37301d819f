"""GPU parity tests: every kernel family of the CUDA path, called through the C ABI, against the FP64 oracle.

Tolerances: plain FP64 form 1e-12 relative L2 (the target of the build); FP32-mixed form 1e-5 relative L2 against
the FP64 oracle; max |div u| after a projection 1e-12 relative to |u|/dy_min.
"""
import numpy as np
import pytest

from conftest import cfl_reference, interior, rel_l2
from dfdm import cases
from dfdm.native import Solver

pytestmark = pytest.mark.gpu

SMALL = ["tgv_small", "chan_small", "chan_les_amd_small", "chan_les_vreman_small"]
TOL64 = 1e-12
TOL32 = 1e-5


def _pair(oracle_mod, name, precision="fp64", **kw):
    c = cases.get(name, **kw) if kw else cases.get(name)
    U, V, W, P = cases.initial_condition(c)
    o = oracle_mod.Oracle(c)
    o.set_state(U, V, W, P)
    s = Solver(c, precision)
    s.set_state(U, V, W, P)
    return c, o, s


@pytest.mark.parametrize("name", SMALL)
def test_rhs_parity(oracle_mod, name):
    c, o, s = _pair(oracle_mod, name)
    if c.sgs_model:
        o.compute_sgs_model()
        s.compute_sgs_model()
    if c.flat_wall_model_flag:
        o.compute_wall_model(True)
        s.compute_wall_model(True)
    fo = o.compute_rhs()
    fg = s.compute_rhs()
    Nx, Ny, Nz = c.cells
    nyv = Ny if c.y_bc_type == 0 else Ny - 1
    lims = [(Nx, Ny, Nz), (Nx, nyv, Nz), (Nx, Ny, Nz)]
    for a, b, (n1, n2, n3) in zip(fg, fo, lims):
        assert rel_l2(a[:n1, :n2, :n3], b[:n1, :n2, :n3]) <= TOL64


@pytest.mark.parametrize("name", ["chan_les_amd_small", "chan_les_vreman_small"])
def test_sgs_parity(oracle_mod, name):
    c, o, s = _pair(oracle_mod, name)
    o.compute_sgs_model()
    s.compute_sgs_model()
    a, b = s.get_nu_t(), o.get_nu_t()
    assert b.max() > 0
    assert rel_l2(a, b) <= TOL64


def test_wall_model_parity(oracle_mod):
    c, o, s = _pair(oracle_mod, "chan_les_amd_small")
    for upd in (True, False, True):
        tx_o, tz_o = o.compute_wall_model(upd)
        tx_g, tz_g = s.compute_wall_model(upd)
        assert rel_l2(tx_g, tx_o) <= TOL64 and rel_l2(tz_g, tz_o) <= TOL64


@pytest.mark.parametrize("name", SMALL)
def test_poisson_parity(oracle_mod, name):
    c, o, s = _pair(oracle_mod, name)
    rhs = o.divergence_rhs()
    want = o.solve_poisson(rhs)
    got = s.solve_poisson_equation(rhs)
    Nx, Ny, Nz = c.cells
    assert rel_l2(got[:Nx, :Ny, :Nz], want[:Nx, :Ny, :Nz]) <= TOL64


@pytest.mark.parametrize("name", SMALL)
def test_projection_parity_and_divergence(oracle_mod, name):
    c, o, s = _pair(oracle_mod, name)
    o.compute_projection_step(save_p=True)
    o.apply_boundary_conditions()
    s.compute_projection_step(save_p=True)
    Uo, Vo, Wo, Po = o.get_state()
    Ug, Vg, Wg, Pg = s.get_state()
    for key, a, b in (("U", Ug, Uo), ("V", Vg, Vo), ("W", Wg, Wo)):
        assert rel_l2(interior(c, key, a), interior(c, key, b)) <= TOL64, key
    umax = max(np.abs(Ug).max(), np.abs(Vg).max(), np.abs(Wg).max())
    dymin = np.diff(cases.faces(c)[1]).min()
    assert s.check_divergence() <= 1e-12 * umax / dymin


@pytest.mark.parametrize("name", SMALL)
def test_full_step_parity_fp64(oracle_mod, name):
    c, o, s = _pair(oracle_mod, name)
    n = 5
    o.step(n)
    t = s.compute_time_step_RK3(n)
    assert abs(t - o.t) < 1e-14
    Uo, Vo, Wo, Po = o.get_state()
    Ug, Vg, Wg, Pg = s.get_state()
    for key, a, b in (("U", Ug, Uo), ("V", Vg, Vo), ("W", Wg, Wo), ("P", Pg, Po)):
        assert rel_l2(a, b) <= TOL64, (key, rel_l2(a, b))
    umax = max(np.abs(Ug).max(), np.abs(Vg).max(), np.abs(Wg).max())
    dymin = np.diff(cases.faces(c)[1]).min()
    assert s.check_divergence() <= 1e-12 * umax / dymin


@pytest.mark.parametrize("name", SMALL)
def test_full_step_parity_fp32_mixed(oracle_mod, name):
    c, o, s = _pair(oracle_mod, name, "fp32")
    n = 5
    o.step(n)
    s.compute_time_step_RK3(n)
    Uo, Vo, Wo, Po = o.get_state()
    Ug, Vg, Wg, Pg = s.get_state()
    for key, a, b in (("U", Ug, Uo), ("V", Vg, Vo), ("W", Wg, Wo), ("P", Pg, Po)):
        assert rel_l2(a, b) <= TOL32, (key, rel_l2(a, b))


@pytest.mark.parametrize("name", ["chan_small", "tgv_small"])
def test_fp32_mixed_100_steps_within_1e5(oracle_mod, name):
    """The FP32-mixed target: <= 1e-5 relative L2 of u, v, w and p against the FP64 oracle after 100 steps."""
    c, o, s = _pair(oracle_mod, name, "fp32")
    o.step(100)
    s.compute_time_step_RK3(100)
    for key, a, b in zip("UVWP", s.get_state(), o.get_state()):
        assert rel_l2(a, b) <= TOL32, (key, rel_l2(a, b))


def test_graphs_match_plain_launches(oracle_mod):
    c = cases.chan_les_amd_small()
    U, V, W, P = cases.initial_condition(c)
    a = Solver(c, "fp64")
    a.set_state(U, V, W, P)
    a.compute_time_step_RK3(4)
    b = Solver(c, "fp64", graphs=True)
    b.set_state(U, V, W, P)
    b.compute_time_step_RK3(4)
    for x, y in zip(a.get_state(), b.get_state()):
        assert np.array_equal(x, y)


def test_bulk_velocity_and_energy_diagnostics(oracle_mod):
    c, o, s = _pair(oracle_mod, "chan_small")
    assert abs(s.compute_bulk_velocity() - o.bulk_velocity()) <= 1e-13 * abs(o.bulk_velocity())
    assert abs(s.kinetic_energy() - o.kinetic_energy()) <= 1e-13 * o.kinetic_energy()
    s.check_finite()


def test_not_finite_guard(oracle_mod):
    c = cases.chan_small()
    U, V, W, P = cases.initial_condition(c)
    U[3, 4, 5] = np.nan
    s = Solver(c, "fp64")
    s.set_state(U, V, W, P)
    from dfdm.native import DfdmError
    with pytest.raises(DfdmError) as e:
        s.check_finite()
    assert e.value.code == 5


@pytest.mark.parametrize("name,prec,tol", [("chan_small", "fp64", 1e-13), ("chan_les_amd_small", "fp64", 1e-13),
                                           ("tgv_small", "fp64", 1e-13), ("chan_small", "fp32", 1e-6)])
def test_cfl_matches_the_reference_formula(name, prec, tol):
    c = cases.get(name)
    s = Solver(c, prec)
    s.set_state(*cases.initial_condition(c))
    s.compute_time_step_RK3(2)
    if c.sgs_model:
        s.compute_sgs_model()
    U, V, W, P = s.get_state()
    nut = s.get_nu_t() if c.sgs_model else np.zeros_like(P)
    want = cfl_reference(c, U, V, W, nut)
    got = s.compute_cfl()
    for g, w in zip(got, want):
        assert abs(g - w) <= tol * w, (got, want)


@pytest.mark.parametrize("variant", [0, 1])
@pytest.mark.parametrize("name", SMALL)
def test_fp32_stage_variants_match_the_oracle(oracle_mod, name, variant):
    """Both FP32 stage kernels (one cell per thread; packed FP32x2 pairs) against the FP64 oracle after 5 steps."""
    c, o, s = _pair(oracle_mod, name, "fp32")
    s.set_stage_variant(variant)
    assert s.stage_variant()[0] == variant
    o.step(5)
    s.compute_time_step_RK3(5)
    for key, a, b in zip("UVWP", s.get_state(), o.get_state()):
        assert rel_l2(a, b) <= TOL32, (key, rel_l2(a, b))


@pytest.mark.parametrize("name", ["chan_les_amd_small", "chan_les_vreman_small", "tgv_small", "chan_small"])
def test_fp32_stage_variants_agree(name):
    c = cases.get(name)
    state = cases.initial_condition(c)
    out = []
    for variant in (0, 1):
        s = Solver(c, "fp32", graphs=True)
        s.set_stage_variant(variant)
        s.set_state(*state)
        s.compute_time_step_RK3(20)
        out.append(s.get_state())
    for key, a, b in zip("UVWP", *out):   # the variants round differently in FP32; P amplifies that to ~2e-6
        assert rel_l2(a, b) <= TOL32, (key, rel_l2(a, b))


def test_stage_variant_tuning_is_reported():
    c = cases.chan_small()
    s = Solver(c, "fp32")
    v, ms0, ms1 = s.stage_variant()
    assert v in (0, 1) and ms0 > 0 and ms1 > 0 and (ms1 < ms0) == (v == 1)
    s.set_stage_variant(-1)
    assert s.stage_variant()[1] > 0
    d = Solver(c, "fp64")
    assert d.stage_variant() == (0, -1.0, -1.0)
    from dfdm.native import DfdmError
    with pytest.raises(DfdmError) as e:
        d.set_stage_variant(1)
    assert e.value.code == 4
