"""CPU tests of the FP64 oracle: third-party arithmetic against numpy/scipy, the reference's own regression
invariants, and analytic known answers (tests/regression/* hold no golden outputs for this path)."""
import math

import numpy as np
import pytest
import scipy.linalg.lapack as lapack

from conftest import cfl_reference, interior, rel_l2
from dfdm import cases


@pytest.mark.parametrize("n", [8, 15, 16, 24, 48, 64, 96, 128, 192, 256])
def test_fft_matches_numpy(oracle_mod, n):
    rng = np.random.default_rng(n)
    z = rng.standard_normal(n) + 1j * rng.standard_normal(n)
    f = oracle_mod.fft(z)
    assert np.max(np.abs(f - np.fft.fft(z))) <= 1e-13 * np.max(np.abs(np.fft.fft(z)))
    b = oracle_mod.fft(z, inverse=True)
    assert np.max(np.abs(b - np.fft.ifft(z) * n)) <= 1e-13 * n * np.max(np.abs(z))


def test_zgtsv_matches_lapack(oracle_mod):
    rng = np.random.default_rng(3)
    n = 40
    for trial in range(5):
        dl = rng.standard_normal(n - 1) + 0j
        du = rng.standard_normal(n - 1) + 0j
        d = rng.standard_normal(n) * (0.5 if trial % 2 else 4.0) + 0j   # odd trials force row interchanges
        b = rng.standard_normal(n) + 1j * rng.standard_normal(n)
        x, info = oracle_mod.zgtsv(dl, d, du, b)
        _, _, _, xs, infos = lapack.zgtsv(dl.copy(), d.copy(), du.copy(), b.copy())
        assert info == infos == 0
        assert np.max(np.abs(x - xs)) <= 1e-12 * np.max(np.abs(xs))


def _with_ic(oracle_mod, case):
    o = oracle_mod.Oracle(case)
    U, V, W, P = cases.initial_condition(case)
    o.set_state(U, V, W, P)
    return o


@pytest.mark.parametrize("name", ["tgv_small", "chan_small", "chan_les_amd_small"])
def test_projection_divergence_free(oracle_mod, name):
    """check_div.py bound of the reference's regressions (1e-9) -- and 1e-12 relative here."""
    c = cases.get(name)
    o = _with_ic(oracle_mod, c)
    o.compute_projection_step()
    o.apply_boundary_conditions()
    U, V, W, P = o.get_state()
    scale = max(np.abs(U).max(), np.abs(V).max(), np.abs(W).max()) / min(np.diff(cases.faces(c)[1]))
    assert o.max_divergence() <= 1e-12 * scale


def test_poisson_manufactured_mode(oracle_mod):
    """A single discrete eigenmode of the periodic x/z, wall-y Laplacian is recovered exactly."""
    c = cases.chan_small().with_(grid_type=2, alpha_grid=1.5)
    o = oracle_mod.Oracle(c)
    nxg, nyg, nzg = c.nxg, c.nyg, c.nzg
    Nx, Ny, Nz = c.cells
    kxx = o.grid_array(3)
    kzz = o.grid_array(4)
    y = cases.faces(c)[1]
    yg = o.grid_array(1)
    # y profile: any vector; build rhs = (Dyy + kxx(1) + kzz(2)) phi for phi = cos(2pi i/Nx) cos(4pi k/Nz) g(j)
    g = np.cos(np.linspace(0.3, 2.5, Ny))
    # Dyy applied to g, rows j=2..nyg-1 (reference indices), Neumann closure at both walls
    Dg = np.zeros(Ny)
    for r in range(Ny):
        j = r + 2
        a = 1.0 / (y[j - 1] - y[j - 2]) / (yg[j] - yg[j - 1])
        cc = 1.0 / (y[j - 1] - y[j - 2]) / (yg[j - 1] - yg[j - 2])
        val = 0.0
        if r + 1 < Ny:
            val += a * (g[r + 1] - g[r])
        if r - 1 >= 0:
            val += cc * (g[r - 1] - g[r])
        Dg[r] = val
    ii = np.arange(Nx)
    kk = np.arange(Nz)
    fx = np.cos(2 * np.pi * ii / Nx)
    fz = np.cos(4 * np.pi * kk / Nz)
    lam = kxx[1] + kzz[2]
    rhs = np.zeros((nxg - 1, nyg - 2, nzg - 1), order="F")
    core = fx[:, None, None] * (Dg + lam * g)[None, :, None] * fz[None, None, :]
    rhs[:Nx, :, :Nz] = core
    phi = o.solve_poisson(rhs)
    want = fx[:, None, None] * g[None, :, None] * fz[None, None, :]
    assert rel_l2(phi[:Nx, :, :Nz], want) <= 1e-12


def test_tgv_decay_matches_analytic(oracle_mod):
    """Viscous decay of the Taylor-Green vortex at early time: E(t)/E(0) = exp(-2 nu k_eff^2 t) with the
    second-order modified wavenumber; the nonlinear term is O(t^2) at this Reynolds number."""
    c = cases.tgv(N=16, Re=50.0, dt=2e-3)
    o = _with_ic(oracle_mod, c)
    e0 = o.kinetic_energy()
    o.step(20)
    t = o.t
    assert abs(t - 0.04) < 1e-14
    dx = 2 * np.pi / 16
    k2 = 3 * (2 - 2 * np.cos(dx)) / dx ** 2   # |k|^2 = 3 with the second-order modified wavenumber
    want = math.exp(-2 * (1.0 / 50.0) * k2 * t)
    assert abs(o.kinetic_energy() / e0 - want) < 2e-4


@pytest.mark.parametrize("name", ["chan_small", "tgv_small"])
def test_uniform_grid_never_pivots(oracle_mod, name):
    c = cases.get(name)
    o = _with_ic(oracle_mod, c)
    o.step(2)
    assert o.gtsv_swaps() == 0


def test_ghost_rules_are_the_reference_boundary_conditions(oracle_mod):
    """The Python IC ghost fill equals the oracle's apply_boundary_conditions (src/boundary_conditions.f90)."""
    for name in ("tgv_small", "chan_small"):
        c = cases.get(name)
        U, V, W, P = cases.initial_condition(c)
        o = oracle_mod.Oracle(c)
        o.set_state(U, V, W, P)
        o.apply_boundary_conditions()
        U2, V2, W2, _ = o.get_state()
        assert np.array_equal(U, U2) and np.array_equal(V, V2) and np.array_equal(W, W2)


def test_restart_equals_uninterrupted(oracle_mod):
    """restart_check.py of the reference: a run restarted from its snapshot equals the uninterrupted run
    (1e-12).  A DNS case: its restart state is U, V, W alone (src/input_output.f90:1225-1341)."""
    c = cases.chan_small()
    a = _with_ic(oracle_mod, c)
    a.step(6)
    Ua, Va, Wa, Pa = a.get_state()
    b = _with_ic(oracle_mod, c)
    b.step(3)
    snap = b.get_state()
    r = oracle_mod.Oracle(c)
    r.set_state(*snap)
    r.step(3)
    Ur, Vr, Wr, Pr = r.get_state()
    for x, y in ((Ur, Ua), (Vr, Va), (Wr, Wa), (Pr, Pa)):
        assert rel_l2(x, y) <= 1e-12


def test_constant_flux_holds_bulk_velocity(oracle_mod):
    c = cases.channel(16, 16, 16, 2 * np.pi, np.pi, 2.0, 180.0, 15.6, 1e-3, 7, 5, "cf")
    o = _with_ic(oracle_mod, c)
    o.step(3)
    assert abs(o.bulk_velocity() - 15.6) <= 1e-12 * 15.6


def test_golden_fixture_regression(oracle_mod):
    """Committed fixtures (tests/golden/make_golden.py) pin the oracle's outputs on the reference's three
    18x17x18 regression grids so that any change of the restatement is caught."""
    import os
    path = os.path.join(os.path.dirname(__file__), "golden", "oracle_small.npz")
    if not os.path.exists(path):
        pytest.skip("golden fixture not generated")
    data = np.load(path)
    for name in ("tgv_small", "chan_small", "chan_les_amd_small"):
        c = cases.get(name)
        o = _with_ic(oracle_mod, c)
        o.step(int(data[f"{name}_steps"]))
        U, V, W, P = o.get_state()
        for key, arr in (("U", U), ("V", V), ("W", W), ("P", P)):
            assert rel_l2(arr, data[f"{name}_{key}"]) <= 1e-13, (name, key)


@pytest.mark.parametrize("name", ["chan_small", "chan_les_amd_small", "tgv_small"])
def test_cfl_matches_the_formula(oracle_mod, name):
    """The oracle's compute_cfl against the numpy restatement of src/monitor.f90:304-424."""
    c = cases.get(name)
    o = _with_ic(oracle_mod, c)
    o.step(2)
    o.compute_sgs_model()
    U, V, W, P = o.get_state()
    nut = o.get_nu_t() if c.sgs_model else np.zeros_like(P)
    want = cfl_reference(c, U, V, W, nut)
    got = o.compute_cfl()
    for g, w in zip(got, want):
        assert abs(g - w) <= 1e-14 * w, (got, want)


@pytest.mark.parametrize("name,target,dt_max", [("chan_les_amd_small", 0.5, 1e10), ("chan_small", 0.8, 1e10),
                                                 ("tgv_small", 0.5, 1e-3)])
def test_adaptive_dt_follows_select_dt(oracle_mod, name, target, dt_max):
    """cfl_adaptive = 1: every step takes dt = max(dt_min, min(dt_max, dt*cfl_target/cfl*cfl_safety)) from the
    start-of-step CFL number, after nu_t (src/time_integration.f90:146-160, src/monitor.f90:429-444)."""
    c = cases.get(name)
    o = _with_ic(oracle_mod, c)
    o.set_adaptive_dt(True, target, 0.9, 1e-10, dt_max)
    dt = c.dt
    for _ in range(4):
        o.compute_sgs_model()
        U, V, W, P = o.get_state()
        nut = o.get_nu_t() if c.sgs_model else np.zeros_like(P)
        cfl = max(cfl_reference(c, U, V, W, nut, dt))
        want = max(1e-10, min(dt_max, dt * target / cfl * 0.9))
        t0 = o.t
        o.step(1)
        assert abs(o.dt - want) <= 1e-13 * want, (o.dt, want)
        assert abs(o.t - (t0 + want)) <= 1e-13 * (t0 + want)
        dt = want
    if dt_max < 1.0:
        assert o.dt == dt_max


def test_landing_dt_lands_on_the_target(oracle_mod):
    """landing_dt (src/monitor.f90:450-458): a remainder below 2 dt is one step, one between dt and 2 dt is two
    equal halves; dt is restored after the shrunk step (src/time_integration.f90:711)."""
    c = cases.get("chan_small")
    o = _with_ic(oracle_mod, c)
    dt = c.dt
    target = 3.7 * dt
    o.set_landing_time(target)
    ts = []
    for _ in range(5):
        o.step(1)
        ts.append(o.t)
        assert o.dt == dt
    # steps: dt, dt, then 1.7 dt is split in two halves 0.85 dt, then the target is reached and the rest are dt
    want = [dt, 2 * dt, 2 * dt + 0.85 * dt, target, target + dt]
    for got, w in zip(ts, want):
        assert abs(got - w) <= 1e-12 * target, (ts, want)


def test_output_monitor_restatement(oracle_mod):
    """The oracle's output_monitor values against numpy on its own state."""
    c = cases.get("chan_les_amd_small")
    o = _with_ic(oracle_mod, c)
    o.step(2)
    m = o.output_monitor()
    U, V, W, P = o.get_state()
    nx, nyg, nzg = c.nx, c.nyg, c.nzg
    assert m["max_u"] == np.abs(U[1:nx - 1, 1:nyg - 1, 1:nzg - 1]).max()
    assert m["mean_u"] == o.bulk_velocity() and m["max_div"] == o.max_divergence()
    assert (m["cfl_conv"], m["cfl_visc"]) == o.compute_cfl()
    assert m["t"] == o.t and m["dt"] == o.dt and m["nan_flag"] == 0.0
    assert 0.5 < m["u_tau_lo"] < 2.0 and 0.5 < m["u_tau_hi"] < 2.0


@pytest.mark.parametrize("order,factor,power", [(3, 4.0 / 3.0, 4), (5, 16.0 / 15.0, 6)])
def test_hybrid_dissipation_symbol(oracle_mod, order, factor, power):
    """advection_scheme = 2 (src/adv_hybrid.f90) on a pure x-mode W = a cos(theta (i-2)) convected by a uniform
    U = u0 > 0 (fully periodic box): the added rhs_w is the known symbol of the dissipation,
    -(4/3) beta u0/dx sin^4(theta/2) W for order 3 and -(16/15) beta u0/dx sin^6(theta/2) W for order 5."""
    base = cases.get("tgv_small")
    Nx = base.cells[0]
    theta, a, u0, beta = 2.0 * math.pi * 3 / Nx, 0.1, 1.0, 0.3
    U, V, W, P = (np.zeros(base.shapes()[k], order="F") for k in "UVWP")
    U[...] = u0
    i = np.arange(W.shape[0])
    W[...] = (a * np.cos(theta * (i - 1)))[:, None, None]   # 0-based index i is the reference's i+1
    out = {}
    for scheme in (0, 2):
        c = base.with_(advection_scheme=scheme, adv_order=order, adv_beta0=beta)
        o = oracle_mod.Oracle(c)
        o.set_state(U, V, W, P)
        out[scheme] = o.compute_rhs()[2]
    dw = out[2] - out[0]
    dx = (cases.faces(base)[0][1] - cases.faces(base)[0][0])
    iw = np.arange(dw.shape[0])   # rhs arrays start at the reference's i = 2
    want = -factor * beta * u0 / dx * math.sin(theta / 2) ** power * (a * np.cos(theta * iw))[:, None, None]
    want = np.broadcast_to(want, dw.shape)
    assert np.abs(dw - want).max() <= 1e-10 * np.abs(want).max()
    # beta = 0 is advection_scheme = 0 (the reference's statement, src/adv_hybrid.f90:4-5)
    c = base.with_(advection_scheme=2, adv_order=order, adv_beta0=0.0)
    o = oracle_mod.Oracle(c)
    o.set_state(U, V, W, P)
    assert np.array_equal(o.compute_rhs()[2], out[0])


@pytest.mark.parametrize("model", [1, 2])
def test_eddy_viscosity_of_a_two_component_shear(oracle_mod, model):
    """Known answer of compute_vreman (src/sgs_model.f90:118-216) for u = s*y, v = r*x on a uniform grid, where
    the only gradients are a21 = s and a12 = r:
      Vreman: B_beta = (dx*r)^2 (dy*s)^2, alpha^2 = s^2 + r^2, nu_t = 2.5 Cs^2 sqrt(B_beta / alpha^2);
      AMD: -beta:S = -(b12 (a12 + a21)) with b12 = dx^2 a11 a12 + dy^2 a21 a22 + dz^2 a31 a32 = 0, so nu_t = 0.
    A single shear (r = 0) gives B_beta = 0, so Vreman also vanishes there (its design property)."""
    c = cases.chan_small().with_(sgs_model=model, flat_wall_model_flag=0)
    x, y, z = cases.faces(c)
    xc, yc = cases.centres(x), cases.centres(y)
    dx, dy = x[1] - x[0], y[1] - y[0]
    for s, r in ((0.7, 0.3), (1.3, 0.0)):
        U, V, W, P = cases.allocate_state(c)
        U[:] = s * yc[None, :, None]           # U(i,j,k) sits at (x_i, yc_j, zc_k)
        V[:] = r * xc[:, None, None]           # V(i,j,k) sits at (xc_i, y_j, zc_k)
        o = oracle_mod.Oracle(c)
        o.set_state(U, V, W, P)
        o.compute_sgs_model()
        nut = o.get_nu_t()[2:-2, 2:-2, 2:-2]   # away from every ghost
        if model == 1:
            want = 2.5 * c.Cs_vreman ** 2 * math.sqrt((dx * r) ** 2 * (dy * s) ** 2 / (s * s + r * r))
        else:
            want = 0.0
        assert np.max(np.abs(nut - want)) <= 1e-13 * max(want, 1e-3), (model, s, r, nut.min(), nut.max(), want)
        o.close()
