"""Adaptive time step (cfl_adaptive = 1) on the device, through the C ABI, against the oracle's select_dt.

Every step starts with the SGS eddy viscosity, the CFL maxima of the start-of-step velocity and
dt = max(dt_min, min(dt_max, dt * cfl_target / cfl * cfl_safety)) (src/monitor.f90:429-444,
src/time_integration.f90:146-160); dt and t stay on the device.  FP64: state within 1e-12 relative L2 and dt, t
within 1e-13 relative of the oracle's; FP32-mixed: 1e-5.
"""
import numpy as np
import pytest

from conftest import rel_l2
from dfdm import cases
from dfdm.native import DfdmError, Solver

pytestmark = pytest.mark.gpu

SMALL = ["tgv_small", "chan_small", "chan_les_amd_small"]


def _pair(oracle_mod, name, precision, target=0.5, safety=0.9, dt_min=1e-10, dt_max=1e10, graphs=False):
    c = cases.get(name)
    U, V, W, P = cases.initial_condition(c)
    o = oracle_mod.Oracle(c)
    o.set_state(U, V, W, P)
    o.set_adaptive_dt(True, target, safety, dt_min, dt_max)
    s = Solver(c, precision)
    s.set_state(U, V, W, P)
    s.enable_graphs(graphs)
    s.set_adaptive_dt(True, target, safety, dt_min, dt_max)
    return c, o, s


@pytest.mark.parametrize("prec,tol,ttol", [("fp64", 1e-12, 1e-13), ("fp32", 1e-5, 1e-5)])
@pytest.mark.parametrize("name", SMALL)
def test_adaptive_dt_matches_the_oracle(oracle_mod, name, prec, tol, ttol):
    c, o, s = _pair(oracle_mod, name, prec, target=0.6)
    for n in range(5):
        o.step(1)
        t = s.compute_time_step_RK3(1)
        assert abs(s.dt - o.dt) <= ttol * o.dt, (n, s.dt, o.dt)
        assert abs(t - o.t) <= ttol * o.t, (n, t, o.t)
        assert s.dt != c.dt
    for key, a, b in zip("UVWP", s.get_state(), o.get_state()):
        assert rel_l2(a, b) <= tol, (key, rel_l2(a, b))
    s.close()


@pytest.mark.parametrize("prec", ["fp64", "fp32"])
def test_adaptive_graph_replays_equal_plain_steps(oracle_mod, prec):
    """dt lives on the device, so the captured step replays the CFL, the dt choice and the step bit for bit."""
    name = "chan_les_amd_small"
    _, _, a = _pair(oracle_mod, name, prec, graphs=False)
    _, _, b = _pair(oracle_mod, name, prec, graphs=True)
    ta = a.compute_time_step_RK3(6)
    tb = b.compute_time_step_RK3(6)
    assert ta == tb and a.dt == b.dt
    for x, y in zip(a.get_state(), b.get_state()):
        assert np.array_equal(x, y)
    a.close()
    b.close()


def test_dt_max_clamps_and_disable_returns_to_the_fixed_dt(oracle_mod):
    c, o, s = _pair(oracle_mod, "tgv_small", "fp64", dt_max=1e-3)
    o.step(2)
    s.compute_time_step_RK3(2)
    assert s.dt == 1e-3 and o.dt == 1e-3
    o.set_adaptive_dt(False)
    s.set_adaptive_dt(False)
    assert s.dt == c.dt
    o.step(2)
    t = s.compute_time_step_RK3(2)
    assert abs(t - o.t) <= 1e-13 * o.t
    for key, x, y in zip("UVWP", s.get_state(), o.get_state()):
        assert rel_l2(x, y) <= 1e-12, key
    s.close()


def test_set_time_under_adaptive_dt():
    c = cases.get("chan_small")
    s = Solver(c, "fp64")
    s.set_state(*cases.initial_condition(c))
    s.set_adaptive_dt(True, 0.5, 0.9)
    s.set_time(5.0)
    assert s.t == 5.0
    t = s.compute_time_step_RK3(1)
    assert t == 5.0 + s.dt
    conv, visc = s.compute_cfl()
    assert conv > 0 and visc > 0
    s.close()


@pytest.mark.parametrize("args", [(0.0, 0.9, 1e-10, 1.0), (0.5, -1.0, 1e-10, 1.0), (0.5, 0.9, 0.0, 1.0),
                                  (0.5, 0.9, 1e-3, 1e-4)])
def test_adaptive_dt_rejects_bad_parameters(args):
    c = cases.get("chan_small")
    s = Solver(c, "fp64")
    with pytest.raises(DfdmError):
        s.set_adaptive_dt(True, *args)
    s.close()


@pytest.mark.parametrize("adaptive", [False, True])
def test_landing_matches_the_oracle(oracle_mod, adaptive):
    """Output landing (landing_dt) with the fixed and with the adaptive dt: the same times and states as the oracle;
    a new target between steps keeps the captured graph (graphs on)."""
    c = cases.get("chan_les_amd_small")
    U, V, W, P = cases.initial_condition(c)
    o = oracle_mod.Oracle(c)
    o.set_state(U, V, W, P)
    s = Solver(c, "fp64")
    s.set_state(U, V, W, P)
    s.enable_graphs(True)
    if adaptive:
        o.set_adaptive_dt(True, 0.6, 0.9)
        s.set_adaptive_dt(True, 0.6, 0.9)
    target = 3.7 * c.dt
    o.set_landing_time(target)
    s.set_landing_time(target)
    for n in range(8):
        if n == 5:
            target = o.t + 2.5 * c.dt
            o.set_landing_time(target)
            s.set_landing_time(target)
        o.step(1)
        t = s.compute_time_step_RK3(1)
        assert abs(t - o.t) <= 1e-13 * o.t, (n, t, o.t)
        assert abs(s.dt - o.dt) <= 1e-13 * o.dt, (n, s.dt, o.dt)
    assert abs(o.t - target) <= 1e-12 * target or o.t > target
    for key, a, b in zip("UVWP", s.get_state(), o.get_state()):
        assert rel_l2(a, b) <= 1e-12, (key, rel_l2(a, b))
    s.close()


@pytest.mark.parametrize("adaptive", [False, True])
def test_several_landing_targets_match_the_oracle(oracle_mod, adaptive):
    """select_dt with three time targets at once (full snapshots, slices, the end time), the targets moved on by
    the host output cadence (dfdm.output.OutputSchedule) after every step: the same times, dt and states as the
    oracle, with the step graph kept across new targets."""
    from dfdm.output import OutputSchedule
    c = cases.get("chan_les_amd_small")
    U, V, W, P = cases.initial_condition(c)
    o = oracle_mod.Oracle(c)
    o.set_state(U, V, W, P)
    s = Solver(c, "fp64")
    s.set_state(U, V, W, P)
    s.enable_graphs(True)
    if adaptive:
        o.set_adaptive_dt(True, 0.6, 0.9)
        s.set_adaptive_dt(True, 0.6, 0.9)

    def sched():
        return OutputSchedule(nsteps=-1, sim_end_time=11.3 * c.dt, nsave=-1, tsave=2.6 * c.dt, n_slices=1,
                              slice_freq=-1, slice_interval=3.7 * c.dt)
    so, ss = sched(), sched()
    istep = 0
    while True:
        istep += 1
        o.set_landing_times(so.targets())
        s.set_landing_times(ss.targets())
        o.step(1)
        t = s.compute_time_step_RK3(1)
        assert abs(t - o.t) <= 1e-13 * o.t, (istep, t, o.t)
        assert abs(s.dt - o.dt) <= 1e-13 * o.dt, (istep, s.dt, o.dt)
        assert ss.after_step(istep, t) == so.after_step(istep, o.t)
        if so.done(istep, o.t):
            assert ss.done(istep, t)
            break
        assert istep < 200
    assert abs(o.t - 11.3 * c.dt) <= 1e-12
    for key, a, b in zip("UVWP", s.get_state(), o.get_state()):
        assert rel_l2(a, b) <= 1e-12, (key, rel_l2(a, b))
    import ctypes
    from dfdm.native import load
    six = (ctypes.c_double * 6)(*([1.0] * 6))
    assert load().dfdm_set_landing_times(s.h, 6, six) != 0        # at most five targets
    inf = (ctypes.c_double * 1)(float("inf"))
    assert load().dfdm_set_landing_times(s.h, 1, inf) != 0        # NaN marks a free slot; inf is an error
    s.close()
