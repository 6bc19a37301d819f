"""output_monitor on the device (dfdm_output_monitor) against the oracle's restatement of src/monitor.f90:21-102.

FP64: t, dt, mean U, max |U|, the CFL numbers and the mean wall u_tau within 1e-12 relative of the oracle's; the
divergence is rounding-level in both, so it is checked against the projection bound 1e-12 |u|/dy_min.  FP32-mixed:
1e-5.  The asynchronous form writes the same ten values into device memory.
"""
import numpy as np
import pytest

from conftest import rel_l2
from dfdm import cases
from dfdm.native import DfdmError, Solver

pytestmark = pytest.mark.gpu

SMALL = ["tgv_small", "chan_small", "chan_les_amd_small"]
KEYS = ("t", "dt", "mean_u", "max_u", "cfl_conv", "cfl_visc", "u_tau_lo", "u_tau_hi")


def _pair(oracle_mod, name, prec, steps):
    c = cases.get(name)
    U, V, W, P = cases.initial_condition(c)
    o = oracle_mod.Oracle(c)
    o.set_state(U, V, W, P)
    s = Solver(c, prec)
    s.set_state(U, V, W, P)
    o.step(steps)
    s.compute_time_step_RK3(steps)
    if c.sgs_model:   # nu_t of the current state in both (the viscous CFL reads it)
        o.compute_sgs_model()
        s.compute_sgs_model()
    return c, o, s


@pytest.mark.parametrize("prec,tol", [("fp64", 1e-12), ("fp32", 1e-5)])
@pytest.mark.parametrize("name", SMALL)
def test_monitor_matches_the_oracle(oracle_mod, name, prec, tol):
    c, o, s = _pair(oracle_mod, name, prec, 3)
    got, want = s.output_monitor(), o.output_monitor()
    for key in KEYS:   # the mean of a periodic TGV field is rounding-level: scaled by max |U|
        scale = max(abs(want[key]), want["max_u"] if key == "mean_u" else 0.0, 1e-300)
        assert abs(got[key] - want[key]) <= tol * scale, (key, got[key], want[key])
    if c.flat_wall_model_flag:
        assert got["u_tau_lo"] > 0 and got["u_tau_hi"] > 0
    else:
        assert got["u_tau_lo"] == 0.0 and got["u_tau_hi"] == 0.0
    umax = max(np.abs(a).max() for a in s.get_state()[:3])
    dymin = np.diff(cases.faces(c)[1]).min()
    assert got["max_div"] <= 1e-12 * umax / dymin if prec == "fp64" else got["max_div"] <= 1e-4 * umax / dymin
    assert got["max_div"] == s.check_divergence()
    assert got["nan_flag"] == 0.0
    s.close()


def test_monitor_async_writes_device_memory(oracle_mod):
    import torch
    c, o, s = _pair(oracle_mod, "chan_les_amd_small", "fp64", 2)
    want = s.output_monitor()
    buf = torch.zeros(10, dtype=torch.float64, device="cuda")
    s.output_monitor_async(buf.data_ptr())
    s.synchronize()
    got = dict(zip(Solver.MONITOR_KEYS, buf.cpu().tolist()))
    assert got == want
    s.close()


def test_monitor_under_adaptive_dt(oracle_mod):
    c = cases.get("chan_small")
    U, V, W, P = cases.initial_condition(c)
    o = oracle_mod.Oracle(c)
    o.set_state(U, V, W, P)
    o.set_adaptive_dt(True, 0.5, 0.9)
    s = Solver(c, "fp64")
    s.set_state(U, V, W, P)
    s.set_adaptive_dt(True, 0.5, 0.9)
    o.step(3)
    s.compute_time_step_RK3(3)
    got, want = s.output_monitor(), o.output_monitor()
    for key in KEYS:
        assert abs(got[key] - want[key]) <= 1e-12 * max(abs(want[key]), 1e-300), (key, got[key], want[key])
    assert got["dt"] == s.dt and got["t"] == s.t
    s.close()


def test_monitor_guard():
    c = cases.chan_small()
    U, V, W, P = cases.initial_condition(c)
    W[5, 6, 7] = 2e8
    s = Solver(c, "fp64")
    s.set_state(U, V, W, P)
    with pytest.raises(DfdmError) as e:
        s.output_monitor()
    assert e.value.code == 5
    s.close()
