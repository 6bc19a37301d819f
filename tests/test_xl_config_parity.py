"""Oracle parity at the benchmark configurations' full sizes and step counts, through the C ABI.

Each configuration is stepped by the FP64 oracle and by the library from the same initial condition with the same
dt, and u, v, w and p are compared after the configuration's own step count:
  Taylor-Green 64^3, 100 steps; channel Re_tau 180 (128 x 96 x 128), 200 steps; wall-modelled AMD LES Re_tau 395
  (96 x 64 x 96), 500 steps; channel Re_tau 550 (256 x 192 x 256), 20 warm-up + 100 timed steps = 120 steps.
Bars: the plain FP64 form within 1e-12 relative L2 of the oracle, with max |div u| <= 1e-12 |u|_max / dy_min after
the final projection; the FP32-mixed form within 1e-5 relative L2 of the oracle.

The oracle runs once per configuration (OpenMP on every host core) and both precisions compare against that run.
The Re_tau 550 oracle takes about five minutes on 16 cores, so these tests are also marked `slow`.
"""
import numpy as np
import pytest

from conftest import rel_l2
from dfdm import cases
from dfdm.native import Solver

pytestmark = [pytest.mark.gpu, pytest.mark.slow]

TOL64 = 1e-12
TOL32 = 1e-5
STEPS = {"tgv64": 100, "chan180": 200, "les395": 500, "chan550": 120}

_ORACLE = {}


def _oracle_run(oracle_mod, name):
    """(case, initial state, oracle final state, oracle t) for one configuration, computed once per session."""
    if name not in _ORACLE:
        _ORACLE.clear()          # keep one configuration's arrays at a time (chan550: ~0.4 GB per state)
        c = cases.get(name)
        state = cases.initial_condition(c)
        o = oracle_mod.Oracle(c)
        o.set_state(*state)
        o.step(STEPS[name])
        _ORACLE[name] = (c, state, o.get_state(), o.t)
        o.close()
    return _ORACLE[name]


def _gpu_run(c, state, precision, n):
    s = Solver(c, precision, graphs=True)
    s.set_state(*state)
    t = s.compute_time_step_RK3(n)
    out = s.get_state()
    div = s.check_divergence()
    s.close()
    return out, t, div


CASES = [(name, prec) for name in ("tgv64", "chan180", "les395", "chan550") for prec in ("fp64", "fp32")]


@pytest.mark.parametrize("name,precision", CASES)
def test_config_parity_against_the_oracle(oracle_mod, name, precision):
    c, state, want, t_oracle = _oracle_run(oracle_mod, name)
    got, t, div = _gpu_run(c, state, precision, STEPS[name])
    assert abs(t - t_oracle) <= 1e-12 * max(1.0, abs(t_oracle))
    errs = {key: rel_l2(a, b) for key, a, b in zip("UVWP", got, want)}
    print(f"{name} {precision} after {STEPS[name]} steps: rel L2 vs oracle " +
          " ".join(f"{k} {v:.3e}" for k, v in errs.items()))
    tol = TOL64 if precision == "fp64" else TOL32
    for key, e in errs.items():
        assert e <= tol, (name, precision, key, e)
    if precision == "fp64":
        umax = max(float(np.abs(a).max()) for a in got[:3])
        dymin = float(np.diff(cases.faces(c)[1]).min())
        assert div <= 1e-12 * umax / dymin, (div, umax / dymin)
