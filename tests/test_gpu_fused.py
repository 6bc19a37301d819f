"""Fused corrections: the projections of RK stages 1 and 2 applied inside the next stage kernel's loader.

The arithmetic is k_correct's, so a step with fused corrections must reproduce the separate-correction step bit for
bit, in FP64 and in FP32-mixed with either stage kernel, with and without the captured step graph.  Cases with an
hybrid scheme keeps the separate corrections (its dissipation kernel reads the corrected velocity), and so does an
LES whose eddy viscosity comes from the separate pass (the default); with it computed in the stage tiles LES fuses.
"""
import numpy as np
import pytest

from dfdm import cases
from dfdm.native import DfdmError, Solver

pytestmark = pytest.mark.gpu


def _run(c, prec, fused, steps=4, variant=None, graphs=False):
    s = Solver(c, prec)
    if variant is not None:
        s.set_stage_variant(variant)
    s.set_fused_correction(fused)
    s.enable_graphs(graphs)
    s.set_state(*cases.initial_condition(c))
    t = s.compute_time_step_RK3(steps)
    out = s.get_state()
    s.close()
    return t, out


@pytest.mark.parametrize("prec,variant", [("fp64", None), ("fp32", 0), ("fp32", 1)])
@pytest.mark.parametrize("name", ["tgv_small", "chan_small"])
def test_fused_step_equals_separate_corrections(name, prec, variant):
    c = cases.get(name)
    ta, a = _run(c, prec, False, variant=variant)
    tb, b = _run(c, prec, True, variant=variant)
    assert ta == tb
    for key, x, y in zip("UVWP", a, b):
        assert np.array_equal(x, y), (key, float(np.abs(x - y).max()))


@pytest.mark.parametrize("prec", ["fp64", "fp32"])
def test_fused_graph_replays_equal_plain_steps(prec):
    c = cases.get("chan_small")
    _, a = _run(c, prec, True, steps=5, graphs=False)
    _, b = _run(c, prec, True, steps=5, graphs=True)
    for x, y in zip(a, b):
        assert np.array_equal(x, y)


def test_fused_corrections_default_and_eligibility():
    s = Solver(cases.get("chan_small"), "fp32")
    assert s.fused_correction
    s.close()
    s = Solver(cases.get("chan_les_amd_small"), "fp32")   # LES with the filtered wall model
    assert not s.fused_correction                          # the eddy-viscosity pass reads the corrected U
    s.set_sgs_in_tile(True)
    assert s.fused_correction
    s.set_sgs_in_tile(False)
    assert not s.fused_correction
    with pytest.raises(DfdmError):
        s.set_fused_correction(True)
    s.close()
    s = Solver(cases.get("chan_small").with_(advection_scheme=2), "fp32")
    assert not s.fused_correction
    with pytest.raises(DfdmError):
        s.set_fused_correction(True)
    s.close()


@pytest.mark.parametrize("prec", ["fp64", "fp32"])
def test_fused_step_equals_separate_corrections_with_the_wall_model(prec):
    """DNS with the filtered wall model: the wall-model kernels read only the filter planes at stages 2 and 3, so
    the fused step is the separate-correction step bit for bit."""
    c = cases.get("chan_les_amd_small").with_(sgs_model=0, name="chan_wm_small")
    ta, a = _run(c, prec, False, variant=0 if prec == "fp32" else None)
    tb, b = _run(c, prec, True, variant=0 if prec == "fp32" else None)
    assert ta == tb
    for key, x, y in zip("UVWP", a, b):
        assert np.array_equal(x, y), (key, float(np.abs(x - y).max()))
