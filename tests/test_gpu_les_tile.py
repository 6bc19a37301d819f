"""LES stage kernels with the eddy viscosity computed in their tiles, through the C ABI.

The in-tile eddy viscosity evaluates compute_vreman's arithmetic on the same velocity the separate pass reads, so a
step with it (dfdm_set_sgs_in_tile, with the fused corrections it brings) must equal a step with the separate pass and
separate corrections up to the compiler's different contraction of the same expressions in another kernel (FP64
within 1e-13, FP32-mixed within 1e-6, its pressure within 1e-5, relative L2 after four steps; a read of a refilled
tile slot, found and fixed once, showed as 2e-7 and 7e-5); from one state the eddy viscosity itself is equal bit for bit; and both paths must
match the FP64 oracle (1e-12 FP64, 1e-5 FP32-mixed relative L2).  Cases: AMD and Vreman with the wall model,
the Re_tau 395 LES grid, and a triply periodic AMD case (wrapped halo rows).
"""
import numpy as np
import pytest

from conftest import rel_l2
from dfdm import cases
from dfdm.native import DfdmError, Solver

pytestmark = pytest.mark.gpu

TOL = {"fp64": 1e-12, "fp32": 1e-5}
SAME = {"fp64": 1e-13, "fp32": 1e-6}   # in-tile against separate pass: the rounding of two compilations


def _case(name):
    if name == "tgv_amd_small":
        return cases.tgv_small().with_(name="tgv_amd_small", sgs_model=2)
    return cases.get(name)


def _run(c, prec, n, tile, graphs=False):
    s = Solver(c, prec, graphs=graphs)
    if prec == "fp32":
        s.set_stage_variant(0)   # the separate pass's stage kernel with k_les's one-cell arithmetic
    s.set_sgs_in_tile(tile)
    assert s.sgs_in_tile() == tile
    s.set_state(*cases.initial_condition(c))
    s.compute_time_step_RK3(n)
    out = s.get_state(), s.get_nu_t(), s.fused_correction
    s.close()
    return out


@pytest.mark.parametrize("prec", ["fp64", "fp32"])
@pytest.mark.parametrize("name", ["chan_les_amd_small", "chan_les_vreman_small", "tgv_amd_small", "les395"])
def test_in_tile_eddy_viscosity_equals_the_separate_pass(name, prec):
    c = _case(name)
    n = 3 if name == "les395" else 4
    (a, nut_a, fused_a) = _run(c, prec, n, tile=True)
    (b, nut_b, fused_b) = _run(c, prec, n, tile=False)
    assert not fused_b
    for key, x, y in zip("UVWP", a, b):
        # FP32-mixed P = phi/(dt 3/4) amplifies velocity rounding by dx/dt (as between the FP32 stage variants)
        bar = 10 * SAME[prec] if (key == "P" and prec == "fp32") else SAME[prec]
        assert rel_l2(x, y) <= bar, (key, rel_l2(x, y))
    assert rel_l2(nut_a, nut_b) <= 100 * SAME[prec]
    assert nut_a.max() > 0


@pytest.mark.parametrize("prec", ["fp64", "fp32"])
@pytest.mark.parametrize("name", ["chan_les_amd_small", "tgv_amd_small", "les395"])
def test_in_tile_eddy_viscosity_equals_the_pass_from_one_state(name, prec):
    """From one state: the field the stage-3 kernel stores (its own tile's eddy viscosity) is the separate pass's,
    bit for bit."""
    c = _case(name)
    s = Solver(c, prec)
    s.set_sgs_in_tile(True)
    s.set_fused_correction(False)
    s.set_state(*cases.initial_condition(c))
    s.launch_kernel_async("stage", 3)
    s.synchronize()
    tile = s.get_nu_t()
    s.compute_sgs_model()
    assert np.array_equal(tile, s.get_nu_t())
    s.close()


@pytest.mark.parametrize("prec", ["fp64", "fp32"])
@pytest.mark.parametrize("name", ["chan_les_amd_small", "chan_les_vreman_small", "tgv_amd_small"])
def test_in_tile_eddy_viscosity_matches_the_oracle(oracle_mod, name, prec):
    c = _case(name)
    st = cases.initial_condition(c)
    o = oracle_mod.Oracle(c)
    o.set_state(*st)
    o.step(5)
    s = Solver(c, prec, graphs=True)
    s.set_sgs_in_tile(True)
    s.set_state(*st)
    s.compute_time_step_RK3(5)
    for key, x, y in zip("UVWP", s.get_state(), o.get_state()):
        assert rel_l2(x, y) <= TOL[prec], (key, rel_l2(x, y))
    # the stored field after the step is the stage-3 nu_t, as the oracle leaves it
    assert rel_l2(s.get_nu_t(), o.get_nu_t()) <= (1e-11 if prec == "fp64" else 1e-4)
    s.close()


def test_filtered_wall_model_les_takes_fused_corrections_with_the_tile_form():
    c = cases.les395()
    s = Solver(c, "fp32")
    assert not s.sgs_in_tile() and not s.fused_correction   # the separate pass is the default
    with pytest.raises(DfdmError) as e:
        s.set_fused_correction(True)
    assert e.value.code == 4
    s.set_sgs_in_tile(True)
    assert s.fused_correction
    s.set_sgs_in_tile(False)
    assert not s.fused_correction
    s.close()
    d = Solver(cases.chan_small(), "fp32")
    with pytest.raises(DfdmError) as e:
        d.set_sgs_in_tile(True)
    assert e.value.code == 4
    d.close()
