"""Full RK3 steps on grids whose sizes leave partial tiles everywhere, against the oracle.

x and z lengths without a two-level split (Stockham transforms), Nx not a multiple of 4 (the scalar correction,
bulk-sum and CFL paths), Ny not a multiple of the 8-row tiles, and more than one 64-cell x tile of the packed stage
kernel with a partial last one.  FP64 within 1e-12 relative L2 of the oracle after 3 steps; FP32-mixed within 1e-5
with each stage kernel; the fused-correction step equal bit for bit to the separate-correction step.
"""
import numpy as np
import pytest

from conftest import rel_l2
from dfdm import cases
from dfdm.native import Solver

pytestmark = pytest.mark.gpu


def _odd_cases():
    ch = cases.channel(18, 13, 10, 3.0, 1.5, 2.0, 180.0, 1.0, 2e-3, 31, 3, "chan_18x13x10")   # Nx/2 = 9, Nz = 10
    wide = cases.channel(72, 9, 12, 6.0, 1.5, 1.5, 180.0, 1.0, 2e-3, 32, 3, "chan_72x9x12")   # two x tiles, Nx/2 = 36
    les = cases.Case(name="les_20x11x12", nx=22, ny=12, nz=14, Lx_i=3.0, Ly_i=2.0, Lz_i=1.5, grid_type=2,
                     alpha_grid=2.0, y_bc_type=1, nu=0.002531645569620253, dt=0.002, dPdx=1.0, sgs_model=2,
                     flat_wall_model_flag=1, ic="reichardt_gauss", ic_amplitude=1.0, noise=0.25, seed=33, nsteps=3)
    tgv = cases.tgv(12, Re=400.0, dt=2e-3, nsteps=3, name="tgv12")   # periodic y of length 12
    return [ch, wide, les, tgv]


CASES = _odd_cases()


def _run(c, prec, variant=None, fused=None, steps=3):
    s = Solver(c, prec)
    if variant is not None:
        s.set_stage_variant(variant)
    if fused is not None:
        s.set_fused_correction(fused)
    s.set_state(*cases.initial_condition(c))
    s.compute_time_step_RK3(steps)
    out = s.get_state()
    s.close()
    return out


@pytest.mark.parametrize("c", CASES, ids=[c.name for c in CASES])
def test_odd_shapes_match_the_oracle(oracle_mod, c):
    o = oracle_mod.Oracle(c)
    o.set_state(*cases.initial_condition(c))
    o.step(3)
    want = o.get_state()
    for key, a, b in zip("UVWP", _run(c, "fp64"), want):
        assert rel_l2(a, b) <= 1e-12, ("fp64", key, rel_l2(a, b))
    for v in (0, 1):
        for key, a, b in zip("UVWP", _run(c, "fp32", variant=v), want):
            assert rel_l2(a, b) <= 1e-5, ("fp32", v, key, rel_l2(a, b))


@pytest.mark.parametrize("c", [c for c in CASES if c.sgs_model == 0], ids=[c.name for c in CASES if c.sgs_model == 0])
def test_odd_shapes_fused_equals_separate(c):
    for prec, variants in (("fp64", [None]), ("fp32", [0, 1])):
        for v in variants:
            a = _run(c, prec, variant=v, fused=False)
            b = _run(c, prec, variant=v, fused=True)
            for key, x, y in zip("UVWP", a, b):
                assert np.array_equal(x, y), (prec, v, key, float(np.abs(x - y).max()))


def test_a_later_context_of_a_smaller_grid_leaves_earlier_launches_valid():
    """Kernels whose shared memory depends on the grid (the staged y solve, the Stockham transforms) keep their
    dynamic shared-memory cap at the device maximum: a context created later, on a smaller grid, must not lower it
    under an earlier context's launches and captured graphs."""
    import math
    big = cases.channel(32, 128, 32, 2 * math.pi, math.pi, 2.0, 180.0, 15.6, 1e-3, 7, 0, "chan_ny128")
    small = cases.channel(32, 24, 32, 2 * math.pi, math.pi, 2.0, 180.0, 15.6, 1e-3, 8, 0, "chan_ny24")
    ref = _run(big, "fp32", steps=2)
    for graphs in (False, True):
        s1 = Solver(big, "fp32", graphs=graphs)
        s1.set_state(*cases.initial_condition(big))
        s1.compute_time_step_RK3(1)
        s2 = Solver(small, "fp32")
        s2.set_state(*cases.initial_condition(small))
        s2.compute_time_step_RK3(1)
        s1.compute_time_step_RK3(1)
        for x, y in zip(s1.get_state(), ref):
            assert np.array_equal(x, y)
        s1.close()
        s2.close()
