"""The packed FP32 stage kernel with TMA plane tiles (stage variant 2), through the C ABI.

Variant 2 evaluates the same packed FP32x2 arithmetic as variant 1; only the way the z-plane tiles reach shared
memory differs (3-D tensor boxes completing on mbarriers, zero-filled wall rows mirrored in a fix pass, x-wrap patch
boxes).  So its steps must equal variant 1's bit for bit, and both must match the FP64 oracle within the FP32-mixed
bar (1e-5 relative L2).  The grids cover one tile (Nx < 64: both x-wrap patches in one block), interior and edge
tiles in x, partial tiles in y, the fused correction and its absence, LES with the wall model, and the hybrid scheme.
"""
import numpy as np
import pytest

from conftest import rel_l2
from dfdm import cases
from dfdm.native import DfdmError, Solver

pytestmark = pytest.mark.gpu

TOL32 = 1e-5


def _wide_channel():
    """256 x 20 x 12 cells: four 64-wide tiles in x (two interior), three tile rows in y (the last partial)."""
    return cases.channel(256, 20, 12, 6.0, 1.5, 1.8, 180.0, 10.0, 1e-3, 7, 20, "chan_wide")


def _get(name):
    return _wide_channel() if name == "chan_wide" else cases.get(name)


def _run(c, variant, n, graphs=False, fused=None):
    s = Solver(c, "fp32", graphs=graphs)
    s.set_stage_variant(variant)
    if fused is not None:
        s.set_fused_correction(fused)
    s.set_state(*cases.initial_condition(c))
    s.compute_time_step_RK3(n)
    out = s.get_state()
    s.close()
    return out


@pytest.mark.parametrize("name", ["chan_small", "chan_les_amd_small", "chan_les_vreman_small", "chan_wide"])
def test_tma_stage_equals_the_cp_async_stage(name):
    c = _get(name)
    a = _run(c, 1, 4)
    b = _run(c, 2, 4)
    for key, x, y in zip("UVWP", a, b):
        assert np.array_equal(x, y), (key, rel_l2(y, x))


@pytest.mark.parametrize("fused", [True, False])
def test_tma_stage_with_and_without_fused_corrections(fused):
    c = _wide_channel()
    a = _run(c, 1, 3, fused=fused)
    b = _run(c, 2, 3, fused=fused)
    for key, x, y in zip("UVWP", a, b):
        assert np.array_equal(x, y), (key, rel_l2(y, x))


@pytest.mark.parametrize("name", ["chan_small", "chan_les_amd_small", "chan_wide"])
def test_tma_stage_matches_the_oracle(oracle_mod, name):
    c = _get(name)
    st = cases.initial_condition(c)
    o = oracle_mod.Oracle(c)
    o.set_state(*st)
    o.step(5)
    got = _run(c, 2, 5)
    for key, a, b in zip("UVWP", got, o.get_state()):
        assert rel_l2(a, b) <= TOL32, (key, rel_l2(a, b))


def test_tma_stage_unit_rhs_matches_the_oracle(oracle_mod):
    c = _wide_channel()
    st = cases.initial_condition(c)
    o = oracle_mod.Oracle(c)
    o.set_state(*st)
    s = Solver(c, "fp32")
    s.set_stage_variant(2)
    s.set_state(*st)
    Nx, Ny, Nz = c.cells
    lims = [(Nx, Ny, Nz), (Nx, Ny - 1, Nz), (Nx, Ny, Nz)]
    for a, b, (n1, n2, n3) in zip(s.compute_rhs(), o.compute_rhs(), lims):
        assert rel_l2(a[:n1, :n2, :n3], b[:n1, :n2, :n3]) <= TOL32


def test_tma_stage_hybrid_scheme_equals_cp_async():
    c = _wide_channel().with_(advection_scheme=2, adv_order=5)
    a = _run(c, 1, 3)
    b = _run(c, 2, 3)
    for key, x, y in zip("UVWP", a, b):
        assert np.array_equal(x, y), (key, rel_l2(y, x))


def test_tma_stage_graph_replays_equal_plain_launches():
    c = _wide_channel()
    a = _run(c, 2, 4)
    b = _run(c, 2, 4, graphs=True)
    for x, y in zip(a, b):
        assert np.array_equal(x, y)


@pytest.mark.parametrize("name,kw", [("tgv_small", {}), ("chan_small", {"nx": 20})])
def test_tma_stage_rejected_where_not_eligible(name, kw):
    """Periodic y, or Nx not a multiple of 4: the TMA variant is refused and the tuner never picks it."""
    c = cases.get(name).with_(**kw)
    s = Solver(c, "fp32")
    with pytest.raises(DfdmError) as e:
        s.set_stage_variant(2)
    assert e.value.code == 4
    assert s.stage_timing(2) == -1.0 and s.stage_variant()[0] in (0, 1)
    s.close()


def test_tuner_times_the_tma_variant():
    s = Solver(_wide_channel(), "fp32")
    assert s.stage_timing(2) > 0 and s.stage_timing(1) > 0 and s.stage_timing(0) > 0
    v = s.stage_variant()[0]
    assert s.stage_timing(v) == min(s.stage_timing(q) for q in (0, 1, 2))
    s.close()
