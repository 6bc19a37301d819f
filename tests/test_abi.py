"""CPU tests of the drop-in boundary: the C-ABI library loads, exports every symbol include/dfdm.h declares,
validates its inputs like the reference's input checks, and refuses to run without a GPU (no CPU fallback)."""
import ctypes
import os
import re

import numpy as np
import pytest

from conftest import ROOT, has_gpu
from dfdm import abi, cases, native


def header_symbols():
    text = open(os.path.join(ROOT, "include", "dfdm.h")).read()
    return sorted(set(re.findall(r"^\s*(?:int|void|const char \*)\s*(dfdm_\w+)\s*\(", text, re.M)))


def test_library_builds_and_exports_every_header_symbol():
    L = native.load()
    declared = header_symbols()
    assert declared, "no declarations parsed from include/dfdm.h"
    assert sorted(native.EXPORTS) == declared
    for name in declared:
        assert hasattr(L, name), name
    assert b"sm_100a" in L.dfdm_version()


def test_default_params_match_reference_defaults():
    L = native.load()
    p = abi.DfdmParams()
    L.dfdm_default_params(ctypes.byref(p))
    assert p.sgs_model == 2 and abs(p.Cs_vreman - 0.17) < 1e-15 and abs(p.C_amd - 1.0 / 3.0) < 1e-15
    assert p.adv_wall_layers == -1 and p.wm_filter_mode == -1 and p.flat_wall_model_flag == 0
    assert p.advection_scheme == 0 and p.adv_order == 3 and abs(p.adv_beta0 - 0.05) < 1e-15   # src/global.f90:71-72


@pytest.mark.parametrize("mutate,code,msg", [
    (dict(nx=17), 1, "even"),
    (dict(sgs_model=3), 1, "sgs_model"),
    (dict(advection_scheme=3), 1, "advection_scheme"),
    (dict(advection_scheme=2, adv_order=4), 1, "adv_order"),
    (dict(advection_scheme=2, adv_beta0=-1.0), 1, "adv_beta0"),
    (dict(flat_wall_model_flag=2), 4, "rough"),
    (dict(dt=0.0), 1, "dt"),
])
def test_invalid_inputs_are_rejected_with_the_reference_message(mutate, code, msg):
    c = cases.chan_small().with_(**mutate)
    with pytest.raises(native.DfdmError) as e:
        native.footprint_bytes(c)
    assert e.value.code == code and msg in str(e.value)


@pytest.mark.parametrize("case,code,msg", [
    (cases.inflow_outflow(260, 17, 18), 4, "at most 257 x cells"),
    (cases.inflow_outflow(18, 17, 18).with_(y_bc_type=0), 1, "requires x_bc_type=0"),
    (cases.duct(18, 17, 514), 4, "at most 512 z cells"),
    (cases.spanwise_wall(18, 18, 18).with_(x_bc_type=1), 4, "spanwise walls with inflow/outflow x"),
    (cases.duct(18, 17, 17), 1, "even"),
])
def test_poisson_only_grids_outside_the_built_paths_are_rejected(case, code, msg):
    """The inflow/outflow and duct pressure solves: their size limits and the boundary combinations the reference's
    GPU build rejects (src/initialization.f90:95-100), refused before any device work."""
    with pytest.raises(native.DfdmError) as e:
        native.footprint_bytes(case)
    assert e.value.code == code and msg in str(e.value)


def test_poisson_only_footprints_at_their_largest_sizes():
    for c in (cases.inflow_outflow(258, 129, 130), cases.duct(258, 129, 512), cases.duct(18, 17, 18),
              cases.spanwise_wall(130, 98, 130), cases.inflow_duct(258, 129, 512)):
        for prec in ("fp32", "fp64"):
            assert native.footprint_bytes(c, prec) > 0


def test_footprint_scales_with_precision():
    c = cases.chan550()
    b64 = native.footprint_bytes(c, "fp64")
    b32 = native.footprint_bytes(c, "fp32")
    # the fields and the spectrum halve in FP32; the FP64 pivot table and the FP64 host staging do not
    assert 1.75 < b64 / b32 < 2.0
    assert b32 < 2e9   # the 13M-cell throughput case fits easily in 180 GB


def test_every_config_has_supported_transform_lengths():
    for name in ("tgv64", "chan180", "les395", "chan550", "tgv_small", "chan_small", "chan_les_amd_small"):
        c = cases.get(name)
        assert native.footprint_bytes(c, "fp64") > 0


@pytest.mark.skipif(has_gpu(), reason="checks the no-GPU behaviour")
def test_no_cpu_fallback_without_gpu():
    with pytest.raises(native.DfdmError) as e:
        native.Solver(cases.chan_small())
    assert e.value.code == 2 and "no CPU fallback" in str(e.value)


def test_case_shapes_follow_the_reference_allocation():
    c = cases.chan550()
    s = c.shapes()
    assert s["U"] == (258, 194, 259) and s["V"] == (259, 193, 259) and s["W"] == (259, 194, 258)
    assert c.cells == (256, 192, 256) and c.n_cells == 12582912
    t = cases.tgv()
    assert t.cells == (64, 64, 64)
