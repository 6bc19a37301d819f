"""dfdm_solve_poisson_noalloc against dfdm_solve_poisson and the FP64 oracle, both called through the C ABI.

The no-allocation variant stages through one library-wide device array that keeps the previous call's contents,
so it is checked on two calls in a row with different right-hand sides, on two contexts of different sizes that
share the array, against the oracle's solve, against the size limit, and for the property it exists for: a first
call on a fresh context leaves the device's free memory unchanged. Collected last (file name) so that it also runs
after every other GPU test in the same process.
"""
import numpy as np
import pytest

from conftest import rel_l2
from dfdm import cases
from dfdm.native import DfdmError, Solver

pytestmark = pytest.mark.gpu

TOL = {"fp64": 1e-12, "fp32": 1e-5}
MAX_POINTS = 2097152   # DFDM_NOALLOC_MAX_POINTS


def _rhs_pair(oracle_mod, c):
    """Two different divergence right-hand sides of the case's shape: the initial field's and a second one."""
    U, V, W, P = cases.initial_condition(c)
    o = oracle_mod.Oracle(c)
    o.set_state(U, V, W, P)
    a = o.divergence_rhs()
    o.set_state(0.5 * U[:, ::-1, :].copy(order="F"), V, 2.0 * W, P)
    b = o.divergence_rhs()
    assert rel_l2(a, b) > 0.1
    return (U, V, W, P), a, b


@pytest.mark.parametrize("precision", ["fp64", "fp32"])
def test_noalloc_matches_solve_poisson_twice_in_a_row(oracle_mod, precision):
    results = []
    for name in ("chan_small", "les395"):
        c = cases.get(name)
        state, a, b = _rhs_pair(oracle_mod, c)
        s = Solver(c, precision)
        s.set_state(*state)
        got = [s.solve_poisson_noalloc(a), s.solve_poisson_noalloc(b)]
        want = [s.solve_poisson_equation(a), s.solve_poisson_equation(b)]
        results.append((s, a, want[0]))
        for g, w in zip(got, want):
            assert g.shape == w.shape
            assert np.abs(w).max() > 0
            assert rel_l2(g, w) <= TOL[precision]
    # the first context again, after the second one has overwritten the shared array
    s, a, w = results[0]
    assert rel_l2(s.solve_poisson_noalloc(a), w) <= TOL[precision]


@pytest.mark.parametrize("precision", ["fp64", "fp32"])
@pytest.mark.parametrize("name", ["chan_small", "les395"])
def test_noalloc_matches_the_oracle(oracle_mod, name, precision):
    """solve_poisson_equation of the oracle (src/projection.f90:100-382) on the same right-hand side."""
    c = cases.get(name)
    state, a, b = _rhs_pair(oracle_mod, c)
    o = oracle_mod.Oracle(c)
    o.set_state(*state)
    s = Solver(c, precision)
    s.set_state(*state)
    Nx, Ny, Nz = c.cells
    for rhs in (a, b):
        got, want = s.solve_poisson_noalloc(rhs), o.solve_poisson(rhs)
        assert rel_l2(got[:Nx, :Ny, :Nz], want[:Nx, :Ny, :Nz]) <= TOL[precision]


def test_noalloc_first_call_allocates_no_device_memory(oracle_mod):
    """A context that has never solved a Poisson problem: its first no-allocation solve leaves cudaMemGetInfo's free
    bytes unchanged (dfdm_solve_poisson would allocate its staging buffer here)."""
    import torch
    c = cases.get("chan_small")
    state, a, _ = _rhs_pair(oracle_mod, c)
    s = Solver(c, "fp64")
    s.set_state(*state)
    s.synchronize()
    torch.cuda.synchronize()
    free0, _ = torch.cuda.mem_get_info()
    s.solve_poisson_noalloc(a)
    torch.cuda.synchronize()
    free1, _ = torch.cuda.mem_get_info()
    assert free1 == free0, (free0, free1)


def test_noalloc_rejects_sizes_beyond_the_limit():
    c = cases.get("chan550")
    shape = c.shapes()["rhs_p"]
    assert int(np.prod(shape)) > MAX_POINTS
    s = Solver(c, "fp32")
    rhs = np.zeros(shape, order="F")
    with pytest.raises(DfdmError) as e:
        s.solve_poisson_noalloc(rhs)
    assert e.value.code == 1 and "at most 2097152" in str(e.value)
