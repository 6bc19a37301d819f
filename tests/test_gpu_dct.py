"""The DCT-IV pressure solve of an inflow/outflow-x grid (src/projection.f90:124-130,334-343) on the GPU against the
oracle: FP64 to 1e-12 and FP32-mixed to 1e-5 (relative L2), the planes the reference leaves alone returned as passed,
and every stepping entry point refusing the context."""
import numpy as np
import pytest

from dfdm.native import DfdmError, Solver

from test_oracle_dct import dct_case

pytestmark = pytest.mark.gpu

DFDM_ERR_UNSUPPORTED = 4


@pytest.fixture(scope="module")
def oracle_mod():
    import oracle
    oracle.build()
    return oracle


def rel_l2(a, b):
    return float(np.linalg.norm((a - b).ravel()) / np.linalg.norm(b.ravel()))


@pytest.mark.parametrize("prec,tol", [("fp64", 1e-12), ("fp32", 1e-5)])
@pytest.mark.parametrize("nx,ny,nz,grid_type", [(18, 17, 18, 2), (34, 21, 22, 1), (130, 65, 34, 2), (258, 33, 18, 1)])
def test_dct_poisson_matches_the_oracle(oracle_mod, prec, tol, nx, ny, nz, grid_type):
    c = dct_case(nx, ny, nz, grid_type)
    o = oracle_mod.Oracle(c)
    rng = np.random.default_rng(nx + ny)
    rhs = np.asfortranarray(rng.standard_normal((nx, ny - 1, nz)))
    want = o.solve_poisson(rhs)
    o.close()
    with Solver(c, prec) as s:
        got = s.solve_poisson_equation(rhs)
        again = s.solve_poisson_equation(rhs)
    N, nzp = nx - 1, nz - 2
    assert rel_l2(got[:N, :, :nzp], want[:N, :, :nzp]) <= tol
    assert np.array_equal(got[N], rhs[N])                   # x plane nxg: the caller's input
    assert np.array_equal(got[:N, :, nzp], got[:N, :, 0])   # periodic z copy
    assert np.array_equal(got[:N, :, nzp + 1], rhs[:N, :, nzp + 1])
    assert np.array_equal(got, again)


def test_dct_context_refuses_the_stepping_entry_points():
    c = dct_case()
    with Solver(c, "fp32") as s:
        sh = c.shapes()
        U, V, W, P = (np.zeros(sh[k], order="F") for k in "UVWP")
        with pytest.raises(DfdmError) as e:
            s.set_state(U, V, W, P)
        assert e.value.code == DFDM_ERR_UNSUPPORTED
        with pytest.raises(DfdmError) as e:
            s.compute_time_step_RK3(1)
        assert e.value.code == DFDM_ERR_UNSUPPORTED
        with pytest.raises(DfdmError) as e:
            s.solve_poisson_noalloc(np.zeros(sh["rhs_p"], order="F"))
        assert e.value.code == DFDM_ERR_UNSUPPORTED
        s.synchronize()
