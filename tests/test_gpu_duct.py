"""The 4-wall duct's pressure solve (z walls with y walls, periodic x; src/projection.f90:172-217) on the GPU against
the oracle: FP64 to 1e-12 and FP32-mixed to 1e-5 (relative L2), the x copy and the untouched z-wall plane as the
reference leaves them, and every stepping entry point refusing the context."""
import numpy as np
import pytest

from dfdm.native import DfdmError, Solver

from test_oracle_duct import duct_rhs
from dfdm.cases import duct

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
@pytest.mark.parametrize("nx,ny,nz,grid_type", [(18, 17, 18, 2), (34, 21, 26, 1), (66, 33, 40, 2), (130, 97, 130, 2)])
def test_duct_poisson_matches_the_oracle(oracle_mod, prec, tol, nx, ny, nz, grid_type):
    c = duct(nx, ny, nz, grid_type)
    o = oracle_mod.Oracle(c)
    rhs = duct_rhs(o, c, nx + nz)
    want = o.solve_poisson(rhs)
    o.close()
    with Solver(c, prec) as s:
        got = s.solve_poisson_equation(rhs)
        again = s.solve_poisson_equation(rhs)
    Nx, Nz = nx - 2, nz - 1
    assert rel_l2(got[:Nx, :, :Nz], want[:Nx, :, :Nz]) <= tol
    assert np.array_equal(got[Nx], got[0])                   # apply_periodic_xz_pressure's x copy
    assert np.array_equal(got[:Nx + 1, :, Nz], want[:Nx + 1, :, Nz])   # the plane nzg as the reference leaves it
    assert np.array_equal(got, again)


def test_duct_context_refuses_the_stepping_entry_points():
    c = duct()
    with Solver(c, "fp32") as s:
        sh = c.shapes()
        U, V, W, P = (np.zeros(sh[k], order="F") for k in "UVWP")
        with pytest.raises(DfdmError) as e:
            s.set_state(U, V, W, P)
        assert e.value.code == DFDM_ERR_UNSUPPORTED
        with pytest.raises(DfdmError) as e:
            s.compute_time_step_RK3(1)
        assert e.value.code == DFDM_ERR_UNSUPPORTED
        s.synchronize()


def test_duct_needs_periodic_x_and_y_walls():
    with pytest.raises(DfdmError) as e:
        Solver(duct().with_(x_bc_type=1), "fp32")
    assert e.value.code == DFDM_ERR_UNSUPPORTED
    with pytest.raises(DfdmError) as e:
        Solver(duct().with_(y_bc_type=0), "fp32")
    assert e.value.code == DFDM_ERR_UNSUPPORTED
