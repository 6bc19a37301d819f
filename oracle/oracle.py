"""ctypes wrapper of the CPU FP64 oracle (TEST INFRASTRUCTURE ONLY).

Loads oracle/liboracle.so (built by oracle/Makefile from dfdm_oracle.cpp).  Only tests/, __graft_entry__.smoke()
and bench.py's CPU-baseline leg use this module; the product library never imports it.  See the header of
dfdm_oracle.cpp for the reference files it restates and for its parity status.
"""
from __future__ import annotations

import ctypes
import os
import subprocess
import sys
from ctypes import POINTER, c_double, c_int, c_long, c_void_p

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_PKG = os.path.join(os.path.dirname(_HERE), "dopamine-fdm_b200")
if _PKG not in sys.path:
    sys.path.insert(0, _PKG)

from dfdm.abi import DfdmGrid, DfdmParams, GridHolder, dptr, make_params  # noqa: E402
from dfdm.cases import Case  # noqa: E402

LIB_PATH = os.path.join(_HERE, "liboracle.so")
_lib = None


def build(force: bool = False) -> str:
    """Compile liboracle.so with the Makefile next to this file."""
    src = os.path.join(_HERE, "dfdm_oracle.cpp")
    if force or not os.path.exists(LIB_PATH) or os.path.getmtime(LIB_PATH) < os.path.getmtime(src):
        subprocess.run(["make", "-s", "-C", _HERE], check=True)
    return LIB_PATH


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            build()
        L = ctypes.CDLL(LIB_PATH)
        L.orc_create.restype = c_void_p
        L.orc_create.argtypes = [POINTER(DfdmGrid), POINTER(DfdmParams)]
        L.orc_destroy.argtypes = [c_void_p]
        for name in ("orc_set_state", "orc_get_state"):
            getattr(L, name).argtypes = [c_void_p] + [POINTER(c_double)] * 4
        for name in ("orc_get_nu_t", "orc_set_nu_t", "orc_divergence_rhs"):
            getattr(L, name).argtypes = [c_void_p, POINTER(c_double)]
        L.orc_apply_bc.argtypes = [c_void_p]
        L.orc_step.argtypes = [c_void_p, c_int]
        L.orc_time.restype = c_double
        L.orc_time.argtypes = [c_void_p]
        L.orc_compute_sgs.argtypes = [c_void_p]
        L.orc_wall_model.argtypes = [c_void_p, c_int, POINTER(c_double), POINTER(c_double)]
        L.orc_compute_rhs.argtypes = [c_void_p] + [POINTER(c_double)] * 3
        L.orc_solve_poisson.restype = c_int
        L.orc_solve_poisson.argtypes = [c_void_p, POINTER(c_double)]
        L.orc_projection.argtypes = [c_void_p, c_int]
        for name in ("orc_bulk_velocity", "orc_max_divergence", "orc_kinetic_energy"):
            getattr(L, name).restype = c_double
            getattr(L, name).argtypes = [c_void_p]
        L.orc_gtsv_swaps.restype = c_long
        L.orc_gtsv_swaps.argtypes = [c_void_p]
        L.orc_grid_array.restype = c_int
        L.orc_grid_array.argtypes = [c_void_p, c_int, POINTER(c_double)]
        L.orc_dct4.restype = c_int
        L.orc_dct4.argtypes = [c_void_p, POINTER(c_double), POINTER(c_double)]
        L.orc_fft.argtypes = [c_int, POINTER(c_double), c_int]
        L.orc_zgtsv.restype = c_int
        L.orc_zgtsv.argtypes = [c_int] + [POINTER(c_double)] * 4
        L.orc_dt.restype = c_double
        L.orc_dt.argtypes = [c_void_p]
        L.orc_set_adaptive.argtypes = [c_void_p, c_int, c_double, c_double, c_double, c_double]
        L.orc_cfl.argtypes = [c_void_p, POINTER(c_double), POINTER(c_double)]
        L.orc_set_landing.argtypes = [c_void_p, c_double]
        L.orc_set_landings.argtypes = [c_void_p, c_int, POINTER(c_double)]
        L.orc_output_monitor.argtypes = [c_void_p, POINTER(c_double)]
        L.orc_set_threads.argtypes = [c_int]
        L.orc_get_threads.restype = c_int
        _lib = L
    return _lib


def set_threads(n: int) -> None:
    lib().orc_set_threads(int(n))


def get_threads() -> int:
    return int(lib().orc_get_threads())


class Oracle:
    """One case held by the CPU restatement; arrays in and out are Fortran-ordered ghosted float64 arrays."""

    def __init__(self, case: Case):
        self.case = case
        self._g = GridHolder(case)
        self._p = make_params(case)
        self.h = lib().orc_create(ctypes.byref(self._g.grid), ctypes.byref(self._p))
        self.shapes = case.shapes()

    def close(self):
        if self.h:
            lib().orc_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _arr(self, key):
        return np.zeros(self.shapes[key], order="F")

    def set_state(self, U, V, W, P=None):
        f = lambda a: None if a is None else np.asfortranarray(a, dtype=np.float64)
        U, V, W, P = f(U), f(V), f(W), f(P)
        lib().orc_set_state(self.h, dptr(U), dptr(V), dptr(W), dptr(P))

    def get_state(self):
        U, V, W, P = self._arr("U"), self._arr("V"), self._arr("W"), self._arr("P")
        lib().orc_get_state(self.h, dptr(U), dptr(V), dptr(W), dptr(P))
        return U, V, W, P

    def get_nu_t(self):
        a = self._arr("P")
        lib().orc_get_nu_t(self.h, dptr(a))
        return a

    def set_nu_t(self, a):
        a = np.asfortranarray(a, dtype=np.float64)
        lib().orc_set_nu_t(self.h, dptr(a))

    def apply_boundary_conditions(self):
        lib().orc_apply_bc(self.h)

    def step(self, n: int = 1):
        lib().orc_step(self.h, int(n))

    @property
    def t(self) -> float:
        return float(lib().orc_time(self.h))

    @property
    def dt(self) -> float:
        return float(lib().orc_dt(self.h))

    def set_adaptive_dt(self, enable=True, cfl_target=0.5, cfl_safety=0.9, dt_min=1e-10, dt_max=1e10):
        """cfl_adaptive = 1: dt from the CFL number at every step start (select_dt, src/monitor.f90:429)."""
        lib().orc_set_adaptive(self.h, int(enable), cfl_target, cfl_safety, dt_min, dt_max)

    def set_landing_time(self, t_land=None):
        """Shrink the coming steps so that t lands on t_land (landing_dt, src/monitor.f90:436-458); None: no target."""
        lib().orc_set_landing(self.h, float("nan") if t_land is None else float(t_land))

    def set_landing_times(self, targets=()):
        """Up to five landing targets in select_dt's order (tsave_next, chunk_tsave_next, slice_tnext, line_tnext,
        sim_end_time; src/monitor.f90:436-440), each applied in turn; None entries are slots without a target."""
        vals = [float("nan") if v is None else float(v) for v in targets]
        if len(vals) > 5:
            raise ValueError("at most five landing targets")
        arr = (c_double * max(1, len(vals)))(*vals)
        lib().orc_set_landings(self.h, len(vals), arr)

    MONITOR_KEYS = ("t", "dt", "mean_u", "max_u", "max_div", "cfl_conv", "cfl_visc", "u_tau_lo", "u_tau_hi", "nan_flag")

    def output_monitor(self) -> dict:
        """The values output_monitor prints (src/monitor.f90:21-102), CFL numbers of the current state."""
        out = np.zeros(10)
        lib().orc_output_monitor(self.h, dptr(out))
        return dict(zip(self.MONITOR_KEYS, out.tolist()))

    def compute_cfl(self):
        a, b = c_double(0.0), c_double(0.0)
        lib().orc_cfl(self.h, ctypes.byref(a), ctypes.byref(b))
        return a.value, b.value

    def compute_sgs_model(self):
        lib().orc_compute_sgs(self.h)

    def compute_wall_model(self, update_filter: bool = True):
        tx, tz = self._arr("tau_x"), self._arr("tau_z")
        lib().orc_wall_model(self.h, int(update_filter), dptr(tx), dptr(tz))
        return tx, tz

    def compute_rhs(self):
        fu, fv, fw = self._arr("rhs_u"), self._arr("rhs_v"), self._arr("rhs_w")
        lib().orc_compute_rhs(self.h, dptr(fu), dptr(fv), dptr(fw))
        return fu, fv, fw

    def divergence_rhs(self):
        a = self._arr("rhs_p")
        lib().orc_divergence_rhs(self.h, dptr(a))
        return a

    def solve_poisson(self, rhs_p):
        a = np.array(rhs_p, dtype=np.float64, order="F", copy=True)
        info = lib().orc_solve_poisson(self.h, dptr(a))
        if info != 0:
            raise RuntimeError(f"oracle zgtsv reported a singular pivot (info={info})")
        return a

    def compute_projection_step(self, save_p: bool = False):
        lib().orc_projection(self.h, int(save_p))

    def bulk_velocity(self) -> float:
        return float(lib().orc_bulk_velocity(self.h))

    def max_divergence(self) -> float:
        return float(lib().orc_max_divergence(self.h))

    def kinetic_energy(self) -> float:
        return float(lib().orc_kinetic_energy(self.h))

    def gtsv_swaps(self) -> int:
        return int(lib().orc_gtsv_swaps(self.h))

    def dct4(self, line) -> np.ndarray:
        """The DCT-IV of one x line (inflow/outflow x only): 2 sum_n x_n cos(pi (2n+1)(2k+1) / (4N))."""
        a = np.ascontiguousarray(line, dtype=np.float64)
        out = np.zeros_like(a)
        n = lib().orc_dct4(self.h, dptr(a), dptr(out))
        if n != a.size:
            raise ValueError("the oracle's DCT-IV needs an inflow/outflow-x case of the line's length")
        return out

    def grid_array(self, which: int) -> np.ndarray:
        out = np.zeros(max(self.case.nx, self.case.ny, self.case.nz) + 8)
        n = lib().orc_grid_array(self.h, int(which), dptr(out))
        return out[:n].copy()


def fft(a: np.ndarray, inverse: bool = False) -> np.ndarray:
    z = np.array(a, dtype=np.complex128, copy=True)
    lib().orc_fft(z.size, z.ctypes.data_as(POINTER(c_double)), int(inverse))
    return z


def zgtsv(dl, d, du, b):
    dl = np.array(dl, dtype=np.complex128, copy=True)
    d = np.array(d, dtype=np.complex128, copy=True)
    du = np.array(du, dtype=np.complex128, copy=True)
    b = np.array(b, dtype=np.complex128, copy=True)
    p = lambda z: z.ctypes.data_as(POINTER(c_double))
    info = lib().orc_zgtsv(b.size, p(dl), p(d), p(du), p(b))
    return b, info
