"""Python host binding of libdfdm.so: one class whose methods carry the names of the reference's subroutines.

Every method calls the C ABI declared in include/dfdm.h.  There is no CPU fallback: if the library is missing
or no GPU is present the calls raise DfdmError.
"""
from __future__ import annotations

import ctypes
import os
from ctypes import POINTER, c_char_p, c_double, c_int, c_size_t, c_void_p
from typing import Optional

import numpy as np

from . import build as _build
from .abi import (DFDM_FP32_MIXED, DFDM_FP64, PRECISIONS, DfdmGrid, DfdmParams, GridHolder, dptr,
                  make_params)
from .cases import Case

_lib = None

KERNELS = {"sgs": 0, "stage": 1, "fwd_x": 2, "fwd_z": 3, "y_solve": 4, "inv_z": 5, "inv_x": 6, "correct": 7,
           "wall_model": 8, "flux_shift": 9, "cfl": 10, "hybrid": 11}

# Every exported symbol of include/dfdm.h (checked by the CPU test suite).
EXPORTS = ["dfdm_default_params", "dfdm_last_error", "dfdm_version", "dfdm_create", "dfdm_destroy",
           "dfdm_footprint_bytes", "dfdm_set_stream", "dfdm_synchronize", "dfdm_set_state", "dfdm_get_state",
           "dfdm_get_nu_t", "dfdm_set_nu_t", "dfdm_set_time", "dfdm_get_time", "dfdm_compute_time_step_rk3",
           "dfdm_compute_time_step_rk3_async", "dfdm_enable_graphs", "dfdm_compute_sgs_model", "dfdm_compute_rhs",
           "dfdm_compute_wall_model", "dfdm_apply_boundary_conditions", "dfdm_compute_projection_step",
           "dfdm_solve_poisson", "dfdm_compute_bulk_velocity", "dfdm_check_divergence", "dfdm_kinetic_energy",
           "dfdm_check_finite", "dfdm_pad_field", "dfdm_launch_kernel_async", "dfdm_kernel_bytes",
           "dfdm_launch_count", "dfdm_solve_poisson_noalloc", "dfdm_write_snapshot", "dfdm_read_snapshot",
           "dfdm_compute_cfl", "dfdm_set_stage_variant", "dfdm_get_stage_variant", "dfdm_set_adaptive_dt",
           "dfdm_get_dt", "dfdm_set_landing_time", "dfdm_output_monitor", "dfdm_output_monitor_async",
           "dfdm_set_fused_correction", "dfdm_get_fused_correction", "dfdm_set_state_async", "dfdm_get_state_async",
           "dfdm_write_box_snapshot", "dfdm_set_landing_times", "dfdm_write_snapshot_ex", "dfdm_get_stage_timing",
           "dfdm_set_sgs_in_tile", "dfdm_get_sgs_in_tile", "dfdm_group_create", "dfdm_group_step_async",
           "dfdm_group_synchronize", "dfdm_group_launch_count", "dfdm_group_destroy", "dfdm_get_stream",
           "dfdm_group_get_stream", "dfdm_group_set_branch_cells", "dfdm_group_set_stage_tiles"]


class DfdmError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__(f"dfdm error {code}: {msg}")
        self.code = code


def lib_path() -> str:
    return _build.LIB_PATH


def load(build_if_missing: bool = True):
    """Load libdfdm.so (building it with nvcc first when it is absent and nvcc exists)."""
    global _lib
    if _lib is not None:
        return _lib
    path = _build.LIB_PATH
    if not os.path.exists(path):
        if not build_if_missing:
            raise DfdmError(2, f"{path} is missing; build it with dfdm.build.build()")
        _build.build()
    L = ctypes.CDLL(path)
    P = POINTER(c_double)
    sig = {
        "dfdm_default_params": (None, [POINTER(DfdmParams)]),
        "dfdm_last_error": (c_char_p, []),
        "dfdm_version": (c_char_p, []),
        "dfdm_create": (c_int, [POINTER(DfdmGrid), POINTER(DfdmParams), POINTER(c_void_p)]),
        "dfdm_destroy": (c_int, [c_void_p]),
        "dfdm_footprint_bytes": (c_int, [POINTER(DfdmGrid), POINTER(DfdmParams), POINTER(c_size_t)]),
        "dfdm_set_stream": (c_int, [c_void_p, c_void_p]),
        "dfdm_synchronize": (c_int, [c_void_p]),
        "dfdm_set_state": (c_int, [c_void_p, P, P, P, P]),
        "dfdm_get_state": (c_int, [c_void_p, P, P, P, P]),
        "dfdm_set_state_async": (c_int, [c_void_p, P, P, P, P]),
        "dfdm_get_state_async": (c_int, [c_void_p, P, P, P, P]),
        "dfdm_get_nu_t": (c_int, [c_void_p, P]),
        "dfdm_set_nu_t": (c_int, [c_void_p, P]),
        "dfdm_set_time": (c_int, [c_void_p, c_double]),
        "dfdm_get_time": (c_int, [c_void_p, P]),
        "dfdm_compute_time_step_rk3": (c_int, [c_void_p, c_int, P]),
        "dfdm_compute_time_step_rk3_async": (c_int, [c_void_p, c_int]),
        "dfdm_enable_graphs": (c_int, [c_void_p, c_int]),
        "dfdm_compute_sgs_model": (c_int, [c_void_p]),
        "dfdm_compute_rhs": (c_int, [c_void_p, P, P, P]),
        "dfdm_compute_wall_model": (c_int, [c_void_p, c_int, P, P]),
        "dfdm_apply_boundary_conditions": (c_int, [c_void_p, c_int]),
        "dfdm_compute_projection_step": (c_int, [c_void_p, c_int]),
        "dfdm_solve_poisson": (c_int, [c_void_p, P, P]),
        "dfdm_compute_bulk_velocity": (c_int, [c_void_p, P]),
        "dfdm_check_divergence": (c_int, [c_void_p, P]),
        "dfdm_kinetic_energy": (c_int, [c_void_p, P]),
        "dfdm_check_finite": (c_int, [c_void_p]),
        "dfdm_pad_field": (c_int, [c_void_p, c_int, c_int, P]),
        "dfdm_launch_kernel_async": (c_int, [c_void_p, c_int, c_int]),
        "dfdm_kernel_bytes": (c_int, [c_void_p, c_int, P]),
        "dfdm_launch_count": (c_int, [c_void_p, POINTER(ctypes.c_longlong)]),
        "dfdm_solve_poisson_noalloc": (c_int, [c_void_p, P, P]),
        "dfdm_write_snapshot": (c_int, [c_void_p, c_char_p]),
        "dfdm_write_snapshot_ex": (c_int, [c_void_p, c_char_p, c_int]),
        "dfdm_read_snapshot": (c_int, [c_void_p, c_char_p]),
        "dfdm_write_box_snapshot": (c_int, [c_void_p, c_char_p, POINTER(ctypes.c_int32), POINTER(ctypes.c_int32), c_int,
                                            ctypes.c_int32]),
        "dfdm_compute_cfl": (c_int, [c_void_p, P, P]),
        "dfdm_set_stage_variant": (c_int, [c_void_p, c_int]),
        "dfdm_get_stage_variant": (c_int, [c_void_p, POINTER(ctypes.c_int), P, P]),
        "dfdm_get_stage_timing": (c_int, [c_void_p, c_int, P]),
        "dfdm_set_sgs_in_tile": (c_int, [c_void_p, c_int]),
        "dfdm_get_sgs_in_tile": (c_int, [c_void_p, POINTER(ctypes.c_int)]),
        "dfdm_set_adaptive_dt": (c_int, [c_void_p, c_int, c_double, c_double, c_double, c_double]),
        "dfdm_get_dt": (c_int, [c_void_p, P]),
        "dfdm_set_landing_time": (c_int, [c_void_p, c_int, c_double]),
        "dfdm_set_landing_times": (c_int, [c_void_p, c_int, P]),
        "dfdm_output_monitor": (c_int, [c_void_p, P]),
        "dfdm_output_monitor_async": (c_int, [c_void_p, c_void_p]),
        "dfdm_set_fused_correction": (c_int, [c_void_p, c_int]),
        "dfdm_get_fused_correction": (c_int, [c_void_p, POINTER(ctypes.c_int)]),
        "dfdm_group_create": (c_int, [POINTER(c_void_p), c_int, c_void_p, POINTER(c_void_p)]),
        "dfdm_group_step_async": (c_int, [c_void_p, c_int]),
        "dfdm_group_synchronize": (c_int, [c_void_p]),
        "dfdm_group_launch_count": (c_int, [c_void_p, POINTER(ctypes.c_longlong)]),
        "dfdm_group_destroy": (c_int, [c_void_p]),
        "dfdm_get_stream": (c_int, [c_void_p, POINTER(c_void_p)]),
        "dfdm_group_get_stream": (c_int, [c_void_p, POINTER(c_void_p)]),
        "dfdm_group_set_branch_cells": (c_int, [c_void_p, ctypes.c_longlong]),
        "dfdm_group_set_stage_tiles": (c_int, [c_void_p, c_int, c_int]),
    }
    for name, (res, args) in sig.items():
        fn = getattr(L, name)
        fn.restype = res
        fn.argtypes = args
    _lib = L
    return L


def last_error() -> str:
    return load().dfdm_last_error().decode()


def _check(rc: int) -> None:
    if rc != 0:
        raise DfdmError(rc, last_error())


def footprint_bytes(case: Case, precision="fp32") -> int:
    g = GridHolder(case)
    p = make_params(case, PRECISIONS.get(precision, precision))
    out = c_size_t(0)
    _check(load().dfdm_footprint_bytes(ctypes.byref(g.grid), ctypes.byref(p), ctypes.byref(out)))
    return int(out.value)


class Solver:
    """One case resident on the GPU, driven through the C ABI.

    Method names follow the reference's subroutines: compute_time_step_RK3 (src/time_integration.f90:120),
    compute_sgs_model (src/sgs_model.f90:27), compute_rhs_u/v/w (src/equations.f90), compute_wall_model
    (src/wallmodel.f90:197), apply_boundary_conditions (src/boundary_conditions.f90:186),
    compute_projection_step (src/projection.f90:21), solve_poisson_equation (src/projection.f90:100),
    compute_bulk_velocity (src/monitor.f90:463) and check_divergence (src/projection.f90:607).
    """

    def __init__(self, case: Case, precision="fp64", graphs: bool = False, stream: Optional[int] = None):
        self.case = case
        self.precision = PRECISIONS.get(precision, precision)
        self._g = GridHolder(case)
        self._p = make_params(case, self.precision)
        self.shapes = case.shapes()
        h = c_void_p()
        _check(load().dfdm_create(ctypes.byref(self._g.grid), ctypes.byref(self._p), ctypes.byref(h)))
        self.h = h
        if stream is not None:
            self.set_stream(stream)
        if graphs:
            _check(load().dfdm_enable_graphs(self.h, 1))

    # ---- lifetime ----
    def close(self):
        if getattr(self, "h", None):
            load().dfdm_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def set_stream(self, stream: Optional[int]):
        _check(load().dfdm_set_stream(self.h, c_void_p(stream) if stream else None))

    def synchronize(self):
        _check(load().dfdm_synchronize(self.h))
        self._pending = []

    @property
    def stream_handle(self) -> int:
        """The cudaStream_t the context runs on, as an integer (torch.cuda.ExternalStream wraps it)."""
        v = c_void_p()
        _check(load().dfdm_get_stream(self.h, ctypes.byref(v)))
        return int(v.value or 0)

    def enable_graphs(self, on: bool = True):
        _check(load().dfdm_enable_graphs(self.h, int(on)))

    # ---- state ----
    def _arr(self, key):
        return np.zeros(self.shapes[key], order="F")

    def set_state(self, U, V, W, P=None):
        f = lambda a: None if a is None else np.asfortranarray(a, dtype=np.float64)
        U, V, W, P = f(U), f(V), f(W), f(P)
        _check(load().dfdm_set_state(self.h, dptr(U), dptr(V), dptr(W), dptr(P)))

    def get_state(self, out=None):
        U, V, W, P = out if out is not None else (self._arr("U"), self._arr("V"), self._arr("W"), self._arr("P"))
        _check(load().dfdm_get_state(self.h, dptr(U), dptr(V), dptr(W), dptr(P)))
        return U, V, W, P

    @staticmethod
    def _async_arg(a):
        """An array an asynchronous copy may use in place: Fortran-ordered float64 (no temporary copy)."""
        if a is None:
            return None
        if a.dtype != np.float64 or not a.flags.f_contiguous:
            raise ValueError("asynchronous transfers need Fortran-ordered float64 arrays (ideally pinned memory)")
        return a

    def set_state_async(self, U, V, W, P=None):
        """Enqueue the upload; the arrays must stay untouched until synchronize()."""
        args = [self._async_arg(a) for a in (U, V, W, P)]
        self._pending = getattr(self, "_pending", []) + args
        _check(load().dfdm_set_state_async(self.h, *[dptr(a) for a in args]))

    def get_state_async(self, out):
        """Enqueue the download into out = (U, V, W, P) (P may be None); valid after synchronize()."""
        args = [self._async_arg(a) for a in out]
        self._pending = getattr(self, "_pending", []) + args
        _check(load().dfdm_get_state_async(self.h, *[dptr(a) for a in args]))

    def get_nu_t(self):
        a = self._arr("P")
        _check(load().dfdm_get_nu_t(self.h, dptr(a)))
        return a

    def set_nu_t(self, a):
        a = np.asfortranarray(a, dtype=np.float64)
        _check(load().dfdm_set_nu_t(self.h, dptr(a)))

    def set_time(self, t: float):
        _check(load().dfdm_set_time(self.h, float(t)))

    @property
    def t(self) -> float:
        v = c_double(0.0)
        _check(load().dfdm_get_time(self.h, ctypes.byref(v)))
        return v.value

    # ---- the step ----
    def compute_time_step_RK3(self, nsteps: int = 1) -> float:
        t = c_double(0.0)
        _check(load().dfdm_compute_time_step_rk3(self.h, int(nsteps), ctypes.byref(t)))
        return t.value

    def compute_time_step_RK3_async(self, nsteps: int = 1) -> None:
        _check(load().dfdm_compute_time_step_rk3_async(self.h, int(nsteps)))

    # ---- unit entry points ----
    def compute_sgs_model(self):
        _check(load().dfdm_compute_sgs_model(self.h))

    def compute_rhs(self):
        fu, fv, fw = self._arr("rhs_u"), self._arr("rhs_v"), self._arr("rhs_w")
        _check(load().dfdm_compute_rhs(self.h, dptr(fu), dptr(fv), dptr(fw)))
        return fu, fv, fw

    def compute_wall_model(self, update_filter: bool = True):
        tx, tz = self._arr("tau_x"), self._arr("tau_z")
        _check(load().dfdm_compute_wall_model(self.h, int(update_filter), dptr(tx), dptr(tz)))
        return tx, tz

    def apply_boundary_conditions(self, after_projection: bool = False):
        _check(load().dfdm_apply_boundary_conditions(self.h, int(after_projection)))

    def compute_projection_step(self, save_p: bool = False):
        _check(load().dfdm_compute_projection_step(self.h, int(save_p)))

    def solve_poisson_equation(self, rhs_p, out=None):
        """phi for rhs_p, both in the reference's (2:nxg, 2:nyg-1, 2:nzg) shape.  out: an FP64 Fortran-order array of
        that shape to write into (rhs_p itself solves in place, as the reference's subroutine does); a caller that
        solves repeatedly should pass one, since a fresh array's first-touch page faults land inside the copy."""
        a = np.asfortranarray(rhs_p, dtype=np.float64)
        if out is None:
            out = np.zeros_like(a, order="F")
        elif out.shape != a.shape or out.dtype != np.float64 or not out.flags.f_contiguous:
            raise ValueError("out must be an FP64 Fortran-order array of rhs_p's shape")
        _check(load().dfdm_solve_poisson(self.h, dptr(a), dptr(out)))
        return out

    def solve_poisson_noalloc(self, rhs_p):
        """dfdm_solve_poisson through the library's fixed staging array: no device allocation in the call."""
        a = np.asfortranarray(rhs_p, dtype=np.float64)
        out = np.zeros_like(a, order="F")
        _check(load().dfdm_solve_poisson_noalloc(self.h, dptr(a), dptr(out)))
        return out

    def write_snapshot(self, path: str, byte_order: str = "big") -> None:
        """The reference's restart file (and <path>.wmf with a seeded wall-model filter), big-endian as the
        reference's builds write it, or little-endian with byte_order="little"."""
        if byte_order not in ("big", "little"):
            raise ValueError("byte_order must be 'big' or 'little'")
        _check(load().dfdm_write_snapshot_ex(self.h, os.fsencode(path), 1 if byte_order == "big" else 0))

    def read_snapshot(self, path: str) -> None:
        """U, V, W, P (and the wall-model filter from <path>.wmf) from a restart file of this grid, in the byte
        order the file holds."""
        _check(load().dfdm_read_snapshot(self.h, os.fsencode(path)))

    def write_box_snapshot(self, path: str, f1, f2, location: int = 0, step: int = 0) -> None:
        """The reference's chunked / cell-centred box snapshot (write_box_snapshot) of the face box f1..f2 (1-based
        faces per direction; dfdm.snapshot.resolve_chunk_box turns the &IO chunk inputs into f1, f2)."""
        a = (ctypes.c_int32 * 3)(*[int(v) for v in f1])
        b = (ctypes.c_int32 * 3)(*[int(v) for v in f2])
        _check(load().dfdm_write_box_snapshot(self.h, os.fsencode(path), a, b, int(location), int(step)))

    def compute_bulk_velocity(self) -> float:
        v = c_double(0.0)
        _check(load().dfdm_compute_bulk_velocity(self.h, ctypes.byref(v)))
        return v.value

    def check_divergence(self) -> float:
        v = c_double(0.0)
        _check(load().dfdm_check_divergence(self.h, ctypes.byref(v)))
        return v.value

    def set_fused_correction(self, enable: bool = True):
        """Stage-1/2 projections inside the next stage kernel (on by default where it applies)."""
        _check(load().dfdm_set_fused_correction(self.h, int(enable)))

    @property
    def fused_correction(self) -> bool:
        v = ctypes.c_int(0)
        _check(load().dfdm_get_fused_correction(self.h, ctypes.byref(v)))
        return bool(v.value)

    def set_stage_variant(self, variant: int) -> None:
        """FP32 stage kernel: 0 one cell per thread, 1 packed pairs, 2 packed pairs with TMA plane tiles (walls in y,
        Nx a multiple of 4), -1 re-time the eligible ones and keep the fastest."""
        _check(load().dfdm_set_stage_variant(self.h, int(variant)))

    def set_sgs_in_tile(self, enable: bool = True) -> None:
        """LES: eddy viscosity computed in the stage tiles (True, the default) or by the separate pass (False)."""
        _check(load().dfdm_set_sgs_in_tile(self.h, int(bool(enable))))

    def sgs_in_tile(self) -> bool:
        v = ctypes.c_int(0)
        _check(load().dfdm_get_sgs_in_tile(self.h, ctypes.byref(v)))
        return bool(v.value)

    def stage_timing(self, variant: int) -> float:
        """ms per launch of a stage-kernel variant from the set-up timing (-1 = not timed)."""
        ms = c_double(0.0)
        _check(load().dfdm_get_stage_timing(self.h, int(variant), ctypes.byref(ms)))
        return ms.value

    def stage_variant(self):
        """(variant in use, ms per launch of variant 0, of variant 1) from the set-up timing (-1 = not timed)."""
        v, a, b = ctypes.c_int(0), c_double(0.0), c_double(0.0)
        _check(load().dfdm_get_stage_variant(self.h, ctypes.byref(v), ctypes.byref(a), ctypes.byref(b)))
        return v.value, a.value, b.value

    def compute_cfl(self):
        """(convective, viscous) CFL numbers of the resident state, as compute_cfl (src/monitor.f90:304)."""
        a, b = c_double(0.0), c_double(0.0)
        _check(load().dfdm_compute_cfl(self.h, ctypes.byref(a), ctypes.byref(b)))
        return a.value, b.value

    def set_adaptive_dt(self, enable=True, cfl_target=0.5, cfl_safety=0.9, dt_min=1e-10, dt_max=1e10):
        """cfl_adaptive = 1: dt chosen on the device from the start-of-step CFL number at every step
        (select_dt, src/monitor.f90:429-444)."""
        _check(load().dfdm_set_adaptive_dt(self.h, int(enable), cfl_target, cfl_safety, dt_min, dt_max))

    def set_landing_time(self, t_land=None):
        """Shrink the coming steps so that t lands on t_land (landing_dt, src/monitor.f90:436-458); None: no target."""
        _check(load().dfdm_set_landing_time(self.h, 0 if t_land is None else 1, 0.0 if t_land is None else float(t_land)))

    def set_landing_times(self, targets=()):
        """Up to five landing targets in select_dt's order (tsave_next, chunk_tsave_next, slice_tnext, line_tnext,
        sim_end_time), applied in turn; None entries are slots without a target (dfdm.output.OutputSchedule keeps
        them)."""
        vals = [float("nan") if v is None else float(v) for v in targets]
        if len(vals) > 5:
            raise ValueError("at most five landing targets")
        arr = (c_double * max(1, len(vals)))(*vals)
        _check(load().dfdm_set_landing_times(self.h, len(vals), arr))

    @property
    def dt(self) -> float:
        v = c_double(0.0)
        _check(load().dfdm_get_dt(self.h, ctypes.byref(v)))
        return v.value

    MONITOR_KEYS = ("t", "dt", "mean_u", "max_u", "max_div", "cfl_conv", "cfl_visc", "u_tau_lo", "u_tau_hi", "nan_flag")

    def output_monitor(self) -> dict:
        """The values output_monitor prints (src/monitor.f90:21-102), from one device pass; raises DfdmError
        (DFDM_ERR_NOT_FINITE) when the NaN / |u| > 1e8 guard trips."""
        out = (c_double * 10)()
        _check(load().dfdm_output_monitor(self.h, out))
        return dict(zip(self.MONITOR_KEYS, list(out)))

    def output_monitor_async(self, out_ptr: int) -> None:
        """Enqueue the monitor into ten doubles at out_ptr (pinned host or device memory)."""
        _check(load().dfdm_output_monitor_async(self.h, ctypes.c_void_p(out_ptr)))

    def kinetic_energy(self) -> float:
        v = c_double(0.0)
        _check(load().dfdm_kinetic_energy(self.h, ctypes.byref(v)))
        return v.value

    def check_finite(self) -> None:
        _check(load().dfdm_check_finite(self.h))

    def pad_field(self, field: int = 1, extra_planes: int = 1):
        _check(load().dfdm_pad_field(self.h, int(field), int(extra_planes), None))

    # ---- profiling hooks ----
    def launch_kernel_async(self, which, rk_stage: int = 2):
        which = KERNELS.get(which, which)
        _check(load().dfdm_launch_kernel_async(self.h, int(which), int(rk_stage)))

    def launch_count(self) -> int:
        v = ctypes.c_longlong(0)
        _check(load().dfdm_launch_count(self.h, ctypes.byref(v)))
        return int(v.value)

    def kernel_bytes(self, which) -> float:
        which = KERNELS.get(which, which)
        v = c_double(0.0)
        _check(load().dfdm_kernel_bytes(self.h, int(which), ctypes.byref(v)))
        return v.value


class Group:
    """Several FP32-mixed DNS solvers stepped together: one grouped launch per kernel family for all members, one
    CUDA graph per group step (dfdm_group_create).  A member's results do not depend on the other members (the same
    case steps bit-identically in a group of one and in any mix); against compute_time_step_RK3 steps of the member
    alone they agree to FP32 rounding.  Members must have taken a first step."""

    def __init__(self, solvers, stream: Optional[int] = None):
        self.solvers = list(solvers)
        hs = (c_void_p * len(self.solvers))(*[s.h.value if isinstance(s.h, c_void_p) else s.h for s in self.solvers])
        h = c_void_p()
        _check(load().dfdm_group_create(hs, len(self.solvers), c_void_p(stream) if stream else None, ctypes.byref(h)))
        self.h = h

    def step_async(self, nsteps: int = 1) -> None:
        _check(load().dfdm_group_step_async(self.h, int(nsteps)))

    def step(self, nsteps: int = 1) -> None:
        self.step_async(nsteps)
        self.synchronize()

    def synchronize(self) -> None:
        _check(load().dfdm_group_synchronize(self.h))

    @property
    def stream_handle(self) -> int:
        """The cudaStream_t the group runs on, as an integer."""
        v = c_void_p()
        _check(load().dfdm_group_get_stream(self.h, ctypes.byref(v)))
        return int(v.value or 0)

    def launch_count(self) -> int:
        v = ctypes.c_longlong(0)
        _check(load().dfdm_group_launch_count(self.h, ctypes.byref(v)))
        return int(v.value)

    def set_branch_cells(self, cells: int) -> None:
        """At most `cells` cells per graph branch (0: one branch per shape class); results do not change."""
        _check(load().dfdm_group_set_branch_cells(self.h, int(cells)))

    def set_stage_tiles(self, kc: int = -1, walk: bool = False) -> None:
        """Fix the grouped stage launches' tile shape: kc > 0 z-planes per block, 0 each member's own, with walking
        resident blocks if walk; kc < 0 returns to the group's timed choice.  Results do not change."""
        _check(load().dfdm_group_set_stage_tiles(self.h, int(kc), int(bool(walk))))

    def close(self):
        if getattr(self, "h", None):
            load().dfdm_group_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()
