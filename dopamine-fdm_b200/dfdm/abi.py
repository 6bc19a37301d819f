"""ctypes mirror of the C ABI structures declared in include/dfdm.h."""
from __future__ import annotations

import ctypes
from ctypes import POINTER, c_double, c_int

import numpy as np

from .cases import Case, faces

DFDM_OK = 0
DFDM_ERR_INVALID = 1
DFDM_ERR_CUDA = 2
DFDM_ERR_NOMEM = 3
DFDM_ERR_UNSUPPORTED = 4
DFDM_ERR_NOT_FINITE = 5
DFDM_ERR_TIMEOUT = 6

DFDM_FP64 = 0
DFDM_FP32_MIXED = 1

PRECISIONS = {"fp64": DFDM_FP64, "fp32": DFDM_FP32_MIXED, "fp32_mixed": DFDM_FP32_MIXED}


class DfdmGrid(ctypes.Structure):
    _fields_ = [("nx", c_int), ("ny", c_int), ("nz", c_int),
                ("x", POINTER(c_double)), ("y", POINTER(c_double)), ("z", POINTER(c_double)),
                ("x_bc_type", c_int), ("y_bc_type", c_int), ("z_bc_type", c_int),
                ("bc_face_ylo", c_int), ("bc_face_yhi", c_int)]


class DfdmParams(ctypes.Structure):
    _fields_ = [("nu", c_double), ("dt", c_double), ("dPdx", c_double), ("dPdz", c_double),
                ("sgs_model", c_int), ("Cs_vreman", c_double), ("C_amd", c_double),
                ("flat_wall_model_flag", c_int), ("advection_scheme", c_int), ("adv_wall_layers", c_int),
                ("wm_filter_mode", c_int), ("wm_filter_Tf_fac", c_double), ("flow_forcing_mode", c_int),
                ("Ub_target", c_double), ("precision", c_int), ("adv_order", c_int), ("adv_beta0", c_double)]


def dptr(a: np.ndarray):
    """double* of a contiguous float64 numpy array (None -> NULL)."""
    if a is None:
        return None
    assert a.dtype == np.float64 and (a.flags.f_contiguous or a.flags.c_contiguous)
    return a.ctypes.data_as(POINTER(c_double))


class GridHolder:
    """Keeps the face arrays alive for as long as the dfdm_grid struct that points at them."""

    def __init__(self, case: Case):
        self.x, self.y, self.z = (np.ascontiguousarray(a, dtype=np.float64) for a in faces(case))
        self.grid = DfdmGrid(case.nx, case.ny, case.nz, dptr(self.x), dptr(self.y), dptr(self.z),
                             case.x_bc_type, case.y_bc_type, case.z_bc_type, 1, 1)


def make_params(case: Case, precision: int = DFDM_FP64) -> DfdmParams:
    return DfdmParams(case.nu, case.dt, case.dPdx, case.dPdz, case.sgs_model, case.Cs_vreman, case.C_amd,
                      case.flat_wall_model_flag, case.advection_scheme, case.adv_wall_layers, case.wm_filter_mode,
                      case.wm_filter_Tf_fac, case.flow_forcing_mode, case.Ub_target, int(precision),
                      case.adv_order, case.adv_beta0)
