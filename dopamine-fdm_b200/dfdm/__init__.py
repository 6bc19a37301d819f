"""dfdm: B200 library for dopamine-fdm's single-phase fractional-step RK3 time step.

The compute path is libdfdm.so (hand-written CUDA for sm_100a behind the C ABI of include/dfdm.h); this package is
its Python host binding plus the case set-up used by the tests, the benchmark and the serving loop.
"""
from . import cases  # noqa: F401
from .abi import DFDM_FP32_MIXED, DFDM_FP64  # noqa: F401

__all__ = ["cases", "DFDM_FP64", "DFDM_FP32_MIXED", "Solver", "DfdmError", "load"]


def __getattr__(name):
    if name in ("Solver", "DfdmError", "load", "footprint_bytes", "KERNELS", "EXPORTS"):
        from . import native
        return getattr(native, name)
    raise AttributeError(name)
