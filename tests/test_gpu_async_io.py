"""Asynchronous state transfer (dfdm_set_state_async / dfdm_get_state_async): the same values as the synchronous
calls, and a pipelined host loop (upload, step, download per step, one synchronisation at the end) produces what
the synchronous loop produces."""
import numpy as np
import pytest

from dfdm import cases
from dfdm.native import Solver

pytestmark = pytest.mark.gpu


def _pinned_like(a):
    import torch
    t = torch.empty(a.shape[::-1], dtype=torch.float64, pin_memory=True)
    v = t.numpy().T   # Fortran-ordered view of pinned memory
    v[...] = a
    return t, v


@pytest.mark.parametrize("prec", ["fp64", "fp32"])
def test_async_round_trip_equals_sync(prec):
    c = cases.get("chan_small")
    st = cases.initial_condition(c)
    a = Solver(c, prec)
    a.set_state(*st)
    a.compute_time_step_RK3(2)
    want = a.get_state()
    keep = [_pinned_like(x) for x in want]
    outs = [_pinned_like(np.zeros_like(x)) for x in want]
    b = Solver(c, prec)
    b.set_state(*st)              # fixes the FP32 base profile as a did
    b.set_state_async(*[v for _, v in keep])
    b.get_state_async([v for _, v in outs])
    b.synchronize()
    for x, (_, y) in zip(want, outs):
        assert np.array_equal(x, y)
    a.close()
    b.close()


@pytest.mark.parametrize("prec", ["fp64", "fp32"])
def test_pipelined_loop_equals_synchronous_loop(prec):
    c = cases.get("chan_small")
    st = cases.initial_condition(c)
    ins = [_pinned_like(x) for x in st[:3]]
    n = 4
    sync_out = []
    a = Solver(c, prec)
    a.set_state(*st)
    for _ in range(n):
        a.set_state(*[v for _, v in ins])
        a.compute_time_step_RK3(1)
        sync_out.append([x.copy() for x in a.get_state()])
    b = Solver(c, prec)
    b.set_state(*st)
    outs = [[_pinned_like(np.zeros_like(x)) for x in st] for _ in range(n)]
    for q in range(n):
        b.set_state_async(*[v for _, v in ins])
        b.compute_time_step_RK3_async(1)
        b.get_state_async([v for _, v in outs[q]])
    b.synchronize()
    for q in range(n):
        for x, (_, y) in zip(sync_out[q], outs[q]):
            assert np.array_equal(x, y)
    a.close()
    b.close()
