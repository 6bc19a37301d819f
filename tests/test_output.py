"""The reference's output cadence (dfdm.output.OutputSchedule: save_due, write_probes, the stop rule) and the
landing of select_dt on several time targets at once, on the host and through the oracle."""
import math

import numpy as np
import pytest

from dfdm import cases
from dfdm.output import OutputSchedule


def _landing_dt(dt_now, rem):   # landing_dt, src/monitor.f90:449-458
    r = dt_now
    if rem < 2.0 * dt_now:
        r = rem
        if rem > dt_now:
            r = 0.5 * rem
    return r


def _run(sched, dt0, t0=0.0, max_steps=10000):
    """main.f90's loop with select_dt's landing on every time target in turn (fixed dt)."""
    t, istep, log = t0, 0, []
    while True:
        istep += 1
        dt = dt0
        for tl in sched.targets():
            if tl is not None and tl - t > 1e-10:
                dt = _landing_dt(dt, tl - t)
        t += dt
        log.append((istep, t, dt, sched.after_step(istep, t)))
        if sched.done(istep, t) or istep >= max_steps:
            return log


def test_time_cadences_land_exactly():
    s = OutputSchedule(nsteps=-1, sim_end_time=0.05, nsave=-1, tsave=0.01, n_slices=2, slice_freq=-1,
                       slice_interval=0.006)
    log = _run(s, 0.004)
    full = [t for _, t, _, d in log if "full" in d]
    slices = [t for _, t, _, d in log if "slices" in d]
    assert np.allclose(full, [0.01 * k for k in range(1, 6)], rtol=0, atol=1e-12)
    assert np.allclose(slices, [0.006 * k for k in range(1, 9)], rtol=0, atol=1e-12)
    assert abs(log[-1][1] - 0.05) < 1e-12
    # no step shorter than half the base dt except a landing remainder (landing_dt never makes slivers)
    assert min(dt for _, _, dt, _ in log) >= 0.0009


def test_step_cadences_and_the_chunk_with_the_full_snapshot():
    s = OutputSchedule(nsteps=12, nsave=3, chunked_snapshot=True, chunk_nsave=0, n_lines=1, line_freq=4)
    log = _run(s, 1e-3)
    assert len(log) == 12
    assert [i for i, _, _, d in log if "full" in d] == [3, 6, 9, 12]
    assert [i for i, _, _, d in log if "chunk" in d] == [3, 6, 9, 12]
    assert [i for i, _, _, d in log if "lines" in d] == [4, 8, 12]
    assert all(tl is None for tl in s.targets())


def test_chunk_on_its_own_time_cadence():
    s = OutputSchedule(t0=1.0, nsteps=-1, sim_end_time=1.03, nsave=5, chunked_snapshot=True, chunk_nsave=-1,
                       chunk_tsave=0.0075)
    assert s.targets() == [None, 1.0075, None, None, 1.03]
    log = _run(s, 0.002, t0=1.0)
    chunks = [t for _, t, _, d in log if "chunk" in d]
    assert np.allclose(chunks, [1.0 + 0.0075 * k for k in range(1, 5)], rtol=0, atol=1e-12)
    assert [i for i, _, _, d in log if "full" in d] == [i for i, _, _, _ in log if i % 5 == 0]


def test_oracle_lands_on_every_target(oracle_mod):
    """The oracle's select_dt with three targets at once: the steps it takes are those of main.f90's loop."""
    c = cases.tgv_small()
    o = oracle_mod.Oracle(c)
    o.set_state(*cases.initial_condition(c))
    sched = OutputSchedule(nsteps=-1, sim_end_time=9.5 * c.dt, nsave=-1, tsave=2.5 * c.dt, n_slices=1,
                           slice_freq=-1, slice_interval=3.5 * c.dt)
    want = _run(OutputSchedule(nsteps=-1, sim_end_time=9.5 * c.dt, nsave=-1, tsave=2.5 * c.dt, n_slices=1,
                               slice_freq=-1, slice_interval=3.5 * c.dt), c.dt)
    istep = 0
    while True:
        istep += 1
        o.set_landing_times(sched.targets())
        o.step(1)
        due = sched.after_step(istep, o.t)
        i, t, dt, d = want[istep - 1]
        assert abs(o.t - t) <= 1e-15 * max(1.0, t) and due == d, (istep, o.t, t, due, d)
        if sched.done(istep, o.t):
            break
    assert istep == len(want) and abs(o.t - 9.5 * c.dt) < 1e-12
