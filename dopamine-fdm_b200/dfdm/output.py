"""The reference's output cadence on the host: which outputs a step makes due and the landing targets of the next
step, as the main loop (src/main.f90:58-92) drives them around compute_time_step_RK3.

  initialisation  tsave_next = t0 + tsave (nsave < 0), chunk_tsave_next = t0 + chunk_tsave (chunk_nsave < 0)
                  (src/initialization.f90:115-118); slice_tnext = t0 + slice_interval, line_tnext = t0 +
                  line_interval (src/probe_output.f90:50)
  select_dt       lands t on tsave_next, chunk_tsave_next, slice_tnext, line_tnext, sim_end_time in that order, each
                  only when its cadence is time-based (src/monitor.f90:436-440)
  output_data     full snapshot when save_due(nsave, tsave_next, tsave); the chunk box with it (chunk_nsave = 0) or
                  when save_due(chunk_nsave, chunk_tsave_next, chunk_tsave) (src/input_output.f90:1790-1796; save_full at :1793)
  write_probes    slices / lines every slice_freq / line_freq steps, or once t reaches slice_tnext / line_tnext, the
                  target then moving on by one interval (src/probe_output.f90:173-211)
  save_due        n > 0: every n steps; otherwise once t >= tnext - 1e-10, then tnext += tint (:1764-1778)
  stop            nsteps > 0: after step nsteps; nsteps < 0: once t >= sim_end_time - 1e-10 (src/main.f90:86-92)

A driver calls ``targets()`` before a step (``Solver.set_landing_times`` / ``Oracle.set_landing_times``), steps once,
then calls ``after_step(istep, t)`` for the outputs due and ``done(istep, t)``.
"""
from __future__ import annotations

from dataclasses import dataclass, field
from typing import List, Optional, Set

TOL = 1e-10


@dataclass
class OutputSchedule:
    t0: float = 0.0
    nsteps: int = 1               # > 0 step count, < 0 run to sim_end_time
    sim_end_time: float = 0.0
    nsave: int = 0                # > 0 every nsave steps, < 0 every tsave in time
    tsave: float = 0.0
    chunked_snapshot: bool = False
    chunk_nsave: int = 0          # 0: with the full snapshot
    chunk_tsave: float = 0.0
    n_slices: int = 0
    slice_freq: int = 0           # > 0 every slice_freq steps, < 0 every slice_interval in time
    slice_interval: float = 0.0
    n_lines: int = 0
    line_freq: int = 0
    line_interval: float = 0.0
    tsave_next: float = field(init=False, default=0.0)
    chunk_tsave_next: float = field(init=False, default=0.0)
    slice_tnext: float = field(init=False, default=0.0)
    line_tnext: float = field(init=False, default=0.0)

    def __post_init__(self):
        if self.nsave < 0:
            self.tsave_next = self.t0 + self.tsave
        if self.chunk_nsave < 0:
            self.chunk_tsave_next = self.t0 + self.chunk_tsave
        self.slice_tnext = self.t0 + self.slice_interval
        self.line_tnext = self.t0 + self.line_interval

    def targets(self) -> List[Optional[float]]:
        """select_dt's five landing targets for the coming step (None: that cadence is not time-based)."""
        return [self.tsave_next if self.nsave < 0 else None,
                self.chunk_tsave_next if (self.chunked_snapshot and self.chunk_nsave < 0) else None,
                self.slice_tnext if (self.n_slices > 0 and self.slice_freq < 0) else None,
                self.line_tnext if (self.n_lines > 0 and self.line_freq < 0) else None,
                self.sim_end_time if self.nsteps < 0 else None]

    @staticmethod
    def _save_due(n: int, tnext: float, tint: float, istep: int, t: float):
        if n > 0:
            return istep % n == 0, tnext
        due = t >= tnext - TOL
        return due, (tnext + tint if due else tnext)

    def after_step(self, istep: int, t: float) -> Set[str]:
        """The outputs due after step istep at time t ("full", "chunk", "slices", "lines"), moving the time targets
        on in the order output_data, write_probes."""
        due: Set[str] = set()
        full, self.tsave_next = self._save_due(self.nsave, self.tsave_next, self.tsave, istep, t)
        chunk = self.chunked_snapshot and full and self.chunk_nsave == 0
        if self.chunked_snapshot and self.chunk_nsave != 0:
            chunk, self.chunk_tsave_next = self._save_due(self.chunk_nsave, self.chunk_tsave_next, self.chunk_tsave,
                                                          istep, t)
        if full:
            due.add("full")
        if chunk:
            due.add("chunk")
        slice_due = ((self.n_slices > 0 and self.slice_freq > 0 and istep % self.slice_freq == 0) or
                     (self.n_slices > 0 and self.slice_freq < 0 and t >= self.slice_tnext - TOL))
        line_due = ((self.n_lines > 0 and self.line_freq > 0 and istep % self.line_freq == 0) or
                    (self.n_lines > 0 and self.line_freq < 0 and t >= self.line_tnext - TOL))
        if slice_due:
            if self.slice_freq < 0:
                self.slice_tnext += self.slice_interval
            due.add("slices")
        if line_due:
            if self.line_freq < 0:
                self.line_tnext += self.line_interval
            due.add("lines")
        return due

    def done(self, istep: int, t: float) -> bool:
        if self.nsteps > 0:
            return istep >= self.nsteps
        return t >= self.sim_end_time - TOL
