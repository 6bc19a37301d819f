"""The request loop's scheduling logic on a simulated device (CPU), and the request stream's statistics."""
import numpy as np
import pytest

from dfdm import serve


class FakeExecutor:
    """Simulated device: one work queue at `rate` cell-steps/s shared by all streams; virtual clock."""

    def __init__(self, rate=5e9, bytes_per_cell=72.0):
        self.t = 0.0
        self.rate = rate
        self.bpc = bytes_per_cell
        self.busy_until = 0.0
        self.steps = {}
        self.started = []
        self.live = 0
        self.max_live = 0
        self.handles = []

    def now(self):
        return self.t

    def idle(self, until_next_arrival):
        cands = [h["t_done"] for h in self._inflight if h["t_done"] > self.t]
        if until_next_arrival is not None:
            cands.append(self.t + max(until_next_arrival, 1e-9))
        self.t = min(cands) if cands else self.t + 1e-3

    @property
    def _inflight(self):
        return [h for h in self.handles if h.get("t_done") is not None]

    def footprint(self, req):
        return int(req.cells * self.bpc)

    def prepare(self, req):
        pass

    def can_enqueue(self, h):
        return True

    def reclaim(self):
        pass

    def start(self, req):
        h = {"rid": req.rid, "t_done": None, "cells": req.cells}
        self.handles = self.handles + [h]
        self.steps[req.rid] = 0
        self.started.append(req.rid)
        self.live += 1
        self.max_live = max(self.max_live, self.live)
        return h

    def enqueue(self, h, k):
        self.steps[h["rid"]] += k
        w = k * h["cells"]
        t0 = max(self.t, self.busy_until)
        self.busy_until = t0 + w / self.rate
        h["t_done"] = self.busy_until

    def ready(self, h):
        return h["t_done"] is not None and h["t_done"] <= self.t

    def finish(self, h, req, keep_state):
        self.live -= 1
        self.handles = [x for x in self.handles if x is not h]
        return None, {"steps": self.steps[req.rid]}


class FakeGroupExecutor(FakeExecutor):
    """Simulated device for GroupScheduler: first steps and group chunks queue on one device at `rate` cell-steps/s;
    a group chunk of k steps costs k times the members' cells."""

    def __init__(self, rate=5e9, bytes_per_cell=72.0):
        super().__init__(rate, bytes_per_cell)
        self.tokens = []
        self.chunk_sizes = []
        self.chunk_keys = []
        self.max_group_inflight = 0
        self.by_class = True

    def idle(self, until_next_arrival):
        cands = [t["t_done"] for t in self.tokens if t["t_done"] > self.t]
        if until_next_arrival is not None:
            cands.append(self.t + max(until_next_arrival, 1e-9))
        self.t = min(cands) if cands else self.t + 1e-3

    def start(self, req):
        h = super().start(req)
        h["nsteps"] = req.nsteps
        h["joined"] = False
        return h

    def _run(self, work, group):
        t0 = max(self.t, self.busy_until)
        self.busy_until = t0 + work / self.rate
        tok = {"t_done": self.busy_until, "group": group}
        self.tokens.append(tok)
        return tok

    def shape_class(self, h):
        return h["cells"]

    def first_step(self, h):
        assert not h["joined"] and self.steps[h["rid"]] == 0
        h["joined"] = True
        self.steps[h["rid"]] += 1
        return self._run(h["cells"], False)

    def group_step(self, hs, k, key=0):
        assert k >= 1 and hs
        for h in hs:
            assert h["joined"]
            assert self.by_class is False or h["cells"] == key      # one shape class per group
            self.steps[h["rid"]] += k
            assert self.steps[h["rid"]] <= h["nsteps"]           # never past a member's last step
        self.chunk_sizes.append(len(hs))
        self.chunk_keys.append(key)
        tok = self._run(k * sum(h["cells"] for h in hs), True)
        tok["key"] = key
        live = sum(1 for t in self.tokens if t["group"] and t.get("key") == key and t["t_done"] > self.t)
        self.max_group_inflight = max(self.max_group_inflight, live)
        return tok

    def done(self, tok):
        return tok["t_done"] <= self.t


@pytest.mark.parametrize("by_class", [True, False])
def test_group_scheduler_issues_every_step_once_within_budget_in_order(by_class):
    reqs = serve.make_stream(64, 4.0, seed=11, steps=(1, 60))
    ex = FakeGroupExecutor(rate=1e8)
    ex.by_class = by_class
    budget = 3 * 128**3 * ex.bpc
    sch = serve.GroupScheduler(ex, budget, chunk_cell_steps=1e6, depth=2, by_class=by_class)
    out = sch.run(reqs)
    assert [r.rid for r in out] == sorted(r.rid for r in reqs)
    for r, q in zip(out, sorted(reqs, key=lambda x: x.rid)):
        assert r.summary["steps"] == q.nsteps                      # first step + group chunks, each step once
        assert r.finished >= r.admitted >= r.arrival - 1e-12
    assert sch.peak_bytes <= budget
    assert ex.started == sorted(ex.started, key=lambda rid: reqs[rid].arrival)
    assert sch.peak_group > 1 and max(ex.chunk_sizes) == sch.peak_group   # cases step together
    assert ex.max_group_inflight <= 2                                      # at most `depth` chunks per class queued
    assert sch.compositions >= 2


def test_group_scheduler_chunk_is_cut_at_the_first_member_to_finish():
    reqs = [serve.Request(0, serve.serve_case("tgv", 32, 800.0, 1), 50, 0.0),
            serve.Request(1, serve.serve_case("tgv", 32, 900.0, 2), 9, 0.0),
            serve.Request(2, serve.serve_case("tgv", 32, 1000.0, 3), 30, 0.0),
            serve.Request(3, serve.serve_case("chan", 48, 0.0, 4), 20, 0.0)]
    ex = FakeGroupExecutor(rate=1e9)
    sch = serve.GroupScheduler(ex, 1e12, chunk_cell_steps=1e9)   # chunks limited only by the members' ends
    out = sch.run(reqs)
    assert [r.summary["steps"] for r in out] == [50, 9, 30, 20]
    sizes = [n for n, key in zip(ex.chunk_sizes, ex.chunk_keys) if key == 32**3]
    assert sizes == [3, 2, 1]                     # the 32^3 class: 3 together, then 2 after rid 1, then rid 0 alone
    assert [n for n, key in zip(ex.chunk_sizes, ex.chunk_keys) if key == 48**3] == [1]


def test_stream_is_seeded_and_matches_its_distribution():
    a = serve.make_stream(256, 4.0, seed=5)
    b = serve.make_stream(256, 4.0, seed=5)
    assert [(r.arrival, r.case.name, r.nsteps) for r in a] == [(r.arrival, r.case.name, r.nsteps) for r in b]
    arr = np.array([r.arrival for r in a])
    assert np.all(np.diff(arr) > 0)
    assert abs(arr[-1] / 256 - 0.25) < 0.05                        # mean inter-arrival 1/4 s
    kinds = [r.case.name.startswith("tgv") for r in a]
    assert 0.4 < np.mean(kinds) < 0.6
    assert {r.case.cells[0] for r in a} <= set(serve.GRIDS)
    assert all(r.case.cells == (r.case.cells[0],) * 3 for r in a)
    assert all(200 <= r.nsteps <= 2000 for r in a)
    res = [1.0 / r.case.nu for r in a if r.case.name.startswith("tgv")]
    assert min(res) >= 400 - 1e-9 and max(res) <= 3200 + 1e-9
    chans = [r.case for r in a if not r.case.name.startswith("tgv")]
    assert all(c.y_bc_type == 1 and c.alpha_grid == 2.0 for c in chans)


def test_scheduler_completes_every_request_within_budget_in_order():
    reqs = serve.make_stream(64, 4.0, seed=11, steps=(20, 60))
    ex = FakeExecutor(rate=1e8)     # slow enough that cases overlap
    budget = 3 * 128**3 * ex.bpc     # room for about three of the largest cases at once
    sch = serve.Scheduler(ex, budget, chunk_cell_steps=1e6)
    out = sch.run(reqs)
    assert [r.rid for r in out] == sorted(r.rid for r in reqs)
    for r, q in zip(out, sorted(reqs, key=lambda x: x.rid)):
        assert r.summary["steps"] == q.nsteps                      # every step issued exactly once
        assert r.finished >= r.admitted >= r.arrival - 1e-12
    assert sch.peak_bytes <= budget
    assert ex.started == sorted(ex.started, key=lambda rid: reqs[rid].arrival)   # FIFO admission
    assert ex.max_live > 1                                          # cases overlap
    s = serve.summarize(out, max(r.finished for r in out))
    assert s["requests"] == 64 and s["p99_latency_s"] >= s["p50_latency_s"] > 0


def test_scheduler_rejects_a_request_larger_than_the_budget():
    reqs = serve.make_stream(3, 4.0, seed=3, grids=(128,), steps=(10, 10))
    ex = FakeExecutor()
    with pytest.raises(ValueError):
        serve.Scheduler(ex, 1000.0).run(reqs)


def test_percentile_nearest_rank():
    xs = list(range(1, 101))
    assert serve.percentile(xs, 50) == 50 and serve.percentile(xs, 99) == 99 and serve.percentile(xs, 100) == 100
