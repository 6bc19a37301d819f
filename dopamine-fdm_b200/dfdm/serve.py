"""Request loop for independent simulations on one GPU (continuous batching of whole cases).

A request is one case (grid, Reynolds number, initial-condition seed) and a step count.  Requests arrive over
time.  They are admitted in arrival order as soon as their device footprint (dfdm_footprint_bytes) fits in the
admission budget, and each admitted case stays resident in its own context on its own CUDA stream.  The loop
advances every active case by chunks of whole steps (one CUDA-graph replay per step).  Chunks of different cases
are enqueued on different streams, so their kernels overlap on the device.  A case that finishes returns its final
state to the host and gives its memory back to the budget, and the next waiting request takes its place.

The scheduling logic (Scheduler) is independent of the device: Scheduler.run drives an executor object, which the
GPU path implements with dfdm contexts (GpuExecutor) and the CPU tests implement with a simulated clock.

The synthetic request stream (make_stream) draws, from one seed, Poisson arrivals at a given rate.  Per request it
draws a case type (Taylor-Green or Re_tau = 180 channel, 50/50), a cubic grid N^3 with N in {32, 48, 64, 96, 128}
(channel: 4pi x 2 x 4pi/3, tanh 2.0), Re log-uniform in [400, 3200] for Taylor-Green, an initial-condition seed and
a step count uniform in [200, 2000].
"""
from __future__ import annotations

import math
import time
from collections import deque
from dataclasses import dataclass, field
from typing import Dict, List, Optional

import numpy as np

from . import cases
from .cases import Case

GRIDS = (32, 48, 64, 96, 128)


@dataclass
class Request:
    rid: int
    case: Case
    nsteps: int
    arrival: float          # seconds after the stream starts
    precision: str = "fp32"

    @property
    def cells(self) -> int:
        return self.case.n_cells

    @property
    def work(self) -> int:  # cell-steps
        return self.cells * self.nsteps


@dataclass
class Result:
    rid: int
    arrival: float
    admitted: float
    finished: float
    nsteps: int
    cells: int
    state: Optional[tuple] = None
    summary: Dict[str, float] = field(default_factory=dict)
    device_s: Optional[float] = None   # run_isolated: device time of the request's steps alone

    @property
    def latency(self) -> float:
        return self.finished - self.arrival


def serve_case(kind: str, N: int, Re: float, seed: int) -> Case:
    """One request's case: Taylor-Green in [0, 2pi]^3 or the Re_tau = 180 channel domain, on N^3 cells."""
    if kind == "tgv":
        c = cases.tgv(N=N, Re=Re, dt=1e-3, name=f"tgv{N}_Re{Re:.0f}")
        c.seed = seed
        return c
    c = cases.channel(N, N, N, 4.0 * math.pi, 4.0 * math.pi / 3.0, 2.0, 180.0, 15.6, 1e-3, seed, 0, f"chan{N}")
    return c


def make_stream(n: int = 256, rate: float = 4.0, seed: int = 5, grids=GRIDS, steps=(200, 2000),
                precision: str = "fp32") -> List[Request]:
    """The synthetic request stream: Poisson arrivals at `rate` per second, all draws from PCG64(seed)."""
    g = np.random.Generator(np.random.PCG64(seed))
    t = 0.0
    out = []
    for rid in range(n):
        t += g.exponential(1.0 / rate)
        kind = "tgv" if g.random() < 0.5 else "chan"
        N = int(grids[g.integers(0, len(grids))])
        Re = float(math.exp(g.uniform(math.log(400.0), math.log(3200.0))))
        ic_seed = int(g.integers(0, 2**31 - 1))
        nsteps = int(g.integers(steps[0], steps[1] + 1))
        out.append(Request(rid, serve_case(kind, N, Re, ic_seed), nsteps, t, precision))
    return out


def percentile(xs: List[float], q: float) -> float:
    """Nearest-rank percentile (q in [0, 100])."""
    if not xs:
        return float("nan")
    s = sorted(xs)
    k = max(0, min(len(s) - 1, int(math.ceil(q / 100.0 * len(s))) - 1))
    return s[k]


class Scheduler:
    """FIFO admission by device footprint, round-robin chunked stepping of the admitted cases.

    executor protocol:
      footprint(req) -> bytes            prepare(req)        (called at arrival; may start work in the background)
      start(req) -> handle               can_enqueue(handle) -> bool  (False while the case is still being set up)
      enqueue(handle, nsteps)            ready(handle) -> bool
      finish(handle, req, keep_state) -> (state, summary)
      reclaim() -> None                  (release the memory of finished cases; may wait for the device)
      now() -> seconds                   idle(seconds or None)        (wait for device progress or an arrival)
      defers_free: bool                  (finished cases hold their memory until reclaim())
    """

    def __init__(self, executor, budget_bytes: float, chunk_cell_steps: float = 2.5e7, max_active: int = 64,
                 keep_state: bool = False):
        self.ex = executor
        self.budget = float(budget_bytes)
        self.chunk_cell_steps = float(chunk_cell_steps)
        self.max_active = int(max_active)
        self.keep_state = keep_state
        self.peak_bytes = 0.0
        self.peak_active = 0
        self.reclaims = 0

    def chunk(self, req: Request, done: int) -> int:
        k = int(max(1, round(self.chunk_cell_steps / max(1, req.cells))))
        return min(k, req.nsteps - done)

    def run(self, requests: List[Request], t0: Optional[float] = None) -> List[Result]:
        ex = self.ex
        defers = getattr(ex, "defers_free", False)
        pending = deque(sorted(requests, key=lambda r: r.arrival))
        waiting: deque = deque()
        active: List[dict] = []
        results: List[Result] = []
        used = 0.0       # footprint of admitted, unfinished cases
        held = 0.0       # footprint of finished cases whose memory is not released yet
        start = ex.now() if t0 is None else t0
        while pending or waiting or active:
            now = ex.now() - start
            while pending and pending[0].arrival <= now:
                r = pending.popleft()
                fp = ex.footprint(r)
                if fp > self.budget:
                    raise ValueError(f"request {r.rid} needs {fp} bytes, more than the whole budget")
                ex.prepare(r)
                waiting.append((r, fp))
            # admission: arrival order, head of line waits until its footprint fits
            while waiting and len(active) < self.max_active:
                r, fp = waiting[0]
                if used + held + fp > self.budget and held > 0:
                    ex.reclaim()
                    held = 0.0
                    self.reclaims += 1
                if used + held + fp > self.budget:
                    break
                waiting.popleft()
                used += fp
                h = ex.start(r)
                active.append({"req": r, "h": h, "fp": fp, "done": 0, "inflight": 0, "admitted": ex.now() - start})
            self.peak_bytes = max(self.peak_bytes, used + held)
            self.peak_active = max(self.peak_active, len(active))
            progressed = False
            for a in list(active):
                r = a["req"]
                if a["inflight"] and not ex.ready(a["h"]):
                    continue
                if not a["inflight"] and not ex.can_enqueue(a["h"]):
                    continue
                a["done"] += a["inflight"]
                a["inflight"] = 0
                if a["done"] >= r.nsteps:
                    state, summary = ex.finish(a["h"], r, self.keep_state)
                    results.append(Result(r.rid, r.arrival, a["admitted"], ex.now() - start, r.nsteps, r.cells,
                                          state, summary))
                    used -= a["fp"]
                    if defers:
                        held += a["fp"]
                    active.remove(a)
                    progressed = True
                    continue
                k = self.chunk(r, a["done"])
                ex.enqueue(a["h"], k)
                a["inflight"] = k
                progressed = True
            if not progressed:
                nxt = pending[0].arrival - (ex.now() - start) if pending else None
                ex.idle(nxt)
        ex.reclaim()
        return sorted(results, key=lambda x: x.rid)


def summarize(results: List[Result], wall: float) -> Dict[str, float]:
    lat = [r.latency for r in results]
    work = sum(r.cells * r.nsteps for r in results)
    return {"requests": len(results), "p50_latency_s": percentile(lat, 50), "p99_latency_s": percentile(lat, 99),
            "mean_latency_s": float(np.mean(lat)) if lat else float("nan"), "cell_steps": float(work),
            "wall_s": wall, "throughput_cell_steps_per_s": work / wall if wall > 0 else float("nan")}


class GpuExecutor:
    """Executor on one GPU: one dfdm context (CUDA-graph steps) and one CUDA stream per admitted request.

    The host-side initial condition of a request is built on worker threads from the moment it arrives (no device
    memory is touched before admission); at admission another worker creates the context and uploads the state, so
    the loop keeps feeding the device meanwhile.  Finished contexts are kept until reclaim(): releasing device
    memory waits for the whole device, which would stall every other case.
    """

    defers_free = True

    def __init__(self, device: int = 0, graphs: bool = True, workers: int = 4):
        import torch
        from concurrent.futures import ThreadPoolExecutor
        from .native import Solver, footprint_bytes
        self.torch = torch
        self.Solver = Solver
        self._footprint = footprint_bytes
        self.device = device
        self.graphs = graphs
        self.ic_pool = ThreadPoolExecutor(max_workers=workers)
        self.setup_pool = ThreadPoolExecutor(max_workers=workers)
        self.ics: Dict[int, object] = {}
        self.finished: List = []
        self.streams: List = []     # CUDA streams of released contexts, reused

    def now(self) -> float:
        return time.perf_counter()

    def idle(self, until_next_arrival: Optional[float]) -> None:
        time.sleep(min(2e-4, max(0.0, until_next_arrival)) if until_next_arrival is not None else 2e-4)

    def footprint(self, req: Request) -> int:
        return self._footprint(req.case, req.precision)

    def prepare(self, req: Request) -> None:
        self.ics[req.rid] = self.ic_pool.submit(cases.initial_condition, req.case)

    def _setup(self, req: Request, ic, st):
        self.torch.cuda.set_device(self.device)
        s = self.Solver(req.case, req.precision, graphs=self.graphs, stream=st.cuda_stream)
        s.set_state(*ic.result())
        return s

    def start(self, req: Request):
        if req.rid not in self.ics:
            self.prepare(req)
        ic = self.ics.pop(req.rid)
        st = self.streams.pop() if self.streams else self.torch.cuda.Stream(device=self.device)
        return {"fut": self.setup_pool.submit(self._setup, req, ic, st), "s": None, "st": st,
                "ev": self.torch.cuda.Event()}

    def can_enqueue(self, h) -> bool:
        if h["s"] is None:
            if not h["fut"].done():
                return False
            h["s"] = h["fut"].result()
        return True

    def enqueue(self, h, nsteps: int) -> None:
        if "ev0" in h:
            h["ev0"].record(h["st"])
        h["s"].compute_time_step_RK3_async(nsteps)
        h["ev"].record(h["st"])

    def time_steps(self, h) -> None:
        """Time the next enqueue on the device (CUDA events around its steps on the case's stream)."""
        h["ev0"] = self.torch.cuda.Event(enable_timing=True)
        h["ev"] = self.torch.cuda.Event(enable_timing=True)

    def device_seconds(self, h) -> float:
        h["ev"].synchronize()
        return h["ev0"].elapsed_time(h["ev"]) * 1e-3

    def ready(self, h) -> bool:
        return h["ev"].query()

    def finish(self, h, req: Request, keep_state: bool):
        s = h["s"]
        summary = {"t": s.t, "kinetic_energy": s.kinetic_energy()}
        try:
            s.check_finite()
            summary["finite"] = 1.0
        except Exception:
            summary["finite"] = 0.0
        state = s.get_state() if keep_state else None
        self.finished.append((s, h["st"]))
        return state, summary

    def reclaim(self) -> None:
        for s, st in self.finished:
            s.close()
            self.streams.append(st)
        self.finished = []


class GroupScheduler:
    """FIFO admission by device footprint, as Scheduler; the admitted cases step TOGETHER, as one serving group.

    A case takes its first step on its own (set-up and the first projection), then joins the group: every chunk of
    steps is one group step of all joined cases (one grouped launch per kernel family, dfdm_group_create), k steps
    at a time, k = chunk_cell_steps / (the group's cells), cut at the first member to finish.  The composition
    changes when a case joins or finishes; the executor keeps one group (one captured graph) per composition.  Up
    to `depth` chunks are in flight, so the device works on one while the host prepares the next.

    executor protocol:
      footprint(req) -> bytes        prepare(req)          start(req) -> handle        can_enqueue(handle) -> bool
      first_step(handle) -> token    group_step([handle], k) -> token                  done(token) -> bool
      finish(handle, req, keep_state) -> (state, summary)   reclaim()   now()   idle(seconds or None)
      defers_free: bool
    """

    def __init__(self, executor, budget_bytes: float, chunk_cell_steps: float = 2.5e7, max_active: int = 256,
                 keep_state: bool = False, depth: int = 2):
        self.ex = executor
        self.budget = float(budget_bytes)
        self.chunk_cell_steps = float(chunk_cell_steps)
        self.max_active = int(max_active)
        self.keep_state = keep_state
        self.depth = int(depth)
        self.peak_bytes = 0.0
        self.peak_active = 0
        self.peak_group = 0
        self.reclaims = 0
        self.chunks = 0
        self.compositions = 0

    def chunk(self, members: List[dict]) -> int:
        cells = sum(a["req"].cells for a in members)
        k = int(max(1, round(self.chunk_cell_steps / max(1, cells))))
        return min([k] + [a["req"].nsteps - a["done"] for a in members])

    def run(self, requests: List[Request], t0: Optional[float] = None) -> List[Result]:
        ex = self.ex
        defers = getattr(ex, "defers_free", False)
        pending = deque(sorted(requests, key=lambda r: r.arrival))
        waiting: deque = deque()
        active: List[dict] = []
        inflight: List[tuple] = []      # (token, [(case, steps)], is a group chunk)
        results: List[Result] = []
        used = 0.0
        held = 0.0
        last = None
        start = ex.now() if t0 is None else t0
        while pending or waiting or active:
            now = ex.now() - start
            while pending and pending[0].arrival <= now:
                r = pending.popleft()
                fp = ex.footprint(r)
                if fp > self.budget:
                    raise ValueError(f"request {r.rid} needs {fp} bytes, more than the whole budget")
                ex.prepare(r)
                waiting.append((r, fp))
            while waiting and len(active) < self.max_active:
                r, fp = waiting[0]
                if used + held + fp > self.budget and held > 0:
                    ex.reclaim()
                    held = 0.0
                    self.reclaims += 1
                if used + held + fp > self.budget:
                    break
                waiting.popleft()
                used += fp
                active.append({"req": r, "h": ex.start(r), "fp": fp, "done": 0, "completed": 0, "joined": False,
                               "admitted": ex.now() - start})
            self.peak_bytes = max(self.peak_bytes, used + held)
            self.peak_active = max(self.peak_active, len(active))
            progressed = False
            # completed chunks (the group's chunks complete in order; first steps on their own streams)
            keep = []
            for item in inflight:
                if ex.done(item[0]):
                    for a, k in item[1]:
                        a["completed"] += k
                    progressed = True
                else:
                    keep.append(item)
            inflight = keep
            for a in list(active):
                r = a["req"]
                if a["completed"] >= r.nsteps:
                    state, summary = ex.finish(a["h"], r, self.keep_state)
                    results.append(Result(r.rid, r.arrival, a["admitted"], ex.now() - start, r.nsteps, r.cells,
                                          state, summary))
                    used -= a["fp"]
                    if defers:
                        held += a["fp"]
                    active.remove(a)
                    progressed = True
                elif not a["joined"] and ex.can_enqueue(a["h"]):
                    inflight.append((ex.first_step(a["h"]), [(a, 1)], False))
                    a["done"] = 1
                    a["joined"] = True
                    progressed = True
            members = [a for a in active if a["joined"] and a["done"] < a["req"].nsteps]
            if members and sum(1 for item in inflight if item[2]) < self.depth:
                k = self.chunk(members)
                key = tuple(a["req"].rid for a in members)
                if key != last:
                    self.compositions += 1
                    last = key
                inflight.append((ex.group_step([a["h"] for a in members], k), [(a, k) for a in members], True))
                for a in members:
                    a["done"] += k
                self.chunks += 1
                self.peak_group = max(self.peak_group, len(members))
                progressed = True
            if not progressed:
                nxt = pending[0].arrival - (ex.now() - start) if pending else None
                ex.idle(nxt)
        ex.reclaim()
        return sorted(results, key=lambda x: x.rid)


class GroupGpuExecutor(GpuExecutor):
    """GroupScheduler's executor on one GPU: one dfdm context and CUDA stream per admitted case (set-up, first step
    and the result transfer run there), and the group steps on one stream of their own, with one dfdm group (one
    captured graph per group step) per composition, kept while the composition lasts.

    The same object runs run_isolated: a case alone is a group of one on the case's own stream, so every result is
    bit-identical alone and in any mix."""

    def __init__(self, device: int = 0, workers: int = 4):
        super().__init__(device=device, graphs=False, workers=workers)
        from .native import Group
        self.Group = Group
        self.gstream = self.torch.cuda.Stream(device=device)
        self.groups: Dict[tuple, object] = {}
        self.retired: List[tuple] = []     # (group, event of its last chunk)

    def _event(self, stream):
        ev = self.torch.cuda.Event()
        ev.record(stream)
        return ev

    def first_step(self, h):
        self.can_enqueue(h)
        h["s"].compute_time_step_RK3_async(1)
        return self._event(h["st"])

    def _group(self, hs):
        key = tuple(id(h) for h in hs)
        g = self.groups.get(key)
        if g is None:
            # compositions not in use any more are released once their last chunk is done
            for k2 in list(self.groups):
                self.retired.append((self.groups.pop(k2), self._event(self.gstream)))
            g = self.Group([h["s"] for h in hs], stream=self.gstream.cuda_stream)
            self.groups[key] = g
        still = []
        for gr, ev in self.retired:
            if ev.query():
                gr.close()
            else:
                still.append((gr, ev))
        self.retired = still
        return g

    def group_step(self, hs, k: int):
        self._group(hs).step_async(k)
        return self._event(self.gstream)

    def done(self, token) -> bool:
        return token.query()

    # run_isolated: first step on the case's stream, then a group of one on the same stream
    def enqueue(self, h, nsteps: int) -> None:
        if "ev0" in h:
            h["ev0"].record(h["st"])
        h["s"].compute_time_step_RK3_async(1)
        if nsteps > 1:
            g = self.Group([h["s"]], stream=h["st"].cuda_stream)
            g.step_async(nsteps - 1)
            g.close()
        h["ev"].record(h["st"])

    def reclaim(self) -> None:
        for key in list(self.groups):
            self.groups.pop(key).close()
        for g, _ in self.retired:
            g.close()
        self.retired = []
        super().reclaim()


def run_isolated(executor, requests: List[Request], keep_state: bool = False) -> List[Result]:
    """Every request alone, back to back (the isolated-run reference for the loop's throughput): set-up, steps,
    result, in turn.  Each Result carries the device time of its steps alone (device_s: CUDA events around the
    steps on the case's own stream, set-up and transfers excluded) where the executor can time them."""
    out = []
    t0 = executor.now()
    timed = hasattr(executor, "time_steps")
    for r in requests:
        a = executor.now() - t0
        executor.prepare(r)
        h = executor.start(r)
        while not executor.can_enqueue(h):
            executor.idle(None)
        if timed:
            executor.time_steps(h)
        executor.enqueue(h, r.nsteps)
        while not executor.ready(h):
            executor.idle(None)
        dev = executor.device_seconds(h) if timed else None
        state, summary = executor.finish(h, r, keep_state)
        out.append(Result(r.rid, a, a, executor.now() - t0, r.nsteps, r.cells, state, summary, dev))
    executor.reclaim()
    return out


def measure_stream(executor, requests: List[Request], rank: int, world: int, gather, budget_bytes: float = 150e9,
                   saturated: int = 48, scheduler=None) -> Dict[str, object]:
    """The serving measurement on one rank of `world` replicas: rank r serves requests r::world of the stream.

    Returns the whole job's figures on every rank: p50/p99 latency from arrival to the result on the host over all
    ranks' requests, the stream's throughput, and the loop's throughput when saturated (the rank's first
    `saturated` requests all arriving at once) against the same requests run alone back to back.  `gather(obj)`
    returns the list of every rank's obj (all_gather_object under torch.distributed, [obj] alone).  `scheduler` is
    the loop's class (Scheduler, the default, or GroupScheduler with a GroupGpuExecutor)."""
    scheduler = scheduler or Scheduler
    mine = requests[rank::world]
    sch = scheduler(executor, budget_bytes)
    t0 = executor.now()
    res = sch.run(mine)
    wall = executor.now() - t0
    sub = [Request(r.rid, r.case, r.nsteps, 0.0, r.precision) for r in mine[:saturated]]
    iso = run_isolated(executor, sub)
    iso_wall = iso[-1].finished if iso else float("nan")
    # the isolated reference is the device time of each request's steps alone (set-up, uploads and results
    # excluded), so the ratio compares the loop against the device's throughput on one case at a time
    iso_dev = sum(r.device_s for r in iso) if iso and all(r.device_s is not None for r in iso) else iso_wall
    t0 = executor.now()
    scheduler(executor, budget_bytes).run(sub)
    sat_wall = executor.now() - t0
    work_sub = float(sum(r.work for r in sub))
    parts = gather({"rids": [r.rid for r in res], "lat": [r.latency for r in res],
                    "work": float(sum(r.work for r in mine)), "wall": wall,
                    "iso": work_sub / iso_dev if iso else 0.0, "iso_wall": work_sub / iso_wall if iso else 0.0,
                    "sat": work_sub / sat_wall if sub else 0.0,
                    "n_sub": len(sub), "finite": all(r.summary.get("finite", 1.0) == 1.0 for r in res),
                    "peak_active": sch.peak_active, "peak_bytes": sch.peak_bytes,
                    "peak_group": getattr(sch, "peak_group", 0), "compositions": getattr(sch, "compositions", 0)})
    lat = [x for p in parts for x in p["lat"]]
    rids = sorted(x for p in parts for x in p["rids"])
    iso_thr = sum(p["iso"] for p in parts)
    iso_wall_thr = sum(p["iso_wall"] for p in parts)
    sat_thr = sum(p["sat"] for p in parts)
    wall_max = max(p["wall"] for p in parts)
    return {"requests": len(lat), "rids": rids, "p50_latency_s": percentile(lat, 50),
            "p99_latency_s": percentile(lat, 99), "max_latency_s": max(lat) if lat else None,
            "stream_wall_s": wall_max, "stream_throughput_cell_steps_per_s": sum(p["work"] for p in parts) / wall_max,
            "saturated_requests": sum(p["n_sub"] for p in parts), "saturated_throughput_cell_steps_per_s": sat_thr,
            "isolated_throughput_cell_steps_per_s": iso_thr,
            "isolated_basis": "device time of each request's steps alone (CUDA events; set-up, transfers excluded)",
            "isolated_wall_throughput_cell_steps_per_s": iso_wall_thr,
            "saturated_over_isolated": sat_thr / iso_thr if iso_thr > 0 else None,
            "all_finite": all(p["finite"] for p in parts), "peak_active": max(p["peak_active"] for p in parts),
            "peak_group": max(p["peak_group"] for p in parts), "group_compositions": sum(p["compositions"] for p in parts),
            "peak_admitted_bytes": max(p["peak_bytes"] for p in parts), "admission_budget_bytes": budget_bytes}
