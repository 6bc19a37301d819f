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

    Each context runs on the non-blocking stream dfdm_create makes for it (wrapped in torch.cuda.ExternalStream for
    the events); streams from torch's pool would not do, since the pool hands out a fixed set of streams in turn, so
    that with more cases than the pool holds two contexts would share one stream and a set-up on a worker thread
    could land inside another context's graph capture.

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

    def now(self) -> float:
        return time.perf_counter()

    def idle(self, until_next_arrival: Optional[float]) -> None:
        time.sleep(min(2e-4, max(0.0, until_next_arrival)) if until_next_arrival is not None else 2e-4)

    def footprint(self, req: Request) -> int:
        return self._footprint(req.case, req.precision)

    def prepare(self, req: Request) -> None:
        self.ics[req.rid] = self.ic_pool.submit(cases.initial_condition, req.case)

    def _setup(self, req: Request, ic):
        self.torch.cuda.set_device(self.device)
        s = self.Solver(req.case, req.precision, graphs=self.graphs)
        s.set_state(*ic.result())
        return s

    def start(self, req: Request):
        if req.rid not in self.ics:
            self.prepare(req)
        ic = self.ics.pop(req.rid)
        return {"fut": self.setup_pool.submit(self._setup, req, ic), "s": None, "st": None,
                "ev": self.torch.cuda.Event()}

    def can_enqueue(self, h) -> bool:
        if h["s"] is None:
            if not h["fut"].done():
                return False
            h["s"] = h["fut"].result()
            h["st"] = self.torch.cuda.ExternalStream(h["s"].stream_handle, device=self.device)
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
        self.finished.append(s)
        return state, summary

    def reclaim(self) -> None:
        for s in self.finished:
            s.close()
        self.finished = []


class GroupScheduler:
    """FIFO admission by device footprint, as Scheduler; the admitted cases step in serving groups.

    A case takes its first step on its own (set-up and the first projection), then joins the group of its shape
    class (grid and boundary type; executor.shape_class): every chunk of a class is one group step of all its joined
    cases (one grouped launch per kernel family, dfdm_group_create), k steps at a time, k = chunk_cell_steps / (the
    class's cells), cut at the class's first member to finish.  Each class steps on its own stream with up to `depth`
    chunks in flight, so classes share the device in cell-steps as the per-context loop's cases do, while the cases
    of a class share their launches.  by_class=False puts every joined case in one group instead.  A composition
    changes when a case joins or finishes; the executor keeps one group (one captured graph) per composition.

    executor protocol:
      footprint(req) -> bytes        prepare(req)          start(req) -> handle        can_enqueue(handle) -> bool
      shape_class(handle) -> key     first_step(handle) -> token
      group_step([handle], k, key) -> token                 done(token) -> bool
      finish(handle, req, keep_state) -> (state, summary)   reclaim()   now()   idle(seconds or None)
      defers_free: bool
    """

    def __init__(self, executor, budget_bytes: float, chunk_cell_steps: float = 2.5e7, max_active: int = 256,
                 keep_state: bool = False, depth: int = 2, by_class: bool = True):
        self.ex = executor
        self.budget = float(budget_bytes)
        self.chunk_cell_steps = float(chunk_cell_steps)
        self.max_active = int(max_active)
        self.keep_state = keep_state
        self.depth = int(depth)
        self.by_class = by_class
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
        inflight: List[tuple] = []      # (token, [(case, steps)], class key or None for a first step)
        results: List[Result] = []
        used = 0.0
        held = 0.0
        last: Dict[object, tuple] = {}  # class -> its last composition
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
            # completed chunks (a class's chunks complete in order; first steps on the cases' own streams)
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
                    inflight.append((ex.first_step(a["h"]), [(a, 1)], None))
                    a["done"] = 1
                    a["joined"] = True
                    a["class"] = ex.shape_class(a["h"]) if self.by_class else 0
                    progressed = True
            classes: Dict[object, List[dict]] = {}
            for a in active:
                if a["joined"] and a["done"] < a["req"].nsteps:
                    classes.setdefault(a["class"], []).append(a)
            busy: Dict[object, int] = {}
            for item in inflight:
                if item[2] is not None:
                    busy[item[2]] = busy.get(item[2], 0) + 1
            for key, members in classes.items():
                if busy.get(key, 0) >= self.depth:
                    continue
                k = self.chunk(members)
                comp = tuple(a["req"].rid for a in members)
                if last.get(key) != comp:
                    self.compositions += 1
                    last[key] = comp
                inflight.append((ex.group_step([a["h"] for a in members], k, key), [(a, k) for a in members], key))
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
    and the result transfer run there); each shape class steps in one dfdm group per composition (one captured graph
    per group step, on the group's own stream), kept while the composition lasts.

    The same object runs run_isolated: a case alone is a group of one on the case's own stream, so every result is
    bit-identical alone and in any mix."""

    def __init__(self, device: int = 0, workers: int = 4):
        super().__init__(device=device, graphs=False, workers=workers)
        from .native import Group
        self.Group = Group
        self.groups: Dict[object, tuple] = {}       # class -> (composition, group, its stream)
        self.retired: List[tuple] = []              # (group, event after its last chunk)

    def _event(self, stream):
        ev = self.torch.cuda.Event()
        ev.record(stream)
        return ev

    def shape_class(self, h):
        c = h["s"].case
        return (c.nx, c.ny, c.nz, c.y_bc_type)

    def first_step(self, h):
        self.can_enqueue(h)
        h["s"].compute_time_step_RK3_async(1)
        return self._event(h["st"])

    def _group(self, hs, key):
        comp = tuple(id(h) for h in hs)
        cur = self.groups.get(key)
        if cur is None or cur[0] != comp:
            if cur is not None:   # released once its last chunk is done
                self.retired.append((cur[1], self._event(cur[2])))
            g = self.Group([h["s"] for h in hs])
            cur = self.groups[key] = (comp, g, self.torch.cuda.ExternalStream(g.stream_handle, device=self.device))
        still = []
        for gr, ev in self.retired:
            if ev.query():
                gr.close()
            else:
                still.append((gr, ev))
        self.retired = still
        return cur[1], cur[2]

    def group_step(self, hs, k: int, key=0):
        g, st = self._group(hs, key)
        g.step_async(k)
        return self._event(st)

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
            self.groups.pop(key)[1].close()
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


def saturated_throughput(executor, scheduler, requests: List[Request], budget_bytes: float = 150e9,
                         reps: int = 3) -> List[float]:
    """Cell-steps/s of the loop with every request arriving at once, `reps` times (wall clock of each run)."""
    sub = [Request(r.rid, r.case, r.nsteps, 0.0, r.precision) for r in requests]
    work = float(sum(r.work for r in sub))
    out = []
    for _ in range(reps):
        t0 = executor.now()
        scheduler(executor, budget_bytes).run(sub)
        out.append(work / (executor.now() - t0))
    return out


def measure_stream(executor, requests: List[Request], rank: int, world: int, gather, budget_bytes: float = 150e9,
                   saturated: int = 48, scheduler=None, reps: int = 3) -> Dict[str, object]:
    """The serving measurement on one rank of `world` replicas: rank r serves requests r::world of the stream.

    Returns the whole job's figures on every rank: p50/p99 latency from arrival to the result on the host over all
    ranks' requests, the stream's throughput, and the loop's throughput when saturated (the rank's first
    `saturated` requests all arriving at once) against the same requests run alone back to back.  `gather(obj)`
    returns the list of every rank's obj (all_gather_object under torch.distributed, [obj] alone).  `scheduler` is
    the loop's class (Scheduler, the default, or GroupScheduler with a GroupGpuExecutor).  The saturated run is
    repeated `reps` times and its median reported: its wall time varies by some 20% from run to run with the order in
    which the cases' set-ups complete."""
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
    sat_runs = saturated_throughput(executor, scheduler, sub, budget_bytes, reps) if sub else [0.0]
    work_sub = float(sum(r.work for r in sub))
    parts = gather({"rids": [r.rid for r in res], "lat": [r.latency for r in res],
                    "work": float(sum(r.work for r in mine)), "wall": wall,
                    "iso": work_sub / iso_dev if iso else 0.0, "iso_wall": work_sub / iso_wall if iso else 0.0,
                    "sat": float(np.median(sat_runs)), "sat_runs": sat_runs,
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
            "saturated_runs_cell_steps_per_s": [sum(x) for x in zip(*[p["sat_runs"] for p in parts])],
            "isolated_throughput_cell_steps_per_s": iso_thr,
            "isolated_basis": "device time of each request's steps alone (CUDA events; set-up, transfers excluded)",
            "isolated_wall_throughput_cell_steps_per_s": iso_wall_thr,
            "saturated_over_isolated": sat_thr / iso_thr if iso_thr > 0 else None,
            "all_finite": all(p["finite"] for p in parts), "peak_active": max(p["peak_active"] for p in parts),
            "peak_group": max(p["peak_group"] for p in parts), "group_compositions": sum(p["compositions"] for p in parts),
            "peak_admitted_bytes": max(p["peak_bytes"] for p in parts), "admission_budget_bytes": budget_bytes}
