#!/usr/bin/env python
"""Throughput benchmark of the single-phase RK3 step: cell-RK3-steps/s, FP32-mixed vs plain FP64.

    python bench.py [--gpus N --steps K --warmup W] [--impl dfdm|reference] [--config chan550]

Workload (default): the Re_tau = 550 constant-flux channel DNS on 256 x 192 x 256 cells (tanh-stretched y,
periodic x/z), seeded Poiseuille + 10 % uniform-noise initial condition.  One step = one full
compute_time_step_RK3 (three stages: RHS + RK update, projection, constant-flux shift).  The state is resident
in HBM; the per-step working set (~0.6 GB FP32) exceeds the 126 MB L2, so no flush is needed between steps.

With N > 1 (torchrun) every rank advances its own independent replica of the case (the requests of the serving
loop shard this way; there is no data-path collective): value = N * cells * K / max-over-ranks(time).

`--impl reference` times the reference's algorithm on the host cores instead: the reference's Fortran/MPI build
cannot be built here, so this is the repository's FP64 C++ restatement (the oracle), OpenMP over all host cores,
on a bounded sample of the same workload (whole RK3 steps of the same grid, as many as fit in ~90 s).
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(ROOT, "dopamine-fdm_b200"))

import numpy as np  # noqa: E402

from dfdm import cases  # noqa: E402

METRIC = "cell-RK3-steps/s"
UNIT = "cell-steps/s"


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=100)
    ap.add_argument("--warmup", type=int, default=20)
    ap.add_argument("--impl", default="dfdm", choices=["dfdm", "reference"])
    ap.add_argument("--config", default="chan550")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--no-fp64", action="store_true")
    ap.add_argument("--no-kernels", action="store_true", help="skip the per-kernel roofline timings")
    ap.add_argument("--cpu-seconds", type=float, default=20.0)
    ap.add_argument("--no-serve", action="store_true", help="skip the serving-stream measurement")
    ap.add_argument("--no-adaptive", action="store_true", help="skip the adaptive-time-step run")
    ap.add_argument("--no-hybrid", action="store_true", help="skip the advection_scheme = 2 runs")
    ap.add_argument("--stage-kernel", choices=["auto", "one-cell", "pairs", "tma"], default="auto",
                    help="FP32 stage kernel: the autotuner's choice (default) or a fixed one (profiling runs, where the "
                         "serialised launches under a profiler skew the autotuner's timing)")
    ap.add_argument("--no-accuracy", action="store_true",
                    help="skip the report of every config's FP32 and FP64 results against the FP64 oracle")
    ap.add_argument("--oracle-steps", type=int, default=20,
                    help="steps of the bench workload compared with the oracle in the accuracy report (the other "
                         "configs use their own step counts; the full 120-step comparison is a GPU test)")
    ap.add_argument("--serve-requests", type=int, default=256)
    ap.add_argument("--serve-rate", type=float, default=4.0, help="Poisson arrival rate, requests/s")
    ap.add_argument("--serve-saturated", type=int, default=48,
                    help="requests of the saturated comparison (all arriving at once vs run alone back to back)")
    return ap.parse_args()


def dist_env():
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return ws, rank, local


def measured_peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        d = json.load(open(p))
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def workload_name(c):
    Nx, Ny, Nz = c.cells
    return f"{c.name}: {Nx}x{Ny}x{Nz} cells"


def data_desc(c):
    """The synthetic input of the workload: its seeded initial condition (there is no dataset)."""
    return {"poiseuille_uniform": "synthetic: seeded laminar Poiseuille + 10% uniform noise, no dataset",
            "reichardt_gauss": "synthetic: seeded Reichardt profile + Gaussian noise, no dataset",
            "tgv": "synthetic: Taylor-Green vortex, no dataset",
            "zero": "synthetic: fluid at rest, no dataset"}.get(c.ic, f"synthetic: initial condition {c.ic}, no dataset")


def config_dict(c, extra=None):
    d = {"workload": workload_name(c), "grid_faces": [c.nx, c.ny, c.nz], "cells": c.n_cells,
         "y": "walls, tanh alpha=%g" % c.alpha_grid if c.y_bc_type == 1 else "periodic",
         "nu": c.nu, "dt": c.dt, "sgs_model": c.sgs_model, "flow_forcing_mode": c.flow_forcing_mode,
         "ic": c.ic, "seed": c.seed, "l2": "per-step working set larger than the 126 MB L2 (no flush)"}
    if extra:
        d.update(extra)
    return d


# ---------------------------------------------------------------------------------------------------------------
class ClockSampler:
    """SM clocks and clock-event (throttle) reasons sampled during the timed region: NVML polled every 10 ms from a
    thread of this process (read-only queries), else nvidia-smi every 200 ms."""
    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
         "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
         "clocks_event_reasons.sw_power_cap")
    # NVML clock-event reason bits (nvml.h): sw_power_cap 0x4, hw_slowdown 0x8, sw_thermal 0x20, hw_thermal 0x40
    BITS = {"sw_power_cap": 0x4, "hw_slowdown": 0x8, "sw_thermal_slowdown": 0x20, "hw_thermal_slowdown": 0x40}

    def __init__(self, gpu_index: int):
        self.idx = gpu_index
        self.proc = None
        self.f = None
        self.nvml = None
        self.thread = None
        self.samples = []
        self.run = False

    def _nvml_handle(self):
        import pynvml
        pynvml.nvmlInit()
        try:   # the CUDA device's own UUID, so that CUDA_VISIBLE_DEVICES cannot map it to another GPU
            uuid = str(torch.cuda.get_device_properties(self.idx).uuid)
            return pynvml, pynvml.nvmlDeviceGetHandleByUUID(("GPU-" + uuid) if not uuid.startswith("GPU-") else uuid)
        except Exception:
            return pynvml, pynvml.nvmlDeviceGetHandleByIndex(self.idx)

    def start(self):
        try:
            nv, h = self._nvml_handle()
            self.nvml = (nv, h)
            smax = nv.nvmlDeviceGetMaxClockInfo(h, nv.NVML_CLOCK_SM)
            self.smax = float(smax)

            def poll():
                while self.run:
                    try:
                        sm = nv.nvmlDeviceGetClockInfo(h, nv.NVML_CLOCK_SM)
                        rs = nv.nvmlDeviceGetCurrentClocksEventReasons(h)
                        self.samples.append((float(sm), int(rs)))
                    except Exception:
                        pass
                    time.sleep(0.01)
            self.run = True
            self.thread = threading.Thread(target=poll, daemon=True)
            self.thread.start()
            return
        except Exception:
            self.nvml = None
        try:
            self.f = tempfile.NamedTemporaryFile("w+", suffix=".csv", delete=False)
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.idx), "--query-gpu=" + self.Q,
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=self.f, stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None

    def stop(self):
        if self.nvml:
            self.run = False
            self.thread.join(timeout=5)
            sm = [v for v, _ in self.samples]
            reasons = sorted(n for n, bit in self.BITS.items() if any(r & bit for _, r in self.samples))
            return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": self.smax, "reasons": reasons,
                    "samples": len(sm), "source": "NVML, every 10 ms"}
        if not self.proc:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        self.f.flush()
        self.f.seek(0)
        rows = [r.strip().split(",") for r in self.f.read().splitlines() if r.strip()]
        os.unlink(self.f.name)
        sm, smax, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for r in rows:
            r = [x.strip() for x in r]
            if len(r) < 9:
                continue
            try:
                sm.append(float(r[1]))
                smax = float(r[2])
            except ValueError:
                continue
            for n, v in zip(names, r[5:9]):
                if v.lower() == "active":
                    reasons.add(n)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": smax, "reasons": sorted(reasons),
                "samples": len(sm), "source": "nvidia-smi, every 200 ms"}


# ---------------------------------------------------------------------------------------------------------------
def run_reference(args, c):
    """Reference arm: the FP64 C++ restatement of the reference (oracle), OpenMP on all host cores."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle
    oracle.build()
    ncores = os.cpu_count() or 1
    oracle.set_threads(ncores)
    o = oracle.Oracle(c)
    U, V, W, P = cases.initial_condition(c)
    o.set_state(U, V, W, P)
    budget = 90.0
    nwarm = max(1, args.warmup)
    t0 = time.perf_counter()
    for w in range(nwarm):   # warm-up: first touch of every array, then as many as the run asks for
        o.step(1)
        if time.perf_counter() - t0 > budget / 3:
            nwarm = w + 1
            break
    t_first = time.perf_counter() - t0
    n = 0
    t0 = time.perf_counter()
    while n < max(1, args.steps):
        o.step(1)
        n += 1
        if time.perf_counter() - t0 + t_first > budget:
            break
    el = time.perf_counter() - t0
    value = c.n_cells * n / el
    sample = f"{n} full RK3 steps of the {workload_name(c)} case after {nwarm} warm-up step(s)"
    return {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": args.gpus, "steps": n, "warmup": nwarm,
            "ms_per_step": 1e3 * el / n, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "f64", "data": data_desc(c),
            "config": config_dict(c), "impl": "reference",
            "cpu_baseline": {"value": value, "unit": UNIT, "cores": ncores, "kind": "port", "sample": sample,
                             "note": "reference Fortran/MPI build unavailable on this box; FP64 C++ restatement"},
            "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}


def cpu_baseline(c, seconds):
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle
    oracle.build()
    ncores = os.cpu_count() or 1
    oracle.set_threads(ncores)
    o = oracle.Oracle(c)
    U, V, W, P = cases.initial_condition(c)
    o.set_state(U, V, W, P)
    n = 0
    t0 = time.perf_counter()
    while True:
        o.step(1)
        n += 1
        if time.perf_counter() - t0 > seconds:
            break
    el = time.perf_counter() - t0
    o.close()
    return {"value": c.n_cells * n / el, "unit": UNIT, "cores": ncores, "kind": "port",
            "sample": f"{n} full RK3 step(s) of the {workload_name(c)} case from the initial condition "
                      f"(FP64 C++ restatement, OpenMP on {ncores} threads)"}


# ---------------------------------------------------------------------------------------------------------------
def group_bench(local):
    """Serving groups against per-context graphs on one stream each: cell-steps/s of 20 steps of the same cases
    (CUDA events, best of 3), for 16 cases of 32^3, 16 of 64^3, a 16-case mix of 32^3-128^3 and 64 cases of 32^3
    (half Taylor-Green, half channel; a case's first steps taken before the timing)."""
    import torch
    from dfdm import cases, serve
    from dfdm.native import Group, Solver

    def ready(c):
        s = Solver(c, "fp32", graphs=True)
        s.set_state(*cases.initial_condition(c))
        s.compute_time_step_RK3(2)
        return s

    def best(fn, st, reps=3):
        """Device seconds of fn's work on the streams st: from an event on st[0] that every stream waits on, to an
        event on st[0] after every stream's work (best of reps)."""
        t = 1e9
        for _ in range(reps):
            torch.cuda.synchronize()
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(st[0])
            for x in st[1:]:
                x.wait_event(e0)
            fn()
            for x in st[1:]:
                ev = torch.cuda.Event()
                ev.record(x)
                st[0].wait_event(ev)
            e1.record(st[0])
            e1.synchronize()
            t = min(t, e0.elapsed_time(e1) * 1e-3)
        return t

    K = 20
    out = {}
    for label, grids, n in [("16x32^3", (32,), 16), ("16x64^3", (64,), 16), ("16-case mix 32^3-128^3", (32, 48, 64, 96, 128), 16),
                            ("64x32^3", (32,), 64)]:
        rng = np.random.default_rng(1)
        cs = [serve.serve_case("tgv" if q % 2 else "chan", int(rng.choice(grids)), 1000.0, q) for q in range(n)]
        cells = sum(c.n_cells for c in cs)
        per = [ready(c) for c in cs]
        pst = [torch.cuda.ExternalStream(s.stream_handle, device=local) for s in per]
        t_per = best(lambda: [s.compute_time_step_RK3_async(K) for s in per], pst)
        grp = [ready(c) for c in cs]
        g = Group(grp)
        g.step(1)
        gst = [torch.cuda.ExternalStream(g.stream_handle, device=local)]
        t_grp = best(lambda: g.step_async(K), gst)
        launches = g.launch_count()
        g.step(1)
        per_step = g.launch_count() - launches
        out[label] = {"cells": cells, "per_context_streams_cell_steps_per_s": cells * K / t_per,
                      "group_cell_steps_per_s": cells * K / t_grp, "group_over_per_context": t_per / t_grp,
                      "group_ms_per_step": t_grp / K * 1e3, "group_launches_per_step": per_step}
        g.close()
        for s in per + grp:
            s.close()
    return out


def serve_bench(args, local, rank, ws, gather):
    """The serving stream (256 requests, Poisson arrivals at 4/s, FP32-mixed, 150 GB admission budget) through the
    grouped loop (serve.GroupScheduler: the admitted cases of each shape class step as one serving group, one grouped
    launch per kernel family, the classes on streams of their own): p50/p99 latency from arrival to the result on the
    host, and the loop's throughput when saturated (median of 3 runs) against the same requests run alone back to
    back (device time of each alone, a group of one).  Beside it, the per-context loop (serve.Scheduler: one context,
    stream and step graph per case) on the same saturated requests.  With N ranks each serves requests rank::N of
    the stream."""
    from dfdm import serve
    warm = serve.make_stream(4, 100.0, seed=99, grids=(32, 48), steps=(10, 10))
    gex = serve.GroupGpuExecutor(device=local)
    serve.GroupScheduler(gex, 150e9).run(warm)
    reqs = serve.make_stream(args.serve_requests, args.serve_rate, seed=5)
    out = serve.measure_stream(gex, reqs, rank, ws, gather, 150e9, args.serve_saturated, serve.GroupScheduler)
    out.pop("rids")
    # the per-context loop on the same saturated requests (all arriving at once), repeated as the grouped loop's
    pex = serve.GpuExecutor(device=local)
    serve.Scheduler(pex, 150e9).run(warm)
    runs = serve.saturated_throughput(pex, serve.Scheduler, reqs[rank::ws][:args.serve_saturated], 150e9)
    per = sum(gather(float(np.median(runs))))
    out["group_steps"] = group_bench(local)
    out.update({"loop": "grouped per shape class (serve.GroupScheduler)", "arrival_rate_per_s": args.serve_rate,
                "precision": "fp32-mixed",
                "per_context_saturated_throughput_cell_steps_per_s": per,
                "per_context_saturated_runs_cell_steps_per_s": runs,
                "grouped_over_per_context_saturated": out["saturated_throughput_cell_steps_per_s"] / per,
                "stream": "seed 5: 50% Taylor-Green (Re log-uniform 400-3200), 50% Re_tau=180 channel domain; "
                          "N^3 cells, N in {32,48,64,96,128}; 200-2000 steps"})
    return out


def main():
    args = parse()
    ws, rank, local = dist_env()
    c = cases.get(args.config)
    if args.impl == "reference":
        if rank == 0:
            print(json.dumps(run_reference(args, c)), flush=True)
        return

    import torch
    import torch.distributed as dist
    from dfdm.native import KERNELS, Solver
    from dfdm.native import load as native_lib

    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    if ws > 1:
        from datetime import timedelta
        dist.init_process_group("nccl", timeout=timedelta(seconds=300), device_id=dev)
    stream = torch.cuda.Stream(device=dev)
    sh = stream.cuda_stream

    def barrier_sync():
        torch.cuda.synchronize()
        if ws > 1:
            dist.barrier()
        torch.cuda.synchronize()

    def max_over_ranks(x: float) -> float:
        if ws == 1:
            return x
        t = torch.tensor([x], dtype=torch.float64, device=dev)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        return float(t.item())

    U, V, W, P = cases.initial_condition(c)

    def timed_run(prec, sample_clocks=False, adaptive=False, case=None):
        s = Solver(case or c, prec, graphs=True)
        s.set_stream(sh)
        if prec == "fp32" and args.stage_kernel != "auto":
            s.set_stage_variant({"one-cell": 0, "pairs": 1, "tma": 2}[args.stage_kernel])
        s.set_state(U, V, W, P)
        if adaptive:
            s.set_adaptive_dt(True, 0.5, 0.9)
        s.compute_time_step_RK3(args.warmup)
        barrier_sync()
        l0 = s.launch_count()
        clk = ClockSampler(local) if sample_clocks else None
        if clk:
            clk.start()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        s.compute_time_step_RK3_async(args.steps)
        e1.record(stream)
        e1.synchronize()
        clocks = clk.stop() if clk else None
        ms = e0.elapsed_time(e1)
        barrier_sync()
        launches = s.launch_count() - l0
        return s, max_over_ranks(ms), clocks, launches

    s32, ms32, clocks, launches = timed_run("fp32", sample_clocks=True)
    variant, ms_one, ms_pairs = s32.stage_variant()
    value = ws * c.n_cells * args.steps / (ms32 / 1e3)
    out = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": ws, "steps": args.steps,
           "warmup": args.warmup, "ms_per_step": ms32 / args.steps, "higher_is_better": True, "scaling": "weak",
           "vs_baseline": None, "dtype": "fp32-mixed (FP32 fields/stencils/FFTs, FP64 y-solves and reductions)",
           "data": data_desc(c),
           "config": config_dict(c), "replicas": ws,
           "clocks": clocks, "gpu_launches": launches,
           "tuning": {"stage_kernel": ["one cell per thread", "packed FP32x2 pairs",
                                       "packed FP32x2 pairs, TMA plane tiles"][variant],
                      "stage_ms_one_cell": ms_one, "stage_ms_packed_pairs": ms_pairs,
                      "stage_ms_tma": s32.stage_timing(2)}}

    # ---- plain FP64 form and the FP32-vs-FP64 error after warmup + K steps from the same state ----
    if not args.no_fp64:
        s64, ms64, _, _ = timed_run("fp64")
        v64 = ws * c.n_cells * args.steps / (ms64 / 1e3)
        a = s32.get_state()
        b = s64.get_state()
        rel = {k: float(np.linalg.norm((x - y).ravel()) / max(np.linalg.norm(y.ravel()), 1e-300))
               for k, x, y in zip("UVWP", a, b)}
        out["fp64"] = {"value": v64, "ms_per_step": ms64 / args.steps,
                       "fp32_speedup": value / v64,
                       "rel_l2_fp32_vs_fp64": rel, "steps_compared": args.warmup + args.steps}
        s64.close()

    # ---- the same step with the adaptive time step (cfl_adaptive = 1): CFL maxima and dt choice on the device ----
    if not args.no_adaptive:
        sa, msa, _, la = timed_run("fp32", adaptive=True)
        out["adaptive_dt"] = {"value": ws * c.n_cells * args.steps / (msa / 1e3), "ms_per_step": msa / args.steps,
                              "overhead_ms_per_step": (msa - ms32) / args.steps, "gpu_launches": la,
                              "dt_last": sa.dt, "cfl_target": 0.5, "cfl_safety": 0.9}
        sa.close()

    # ---- the same step with advection_scheme = 2 (upwind-biased dissipation, orders 3 and 5) ----
    if not args.no_hybrid:
        hyb = {}
        for order in (3, 5):
            ch = c.with_(advection_scheme=2, adv_order=order, adv_beta0=0.05)
            sh_, msh, _, lh = timed_run("fp32", case=ch)
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            for _ in range(3):
                sh_.launch_kernel_async("hybrid", 2)
            e0.record(stream)
            for _ in range(20):
                sh_.launch_kernel_async("hybrid", 2)
            e1.record(stream)
            e1.synchronize()
            kms = e0.elapsed_time(e1) / 20
            kb = sh_.kernel_bytes("hybrid")
            hyb[f"order{order}"] = {"value": ws * c.n_cells * args.steps / (msh / 1e3), "ms_per_step": msh / args.steps,
                                    "gpu_launches": lh, "k_adv_hybrid_ms": kms,
                                    "k_adv_hybrid_GBps": kb / (kms * 1e-3) / 1e9}
            sh_.close()
        out["hybrid_scheme"] = hyb

    # ---- roofline: per-kernel-family device time of one stage, dominant family against HBM peak ----
    peak, peak_kind = measured_peaks()
    if args.no_kernels:
        s32.close()
        if rank == 0:
            print(json.dumps(out), flush=True)
        return
    fams = ["stage", "fwd_x", "fwd_z", "y_solve", "inv_z", "inv_x", "correct", "cfl"]
    if c.flow_forcing_mode == 1:
        fams.append("flux_shift")
    iters = 20
    kt = {}
    for fam in fams:
        for _ in range(3):
            s32.launch_kernel_async(fam, 2)
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(iters):
            s32.launch_kernel_async(fam, 2)
        e1.record(stream)
        e1.synchronize()
        ms = e0.elapsed_time(e1) / iters
        b = s32.kernel_bytes(fam)
        kt[fam] = {"ms": ms, "alg_bytes": b, "GBps": b / (ms * 1e-3) / 1e9, "frac": b / (ms * 1e-3) / 1e9 / peak}
    dom = max(kt, key=lambda k: kt[k]["ms"])
    # DRAM bytes (read + write) per launch of each kernel family from the committed ncu capture:
    # lines "<config> <family> <bytes>" in profiles/traffic.txt
    traffic = None
    tfile = os.path.join(ROOT, "profiles", "traffic.txt")
    if os.path.exists(tfile):
        for line in open(tfile):
            f = line.split()
            if len(f) >= 3 and not line.startswith("#") and f[0] == c.name and f[1] == dom:
                traffic = float(f[2])
    out["roofline"] = {"bound": "hbm", "kernel": dom, "achieved": kt[dom]["GBps"], "peak": peak, "unit": "GB/s",
                       "frac": kt[dom]["GBps"] / peak, "traffic": traffic, "peak_kind": peak_kind,
                       "alg_bytes_per_launch": kt[dom]["alg_bytes"], "avg_launch_ms": kt[dom]["ms"]}
    # whole-step roofline of the M1 model: 88 words per cell-step + 2 for the constant-flux shift
    words = 88 + (2 if c.flow_forcing_mode == 1 else 0)
    step_bytes = words * 4 * c.n_cells
    out["step_roofline"] = {"model": f"M1 {words} words/cell-step", "bytes_per_step": step_bytes,
                            "achieved_GBps": step_bytes / (ms32 / args.steps * 1e-3) / 1e9,
                            "frac_of_peak": step_bytes / (ms32 / args.steps * 1e-3) / 1e9 / peak}
    out["kernels"] = kt

    # ---- end to end through the C ABI with host buffers (the reference's FP64 ghosted arrays, pinned) ----
    if not args.no_e2e:
        shp = c.shapes()

        def pinned(key):
            n1, n2, n3 = shp[key]
            t = torch.empty((n3, n2, n1), dtype=torch.float64, pin_memory=True)
            return t.numpy().T   # Fortran-ordered view of pinned memory

        hU, hV, hW, hP = pinned("U"), pinned("V"), pinned("W"), pinned("P")
        hU[...] = U; hV[...] = V; hW[...] = W; hP[...] = P
        oU, oV, oW, oP = pinned("U"), pinned("V"), pinned("W"), pinned("P")
        ne = max(1, min(args.steps, 10))
        s32.set_state(hU, hV, hW, hP)
        s32.compute_time_step_RK3(1)
        barrier_sync()
        # synchronous calls: upload, step, download, one after the other
        t0 = time.perf_counter()
        for _ in range(ne):
            s32.set_state(hU, hV, hW)                 # H2D of the step's input state
            s32.compute_time_step_RK3(1)
            s32.get_state((oU, oV, oW, oP))           # D2H of the step's result
        ms_sync = max_over_ranks((time.perf_counter() - t0) * 1e3)
        # the asynchronous calls: one step's download overlaps the next step's upload (one copy engine each way);
        # every step still uploads its input and downloads its result, and the clock stops after the last one.  One
        # untimed iteration first: the context makes its copy streams and staging buffers on first use (about 800 MB
        # of device allocations at this size, timed separately as setup_ms)
        barrier_sync()
        t0 = time.perf_counter()
        s32.set_state_async(hU, hV, hW)
        s32.compute_time_step_RK3_async(1)
        s32.get_state_async((oU, oV, oW, oP))
        s32.synchronize()
        setup_ms = (time.perf_counter() - t0) * 1e3
        barrier_sync()
        t0 = time.perf_counter()
        for _ in range(ne):
            s32.set_state_async(hU, hV, hW)
            s32.compute_time_step_RK3_async(1)
            s32.get_state_async((oU, oV, oW, oP))
        s32.synchronize()
        ms_e = max_over_ranks((time.perf_counter() - t0) * 1e3)
        bi = 8 * (hU.size + hV.size + hW.size)
        bo = 8 * (oU.size + oV.size + oW.size + oP.size)
        out["e2e"] = {"value": ws * c.n_cells * ne / (ms_e / 1e3), "unit": UNIT, "h2d_bytes_per_step": bi,
                      "d2h_bytes_per_step": bo, "steps": ne,
                      "path": "dfdm_set_state_async(U,V,W) + dfdm_compute_time_step_rk3_async(1) + "
                              "dfdm_get_state_async(U,V,W,P) per step, then dfdm_synchronize; FP64 ghosted host "
                              "arrays in pinned memory; host wall clock; after one untimed iteration that sets the "
                              "asynchronous transfers up",
                      "first_iteration_with_setup_ms": setup_ms,
                      "synchronous_calls": {"value": ws * c.n_cells * ne / (ms_sync / 1e3),
                                            "path": "dfdm_set_state + dfdm_compute_time_step_rk3(1) + dfdm_get_state "
                                                    "per step"}}

    # ---- every config at its stated step count: FP32-mixed and FP64 against the FP64 oracle and each other ----
    if not args.no_accuracy and rank == 0:
        sys.path.insert(0, os.path.join(ROOT, "oracle"))
        import oracle
        oracle.build()
        oracle.set_threads(os.cpu_count() or 1)

        def rel_l2(a, b):
            return {k: float(np.linalg.norm((x - y).ravel()) / max(np.linalg.norm(y.ravel()), 1e-300))
                    for k, x, y in zip("UVWP", a, b)}

        acc = {}
        runs = [("tgv64", None), ("chan180", None), ("les395", None), (args.config, args.oracle_steps)]
        for name, nsteps in runs:
            cc = cases.get(name)
            nsteps = cc.nsteps if nsteps is None else nsteps
            st = cases.initial_condition(cc)
            res = {}
            for prec in ("fp32", "fp64"):
                sv = Solver(cc, prec, graphs=True)
                sv.set_stream(sh)
                sv.set_state(*st)
                torch.cuda.synchronize()
                a0 = torch.cuda.Event(enable_timing=True)
                a1 = torch.cuda.Event(enable_timing=True)
                a0.record(stream)
                sv.compute_time_step_RK3_async(nsteps)
                a1.record(stream)
                a1.synchronize()
                res[prec] = (sv.get_state(), cc.n_cells * nsteps / (a0.elapsed_time(a1) * 1e-3))
                sv.close()
            o = oracle.Oracle(cc)
            o.set_state(*st)
            t0 = time.perf_counter()
            o.step(nsteps)
            t_oracle = time.perf_counter() - t0
            want = o.get_state()
            o.close()
            acc[name] = {"steps": nsteps, "cells": cc.n_cells,
                         "rel_l2_fp32_vs_oracle": rel_l2(res["fp32"][0], want),
                         "rel_l2_fp64_vs_oracle": rel_l2(res["fp64"][0], want),
                         "rel_l2_fp32_vs_fp64": rel_l2(res["fp32"][0], res["fp64"][0]),
                         "fp32_cell_steps_per_s": res["fp32"][1], "fp64_cell_steps_per_s": res["fp64"][1],
                         "oracle_s": t_oracle,
                         "note": "timing includes the first (ungraphed) step and the graph capture"}
        acc["bars"] = {"fp64_vs_oracle": 1e-12, "fp32_vs_oracle": 1e-5,
                       "oracle": "FP64 C++ restatement of the reference, same grid, initial condition and dt"}
        out["accuracy"] = acc

        def poisson_call_time(fn):
            """Best of 3 batches of 10 calls, after 3 warm-up calls (seconds per call, host wall clock)."""
            for _ in range(3):
                fn()
            best = 1e30
            for _ in range(3):
                t0 = time.perf_counter()
                for _ in range(10):
                    fn()
                best = min(best, (time.perf_counter() - t0) / 10)
            return best

        def pinned_solve(sv, rhs):
            """dfdm_solve_poisson from and to page-locked copies of rhs (the C call a host with pinned arrays makes)."""
            import ctypes
            pin_in = torch.from_numpy(rhs.ravel(order="K")).pin_memory()
            pin_out = torch.empty_like(pin_in).pin_memory()
            P = ctypes.POINTER(ctypes.c_double)
            lib = native_lib()
            call = lambda: lib.dfdm_solve_poisson(sv.h, ctypes.cast(pin_in.data_ptr(), P),   # noqa: E731
                                                  ctypes.cast(pin_out.data_ptr(), P))
            if call() != 0:
                raise RuntimeError("dfdm_solve_poisson from pinned arrays failed")
            return call

        # the DCT-IV pressure solve of an inflow/outflow-x grid (257 x 128 x 128 independent cells)
        cc = cases.inflow_outflow(258, 129, 130, grid_type=2)
        rhs = np.asfortranarray(np.random.default_rng(258).standard_normal(cc.shapes()["rhs_p"]))
        o = oracle.Oracle(cc)
        t0 = time.perf_counter()
        want = o.solve_poisson(rhs)
        t_oracle = time.perf_counter() - t0
        o.close()
        N, nzp = cc.nx - 1, cc.nz - 2
        cells = N * (cc.ny - 1) * nzp
        io = {"grid": [N, cc.ny - 1, nzp], "oracle_s_per_solve": t_oracle,
              "path": "dfdm_solve_poisson (FP64 pageable host arrays in and out, the output array reused, synchronous), "
                      "host wall clock, best of 3 batches of 10 after 3 warm-up calls; pinned: the same from page-locked "
                      "arrays"}
        for prec in ("fp32", "fp64"):
            with Solver(cc, prec) as sv:
                got = np.zeros_like(rhs, order="F")
                best = poisson_call_time(lambda: sv.solve_poisson_equation(rhs, out=got))
                best_pinned = poisson_call_time(pinned_solve(sv, rhs))
            err = float(np.linalg.norm((got[:N, :, :nzp] - want[:N, :, :nzp]).ravel()) /
                        np.linalg.norm(want[:N, :, :nzp].ravel()))
            io[prec] = {"ms_per_solve": best * 1e3, "cells_per_s": cells / best, "rel_l2_vs_oracle": err,
                        "pinned_ms_per_solve": best_pinned * 1e3}
        out["inflow_outflow_poisson"] = io

        # the 4-wall duct's pressure solve (256 x 128 x 129 independent cells); its right-hand side is the discrete
        # operator applied to a seeded random field, so that it lies in the operator's range
        cc = cases.duct(258, 129, 130, grid_type=2)
        o = oracle.Oracle(cc)
        rng = np.random.default_rng(130)
        rhs = np.asfortranarray(rng.standard_normal(cc.shapes()["rhs_p"]))
        Nx, Ny, Nz = cc.nx - 2, cc.ny - 1, cc.nz - 1
        q = rng.standard_normal((Nx, Ny, Nz))
        dx = o.grid_array(7)[0]
        dy, ly, uy = o.grid_array(5), o.grid_array(8), o.grid_array(9)
        dzz, lz, uz = o.grid_array(10), o.grid_array(11), o.grid_array(12)
        a = (np.roll(q, -1, axis=0) - 2.0 * q + np.roll(q, 1, axis=0)) / dx**2 + dy[None, :, None] * q + dzz[None, None, :] * q
        a[:, 1:, :] += ly[None, 1:, None] * q[:, :-1, :]
        a[:, :-1, :] += uy[None, :-1, None] * q[:, 1:, :]
        a[:, :, 1:] += lz[None, None, 1:] * q[:, :, :-1]
        a[:, :, :-1] += uz[None, None, :-1] * q[:, :, 1:]
        rhs[:Nx, :Ny, :Nz] = a
        t0 = time.perf_counter()
        want = o.solve_poisson(rhs)
        t_oracle = time.perf_counter() - t0
        o.close()
        dp = {"grid": [Nx, Ny, Nz], "oracle_s_per_solve": t_oracle, "path": io["path"]}
        for prec in ("fp32", "fp64"):
            with Solver(cc, prec) as sv:
                got = np.zeros_like(rhs, order="F")
                best = poisson_call_time(lambda: sv.solve_poisson_equation(rhs, out=got))
                best_pinned = poisson_call_time(pinned_solve(sv, rhs))
            err = float(np.linalg.norm((got[:Nx, :, :Nz] - want[:Nx, :, :Nz]).ravel()) /
                        np.linalg.norm(want[:Nx, :, :Nz].ravel()))
            dp[prec] = {"ms_per_solve": best * 1e3, "cells_per_s": Nx * Ny * Nz / best, "rel_l2_vs_oracle": err,
                        "pinned_ms_per_solve": best_pinned * 1e3}
        out["duct_poisson"] = dp

        # spanwise walls alone (256 x 128 x 129 independent cells: periodic x and y, z walls)
        cc = cases.spanwise_wall(258, 130, 130)
        o = oracle.Oracle(cc)
        rng = np.random.default_rng(131)
        rhs = np.asfortranarray(rng.standard_normal(cc.shapes()["rhs_p"]))
        t0 = time.perf_counter()
        want = o.solve_poisson(rhs)
        t_oracle = time.perf_counter() - t0
        o.close()
        Nx, nyp, Nz = cc.nx - 2, cc.ny - 2, cc.nz - 1
        sw = {"grid": [Nx, nyp, Nz], "oracle_s_per_solve": t_oracle, "path": io["path"]}
        for prec in ("fp32", "fp64"):
            with Solver(cc, prec) as sv:
                got = np.zeros_like(rhs, order="F")
                best = poisson_call_time(lambda: sv.solve_poisson_equation(rhs, out=got))
                best_pinned = poisson_call_time(pinned_solve(sv, rhs))
            err = float(np.linalg.norm((got[:Nx, :nyp, :Nz] - want[:Nx, :nyp, :Nz]).ravel()) /
                        np.linalg.norm(want[:Nx, :nyp, :Nz].ravel()))
            sw[prec] = {"ms_per_solve": best * 1e3, "cells_per_s": Nx * nyp * Nz / best, "rel_l2_vs_oracle": err,
                        "pinned_ms_per_solve": best_pinned * 1e3}
        out["spanwise_wall_poisson"] = sw

    # ---- serving stream ----
    if not args.no_serve:
        def gather(obj):
            if ws == 1:
                return [obj]
            parts = [None] * ws
            dist.all_gather_object(parts, obj)
            return parts
        out["serve"] = serve_bench(args, local, rank, ws, gather)

    # ---- CPU baseline: the FP64 restatement on the host cores (rank 0 at N = 1 only) ----
    if rank == 0 and ws == 1 and not args.no_cpu:
        out["cpu_baseline"] = cpu_baseline(c, args.cpu_seconds)

    s32.close()
    if rank == 0:
        print(json.dumps(out), flush=True)
    if ws > 1:
        dist.barrier()
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
