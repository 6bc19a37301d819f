"""The N-GPU replica path of the serving measurement, as world_size-2 gloo ranks on CPU: each rank serves requests
rank::N of the stream on its own (simulated) device, and every rank ends with the whole job's figures."""
import os
import socket

import pytest
import torch.distributed as dist
import torch.multiprocessing as mp

from dfdm import serve
from test_serve import FakeExecutor


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, q):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        reqs = serve.make_stream(40, 4.0, seed=8, steps=(20, 50))

        def gather(obj):
            parts = [None] * world
            dist.all_gather_object(parts, obj)
            return parts

        out = serve.measure_stream(FakeExecutor(rate=2e8), reqs, rank, world, gather, budget_bytes=2e9, saturated=6)
        q.put((rank, out))
    finally:
        dist.destroy_process_group()


def test_two_replicas_split_the_stream_and_agree_on_the_job_figures():
    world = 2
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    got = dict(q.get(timeout=120) for _ in range(world))
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    a, b = got[0], got[1]
    assert a["rids"] == list(range(40))                  # every request served exactly once, across the ranks
    assert a["requests"] == 40 and a["saturated_requests"] == 12
    for key in ("p50_latency_s", "p99_latency_s", "saturated_throughput_cell_steps_per_s",
                "isolated_throughput_cell_steps_per_s", "stream_wall_s"):
        assert a[key] == pytest.approx(b[key])            # the same whole-job figures on every rank
    assert a["p99_latency_s"] >= a["p50_latency_s"] > 0
