"""The request loop on the GPU: every result is the same alone and in the mix."""
import numpy as np
import pytest

from dfdm import serve

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("seed,grids,n", [(21, (32, 48), 8), (1, (48, 64, 96, 128), 10)])
def test_results_alone_equal_results_in_the_mix(seed, grids, n):
    """Each result is bit-identical alone and in the mix: small grids, and a mix that reaches 96^3 and 128^3 with
    several channel and Taylor-Green cases."""
    reqs = serve.make_stream(n, rate=200.0, seed=seed, grids=grids, steps=(20, 60))
    kinds = {r.case.name[:3] for r in reqs}
    assert kinds == {"tgv", "cha"}
    if max(grids) >= 96:
        assert {96, 128} <= {r.case.cells[0] for r in reqs}
    mix = serve.Scheduler(serve.GpuExecutor(), 150e9, chunk_cell_steps=2e5, keep_state=True)
    got = mix.run(reqs)
    assert mix.peak_active > 1
    alone = serve.run_isolated(serve.GpuExecutor(), reqs, keep_state=True)
    assert [r.rid for r in got] == [r.rid for r in alone]
    assert all(r.device_s is not None and r.device_s > 0 for r in alone)
    for a, b in zip(got, alone):
        assert a.summary["finite"] == 1.0
        for x, y in zip(a.state, b.state):
            assert np.array_equal(x, y), a.rid
        assert a.summary["kinetic_energy"] == b.summary["kinetic_energy"]


@pytest.mark.parametrize("seed,grids,n,by_class", [(21, (32, 48), 8, True), (1, (48, 64, 96, 128), 10, True),
                                                   (1, (48, 64, 96, 128), 10, False)])
def test_grouped_loop_results_alone_equal_results_in_the_mix(seed, grids, n, by_class):
    """The grouped loop (one group per shape class, or one group for all): each case steps inside serving groups
    whose composition changes as cases join and finish; every result is bit-identical to the case alone (a group of
    one) and agrees with the per-context loop to FP32 rounding."""
    reqs = serve.make_stream(n, rate=200.0, seed=seed, grids=grids, steps=(20, 60))
    ex = serve.GroupGpuExecutor()
    mix = serve.GroupScheduler(ex, 150e9, chunk_cell_steps=2e5, keep_state=True, by_class=by_class)
    got = mix.run(reqs)
    assert mix.compositions > 2
    if not by_class:
        assert mix.peak_group > 1
    alone = serve.run_isolated(serve.GroupGpuExecutor(), reqs, keep_state=True)
    per_ctx = serve.run_isolated(serve.GpuExecutor(), reqs, keep_state=True)
    assert [r.rid for r in got] == [r.rid for r in alone] == [r.rid for r in per_ctx]
    for a, b, c in zip(got, alone, per_ctx):
        assert a.summary["finite"] == 1.0
        for x, y, z in zip(a.state, b.state, c.state):
            assert np.array_equal(x, y), a.rid
            assert np.linalg.norm((x - z).ravel()) <= 1e-5 * np.linalg.norm(z.ravel()), a.rid
        assert a.summary["t"] == c.summary["t"]


@pytest.mark.parametrize("name,prec",[("chan180", "fp32"), ("chan180", "fp64"), ("tgv64", "fp32"), ("les395", "fp32")])
def test_footprint_bounds_the_device_memory_of_a_context(name, prec):
    """Admission relies on dfdm_footprint_bytes being an upper bound of what a stepping context holds."""
    import torch
    from dfdm import cases
    from dfdm.native import Solver, footprint_bytes
    warm = Solver(cases.get("chan_small"), "fp32")   # module and runtime set-up outside the measurement
    c = cases.get(name)
    U, V, W, P = cases.initial_condition(c)
    torch.cuda.synchronize()
    free0, _ = torch.cuda.mem_get_info()
    s = Solver(c, prec, graphs=True)
    s.set_state(U, V, W, P)
    s.compute_time_step_RK3(2)
    s.get_state()
    torch.cuda.synchronize()
    free1, _ = torch.cuda.mem_get_info()
    used = free0 - free1
    fp = footprint_bytes(c, prec)
    s.close()
    warm.close()
    assert 0 < used <= 1.02 * fp + (8 << 20), (name, prec, used, fp)
