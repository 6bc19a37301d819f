"""The request loop on the GPU: every result is the same alone and in the mix."""
import numpy as np
import pytest

from dfdm import serve

pytestmark = pytest.mark.gpu


def test_results_alone_equal_results_in_the_mix():
    reqs = serve.make_stream(8, rate=200.0, seed=21, grids=(32, 48), steps=(20, 60))
    mix = serve.Scheduler(serve.GpuExecutor(), 150e9, chunk_cell_steps=2e5, keep_state=True)
    got = mix.run(reqs)
    assert mix.peak_active > 1
    alone = serve.run_isolated(serve.GpuExecutor(), reqs, keep_state=True)
    assert [r.rid for r in got] == [r.rid for r in alone]
    for a, b in zip(got, alone):
        assert a.summary["finite"] == 1.0
        for x, y in zip(a.state, b.state):
            assert np.array_equal(x, y), a.rid
        assert a.summary["kinetic_energy"] == b.summary["kinetic_energy"]
