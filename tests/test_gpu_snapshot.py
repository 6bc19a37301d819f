"""Snapshots in the reference's restart format through the C ABI: the library writes what the host format reader
reads, reads what the host writer writes, and a run restarted from its own file continues exactly."""
import os

import numpy as np
import pytest

from conftest import rel_l2
from dfdm import cases, snapshot
from dfdm.native import DfdmError, Solver

pytestmark = pytest.mark.gpu


def test_restart_from_the_library_snapshot_continues_the_run(tmp_path):
    c = cases.chan_les_amd_small()          # AMD + wall model with the temporal filter: the .wmf is needed too
    U, V, W, P = cases.initial_condition(c)
    a = Solver(c, "fp64")
    a.set_state(U, V, W, P)
    a.compute_time_step_RK3(3)
    f = str(tmp_path / "snap.00000003")
    a.write_snapshot(f)
    assert os.path.exists(f + ".wmf")
    host = snapshot.read_restart(f, c, read_nut=True)
    for key, x in zip("UVWP", a.get_state()):
        assert np.array_equal(host[key], x), key
    assert np.array_equal(host["nu_t"], a.get_nu_t())
    assert snapshot.read_wmf(f + ".wmf", c) is not None
    b = Solver(c, "fp64")
    b.read_snapshot(f)
    a.compute_time_step_RK3(2)
    b.compute_time_step_RK3(2)
    for x, y in zip(a.get_state(), b.get_state()):
        assert rel_l2(x, y) <= 1e-13


def test_library_reads_the_host_written_restart(tmp_path):
    c = cases.chan_small()
    U, V, W, P = cases.initial_condition(c)
    f = str(tmp_path / "ic")
    snapshot.write_restart(f, c, U, V, W, P)
    s = Solver(c, "fp64")
    s.read_snapshot(f)
    ref = Solver(c, "fp64")
    ref.set_state(U, V, W, P)
    for x, y in zip(s.get_state(), ref.get_state()):
        assert np.array_equal(x, y)
    other = Solver(cases.chan_small().with_(Lz_i=2.0), "fp64")
    with pytest.raises(DfdmError) as e:
        other.read_snapshot(f)
    assert e.value.code == 1 and "coordinates" in str(e.value)
