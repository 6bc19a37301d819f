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


@pytest.mark.parametrize("order", ["big", "little"])
def test_library_reads_the_host_written_restart(tmp_path, order):
    c = cases.chan_small()
    U, V, W, P = cases.initial_condition(c)
    f = str(tmp_path / "ic")
    snapshot.write_restart(f, c, U, V, W, P, byte_order=order)
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


@pytest.mark.parametrize("order", ["big", "little"])
def test_library_writes_what_the_host_writer_writes(tmp_path, order):
    """The library's restart and .wmf are byte for byte the host restatement's, big-endian by default (as the
    reference's builds write them) and little-endian on request."""
    c = cases.chan_les_amd_small()
    s = Solver(c, "fp64")
    s.set_state(*cases.initial_condition(c))
    s.compute_time_step_RK3(2)
    a, b = str(tmp_path / "lib"), str(tmp_path / "host")
    if order == "big":
        s.write_snapshot(a)
    else:
        s.write_snapshot(a, byte_order="little")
    snapshot.write_restart(b, c, *s.get_state(), nu_t=s.get_nu_t(), byte_order=order)
    assert open(a, "rb").read() == open(b, "rb").read()
    assert snapshot.detect_byte_order(a + ".wmf", c.nx) == order
    snapshot.write_wmf(b + ".wmf", c, snapshot.read_wmf(a + ".wmf", c), byte_order=order)
    assert open(a + ".wmf", "rb").read() == open(b + ".wmf", "rb").read()
    s.close()


@pytest.mark.parametrize("name", ["chan_les_amd_small", "tgv_small"])
@pytest.mark.parametrize("location", [0, 1])
def test_box_snapshot_equals_the_host_restatement(tmp_path, name, location):
    """dfdm_write_box_snapshot writes, byte for byte, what the host restatement of write_box_snapshot writes from
    the same state, time and step: a sub-box and the whole domain (the cell-centred full snapshot at location 1)."""
    c = cases.get(name)
    s = Solver(c, "fp64")
    s.set_state(*cases.initial_condition(c))
    s.compute_time_step_RK3(2)
    U, V, W, P = s.get_state()
    nut = s.get_nu_t() if c.sgs_model else None
    for f1, f2 in (((2, 3, 2), (c.nx - 2, c.ny - 1, c.nz - 3)), ((1, 1, 1), (c.nx, c.ny, c.nz))):
        a, b = str(tmp_path / "lib"), str(tmp_path / "host")
        s.write_box_snapshot(a, f1, f2, location=location, step=7)
        snapshot.write_box(b, c, f1, f2, U, V, W, P, nut, location=location, step=7, t=s.t)
        assert open(a, "rb").read() == open(b, "rb").read(), (f1, f2)
    s.close()


def test_box_snapshot_rejections(tmp_path):
    c = cases.chan_small()
    s = Solver(c, "fp64")
    s.set_state(*cases.initial_condition(c))
    f = str(tmp_path / "box")
    for f1, f2, loc in (((1, 1, 1), (c.nx + 1, 3, 3), 0), ((2, 2, 2), (2, 5, 5), 0), ((1, 1, 1), (3, 3, 3), 2)):
        with pytest.raises(DfdmError):
            s.write_box_snapshot(f, f1, f2, location=loc)
    s.write_box_snapshot(f, (1, 1, 1), (3, 3, 3))
    with pytest.raises(DfdmError, match="cannot be used for restart"):
        s.read_snapshot(f)
    s.close()
