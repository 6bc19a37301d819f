"""The reference's restart/snapshot file format on the host, and restart = uninterrupted through a file."""
import os

import numpy as np
import pytest

from conftest import rel_l2
from dfdm import cases, snapshot


def _state(c):
    U, V, W, P = cases.initial_condition(c)
    P = np.asfortranarray(np.random.Generator(np.random.PCG64(3)).standard_normal(P.shape))
    return U, V, W, P


def test_round_trip_and_byte_layout(tmp_path):
    c = cases.chan_les_amd_small()
    U, V, W, P = _state(c)
    nut = np.asfortranarray(np.abs(P) * 1e-3)
    f = str(tmp_path / "snap.00000010")
    snapshot.write_restart(f, c, U, V, W, P, nut)
    assert os.path.getsize(f) == snapshot.expected_size(c, with_p=True, with_nut=True)
    raw = open(f, "rb").read()
    x, y, z = cases.faces(c)
    assert np.frombuffer(raw[:4], "<i4")[0] == c.nx
    assert np.array_equal(np.frombuffer(raw[4:4 + 8 * c.nx], "<f8"), x)
    off = 6 * 4 + 8 * (c.nx + c.ny + c.nz + c.nx - 1 + c.ny - 1 + c.nz - 1)
    assert tuple(np.frombuffer(raw[off:off + 12], "<i4")) == c.shapes()["U"]
    assert np.array_equal(np.frombuffer(raw[off + 12:off + 12 + 8 * U.size], "<f8"), U.ravel(order="F"))
    got = snapshot.read_restart(f, c, read_nut=True)
    for key, a in (("U", U), ("V", V), ("W", W), ("P", P), ("nu_t", nut)):
        assert np.array_equal(got[key], a), key


def test_rejections(tmp_path):
    c = cases.chan_small()
    U, V, W, P = _state(c)
    f = str(tmp_path / "snap")
    snapshot.write_restart(f, c, U, V, W, P)
    with pytest.raises(ValueError, match="smaller than expected"):
        snapshot.read_restart(f, cases.chan_les_amd_small().with_(nz=20))
    with pytest.raises(ValueError, match="coordinates"):
        snapshot.read_restart(f, c.with_(Lx_i=3.5))
    short = str(tmp_path / "short")
    open(short, "wb").write(open(f, "rb").read()[:-8])
    with pytest.raises(ValueError, match="smaller than expected"):
        snapshot.read_restart(short, c)
    box = str(tmp_path / "box")
    open(box, "wb").write(np.asarray([snapshot.SNAP_MAGIC], "<i4").tobytes() + b"\0" * 64)
    with pytest.raises(ValueError, match="chunked"):
        snapshot.read_restart(box, c)


def test_wmf_round_trip_zeroes_the_ghost_planes(tmp_path):
    c = cases.chan_les_amd_small()
    g = np.random.Generator(np.random.PCG64(4))
    planes = {k: np.asfortranarray(g.standard_normal((c.nx, 2, c.nzg))) for k in ("ux", "wx", "tx")}
    planes.update({k: np.asfortranarray(g.standard_normal((c.nxg, 2, c.nz))) for k in ("uz", "wz", "tz")})
    f = str(tmp_path / "snap.wmf")
    snapshot.write_wmf(f, c, planes)
    back = snapshot.read_wmf(f, c)
    for k, a in planes.items():
        b = back[k]
        assert np.array_equal(b[1:-1, :, 1:-1], a[1:-1, :, 1:-1])
        assert not b[0].any() and not b[-1].any() and not b[:, :, 0].any() and not b[:, :, -1].any()
    assert snapshot.read_wmf(str(tmp_path / "missing.wmf"), c) is None


def test_oracle_restart_through_a_file_equals_the_uninterrupted_run(oracle_mod, tmp_path):
    """The reference's restart invariant (CMakeLists.txt:609-619) with the state passing through the file."""
    c = cases.chan_small()
    U, V, W, P = cases.initial_condition(c)
    full = oracle_mod.Oracle(c)
    full.set_state(U, V, W, P)
    full.step(5)
    a = oracle_mod.Oracle(c)
    a.set_state(U, V, W, P)
    a.step(3)
    f = str(tmp_path / "restart")
    snapshot.write_restart(f, c, *a.get_state())
    r = snapshot.read_restart(f, c)
    b = oracle_mod.Oracle(c)
    b.set_state(r["U"], r["V"], r["W"], r["P"])
    b.step(2)
    for x, y in zip(b.get_state()[:3], full.get_state()[:3]):
        assert rel_l2(x, y) <= 1e-12
