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


@pytest.mark.parametrize("order,e", [("big", ">"), ("little", "<")])
def test_round_trip_and_byte_layout(tmp_path, order, e):
    """Every word of the staggered restart in the requested byte order: big-endian is what the reference's builds
    write and read (CMakeLists.txt:210 sets -fconvert=big-endian, -convert big_endian or -Mbyteswapio, and
    output_data opens the file without convert=, src/input_output.f90:1842)."""
    c = cases.chan_les_amd_small()
    U, V, W, P = _state(c)
    nut = np.asfortranarray(np.abs(P) * 1e-3)
    f = str(tmp_path / "snap.00000010")
    if order == "big":
        snapshot.write_restart(f, c, U, V, W, P, nut)      # the default
    else:
        snapshot.write_restart(f, c, U, V, W, P, nut, byte_order="little")
    assert os.path.getsize(f) == snapshot.expected_size(c, with_p=True, with_nut=True)
    assert snapshot.detect_byte_order(f, c.nx) == order
    raw = open(f, "rb").read()
    x, y, z = cases.faces(c)
    xm, ym, zm = (0.5 * (a[:-1] + a[1:]) for a in (x, y, z))
    off = 0
    for a in (x, y, z, xm, ym, zm):                         # the mesh: int32 n, then n doubles
        assert np.frombuffer(raw[off:off + 4], e + "i4")[0] == a.size
        assert np.array_equal(np.frombuffer(raw[off + 4:off + 4 + 8 * a.size], e + "f8"), a)
        off += 4 + 8 * a.size
    for key, a in (("U", U), ("V", V), ("W", W), ("P", P), ("nu_t", nut)):   # int32 n1, n2, n3, then the array
        shape = c.shapes()["P" if key == "nu_t" else key]
        assert tuple(np.frombuffer(raw[off:off + 12], e + "i4")) == shape, key
        assert np.array_equal(np.frombuffer(raw[off + 12:off + 12 + 8 * a.size], e + "f8"), a.ravel(order="F")), key
        off += 12 + 8 * a.size
    assert off == len(raw)
    got = snapshot.read_restart(f, c, read_nut=True)
    for key, a in (("U", U), ("V", V), ("W", W), ("P", P), ("nu_t", nut)):
        assert np.array_equal(got[key], a), key


def test_byte_order_detection_rejects_another_grid(tmp_path):
    c = cases.chan_small()
    U, V, W, P = _state(c)
    f = str(tmp_path / "snap")
    snapshot.write_restart(f, c, U, V, W, P)
    with pytest.raises(ValueError, match="nx"):
        snapshot.detect_byte_order(f, c.nx + 2)


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


@pytest.mark.parametrize("order,e", [("big", ">"), ("little", "<")])
def test_wmf_round_trip_zeroes_the_ghost_planes(tmp_path, order, e):
    c = cases.chan_les_amd_small()
    g = np.random.Generator(np.random.PCG64(4))
    planes = {k: np.asfortranarray(g.standard_normal((c.nx, 2, c.nzg))) for k in ("ux", "wx", "tx")}
    planes.update({k: np.asfortranarray(g.standard_normal((c.nxg, 2, c.nz))) for k in ("uz", "wz", "tz")})
    f = str(tmp_path / "snap.wmf")
    snapshot.write_wmf(f, c, planes, byte_order=order)
    raw = open(f, "rb").read()
    assert tuple(np.frombuffer(raw[:12], e + "i4")) == (c.nx, 2, c.nzg)   # the first block header, in that order
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
