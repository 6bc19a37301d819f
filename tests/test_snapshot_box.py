"""The reference's chunked / cell-centred box snapshot (write_box_snapshot, src/input_output.f90:1699-1767) and the
&IO chunk-box resolution (resolve_chunk_box, :1538-1583) on the host: header layout, the stagger and index rules of
field_box / fill_box_block checked element by element, and the reference's rejections."""
import os

import numpy as np
import pytest

from dfdm import cases, snapshot


def _state(c, seed=4):
    g = np.random.Generator(np.random.PCG64(seed))
    return [np.asfortranarray(g.standard_normal(c.shapes()[k])) for k in ("U", "V", "W", "P")]


def _expected(A, ic, f1, f2, location):
    """fill_box_block of one rank written out with explicit 1-based loops."""
    st = [1 if (location == 0 and ic == a + 1) else 0 for a in range(3)]
    gl = list(f1)
    gh = [f2[a] - 1 + st[a] for a in range(3)]
    out = np.empty([gh[a] - gl[a] + 1 for a in range(3)])
    for k in range(gl[2], gh[2] + 1):
        for j in range(gl[1], gh[1] + 1):
            for i in range(gl[0], gh[0] + 1):
                ia, ja, ka = i + 1 - st[0], j + 1 - st[1], k + 1 - st[2]   # 1-based ghosted indices
                val = lambda p, q, r: A[p - 1, q - 1, r - 1]
                if location == 1 and ic == 1:
                    v = 0.5 * (val(ia - 1, ja, ka) + val(ia, ja, ka))
                elif location == 1 and ic == 2:
                    v = 0.5 * (val(ia, ja - 1, ka) + val(ia, ja, ka))
                elif location == 1 and ic == 3:
                    v = 0.5 * (val(ia, ja, ka - 1) + val(ia, ja, ka))
                else:
                    v = val(ia, ja, ka)
                out[i - gl[0], j - gl[1], k - gl[2]] = v
    return out


@pytest.mark.parametrize("location", [0, 1])
@pytest.mark.parametrize("box", [((2, 3, 4), (7, 9, 11)), ((1, 1, 1), None)], ids=["sub-box", "whole domain"])
def test_box_layout_and_values(tmp_path, location, box):
    c = cases.chan_les_amd_small()
    f1, f2 = box
    if f2 is None:
        f2 = (c.nx, c.ny, c.nz)
    U, V, W, P = _state(c)
    nut = np.asfortranarray(np.abs(P) * 1e-3)
    path = str(tmp_path / "box.00000012")
    snapshot.write_box(path, c, f1, f2, U, V, W, P, nut, location=location, step=12, t=0.375)
    raw = open(path, "rb").read()
    assert tuple(np.frombuffer(raw[:16], "<i4")) == (-4242, location, 12, 5)
    assert np.frombuffer(raw[16:24], "<f8")[0] == 0.375
    assert tuple(np.frombuffer(raw[24:48], "<i4")) == tuple(f1) + tuple(f2)
    got = snapshot.read_box(path)
    assert got["location"] == location and got["step"] == 12 and got["t"] == 0.375
    assert got["f1"] == tuple(f1) and got["f2"] == tuple(f2)
    for a, key in enumerate("xyz"):
        face = cases.faces(c)[a]
        assert np.array_equal(got[key], face[f1[a] - 1:f2[a]])
        assert np.array_equal(got[key + "m"], 0.5 * (face[f1[a] - 1:f2[a] - 1] + face[f1[a]:f2[a]]))
    assert list(got["fields"]) == ["U", "V", "W", "P", "nu_t"]
    for (name, A, ic) in (("U", U, 1), ("V", V, 2), ("W", W, 3), ("P", P, 0), ("nu_t", nut, 0)):
        fl = got["fields"][name]
        st = tuple(1 if (location == 0 and ic == a + 1) else 0 for a in range(3))
        assert fl["st"] == st and fl["gl"] == tuple(f1)
        assert fl["gh"] == tuple(f2[a] - 1 + st[a] for a in range(3))
        assert np.array_equal(fl["data"], _expected(A, ic, f1, f2, location)), name
    # the size: header, axes, per-field heads and the blocks
    n = 16 + 8 + 24 + 8 * sum(2 * (f2[a] - f1[a]) + 1 for a in range(3)) + 5 * (8 + 36)
    n += 8 * sum(int(np.prod(f["data"].shape)) for f in got["fields"].values())
    assert os.path.getsize(path) == n


def test_dns_box_has_four_fields_and_is_not_a_restart(tmp_path):
    c = cases.chan_small()
    U, V, W, P = _state(c, 5)
    path = str(tmp_path / "box")
    snapshot.write_box(path, c, (1, 1, 1), (c.nx, c.ny, c.nz), U, V, W, P, location=1)
    got = snapshot.read_box(path)
    assert list(got["fields"]) == ["U", "V", "W", "P"]
    for f in got["fields"].values():   # cell-centred: every field on the (nx-1, ny-1, nz-1) cells
        assert f["data"].shape == (c.nx - 1, c.ny - 1, c.nz - 1)
    with pytest.raises(ValueError, match="cannot be used for restart"):
        snapshot.read_restart(path, c)
    with pytest.raises(ValueError, match="snapshot_location"):
        snapshot.write_box(path, c, (1, 1, 1), (3, 3, 3), U, V, W, P, location=2)


def test_chunk_box_index_mode():
    c = cases.chan_small()
    # all six negative: -v is the 1-based face, 0 <= -v-1 < n
    assert snapshot.resolve_chunk_box(c, -1, -5, -2, -4, -3, -c.nz) == ((1, 2, 3), (5, 4, c.nz))
    for bad in ((-1, -1, -2, -4, -3, -6),            # empty in x
                (-1, -(c.nx + 1), -2, -4, -3, -6),   # beyond the last face
                (-3, -2, -2, -4, -3, -6)):           # start after end
        with pytest.raises(ValueError, match="empty or outside"):
            snapshot.resolve_chunk_box(c, *bad)
    with pytest.raises(ValueError, match="all lengths"):
        snapshot.resolve_chunk_box(c, -1, 2.0, -2, -4, -3, -6)


def test_chunk_box_coordinate_mode():
    c = cases.chan_small()
    x, y, z = cases.faces(c)
    # nearest faces of the clamped coordinates
    f1, f2 = snapshot.resolve_chunk_box(c, x[2] + 0.1 * (x[3] - x[2]), x[6] - 0.2 * (x[6] - x[5]), -0.5 * 0 + y[0],
                                        1e9, z[1], z[4])
    assert f1 == (3, 1, 2) and f2 == (7, c.ny, 5)
    # start and end on one face: widened to one cell (upwards, or downwards at the last face)
    assert snapshot.resolve_chunk_box(c, x[3], x[3], y[2], y[2], z[-1], z[-1]) == ((4, 3, c.nz - 1), (5, 4, c.nz))
    with pytest.raises(ValueError, match="empty or outside"):
        snapshot.resolve_chunk_box(c, x[-1] + 1.0, x[-1] + 2.0, 0.0, 1.0, 0.0, 1.0)
    with pytest.raises(ValueError, match="empty or outside"):
        snapshot.resolve_chunk_box(c, 2.0, 1.0, 0.0, 1.0, 0.0, 1.0)
