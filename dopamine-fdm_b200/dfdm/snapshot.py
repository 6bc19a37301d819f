"""The reference's staggered restart/snapshot format, on the host (numpy).

Layout of a one-rank file (output_data, src/input_output.f90:1782-1880; read back by read_input_data, :1225-1341),
a stream with no record markers, big-endian by default:
  int32 nx,  float64 x(nx)        face coordinates        int32 nxm, float64 xm(nxm)   centres, nxm = nx-1
  int32 ny,  float64 y(ny)                                int32 nym, float64 ym(nym)
  int32 nz,  float64 z(nz)                                int32 nzm, float64 zm(nzm)
  then one block per field: int32 n1, n2, n3 and n1*n2*n3 float64 in Fortran order:
  U(nx,nyg,nzg), V(nxg,ny,nzg), W(nxg,nyg,nz), P(nxg,nyg,nzg) and, with an SGS model, nu_t(nxg,nyg,nzg).
(The mesh blocks come in the order x, y, z, xm, ym, zm.)  A file that starts with -4242 (read little-endian, as the
reference's probe at :1235 reads it) is a cell-centred/chunked box snapshot, which cannot serve as a restart.

Byte order: output_data and read_input_data open the restart without convert= (:1272, :1842), and so do the .wmf
writer and reader (:1996, :2019), so these files take the build's default byte order, which the reference's
CMakeLists.txt:210 sets to big-endian for gfortran (-fconvert=big-endian), Intel (-convert big_endian) and NVHPC
(-Mbyteswapio).  They are written big-endian here unless byte_order="little" is asked for, and read in the order
their first word (nx) shows.  The box snapshot is explicitly little-endian (:1723) and stays so.

The box snapshot (write_box_snapshot, :1699-1767) holds the face box f1..f2 (1-based faces) of every field:
  int32 -4242, snapshot_location, step, nfields; float64 t; int32 f1(3), f2(3);
  per direction float64 faces x(f1:f2) and centres xm(f1:f2-1);
  per field char name(8) (blank-padded), int32 st(3), gl(3), gh(3);
  then each field's box gl:gh as float64 in Fortran order.
field_box (:1586-1598): st(a) = 1 for the velocity of direction a when snapshot_location = 0, else 0; gl = f1,
gh = f2 - 1 + st.  fill_box_block (:1623-1659) reads global index g of a one-rank run at ghosted index g + 1 - st and,
with snapshot_location = 1, averages each velocity over the two faces of its own direction.  The reference writes it
for chunked_snapshot (the box resolve_chunk_box gives, :1538-1583) and for a cell-centred full snapshot
(snapshot_location = 1, f1 = 1, f2 = n).

The wall-model filter state goes next to it as <file>.wmf (write_wm_filter_state, :1990-2009): six blocks
wmf_ux, wmf_wx, wmf_tx (nx,2,nzg) and wmf_uz, wmf_wz, wmf_tz (nxg,2,nz), with the x/z ghost planes written as zero.
"""
from __future__ import annotations

import os
from typing import Dict, Optional, Tuple

import numpy as np

from . import cases
from .cases import Case

SNAP_MAGIC = -4242


def _centres(f: np.ndarray) -> np.ndarray:
    return 0.5 * (f[:-1] + f[1:])


def _prefix(byte_order: str) -> str:
    if byte_order not in ("big", "little"):
        raise ValueError("byte_order must be 'big' or 'little'")
    return ">" if byte_order == "big" else "<"


def detect_byte_order(path: str, nx: int) -> str:
    """'big' or 'little': the order in which the file's first word reads as nx (a restart starts with nx, a .wmf
    with its first block's n1 = nx); ValueError when it reads as nx in neither."""
    raw = open(path, "rb").read(4)
    if len(raw) < 4:
        raise ValueError("restart file is empty")
    be, le = int(np.frombuffer(raw, ">i4")[0]), int(np.frombuffer(raw, "<i4")[0])
    if be == nx:
        return "big"
    if le == nx:
        return "little"
    raise ValueError(f"restart file nx = {be} (big-endian) or {le} (little-endian) but the grid gives {nx}")


def _write_block(fh, a: np.ndarray, e: str = ">") -> None:
    a = np.asfortranarray(a, dtype=e + "f8")
    np.asarray(a.shape, dtype=e + "i4").tofile(fh)
    fh.write(a.tobytes(order="F"))


def _read_block(fh, shape: Tuple[int, int, int], what: str, e: str = ">") -> np.ndarray:
    nn = np.fromfile(fh, dtype=e + "i4", count=3)
    if nn.size != 3 or tuple(int(v) for v in nn) != tuple(shape):
        raise ValueError(f"restart file field block size mismatch for {what}: found {tuple(nn)} expected {shape}")
    n = int(np.prod(shape))
    data = np.fromfile(fh, dtype=e + "f8", count=n)
    if data.size != n:
        raise ValueError(f"restart file ends inside the {what} block")
    return data.reshape(shape, order="F").astype(np.float64)


def expected_size(case: Case, with_p: bool = True, with_nut: bool = False) -> int:
    """Bytes of a restart file of this grid: read_input_data's size check (which counts U, V, W and P)."""
    sh = case.shapes()
    n = 6 * 4 + 8 * (case.nx + case.ny + case.nz + (case.nx - 1) + (case.ny - 1) + (case.nz - 1))
    for key in ("U", "V", "W") + (("P",) if with_p else ()) + (("P",) if with_nut else ()):
        n += 3 * 4 + 8 * int(np.prod(sh[key]))
    return n


def write_restart(path: str, case: Case, U, V, W, P, nu_t=None, byte_order: str = "big") -> None:
    """The staggered full snapshot (snapshot_location = 0) of one rank, big-endian as the reference's builds
    write it (byte_order="little" for a build without the CMakeLists.txt:210 flags)."""
    e = _prefix(byte_order)
    x, y, z = cases.faces(case)
    with open(path, "wb") as fh:
        for f in (x, y, z, _centres(x), _centres(y), _centres(z)):
            np.asarray([f.size], dtype=e + "i4").tofile(fh)
            np.asarray(f, dtype=e + "f8").tofile(fh)
        for a in (U, V, W, P):
            _write_block(fh, a, e)
        if nu_t is not None:
            _write_block(fh, nu_t, e)


def read_restart(path: str, case: Case, read_nut: bool = False, rtol: float = 1e-12) -> Dict[str, np.ndarray]:
    """U, V, W, P (and nu_t) of a restart file written for this case's grid, in the byte order its first word shows;
    raises ValueError as the reference aborts: chunked snapshot, short file, face-count mismatch, block-shape
    mismatch, or (here) coordinates that do not match the case's grid."""
    with open(path, "rb") as fh:
        first = np.fromfile(fh, dtype="<i4", count=1)
        if first.size == 1 and int(first[0]) == SNAP_MAGIC:
            raise ValueError("the file is a cell-centred/chunked box snapshot and cannot be used for restart")
    size = os.path.getsize(path)
    need = expected_size(case, with_p=True)
    if size < need:
        raise ValueError(f"restart file is smaller than expected for the grid: {size} < {need} bytes")
    e = _prefix(detect_byte_order(path, case.nx))
    x, y, z = cases.faces(case)
    want = [("nx", x), ("ny", y), ("nz", z), ("nxm", _centres(x)), ("nym", _centres(y)), ("nzm", _centres(z))]
    out: Dict[str, np.ndarray] = {}
    sh = case.shapes()
    with open(path, "rb") as fh:
        for name, ref in want:
            n = int(np.fromfile(fh, dtype=e + "i4", count=1)[0])
            if n != ref.size:
                raise ValueError(f"restart file {name} = {n} but the grid gives {ref.size}")
            f = np.fromfile(fh, dtype=e + "f8", count=n)
            scale = max(1.0, float(np.abs(ref).max()))
            if np.abs(f - ref).max() > rtol * scale:
                raise ValueError(f"restart file coordinates ({name}) differ from the grid")
        for key in ("U", "V", "W", "P"):
            out[key] = _read_block(fh, sh[key], key, e)
        if read_nut:
            out["nu_t"] = _read_block(fh, sh["P"], "nu_t", e)
    return out


def write_wmf(path: str, case: Case, planes: Dict[str, np.ndarray], byte_order: str = "big") -> None:
    """<snapshot>.wmf from the filter planes in the reference shapes (ux/wx/tx (nx,2,nzg), uz/wz/tz (nxg,2,nz));
    the x/z ghost planes are written as zero, as write_distributed_field_block(..., interior_only) leaves them."""
    e = _prefix(byte_order)
    with open(path, "wb") as fh:
        for key in ("ux", "wx", "tx", "uz", "wz", "tz"):
            a = np.array(planes[key], dtype=np.float64, order="F", copy=True)
            a[0, :, :] = 0.0
            a[-1, :, :] = 0.0
            a[:, :, 0] = 0.0
            a[:, :, -1] = 0.0
            _write_block(fh, a, e)


def read_wmf(path: str, case: Case) -> Optional[Dict[str, np.ndarray]]:
    """The filter planes of <snapshot>.wmf, or None when the file does not exist (the filter then re-seeds); read in
    the byte order its first word shows."""
    if not os.path.exists(path):
        return None
    nx, nz, nxg, nzg = case.nx, case.nz, case.nxg, case.nzg
    e = _prefix(detect_byte_order(path, nx))
    out = {}
    with open(path, "rb") as fh:
        for key in ("ux", "wx", "tx"):
            out[key] = _read_block(fh, (nx, 2, nzg), "wmf_" + key, e)
        for key in ("uz", "wz", "tz"):
            out[key] = _read_block(fh, (nxg, 2, nz), "wmf_" + key, e)
    return out


def coordinate_face_range(xf: np.ndarray, s: float, e: float) -> Tuple[int, int, bool]:
    """coordinate_face_range (src/input_output.f90:1517-1535): the faces nearest the clamped start and end
    coordinates (1-based, first of equal distances), widened to one cell when they coincide."""
    nf = xf.size
    ok = (s <= e) and (e >= xf[0]) and (s <= xf[nf - 1])
    f1 = int(np.argmin(np.abs(xf - min(max(s, xf[0]), xf[nf - 1])))) + 1
    f2 = int(np.argmin(np.abs(xf - min(max(e, xf[0]), xf[nf - 1])))) + 1
    if f2 <= f1:
        if f1 < nf:
            f2 = f1 + 1
        else:
            f1 = f2 - 1
    return f1, f2, ok


def resolve_chunk_box(case: Case, x_start: float, x_end: float, y_start: float, y_end: float, z_start: float,
                      z_end: float) -> Tuple[Tuple[int, int, int], Tuple[int, int, int]]:
    """check_snapshot_inputs and resolve_chunk_box (src/input_output.f90:913-925, 1538-1583): the &IO chunk box as
    1-based face indices f1, f2.  All six inputs negative: index mode, -v is the 1-based face (0 <= -v-1 < n);
    none negative: coordinates, mapped by coordinate_face_range.  Raises ValueError where the reference aborts."""
    vals = [x_start, x_end, y_start, y_end, z_start, z_end]
    nneg = sum(1 for v in vals if v < 0.0)
    if nneg not in (0, 6):
        raise ValueError("chunk box x/y/z_start/end must be all lengths (>= 0) or all negative face indices")
    faces_ = cases.faces(case)
    nf = (case.nx, case.ny, case.nz)
    index_mode = x_start < 0.0
    f1, f2 = [0, 0, 0], [0, 0, 0]
    for a, (st, en) in enumerate(((x_start, x_end), (y_start, y_end), (z_start, z_end))):
        if index_mode:
            n1 = int(round(-st)) - 1
            n2 = int(round(-en)) - 1
            ok = n1 >= 0 and n2 <= nf[a] - 1 and n1 < n2
            f1[a], f2[a] = n1 + 1, n2 + 1
        else:
            f1[a], f2[a], ok = coordinate_face_range(faces_[a], st, en)
        if not ok:
            raise ValueError(f"chunk box is empty or outside the domain in direction {a + 1}")
    return (f1[0], f1[1], f1[2]), (f2[0], f2[1], f2[2])


def field_box(ic: int, f1, f2, location: int) -> Tuple[Tuple[int, ...], Tuple[int, ...], Tuple[int, ...]]:
    """field_box: stagger flags and the global index range gl:gh of field kind ic (0 scalar, 1/2/3 = U/V/W)."""
    st = [0, 0, 0]
    if location == 0 and ic > 0:
        st[ic - 1] = 1
    gl = tuple(int(v) for v in f1)
    gh = tuple(int(f2[a]) - 1 + st[a] for a in range(3))
    return tuple(st), gl, gh


def box_block(A: np.ndarray, ic: int, f1, f2, location: int) -> np.ndarray:
    """fill_box_block of a one-rank run: the box gl:gh of the ghosted array A (reference shape, Fortran order)."""
    st, gl, gh = field_box(ic, f1, f2, location)
    sl = tuple(slice(gl[a] - st[a], gh[a] - st[a] + 1) for a in range(3))   # 0-based ghosted index g - st
    if location == 1 and ic > 0:
        a = ic - 1
        lo = list(sl)
        lo[a] = slice(sl[a].start - 1, sl[a].stop - 1)
        return 0.5 * (A[tuple(lo)] + A[sl])
    return np.array(A[sl], dtype=np.float64)


def write_box(path: str, case: Case, f1, f2, U, V, W, P, nu_t=None, location: int = 0, step: int = 0,
              t: float = 0.0) -> None:
    """write_box_snapshot of a one-rank run (the restatement that the library's dfdm_write_box_snapshot is checked
    against)."""
    if location not in (0, 1):
        raise ValueError("snapshot_location must be 0 (staggered) or 1 (cell-centred)")
    fields = [("U", U, 1), ("V", V, 2), ("W", W, 3), ("P", P, 0)]
    if nu_t is not None:
        fields.append(("nu_t", nu_t, 0))
    faces_ = cases.faces(case)
    with open(path, "wb") as fh:
        np.asarray([SNAP_MAGIC, location, step, len(fields)], dtype="<i4").tofile(fh)
        np.asarray([t], dtype="<f8").tofile(fh)
        np.asarray(list(f1) + list(f2), dtype="<i4").tofile(fh)
        for a in range(3):
            f = faces_[a]
            np.asarray(f[f1[a] - 1:f2[a]], dtype="<f8").tofile(fh)
            np.asarray(_centres(f)[f1[a] - 1:f2[a] - 1], dtype="<f8").tofile(fh)
        for name, _, ic in fields:
            fh.write(name.ljust(8).encode("ascii"))
            st, gl, gh = field_box(ic, f1, f2, location)
            np.asarray(list(st) + list(gl) + list(gh), dtype="<i4").tofile(fh)
        for _, A, ic in fields:
            fh.write(np.asfortranarray(box_block(np.asarray(A), ic, f1, f2, location), dtype="<f8").tobytes(order="F"))


def read_box(path: str) -> Dict[str, object]:
    """A box snapshot: its header (location, step, t, f1, f2, the face and centre coordinates) and fields by name."""
    with open(path, "rb") as fh:
        head = np.fromfile(fh, dtype="<i4", count=4)
        if head.size != 4 or int(head[0]) != SNAP_MAGIC:
            raise ValueError("not a box snapshot (no -4242 magic)")
        out: Dict[str, object] = {"location": int(head[1]), "step": int(head[2])}
        nf = int(head[3])
        out["t"] = float(np.fromfile(fh, dtype="<f8", count=1)[0])
        ff = np.fromfile(fh, dtype="<i4", count=6)
        f1, f2 = tuple(int(v) for v in ff[:3]), tuple(int(v) for v in ff[3:])
        out["f1"], out["f2"] = f1, f2
        for a, key in enumerate("xyz"):
            out[key] = np.fromfile(fh, dtype="<f8", count=f2[a] - f1[a] + 1)
            out[key + "m"] = np.fromfile(fh, dtype="<f8", count=f2[a] - f1[a])
        heads = []
        for _ in range(nf):
            name = fh.read(8).decode("ascii").rstrip()
            v = np.fromfile(fh, dtype="<i4", count=9)
            heads.append((name, tuple(int(x) for x in v[:3]), tuple(int(x) for x in v[3:6]), tuple(int(x) for x in v[6:])))
        out["fields"] = {}
        for name, st, gl, gh in heads:
            shape = tuple(gh[a] - gl[a] + 1 for a in range(3))
            n = int(np.prod(shape))
            data = np.fromfile(fh, dtype="<f8", count=n)
            if data.size != n:
                raise ValueError(f"box snapshot ends inside the {name} block")
            out["fields"][name] = {"st": st, "gl": gl, "gh": gh, "data": data.reshape(shape, order="F")}
    return out
