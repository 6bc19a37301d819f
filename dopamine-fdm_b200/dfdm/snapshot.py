"""The reference's staggered restart/snapshot format, on the host (numpy).

Layout of a one-rank file (output_data, src/input_output.f90:1782-1880; read back by read_input_data, :1225-1341),
a little-endian stream with no record markers:
  int32 nx,  float64 x(nx)        face coordinates        int32 nxm, float64 xm(nxm)   centres, nxm = nx-1
  int32 ny,  float64 y(ny)                                int32 nym, float64 ym(nym)
  int32 nz,  float64 z(nz)                                int32 nzm, float64 zm(nzm)
  then one block per field: int32 n1, n2, n3 and n1*n2*n3 float64 in Fortran order:
  U(nx,nyg,nzg), V(nxg,ny,nzg), W(nxg,nyg,nz), P(nxg,nyg,nzg) and, with an SGS model, nu_t(nxg,nyg,nzg).
(The mesh blocks come in the order x, y, z, xm, ym, zm.)  A file that starts with -4242 is a cell-centred/chunked
box snapshot, which cannot serve as a restart.

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


def _write_block(fh, a: np.ndarray) -> None:
    a = np.asfortranarray(a, dtype="<f8")
    np.asarray(a.shape, dtype="<i4").tofile(fh)
    fh.write(a.tobytes(order="F"))


def _read_block(fh, shape: Tuple[int, int, int], what: str) -> np.ndarray:
    nn = np.fromfile(fh, dtype="<i4", count=3)
    if nn.size != 3 or tuple(int(v) for v in nn) != tuple(shape):
        raise ValueError(f"restart file field block size mismatch for {what}: found {tuple(nn)} expected {shape}")
    n = int(np.prod(shape))
    data = np.fromfile(fh, dtype="<f8", count=n)
    if data.size != n:
        raise ValueError(f"restart file ends inside the {what} block")
    return data.reshape(shape, order="F")


def expected_size(case: Case, with_p: bool = True, with_nut: bool = False) -> int:
    """Bytes of a restart file of this grid: read_input_data's size check (which counts U, V, W and P)."""
    sh = case.shapes()
    n = 6 * 4 + 8 * (case.nx + case.ny + case.nz + (case.nx - 1) + (case.ny - 1) + (case.nz - 1))
    for key in ("U", "V", "W") + (("P",) if with_p else ()) + (("P",) if with_nut else ()):
        n += 3 * 4 + 8 * int(np.prod(sh[key]))
    return n


def write_restart(path: str, case: Case, U, V, W, P, nu_t=None) -> None:
    """The staggered full snapshot (snapshot_location = 0) of one rank."""
    x, y, z = cases.faces(case)
    with open(path, "wb") as fh:
        for f in (x, y, z, _centres(x), _centres(y), _centres(z)):
            np.asarray([f.size], dtype="<i4").tofile(fh)
            np.asarray(f, dtype="<f8").tofile(fh)
        for a in (U, V, W, P):
            _write_block(fh, a)
        if nu_t is not None:
            _write_block(fh, nu_t)


def read_restart(path: str, case: Case, read_nut: bool = False, rtol: float = 1e-12) -> Dict[str, np.ndarray]:
    """U, V, W, P (and nu_t) of a restart file written for this case's grid; raises ValueError as the reference
    aborts: chunked snapshot, short file, face-count mismatch, block-shape mismatch, or (here) coordinates that do
    not match the case's grid."""
    with open(path, "rb") as fh:
        first = np.fromfile(fh, dtype="<i4", count=1)
        if first.size == 1 and int(first[0]) == SNAP_MAGIC:
            raise ValueError("the file is a cell-centred/chunked box snapshot and cannot be used for restart")
    size = os.path.getsize(path)
    need = expected_size(case, with_p=True)
    if size < need:
        raise ValueError(f"restart file is smaller than expected for the grid: {size} < {need} bytes")
    x, y, z = cases.faces(case)
    want = [("nx", x), ("ny", y), ("nz", z), ("nxm", _centres(x)), ("nym", _centres(y)), ("nzm", _centres(z))]
    out: Dict[str, np.ndarray] = {}
    sh = case.shapes()
    with open(path, "rb") as fh:
        for name, ref in want:
            n = int(np.fromfile(fh, dtype="<i4", count=1)[0])
            if n != ref.size:
                raise ValueError(f"restart file {name} = {n} but the grid gives {ref.size}")
            f = np.fromfile(fh, dtype="<f8", count=n)
            scale = max(1.0, float(np.abs(ref).max()))
            if np.abs(f - ref).max() > rtol * scale:
                raise ValueError(f"restart file coordinates ({name}) differ from the grid")
        for key in ("U", "V", "W", "P"):
            out[key] = _read_block(fh, sh[key], key)
        if read_nut:
            out["nu_t"] = _read_block(fh, sh["P"], "nu_t")
    return out


def write_wmf(path: str, case: Case, planes: Dict[str, np.ndarray]) -> None:
    """<snapshot>.wmf from the filter planes in the reference shapes (ux/wx/tx (nx,2,nzg), uz/wz/tz (nxg,2,nz));
    the x/z ghost planes are written as zero, as write_distributed_field_block(..., interior_only) leaves them."""
    with open(path, "wb") as fh:
        for key in ("ux", "wx", "tx", "uz", "wz", "tz"):
            a = np.array(planes[key], dtype=np.float64, order="F", copy=True)
            a[0, :, :] = 0.0
            a[-1, :, :] = 0.0
            a[:, :, 0] = 0.0
            a[:, :, -1] = 0.0
            _write_block(fh, a)


def read_wmf(path: str, case: Case) -> Optional[Dict[str, np.ndarray]]:
    """The filter planes of <snapshot>.wmf, or None when the file does not exist (the filter then re-seeds)."""
    if not os.path.exists(path):
        return None
    nx, nz, nxg, nzg = case.nx, case.nz, case.nxg, case.nzg
    out = {}
    with open(path, "rb") as fh:
        for key in ("ux", "wx", "tx"):
            out[key] = _read_block(fh, (nx, 2, nzg), "wmf_" + key)
        for key in ("uz", "wz", "tz"):
            out[key] = _read_block(fh, (nxg, 2, nz), "wmf_" + key)
    return out
