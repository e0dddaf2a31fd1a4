"""Legacy binary VTK export of the fields (for ParaView).

Writes the file the reference's post-processor writes
(post/paraview_fields/generate_output.f90:45-143): ``OUTPAR_%08d.vtk``, a
legacy VTK 3.0 ``RECTILINEAR_GRID`` in BINARY (big-endian float32) with the x,
y, z coordinates x(i) = (i-1) dx, dx = 2 pi/(nx-1), and one ``FIELD FieldData``
block holding the requested fields (u, v, w, phi) in x-fastest order.  Header
numbers are right-justified in Fortran's i8 / i16 widths, as there.
"""
from __future__ import annotations

import math
import os

import numpy as np


def _coords(n: int, grid_mode: int = 0) -> np.ndarray:
    dx = 2 * (4 * math.atan(1.0)) / (n - 1) if grid_mode == 0 else 2 * math.pi / n
    x = np.zeros(n)
    for i in range(1, n):  # cumulative, as x(i+1) = x(i) + dx
        x[i] = x[i - 1] + dx
    return x


def write_vtk(path: str, fields: dict, grid_mode: int = 0) -> str:
    """fields: ordered {name: array indexed [i, j, k]} (names u, v, w, phi)."""
    arrays = [(k, np.asarray(v)) for k, v in fields.items() if v is not None]
    n = arrays[0][1].shape[0]
    x = _coords(n, grid_mode)
    lf = b"\n"
    out = bytearray()
    out += b"# vtk DataFile Version 3.0" + lf
    out += b"Phase field" + lf
    out += b"BINARY" + lf
    out += b"DATASET RECTILINEAR_GRID" + lf
    s8 = f"{n:8d}".encode()
    out += b"DIMENSIONS " + s8 + s8 + s8 + lf
    for axis in (b"X", b"Y", b"Z"):
        out += axis + b"_COORDINATES " + s8 + b"  float" + lf
        out += x.astype(">f4").tobytes()
    total = f"{n * n * n:16d}".encode()
    out += b"POINT_DATA " + total + lf
    out += b"FIELD FieldData " + f"{len(arrays):8d}".encode() + lf
    for name, a in arrays:
        out += name.encode() + b" 1 " + total + b" float" + lf
        out += np.asfortranarray(a).ravel(order="F").astype(">f4").tobytes()
    with open(path, "wb") as f:
        f.write(bytes(out))
    return path


def vtk_name(outdir: str, t: int) -> str:
    return os.path.join(outdir, f"OUTPAR_{t:08d}.vtk")


def read_vtk(path: str) -> dict:
    """Parse a file written by write_vtk (for tests and tools)."""
    data = open(path, "rb").read()
    pos = 0

    def line():
        nonlocal pos
        e = data.index(b"\n", pos)
        s = data[pos:e].decode()
        pos = e + 1
        return s

    assert line().startswith("# vtk DataFile")
    line()
    assert line() == "BINARY"
    assert line() == "DATASET RECTILINEAR_GRID"
    dims = [int(v) for v in line().split()[1:]]
    n = dims[0]
    coords = []
    for _ in range(3):
        line()
        coords.append(np.frombuffer(data, dtype=">f4", count=n, offset=pos))
        pos += 4 * n
    npts = int(line().split()[1])
    nf = int(line().split()[2])
    out = {"dims": dims, "coords": coords}
    for _ in range(nf):
        name = line().split()[0]
        a = np.frombuffer(data, dtype=">f4", count=npts, offset=pos).reshape((n, n, n), order="F")
        pos += 4 * npts
        out[name] = a
    return out
