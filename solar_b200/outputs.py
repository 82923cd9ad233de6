"""The reference's output files: host writers (through the C library) and readers.

Formats (output.f90):
* restart  ``Restart/restart.NNN.<zone>`` -- int32 nx, ny, nr, 5; float64 time; int32 step;
  then q(nx, ny, nr, 5) float64 in Fortran order (WRITE_RESTART, :86-190).
* visual   ``Visual/NNN/vis_<rank>`` -- one Fortran unformatted record of q(:, :, o_rad, 1:5)
  (WRITE_VISUAL, :192-240).
* grid     ``Visual/grid/grid_<rank>`` -- FORMAT(1x, 7i5) (WRITE_GRID, :242-267).
* trace    ``trace_<zone>`` -- appended ((q(1,1,k,l), k=1,nr), l=1,5), FORMAT(1x, 5(ES13.5))
  (WRITE_RADIAL_TRACE, :309-343).
Arrays returned here use this package's zone layout: q[field][k][j][i].
"""
from __future__ import annotations

import ctypes
import os
import struct

import numpy as np

from . import _lib


def cue_name(cue: int) -> str:
    buf = ctypes.create_string_buffer(32)
    _lib.check(_lib.load().solar_io_cue_name(int(cue), buf, 32))
    return buf.value.decode()


def format_es(v: float, w: int = 13, d: int = 5) -> str:
    """Fortran ESw.d of one value (the trace files' number format)."""
    buf = ctypes.create_string_buffer(w + 1)
    _lib.check(_lib.load().solar_io_format_es(float(v), w, d, buf))
    return buf.value.decode()


def read_restart(path: str):
    """(q[5][nr][ny][nx], time, step) of one zone's restart file."""
    with open(path, "rb") as f:
        head = f.read(28)
        nx, ny, nr, nf, time, step = struct.unpack("<4idi", head)
        data = np.fromfile(f, dtype="<f8", count=nx * ny * nr * nf)
    if nf != 5 or data.size != nx * ny * nr * 5:
        raise ValueError(f"{path}: not a restart file of a 5-field state")
    return data.reshape(5, nr, ny, nx), time, step


def read_visual(path: str, nx: int, ny: int | None = None) -> np.ndarray:
    """q[5][ny][nx] of one zone's visual dump (one unformatted sequential record)."""
    ny = nx if ny is None else ny
    raw = open(path, "rb").read()
    n = nx * ny * 5 * 8
    head, tail = struct.unpack("<i", raw[:4])[0], struct.unpack("<i", raw[4 + n:8 + n])[0]
    if head != n or tail != n or len(raw) != n + 8:
        raise ValueError(f"{path}: record markers {head}, {tail} do not match {n} bytes")
    return np.frombuffer(raw[4:4 + n], dtype="<f8").reshape(5, ny, nx)


def read_grid(path: str):
    """The seven integers of a grid file: start/end of xi, eta, r (0-based) and the zone id."""
    line = open(path).read().splitlines()[0]
    return [int(line[1 + 5 * q:6 + 5 * q]) for q in range(7)]


def parse_es(cell: str) -> float:
    """A Fortran ES field, including the E-less form of three-digit exponents (1.23457+100)."""
    t = cell.strip()
    if "E" in t or t in ("NaN", "Infinity", "-Infinity"):
        return float(t.replace("Infinity", "inf"))
    p = max(t.rfind("+"), t.rfind("-"))
    return float(t[:p] + "E" + t[p:])


def read_trace(path: str, nr: int) -> np.ndarray:
    """Every record of a trace file: array (records, 5, nr) of q(1,1,k,l).  Lines hold five
    13-character fields; the first line of each record starts with one blank."""
    vals = []
    for line in open(path).read().splitlines():
        body = line[1:] if len(line) % 13 == 1 else line
        vals += [parse_es(body[13 * q:13 * q + 13]) for q in range(len(body) // 13)]
    return np.array(vals).reshape(-1, 5, nr)


def write_forcing(path: str, f: np.ndarray) -> None:
    """A forcing_cubesph file: one unformatted record of f(nx, ny, nt) with n fastest;
    ``f`` has shape (nx, ny, nt) indexed [i][j][n]."""
    f = np.ascontiguousarray(f, dtype="<f8")
    d = os.path.dirname(path)
    if d:
        os.makedirs(d, exist_ok=True)
    with open(path, "wb") as fp:
        marker = struct.pack("<i", f.nbytes)
        fp.write(marker)
        fp.write(f.tobytes())
        fp.write(marker)


def read_forcing(path: str, nx: int, ny: int, nt: int) -> np.ndarray:
    """f[i][j][n] of a forcing_cubesph file."""
    out = np.empty(nx * ny * nt)
    _lib.check(_lib.load().solar_io_read_forcing(path.encode(), nx, ny, nt,
                                                 out.ctypes.data_as(ctypes.POINTER(ctypes.c_double))))
    return out.reshape(nx, ny, nt)
