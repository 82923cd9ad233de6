"""The reference's output formats (output.f90) through the library's host writers, on CPU.

Expected strings follow the Fortran rules the reference relies on: ES13.5 (one digit, five
decimals, E+zz exponent, or +zzz without the E beyond two digits), FORMAT(1x, 7i5),
format reversion to 5(ES13.5) after the first record line, unformatted sequential records
with 4-byte length markers, and the WRITE_RESTART header of four int32, one float64 and one
int32 before the Fortran-order float64 state at byte 28.
"""
import struct

import numpy as np
import pytest

from solar_b200 import _lib, outputs


@pytest.mark.parametrize("v,want", [
    (1.0, "  1.00000E+00"), (-2.5e-7, " -2.50000E-07"), (0.0, "  0.00000E+00"),
    (9.999996, "  1.00000E+01"), (123456.789, "  1.23457E+05"), (1.234567e100, "  1.23457+100"),
    (-1.5e-150, " -1.50000-150"), (6.02214076e23, "  6.02214E+23"),
])
def test_es13_5(v, want):
    assert outputs.format_es(v) == want
    assert outputs.parse_es(want) == pytest.approx(v, rel=1e-5, abs=0)


@pytest.mark.parametrize("cue,want", [(0, "000"), (7, "007"), (42, "042"), (123, "123"), (1234, "1234")])
def test_cue_names(cue, want):
    assert outputs.cue_name(cue) == want


def _dp(a):
    return a.ctypes.data_as(_lib.ctypes.POINTER(_lib.ctypes.c_double))


def test_restart_layout_and_roundtrip(tmp_path):
    lib = _lib.load()
    nx, nr = 6, 5
    q = np.random.default_rng(0).standard_normal((5, nr, nx, nx))      # Fortran (nx, ny, nr, 5)
    path = str(tmp_path / "Restart" / "restart.003.2")
    assert lib.solar_io_write_restart(path.encode(), _dp(q), nx, nx, nr, 1.25, 17) == 0
    raw = open(path, "rb").read()
    assert len(raw) == 28 + q.size * 8
    assert struct.unpack("<4idi", raw[:28]) == (nx, nx, nr, 5, 1.25, 17)
    np.testing.assert_array_equal(np.frombuffer(raw[28:], "<f8"), q.ravel())
    back, t, s = outputs.read_restart(path)
    np.testing.assert_array_equal(back, q)
    assert (t, s) == (1.25, 17)
    out = np.zeros_like(q)
    tt, ss = _lib.ctypes.c_double(), _lib.ctypes.c_int()
    assert lib.solar_io_read_restart(path.encode(), _dp(out), nx, nx, nr, _lib.ctypes.byref(tt),
                                     _lib.ctypes.byref(ss)) == 0
    np.testing.assert_array_equal(out, q)
    assert lib.solar_io_read_restart(path.encode(), _dp(out), nx, nx, nr + 1, None, None) == _lib.SOLAR_ERR_ARG
    assert "expected" in _lib.last_error()


def test_visual_record(tmp_path):
    lib = _lib.load()
    nx = 7
    plane = np.arange(5 * nx * nx, dtype=np.float64).reshape(5, nx, nx)
    path = str(tmp_path / "Visual" / "000" / "vis_3")
    assert lib.solar_io_write_visual(path.encode(), _dp(plane), nx, nx) == 0
    raw = open(path, "rb").read()
    n = plane.size * 8
    assert struct.unpack("<i", raw[:4])[0] == n and struct.unpack("<i", raw[-4:])[0] == n
    np.testing.assert_array_equal(outputs.read_visual(path, nx), plane)


def test_grid_line(tmp_path):
    lib = _lib.load()
    path = str(tmp_path / "Visual" / "grid" / "grid_4")
    seven = (_lib.ctypes.c_int * 7)(0, 127, 0, 127, 0, 399, 5)
    assert lib.solar_io_write_grid(path.encode(), seven) == 0
    assert open(path).read() == "     0  127    0  127    0  399    5\n"
    assert outputs.read_grid(path) == [0, 127, 0, 127, 0, 399, 5]


def test_trace_records_append(tmp_path):
    lib = _lib.load()
    nr = 4
    path = str(tmp_path / "trace_1")
    recs = [np.linspace(-1, 1, 5 * nr) * 10.0 ** e for e in (0, -3)]
    for r in recs:
        assert lib.solar_io_append_trace(path.encode(), _dp(np.ascontiguousarray(r)), r.size) == 0
    lines = open(path).read().splitlines()
    assert len(lines) == 2 * nr                       # 5 values per line, 5*nr values per record
    assert lines[0].startswith(" ") and len(lines[0]) == 66
    assert len(lines[1]) == 65                        # format reversion: no 1x after the first line
    got = outputs.read_trace(path, nr)
    assert got.shape == (2, 5, nr)
    for g, r in zip(got, recs):
        np.testing.assert_allclose(g.ravel(), r, rtol=6e-6, atol=1e-300)


def test_forcing_file_roundtrip(tmp_path):
    nx, nt = 5, 7
    f = np.random.default_rng(2).standard_normal((nx, nx, nt))
    path = str(tmp_path / "forcing" / "forcing_cubesph.3")
    outputs.write_forcing(path, f)
    raw = open(path, "rb").read()
    assert len(raw) == f.size * 8 + 8
    assert struct.unpack("<i", raw[:4])[0] == f.size * 8
    np.testing.assert_array_equal(outputs.read_forcing(path, nx, nx, nt), f)
    with pytest.raises(_lib.SolarError):
        outputs.read_forcing(path, nx, nx, nt + 1)
