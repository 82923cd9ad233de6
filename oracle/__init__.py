"""ctypes binding of the FP64 CPU oracle (test infrastructure only).

Only the test suite, ``__graft_entry__.smoke()`` and the benchmark's CPU-baseline /
reference arm may import this package.  It checks the GPU solver; it is never the
thing measured as the product.  See ``solar_oracle.h`` for the restated reference
routines and the array layouts.  Parity status: unpinned against golden vectors
(the reference ships none and cannot be built here); pinned to the reference's own
analytic checks (testcode.f90) by the test suite.
"""
from __future__ import annotations

import ctypes
import os
import subprocess
from typing import Optional

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_HERE, "_build", "liboracle.so")
_lib = None

_D = ctypes.POINTER(ctypes.c_double)


def build() -> str:
    """Compile the oracle with its Makefile (system g++ + OpenMP)."""
    subprocess.check_call(["make", "-s", "-C", _HERE])
    return _LIB_PATH


def _load():
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(_LIB_PATH):
        build()
    lib = ctypes.CDLL(_LIB_PATH)
    lib.oracle_create.restype = ctypes.c_void_p
    lib.oracle_create.argtypes = [ctypes.c_int, ctypes.c_int, _D, ctypes.c_double, ctypes.c_double,
                                  ctypes.c_double, ctypes.c_int, ctypes.c_int, ctypes.c_int, _D]
    lib.oracle_destroy.argtypes = [ctypes.c_void_p]
    lib.oracle_set_threads.argtypes = [ctypes.c_int]
    lib.oracle_set_fix_reversed_rotation.argtypes = [ctypes.c_void_p, ctypes.c_int]
    lib.oracle_get_grid.argtypes = [ctypes.c_void_p, ctypes.c_int, _D]
    lib.oracle_get_grid.restype = ctypes.c_int
    lib.oracle_add_gaussian.argtypes = [ctypes.c_void_p, _D] + [ctypes.c_double] * 5
    for name in ("oracle_interpolate_strips", "oracle_ddx", "oracle_ddy", "oracle_ddr",
                 "oracle_compute_rhs", "oracle_sponge", "oracle_filter_exp"):
        getattr(lib, name).argtypes = [ctypes.c_void_p, _D, _D]
    lib.oracle_bc_rhs.argtypes = [ctypes.c_void_p, _D]
    lib.oracle_gradient.argtypes = [ctypes.c_void_p, _D, _D, _D, _D]
    lib.oracle_divergence.argtypes = [ctypes.c_void_p, _D, _D, _D, _D]
    lib.oracle_filter_field.argtypes = [ctypes.c_void_p, _D, _D, ctypes.c_int]
    lib.oracle_rk4.argtypes = [ctypes.c_void_p, _D, ctypes.c_int]
    lib.oracle_norm.argtypes = [ctypes.c_void_p, _D, ctypes.c_int]
    lib.oracle_norm.restype = ctypes.c_double
    lib.oracle_curl.argtypes = [ctypes.c_void_p, _D, _D, _D, _D, _D, _D]
    lib.oracle_set_forcing.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_int, ctypes.c_int]
    lib.oracle_set_forcing.restype = ctypes.c_int
    lib.oracle_set_forcing_samples.argtypes = [ctypes.c_void_p, ctypes.c_int, _D, ctypes.c_int]
    lib.oracle_set_forcing_samples.restype = ctypes.c_int
    lib.oracle_set_clock.argtypes = [ctypes.c_void_p, ctypes.c_double, ctypes.c_int]
    lib.oracle_get_clock.argtypes = [ctypes.c_void_p, _D, ctypes.POINTER(ctypes.c_int)]
    _lib = lib
    return lib


def _p(a: np.ndarray):
    assert a.dtype == np.float64 and a.flags.c_contiguous
    return a.ctypes.data_as(_D)


def set_threads(n: int) -> None:
    _load().oracle_set_threads(int(n))


class Oracle:
    """All six zones of one run, FP64, reference arithmetic."""

    def __init__(self, cfg, c2_3d: Optional[np.ndarray] = None, fix_reversed_rotation: bool = False):
        lib = _load()
        self.cfg = cfg
        self.nx, self.nr = cfg.nx, cfg.nr
        self._model = np.ascontiguousarray(cfg.model, dtype=np.float64)
        sp = cfg.sponge
        self._c2 = None if c2_3d is None else np.ascontiguousarray(c2_3d, dtype=np.float64)
        self._h = lib.oracle_create(cfg.nx, cfg.nr, _p(self._model), float(cfg.dt), float(sp.amp),
                                    float(sp.exp), int(sp.length), int(sp.lower), int(sp.upper),
                                    None if self._c2 is None else _p(self._c2))
        if not self._h:
            raise ValueError("oracle_create rejected the configuration")
        self._lib = lib
        if fix_reversed_rotation:
            lib.oracle_set_fix_reversed_rotation(self._h, 1)

    def __del__(self):
        h = getattr(self, "_h", None)
        if h:
            self._lib.oracle_destroy(h)
            self._h = None

    # shapes
    @property
    def field_shape(self):
        return (6, self.nr, self.nx, self.nx)

    @property
    def state_shape(self):
        return (6, 5, self.nr, self.nx, self.nx)

    def zeros_state(self) -> np.ndarray:
        return np.zeros(self.state_shape)

    def grid(self, which: int) -> np.ndarray:
        n, nr = self.nx, self.nr
        size = {0: 6 * n * n, 1: 6 * n * n, 2: n, 3: nr, 4: nr, 5: 3 * n * 9, 6: 3 * n,
                7: nr, 8: nr, 9: nr, 10: nr, 11: nr}[which]
        out = np.zeros(size)
        self._lib.oracle_get_grid(self._h, which, _p(out))
        return out

    def initial_state(self, sources=None) -> np.ndarray:
        q = self.zeros_state()
        for s in (self.cfg.sources if sources is None else sources):
            self._lib.oracle_add_gaussian(self._h, _p(q), *map(float, s.x0), float(s.width), float(s.amp))
        return q

    # operators
    def strips(self, f):
        out = np.zeros((6, 4, self.nr, 3, self.nx))
        self._lib.oracle_interpolate_strips(self._h, _p(f), _p(out))
        return out

    def _unary(self, name, f):
        f = np.ascontiguousarray(f, dtype=np.float64)
        out = np.zeros_like(f)
        getattr(self._lib, name)(self._h, _p(f), _p(out))
        return out

    def ddx(self, f): return self._unary("oracle_ddx", f)
    def ddy(self, f): return self._unary("oracle_ddy", f)
    def ddr(self, f): return self._unary("oracle_ddr", f)

    def gradient(self, p):
        p = np.ascontiguousarray(p, dtype=np.float64)
        gx, ge, gr = np.zeros_like(p), np.zeros_like(p), np.zeros_like(p)
        self._lib.oracle_gradient(self._h, _p(p), _p(gx), _p(ge), _p(gr))
        return gx, ge, gr

    def divergence(self, vxi, veta, vr):
        a = [np.ascontiguousarray(x, dtype=np.float64) for x in (vxi, veta, vr)]
        out = np.zeros_like(a[0])
        self._lib.oracle_divergence(self._h, _p(a[0]), _p(a[1]), _p(a[2]), _p(out))
        return out

    def curl(self, axi, aeta, ar):
        """COMPUTE_CURL (grad.f90:140-255): returns (curl_xi, curl_eta, curl_r)."""
        a = [np.ascontiguousarray(x, dtype=np.float64) for x in (axi, aeta, ar)]
        out = [np.zeros(self.field_shape) for _ in range(3)]
        self._lib.oracle_curl(self._h, *(_p(x) for x in a), *(_p(x) for x in out))
        return tuple(out)

    def filter_field(self, f, which: int):
        f = np.ascontiguousarray(f, dtype=np.float64)
        out = np.zeros_like(f)
        self._lib.oracle_filter_field(self._h, _p(f), _p(out), int(which))
        return out

    def compute_rhs(self, q):
        return self._unary("oracle_compute_rhs", q)

    def bc_rhs(self, rhs):
        rhs = np.ascontiguousarray(rhs, dtype=np.float64).copy()
        self._lib.oracle_bc_rhs(self._h, _p(rhs))
        return rhs

    def sponge(self, q, rhs):
        q = np.ascontiguousarray(q, dtype=np.float64)
        rhs = np.ascontiguousarray(rhs, dtype=np.float64).copy()
        self._lib.oracle_sponge(self._h, _p(q), _p(rhs))
        return rhs

    def filter_exp(self, q):
        return self._unary("oracle_filter_exp", q)

    def rk4(self, q, nsteps: int = 1) -> np.ndarray:
        q = np.ascontiguousarray(q, dtype=np.float64).copy()
        self._lib.oracle_rk4(self._h, _p(q), int(nsteps))
        return q

    # source term and clock (compute_rhs_acoustic.f90:92-116, timestep.f90:82)
    def set_forcing(self, kind: int, k_center: int = 0, nstep: int = 0) -> None:
        if self._lib.oracle_set_forcing(self._h, int(kind), int(k_center), int(nstep)) != 0:
            raise ValueError("bad forcing arguments")

    def set_forcing_samples(self, zone: int, f, nt: int) -> None:
        f = np.ascontiguousarray(f, dtype=np.float64)
        if self._lib.oracle_set_forcing_samples(self._h, int(zone), _p(f), int(nt)) != 0:
            raise ValueError("bad forcing samples")

    def set_clock(self, time: float, step: int = 0) -> None:
        self._lib.oracle_set_clock(self._h, float(time), int(step))

    def get_clock(self):
        t, s = ctypes.c_double(), ctypes.c_int()
        self._lib.oracle_get_clock(self._h, ctypes.byref(t), ctypes.byref(s))
        return t.value, s.value

    def norm(self, q, field: int = 4) -> float:
        q = np.ascontiguousarray(q, dtype=np.float64)
        return float(self._lib.oracle_norm(self._h, _p(q), int(field)))
