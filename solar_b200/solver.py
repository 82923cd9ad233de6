"""Host-side mirror of the reference's time-stepping call surface.

The reference (Fortran 90 + MPI) exposes its hot path as the subroutines ``RK4``
(timestep.f90:41), ``COMPUTE_RHS`` (compute_rhs_acoustic.f90:1), ``BC_RHS``
(bc_acoustic_wave.f90:1), ``SPONGE`` (sponge.f90:1), ``FILTER_EXP`` (filter.f90:9),
``COMPUTE_GRADIENT`` / ``COMPUTE_DIVERGENCE`` (grad.f90:13, 62) and the diagnostic
``norm`` (auxiliary.f90:100).  :class:`Solver` offers the same operations, with the same
array meaning, over the C-ABI of ``include/solar_gpu.h``.  Arrays are numpy float64 in
"six-zone Fortran order": a field is ``f[zone, k, j, i]`` and a state is
``q[zone, m, k, j, i]`` with m = rho, v_xi, v_eta, v_r, p -- the reference's per-zone
arrays ``f(mx,my,mr)`` / ``q(mx,my,mr,5)`` stacked over the six zones.

Errors from the library raise :class:`solar_b200._lib.SolarError`; there is no CPU
fallback.
"""
from __future__ import annotations

import ctypes
from typing import Iterable, Optional, Sequence

import numpy as np

from . import _lib
from .configs import Config, Source

_D = ctypes.POINTER(ctypes.c_double)


def _ptr(a: np.ndarray):
    if a.dtype != np.float64 or not a.flags.c_contiguous:
        raise TypeError("arrays must be C-contiguous float64")
    return a.ctypes.data_as(_D)


class Solver:
    """One GPU context holding ``nruns`` independent six-face runs of one grid."""

    def __init__(self, cfg: Config, precision: str = "fp64", nfields: int = 5, nruns: int = 1,
                 device: int = 0, fix_reversed_rotation: bool = False,
                 c2_3d: Optional[np.ndarray] = None, tile: Optional[Sequence[int]] = None,
                 tuned: bool = True):
        self.lib = _lib.load()
        self.cfg = cfg
        self.nx, self.nr = cfg.nx, cfg.nr
        self.nruns = nruns
        self.nfields = nfields
        self.precision = precision
        d = _lib.SolarDesc()
        self.lib.solar_desc_defaults(ctypes.byref(d))
        self._model = np.ascontiguousarray(cfg.model, dtype=np.float64)
        self._c2 = None if c2_3d is None else np.ascontiguousarray(c2_3d, dtype=np.float64)
        d.nx, d.nr = cfg.nx, cfg.nr
        d.precision = {"fp64": _lib.SOLAR_FP64, "fp32": _lib.SOLAR_FP32}[precision]
        d.nfields = nfields
        d.nruns = nruns
        d.device = device
        d.dt = float(cfg.dt)
        d.model = _ptr(self._model)
        d.c2_3d = _ptr(self._c2) if self._c2 is not None else None
        sp = cfg.sponge
        d.sponge_amp, d.sponge_exp, d.sponge_len = float(sp.amp), float(sp.exp), int(sp.length)
        d.sponge_lower, d.sponge_upper = int(sp.lower), int(sp.upper)
        d.fix_reversed_rotation = int(bool(fix_reversed_rotation))
        if tile is None and tuned:
            from . import autotune
            tile = autotune.lookup(cfg.nx, cfg.nr, precision, nfields, nruns, device)
        if tile is not None:
            d.tile_x, d.tile_y, d.kchunk = (list(tile) + [0, 0, 0])[:3]
        self.tile = tile
        self.desc = d
        h = ctypes.c_void_p()
        _lib.check(self.lib.solar_gpu_init(ctypes.byref(d), ctypes.byref(h)))
        self._h = h

    # ------------------------------------------------------------------ lifetime
    def close(self) -> None:
        if getattr(self, "_h", None):
            self.lib.solar_gpu_finalize(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    # ------------------------------------------------------------------ shapes
    @property
    def field_shape(self):
        return (6, self.nr, self.nx, self.nx)

    @property
    def state_shape(self):
        return (6, 5, self.nr, self.nx, self.nx)

    @property
    def points(self) -> int:
        return 6 * self.nx * self.nx * self.nr

    # ------------------------------------------------------------------ state (COMMON /RKWORK/ q)
    def set_state(self, q: np.ndarray, run: int = 0) -> None:
        q = np.ascontiguousarray(q, dtype=np.float64)
        if q.shape != self.state_shape:
            raise ValueError(f"state shape {q.shape} != {self.state_shape}")
        _lib.check(self.lib.solar_gpu_set_state(self._h, run, _ptr(q)))

    def get_state(self, run: int = 0, out: Optional[np.ndarray] = None) -> np.ndarray:
        q = np.empty(self.state_shape) if out is None else out
        _lib.check(self.lib.solar_gpu_get_state(self._h, run, _ptr(q)))
        return q

    def add_gaussian(self, src: Source, run: int = 0) -> None:
        x0, y0, z0 = map(float, src.x0)
        _lib.check(self.lib.solar_gpu_add_gaussian(self._h, run, x0, y0, z0, float(src.width), float(src.amp)))

    def init_sources(self, sources: Optional[Iterable[Source]] = None, run: int = 0) -> None:
        """GENERATE_IC slot: zero state plus the configuration's Gaussian pulses."""
        self.set_state(np.zeros(self.state_shape), run)
        for s in (self.cfg.sources if sources is None else sources):
            self.add_gaussian(s, run)

    # ------------------------------------------------------------------ time stepping
    def rk4(self, nsteps: int = 1) -> None:
        """``nsteps`` calls of the reference's RK4 (timestep.f90:41-86) on every run."""
        _lib.check(self.lib.solar_gpu_rk4(self._h, int(nsteps)))

    def rk4_norms(self, nsteps: int, field: int = 4, run: int = 0, out: Optional[np.ndarray] = None) -> np.ndarray:
        """The loop of cube.f90:71-79: ``nsteps`` RK4 calls, each followed by the norm of
        ``field`` (auxiliary.f90:100-125); the norms are read back once, after the last step."""
        norms = np.empty(int(nsteps)) if out is None else out
        _lib.check(self.lib.solar_gpu_rk4_norms(self._h, int(run), int(field), int(nsteps), _ptr(norms)))
        return norms

    def set_watchdog(self, every: int) -> None:
        """Scan the state for NaN/Inf every ``every`` steps (0 = off); a hit makes the
        stepping call raise SolarError with status SOLAR_ERR_NAN."""
        _lib.check(self.lib.solar_gpu_set_watchdog(self._h, int(every)))

    def rk4_runs(self, steps: Sequence[int]) -> None:
        """Advance run r by steps[r] RK4 steps (uneven counts, one batched graph)."""
        s = np.ascontiguousarray(np.asarray(steps, dtype=np.int32))
        if s.shape != (self.nruns,):
            raise ValueError("need one step count per run")
        _lib.check(self.lib.solar_gpu_rk4_runs(self._h, s.ctypes.data_as(ctypes.POINTER(ctypes.c_int))))

    def time_rk4_runs(self, steps: Sequence[int]) -> float:
        """rk4_runs, returning the batch's device time in ms (CUDA events)."""
        s = np.ascontiguousarray(np.asarray(steps, dtype=np.int32))
        if s.shape != (self.nruns,):
            raise ValueError("need one step count per run")
        ms = ctypes.c_double()
        _lib.check(self.lib.solar_gpu_time_rk4_runs(self._h, s.ctypes.data_as(ctypes.POINTER(ctypes.c_int)),
                                                    ctypes.byref(ms)))
        return ms.value

    # ------------------------------------------------------------------ operators
    def compute_rhs(self, q: np.ndarray) -> np.ndarray:
        q = np.ascontiguousarray(q, dtype=np.float64)
        rhs = np.empty(self.state_shape)
        _lib.check(self.lib.solar_gpu_compute_rhs(self._h, _ptr(q), _ptr(rhs)))
        return rhs

    def bc_rhs(self, rhs: np.ndarray) -> np.ndarray:
        out = np.ascontiguousarray(rhs, dtype=np.float64).copy()
        _lib.check(self.lib.solar_gpu_bc_rhs(self._h, _ptr(out)))
        return out

    def sponge(self, q: np.ndarray, rhs: np.ndarray) -> np.ndarray:
        q = np.ascontiguousarray(q, dtype=np.float64)
        out = np.ascontiguousarray(rhs, dtype=np.float64).copy()
        _lib.check(self.lib.solar_gpu_sponge(self._h, _ptr(q), _ptr(out)))
        return out

    def filter_exp(self, q: np.ndarray) -> np.ndarray:
        q = np.ascontiguousarray(q, dtype=np.float64)
        qf = np.empty(self.state_shape)
        _lib.check(self.lib.solar_gpu_filter_exp(self._h, _ptr(q), _ptr(qf)))
        return qf

    def gradient(self, p: np.ndarray):
        p = np.ascontiguousarray(p, dtype=np.float64)
        gx, ge, gr = (np.empty(self.field_shape) for _ in range(3))
        _lib.check(self.lib.solar_gpu_gradient(self._h, _ptr(p), _ptr(gx), _ptr(ge), _ptr(gr)))
        return gx, ge, gr

    def divergence(self, vxi: np.ndarray, veta: np.ndarray, vr: np.ndarray) -> np.ndarray:
        a = [np.ascontiguousarray(x, dtype=np.float64) for x in (vxi, veta, vr)]
        out = np.empty(self.field_shape)
        _lib.check(self.lib.solar_gpu_divergence(self._h, _ptr(a[0]), _ptr(a[1]), _ptr(a[2]), _ptr(out)))
        return out

    def curl(self, axi: np.ndarray, aeta: np.ndarray, ar: np.ndarray):
        """COMPUTE_CURL (grad.f90:140-255): returns (curl_xi, curl_eta, curl_r)."""
        a = [np.ascontiguousarray(x, dtype=np.float64) for x in (axi, aeta, ar)]
        out = [np.empty(self.field_shape) for _ in range(3)]
        _lib.check(self.lib.solar_gpu_curl(self._h, *(_ptr(x) for x in a), *(_ptr(x) for x in out)))
        return tuple(out)

    # ------------------------------------------------------------------ diagnostics
    def norm(self, field: int = 4, run: int = 0) -> float:
        out = ctypes.c_double()
        _lib.check(self.lib.solar_gpu_norm(self._h, run, field, ctypes.byref(out)))
        return out.value

    def diag(self, run: int = 0) -> dict:
        out = (ctypes.c_double * 4)()
        _lib.check(self.lib.solar_gpu_diag(self._h, run, out))
        return {"energy": out[0], "mass": out[1], "max_abs_p": out[2], "nonfinite": bool(out[3])}

    def time_rk4(self, nsteps: int, per_kernel: bool = False) -> dict:
        out = (ctypes.c_double * 7)()
        _lib.check(self.lib.solar_gpu_time_rk4(self._h, int(nsteps), int(per_kernel), out))
        return {"total_ms": out[0], "stage_ms": out[1], "filter_ms": out[2], "edge_ms": out[3],
                "stage_launches": int(out[4]), "filter_launches": int(out[5]), "edge_launches": int(out[6])}

    def synchronize(self) -> None:
        _lib.check(self.lib.solar_gpu_synchronize(self._h))

    # ------------------------------------------------------------------ source term
    def set_forcing(self, kind: int, k_center: int = 0, nstep: int = 0) -> None:
        """v_r source of COMPUTE_RHS: 0 off, 1 analytic (compute_rhs_acoustic.f90:92-104,
        centre plane k_center), 2 sampled S_t with LAGRANGE_INTERP at plane e_rad."""
        _lib.check(self.lib.solar_gpu_set_forcing(self._h, int(kind), int(k_center), int(nstep)))

    def set_forcing_samples(self, zone: int, f: np.ndarray, nt: int) -> None:
        """Samples of one zone in READ_FORCING_FUNC order: f[(i*nx + j)*nt + n]."""
        f = np.ascontiguousarray(f, dtype=np.float64)
        _lib.check(self.lib.solar_gpu_set_forcing_samples(self._h, int(zone), _ptr(f), int(nt)))

    def load_forcing(self, dir: str, nt: int) -> None:
        """READ_FORCING_FUNC: dir/forcing/forcing_cubesph.<zone> for the six zones."""
        _lib.check(self.lib.solar_gpu_load_forcing(self._h, dir.encode(), int(nt)))

    def set_clock(self, time: float, step: int = 0) -> None:
        _lib.check(self.lib.solar_gpu_set_clock(self._h, float(time), int(step)))

    def get_clock(self):
        t, s = ctypes.c_double(), ctypes.c_int()
        _lib.check(self.lib.solar_gpu_get_clock(self._h, ctypes.byref(t), ctypes.byref(s)))
        return t.value, s.value

    # ------------------------------------------------------------------ output files
    def write_restart(self, dir: str, cue: int, time: float, step: int, run: int = 0) -> None:
        """WRITE_RESTART (output.f90:86-190) for the six zones of `run`."""
        _lib.check(self.lib.solar_gpu_write_restart(self._h, run, dir.encode(), int(cue), float(time), int(step)))

    def read_restart(self, dir: str, cue: int, run: int = 0):
        """Load the six restart files of `cue` into the state; returns (time, step)."""
        t, s = ctypes.c_double(), ctypes.c_int()
        _lib.check(self.lib.solar_gpu_read_restart(self._h, run, dir.encode(), int(cue), ctypes.byref(t), ctypes.byref(s)))
        return t.value, s.value

    def write_visual(self, dir: str, cue: int, run: int = 0) -> None:
        """WRITE_VISUAL (output.f90:192-240): plane o_rad of every zone."""
        _lib.check(self.lib.solar_gpu_write_visual(self._h, run, dir.encode(), int(cue)))

    def write_grid(self, dir: str) -> None:
        """WRITE_GRID (output.f90:242-267)."""
        _lib.check(self.lib.solar_gpu_write_grid(self._h, dir.encode()))

    def write_radial_trace(self, dir: str, run: int = 0) -> None:
        """WRITE_RADIAL_TRACE (output.f90:309-343): appends column (1, 1) of every zone."""
        _lib.check(self.lib.solar_gpu_write_radial_trace(self._h, run, dir.encode()))

    def output_plane(self) -> int:
        k = ctypes.c_int()
        _lib.check(self.lib.solar_gpu_output_plane(self._h, ctypes.byref(k)))
        return k.value

    # ------------------------------------------------------------------ adjoint
    def set_receivers(self, loc) -> None:
        """Receivers as rows (zone 0..5, i, j, k) of fractional 0-based grid indices."""
        loc = np.ascontiguousarray(loc, dtype=np.float64).reshape(-1, 4)
        self.nrec = loc.shape[0]
        _lib.check(self.lib.solar_gpu_set_receivers(self._h, self.nrec, _ptr(loc)))

    def record(self, nsteps: int) -> np.ndarray:
        """Run nsteps and return p at the receivers after every step, shape (nsteps, nrec)."""
        out = np.empty((int(nsteps), self.nrec))
        _lib.check(self.lib.solar_gpu_record(self._h, int(nsteps), _ptr(out)))
        return out

    def misfit_gradient(self, nsteps: int, checkpoint_every: int, data: np.ndarray,
                        want_lambda: bool = False, inner_every: Optional[int] = None) -> dict:
        """Misfit of the receiver traces against ``data`` (nsteps, nrec) and dJ/dc per point.
        ``inner_every`` < ``checkpoint_every`` selects the two-level checkpointed sweep."""
        data = np.ascontiguousarray(data, dtype=np.float64)
        if data.shape != (int(nsteps), self.nrec):
            raise ValueError(f"data must have shape {(int(nsteps), self.nrec)}")
        J = ctypes.c_double()
        grad = np.empty(self.field_shape)
        lam = np.empty(self.state_shape) if want_lambda else None
        times = (ctypes.c_double * 3)()
        inner = int(checkpoint_every if inner_every is None else inner_every)
        _lib.check(self.lib.solar_gpu_misfit_gradient_nested(
            self._h, int(nsteps), int(checkpoint_every), inner, _ptr(data), ctypes.byref(J), _ptr(grad),
            _ptr(lam) if lam is not None else None, times))
        out = {"misfit": J.value, "grad_c": grad,
               "forward_ms": times[0], "recompute_ms": times[1], "adjoint_ms": times[2]}
        if lam is not None:
            out["lambda0"] = lam
        return out

    def rhs_adjoint(self, mu: np.ndarray) -> np.ndarray:
        mu = np.ascontiguousarray(mu, dtype=np.float64)
        out = np.empty(self.state_shape)
        _lib.check(self.lib.solar_gpu_rhs_adjoint(self._h, _ptr(mu), _ptr(out)))
        return out

    def filter_adjoint(self, lam: np.ndarray) -> np.ndarray:
        lam = np.ascontiguousarray(lam, dtype=np.float64)
        out = np.empty(self.state_shape)
        _lib.check(self.lib.solar_gpu_filter_adjoint(self._h, _ptr(lam), _ptr(out)))
        return out

    def rk4_adjoint(self, nsteps: int, lam: np.ndarray) -> np.ndarray:
        lam = np.ascontiguousarray(lam, dtype=np.float64)
        out = np.empty(self.state_shape)
        _lib.check(self.lib.solar_gpu_rk4_adjoint(self._h, int(nsteps), _ptr(lam), _ptr(out)))
        return out
