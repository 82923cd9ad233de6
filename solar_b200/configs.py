"""Synthetic inputs for the solver's benchmark workloads.

The reference reads its background from a file ``solar_model`` (nr rows of
r/R, c, rho, p, T, g, Gamma, unused; ic_acoustic_wave.f90:61-66) and
normalises it by its first row (ic_acoustic_wave.f90:73-108).  It seeds its
state with ``GENERATE_IC`` (ic_acoustic_wave.f90:4-29), a plug-in slot selected at
link time (makefile:16).  Neither the model file nor a public dataset exists
here, so this module builds seeded synthetic ``solar_model`` tables and source
parameters with the shapes the workloads call for:

* ``c1``  6 x 32^3 shell r in [0.5, 1], c = rho = 1, g = 0, one Gaussian pressure
  pulse (width 0.05) at x0 = (0, 0, 0.75); the reference's own sponge
  (a = 0.1, cubic, 30 points at both radial ends); 100 steps.
* ``c2``  6 x 128^3 stratified shell r in [0.7, 1], s = (1-r)/0.3,
  c = 0.1 + 0.9 s^0.5, rho0 = (s + 0.01)^1.5; sponge on the outer 5% of r only;
  one pulse of width 0.02 at r = 0.95 in a seeded uniform direction; 1000 steps.
* ``c3``  64 independent runs on 6 x 64^3 with the c2 background, per-run seeded
  direction, width U[0.01, 0.03], amplitude U[0.5, 2], steps U{200..1000}.
* ``c4``  6 x 96^3 c2 background, one pulse (width 0.02) at r = 0.95, a seeded
  sound-speed perturbation (eight Gaussian blobs of width 0.03, relative amplitude
  0.01, between the source and the receivers) and 32 receivers at r = 0.98 within
  0.05-0.25 rad of the source direction (the distance sound travels near r = 0.95
  in 500 steps is about 0.3), 500 steps.
* ``c5``  6 x 384^3 c2 background, 16 seeded sources, 200 steps.

The time step follows a CFL of 0.5 (the reference overrides its own CFL estimate
with a constant at timestep.f90:35): dt = 0.5 min_k min(r_k dxi, dr_k) / c_k.
Every function here emits parameters only (tables, centres, widths); fields are
generated by the solver or the oracle from them.
"""
from __future__ import annotations

import math
from dataclasses import dataclass, field
from typing import List, Optional, Tuple

import numpy as np

RSUN = 695.9894e8  # ic_acoustic_wave.f90:76


@dataclass
class Source:
    """A Gaussian pressure pulse p += amp * exp(-|x - x0|^2 / (2 width^2))."""

    x0: Tuple[float, float, float]
    width: float
    amp: float = 1.0


@dataclass
class Sponge:
    """Radial sponge of sponge.f90:18-46: sigma = a ((distance in points)/len)^exp.

    ``lower``/``upper`` keep the inner / outer branch of the reference's test
    (sponge.f90:40-46); the reference keeps both with len = 30."""

    amp: float = 0.1
    exp: float = 3.0
    length: int = 30
    lower: bool = True
    upper: bool = True


@dataclass
class Config:
    name: str
    nx: int
    nr: int
    model: np.ndarray                 # (nr, 8) solar_model rows
    dt: float
    nsteps: int
    sponge: Sponge
    sources: List[Source] = field(default_factory=list)
    # batched workloads: per-run sources and step counts
    runs: Optional[List[List[Source]]] = None
    run_steps: Optional[List[int]] = None
    # adjoint workload extras
    dc_blobs: Optional[List[Tuple[Tuple[float, float, float], float, float]]] = None
    receivers: Optional[np.ndarray] = None

    @property
    def points(self) -> int:
        """Grid points of one run (six faces)."""
        return 6 * self.nx * self.nx * self.nr


# --------------------------------------------------------------------- tables
def uniform_radius(nr: int, rmin: float, rmax: float) -> np.ndarray:
    k = np.arange(nr, dtype=np.float64)
    return rmin + (rmax - rmin) * k / (nr - 1)


def model_uniform(nr: int, rmin: float = 0.5, rmax: float = 1.0) -> np.ndarray:
    """solar_model rows for a uniform medium c = rho = p = 1, g = 0."""
    m = np.zeros((nr, 8))
    m[:, 0] = uniform_radius(nr, rmin, rmax)
    m[:, 1] = 1.0
    m[:, 2] = 1.0
    m[:, 3] = 1.0
    m[:, 4] = 1.0
    m[:, 5] = 0.0
    m[:, 6] = 1.67
    return m


def model_stratified(nr: int, rmin: float = 0.7, rmax: float = 1.0) -> np.ndarray:
    """solar_model rows for the stratified shell: s = (1-r)/0.3,
    c = 0.1 + 0.9 s^0.5, rho = (s + 0.01)^1.5, g = 0."""
    r = uniform_radius(nr, rmin, rmax)
    s = np.clip((1.0 - r) / 0.3, 0.0, None)
    c = 0.1 + 0.9 * np.sqrt(s)
    rho = (s + 0.01) ** 1.5
    m = np.zeros((nr, 8))
    m[:, 0] = r
    m[:, 1] = c
    m[:, 2] = rho
    m[:, 3] = rho * c * c / 1.67
    m[:, 4] = 1.0
    m[:, 5] = 0.0
    m[:, 6] = 1.67
    return m


def normalise(model: np.ndarray):
    """SOLAR_DATA (ic_acoustic_wave.f90:73-108): background normalised by row 1.

    Returns (gr, c2, rho0, g0) as float64 arrays of length nr."""
    dimc = model[0, 1]
    dimrho = model[0, 2]
    gr = model[:, 0].copy()
    c2 = (model[:, 1] / dimc) ** 2.0
    rho0 = model[:, 2] / dimrho
    g0 = model[:, 5] * RSUN / dimc ** 2.0
    return gr, c2, rho0, g0


def cfl_dt(nx: int, model: np.ndarray, cfl: float = 0.5) -> float:
    """dt = cfl * min_k min(r_k dxi, dr_k) / c_k with c normalised by row 1."""
    gr, c2, _, _ = normalise(model)
    c = np.sqrt(c2)
    dxi = (math.pi * 0.5) / (nx - 1)
    d = np.diff(gr)
    dr = np.empty_like(gr)
    dr[0] = d[0]
    dr[-1] = d[-1]
    dr[1:-1] = np.minimum(d[:-1], d[1:])
    return float(cfl * np.min(np.minimum(gr * dxi, dr) / c))


def outer_sponge(nr: int, frac: float = 0.05) -> Sponge:
    """Sponge over the outer ``frac`` of the radial extent: the points with
    chi >= 1 - frac, upper branch only."""
    length = nr - int(math.ceil((1.0 - frac) * (nr - 1) - 1e-9))
    return Sponge(amp=0.1, exp=3.0, length=max(length, 1), lower=False, upper=True)


def unit_vectors(rng: np.random.Generator, n: int) -> np.ndarray:
    v = rng.standard_normal((n, 3))
    return v / np.linalg.norm(v, axis=1, keepdims=True)


# --------------------------------------------------------------------- configs
def c1(nx: int = 32, nr: Optional[int] = None, nsteps: int = 100) -> Config:
    nr = nx if nr is None else nr
    model = model_uniform(nr, 0.5, 1.0)
    return Config("c1", nx, nr, model, cfl_dt(nx, model), nsteps, Sponge(),
                  [Source((0.0, 0.0, 0.75), 0.05, 1.0)])


def c2(nx: int = 128, nr: Optional[int] = None, nsteps: int = 1000) -> Config:
    nr = nx if nr is None else nr
    model = model_stratified(nr)
    d = unit_vectors(np.random.default_rng(2), 1)[0] * 0.95
    return Config("c2", nx, nr, model, cfl_dt(nx, model), nsteps, outer_sponge(nr),
                  [Source(tuple(d), 0.02, 1.0)])


def c3(nx: int = 64, nruns: int = 64, smin: int = 200, smax: int = 1000) -> Config:
    nr = nx
    model = model_stratified(nr)
    rng = np.random.default_rng(3)
    dirs = unit_vectors(rng, nruns) * 0.95
    widths = rng.uniform(0.01, 0.03, nruns)
    amps = rng.uniform(0.5, 2.0, nruns)
    steps = rng.integers(smin, smax + 1, nruns)
    runs = [[Source(tuple(dirs[i]), float(widths[i]), float(amps[i]))] for i in range(nruns)]
    return Config("c3", nx, nr, model, cfl_dt(nx, model), int(steps.max()), outer_sponge(nr),
                  runs[0], runs=runs, run_steps=[int(s) for s in steps])


def c4(nx: int = 96, nsteps: int = 500, receiver_r: float = 0.98) -> Config:
    """Adjoint workload.  Receivers sit at r = 0.98: the reference filter zeroes the
    five outermost radial planes every step (filter.f90:726-775), which at nr = 96
    covers r >= 0.987, so receivers at r = 0.99 would read p = 0.  Receivers and
    anomalies lie within reach of the pulse in 500 steps."""
    nr = nx
    model = model_stratified(nr)
    rng = np.random.default_rng(4)
    d = unit_vectors(rng, 1)[0]

    def around(m, lo, hi):
        """m unit vectors at angular distance U[lo, hi] from d, uniform azimuth."""
        a = np.cross(d, [0.0, 0.0, 1.0] if abs(d[2]) < 0.9 else [1.0, 0.0, 0.0])
        a /= np.linalg.norm(a)
        b = np.cross(d, a)
        ang = rng.uniform(lo, hi, m)
        az = rng.uniform(0.0, 2 * np.pi, m)
        return (np.cos(ang)[:, None] * d + np.sin(ang)[:, None] *
                (np.cos(az)[:, None] * a + np.sin(az)[:, None] * b))

    centres = around(8, 0.03, 0.2) * rng.uniform(0.9, 0.97, (8, 1))
    blobs = [(tuple(centres[i]), 0.03, 0.01) for i in range(8)]
    rec = around(32, 0.05, 0.25) * receiver_r
    return Config("c4", nx, nr, model, cfl_dt(nx, model), nsteps, outer_sponge(nr),
                  [Source(tuple(d * 0.95), 0.02, 1.0)], dc_blobs=blobs, receivers=rec)


def c5(nx: int = 384, nsteps: int = 200, nsrc: int = 16) -> Config:
    nr = nx
    model = model_stratified(nr)
    rng = np.random.default_rng(5)
    dirs = unit_vectors(rng, nsrc) * 0.95
    widths = rng.uniform(0.01, 0.03, nsrc)
    amps = rng.uniform(0.5, 2.0, nsrc)
    src = [Source(tuple(dirs[i]), float(widths[i]), float(amps[i])) for i in range(nsrc)]
    return Config("c5", nx, nr, model, cfl_dt(nx, model), nsteps, outer_sponge(nr), src)


CONFIGS = {"c1": c1, "c2": c2, "c3": c3, "c4": c4, "c5": c5}


def get(name: str, **kw) -> Config:
    return CONFIGS[name](**kw)
