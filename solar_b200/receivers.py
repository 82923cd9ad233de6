"""Receivers and sound-speed fields for the adjoint entry points.

The adjoint C-ABI takes receiver positions as (zone, i, j, k) fractional grid indices.
This module maps Cartesian points to that form with the reference's face frames
(metric.f90:95-158: with X = tan(xi), Y = tan(eta), zone 1 points along (1, X, Y),
zone 2 (-X, 1, Y), zone 3 (-1, -X, Y), zone 4 (X, -1, Y), zone 5 (-Y, X, 1),
zone 6 (Y, X, -1)), and builds per-point sound-speed fields (the c2_3d descriptor
input) from the radial model plus Gaussian anomalies.
"""
from __future__ import annotations

import numpy as np

from .configs import Config, normalise


def _grid(cfg: Config):
    n = cfg.nx
    g = -np.pi / 4 + np.arange(n) * (np.pi / 2) / (n - 1)
    gr = normalise(cfg.model)[0]
    return g, gr


def locate(cfg: Config, points) -> np.ndarray:
    """Cartesian points (m, 3) -> rows (zone 0..5, i, j, k) of fractional grid indices."""
    p = np.asarray(points, dtype=np.float64).reshape(-1, 3)
    _, gr = _grid(cfg)
    n = cfg.nx
    out = np.zeros((p.shape[0], 4))
    for r, (x, y, z) in enumerate(p):
        a = np.abs([x, y, z])
        m = int(np.argmax(a))
        if m == 0 and x > 0:
            face, X, Y = 0, y / x, z / x
        elif m == 1 and y > 0:
            face, X, Y = 1, -x / y, z / y
        elif m == 0:
            face, X, Y = 2, y / x, -z / x
        elif m == 1:
            face, X, Y = 3, -x / y, -z / y
        elif z > 0:
            face, X, Y = 4, y / z, -x / z
        else:
            face, X, Y = 5, -y / z, -x / z
        fi = (np.arctan(X) + np.pi / 4) / (np.pi / 2) * (n - 1)
        fj = (np.arctan(Y) + np.pi / 4) / (np.pi / 2) * (n - 1)
        rad = float(np.sqrt(x * x + y * y + z * z))
        tol = 1e-12 * gr[-1]
        if not (gr[0] - tol <= rad <= gr[-1] + tol):
            raise ValueError(f"receiver {r} at radius {rad} lies outside the shell [{gr[0]}, {gr[-1]}]")
        fk = float(np.interp(min(max(rad, gr[0]), gr[-1]), gr, np.arange(len(gr))))
        out[r] = (face, min(max(fi, 0.0), n - 1), min(max(fj, 0.0), n - 1), fk)
    return out


def points(cfg: Config) -> np.ndarray:
    """Cartesian coordinates of every grid point, shape (6, nr, n, n, 3)."""
    g, gr = _grid(cfg)
    X = np.tan(g)[None, :]
    Y = np.tan(g)[:, None]
    one = np.ones((cfg.nx, cfg.nx))
    X, Y = np.broadcast_arrays(X, Y)
    frames = [(one, X, Y), (-X, one, Y), (-one, -X, Y), (X, -one, Y), (-Y, X, one), (Y, X, -one)]
    out = np.zeros((6, cfg.nr, cfg.nx, cfg.nx, 3))
    for z, v in enumerate(frames):
        v = np.stack(v, axis=-1)
        v = v / np.linalg.norm(v, axis=-1, keepdims=True)
        out[z] = gr[:, None, None, None] * v[None]
    return out


def sound_speed(cfg: Config, blobs=None) -> np.ndarray:
    """Per-point sound speed c (6, nr, n, n): the radial model times (1 + sum of relative
    Gaussian anomalies), blobs = [(centre (3,), width, relative amplitude), ...]."""
    c_r = np.sqrt(normalise(cfg.model)[1])
    c = np.broadcast_to(c_r[None, :, None, None], (6, cfg.nr, cfg.nx, cfg.nx)).copy()
    if blobs:
        xyz = points(cfg)
        rel = np.zeros(c.shape)
        for centre, width, amp in blobs:
            d2 = ((xyz - np.asarray(centre, dtype=np.float64)) ** 2).sum(-1)
            rel += amp * np.exp(-d2 / (2.0 * width * width))
        c *= 1.0 + rel
    return c
