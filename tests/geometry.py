"""Analytic cubed-sphere geometry used by the known-answer tests.

Face frames follow the reference's spherical coordinates (metric.f90:95-158): with
X = tan(xi), Y = tan(eta) the face points are F1 (1, X, Y), F2 (-X, 1, Y), F3 (-1, -X, Y),
F4 (X, -1, Y), F5 (-Y, X, 1), F6 (Y, X, -1), normalised.
"""
from __future__ import annotations

import numpy as np


def cube_point(face: int, X, Y):
    """Unit vector of zone ``face`` (1..6) at tangent coordinates X, Y."""
    X, Y = np.broadcast_arrays(np.asarray(X, float), np.asarray(Y, float))
    one = np.ones_like(X)
    v = {1: (one, X, Y), 2: (-X, one, Y), 3: (-one, -X, Y), 4: (X, -one, Y),
         5: (-Y, X, one), 6: (Y, X, -one)}[face]
    v = np.array(v)
    return v / np.linalg.norm(v, axis=0)


def theta_phi(face: int, X, Y):
    x, y, z = cube_point(face, X, Y)
    return np.arccos(np.clip(z, -1, 1)), np.mod(np.arctan2(y, x), 2 * np.pi)


def tp_to_xe(face: int, X, Y, a_th, a_ph):
    """CONVERT_THETA_PHI_TO_XI_ETA (transform.f90:63-111): global (theta, phi) components
    to the zone's (xi, eta) components."""
    C = np.sqrt(1 + X * X)
    D = np.sqrt(1 + Y * Y)
    dl = 1 + X * X + Y * Y
    sd = np.sqrt(dl)
    if face <= 4:
        return C * D / sd * a_ph, -a_th + X * Y / sd * a_ph
    f = 1 / np.sqrt(dl - 1)
    if face == 5:
        return (f * (D * X * a_th - D * Y / sd * a_ph), f * (C * Y * a_th + C * X / sd * a_ph))
    return (f * (-D * X * a_th + D * Y / sd * a_ph), -f * (C * Y * a_th + C * X / sd * a_ph))


def grid_xy(n: int):
    g = -np.pi / 4 + np.arange(n) * (np.pi / 2) / (n - 1)
    X = np.tan(g)[None, :]
    Y = np.tan(g)[:, None]
    return g, X, Y


def rotation_field(n: int, gr: np.ndarray, axis=(1.0, 0.0, 0.0)):
    """Solid-body rotation v = w x x (divergence free) as six-zone (v_xi, v_eta) fields."""
    _, X, Y = grid_xy(n)
    nr = len(gr)
    vxi = np.zeros((6, nr, n, n))
    veta = np.zeros_like(vxi)
    w = np.asarray(axis, float)
    for z in range(1, 7):
        th, ph = theta_phi(z, X, Y)
        x = np.array([np.sin(th) * np.cos(ph), np.sin(th) * np.sin(ph), np.cos(th)])
        V = np.cross(w, x, axis=0)
        e_th = np.array([np.cos(th) * np.cos(ph), np.cos(th) * np.sin(ph), -np.sin(th)])
        e_ph = np.array([-np.sin(ph), np.cos(ph), 0 * ph])
        a, b = tp_to_xe(z, X, Y, (V * e_th).sum(0), (V * e_ph).sum(0))
        vxi[z - 1] = a[None] * gr[:, None, None]
        veta[z - 1] = b[None] * gr[:, None, None]
    return vxi, veta


# the eight source strips whose receiver reverses them (face index 1..6, edge name)
REVERSED_RECEIVER_EDGES = {(2, "S"), (3, "S"), (3, "N"), (4, "N"), (5, "N"), (5, "W"), (6, "S"), (6, "E")}


def edge_maxima(err: np.ndarray, depth: int = 3, margin: int = 4):
    """max |err| near each edge of each zone (corners excluded): {(zone, edge): value}."""
    out = {}
    e = np.abs(err).max(axis=1)  # over k
    for z in range(6):
        out[(z + 1, "S")] = e[z, :depth, margin:-margin].max()
        out[(z + 1, "N")] = e[z, -depth:, margin:-margin].max()
        out[(z + 1, "W")] = e[z, margin:-margin, :depth].max()
        out[(z + 1, "E")] = e[z, margin:-margin, -depth:].max()
    return out
