"""The oracle's source term (compute_rhs_acoustic.f90:92-116) against independent numpy
restatements, on the CPU: the analytic S(theta, phi, r, t) and LAGRANGE_INTERP
(interpolation.f90:385-451) with its saved nodes and coefficients."""
import dataclasses

import numpy as np
import pytest

from solar_b200 import configs

RSUN = 695.9894e8


def scaled(cfg, dimc=RSUN / 1000.0):
    """Same normalised medium with a dimensional sound-speed scale, so that the physical
    time tau = t * rsun / dimc advances 1000 s per unit of normalised time."""
    m = cfg.model.copy()
    m[:, 1] *= dimc
    return dataclasses.replace(cfg, model=m)


@pytest.fixture(scope="module")
def cfg():
    return scaled(configs.c1(nx=16, nr=16))


def test_analytic_source_matches_formula(oracle_mod, cfg):
    o = oracle_mod.Oracle(cfg)
    kc = 9
    o.set_forcing(1, kc)
    n, nr = cfg.nx, cfg.nr
    th = o.grid(0).reshape(6, n, n)
    ph = o.grid(1).reshape(6, n, n)
    gr = o.grid(3)
    dxi = o.grid(2)[1] - o.grid(2)[0]
    dchi = 1.0 / (nr - 1)
    for t in (0.60, 0.65, 0.70):
        o.set_clock(t, 0)
        rhs = o.compute_rhs(np.zeros(o.state_shape))
        u = t * 1000.0 - 650.0
        mag = np.exp(-u * u / (2 * 200.0 ** 2)) * np.cos(4 * np.pi * u / 700.0)
        want = mag * np.exp(-((th[:, None] - np.pi / 2) / (20 * dxi)) ** 2 - (ph[:, None] / (20 * dxi)) ** 2
                            - ((gr[None, :, None, None] - gr[kc]) / (20 * dchi)) ** 2)
        np.testing.assert_allclose(rhs[:, 3], want, rtol=1e-13, atol=1e-15 * abs(mag))
        for f in (0, 1, 2, 4):
            assert not rhs[:, f].any()


def lagrange_reference(samples, nstep, dt, cad, steps):
    """interpolation.f90:385-451 for one point: the forcing value at each step in `steps`
    (called once per step, in order, from step_old = 0)."""
    step_old, x, lc, out = 0, [0.0] * 7, [0.0] * 7, []
    for step in steps:
        xt = step * dt / cad + 1.0
        fl = int(np.floor(xt))
        if step_old < fl:
            x = [(xt - 4.0 + m) * cad for m in range(7)]
            lc = [0.0] * 7
            for m in range(7):
                on = x[m] >= 0 if m <= 3 else (m == 4 or (m == 5 and fl < nstep) or (m == 6 and fl < nstep - 1))
                if on:
                    den = None
                    for j in range(7):
                        if j != m:
                            den = (x[m] - x[j]) if den is None else den * (x[m] - x[j])
                    lc[m] = samples[fl - 4 + m] / den
            step_old = fl
        xe = (step - 1.0) * dt
        f = None
        for m in range(7):
            t = lc[m]
            for j in range(7):
                if j != m:
                    t = t * (xe - x[j])
            f = t if f is None else f + t
        out.append(f)
    return np.array(out)


def test_sampled_source_follows_lagrange_interp(oracle_mod, cfg):
    o = oracle_mod.Oracle(cfg)
    n, nt, nstep = cfg.nx, 24, 200
    rng = np.random.default_rng(1)
    S = rng.standard_normal((6, n, n, nt))          # per zone f(i, j, n): i slowest
    for z in range(6):
        o.set_forcing_samples(z, S[z].ravel(), nt)
    o.set_forcing(2, 0, nstep)
    gr = o.grid(3)
    d = np.abs(gr - (1 - 100e5 / RSUN))
    e_rad = int(np.flatnonzero(d == d.min())[-1])
    cad = 60.0 * (RSUN / 1000.0) / RSUN
    got = []
    q = np.zeros(o.state_shape)
    o.set_clock(0.0, 0)
    for step in range(30):
        rhs = o.compute_rhs(q)
        got.append(rhs[:, 3, e_rad].copy())
        assert not np.delete(rhs[:, 3], e_rad, axis=1).any()
        q = o.rk4(q, 1) * 0.0                      # advance the clock only
    got = np.array(got)                            # [step][zone][j][i]
    for (z, j, i) in [(0, 3, 5), (4, 10, 2), (5, 15, 15)]:
        want = lagrange_reference(S[z, i, j], nstep, cfg.dt, cad, range(30))
        np.testing.assert_allclose(got[:, z, j, i], want, rtol=1e-12, atol=1e-14)


def test_constant_samples_interpolate_to_the_constant(oracle_mod, cfg):
    o = oracle_mod.Oracle(cfg)
    n, nt = cfg.nx, 40
    for z in range(6):
        o.set_forcing_samples(z, np.full(n * n * nt, 2.5), nt)
    o.set_forcing(2, 0, 500)
    cad = 60.0 * (RSUN / 1000.0) / RSUN
    first_full = int(np.ceil(3 * cad / cfg.dt)) + 1          # every node at t >= 0
    o.set_clock(first_full * cfg.dt, first_full)
    rhs = o.compute_rhs(np.zeros(o.state_shape))
    gr = o.grid(3)
    d = np.abs(gr - (1 - 100e5 / RSUN))
    e_rad = int(np.flatnonzero(d == d.min())[-1])          # ties go to the outer plane
    np.testing.assert_allclose(rhs[:, 3, e_rad], 2.5, rtol=1e-10)
