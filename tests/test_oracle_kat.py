"""Known-answer tests that pin the FP64 oracle.

The reference has no automated tests or golden vectors.  Its scratch file testcode.f90
holds analytic print-checks (interpolation of sin(theta), DDY / DDX of sin(theta) on
zone 6 against closed forms, the divergence of v_theta = sin(theta), FILTER_ETA of
sin(theta), DDR of sin(r)); each becomes an assertion here.  Two further checks pin the
oracle's restatement of the vector edge exchange: a divergence-free rotation must give
div = 0 near every edge the reference handles correctly, and the reference's own defect
on the eight reversed vector strips must appear exactly there.
"""
import numpy as np
import pytest

from solar_b200 import configs
from tests import geometry as G


@pytest.fixture(scope="module")
def c1_16(oracle_mod):
    cfg = configs.c1(nx=32, nr=16)
    return cfg, oracle_mod.Oracle(cfg)


def sin_theta_field(o, n, nr):
    th = o.grid(0).reshape(6, n, n)
    return np.broadcast_to(np.sin(th)[:, None], (6, nr, n, n)).copy()


def test_grid_theta_phi_matches_cube_geometry(c1_16):
    cfg, o = c1_16
    n = cfg.nx
    th = o.grid(0).reshape(6, n, n)
    ph = o.grid(1).reshape(6, n, n)
    _, X, Y = G.grid_xy(n)
    for z in range(1, 7):
        t, p = G.theta_phi(z, X, Y)
        assert np.abs(t - th[z - 1]).max() < 1e-13
        assert np.abs(np.angle(np.exp(1j * (p - ph[z - 1])))).max() < 1e-13


def test_interpolation_of_sin_theta(c1_16):
    """testcode.f90:53-96: edge strips interpolated along x / y reproduce sin(theta) at the
    interpolation targets (metric.f90:89-91)."""
    cfg, o = c1_16
    n, nr = cfg.nx, cfg.nr
    f = sin_theta_field(o, n, nr)
    strips = o.strips(f)                       # [zone][S,N,W,E][k][layer][t]
    g = o.grid(2)
    ip = o.grid(6).reshape(3, n)
    worst = 0.0
    for z in range(1, 7):
        for e, name in enumerate("SNWE"):
            for l in range(3):
                if name == "S":
                    xi, eta = np.arctan(np.tan(ip[l])), np.full(n, g[l + 1])
                elif name == "N":
                    xi, eta = ip[l], np.full(n, g[n - 2 - l])
                elif name == "W":
                    xi, eta = np.full(n, g[l + 1]), ip[l]
                else:
                    xi, eta = np.full(n, g[n - 2 - l]), ip[l]
                th, _ = G.theta_phi(z, np.tan(xi), np.tan(eta))
                err = np.abs(strips[z - 1, e, :, l, :] - np.sin(th)[None]).max()
                worst = max(worst, err)
    assert worst < 2e-6


def test_ddy_ddx_sin_theta_zone6(c1_16):
    """testcode.f90:99-162: DDY / DDX of sin(theta) on zone 6 against the closed form
    Y D^2 (delta^-1/2 (delta-1)^-1/2 - delta^-3/2 (delta-1)^1/2)."""
    cfg, o = c1_16
    n, nr = cfg.nx, cfg.nr
    f = sin_theta_field(o, n, nr)
    _, X, Y = G.grid_xy(n)
    dl = 1 + X * X + Y * Y
    D2, C2 = 1 + Y * Y, 1 + X * X
    core = dl ** -0.5 * (dl - 1) ** -0.5 - dl ** -1.5 * (dl - 1) ** 0.5
    dy = o.ddy(f)[5, 0]
    dx = o.ddx(f)[5, 0]
    # sin(theta) has a cusp at the pole (face centre): compare where it is smooth
    away = (X * X + Y * Y) > 0.15
    assert np.abs(dy - Y * D2 * core)[away].max() < 2e-4
    assert np.abs(dx - X * C2 * core)[away].max() < 2e-4
    # the reference's own check prints the edge row j = my (testcode.f90:120-124)
    assert np.abs(dy[-1] - (Y * D2 * core)[-1]).max() < 2e-4


def test_filter_eta_of_sin_theta(c1_16):
    """testcode.f90:212-253: FILTER_ETA leaves a smooth field (nearly) unchanged."""
    cfg, o = c1_16
    n = cfg.nx
    f = sin_theta_field(o, n, cfg.nr)
    _, X, Y = G.grid_xy(n)
    away = np.broadcast_to((X * X + Y * Y) > 0.15, (n, n))
    smooth = np.ones((6, 1, n, n), bool)
    smooth[4:, 0] = away  # sin(theta) has a cusp at the poles (centres of faces 5, 6)
    smooth = np.broadcast_to(smooth, f.shape)
    th = o.grid(0).reshape(6, n, n)
    g = np.broadcast_to(np.cos(th)[:, None], f.shape).copy()  # smooth everywhere
    for which in (0, 1):
        assert np.abs(o.filter_field(f, which) - f)[smooth].max() < 1e-6
        assert np.abs(o.filter_field(g, which) - g).max() < 1e-6


def test_filter_r_zeroes_end_planes(c1_16):
    cfg, o = c1_16
    f = sin_theta_field(o, cfg.nx, cfg.nr) + 1.0
    out = o.filter_field(f, 2)
    assert np.all(out[:, :5] == 0) and np.all(out[:, -5:] == 0)
    assert np.abs(out[:, 5:-5] - f[:, 5:-5]).max() < 5e-6  # radial weights sum to 0.999998


@pytest.mark.parametrize("nr", [32, 64])
def test_ddr_sin_r(oracle_mod, nr):
    """testcode.f90:257-280: DDR of sin(r) against cos(r), one-sided rows included."""
    cfg = configs.c1(nx=16, nr=nr)
    o = oracle_mod.Oracle(cfg)
    r = o.grid(3)
    f = np.broadcast_to(np.sin(r)[None, :, None, None], (6, nr, 16, 16)).copy()
    d = o.ddr(f)
    err = np.abs(d - np.cos(r)[None, :, None, None]).max()
    assert err < (2e-5 if nr == 32 else 1e-6)


def test_divergence_of_sin_theta(c1_16):
    """testcode.f90:164-205: div of v_theta = sin(theta) is 2 cos(theta)/r."""
    cfg, o = c1_16
    n, nr = cfg.nx, cfg.nr
    r = o.grid(3)
    _, X, Y = G.grid_xy(n)
    vxi = np.zeros((6, nr, n, n))
    veta = np.zeros_like(vxi)
    exact = np.zeros_like(vxi)
    for z in range(1, 7):
        th, _ = G.theta_phi(z, X, Y)
        a, b = G.tp_to_xe(z, X, Y, np.sin(th), 0 * th)
        vxi[z - 1] = a[None]
        veta[z - 1] = b[None]
        exact[z - 1] = 2 * np.cos(th)[None] / r[:, None, None]
    div = o.divergence(vxi, veta, np.zeros_like(vxi))
    # interior: scheme accuracy; edges: v_phi = 0 so the rotation defect does not enter
    assert np.abs(div - exact).max() < 5e-4


def test_rotation_divergence_free_and_reference_defect(oracle_mod):
    """A solid-body rotation is divergence free.  With the reference's arithmetic the
    eight reversed vector strips (transform.f90:184-274 evaluated at the sender's own
    edge index) give O(1) errors on exactly those receiver edges; with the corrected
    option every edge is at truncation level."""
    cfg = configs.c1(nx=32, nr=16)
    ref = oracle_mod.Oracle(cfg)
    fix = oracle_mod.Oracle(cfg, fix_reversed_rotation=True)
    r = ref.grid(3)
    vxi, veta = G.rotation_field(cfg.nx, r)
    vr = np.zeros_like(vxi)
    d_ref = G.edge_maxima(ref.divergence(vxi, veta, vr))
    d_fix = G.edge_maxima(fix.divergence(vxi, veta, vr))
    for key, v in d_fix.items():
        assert v < 1e-4, key
    for key, v in d_ref.items():
        if key in G.REVERSED_RECEIVER_EDGES:
            assert v > 0.1, key
        else:
            assert v < 1e-4, key


def test_rk4_short_run_is_finite_and_damped(oracle_mod):
    cfg = configs.c1(nx=16, nr=16)
    o = oracle_mod.Oracle(cfg)
    q0 = o.initial_state()
    n0 = o.norm(q0, 5)
    q = o.rk4(q0, 10)
    assert np.isfinite(q).all()
    assert 0 < o.norm(q, 5) < 2 * n0


def test_bc_and_sponge_semantics(c1_16):
    cfg, o = c1_16
    rng = np.random.default_rng(0)
    q = rng.standard_normal(o.state_shape)
    rhs = rng.standard_normal(o.state_shape)
    bc = o.bc_rhs(rhs)
    assert np.all(bc[:, :, 0] == 0) and np.all(bc[:, :, -1] == 0)
    assert np.array_equal(bc[:, :, 1:-1], rhs[:, :, 1:-1])
    sp = o.sponge(q, rhs)
    sig = o.grid(10)
    for m in range(5):
        want = rhs[:, m] - (sig[None, :, None, None] * q[:, m] if m in (0, 3, 4) else 0)
        assert np.allclose(sp[:, m], want, rtol=0, atol=1e-15)


def test_sponge_profile_single_precision_ratio(oracle_mod):
    """sponge.f90:40-46: sigma = 0.1 (REAL(d)/REAL(30))^3 with a single-precision ratio;
    with nr = 32 and 30-point sponges the two branches overlap (upper wins for gk >= 3)."""
    cfg = configs.c1(nx=16, nr=32)
    sig = oracle_mod.Oracle(cfg).grid(10)
    gk = np.arange(1, 33)
    want = np.where(gk >= 3, 0.1 * (np.float32(gk - 3) / np.float32(30)).astype(np.float64) ** 3,
                    0.1 * (np.float32(30 - gk) / np.float32(30)).astype(np.float64) ** 3)
    assert np.allclose(sig, want, rtol=1e-14, atol=0)
    # a double-precision ratio differs at the 1e-8 level: the oracle keeps the float one
    dbl = np.where(gk >= 3, 0.1 * ((gk - 3) / 30.0) ** 3, 0.1 * ((30 - gk) / 30.0) ** 3)
    assert np.abs(sig - dbl).max() > 1e-10
