"""Discrete adjoint through the C-ABI: transposition checks and gradient checks.

* Dot-product tests: <L q, mu> = <q, L^T mu> with the forward operator L taken from the
  FP64 oracle (COMPUTE_RHS + BC_RHS + SPONGE, FILTER_EXP, the RK4 step), so the GPU
  transposes are checked against an independent CPU restatement of the forward path.
  Tolerance: 1e-11 of ||L q|| ||mu|| (FP64).
* Misfit gradient dJ/dc against central finite differences of the misfit, computed with
  the GPU FP64 forward path and with the FP64 oracle (the CPU reference gradient), along
  random and smooth directions.  Tolerance: 1e-4 relative.
* dJ/dq0 against finite differences in the initial state; checkpoint-interval
  invariance; FP32 gradient against the FP64 gradient.
"""
import numpy as np
import pytest

from solar_b200 import _lib, configs, receivers
from solar_b200.solver import Solver

pytestmark = pytest.mark.gpu

DOT_TOL = 1e-11      # FP64 transposition, relative to ||L q|| ||mu||
FD_TOL = 1e-4        # adjoint gradient vs central finite differences


def dot(a, b):
    return float(np.vdot(np.ravel(a), np.ravel(b)))


@pytest.fixture(scope="module")
def c1s():
    return configs.c1(nx=32, nr=32)


@pytest.fixture(scope="module")
def c2s():
    return configs.c2(nx=32, nr=32, nsteps=30)


def random_state(shape, seed):
    return np.random.default_rng(seed).standard_normal(shape)


def near_source_receivers(cfg, m, seed, spread=0.12):
    """m receivers scattered around the configuration's first source."""
    rng = np.random.default_rng(seed)
    x0 = np.asarray(cfg.sources[0].x0)
    gr = configs.normalise(cfg.model)[0]
    pts = []
    while len(pts) < m:
        p = x0 + rng.uniform(-spread, spread, 3)
        r = np.linalg.norm(p)
        if gr[0] + 0.1 * (gr[-1] - gr[0]) < r < gr[-1] - 0.2 * (gr[-1] - gr[0]):
            pts.append(p)
    return receivers.locate(cfg, np.array(pts))


def sample_host(q, loc):
    """Trilinear p at the receivers from a host state (the formula of the C library)."""
    n, nr = q.shape[-1], q.shape[2]
    out = np.zeros(len(loc))
    for r, (f, x, y, z) in enumerate(loc):
        i0, j0, k0 = min(int(x), n - 2), min(int(y), n - 2), min(int(z), nr - 2)
        wx, wy, wz = x - i0, y - j0, z - k0
        s = 0.0
        for dk in (0, 1):
            for dj in (0, 1):
                for di in (0, 1):
                    w = (wx if di else 1 - wx) * (wy if dj else 1 - wy) * (wz if dk else 1 - wz)
                    s += w * q[int(f), 4, k0 + dk, j0 + dj, i0 + di]
        out[r] = s
    return out


def gpu_traces(cfg, c, q0, loc, nsteps, precision="fp64", nfields=5):
    with Solver(cfg, precision=precision, nfields=nfields, c2_3d=c ** 2) as s:
        s.set_state(q0)
        s.set_receivers(loc)
        return s.record(nsteps)


def oracle_traces(oracle_mod, cfg, c, q0, loc, nsteps):
    o = oracle_mod.Oracle(cfg, c2_3d=c ** 2)
    q = q0.copy()
    out = np.zeros((nsteps, len(loc)))
    for n in range(nsteps):
        q = o.rk4(q, 1)
        out[n] = sample_host(q, loc)
    return out


def misfit(tr, data):
    return 0.5 * float(((tr - data) ** 2).sum())


def gradient_case(oracle_mod, cfg, nsteps, nrec=8, seed=0):
    """Initial state, receivers, synthetic data from a model with a sound-speed anomaly
    between source and receivers, and the background model."""
    o = oracle_mod.Oracle(cfg)
    q0 = o.initial_state()
    loc = near_source_receivers(cfg, nrec, seed)
    x0 = np.asarray(cfg.sources[0].x0)
    c0 = receivers.sound_speed(cfg)
    c_true = receivers.sound_speed(cfg, [(tuple(x0 * 0.97), 0.08, 0.05)])
    data = gpu_traces(cfg, c_true, q0, loc, nsteps)
    return q0, loc, c0, data


def adjoint_gradient(cfg, c, q0, loc, data, nsteps, k, precision="fp64", nfields=5, want_lambda=False):
    with Solver(cfg, precision=precision, nfields=nfields, c2_3d=c ** 2) as s:
        s.set_state(q0)
        s.set_receivers(loc)
        return s.misfit_gradient(nsteps, k, data, want_lambda=want_lambda)


def interior_direction(cfg, seed, smooth=False):
    rng = np.random.default_rng(seed)
    if smooth:     # a blob in the region the receivers are sensitive to
        centre = np.asarray(cfg.sources[0].x0) * 0.95 + rng.uniform(-0.05, 0.05, 3)
        d = receivers.sound_speed(cfg, [(tuple(centre), 0.1, 1.0)]) - receivers.sound_speed(cfg)
    else:
        d = rng.standard_normal((6, cfg.nr, cfg.nx, cfg.nx)) * receivers.sound_speed(cfg)
    d[:, 0] = 0.0
    d[:, -1] = 0.0
    return d


# ---------------------------------------------------------------- transposition
@pytest.mark.parametrize("cfgname", ["c1s", "c2s"])
def test_rhs_adjoint_is_transpose_of_oracle_rhs(oracle_mod, cfgname, request):
    cfg = request.getfixturevalue(cfgname)
    o = oracle_mod.Oracle(cfg)
    q = random_state(o.state_shape, 1)
    mu = random_state(o.state_shape, 2)
    Lq = o.sponge(q, o.bc_rhs(o.compute_rhs(q)))
    with Solver(cfg) as s:
        LTmu = s.rhs_adjoint(mu)
    a, b = dot(Lq, mu), dot(q, LTmu)
    scale = np.linalg.norm(Lq) * np.linalg.norm(mu)
    assert abs(a - b) <= DOT_TOL * scale, (a, b, abs(a - b) / scale)


@pytest.mark.parametrize("cfgname", ["c1s", "c2s"])
def test_filter_adjoint_is_transpose_of_oracle_filter(oracle_mod, cfgname, request):
    cfg = request.getfixturevalue(cfgname)
    o = oracle_mod.Oracle(cfg)
    q = random_state(o.state_shape, 3)
    lam = random_state(o.state_shape, 4)
    Fq = o.filter_exp(q)
    with Solver(cfg) as s:
        FTlam = s.filter_adjoint(lam)
    a, b = dot(Fq, lam), dot(q, FTlam)
    scale = np.linalg.norm(Fq) * np.linalg.norm(lam)
    assert abs(a - b) <= DOT_TOL * scale, (a, b, abs(a - b) / scale)


def test_rhs_adjoint_fixed_rotation_option(oracle_mod, c1s):
    o = oracle_mod.Oracle(c1s, fix_reversed_rotation=True)
    q = random_state(o.state_shape, 5)
    mu = random_state(o.state_shape, 6)
    Lq = o.sponge(q, o.bc_rhs(o.compute_rhs(q)))
    with Solver(c1s, fix_reversed_rotation=True) as s:
        LTmu = s.rhs_adjoint(mu)
    a, b = dot(Lq, mu), dot(q, LTmu)
    assert abs(a - b) <= DOT_TOL * np.linalg.norm(Lq) * np.linalg.norm(mu)


def test_rk4_adjoint_is_transpose_of_oracle_steps(oracle_mod, c2s):
    o = oracle_mod.Oracle(c2s)
    q = random_state(o.state_shape, 7)
    lam = random_state(o.state_shape, 8)
    Sq = o.rk4(q, 3)
    with Solver(c2s) as s:
        STlam = s.rk4_adjoint(3, lam)
    a, b = dot(Sq, lam), dot(q, STlam)
    scale = np.linalg.norm(Sq) * np.linalg.norm(lam)
    assert abs(a - b) <= DOT_TOL * scale, (a, b, abs(a - b) / scale)


def test_receiver_sampling_matches_host_trilinear(c1s):
    with Solver(c1s) as s:
        s.init_sources()
        loc = near_source_receivers(c1s, 6, 9)
        s.set_receivers(loc)
        tr = s.record(2)
        q = s.get_state()
    want = sample_host(q, loc)
    np.testing.assert_allclose(tr[-1], want, rtol=1e-13, atol=1e-15 * np.abs(want).max())


# ---------------------------------------------------------------- gradients
@pytest.fixture(scope="module")
def c2_case(oracle_mod, c2s):
    nsteps = 24
    q0, loc, c0, data = gradient_case(oracle_mod, c2s, nsteps)
    res = adjoint_gradient(c2s, c0, q0, loc, data, nsteps, 5, want_lambda=True)
    return dict(cfg=c2s, nsteps=nsteps, q0=q0, loc=loc, c0=c0, data=data, res=res)


def test_misfit_matches_oracle(oracle_mod, c2_case):
    cs = c2_case
    J_oracle = misfit(oracle_traces(oracle_mod, cs["cfg"], cs["c0"], cs["q0"], cs["loc"], cs["nsteps"]), cs["data"])
    assert cs["res"]["misfit"] > 0
    assert abs(cs["res"]["misfit"] - J_oracle) <= 1e-9 * J_oracle


@pytest.mark.parametrize("smooth", [False, True])
def test_gradient_matches_gpu_finite_differences(c2_case, smooth):
    cs = c2_case
    cfg, c0 = cs["cfg"], cs["c0"]
    d = interior_direction(cfg, 10 + smooth, smooth)
    eps = 1e-6 / np.abs(d / c0).max()
    Jp = misfit(gpu_traces(cfg, c0 + eps * d, cs["q0"], cs["loc"], cs["nsteps"]), cs["data"])
    Jm = misfit(gpu_traces(cfg, c0 - eps * d, cs["q0"], cs["loc"], cs["nsteps"]), cs["data"])
    fd = (Jp - Jm) / (2 * eps)
    ad = dot(cs["res"]["grad_c"], d)
    assert abs(ad) > 0
    assert abs(fd - ad) <= FD_TOL * abs(ad), (fd, ad, abs(fd - ad) / abs(ad))


def test_gradient_matches_oracle_finite_differences(oracle_mod, c2_case):
    """The CPU reference gradient: central differences of the FP64 oracle's misfit."""
    cs = c2_case
    cfg, c0 = cs["cfg"], cs["c0"]
    d = interior_direction(cfg, 12, smooth=True)
    eps = 1e-6 / np.abs(d / c0).max()
    Jp = misfit(oracle_traces(oracle_mod, cfg, c0 + eps * d, cs["q0"], cs["loc"], cs["nsteps"]), cs["data"])
    Jm = misfit(oracle_traces(oracle_mod, cfg, c0 - eps * d, cs["q0"], cs["loc"], cs["nsteps"]), cs["data"])
    fd = (Jp - Jm) / (2 * eps)
    ad = dot(cs["res"]["grad_c"], d)
    assert abs(fd - ad) <= FD_TOL * abs(ad), (fd, ad, abs(fd - ad) / abs(ad))


def test_gradient_is_zero_on_boundary_planes(c2_case):
    g = c2_case["res"]["grad_c"]
    assert np.all(g[:, 0] == 0) and np.all(g[:, -1] == 0)
    assert np.abs(g).max() > 0


def test_lambda0_is_gradient_wrt_initial_state(c2_case):
    cs = c2_case
    cfg = cs["cfg"]
    dq = random_state(cs["q0"].shape, 13) * np.abs(cs["q0"]).max()
    eps = 1e-3
    Jp = misfit(gpu_traces(cfg, cs["c0"], cs["q0"] + eps * dq, cs["loc"], cs["nsteps"]), cs["data"])
    Jm = misfit(gpu_traces(cfg, cs["c0"], cs["q0"] - eps * dq, cs["loc"], cs["nsteps"]), cs["data"])
    fd = (Jp - Jm) / (2 * eps)          # exact up to rounding: J is quadratic in q0
    ad = dot(cs["res"]["lambda0"], dq)
    assert abs(fd - ad) <= 1e-8 * abs(ad), (fd, ad)


def test_checkpoint_interval_does_not_change_gradient(c2_case):
    cs = c2_case
    other = adjoint_gradient(cs["cfg"], cs["c0"], cs["q0"], cs["loc"], cs["data"], cs["nsteps"], cs["nsteps"])
    g0, g1 = cs["res"]["grad_c"], other["grad_c"]
    assert other["misfit"] == cs["res"]["misfit"]
    assert np.linalg.norm(g1 - g0) <= 1e-12 * np.linalg.norm(g0)


@pytest.mark.parametrize("outer,inner", [(10, 3), (24, 5), (7, 1)])
def test_nested_checkpoints_give_the_same_gradient(c2_case, outer, inner):
    """Two checkpoint levels (ragged outer and inner segments included) reproduce the
    single-level sweep."""
    cs = c2_case
    with Solver(cs["cfg"], c2_3d=cs["c0"] ** 2) as s:
        s.set_state(cs["q0"])
        s.set_receivers(cs["loc"])
        r = s.misfit_gradient(cs["nsteps"], outer, cs["data"], want_lambda=True, inner_every=inner)
        np.testing.assert_array_equal(s.get_state(), cs["q0"])
    g0 = cs["res"]["grad_c"]
    assert r["misfit"] == cs["res"]["misfit"]
    assert np.linalg.norm(r["grad_c"] - g0) <= 1e-12 * np.linalg.norm(g0)
    assert np.linalg.norm(r["lambda0"] - cs["res"]["lambda0"]) <= 1e-12 * np.linalg.norm(cs["res"]["lambda0"])


def test_state_is_restored_after_gradient(c2s, c2_case):
    cs = c2_case
    with Solver(c2s, c2_3d=cs["c0"] ** 2) as s:
        s.set_state(cs["q0"])
        s.set_receivers(cs["loc"])
        s.misfit_gradient(cs["nsteps"], 7, cs["data"])
        np.testing.assert_array_equal(s.get_state(), cs["q0"])


def test_fp32_gradient_close_to_fp64(c2_case):
    cs = c2_case
    r32 = adjoint_gradient(cs["cfg"], cs["c0"], cs["q0"], cs["loc"], cs["data"], cs["nsteps"], 5,
                           precision="fp32", nfields=4)
    g64, g32 = cs["res"]["grad_c"], r32["grad_c"]
    assert np.linalg.norm(g32 - g64) <= 1e-3 * np.linalg.norm(g64)
    assert abs(r32["misfit"] - cs["res"]["misfit"]) <= 1e-4 * cs["res"]["misfit"]


# ---------------------------------------------------------------- errors
def test_adjoint_argument_errors(c1s):
    with Solver(c1s) as s:
        with pytest.raises(_lib.SolarError) as e:
            s.nrec = 1
            s.misfit_gradient(2, 1, np.zeros((2, 1)))
        assert e.value.status == _lib.SOLAR_ERR_STATE
        with pytest.raises(_lib.SolarError) as e:
            s.set_receivers([[0, 1.0, 1.0, c1s.nr]])            # k beyond the last plane
        assert e.value.status == _lib.SOLAR_ERR_ARG
        s.set_receivers([[0, 1.0, 1.0, 1.0]])
        with pytest.raises(_lib.SolarError):
            s.misfit_gradient(2, 0, np.zeros((2, 1)))           # checkpoint interval 0
    with Solver(c1s, nruns=2) as s:
        with pytest.raises(_lib.SolarError) as e:
            s.set_receivers([[0, 1.0, 1.0, 1.0]])
        assert e.value.status == _lib.SOLAR_ERR_ARG
