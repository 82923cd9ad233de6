"""The v_r source term on the GPU against the FP64 oracle (compute_rhs_acoustic.f90:92-116,
LAGRANGE_INTERP interpolation.f90:385-451), through the C-ABI."""
import dataclasses

import numpy as np
import pytest

from solar_b200 import _lib, configs, receivers
from solar_b200.solver import Solver
from tests.test_oracle_forcing import scaled

pytestmark = pytest.mark.gpu


def rel(a, b):
    return np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300)


@pytest.fixture(scope="module")
def cfg():
    """A shell reaching past r = 1 (as the reference's grids do), so that the sampled
    source's plane e_rad (r nearest 1 - 100 km / R_sun) lies inside the 5 outer planes that
    FILTER_R zeroes; uniform medium, outer sponge."""
    model = configs.model_uniform(32, 0.6, 1.1)
    base = dataclasses.replace(configs.c2(nx=32, nr=32, nsteps=20), model=model, dt=configs.cfl_dt(32, model))
    return scaled(base)


def samples(cfg, nt, seed=3):
    return np.random.default_rng(seed).standard_normal((6, cfg.nx * cfg.nx * nt))


def test_compute_rhs_with_analytic_source(oracle_mod, cfg):
    o = oracle_mod.Oracle(cfg)
    q = o.initial_state()
    o.set_forcing(1, 20)
    o.set_clock(0.63, 5)
    want = o.compute_rhs(q)
    with Solver(cfg) as s:
        s.set_forcing(1, 20)
        s.set_clock(0.63, 5)
        got = s.compute_rhs(q)
        assert s.get_clock() == (0.63, 5)          # the operator does not advance the clock
    for f in range(5):
        assert rel(got[:, f], want[:, f]) <= 1e-12, f


@pytest.mark.parametrize("kind", [1, 2])
def test_rk4_with_source_fp64(oracle_mod, cfg, kind):
    o = oracle_mod.Oracle(cfg)
    nt = 24
    with Solver(cfg) as s:
        if kind == 2:
            S = samples(cfg, nt)
            for z in range(6):
                o.set_forcing_samples(z, S[z], nt)
                s.set_forcing_samples(z, S[z], nt)
        o.set_forcing(kind, 20, 200)
        s.set_forcing(kind, 20, 200)
        t0 = 0.62 if kind == 1 else 0.0
        o.set_clock(t0, 0)
        s.set_clock(t0, 0)
        q0 = np.zeros(o.state_shape)
        want = o.rk4(q0, 30)
        s.set_state(q0)
        s.rk4(30)
        got = s.get_state()
        tg, sg = s.get_clock()
    assert np.abs(want[:, 3]).max() > 0
    for f in range(5):
        assert rel(got[:, f], want[:, f]) <= 1e-11, (f, rel(got[:, f], want[:, f]))
    to, so = o.get_clock()
    assert sg == so == 30 and tg == to


def test_rk4_with_sampled_source_fp32(oracle_mod, cfg):
    o = oracle_mod.Oracle(cfg)
    nt = 24
    S = samples(cfg, nt, 4)
    with Solver(cfg, precision="fp32", nfields=4) as s:
        for z in range(6):
            o.set_forcing_samples(z, S[z], nt)
            s.set_forcing_samples(z, S[z], nt)
        o.set_forcing(2, 0, 200)
        s.set_forcing(2, 0, 200)
        q0 = np.zeros(o.state_shape)
        want = o.rk4(q0, 30)
        s.set_state(q0)
        s.rk4(30)
        got = s.get_state()
    for f in (1, 2, 3, 4):
        assert rel(got[:, f], want[:, f]) <= 1e-5, f


def test_phases_and_graph_agree_with_source(cfg):
    with Solver(cfg) as a, Solver(cfg) as b:
        for s in (a, b):
            s.set_forcing(1, 20)
            s.set_clock(0.62, 0)
            s.set_state(np.zeros(s.state_shape))
        a.rk4(3)
        for _ in range(3):
            for phase in range(6):
                _lib.check(b.lib.solar_gpu_step_phase(b._h, phase))
        b.synchronize()
        np.testing.assert_array_equal(a.get_state(), b.get_state())
        assert a.get_clock() == b.get_clock()


def test_source_errors(cfg):
    with Solver(cfg) as s:
        with pytest.raises(_lib.SolarError) as e:
            s.set_forcing(2, 0, 100)                    # no samples yet
        assert e.value.status == _lib.SOLAR_ERR_STATE
        with pytest.raises(_lib.SolarError):
            s.set_forcing(1, cfg.nr)                    # centre plane outside the grid
        nt = 6
        for z in range(6):
            s.set_forcing_samples(z, np.ones(cfg.nx * cfg.nx * nt), nt)
        s.set_forcing(2, 0, 1000)
        s.set_state(np.zeros(s.state_shape))
        with pytest.raises(_lib.SolarError) as e:       # runs past the last sample
            s.rk4(60)
        assert "sample" in str(e.value)


def test_adjoint_gradient_with_source(cfg):
    """Wave driven by the analytic source from rest: the checkpointed recomputation must
    replay the source clock; the gradient still matches central differences."""
    nsteps = 16
    loc = receivers.locate(cfg, [[0.95, 0.02, 0.01], [0.93, -0.05, 0.03], [0.96, 0.0, -0.04]])
    c0 = receivers.sound_speed(cfg)

    def run(c, grad=False):
        with Solver(cfg, c2_3d=c ** 2) as s:
            s.set_forcing(1, 28)
            s.set_clock(0.62, 0)
            s.set_state(np.zeros(s.state_shape))
            s.set_receivers(loc)
            if grad:
                return s.misfit_gradient(nsteps, 5, np.zeros((nsteps, len(loc))))
            return s.record(nsteps)

    res = run(c0, grad=True)
    assert res["misfit"] > 0
    d = np.random.default_rng(5).standard_normal(c0.shape) * c0
    eps = 1e-6
    jp = 0.5 * (run(c0 + eps * d) ** 2).sum()
    jm = 0.5 * (run(c0 - eps * d) ** 2).sum()
    fd = (jp - jm) / (2 * eps)
    ad = float(np.vdot(res["grad_c"].ravel(), d.ravel()))
    assert abs(fd - ad) <= 1e-4 * abs(ad), (fd, ad)


def test_forcing_files_load_like_set_samples(cfg, tmp_path):
    from solar_b200 import outputs
    nt = 24
    S = samples(cfg, nt, 7)
    for z in range(6):
        outputs.write_forcing(str(tmp_path / "forcing" / f"forcing_cubesph.{z + 1}"), S[z].reshape(cfg.nx, cfg.nx, nt))
    with Solver(cfg) as a, Solver(cfg) as b:
        a.load_forcing(str(tmp_path), nt)
        for z in range(6):
            b.set_forcing_samples(z, S[z], nt)
        for s in (a, b):
            s.set_forcing(2, 0, 200)
            s.set_state(np.zeros(s.state_shape))
            s.rk4(12)
        np.testing.assert_array_equal(a.get_state(), b.get_state())
