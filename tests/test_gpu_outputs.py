"""The reference's output files written from a GPU context, read back with independent
readers and compared with the state (FP64 exact for binary files, ES13.5 for traces)."""
import numpy as np
import pytest

from solar_b200 import configs, outputs
from solar_b200.solver import Solver

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def cfg():
    return configs.c2(nx=32, nr=32, nsteps=5)


def stepped(s, n=4):
    s.init_sources()
    s.rk4(n)
    return s.get_state()


def test_restart_roundtrip_fp64(cfg, tmp_path):
    d = str(tmp_path)
    with Solver(cfg) as s:
        q = stepped(s)
        s.write_restart(d, 3, 0.75, 4)
    for z in range(6):
        qz, t, st = outputs.read_restart(f"{d}/Restart/restart.003.{z + 1}")
        np.testing.assert_array_equal(qz, q[z])
        assert (t, st) == (0.75, 4)
    with Solver(cfg) as r:
        assert r.read_restart(d, 3) == (0.75, 4)
        np.testing.assert_array_equal(r.get_state(), q)
        # continuing from the restart gives the same run
        r.rk4(2)
        with Solver(cfg) as s2:
            s2.set_state(q)
            s2.rk4(2)
            np.testing.assert_array_equal(r.get_state(), s2.get_state())


def test_restart_fp32_state(cfg, tmp_path):
    d = str(tmp_path)
    with Solver(cfg, precision="fp32", nfields=4) as s:
        q = stepped(s)
        s.write_restart(d, 0, 0.0, 0)
    with Solver(cfg, precision="fp32", nfields=4) as r:
        r.read_restart(d, 0)
        np.testing.assert_array_equal(r.get_state(), q)


def test_restart_size_mismatch_is_an_error(cfg, tmp_path):
    d = str(tmp_path)
    with Solver(cfg) as s:
        s.write_restart(d, 1, 0.0, 0)
    with Solver(configs.c2(nx=32, nr=48, nsteps=1)) as r:
        with pytest.raises(Exception):
            r.read_restart(d, 1)


def test_visual_grid_and_trace(cfg, tmp_path):
    d = str(tmp_path)
    gr = configs.normalise(cfg.model)[0]
    obs = 1.0 + 200e5 / configs.RSUN
    temp, o_rad = 1.0, None                      # ic_acoustic_wave.f90:124-132, 0-based here
    for k in range(cfg.nr):
        if abs(gr[k] - obs) <= temp:
            temp, o_rad = abs(gr[k] - obs), k
    with Solver(cfg) as s:
        q = stepped(s)
        assert s.output_plane() == o_rad
        s.write_visual(d, 12)
        s.write_grid(d)
        s.write_radial_trace(d)
        s.rk4(1)
        q2 = s.get_state()
        s.write_radial_trace(d)
    for z in range(6):
        np.testing.assert_array_equal(outputs.read_visual(f"{d}/Visual/012/vis_{z}", cfg.nx), q[z][:, o_rad])
        assert outputs.read_grid(f"{d}/Visual/grid/grid_{z}") == [0, cfg.nx - 1, 0, cfg.nx - 1, 0, cfg.nr - 1, z + 1]
        tr = outputs.read_trace(f"{d}/trace_{z + 1}", cfg.nr)
        assert tr.shape == (2, 5, cfg.nr)
        for rec, qq in zip(tr, (q, q2)):
            want = qq[z][:, :, 0, 0]
            np.testing.assert_allclose(rec, want, rtol=6e-6, atol=1e-300)
