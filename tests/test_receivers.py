"""Receiver placement (Cartesian -> zone and fractional grid indices) and per-point
sound-speed fields, on the CPU."""
import numpy as np
import pytest

from solar_b200 import configs, receivers


@pytest.fixture(scope="module")
def cfg():
    return configs.c2(nx=16, nr=16, nsteps=1)


def test_grid_points_locate_to_their_indices(cfg):
    xyz = receivers.points(cfg)
    rng = np.random.default_rng(0)
    for _ in range(200):
        z = int(rng.integers(6))
        k = int(rng.integers(cfg.nr))
        j, i = (int(v) for v in rng.integers(1, cfg.nx - 1, 2))   # face edges are shared
        loc = receivers.locate(cfg, xyz[z, k, j, i])[0]
        np.testing.assert_allclose(loc, [z, i, j, k], atol=1e-9)


def test_points_between_planes_get_fractional_radius(cfg):
    gr = configs.normalise(cfg.model)[0]
    r = 0.5 * (gr[3] + gr[4])
    loc = receivers.locate(cfg, [[r, 0.0, 0.0]])[0]
    assert loc[0] == 0 and 3.0 < loc[3] < 4.0
    np.testing.assert_allclose(loc[1:3], (cfg.nx - 1) / 2, atol=1e-12)


def test_points_outside_the_shell_are_rejected(cfg):
    with pytest.raises(ValueError):
        receivers.locate(cfg, [[0.0, 0.0, 1.5]])


def test_sound_speed_background_and_anomaly(cfg):
    c0 = receivers.sound_speed(cfg)
    c2 = configs.normalise(cfg.model)[1]
    np.testing.assert_allclose(c0[3, :, 5, 7], np.sqrt(c2))
    xyz = receivers.points(cfg)
    centre = xyz[4, 8, 7, 7]
    c1 = receivers.sound_speed(cfg, [(tuple(centre), 0.05, 0.1)])
    np.testing.assert_allclose(c1[4, 8, 7, 7], c0[4, 8, 7, 7] * 1.1)
    far = np.linalg.norm(xyz - centre, axis=-1) > 0.6
    np.testing.assert_allclose(c1[far], c0[far], rtol=1e-15)
