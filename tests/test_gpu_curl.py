"""COMPUTE_CURL on the GPU against the FP64 oracle, through the C-ABI (FP64 operators:
1e-12 relative L2 per component, as the other operators; FP32: 1e-5)."""
import numpy as np
import pytest

from solar_b200 import configs
from solar_b200.solver import Solver
from tests import geometry as G

pytestmark = pytest.mark.gpu


def rel(a, b):
    return np.linalg.norm(a - b) / np.linalg.norm(b)


@pytest.fixture(scope="module")
def cfg():
    return configs.c2(nx=32, nr=32, nsteps=1)


def fields(o, cfg, kind):
    if kind == "random":
        rng = np.random.default_rng(5)
        return [rng.standard_normal(o.field_shape) for _ in range(3)]
    gr = o.grid(3)
    vxi, veta = G.rotation_field(cfg.nx, gr, axis=(0.3, -0.5, 0.8))
    return [vxi, veta, np.sin(3 * gr)[None, :, None, None] * np.ones(o.field_shape)]


@pytest.mark.parametrize("kind", ["smooth", "random"])
@pytest.mark.parametrize("fix", [False, True])
def test_curl_fp64(oracle_mod, cfg, kind, fix):
    o = oracle_mod.Oracle(cfg, fix_reversed_rotation=fix)
    a = fields(o, cfg, kind)
    want = o.curl(*a)
    with Solver(cfg, fix_reversed_rotation=fix) as s:
        got = s.curl(*a)
    for g, w in zip(got, want):
        assert rel(g, w) <= 1e-12, rel(g, w)


def test_curl_fp32(oracle_mod, cfg):
    o = oracle_mod.Oracle(cfg)
    a = fields(o, cfg, "smooth")
    want = o.curl(*a)
    with Solver(cfg, precision="fp32", nfields=4) as s:
        got = s.curl(*a)
    for g, w in zip(got, want):
        assert rel(g, w) <= 1e-5, rel(g, w)
