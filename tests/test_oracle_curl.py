"""The oracle's COMPUTE_CURL (grad.f90:140-255) with its halo transform
(transform.f90:279-498) against analytic curls, on the CPU.

With the receiver-frame rotation evaluated at the receiver's edge index
(fix_reversed_rotation) the curl of a gradient vanishes and a solid-body rotation has
curl_r = 2 w.e_r, to truncation error.  With the reference's own arithmetic the same
O(1) defect as in the divergence appears, exactly on the eight receiver edges whose strip
the receiver reverses."""
import numpy as np
import pytest

from solar_b200 import configs
from tests import geometry as G


@pytest.fixture(scope="module")
def cfg():
    return configs.c1(nx=32, nr=32)


def radial_z(o, cfg):
    """phi = r^2 z: a smooth scalar whose gradient is curl-free."""
    _, X, Y = G.grid_xy(cfg.nx)
    gr = o.grid(3)
    phi = np.zeros(o.field_shape)
    for z in range(6):
        phi[z] = gr[:, None, None] ** 2 * G.cube_point(z + 1, X, Y)[2][None]
    return phi


def test_curl_of_gradient_vanishes(oracle_mod, cfg):
    o = oracle_mod.Oracle(cfg, fix_reversed_rotation=True)
    cx, ce, cr = o.curl(*o.gradient(radial_z(o, cfg)))
    # xi/eta: exact cancellation of the same stencils; r: truncation error of the
    # cross derivatives near the edges
    assert np.abs(cx[:, 4:-4]).max() < 1e-10
    assert np.abs(ce[:, 4:-4]).max() < 1e-10
    assert np.abs(cr[:, 4:-4]).max() < 1e-4


def test_rotation_curl_and_reference_defect(oracle_mod, cfg):
    n = cfg.nx
    fixed = oracle_mod.Oracle(cfg, fix_reversed_rotation=True)
    ref = oracle_mod.Oracle(cfg)
    gr = ref.grid(3)
    th = ref.grid(0).reshape(6, n, n)
    vxi, veta = G.rotation_field(n, gr, axis=(0.0, 0.0, 1.0))
    want = 2.0 * np.cos(th)[:, None]
    _, _, cr_fixed = fixed.curl(vxi, veta, np.zeros_like(vxi))
    assert np.abs(cr_fixed - want)[:, 4:-4].max() < 1e-5
    _, _, cr = ref.curl(vxi, veta, np.zeros_like(vxi))
    edges = G.edge_maxima(cr - want)
    for key, v in edges.items():
        if key in G.REVERSED_RECEIVER_EDGES:
            assert v > 0.1, key
        else:
            assert v < 1e-5, key
