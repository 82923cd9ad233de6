"""GPU parity against the FP64 oracle, through the C-ABI.

Tolerances (relative L2 per field, ||gpu - oracle|| / ||oracle||):
  * FP64 operators (gradient, divergence, COMPUTE_RHS, BC_RHS, SPONGE, FILTER_EXP): 1e-12
  * FP64 time stepping, 100 steps: 1e-11
  * FP32 time stepping against the FP64 oracle: 1e-5 (precision-path target)
"""
import numpy as np
import pytest

from solar_b200 import configs
from solar_b200.solver import Solver
from tests import geometry as G

pytestmark = pytest.mark.gpu

FIELDS = ("rho", "v_xi", "v_eta", "v_r", "p")


def rel_l2(a, b):
    nb = np.linalg.norm(b)
    return np.linalg.norm(a - b) / (nb if nb > 0 else 1.0)


def per_field(a, b, fields=range(5)):
    return {FIELDS[m]: rel_l2(a[:, m], b[:, m]) for m in fields}


@pytest.fixture(scope="module")
def c1_small():
    return configs.c1(nx=32, nr=32)


@pytest.fixture(scope="module")
def c2_small():
    return configs.c2(nx=32, nr=32, nsteps=100)


def random_state(shape, seed):
    rng = np.random.default_rng(seed)
    return rng.standard_normal(shape)


def smooth_state(o, seed):
    """A state whose five fields are sums of seeded Gaussian blobs (smooth, nonzero
    everywhere that matters)."""
    rng = np.random.default_rng(seed)
    q = np.zeros(o.state_shape)
    for m in range(5):
        for _ in range(3):
            d = rng.standard_normal(3)
            d = d / np.linalg.norm(d) * rng.uniform(0.6, 0.95)
            src = configs.Source(tuple(d), 0.08, rng.uniform(0.5, 1.5))
            g = o.initial_state([src])[:, 4]
            q[:, m] += g
    return q


# ---------------------------------------------------------------- operators, FP64
def test_state_roundtrip_fp64(oracle_mod, c1_small):
    with Solver(c1_small) as s:
        q = random_state(s.state_shape, 1)
        s.set_state(q)
        assert np.array_equal(s.get_state(), q)


@pytest.mark.parametrize("nfields", [4, 5])
def test_state_roundtrip_fp32(c1_small, nfields):
    """An FP32 context stores the FP64 state rounded to nearest float (rounded by host
    threads before the copy, as the device would round it); reading it back is exact.  Values span normal, large, subnormal
    and underflowing magnitudes; with 4 fields rho is not stored and reads back as zero."""
    rng = np.random.default_rng(5)
    with Solver(c1_small, precision="fp32", nfields=nfields) as s:
        q = random_state(s.state_shape, 2)
        flat = q.reshape(-1)
        flat[:64] = rng.standard_normal(64) * 1e-42          # float subnormals
        flat[64:128] = rng.standard_normal(64) * 1e-47       # below the float range
        flat[128:192] = rng.standard_normal(64) * 1e37
        want = q.astype(np.float32).astype(np.float64)
        if nfields == 4:
            want[:, 0] = 0.0
        for _ in range(2):                                   # the second call reuses the pinned blocks
            s.set_state(q)
            got = s.get_state()
            assert np.array_equal(got, want)


def test_gaussian_ic_matches_oracle(oracle_mod, c1_small):
    o = oracle_mod.Oracle(c1_small)
    with Solver(c1_small) as s:
        s.init_sources()
        assert rel_l2(s.get_state()[:, 4], o.initial_state()[:, 4]) < 1e-12


@pytest.mark.parametrize("cfgname", ["c1_small", "c2_small"])
def test_gradient_and_divergence_fp64(oracle_mod, cfgname, request):
    cfg = request.getfixturevalue(cfgname)
    o = oracle_mod.Oracle(cfg)
    q = smooth_state(o, 2)
    with Solver(cfg) as s:
        g_gpu = s.gradient(q[:, 4])
        g_ref = o.gradient(q[:, 4])
        for a, b in zip(g_gpu, g_ref):
            assert rel_l2(a, b) < 1e-12
        d_gpu = s.divergence(q[:, 1], q[:, 2], q[:, 3])
        d_ref = o.divergence(q[:, 1], q[:, 2], q[:, 3])
        assert rel_l2(d_gpu, d_ref) < 1e-12


def test_divergence_fixed_rotation_option(oracle_mod, c1_small):
    o = oracle_mod.Oracle(c1_small, fix_reversed_rotation=True)
    vxi, veta = G.rotation_field(c1_small.nx, o.grid(3))
    vr = np.zeros_like(vxi)
    with Solver(c1_small, fix_reversed_rotation=True) as s:
        d = s.divergence(vxi, veta, vr)
    assert rel_l2(d, o.divergence(vxi, veta, vr)) < 1e-12 or np.abs(d - o.divergence(vxi, veta, vr)).max() < 1e-12
    assert max(G.edge_maxima(d).values()) < 1e-4


@pytest.mark.parametrize("cfgname", ["c1_small", "c2_small"])
def test_compute_rhs_bc_sponge_fp64(oracle_mod, cfgname, request):
    cfg = request.getfixturevalue(cfgname)
    o = oracle_mod.Oracle(cfg)
    q = smooth_state(o, 3)
    with Solver(cfg) as s:
        rhs = s.compute_rhs(q)
        ref = o.compute_rhs(q)
        for name, e in per_field(rhs, ref).items():
            assert e < 1e-12, (name, e)
        bc = s.bc_rhs(ref)
        assert np.array_equal(bc, o.bc_rhs(ref))
        sp = s.sponge(q, ref)
        assert np.abs(sp - o.sponge(q, ref)).max() <= 1e-14 * np.abs(ref).max()


@pytest.mark.parametrize("cfgname", ["c1_small", "c2_small"])
def test_filter_exp_fp64(oracle_mod, cfgname, request):
    cfg = request.getfixturevalue(cfgname)
    o = oracle_mod.Oracle(cfg)
    q = smooth_state(o, 4)
    with Solver(cfg) as s:
        qf = s.filter_exp(q)
    ref = o.filter_exp(q)
    for name, e in per_field(qf, ref).items():
        assert e < 1e-12, (name, e)
    assert np.all(qf[:, :, :5] == 0) and np.all(qf[:, :, -5:] == 0)


def test_filter_exp_random_fields_fp64(oracle_mod, c1_small):
    """Rough input: every halo value matters at full weight."""
    o = oracle_mod.Oracle(c1_small)
    q = random_state(o.state_shape, 5)
    with Solver(c1_small) as s:
        qf = s.filter_exp(q)
        rhs = s.compute_rhs(q)
    for name, e in per_field(qf, o.filter_exp(q)).items():
        assert e < 1e-12, (name, e)
    for name, e in per_field(rhs, o.compute_rhs(q)).items():
        assert e < 1e-12, (name, e)


def test_filter_exp_radial_chunks_fp64(oracle_mod):
    """6 x 96^2 x 44 has 540 (tile, field, face) filter columns: more than the resident
    filter CTAs of a 148-SM B200, so the columns of the last wave are filtered in radial
    chunks that each re-read 5 planes on either side.  Random input makes every plane of a
    chunk's halo count at full weight."""
    cfg = configs.c1(nx=96, nr=44)
    o = oracle_mod.Oracle(cfg)
    q = random_state(o.state_shape, 6)
    with Solver(cfg) as s:
        qf = s.filter_exp(q)
    for name, e in per_field(qf, o.filter_exp(q)).items():
        assert e < 1e-12, (name, e)
    assert np.all(qf[:, :, :5] == 0) and np.all(qf[:, :, -5:] == 0)


@pytest.fixture(scope="module")
def c2_long_edges():
    """6 x 144^2 x 24: the edge kernel cuts every 144-point edge into a 128-point segment and
    a ragged 16-point one (whose idle threads must stay out of the staged window)."""
    return configs.c2(nx=144, nr=24, nsteps=10)


def test_long_edges_fp64(oracle_mod, c2_long_edges):
    """COMPUTE_RHS (p and rotated-velocity halos) and FILTER_EXP (every field's halos) on
    random input with segmented edges: relative L2 <= 1e-12 per field."""
    o = oracle_mod.Oracle(c2_long_edges)
    q = random_state(o.state_shape, 7)
    with Solver(c2_long_edges) as s:
        rhs = s.compute_rhs(q)
        qf = s.filter_exp(q)
    for name, e in per_field(rhs, o.compute_rhs(q)).items():
        assert e < 1e-12, (name, e)
    for name, e in per_field(qf, o.filter_exp(q)).items():
        assert e < 1e-12, (name, e)


def test_long_edges_rk4_fp32(oracle_mod, c2_long_edges):
    """Ten FP32 steps (4 fields) with segmented edges against the FP64 oracle: <= 1e-5."""
    o = oracle_mod.Oracle(c2_long_edges)
    q0 = o.initial_state()
    ref = o.rk4(q0, 10)
    with Solver(c2_long_edges, precision="fp32", nfields=4) as s:
        s.set_state(q0)
        s.rk4(10)
        q = s.get_state()
    for name, e in per_field(q, ref, fields=(1, 2, 3, 4)).items():
        assert e < 1e-5, (name, e)


# ---------------------------------------------------------------- time stepping
def test_rk4_c1_100_steps_fp64(oracle_mod, c1_small):
    """Config 1 (6 x 32^3, 100 steps): per-field relative L2 <= 1e-11."""
    o = oracle_mod.Oracle(c1_small)
    q0 = o.initial_state()
    ref = o.rk4(q0, 100)
    with Solver(c1_small) as s:
        s.set_state(q0)
        s.rk4(100)
        q = s.get_state()
        assert abs(s.norm(4) - o.norm(ref, 4)) <= 1e-11 * o.norm(ref, 4)
    for name, e in per_field(q, ref).items():
        assert e < 1e-11, (name, e)


def test_rk4_stratified_fp64_and_fp32(oracle_mod, c2_small):
    """Stratified shell at 6 x 32^3, 100 steps: FP64 <= 1e-11; FP32 (4 fields) <= 1e-5."""
    o = oracle_mod.Oracle(c2_small)
    q0 = o.initial_state()
    ref = o.rk4(q0, 100)
    with Solver(c2_small) as s:
        s.set_state(q0)
        s.rk4(100)
        for name, e in per_field(s.get_state(), ref).items():
            assert e < 1e-11, (name, e)
    with Solver(c2_small, precision="fp32", nfields=4) as s:
        s.set_state(q0)
        s.rk4(100)
        q = s.get_state()
        assert np.all(q[:, 0] == 0)
        for name, e in per_field(q, ref, fields=(1, 2, 3, 4)).items():
            assert e < 1e-5, (name, e)


def test_rk4_fp32_five_fields_c1(oracle_mod, c1_small):
    o = oracle_mod.Oracle(c1_small)
    q0 = o.initial_state()
    ref = o.rk4(q0, 100)
    with Solver(c1_small, precision="fp32") as s:
        s.set_state(q0)
        s.rk4(100)
        for name, e in per_field(s.get_state(), ref, fields=(1, 2, 3, 4)).items():
            assert e < 1e-5, (name, e)


def test_graph_and_direct_launch_agree(c1_small):
    with Solver(c1_small) as s:
        s.init_sources()
        q0 = s.get_state()
        s.rk4(3)
        a = s.get_state()
        s.set_state(q0)
        s.time_rk4(3, per_kernel=True)
        b = s.get_state()
    assert np.array_equal(a, b)


def test_batched_uneven_runs_match_single_runs(c1_small):
    steps = [3, 7, 0, 5]
    srcs = [configs.Source((0.0, 0.0, 0.75), 0.05, 1.0), configs.Source((0.75, 0.0, 0.0), 0.04, 0.5),
            configs.Source((0.0, -0.7, 0.2), 0.06, 2.0), configs.Source((0.3, 0.3, -0.6), 0.05, 1.0)]
    with Solver(c1_small, nruns=4) as b:
        for r, src in enumerate(srcs):
            b.init_sources([src], run=r)
        b.rk4_runs(steps)
        got = [b.get_state(r) for r in range(4)]
    with Solver(c1_small) as s:
        for r, src in enumerate(srcs):
            s.init_sources([src])
            s.rk4(steps[r])
            assert np.array_equal(s.get_state(), got[r]), r


def test_batched_runs_twice_reorders_live_runs(c1_small):
    """Two batched calls with different step counts: the second reorders the runs, reuses
    the graphs kept per live-run count, and still matches each run advanced on its own."""
    srcs = [configs.Source((0.0, 0.0, 0.75), 0.05, 1.0), configs.Source((0.75, 0.0, 0.0), 0.04, 0.5),
            configs.Source((0.0, -0.7, 0.2), 0.06, 2.0)]
    first, second = [2, 5, 3], [4, 1, 4]
    with Solver(c1_small, nruns=3) as b:
        for r, src in enumerate(srcs):
            b.init_sources([src], run=r)
        b.rk4_runs(first)
        b.rk4_runs(second)
        got = [b.get_state(r) for r in range(3)]
    with Solver(c1_small) as s:
        for r, src in enumerate(srcs):
            s.init_sources([src])
            s.rk4(first[r] + second[r])
            assert np.array_equal(s.get_state(), got[r]), r


def test_norm_and_diag(oracle_mod, c1_small):
    o = oracle_mod.Oracle(c1_small)
    q = smooth_state(o, 6)
    with Solver(c1_small) as s:
        s.set_state(q)
        for m in range(1, 6):
            assert abs(s.norm(m) - o.norm(q, m)) <= 1e-12 * o.norm(q, m)
        d = s.diag()
        assert d["energy"] > 0 and not d["nonfinite"]
        assert d["max_abs_p"] == pytest.approx(np.abs(q[:, 4]).max(), rel=1e-15)


def test_bad_run_index_raises(c1_small):
    from solar_b200._lib import SolarError
    with Solver(c1_small) as s:
        with pytest.raises(SolarError):
            s.get_state(run=3)


def test_unsupported_tile_is_rejected(c1_small):
    """A stage tile the library does not build, or one that does not divide nx, is refused at
    set-up with SOLAR_ERR_ARG and a message naming it; a valid context still opens after it."""
    from solar_b200._lib import SolarError
    for tile in ((48, 8, 0), (64, 8, 0)):          # unknown shape; 64 does not divide nx = 32
        with pytest.raises(SolarError, match="unsupported stage tile"):
            Solver(c1_small, tile=tile)
    with Solver(c1_small, tile=(16, 16, 0)) as s:
        s.init_sources()
        assert s.norm(5) > 0
