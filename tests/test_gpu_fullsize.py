"""Parity at the workloads' full sizes.

Against the oracle at the benchmark's 6 x 128^3 (ten full RK4 steps from a state with
Gaussian blobs on every cube corner and edge, so every inter-zone edge and both radial
ends take part): the FP64 path <= 1e-11 relative L2 per field, the FP32 path <= 1e-5 per
field; the per-field maximum errors are printed (run with -s).

Through properties that do not need the oracle (too slow for more steps at these sizes):

* linearity of the FP64 step at 6 x 128^3: STEP(a q1 + b q2) = a STEP(q1) + b STEP(q2), to
  rounding (1e-12 relative);
* the FP32 path against the FP64 path at 6 x 128^3 after 50 steps: <= 1e-5 relative L2
  per field (the precision-path target);
* the adjoint at 6 x 96^3: <STEP^2 q, lam> = <q, (STEP^T)^2 lam> to 1e-11 of |STEP^2 q| |lam|;
* batched uneven runs at 64 x 6 x 64^3 equal the same runs stepped alone, bit for bit;
* the zones split over 3 emulated processes at 6 x 128^3 equal the one-context run, bit for bit.
"""
import json
import os

import numpy as np
import pytest

from solar_b200 import _lib, configs
from solar_b200 import distributed as D
from solar_b200.solver import Solver

pytestmark = pytest.mark.gpu


def rel(a, b):
    return np.linalg.norm(a - b) / np.linalg.norm(b)


def blobs(cfg, seed, n=4):
    """A smooth random state: Gaussian pulses in p and the velocity components."""
    rng = np.random.default_rng(seed)
    q = np.zeros((6, 5, cfg.nr, cfg.nx, cfg.nx))
    with Solver(cfg) as s:
        for f in (1, 2, 3, 4):
            s.set_state(np.zeros_like(q))
            for _ in range(n):
                d = configs.unit_vectors(rng, 1)[0] * rng.uniform(0.75, 0.95)
                s.add_gaussian(configs.Source(tuple(d), 0.04, rng.uniform(0.5, 1.5)))
            q[:, f] = s.get_state()[:, 4]
    return q


@pytest.fixture(scope="module")
def c2():
    return configs.c2()


def edge_and_corner_blobs(o, cfg):
    """Five fields of Gaussian blobs (width 0.08): v_xi and v_eta on the 8 cube corners,
    rho, v_r and p on the 12 cube-edge midpoints, at seeded radii inside the shell."""
    rng = np.random.default_rng(12)
    corners = np.array([(x, y, z) for x in (-1, 1) for y in (-1, 1) for z in (-1, 1)], float)
    mids = np.array([v for i in range(3) for a in (-1, 1) for b in (-1, 1)
                     for v in [np.insert(np.array([a, b], float), i, 0.0)]])
    r0, r1 = float(cfg.model[0, 0]), float(cfg.model[-1, 0])
    q = np.zeros(o.state_shape)
    for f, dirs in ((0, mids), (1, corners), (2, corners), (3, mids), (4, mids)):
        srcs = []
        for d in dirs:
            d = d / np.linalg.norm(d) * rng.uniform(r0 + 0.25 * (r1 - r0), r0 + 0.8 * (r1 - r0))
            srcs.append(configs.Source(tuple(d), 0.08, rng.uniform(0.5, 1.5)))
        q[:, f] = o.initial_state(srcs)[:, 4]
    return q


ORACLE_STEPS = 10


def test_fp64_and_fp32_match_the_oracle_at_c2(c2, oracle_mod):
    oracle_mod.set_threads(os.cpu_count() or 1)
    o = oracle_mod.Oracle(c2)
    q0 = edge_and_corner_blobs(o, c2)
    ref = o.rk4(q0, ORACLE_STEPS)
    got = {}
    for prec, nf in (("fp64", 5), ("fp32", 4)):
        with Solver(c2, precision=prec, nfields=nf) as s:
            s.set_state(q0)
            s.rk4(ORACLE_STEPS)
            got[prec] = s.get_state()
    names = ("rho", "v_xi", "v_eta", "v_r", "p")
    report = {}
    for prec, fields in (("fp64", range(5)), ("fp32", range(1, 5))):
        for f in fields:
            d = got[prec][:, f] - ref[:, f]
            report[f"{prec}.{names[f]}"] = {"rel_l2": rel(got[prec][:, f], ref[:, f]),
                                           "max_abs_over_max_ref": float(np.abs(d).max() / np.abs(ref[:, f]).max())}
    print("c2 6x128^3, %d steps vs the oracle: %s" % (ORACLE_STEPS, json.dumps(report)))
    for f in range(5):
        assert report[f"fp64.{names[f]}"]["rel_l2"] <= 1e-11, (names[f], report)
    for f in range(1, 5):
        assert report[f"fp32.{names[f]}"]["rel_l2"] <= 1e-5, (names[f], report)


def test_step_is_linear_at_c2(c2):
    q1, q2 = blobs(c2, 1), blobs(c2, 2)
    a, b = 0.7, -1.3
    with Solver(c2) as s:
        out = []
        for q in (q1, q2, a * q1 + b * q2):
            s.set_state(q)
            s.rk4(3)
            out.append(s.get_state())
    lin = a * out[0] + b * out[1]
    for f in range(1, 5):
        assert rel(out[2][:, f], lin[:, f]) <= 1e-12, f


def test_fp32_tracks_fp64_at_c2(c2):
    q = blobs(c2, 3)
    res = {}
    for prec, nf in (("fp64", 5), ("fp32", 4)):
        with Solver(c2, precision=prec, nfields=nf) as s:
            s.set_state(q)
            s.rk4(50)
            res[prec] = s.get_state()
    for f in (1, 2, 3, 4):
        assert rel(res["fp32"][:, f], res["fp64"][:, f]) <= 1e-5, f


def test_adjoint_dot_product_at_c4():
    cfg = configs.c4()
    rng = np.random.default_rng(4)
    q = rng.standard_normal((6, 5, cfg.nr, cfg.nx, cfg.nx))
    lam = rng.standard_normal(q.shape)
    with Solver(cfg) as s:
        s.set_state(q)
        s.rk4(2)
        Sq = s.get_state()
        STlam = s.rk4_adjoint(2, lam)
    a, b = float(np.vdot(Sq, lam)), float(np.vdot(q, STlam))
    assert abs(a - b) <= 1e-11 * np.linalg.norm(Sq) * np.linalg.norm(lam)


def test_batched_runs_equal_single_runs_at_c3():
    cfg = configs.c3()
    R = len(cfg.runs)
    steps = [5 + (r * 7) % 13 for r in range(R)]          # uneven, 5..17
    picks = (0, 21, R - 1)
    with Solver(cfg, precision="fp32", nfields=4, nruns=R) as s:
        for r in range(R):
            s.init_sources(cfg.runs[r], run=r)
        s.rk4_runs(steps)
        got = {r: s.get_state(run=r) for r in picks}
    for r in picks:
        with Solver(cfg, precision="fp32", nfields=4) as s1:
            s1.init_sources(cfg.runs[r])
            s1.rk4(steps[r])
            np.testing.assert_array_equal(got[r], s1.get_state())


def test_zone_split_equals_single_context_at_c2(c2):
    import torch
    q0 = blobs(c2, 5, n=2)
    world = 3
    parts = D.partition(world)
    routes = D.route_table()
    ranks = []
    try:
        for r in range(world):
            s = Solver(c2, precision="fp32", nfields=4)
            s.set_state(q0)
            _lib.check(s.lib.solar_gpu_set_owned_zones(s._h, *parts[r]))
            ex = D.LineExchange(D.exchange_plan(routes, parts, r), D._LibPacker(s), None,
                                lambda n: torch.zeros(n, dtype=torch.float32, device="cuda"))
            ranks.append((s, ex))
        for _ in range(3):
            for phase in range(6):
                for s, ex in ranks:
                    ex.pack(phase)
                for s, _ in ranks:
                    s.synchronize()
                for r, (s, ex) in enumerate(ranks):
                    for peer, buf in ex.buffers(phase)[1].items():
                        buf.copy_(ranks[peer][1].buffers(phase)[0][r])
                torch.cuda.synchronize()
                for s, ex in ranks:
                    ex.unpack(phase)
                    _lib.check(s.lib.solar_gpu_step_phase(s._h, phase))
        got = np.zeros_like(q0)
        for r, (s, _) in enumerate(ranks):
            z0, nz = parts[r]
            got[z0:z0 + nz] = s.get_state()[z0:z0 + nz]
    finally:
        for s, _ in ranks:
            s.close()
    with Solver(c2, precision="fp32", nfields=4) as s:
        s.set_state(q0)
        s.rk4(3)
        np.testing.assert_array_equal(got, s.get_state())
