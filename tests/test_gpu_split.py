"""The sphere split across processes, on one GPU.

Each emulated rank is its own context owning a zone range (and, for 4 and 8 ranks, a radial
slab: 2 zone groups x 2 or 4 slabs); the ranks are stepped phase by phase from one host
thread, with the edge lines and boundary planes of every phase packed by the library,
copied between the ranks' buffers and unpacked (no kernel waits on another).  The assembled
owned parts must equal the single-context run bit for bit: the split path runs the same
kernels on the same inputs.  A one-rank NCCL process group also runs the torch.distributed
path (ZoneSplitSolver) end to end.
"""
import os
import socket

import numpy as np
import pytest

from solar_b200 import _lib, configs
from solar_b200 import distributed as D
from solar_b200.solver import Solver

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def cfg():
    return configs.c2(nx=32, nr=32, nsteps=5)


def initial_state(cfg):
    with Solver(cfg) as s:
        s.init_sources()
        return s.get_state()


def emulate(cfg, world, nsteps, q0, precision, nfields):
    import torch
    parts = D.partition(world)
    routes = D.route_table()
    dtype = torch.float32 if precision == "fp32" else torch.float64
    ranks = []
    for r in range(world):
        s = Solver(cfg, precision=precision, nfields=nfields)
        s.set_state(q0)
        _lib.check(s.lib.solar_gpu_set_owned_zones(s._h, *parts[r]))
        ex = D.LineExchange(D.exchange_plan(routes, parts, r), D._LibPacker(s), None,
                            lambda n: torch.zeros(n, dtype=dtype, device="cuda"))
        ranks.append((s, ex))
    try:
        for _ in range(nsteps):
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
        q = np.zeros_like(q0)
        norm_parts = 0.0
        for r, (s, _) in enumerate(ranks):
            z0, nz = parts[r]
            q[z0:z0 + nz] = s.get_state()[z0:z0 + nz]
            out = (__import__("ctypes").c_double * 5)()
            _lib.check(s.lib.solar_gpu_reduce_owned(s._h, 0, 4, out))
            norm_parts += out[0]
        return q, norm_parts
    finally:
        for s, _ in ranks:
            s.close()


@pytest.mark.parametrize("world", [2, 3, 6])
@pytest.mark.parametrize("precision,nfields", [("fp64", 5), ("fp32", 4)])
def test_split_run_equals_single_context(cfg, world, precision, nfields):
    q0 = initial_state(cfg)
    nsteps = 5
    with Solver(cfg, precision=precision, nfields=nfields) as s:
        s.set_state(q0)
        s.rk4(nsteps)
        want = s.get_state()
        want_norm = s.norm(4)
    got, sumsq = emulate(cfg, world, nsteps, q0, precision, nfields)
    np.testing.assert_array_equal(got, want)
    norm = (sumsq / (cfg.nx * cfg.nx * cfg.nr) * 6.0) ** 0.5
    assert abs(norm - want_norm) <= 1e-12 * want_norm


def emulate_slabs(cfg, world, nsteps, q0, precision, nfields, parts=False, tile=None):
    """World ranks laid out as D.layout(world) zone groups x radial slabs, one context each.
    With ``parts`` every stage runs as solar_gpu_step_phase_part: part 0 (interior tiles) on
    every rank before any line of the phase is delivered, part 1 after."""
    import ctypes

    import torch
    ngroups, nsl = D.layout(world)
    dtype = torch.float32 if precision == "fp32" else torch.float64
    alloc = lambda n: torch.zeros(n, dtype=dtype, device="cuda")
    ranks = []
    try:
        for r in range(world):
            zg, sl = divmod(r, nsl)
            z0, nz = D.partition(ngroups)[zg]
            k0, k1 = D.slabs(cfg.nr, nsl)[sl]
            s = Solver(cfg, precision=precision, nfields=nfields, tile=tile)
            s.set_state(q0)
            _lib.check(s.lib.solar_gpu_set_owned_zones(s._h, z0, nz))
            _lib.check(s.lib.solar_gpu_set_owned_planes(s._h, k0, k1))
            plan, below, above = D.slab_plan(world, r)
            lx = D.LineExchange(plan, D._LibPacker(s), None, alloc)
            px = D.PlaneExchange(below, above, D._LibPlanePacker(s), None, alloc)
            ranks.append((s, lx, px, (z0, nz, k0, k1)))

        def lines(phase, between=None):
            for s, lx, _, _ in ranks:
                lx.pack(phase)
            if between is not None:
                between()
            for s, _, _, _ in ranks:
                s.synchronize()
            for r, (_, lx, _, _) in enumerate(ranks):
                for peer, buf in lx.buffers(phase)[1].items():
                    buf.copy_(ranks[peer][1].buffers(phase)[0][r])
            torch.cuda.synchronize()
            for _, lx, _, _ in ranks:
                lx.unpack(phase)

        def planes(phase):
            for _, _, px, _ in ranks:
                px.pack(phase)
            for s, _, _, _ in ranks:
                s.synchronize()
            for r, (_, _, px, _) in enumerate(ranks):
                for side, buf in px.buffers(phase)[1].items():
                    peer = px.peers[side]
                    buf.copy_(ranks[peer][2].buffers(phase)[0][1 - side])   # the peer's send toward me
            torch.cuda.synchronize()
            for _, _, px, _ in ranks:
                px.unpack(phase)

        def step(phase):
            for s, _, _, _ in ranks:
                _lib.check(s.lib.solar_gpu_step_phase(s._h, phase))

        def part(phase, p):
            for s, _, _, _ in ranks:
                _lib.check(s.lib.solar_gpu_step_phase_part(s._h, phase, p))

        for _ in range(nsteps):
            for phase in range(5):
                if parts:
                    planes(phase)
                    lines(phase, between=lambda: part(phase, 0))
                    part(phase, 1)
                    continue
                lines(phase)
                planes(phase)
                step(phase)
            lines(5)
            step(6)
            planes(5)
            step(7)
        q = np.zeros_like(q0)
        sumsq = 0.0
        for s, _, _, (z0, nz, k0, k1) in ranks:
            q[z0:z0 + nz, :, k0:k1] = s.get_state()[z0:z0 + nz, :, k0:k1]
            out = (ctypes.c_double * 5)()
            _lib.check(s.lib.solar_gpu_reduce_owned(s._h, 0, 4, out))
            sumsq += out[0]
        return q, sumsq
    finally:
        for s, _, _, _ in ranks:
            s.close()


@pytest.mark.parametrize("world", [4, 8])
@pytest.mark.parametrize("precision,nfields", [("fp64", 5), ("fp32", 4)])
def test_zone_and_slab_split_equals_single_context(cfg, world, precision, nfields):
    q0 = initial_state(cfg)
    nsteps = 5
    with Solver(cfg, precision=precision, nfields=nfields) as s:
        s.set_state(q0)
        s.rk4(nsteps)
        want = s.get_state()
        want_norm = s.norm(4)
    got, sumsq = emulate_slabs(cfg, world, nsteps, q0, precision, nfields)
    np.testing.assert_array_equal(got, want)
    norm = (sumsq / (cfg.nx * cfg.nx * cfg.nr) * 6.0) ** 0.5
    assert abs(norm - want_norm) <= 1e-12 * want_norm


@pytest.fixture(scope="module")
def cfg64():
    return configs.c2(nx=64, nr=32, nsteps=3)


TILE16 = (16, 16, 0)          # 4 x 4 stage tiles per face: 4 interior, 12 along the edges


@pytest.mark.parametrize("tile", [TILE16, None], ids=["16x16", "default"])
@pytest.mark.parametrize("precision,nfields", [("fp64", 5), ("fp32", 4)])
def test_phase_parts_equal_rk4(cfg64, tile, precision, nfields):
    """Parts 0 and 1 of each stage (interior tiles, then edge kernel + edge tiles) give the
    RK4 step bit for bit; with the default 64 x 8 tile a 64^2 face has no interior tile."""
    q0 = initial_state(cfg64)
    with Solver(cfg64, precision=precision, nfields=nfields, tile=tile) as a, \
            Solver(cfg64, precision=precision, nfields=nfields, tile=tile) as b:
        a.set_state(q0)
        b.set_state(q0)
        a.rk4(2)
        for _ in range(2):
            for phase in range(5):
                _lib.check(b.lib.solar_gpu_step_phase_part(b._h, phase, 0))
                _lib.check(b.lib.solar_gpu_step_phase_part(b._h, phase, 1))
            _lib.check(b.lib.solar_gpu_step_phase(b._h, 5))
        b.synchronize()
        np.testing.assert_array_equal(a.get_state(), b.get_state())


@pytest.mark.parametrize("world", [2, 4])
@pytest.mark.parametrize("precision,nfields", [("fp64", 5), ("fp32", 4)])
def test_overlapped_split_equals_single_context(cfg64, world, precision, nfields):
    """Every rank runs its interior tiles before the phase's lines are delivered."""
    q0 = initial_state(cfg64)
    with Solver(cfg64, precision=precision, nfields=nfields, tile=TILE16) as s:
        s.set_state(q0)
        s.rk4(3)
        want = s.get_state()
    got, _ = emulate_slabs(cfg64, world, 3, q0, precision, nfields, parts=True, tile=TILE16)
    np.testing.assert_array_equal(got, want)


def test_phase_part_arguments(cfg):
    with Solver(cfg) as s:
        assert s.lib.solar_gpu_step_phase_part(s._h, 5, 0) == _lib.SOLAR_ERR_ARG     # the filter phase
        assert s.lib.solar_gpu_step_phase_part(s._h, 0, 2) == _lib.SOLAR_ERR_ARG
        assert s.lib.solar_gpu_step_phase_part(s._h, -1, 0) == _lib.SOLAR_ERR_ARG


def test_plane_exchange_arguments(cfg):
    import ctypes

    import torch
    with Solver(cfg) as s:
        assert s.lib.solar_gpu_set_owned_planes(s._h, 0, 4) == _lib.SOLAR_ERR_ARG      # fewer than 5 planes
        assert s.lib.solar_gpu_set_owned_planes(s._h, 10, cfg.nr + 1) == _lib.SOLAR_ERR_ARG
        _lib.check(s.lib.solar_gpu_set_owned_planes(s._h, 0, 16))
        n = s.lib.solar_gpu_planes_size(s._h, 0)
        assert n == 6 * 2 * 3 * (cfg.nx + 16) * (cfg.nx + 6)      # zones x {p, v_r} x 3 planes x padded plane
        assert s.lib.solar_gpu_planes_size(s._h, 5) == 6 * 5 * 5 * (cfg.nx + 16) * (cfg.nx + 6)
        buf = torch.zeros(n, dtype=torch.float64, device="cuda")
        p = ctypes.c_void_p(buf.data_ptr())
        assert s.lib.solar_gpu_pack_planes(s._h, 0, 0, p) == _lib.SOLAR_ERR_ARG     # no slab below plane 0
        _lib.check(s.lib.solar_gpu_pack_planes(s._h, 0, 1, p))


def test_step_phases_equal_rk4(cfg):
    q0 = initial_state(cfg)
    with Solver(cfg) as a, Solver(cfg) as b:
        a.set_state(q0)
        b.set_state(q0)
        a.rk4(2)
        for _ in range(2):
            for phase in (0, 1, 2, 3, 4, 6, 7):             # the filter phase in its two halves
                _lib.check(b.lib.solar_gpu_step_phase(b._h, phase))
        b.synchronize()
        np.testing.assert_array_equal(a.get_state(), b.get_state())


def test_line_pack_roundtrip_and_errors(cfg):
    import ctypes
    import torch
    q0 = np.random.default_rng(3).standard_normal((6, 5, cfg.nr, cfg.nx, cfg.nx))
    with Solver(cfg) as s, Solver(cfg) as t:
        s.set_state(q0)
        pairs = [(z, e) for z in range(6) for e in range(4)]
        per = s.lib.solar_gpu_lines_size(s._h, 0)          # phase 0 reads the state buffer
        assert per == 3 * cfg.nx * cfg.nr * 3
        assert s.lib.solar_gpu_lines_size(s._h, 5) == 3 * cfg.nx * cfg.nr * 5
        buf = torch.zeros(per * 24, dtype=torch.float64, device="cuda")
        D._LibPacker(s).pack(0, pairs, buf)
        s.synchronize()
        lines = buf.cpu().numpy().reshape(24, 3, cfg.nr, 3, cfg.nx)
        fields = [4, 1, 2]                                   # p, v_xi, v_eta
        n = cfg.nx
        for q, (z, e) in enumerate(pairs):   # rows 1..3 / n-2..n-4, columns likewise
            for l in range(3):
                want = {0: q0[z, fields, :, l + 1, :], 1: q0[z, fields, :, n - 2 - l, :],
                        2: q0[z, fields, :, :, l + 1], 3: q0[z, fields, :, :, n - 2 - l]}[e]
                np.testing.assert_array_equal(lines[q, :, :, l, :], want)
        # unpacking into a zeroed context writes exactly those lines
        D._LibPacker(t).unpack(0, pairs, buf)
        t.synchronize()
        back = t.get_state()
        mask = np.zeros(q0.shape, bool)
        sel = np.zeros(5, bool)
        sel[fields] = True
        for a, b in ((slice(1, 4), slice(None)), (slice(n - 4, n - 1), slice(None)),
                     (slice(None), slice(1, 4)), (slice(None), slice(n - 4, n - 1))):
            mask[:, sel, :, a, b] = True
        np.testing.assert_array_equal(back[mask], q0[mask])
        assert not back[~mask].any()
        bad = (ctypes.c_int * 2)(6, 0)
        assert s.lib.solar_gpu_pack_lines(s._h, 0, bad, 1, ctypes.c_void_p(buf.data_ptr())) == _lib.SOLAR_ERR_ARG
        assert s.lib.solar_gpu_step_phase(s._h, 8) == _lib.SOLAR_ERR_ARG
        assert s.lib.solar_gpu_set_owned_zones(s._h, 4, 3) == _lib.SOLAR_ERR_ARG


def test_zone_split_solver_single_rank_nccl(cfg):
    import torch.distributed as dist
    q0 = initial_state(cfg)
    with socket.socket() as sk:
        sk.bind(("127.0.0.1", 0))
        port = sk.getsockname()[1]
    dist.init_process_group("nccl", init_method=f"tcp://127.0.0.1:{port}", rank=0, world_size=1)
    try:
        zs = D.ZoneSplitSolver(cfg, precision="fp64", nfields=5)
        zs.set_state(q0)
        zs.rk4(3)
        got = zs.gather_state()
        got_norm = zs.norm(4)
        zs.close()
    finally:
        dist.destroy_process_group()
    with Solver(cfg) as s:
        s.set_state(q0)
        s.rk4(3)
        np.testing.assert_array_equal(got, s.get_state())
        assert abs(got_norm - s.norm(4)) <= 1e-12 * s.norm(4)
