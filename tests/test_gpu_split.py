"""Zones split across processes, on one GPU.

Each emulated rank is its own context owning partition(world)[rank] zones; the ranks are
stepped phase by phase from one host thread, with the edge lines of every phase packed by
the library, copied between the ranks' buffers and unpacked (no kernel waits on another).
The assembled owned zones must equal the single-context run bit for bit: the split path
runs the same kernels on the same inputs.  A one-rank NCCL process group also runs the
torch.distributed path (ZoneSplitSolver) end to end.
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


def test_step_phases_equal_rk4(cfg):
    q0 = initial_state(cfg)
    with Solver(cfg) as a, Solver(cfg) as b:
        a.set_state(q0)
        b.set_state(q0)
        a.rk4(2)
        for _ in range(2):
            for phase in range(6):
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
        assert s.lib.solar_gpu_step_phase(s._h, 6) == _lib.SOLAR_ERR_ARG
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
