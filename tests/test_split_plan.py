"""Zones split across processes: the exchange plan and its transport, on the CPU.

The plan decides which (zone, edge) source lines each rank sends to and receives from
each peer before every phase of a step.  These tests check it against the route table of
the library (the reference's halo routing, derivative.f90:8-323) and run the exchange over
the gloo backend with 2, 3 and 6 processes, with a packer that stores each line set as
numbers encoding (zone, edge, phase, slot, k, layer, t), so every received value can be
checked.  The GPU packing kernels and the split step itself are tested on the GPU
(tests/test_gpu_split.py) against the single-process run.
"""
import os
import socket

import numpy as np
import pytest

from solar_b200 import distributed as D


@pytest.fixture(scope="module")
def routes():
    return D.route_table()


def test_route_table_is_a_bijection(routes):
    src = {(int(routes[z, e, 0]), int(routes[z, e, 1])) for z in range(6) for e in range(4)}
    assert len(src) == 24
    assert all(routes[z, e, 0] != z for z in range(6) for e in range(4))


def test_partition():
    assert D.partition(1) == [(0, 6)]
    assert D.partition(2) == [(0, 3), (3, 3)]
    assert D.partition(3) == [(0, 2), (2, 2), (4, 2)]
    assert D.partition(6) == [(z, 1) for z in range(6)]
    for bad in (0, 4, 5, 7, 8):
        with pytest.raises(ValueError):
            D.partition(bad)


@pytest.mark.parametrize("world", [1, 2, 3, 6])
def test_plans_of_sender_and_receiver_agree(routes, world):
    parts = D.partition(world)
    own = D.owners(parts)
    plans = [D.exchange_plan(routes, parts, r) for r in range(world)]
    for r in range(world):
        sends, recvs = plans[r]
        assert r not in sends and r not in recvs
        for peer, pairs in sends.items():
            assert plans[peer][1][r] == pairs          # same pairs, same order
        # every ghost frame of an owned zone is fed: by the owner itself or by a receive
        need = {(int(routes[z, e, 0]), int(routes[z, e, 1])) for z in range(6) for e in range(4)
                if own[z] == r and own[int(routes[z, e, 0])] != r}
        got = {p for pairs in recvs.values() for p in pairs}
        assert got == need
    if world == 1:
        assert plans[0] == ({}, {})


NX, NR = 8, 5


def _code(pair, phase, ns):
    z, e = pair
    idx = np.arange(ns * NR * 3 * NX, dtype=np.float64)
    return (z * 4 + e) * 1e6 + phase * 1e5 + idx


class _FakePacker:
    """Line store of one rank: its owned zones' lines hold their codes, the rest NaN."""

    def __init__(self, own, rank):
        self.own, self.rank = own, rank
        self.store = {}

    def size(self, phase):
        return (3 if phase < 5 else 5) * NR * 3 * NX

    def fill(self, phase):
        ns = 3 if phase < 5 else 5
        for z in range(6):
            for e in range(4):
                self.store[(z, e)] = _code((z, e), phase, ns) if self.own[z] == self.rank else np.full(ns * NR * 3 * NX, np.nan)

    def pack(self, phase, pairs, buf):
        buf.copy_(__import__("torch").from_numpy(np.concatenate([self.store[p] for p in pairs])))

    def unpack(self, phase, pairs, buf):
        per = self.size(phase)
        a = buf.numpy()
        for q, p in enumerate(pairs):
            self.store[p] = a[q * per:(q + 1) * per].copy()


def _rank_main(rank, world, port, out):
    import torch
    import torch.distributed as dist
    dist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port}", rank=rank, world_size=world)
    try:
        routes = D.route_table()
        parts = D.partition(world)
        own = D.owners(parts)
        packer = _FakePacker(own, rank)
        ex = D.LineExchange(D.exchange_plan(routes, parts, rank), packer, D.p2p_transport(None),
                            lambda n: torch.zeros(n, dtype=torch.float64))
        bad = 0
        for phase in range(6):
            packer.fill(phase)
            ex.run(phase)
            ns = 3 if phase < 5 else 5
            for z in range(6):
                if own[z] != rank:
                    continue
                for e in range(4):
                    pair = (int(routes[z, e, 0]), int(routes[z, e, 1]))
                    if not np.array_equal(packer.store[pair], _code(pair, phase, ns)):
                        bad += 1
        out.put((rank, bad))
    finally:
        dist.destroy_process_group()


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


@pytest.mark.parametrize("world", [2, 3, 6])
def test_line_exchange_over_gloo(world):
    import torch.multiprocessing as mp
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    res = dict(q.get(timeout=120) for _ in range(world))
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert res == {r: 0 for r in range(world)}


# ---------------------------------------------------------------- zones x radial slabs
def test_layout_and_slabs():
    assert [D.layout(w) for w in (1, 2, 3, 4, 6, 8, 12)] == [(1, 1), (2, 1), (3, 1), (2, 2), (6, 1), (2, 4), (6, 2)]
    assert D.layout(5) == (1, 5)
    assert D.slabs(128, 4) == [(0, 32), (32, 64), (64, 96), (96, 128)]
    assert D.slabs(20, 4) == [(0, 5), (5, 10), (10, 15), (15, 20)]
    with pytest.raises(ValueError):
        D.slabs(16, 4)                       # 4 planes per slab: the 5-plane filter halo would span two


@pytest.mark.parametrize("world", [4, 8])
def test_slab_plans_of_neighbours_agree(routes, world):
    ngroups, nsl = D.layout(world)
    plans = [D.slab_plan(world, r) for r in range(world)]
    for r in range(world):
        (sends, recvs), below, above = plans[r]
        zg, sl = divmod(r, nsl)
        for peer, pairs in sends.items():
            assert peer % nsl == sl                              # zone lines stay inside the slab
            assert plans[peer][0][1][r] == pairs
        assert (below is None) == (sl == 0) and (above is None) == (sl == nsl - 1)
        if below is not None:
            assert plans[below][2] == r                          # I am my lower neighbour's upper one
        if above is not None:
            assert plans[above][1] == r


class _FakePlanePacker:
    """Boundary planes of one rank, coded by (rank, side, phase); received codes are kept."""

    def __init__(self, rank):
        self.rank = rank
        self.got = {}

    def size(self, phase):
        return 7 if phase < 5 else 12         # stages share one size, the filter another

    def pack(self, phase, side, buf):
        import torch
        buf.copy_(torch.full((self.size(phase),), float(self.rank * 100 + side * 10 + phase), dtype=torch.float64))

    def unpack(self, phase, side, buf):
        self.got[(phase, side)] = buf.numpy().copy()


def _slab_rank_main(rank, world, port, out):
    import datetime

    import torch
    import torch.distributed as dist
    dist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port}", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=60))
    try:
        ngroups, nsl = D.layout(world)
        zg, sl = divmod(rank, nsl)
        plan, below, above = D.slab_plan(world, rank)
        own = D.owners(D.partition(ngroups))
        own_rank = [D.rank_of(g, sl, nsl) for g in own]          # owner of each zone in my slab
        lines = _FakePacker(own_rank, rank)
        planes = _FakePlanePacker(rank)
        alloc = lambda n: torch.zeros(n, dtype=torch.float64)
        lx = D.LineExchange(plan, lines, D.p2p_transport(None), alloc)
        px = D.PlaneExchange(below, above, planes, D.p2p_transport(None), alloc)
        phases = []

        def step(phase):                     # the kernels of a phase (nothing to move here)
            phases.append(phase)
        bad = 0
        routes = D.route_table()
        for phase in range(5):
            lines.fill(phase)
            lx.run(phase)
            px.run(phase)
            step(phase)
            for z in range(6):
                if own_rank[z] != rank:
                    continue
                for e in range(4):
                    pair = (int(routes[z, e, 0]), int(routes[z, e, 1]))
                    if not np.array_equal(lines.store[pair], _code(pair, phase, 3)):
                        bad += 1
        lines.fill(5)
        lx.run(5)
        step(6)
        px.run(5)
        step(7)
        if phases != [0, 1, 2, 3, 4, 6, 7]:
            bad += 1
        for phase in (0, 1, 2, 3, 4, 5):
            for side, peer in ((0, below), (1, above)):
                if peer is None:
                    continue
                want = float(peer * 100 + (1 - side) * 10 + phase)      # the peer's send toward me
                if not np.all(planes.got[(phase, side)] == want):
                    bad += 1
        out.put((rank, bad))
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("world", [4, 8])
def test_zone_and_slab_exchange_over_gloo(world):
    import torch.multiprocessing as mp
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_slab_rank_main, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    res = dict(q.get(timeout=180) for _ in range(world))
    for p in procs:
        p.join(timeout=60)
    assert res == {r: 0 for r in range(world)}


def _overlap_rank_main(rank, world, port, out):
    """One RK4 call through D.step_sequence with phase parts: each stage's lines are
    started, part 0 runs, and by part 1 the lines of the phase must have arrived."""
    import datetime

    import torch
    import torch.distributed as dist
    dist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port}", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=60))
    try:
        ngroups, nsl = D.layout(world)
        zg, sl = divmod(rank, nsl)
        plan, below, above = D.slab_plan(world, rank)
        own = D.owners(D.partition(ngroups))
        own_rank = [D.rank_of(g, sl, nsl) for g in own]
        lines = _FakePacker(own_rank, rank)
        planes = _FakePlanePacker(rank)
        alloc = lambda n: torch.zeros(n, dtype=torch.float64)
        lx = D.LineExchange(plan, lines, D.p2p_transport(None), alloc)
        px = D.PlaneExchange(below, above, planes, D.p2p_transport(None), alloc)
        routes = D.route_table()
        events = []
        bad = 0

        def lines_bad(phase):
            ns = 3 if phase < 5 else 5
            n = 0
            for z in range(6):
                if own_rank[z] != rank:
                    continue
                for e in range(4):
                    pair = (int(routes[z, e, 0]), int(routes[z, e, 1]))
                    n += not np.array_equal(lines.store[pair], _code(pair, phase, ns))
            return n

        def step(phase):                     # the filter phase: its lines came before it
            nonlocal bad
            events.append(("phase", phase))
            if phase in (5, 6):
                bad += lines_bad(5)

        def part(phase, p):
            nonlocal bad
            events.append(("part", phase, p))
            if p == 1:
                bad += lines_bad(phase)
                lines.fill(phase + 1)        # the owned lines that the next phase sends
        lines.fill(0)
        D.step_sequence(lx, px, step, part)
        tail = [("phase", 5)] if px.empty else [("phase", 6), ("phase", 7)]
        bad += events != [("part", ph, p) for ph in range(5) for p in (0, 1)] + tail
        for phase in range(6):
            for side, peer in ((0, below), (1, above)):
                if peer is not None:
                    bad += not np.all(planes.got[(phase, side)] == float(peer * 100 + (1 - side) * 10 + phase))
        out.put((rank, int(bad)))
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("world", [2, 4, 8])
def test_overlapped_step_sequence_over_gloo(world):
    import torch.multiprocessing as mp
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_overlap_rank_main, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    res = dict(q.get(timeout=180) for _ in range(world))
    for p in procs:
        p.join(timeout=60)
    assert res == {r: 0 for r in range(world)}
