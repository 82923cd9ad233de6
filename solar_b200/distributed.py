"""The sphere split across processes, one GPU per process: zones and radial slabs.

The reference decomposes the sphere into zone blocks of px x py x pr ranks (header:4-6,
init_mpi.f90): interpolated 3-deep halo strips cross zone edges inside every derivative and
filter (derivative.f90:8-323, filter.f90:9-48, routed by the intercommunicator partner map
of init_mpi.f90:164-304), and radial neighbours exchange 3 planes for DDR and 5 for the
radial filter (derivative.f90:605-758, filter.f90:633-781).  Here a job of W processes is
laid out as G zone groups x S radial slabs, G = gcd(W, 6): each process owns a contiguous
range of 6/G zones and of about nr/S radial planes and runs the same fused kernels on them
(``solar_gpu_set_owned_zones``, ``solar_gpu_set_owned_planes``).

* Zone edges: before each phase of a step (five stages, then the filter) a process sends, to
  every process of its slab owning a neighbouring zone, the three raw lines next to each
  shared edge over its owned planes; the receiver interpolates and rotates them into its
  ghost frame with its own edge kernel, exactly as for a zone it owns.
* Radial slabs: before each stage a process sends the 3 planes of p and v_r next to each slab
  boundary to the neighbouring slab of its zone group; the filter phase is split around its
  edge exchange, and between the halves the 5 planes of every field (frames included) move.

The plans (which pairs and planes go where, in which order) are pure host logic, tested on
CPU with the gloo backend; the transfer is ``torch.distributed`` point-to-point (NCCL between
GPUs) ordered on the library's CUDA stream.  No kernel reads another GPU's memory.
"""
from __future__ import annotations

import ctypes
import math
from typing import Dict, List, Optional, Sequence, Tuple

import numpy as np

from . import _lib

Pair = Tuple[int, int]            # (source zone, source edge), 0-based; edges 0 S, 1 N, 2 W, 3 E


def partition(world: int) -> List[Tuple[int, int]]:
    """Contiguous zone ranges (zone0, nzones) of each zone group; world must divide 6."""
    if world < 1 or 6 % world:
        raise ValueError(f"zone splitting needs 1, 2, 3 or 6 processes, not {world}")
    per = 6 // world
    return [(r * per, per) for r in range(world)]


def layout(world: int) -> Tuple[int, int]:
    """(zone groups, radial slabs) of a job of `world` processes: G = gcd(world, 6) zone
    groups, world / G slabs (2 -> 2 x 1, 4 -> 2 x 2, 8 -> 2 x 4, 12 -> 6 x 2, 5 -> 1 x 5)."""
    if world < 1:
        raise ValueError("world must be >= 1")
    g = math.gcd(world, 6)
    return g, world // g


def slabs(nr: int, nslabs: int) -> List[Tuple[int, int]]:
    """Owned plane ranges [k0, k1) of the radial slabs; each holds >= 5 planes, so the
    5-plane filter halo of a slab comes from its neighbour alone."""
    if nslabs < 1 or nr // nslabs < 5:
        raise ValueError(f"{nslabs} radial slabs of {nr} planes would hold fewer than 5 planes each")
    return [(s * nr // nslabs, (s + 1) * nr // nslabs) for s in range(nslabs)]


def rank_of(zone_group: int, slab: int, nslabs: int) -> int:
    return zone_group * nslabs + slab


def route_table() -> np.ndarray:
    """(6, 4, 3) array: for receiving zone z and edge e, (source zone, source edge,
    reversed) -- the library's copy of the reference's halo routing."""
    out = (ctypes.c_int * 72)()
    _lib.check(_lib.load().solar_gpu_edge_routes(out))
    return np.array(out, dtype=np.int64).reshape(6, 4, 3)


def owners(parts: Sequence[Tuple[int, int]]) -> List[int]:
    own = [-1] * 6
    for r, (z0, nz) in enumerate(parts):
        for z in range(z0, z0 + nz):
            own[z] = r
    return own


def exchange_plan(routes: np.ndarray, parts: Sequence[Tuple[int, int]], rank: int):
    """(sends, recvs): for each peer rank, the ordered (zone, edge) source pairs this rank
    sends to / receives from it.  Both sides enumerate receivers in the same global order
    (receiving zone, then edge), so the lists of a sender and its receiver match."""
    own = owners(parts)
    sends: Dict[int, List[Pair]] = {}
    recvs: Dict[int, List[Pair]] = {}
    for z in range(6):
        for e in range(4):
            sz, se = int(routes[z, e, 0]), int(routes[z, e, 1])
            src, dst = own[sz], own[z]
            if src == dst:
                continue
            if src == rank:
                sends.setdefault(dst, []).append((sz, se))
            if dst == rank:
                recvs.setdefault(src, []).append((sz, se))
    return sends, recvs


def _pairs_array(pairs: Sequence[Pair]):
    a = (ctypes.c_int * (2 * len(pairs)))()
    for q, (z, e) in enumerate(pairs):
        a[2 * q], a[2 * q + 1] = z, e
    return a


class LineExchange:
    """Moves the edge lines of one phase between ranks.

    ``packer`` provides ``size(phase)`` (values per pair), ``pack(phase, pairs, buf)`` and
    ``unpack(phase, pairs, buf)``; ``transport(sends, recvs)`` delivers every send buffer to
    its peer and fills every receive buffer (``{peer: buffer}`` dicts).  ``alloc(n)``
    returns an n-value buffer."""

    def __init__(self, plan, packer, transport, alloc):
        self.sends, self.recvs = plan
        self.packer, self.transport = packer, transport
        self._buf = {}
        for kind, phase in (("stage", 0), ("filter", 5)):
            per = packer.size(phase)
            self._buf[kind] = ({p: alloc(len(v) * per) for p, v in self.sends.items()},
                               {p: alloc(len(v) * per) for p, v in self.recvs.items()})

    @property
    def empty(self) -> bool:
        return not self.sends and not self.recvs

    def buffers(self, phase: int):
        """({peer: send buffer}, {peer: receive buffer}) of this phase."""
        return self._buf["filter" if phase == 5 else "stage"]

    def pack(self, phase: int) -> None:
        sbuf, _ = self.buffers(phase)
        for peer, pairs in self.sends.items():
            self.packer.pack(phase, pairs, sbuf[peer])

    def unpack(self, phase: int) -> None:
        _, rbuf = self.buffers(phase)
        for peer, pairs in self.recvs.items():
            self.packer.unpack(phase, pairs, rbuf[peer])

    def run(self, phase: int) -> None:
        if self.empty:
            return
        self.pack(phase)
        self.transport(*self.buffers(phase))
        self.unpack(phase)

    def start(self, phase: int):
        """Pack this phase's lines and start their transfer without waiting for it; returns
        the pending transfer for finish().  A transport without ``start``/``finish``
        attributes moves the lines here, at once."""
        if self.empty:
            return None
        self.pack(phase)
        begin = getattr(self.transport, "start", None)
        if begin is None:
            self.transport(*self.buffers(phase))
            return None
        return begin(*self.buffers(phase))

    def finish(self, phase: int, pending) -> None:
        """Wait for the transfer start() began, then unpack the received lines."""
        if self.empty:
            return
        if pending is not None:
            self.transport.finish(pending)
        self.unpack(phase)


class _LibPacker:
    """pack/unpack through the C-ABI into CUDA tensors, on the context's stream."""

    def __init__(self, solver):
        self.s = solver

    def size(self, phase):
        return int(self.s.lib.solar_gpu_lines_size(self.s._h, phase))

    def pack(self, phase, pairs, buf):
        _lib.check(self.s.lib.solar_gpu_pack_lines(self.s._h, phase, _pairs_array(pairs), len(pairs),
                                                   ctypes.c_void_p(buf.data_ptr())))

    def unpack(self, phase, pairs, buf):
        _lib.check(self.s.lib.solar_gpu_unpack_lines(self.s._h, phase, _pairs_array(pairs), len(pairs),
                                                     ctypes.c_void_p(buf.data_ptr())))


def slab_plan(world: int, rank: int):
    """(line plan, below, above) of a rank: the zone-edge exchange among the ranks of its
    slab (peers as global ranks) and its radial neighbours in its zone group (None at the
    two ends of the shell)."""
    ngroups, nsl = layout(world)
    zg, sl = divmod(rank, nsl)
    sends, recvs = exchange_plan(route_table(), partition(ngroups), zg)
    glob = lambda d: {rank_of(p, sl, nsl): v for p, v in d.items()}
    below = rank_of(zg, sl - 1, nsl) if sl > 0 else None
    above = rank_of(zg, sl + 1, nsl) if sl < nsl - 1 else None
    return (glob(sends), glob(recvs)), below, above


class PlaneExchange:
    """Moves the boundary planes of one phase between radially neighbouring ranks.

    ``packer`` provides ``size(phase)``, ``pack(phase, side, buf)`` and
    ``unpack(phase, side, buf)`` (side 0 = the neighbour below, 1 = above); ``transport``
    as for :class:`LineExchange`."""

    def __init__(self, below: Optional[int], above: Optional[int], packer, transport, alloc):
        self.peers = {0: below, 1: above}
        self.packer, self.transport = packer, transport
        self._buf = {}
        for kind, phase in (("stage", 0), ("filter", 5)):
            per = packer.size(phase)
            self._buf[kind] = ({sd: alloc(per) for sd, p in self.peers.items() if p is not None},
                               {sd: alloc(per) for sd, p in self.peers.items() if p is not None})

    @property
    def empty(self) -> bool:
        return all(p is None for p in self.peers.values())

    def buffers(self, phase: int):
        """({side: send buffer}, {side: receive buffer}) of this phase."""
        return self._buf["filter" if phase == 5 else "stage"]

    def pack(self, phase: int) -> None:
        for sd, b in self.buffers(phase)[0].items():
            self.packer.pack(phase, sd, b)

    def unpack(self, phase: int) -> None:
        for sd, b in self.buffers(phase)[1].items():
            self.packer.unpack(phase, sd, b)

    def run(self, phase: int) -> None:
        if self.empty:
            return
        self.pack(phase)
        sbuf, rbuf = self.buffers(phase)
        self.transport({self.peers[sd]: b for sd, b in sbuf.items()}, {self.peers[sd]: b for sd, b in rbuf.items()})
        self.unpack(phase)


class _LibPlanePacker:
    """Boundary planes through the C-ABI into CUDA tensors, on the context's stream."""

    def __init__(self, solver):
        self.s = solver

    def size(self, phase):
        return int(self.s.lib.solar_gpu_planes_size(self.s._h, phase))

    def pack(self, phase, side, buf):
        _lib.check(self.s.lib.solar_gpu_pack_planes(self.s._h, phase, side, ctypes.c_void_p(buf.data_ptr())))

    def unpack(self, phase, side, buf):
        _lib.check(self.s.lib.solar_gpu_unpack_planes(self.s._h, phase, side, ctypes.c_void_p(buf.data_ptr())))


def step_sequence(lines: "LineExchange", planes: "PlaneExchange", step_phase, step_part=None) -> None:
    """One RK4 call of a rank: edge lines and boundary planes before each stage; the filter
    phase split around its edge exchange, with the filter's boundary planes in between.

    With ``step_part(phase, part)`` (solar_gpu_step_phase_part) each stage overlaps its line
    transfer: the boundary planes move first, then the lines are packed and sent, the stage
    runs on the interior tiles (part 0, which needs no line) while they are in transit, and
    after they are unpacked the edge kernel and the face-edge tiles run (part 1)."""
    for phase in range(5):
        if step_part is None:
            lines.run(phase)
            planes.run(phase)
            step_phase(phase)
            continue
        planes.run(phase)
        pending = lines.start(phase)
        step_part(phase, 0)
        lines.finish(phase, pending)
        step_part(phase, 1)
    lines.run(5)
    if planes.empty:
        step_phase(5)
    else:
        step_phase(6)
        planes.run(5)
        step_phase(7)


def p2p_transport(stream=None, group=None):
    """torch.distributed point-to-point exchange, issued on ``stream`` (a torch stream;
    the library's stream for GPU buffers) so that it is ordered after the packing and
    before the unpacking."""
    import contextlib

    import torch
    import torch.distributed as dist

    def ctx():
        return torch.cuda.stream(stream) if stream is not None else contextlib.nullcontext()

    def start(sends, recvs):
        """Issue the sends and receives; NCCL runs them on its own stream after the packing."""
        with ctx():
            ops = [dist.P2POp(dist.isend, b, p, group) for p, b in sorted(sends.items())]
            ops += [dist.P2POp(dist.irecv, b, p, group) for p, b in sorted(recvs.items())]
            return dist.batch_isend_irecv(ops) if ops else []

    def finish(reqs):
        """Order ``stream`` after the transfers (NCCL: a stream wait, not a host wait)."""
        with ctx():
            for req in reqs:
                req.wait()

    def run(sends, recvs):
        finish(start(sends, recvs))
    run.start, run.finish = start, finish
    return run


class ZoneSplitSolver:
    """One rank's share of a six-zone run: owns the zones of its zone group and the planes
    of its radial slab (``layout(world)``) of a :class:`solar_b200.solver.Solver` on this
    process's GPU, and exchanges edge lines and boundary planes with the other ranks every
    phase.  ``torch.distributed`` must be initialised (NCCL)."""

    def __init__(self, cfg, precision: str = "fp64", nfields: int = 5, device: int = 0, group=None,
                 overlap: bool = True, **kw):
        import torch
        import torch.distributed as dist

        from .solver import Solver

        self.overlap = overlap               # stage interiors run while the lines are in transit
        self.world = dist.get_world_size(group)
        self.rank = dist.get_rank(group)
        self.group = group
        ngroups, nsl = layout(self.world)
        zg, sl = divmod(self.rank, nsl)
        self.parts = partition(ngroups)
        self.zone0, self.nzones = self.parts[zg]
        self.k0, self.k1 = slabs(cfg.nr, nsl)[sl]
        self.solver = Solver(cfg, precision=precision, nfields=nfields, device=device, **kw)
        s = self.solver
        _lib.check(s.lib.solar_gpu_set_owned_zones(s._h, self.zone0, self.nzones))
        _lib.check(s.lib.solar_gpu_set_owned_planes(s._h, self.k0, self.k1))
        self.stream = torch.cuda.ExternalStream(s.lib.solar_gpu_stream(s._h), device=torch.device("cuda", device))
        dtype = torch.float32 if precision == "fp32" else torch.float64
        alloc = lambda n: torch.empty(n, dtype=dtype, device=torch.device("cuda", device))
        plan, below, above = slab_plan(self.world, self.rank)
        transport = p2p_transport(self.stream, group)
        self.exchange = LineExchange(plan, _LibPacker(s), transport, alloc)
        self.planes = PlaneExchange(below, above, _LibPlanePacker(s), transport, alloc)

    def set_state(self, q: np.ndarray) -> None:
        """Every rank loads the whole six-zone state (it computes only its own share)."""
        self.solver.set_state(q)

    def rk4(self, nsteps: int = 1) -> None:
        s = self.solver
        step = lambda phase: _lib.check(s.lib.solar_gpu_step_phase(s._h, phase))
        part = lambda phase, p: _lib.check(s.lib.solar_gpu_step_phase_part(s._h, phase, p))
        for _ in range(int(nsteps)):
            step_sequence(self.exchange, self.planes, step, part if self.overlap else None)
        s.synchronize()

    def norm(self, field: int = 4) -> float:
        """auxiliary.f90:100-125 over the whole sphere: owned partial sums, all-reduced."""
        import torch
        import torch.distributed as dist

        out = (ctypes.c_double * 5)()
        _lib.check(self.solver.lib.solar_gpu_reduce_owned(self.solver._h, 0, field, out))
        t = torch.tensor([out[0]], dtype=torch.float64, device=torch.device("cuda", torch.cuda.current_device()))
        dist.all_reduce(t, group=self.group)
        n, nr = self.solver.nx, self.solver.nr
        return float((t.item() / (n * n * nr) * 6.0) ** 0.5)

    def gather_state(self) -> np.ndarray:
        """The whole six-zone state, assembled from every rank's owned zones and planes."""
        import torch.distributed as dist

        q = self.solver.get_state()
        mine = (self.zone0, self.k0, q[self.zone0:self.zone0 + self.nzones, :, self.k0:self.k1])
        allp = [None] * self.world
        dist.all_gather_object(allp, mine, group=self.group)
        for z0, k0, part in allp:
            q[z0:z0 + part.shape[0], :, k0:k0 + part.shape[2]] = part
        return q

    def close(self) -> None:
        self.solver.close()
