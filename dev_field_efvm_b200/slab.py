"""One grid split into row slabs over several GPUs (one process per GPU).

field_core decomposes a mesh over MPI ranks; every substage each rank fills
the ghosts on its rank edges from its neighbours (halo_exchange_forward_all)
and the solver takes the smallest dt over ranks (all_reduce_min_f64).  Here a
grid of ny rows is split into contiguous row slabs, one device context per
slab (efvm_create_slab), and every RK stage exchanges the two rows next to each
slab edge with the neighbouring slab; once per step the largest wave speed is
max-reduced over slabs (the same dt as the minimum of the per-slab dt).  The
periodic wrap of a periodic y axis is one more slab edge, between the last
slab and the first.

The data path per stage is two rows of four FP64 planes per neighbour
(8 * nx doubles each way), so the exchange is small next to a stage's compute;
it runs on the context's stream and needs no host round trip.

Transports:
  * DistTransport: torch.distributed point-to-point send/recv and all_reduce
    (NCCL with device tensors across GPUs; gloo with CPU tensors in the CPU tests).
  * LocalTransport: all slabs in one process, copied on the device
    (several slabs on one GPU, used to check the split on a single GPU).

An engine is one slab's compute: the device Context (DeviceSlab) or any object
with the same five methods (prepare, pack, unpack, substep, slot).
"""
from __future__ import annotations

from dataclasses import dataclass

import torch

from . import abi

YLO, YHI = abi.YLO, abi.YHI
# tags of the two directions, for transports that match messages by tag
TAG_UP, TAG_DOWN = 11, 12


def split_rows(ny: int, parts: int) -> list[tuple[int, int]]:
    """Contiguous (row0, rows) slabs, sizes differing by at most one, each >= 2."""
    if parts < 1 or ny < 2 * parts:
        raise ValueError(f"cannot split {ny} rows into {parts} slabs of at least 2 rows")
    base, extra = divmod(ny, parts)
    out, r = [], 0
    for k in range(parts):
        n = base + (1 if k < extra else 0)
        out.append((r, n))
        r += n
    return out


@dataclass
class Neighbours:
    lower: int | None  # slab below (rows with smaller j), or None at a wall
    upper: int | None


def neighbours(rank: int, world: int, periodic_y: bool) -> Neighbours:
    lo = rank - 1 if rank > 0 else (world - 1 if periodic_y else None)
    hi = rank + 1 if rank < world - 1 else (0 if periodic_y else None)
    return Neighbours(lo, hi)


class DeviceSlab:
    """The device engine of one slab: a Context made with efvm_create_slab."""

    def __init__(self, grid: abi.EfvmGrid, params: abi.EfvmParams, row0: int, rows: int):
        from .device import Context

        self.ctx = Context(grid, params, rows=(row0, rows))
        self.nx, self.ny = grid.nx, rows
        self.device = torch.device("cuda", torch.cuda.current_device())
        self.stream = torch.cuda.ExternalStream(self.ctx.stream())
        ptr = self.ctx.wave_speed_slot()
        # a zero-copy int64 view of the slot (non-negative doubles' bits order like the values)
        self._slot = torch.as_tensor(_CudaWord(ptr), device=self.device)

    def new_buffer(self) -> torch.Tensor:
        return torch.empty(8 * self.nx, dtype=torch.float64, device=self.device)

    def prepare(self) -> None:
        self.ctx.prepare()

    def pack(self, side: int, buf: torch.Tensor) -> None:
        self.ctx.halo_pack(side, buf.data_ptr())

    def unpack(self, side: int, buf: torch.Tensor) -> None:
        self.ctx.halo_unpack(side, buf.data_ptr())

    def substep(self) -> None:
        self.ctx.substep()

    def slot(self) -> torch.Tensor:
        return self._slot

    def synchronize(self) -> None:
        self.stream.synchronize()

    # halo peers across processes (DistPeerSlabs)
    def export_peer(self) -> tuple[bytes, int, int]:
        """CUDA IPC handles of this slab's state buffers, their plane and rows."""
        _, plane, rows = self.ctx.state_buffers()
        return self.ctx.state_ipc(), plane, rows

    def map_peer(self, side: int, handles: bytes, plane: int, rows: int) -> None:
        self.ctx.set_halo_peer_ipc(side, handles, plane, rows)

    def map_self(self, side: int) -> None:
        """One slab on a periodic axis: its own buffers are the peer across the wrap."""
        bufs, plane, rows = self.ctx.state_buffers()
        self.ctx.set_halo_peer(side, bufs, plane, rows)

    def token(self) -> torch.Tensor:
        return torch.zeros(1, dtype=torch.int64, device=self.device)


class _CudaWord:
    """__cuda_array_interface__ of one int64 at a device address."""

    def __init__(self, ptr: int):
        self.__cuda_array_interface__ = {"shape": (1,), "typestr": "<i8", "data": (ptr, False), "version": 3}


class DistTransport:
    """Halo rows and the wave-speed maximum over torch.distributed.

    Every rank posts the same pattern: sends to the upper then the lower
    neighbour, receives from the lower then the upper one, so that with two
    slabs on a periodic axis (the same peer above and below) the messages pair
    up in order; tags make the pairing explicit for transports that use them."""

    def __init__(self, group=None):
        import torch.distributed as dist

        self.dist = dist
        self.group = group
        self.rank = dist.get_rank(group)
        self.world = dist.get_world_size(group)

    def exchange(self, nb: Neighbours, send_lo, send_hi, recv_lo, recv_hi) -> None:
        dist = self.dist
        ops = []
        if nb.upper is not None and nb.upper != self.rank:
            ops.append(dist.P2POp(dist.isend, send_hi, nb.upper, self.group, TAG_UP))
        if nb.lower is not None and nb.lower != self.rank:
            ops.append(dist.P2POp(dist.isend, send_lo, nb.lower, self.group, TAG_DOWN))
        if nb.lower is not None and nb.lower != self.rank:
            ops.append(dist.P2POp(dist.irecv, recv_lo, nb.lower, self.group, TAG_UP))
        if nb.upper is not None and nb.upper != self.rank:
            ops.append(dist.P2POp(dist.irecv, recv_hi, nb.upper, self.group, TAG_DOWN))
        if nb.lower == self.rank:  # one slab on a periodic axis: the wrap is local
            recv_lo.copy_(send_hi)
        if nb.upper == self.rank:
            recv_hi.copy_(send_lo)
        if ops:
            for w in dist.batch_isend_irecv(ops):
                w.wait()

    def max_reduce(self, word: torch.Tensor) -> None:
        if self.world > 1:
            self.dist.all_reduce(word, op=self.dist.ReduceOp.MAX, group=self.group)


class SlabRank:
    """This process's slab of the grid, stepped in lockstep with the others."""

    def __init__(self, engine, nb: Neighbours, transport):
        self.e, self.nb, self.t = engine, nb, transport
        mk = getattr(engine, "new_buffer")
        self.send = {YLO: mk(), YHI: mk()}
        self.recv = {YLO: mk(), YHI: mk()}
        self.stream = getattr(engine, "stream", None)

    def _ctx(self):
        if self.stream is not None:
            return torch.cuda.stream(self.stream)
        return _Null()

    def exchange(self) -> None:
        """Fill both halo sides of the next substep's input from the neighbours."""
        e, nb = self.e, self.nb
        if nb.lower is not None:
            e.pack(YLO, self.send[YLO])
        if nb.upper is not None:
            e.pack(YHI, self.send[YHI])
        with self._ctx():
            self.t.exchange(nb, self.send[YLO], self.send[YHI], self.recv[YLO], self.recv[YHI])
        if nb.lower is not None:
            e.unpack(YLO, self.recv[YLO])
        if nb.upper is not None:
            e.unpack(YHI, self.recv[YHI])

    def step(self, n_steps: int) -> None:
        """n whole SSP-RK3 steps (every rank calls this with the same n)."""
        for _ in range(n_steps):
            self.e.prepare()
            with self._ctx():
                self.t.max_reduce(self.e.slot())
            for _s in range(3):
                self.exchange()
                self.e.substep()


class _Null:
    def __enter__(self):
        return self

    def __exit__(self, *a):
        return False


class LocalTransport:
    """Every slab in this process: the exchange and the reduction are device
    copies between the slabs' buffers, ordered by synchronising the slabs'
    streams (a single-GPU stand-in for the multi-GPU transport)."""

    def __init__(self, engines, periodic_y: bool):
        self.engines = engines
        self.world = len(engines)
        self.nbs = [neighbours(k, self.world, periodic_y) for k in range(self.world)]
        mk = [e.new_buffer for e in engines]
        self.send = [{YLO: mk[k](), YHI: mk[k]()} for k in range(self.world)]
        self.recv = [{YLO: mk[k](), YHI: mk[k]()} for k in range(self.world)]

    def _sync(self):
        for e in self.engines:
            if hasattr(e, "synchronize"):
                e.synchronize()

    def exchange(self) -> None:
        for k, e in enumerate(self.engines):
            if self.nbs[k].lower is not None:
                e.pack(YLO, self.send[k][YLO])
            if self.nbs[k].upper is not None:
                e.pack(YHI, self.send[k][YHI])
        self._sync()
        for k in range(self.world):
            nb = self.nbs[k]
            if nb.lower is not None:
                self.recv[k][YLO].copy_(self.send[nb.lower][YHI])
            if nb.upper is not None:
                self.recv[k][YHI].copy_(self.send[nb.upper][YLO])
        if torch.cuda.is_available():
            torch.cuda.synchronize()
        for k, e in enumerate(self.engines):
            if self.nbs[k].lower is not None:
                e.unpack(YLO, self.recv[k][YLO])
            if self.nbs[k].upper is not None:
                e.unpack(YHI, self.recv[k][YHI])

    def reduce(self) -> None:
        self._sync()
        words = [e.slot() for e in self.engines]
        m = torch.stack([w.clone() for w in words]).max(dim=0).values
        for w in words:
            w.copy_(m)
        if torch.cuda.is_available():
            torch.cuda.synchronize()

    def step(self, n_steps: int) -> None:
        for _ in range(n_steps):
            for e in self.engines:
                e.prepare()
            self.reduce()
            for _s in range(3):
                self.exchange()
                for e in self.engines:
                    e.substep()
        self._sync()


class PeerLocalSlabs:
    """Every slab on this GPU, with the halo exchange fused into the stage
    kernels (efvm_set_halo_peer): each stage stores its edge rows straight into
    the neighbouring slabs' ghost rows of the same stage's output, so no pack,
    copy or unpack runs between stages.  Stage t of a slab waits (a stream
    event, no host round trip) for stage t - 1 of both neighbours: their rows
    in its input have been written, and its own stores cannot overtake their
    reads of the buffer it writes.  One pack / unpack exchange fills the ghost
    rows of the uploaded state before the first step; the wave-speed slot is
    max-reduced once per step on the device, ordered by events, so a run of
    steps makes no host round trip."""

    def __init__(self, engines, periodic_y: bool):
        self.engines = engines
        self.local = LocalTransport(engines, periodic_y)
        self.nbs = self.local.nbs
        for k, e in enumerate(engines):
            for side, other in ((YLO, self.nbs[k].lower), (YHI, self.nbs[k].upper)):
                if other is not None:
                    bufs, plane, rows = engines[other].ctx.state_buffers()
                    e.ctx.set_halo_peer(side, bufs, plane, rows)
        self.events = [[torch.cuda.Event() for _ in engines] for _ in range(2)]
        self.rstream = torch.cuda.Stream()
        self.prepared = [torch.cuda.Event() for _ in engines]
        self.reduced = torch.cuda.Event()
        self.stage = 0
        self.primed = False

    def _reduce(self) -> None:
        """Max of the slabs' wave-speed words on the device: after every slab's
        set-up work (and so after its last stage), before any slab's next stage,
        with no host round trip (the words are the bits of non-negative doubles,
        so their integer max is the max wave speed)."""
        for ev, e in zip(self.prepared, self.engines):
            ev.record(e.stream)
            self.rstream.wait_event(ev)
        with torch.cuda.stream(self.rstream):
            words = [e.slot() for e in self.engines]
            m = torch.stack(words).max(dim=0).values
            for w in words:
                w.copy_(m)
        self.reduced.record(self.rstream)
        for e in self.engines:
            e.stream.wait_event(self.reduced)

    def step(self, n_steps: int) -> None:
        if not self.primed:  # the ghost rows of the uploaded state
            for e in self.engines:
                e.prepare()
            self.local.exchange()
            self.primed = True
        for _ in range(n_steps):
            for e in self.engines:
                e.prepare()
            self._reduce()
            for _s in range(3):
                prev, cur = self.events[(self.stage + 1) % 2], self.events[self.stage % 2]
                for k, e in enumerate(self.engines):
                    if self.stage > 0:
                        for o in {self.nbs[k].lower, self.nbs[k].upper} - {None, k}:
                            e.stream.wait_event(prev[o])
                    e.substep()
                    cur[k].record(e.stream)
                self.stage += 1
        self.local._sync()


class DistPeerSlabs:
    """This process's slab, one process per GPU, with the halo exchange fused
    into its stage kernels over peer memory: every rank exports its three state
    buffers as CUDA IPC handles, all ranks gather them, and each slab maps its
    neighbours' buffers (peer access over NVLink) and stores its edge rows into
    their ghost rows as it writes them.  What remains of the collective is
    ordering: after stages 1 and 2 every rank all-reduces an 8-byte token on the
    context's stream, so no rank starts a stage before every rank has finished
    the one before (its rows have landed, and the buffer it writes is no longer
    read); before stage 1 the per-step max-reduce of the wave-speed slot does the
    same.  One pack / exchange / unpack through DistTransport fills the ghost
    rows of the uploaded state first.  Every rank takes the same collective
    steps in the same order."""

    def __init__(self, engine, nb: Neighbours, group=None):
        import torch.distributed as dist

        self.e, self.nb, self.dist, self.group = engine, nb, dist, group
        rank = dist.get_rank(group)
        exports = [None] * dist.get_world_size(group)
        dist.all_gather_object(exports, engine.export_peer(), group=group)
        self.mapped = {}
        for side, other in ((YLO, nb.lower), (YHI, nb.upper)):
            if other is None:
                continue
            if other == rank:
                engine.map_self(side)
            else:
                engine.map_peer(side, *exports[other])
            self.mapped[side] = other
        self.token = engine.token()
        self.rank = SlabRank(engine, nb, DistTransport(group))
        self.primed = False

    def _all_reduce(self, t) -> None:
        with self.rank._ctx():
            self.dist.all_reduce(t, op=self.dist.ReduceOp.MAX, group=self.group)

    def step(self, n_steps: int) -> None:
        if not self.primed:
            self.e.prepare()
            self.rank.exchange()
            self.primed = True
        for _ in range(n_steps):
            self.e.prepare()
            self._all_reduce(self.e.slot())
            for s in range(3):
                self.e.substep()
                if s < 2:
                    self._all_reduce(self.token)
