"""Row-slab decomposition: the host logic on CPU (gloo ranks and in-process
slabs) and the device slabs on one GPU.

The reference checks its MPI decomposition by running one periodic case on
1..4 ranks and comparing global moments to 1e-12 (tests/periodic_mpi.rs).
Here the CPU tests drive the slab orchestration (row split, neighbour pattern,
halo exchange order, wave-speed reduction, periodic wrap) with a small NumPy
stand-in engine whose one-slab run is the plain global scheme, over world sizes
1, 2 and 4 with torch.distributed (gloo) and in one process.  The GPU tests run
the device slabs (efvm_create_slab) for 1..4 slabs on one GPU and require the
result of the unsplit context bit for bit."""
from __future__ import annotations

import os
import tempfile

import numpy as np
import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

from dev_field_efvm_b200 import abi, cases, slab


# ---------------------------------------------------------------------------
# a stand-in engine: 2-D Burgers u_t + (u^2/2)_x + (u^2/2)_y = 0, Rusanov flux,
# SSP-RK3, dt = cfl h / max|u| over the whole grid; periodic in x; in y periodic
# (through the halo) or zero-gradient walls.  The same call pattern as a device
# slab: stage input with two ghost rows per side, pack/unpack of two rows, an
# external max slot read by the step's first stage.
# ---------------------------------------------------------------------------
class FakeSlab:
    def __init__(self, u_global: np.ndarray, row0: int, rows: int, lo_wall: bool, hi_wall: bool, cfl=0.4):
        self.nx = u_global.shape[1]
        self.ny = rows
        self.h = 1.0 / self.nx
        self.cfl = cfl
        self.lo_wall, self.hi_wall = lo_wall, hi_wall
        self.U = [np.zeros((rows + 4, self.nx)) for _ in range(3)]
        self.U[0][2:-2] = u_global[row0:row0 + rows]
        self.stage = 0
        self.word = torch.zeros(1, dtype=torch.int64)
        self.stale = True
        self.dt = 0.0

    def new_buffer(self):
        return torch.zeros(2 * self.nx, dtype=torch.float64)

    def _max_into_slot(self, q):
        m = float(np.max(np.abs(q[2:-2])))
        self.word[0] = max(int(self.word[0]), int(np.float64(m).view(np.int64)))

    def prepare(self):
        if self.stage == 0 and self.stale:
            self.word.zero_()
            self._max_into_slot(self.U[0])
            self.stale = False

    def slot(self):
        return self.word

    def pack(self, side, buf):
        q = self.U[self.stage]
        rows = q[2:4] if side == abi.YLO else q[-4:-2]
        buf.copy_(torch.from_numpy(rows.reshape(-1).copy()))

    def unpack(self, side, buf):
        q = self.U[self.stage]
        r = buf.numpy().reshape(2, self.nx)
        if side == abi.YLO:
            q[0:2] = r
        else:
            q[-2:] = r

    def _rhs(self, q):
        if self.lo_wall:
            q[0:2] = q[2]
        if self.hi_wall:
            q[-2:] = q[-3]
        f = 0.5 * q * q
        # x faces (periodic): between i-1 and i
        ql, fl = np.roll(q, 1, axis=1), np.roll(f, 1, axis=1)
        ax = np.maximum(np.abs(ql), np.abs(q))
        fx = 0.5 * (fl + f) - 0.5 * ax * (q - ql)
        # y faces: between row r and r+1 of the padded array
        ay = np.maximum(np.abs(q[:-1]), np.abs(q[1:]))
        fy = 0.5 * (f[:-1] + f[1:]) - 0.5 * ay * (q[1:] - q[:-1])
        rhs = np.zeros_like(q)
        rhs[2:-2] = -(np.roll(fx, -1, axis=1)[2:-2] - fx[2:-2]) / self.h - (fy[2:-1] - fy[1:-2]) / self.h
        return rhs

    def substep(self):
        s = self.stage
        if s == 0:
            lam = float(np.int64(self.word[0]).view(np.float64))
            self.dt = self.cfl * self.h / lam
            self.word.zero_()
        q = self.U[s]
        r = self._rhs(q)
        if s == 0:
            new = q + self.dt * r
        elif s == 1:
            new = 0.75 * self.U[0] + 0.25 * (q + self.dt * r)
        else:
            new = (1.0 / 3.0) * self.U[0] + (2.0 / 3.0) * (q + self.dt * r)
        out = (s + 1) % 3
        self.U[out][2:-2] = new[2:-2]
        if s == 2:
            self._max_into_slot(self.U[0])
        self.stage = out

    def interior(self):
        return self.U[0][2:-2].copy()


class FakePeerSlab(FakeSlab):
    """FakeSlab whose three buffers live in shared memory-mapped files, so that
    gloo ranks can act as halo peers of one another (the host-side stand-in for
    CUDA IPC mappings): export_peer names the files, map_peer opens a
    neighbour's, and each stage stores its two edge rows straight into the
    neighbour's ghost rows of the same stage's output, as the device stage
    kernel does with efvm_set_halo_peer."""

    def __init__(self, u_global, row0, rows, lo_wall, hi_wall, folder, rank):
        super().__init__(u_global, row0, rows, lo_wall, hi_wall)
        self.paths = [os.path.join(folder, f"slab{rank}_U{k}.bin") for k in range(3)]
        mm = []
        for k, path in enumerate(self.paths):
            m = np.memmap(path, dtype=np.float64, mode="w+", shape=self.U[k].shape)
            m[:] = self.U[k]
            m.flush()
            mm.append(m)
        self.U = mm
        self.peer = {}

    def export_peer(self):
        return "\n".join(self.paths).encode(), 0, self.ny

    def map_peer(self, side, handles, plane, rows):
        self.peer[side] = [np.memmap(p, dtype=np.float64, mode="r+", shape=(rows + 4, self.nx))
                           for p in handles.decode().split("\n")]

    def map_self(self, side):
        self.peer[side] = self.U

    def token(self):
        return torch.zeros(1, dtype=torch.int64)

    def substep(self):
        out = (self.stage + 1) % 3
        super().substep()
        q = self.U[out]
        if abi.YLO in self.peer:  # rows 0, 1 -> the lower slab's top ghost rows
            lo = self.peer[abi.YLO][out]
            lo[-2:] = q[2:4]
            lo.flush()
        if abi.YHI in self.peer:  # rows ny-2, ny-1 -> the upper slab's bottom ghost rows
            hi = self.peer[abi.YHI][out]
            hi[0:2] = q[-4:-2]
            hi.flush()
        q.flush()


def initial(ny=24, nx=20, seed=3):
    rng = np.random.default_rng(seed)
    y, x = np.meshgrid(np.arange(ny) / ny, np.arange(nx) / nx, indexing="ij")
    return 0.5 + 0.3 * np.sin(2 * np.pi * x) * np.cos(2 * np.pi * y) + 0.05 * rng.random((ny, nx))


def run_local(u, world, periodic, steps=6):
    parts = slab.split_rows(u.shape[0], world)
    engines = []
    for k, (r0, n) in enumerate(parts):
        nb = slab.neighbours(k, world, periodic)
        engines.append(FakeSlab(u, r0, n, lo_wall=nb.lower is None, hi_wall=nb.upper is None))
    slab.LocalTransport(engines, periodic).step(steps)
    return np.concatenate([e.interior() for e in engines]), engines[0].dt


def test_split_rows_and_neighbours():
    assert slab.split_rows(10, 3) == [(0, 4), (4, 3), (7, 3)]
    assert slab.split_rows(8, 4) == [(0, 2), (2, 2), (4, 2), (6, 2)]
    with pytest.raises(ValueError):
        slab.split_rows(7, 4)
    assert slab.neighbours(0, 3, True) == slab.Neighbours(2, 1)
    assert slab.neighbours(2, 3, True) == slab.Neighbours(1, 0)
    assert slab.neighbours(0, 3, False) == slab.Neighbours(None, 1)
    assert slab.neighbours(0, 1, True) == slab.Neighbours(0, 0)


@pytest.mark.parametrize("periodic", [True, False])
def test_local_slabs_match_one_slab(periodic):
    u = initial()
    ref, dt_ref = run_local(u, 1, periodic)
    assert not np.array_equal(ref, u)
    for world in (2, 3, 4):
        got, dt = run_local(u, world, periodic)
        assert dt == dt_ref
        assert np.array_equal(got, ref), f"{world} slabs differ from one"


def _gloo_worker(rank, world, periodic, port, out_dir):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        u = initial()
        r0, n = slab.split_rows(u.shape[0], world)[rank]
        nb = slab.neighbours(rank, world, periodic)
        eng = FakeSlab(u, r0, n, lo_wall=nb.lower is None, hi_wall=nb.upper is None)
        slab.SlabRank(eng, nb, slab.DistTransport()).step(6)
        np.save(os.path.join(out_dir, f"r{rank}.npy"), eng.interior())
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("world", [2, 4])
@pytest.mark.parametrize("periodic", [True, False])
def test_gloo_ranks_match_one_slab(world, periodic):
    """World sizes 2 and 4 as gloo processes on CPU: the gathered slabs equal
    the one-slab run bit for bit."""
    ref, _ = run_local(initial(), 1, periodic)
    with tempfile.TemporaryDirectory() as d:
        port = 29500 + (os.getpid() % 1000) + 7 * world + (1 if periodic else 0)
        mp.start_processes(_gloo_worker, args=(world, periodic, port, d), nprocs=world, join=True,
                           start_method="spawn")
        got = np.concatenate([np.load(os.path.join(d, f"r{k}.npy")) for k in range(world)])
    assert np.array_equal(got, ref)


def _gloo_peer_worker(rank, world, periodic, port, out_dir):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        u = initial()
        r0, n = slab.split_rows(u.shape[0], world)[rank]
        nb = slab.neighbours(rank, world, periodic)
        eng = FakePeerSlab(u, r0, n, nb.lower is None, nb.upper is None, out_dir, rank)
        drv = slab.DistPeerSlabs(eng, nb)
        assert set(drv.mapped) == {s for s, o in ((abi.YLO, nb.lower), (abi.YHI, nb.upper)) if o is not None}
        drv.step(2)
        drv.step(4)
        np.save(os.path.join(out_dir, f"r{rank}.npy"), eng.interior())
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("world", [1, 2, 4])
@pytest.mark.parametrize("periodic", [True, False])
def test_gloo_peer_ranks_match_one_slab(world, periodic):
    """DistPeerSlabs over gloo ranks on CPU: each rank maps its neighbours'
    buffers (shared files standing in for CUDA IPC), stores its edge rows into
    their ghost rows during the stage, and orders the stages with token
    all-reduces; the gathered slabs equal the one-slab run bit for bit."""
    ref, _ = run_local(initial(), 1, periodic)
    with tempfile.TemporaryDirectory() as d:
        port = 29900 + (os.getpid() % 500) + 5 * world + (1 if periodic else 0)
        mp.start_processes(_gloo_peer_worker, args=(world, periodic, port, d), nprocs=world, join=True,
                           start_method="spawn")
        got = np.concatenate([np.load(os.path.join(d, f"r{k}.npy")) for k in range(world)])
    assert np.array_equal(got, ref)


# ---------------------------------------------------------------------------
# device slabs on one GPU
# ---------------------------------------------------------------------------
def _device_run(builder, n_slabs, steps, peers=False):
    from dev_field_efvm_b200.device import Context

    grid, params, u, ex = builder()
    per_y = grid.bc[abi.YLO].kind == abi.BC_PERIODIC
    if n_slabs == 0:  # the unsplit context
        c = Context(grid, params)
        c.upload(u)
        c.step(steps)
        return c.download(), c.solver_state(), ex, grid
    engines = []
    for r0, n in slab.split_rows(grid.ny, n_slabs):
        e = slab.DeviceSlab(grid, params, r0, n)
        e.ctx.upload(u[r0:r0 + n])
        engines.append(e)
    if peers:  # the exchange fused into the stage kernels, in two calls to check the stage chain
        drv = slab.PeerLocalSlabs(engines, per_y)
        drv.step(steps // 2)
        drv.step(steps - steps // 2)
    else:
        slab.LocalTransport(engines, per_y).step(steps)
    return np.concatenate([e.ctx.download() for e in engines]), engines[0].ctx.solver_state(), ex, grid


def _vortex(seam, muscl=True):
    return lambda: cases.vortex_case(64, periodic=True, muscl=muscl, mean=(1.0, 1.0), cfl=0.4, seam=seam)


def _vortex_fp32():
    """FP32 fluxes: the built-in stage form is the TMA-fed kernel, with the peer stores in its epilogue."""
    return cases.vortex_case(256, periodic=True, muscl=True, mean=(1.0, 1.0), cfl=0.4, precision=abi.PREC_FP32_FLUX,
                             ny=96)


def _channel():
    grid, params, u, ex = cases.poiseuille_case(ny=32, nx=8)
    params.reconstruction = abi.RECON_MUSCL
    return grid, params, u, ex


@pytest.mark.gpu
@pytest.mark.parametrize("name,builder,steps", [
    ("mpi_pulse", cases.mpi_pulse_case, 10),
    ("vortex_muscl_reference_seam", _vortex(abi.SEAM_REFERENCE), 8),
    ("vortex_muscl_true_periodic", _vortex(abi.SEAM_TRUE_PERIODIC), 8),
    ("channel_walls_viscous_muscl", _channel, 8),
])
def test_device_slabs_match_unsplit_context(name, builder, steps):
    ref, s_ref, ex, grid = _device_run(builder, 0, steps)
    for n in (1, 2, 3, 4):
        got, s, _, _ = _device_run(builder, n, steps)
        assert s.step == s_ref.step == steps
        assert s.time == s_ref.time, (n, s.time, s_ref.time)
        assert np.array_equal(got, ref), f"{name}: {n} slabs differ from the unsplit context"
    if name == "mpi_pulse":
        vol = (grid.hi[0] - grid.lo[0]) / grid.nx * (grid.hi[1] - grid.lo[1]) / grid.ny * (grid.hi[2] - grid.lo[2])
        m = cases.moments(ref, ex["x"], vol)
        assert np.all(np.isfinite(m)) and m[0] > 0


@pytest.mark.gpu
@pytest.mark.parametrize("name,builder,steps", [
    ("mpi_pulse", cases.mpi_pulse_case, 10),
    ("vortex_muscl_reference_seam", _vortex(abi.SEAM_REFERENCE), 8),
    ("vortex_muscl_true_periodic", _vortex(abi.SEAM_TRUE_PERIODIC), 8),
    ("channel_walls_viscous_muscl", _channel, 8),
    ("vortex_fp32_flux_tma_form", _vortex_fp32, 6),
])
def test_halo_peer_slabs_match_unsplit_context(name, builder, steps):
    """The exchange fused into the stage kernels (efvm_set_halo_peer): each
    stage stores its edge rows into the neighbours' ghost rows; 1-4 slabs equal
    the unsplit context bit for bit."""
    ref, s_ref, _, _ = _device_run(builder, 0, steps)
    for n in (1, 2, 3, 4):
        got, s, _, _ = _device_run(builder, n, steps, peers=True)
        assert s.step == s_ref.step == steps
        assert s.time == s_ref.time, (n, s.time, s_ref.time)
        assert np.array_equal(got, ref), f"{name}: {n} peer slabs differ from the unsplit context"


@pytest.mark.gpu
def test_halo_peer_argument_checks():
    from dev_field_efvm_b200.device import Context, EfvmError

    grid, params, u, ex = _channel()  # walls in y: the outer sides face no slab
    lo = Context(grid, params, rows=(0, 16))
    hi = Context(grid, params, rows=(16, 16))
    bufs, plane, rows = hi.state_buffers()
    assert rows == 16 and plane >= (rows + 4) * 8
    with pytest.raises(EfvmError):
        lo.set_halo_peer(abi.YLO, bufs, plane, rows)  # a wall side
    with pytest.raises(EfvmError):
        lo.set_halo_peer(abi.YHI, bufs, plane, 1)  # too few rows
    with pytest.raises(EfvmError):
        lo.set_halo_peer(abi.YHI, bufs, 8, rows)  # plane too small
    lo.set_halo_peer(abi.YHI, bufs, plane, rows)
    lo.set_halo_peer(abi.YHI, None)


@pytest.mark.gpu
def test_slab_refuses_cylinders_and_whole_step_calls():
    from dev_field_efvm_b200.device import Context, EfvmError

    grid, params, u, ex = cases.cylinder_case(110, 41)
    c = Context(grid, params, rows=(0, 20))
    with pytest.raises(EfvmError):
        c.set_cylinders(ex["cylinders"], ex["freestream"])
    with pytest.raises(EfvmError):
        c.step(1)
