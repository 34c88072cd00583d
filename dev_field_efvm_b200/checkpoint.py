"""Checkpoint and restart of a running case.

A checkpoint holds what the reference's grass_io::save_app / restore_app pair
carries for a CFD case (crates/cfd_solver/tests/restart.rs:1-3,86-105): the
conserved fields CfdState.u and the solver clock SolverState {dt, time, step,
rk_stage}.  It is taken at a step boundary (rk_stage == 0), where nothing else
carries from one step to the next: the next step's dt is recomputed from the
restored fields by the same wave-speed maximum the running case would use, and
the IBM mirror and force buffers are rebuilt within each step.  A restored
context therefore continues bit for bit.

The file format is a NumPy .npz archive: `u` (ny, nx, 5) FP64 in the order
(rho, rho_u, rho_v, rho_w, rho_e), and the FP64 scalars `dt`, `time` plus the
integers `step`, `rk_stage`, `completed_full_step`.

Works with any context that has download, upload, apply_geometry,
solver_state and set_solver_state (the device Context).
"""
from __future__ import annotations

import numpy as np

from . import abi

FORMAT_VERSION = 1


def snapshot(ctx) -> dict:
    """The state of `ctx` at a step boundary, as host arrays."""
    s = ctx.solver_state()
    if s.rk_stage != 0:
        raise ValueError(f"checkpoint needs a step boundary (rk_stage == 0), got rk_stage {s.rk_stage}")
    return {
        "format_version": np.int64(FORMAT_VERSION),
        "u": np.array(ctx.download(), dtype=np.float64, copy=True),
        "dt": np.float64(s.dt),
        "time": np.float64(s.time),
        "step": np.uint64(s.step),
        "rk_stage": np.int32(s.rk_stage),
        "completed_full_step": np.int32(s.completed_full_step),
    }


def restore(ctx, snap: dict) -> None:
    """Load a snapshot into `ctx` (same grid, parameters and cylinders as the
    one saved; set the cylinders before calling this).

    A fresh context re-seeds the cells that turn solid when its cylinders are
    first applied (refresh_cylinder_mask, crates/cfd_ibm/src/lib.rs:155-183).
    The reference's restore brings the solid mask back with the fields, so
    nothing is re-seeded after it: restore() therefore applies the geometry to
    the loaded fields and then loads them again over the re-seeded cells."""
    if int(snap["format_version"]) != FORMAT_VERSION:
        raise ValueError(f"unknown checkpoint format {int(snap['format_version'])}")
    u = np.ascontiguousarray(snap["u"], dtype=np.float64)
    ctx.upload(u)
    ctx.apply_geometry()
    ctx.upload(u)
    s = abi.EfvmSolverState()
    s.dt = float(snap["dt"])
    s.time = float(snap["time"])
    s.step = int(snap["step"])
    s.rk_stage = int(snap["rk_stage"])
    s.completed_full_step = int(snap["completed_full_step"])
    ctx.set_solver_state(s)


def save(ctx, path: str) -> None:
    """Write a checkpoint of `ctx` to `path` (.npz)."""
    np.savez(path, **snapshot(ctx))


def load(ctx, path: str) -> None:
    """Restore `ctx` from a checkpoint file written by save()."""
    with np.load(path) as f:
        restore(ctx, {k: f[k] for k in f.files})
