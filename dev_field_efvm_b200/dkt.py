"""Drafting-kissing-tumbling: two discs settling in a closed box, the reference's
resolved-FSI example (examples/dkt_sedimentation/main.rs with config.toml),
driven through the library's moving-disc IBM (efvm_set_discs).

The fluid runs on the engine (a device Context, or the CPU oracle for parity
checks).  Once per completed RK3 step this driver does what the example's
Output-phase fsi_step_system does (main.rs:332-402): read each disc's marker
load and torque (efvm_body_loads), add the reduced-gravity buoyant weight and
the soft-sphere contact springs (contact_forces, main.rs:289-330), advance the
velocities, positions and spins semi-implicitly with the step's dt, and hand the
new discs back (efvm_set_discs) before the next step.  The phase analysis and
its gates are main.rs:620-720.

    python -m dev_field_efvm_b200.dkt [--substeps N]
"""
from __future__ import annotations

import argparse
import json
import math
import time
from dataclasses import dataclass, field

import numpy as np

from . import abi

R_GAS = 287.058

# examples/dkt_sedimentation/config.toml
CONFIG = dict(nx=120, ny=390, hi=(0.024, 0.078, 0.0002), rho=1.0, p=1.0e5, diameter=0.002, density_ratio=1.5,
              u_grav=40.0, re_settle=40.0, n_theta=100, lead=(0.012, 0.060), trail=(0.0120160, 0.0632),
              range_cells=3.0, stiffness_scale=150.0, cfl=0.3, substeps=62000, draft_close_frac=0.4,
              kiss_gap_cells=5.0, tumble_lateral_d=0.5, max_mach=0.30)


@dataclass
class Disc:
    centre: list
    vel: list
    omega: float
    radius: float
    mass: float
    inertia: float


@dataclass
class Fsi:
    rho_f: float
    g: float
    lz: float
    n_theta: int
    contact_range: float
    k_n: float
    walls: tuple  # x_lo, x_hi, y_lo, y_hi


@dataclass
class Trace:
    t: list = field(default_factory=list)
    y0: list = field(default_factory=list)
    y1: list = field(default_factory=list)
    x0: list = field(default_factory=list)
    x1: list = field(default_factory=list)
    gap: list = field(default_factory=list)


def setup(cfg=CONFIG):
    """Grid, params, initial state, discs, driver parameters and the freestream
    (main.rs:450-540)."""
    d = cfg["diameter"]
    r = 0.5 * d
    s = cfg["density_ratio"]
    g = cfg["u_grav"] ** 2 / ((s - 1.0) * d)
    nu = cfg["u_grav"] * d / cfg["re_settle"]
    mu = cfg["rho"] * nu
    rho_p = s * cfg["rho"]
    nx, ny = cfg["nx"], cfg["ny"]
    hi = cfg["hi"]
    dx = hi[0] / nx
    lz = hi[2]
    bcs = {abi.XLO: abi.BC_NO_SLIP_WALL, abi.XHI: abi.BC_NO_SLIP_WALL, abi.YLO: abi.BC_NO_SLIP_WALL,
           abi.YHI: abi.BC_NO_SLIP_WALL, abi.ZLO: abi.BC_SLIP_WALL, abi.ZHI: abi.BC_SLIP_WALL}
    grid = abi.make_grid(nx, ny, lo=(0.0, 0.0, 0.0), hi=hi, bcs=bcs)
    params = abi.make_params(cfl=cfg["cfl"], viscous=1, viscosity_model=abi.VISC_CONSTANT, mu=mu,
                             reconstruction=abi.RECON_FIRST_ORDER)
    gm1 = params.gamma - 1.0
    fs = np.array([cfg["rho"], 0.0, 0.0, 0.0, cfg["p"] / gm1])
    u = np.broadcast_to(fs, (ny, nx, 5)).copy()
    vol = math.pi * r * r * lz
    mass = rho_p * vol
    inertia = 0.5 * mass * r * r
    discs = [Disc(list(cfg["lead"]), [0.0, 0.0], 0.0, r, mass, inertia),
             Disc(list(cfg["trail"]), [0.0, 0.0], 0.0, r, mass, inertia)]
    w_net = (rho_p - cfg["rho"]) * vol * g
    fsi = Fsi(rho_f=cfg["rho"], g=g, lz=lz, n_theta=max(cfg["n_theta"], 16),
              contact_range=cfg["range_cells"] * dx, k_n=cfg["stiffness_scale"] * w_net / dx,
              walls=(0.0, hi[0], 0.0, hi[1]))
    return grid, params, u, discs, fsi, fs


def efvm_discs(discs):
    return [abi.EfvmDisc(d.centre[0], d.centre[1], d.radius, d.vel[0], d.vel[1], d.omega) for d in discs]


def contact_forces(discs, p: Fsi):
    """Linear-spring contact between the discs and against the four walls inside
    the contact band (contact_forces, main.rs:293-330)."""
    f = [[0.0, 0.0], [0.0, 0.0]]
    if len(discs) == 2:
        a, b = discs
        dx = b.centre[0] - a.centre[0]
        dy = b.centre[1] - a.centre[1]
        dist = max(math.sqrt(dx * dx + dy * dy), 1e-12)
        overlap = (a.radius + b.radius + p.contact_range) - dist
        if overlap > 0.0:
            nx, ny = dx / dist, dy / dist
            fmag = p.k_n * overlap
            f[0][0] -= fmag * nx
            f[0][1] -= fmag * ny
            f[1][0] += fmag * nx
            f[1][1] += fmag * ny
    x_lo, x_hi, y_lo, y_hi = p.walls
    for i, d in enumerate(discs):
        gaps = ((d.centre[0] - x_lo - d.radius, (1.0, 0.0)), (x_hi - d.centre[0] - d.radius, (-1.0, 0.0)),
                (d.centre[1] - y_lo - d.radius, (0.0, 1.0)), (y_hi - d.centre[1] - d.radius, (0.0, -1.0)))
        for gap, dr in gaps:
            overlap = p.contact_range - gap
            if overlap > 0.0:
                fmag = p.k_n * overlap
                f[i][0] += fmag * dr[0]
                f[i][1] += fmag * dr[1]
    return f


def fsi_update(discs, loads: np.ndarray, dt: float, p: Fsi) -> None:
    """fsi_step_system's rigid-body update (main.rs:368-385): fluid load (pressure
    + viscous) plus contact, minus the buoyant weight; velocity, then position,
    then spin from the torque's z component."""
    contact = contact_forces(discs, p)
    for i, d in enumerate(discs):
        ld = loads[i]
        f_fluid = ld[0:3] + ld[3:6]
        v = math.pi * d.radius * d.radius * p.lz
        rho_p = d.mass / v
        w_net = (rho_p - p.rho_f) * v * p.g
        fx = f_fluid[0] + contact[i][0]
        fy = f_fluid[1] - w_net + contact[i][1]
        d.vel[0] += fx / d.mass * dt
        d.vel[1] += fy / d.mass * dt
        d.centre[0] += d.vel[0] * dt
        d.centre[1] += d.vel[1] * dt
        d.omega += ld[8] / d.inertia * dt


def max_mach(u: np.ndarray, gamma: float = 1.4) -> float:
    rho = u[..., 0]
    ok = np.isfinite(rho) & (rho > 0)
    rho = np.where(ok, rho, 1.0)
    vel = u[..., 1:4] / rho[..., None]
    ke = 0.5 * rho * np.sum(vel * vel, axis=-1)
    p = (gamma - 1.0) * (u[..., 4] - ke)
    a = np.sqrt(np.maximum(gamma * p / rho, 1e-300))
    m = np.sqrt(np.sum(vel * vel, axis=-1)) / a
    return float(np.max(np.where(ok, m, 0.0)))


def run(engine, discs, fsi: Fsi, fs, steps: int, mach_every: int = 200):
    """Advance `steps` whole RK3 steps with the driver between them.  Returns the
    trace and the largest Mach number over the field (solid cells included) after
    every `mach_every`-th substep, counting substeps from 0 as the reference's
    run loop does (main.rs:567-582); a step holding such a substep runs as three
    substeps so that the field is read at the same instant."""
    engine.set_discs(efvm_discs(discs), fs, fsi.n_theta)
    tr = Trace()
    mach = 0.0
    for step in range(steps):
        due = [r for r in range(3) if (3 * step + r) % mach_every == 0]
        if due:
            for r in range(3):
                engine.substep()
                if r in due:
                    mach = max(mach, max_mach(engine.download()))
        else:
            engine.step(1)
        st = engine.solver_state()
        loads = engine.body_loads(len(discs))
        fsi_update(discs, loads, st.dt, fsi)
        engine.set_discs(efvm_discs(discs), fs, fsi.n_theta)
        a, b = discs
        gap = math.hypot(b.centre[0] - a.centre[0], b.centre[1] - a.centre[1]) - a.radius - b.radius
        tr.t.append(st.time)
        tr.y0.append(a.centre[1])
        tr.y1.append(b.centre[1])
        tr.x0.append(a.centre[0])
        tr.x1.append(b.centre[0])
        tr.gap.append(gap)
    return tr, mach


def analyse(tr: Trace, mach: float, cfg=CONFIG) -> dict:
    """The DKT phase analysis and gates (main.rs:620-720)."""
    d = cfg["diameter"]
    dx = cfg["hi"][0] / cfg["nx"]
    gap = np.asarray(tr.gap)
    kiss_i = int(np.argmin(gap))
    kiss_gap = float(gap[kiss_i])
    gap_max_pre = float(np.max(gap[:kiss_i + 1]))
    draft_closed = (gap_max_pre - kiss_gap) / gap_max_pre
    y0, y1, x0, x1 = (np.asarray(a) for a in (tr.y0, tr.y1, tr.x0, tr.x1))
    caught_up = bool(np.any((y1[1:kiss_i + 1] - y1[:kiss_i]) < (y0[1:kiss_i + 1] - y0[:kiss_i]) - 1e-9))
    tumble = float(np.max(np.abs(x1[kiss_i:] - x0[kiss_i:]))) / d
    overtook = bool(np.any(y1[kiss_i:] < y0[kiss_i:]))
    res = {"draft_closed": draft_closed, "trailing_caught_up": caught_up, "kiss_gap_cells": kiss_gap / dx,
           "t_kiss": float(tr.t[kiss_i]), "tumble_d": tumble, "overtook": overtook, "max_mach": mach}
    res["pass_draft"] = draft_closed >= cfg["draft_close_frac"] and caught_up
    res["pass_kiss"] = kiss_gap / dx <= cfg["kiss_gap_cells"]
    res["pass_tumble"] = tumble >= cfg["tumble_lateral_d"] and overtook
    res["pass_mach"] = mach <= cfg["max_mach"]
    res["pass"] = res["pass_draft"] and res["pass_kiss"] and res["pass_tumble"] and res["pass_mach"]
    return res


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--substeps", type=int, default=CONFIG["substeps"])
    args = ap.parse_args()
    from .device import Context
    grid, params, u, discs, fsi, fs = setup()
    c = Context(grid, params)
    c.upload(u)
    t0 = time.perf_counter()
    tr, mach = run(c, discs, fsi, fs, args.substeps // 3)
    res = analyse(tr, mach)
    res["wall_s"] = time.perf_counter() - t0
    print(json.dumps(res))


if __name__ == "__main__":
    main()
