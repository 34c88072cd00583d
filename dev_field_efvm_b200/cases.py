"""Case builders: the reference's case drivers and the benchmark workloads.

Each builder returns (grid, params, initial interior state (ny, nx, 5), extras)
for one of the reference's drivers (vortex gates, Sod, periodic pulse,
Poiseuille, DFG cylinder) or a benchmark configuration.  Plain numpy: these
generate synthetic inputs and exact solutions; nothing here runs a solver.
"""
from __future__ import annotations

import math

import numpy as np

from . import abi

R_GAS_AIR = 287.058


def prim_to_cons(rho, u, v, p, gamma=1.4):
    """IdealGas::prim_to_cons (crates/cfd_eos/src/lib.rs:55-59), vectorised."""
    rho = np.asarray(rho, dtype=np.float64)
    u = np.broadcast_to(np.asarray(u, dtype=np.float64), rho.shape)
    v = np.broadcast_to(np.asarray(v, dtype=np.float64), rho.shape)
    p = np.broadcast_to(np.asarray(p, dtype=np.float64), rho.shape)
    ke = 0.5 * rho * (u * u + v * v + 0.0 * 0.0)
    rho_e = p / (gamma - 1.0) + ke
    return np.stack([rho, rho * u, rho * v, np.zeros_like(rho), rho_e], -1)


def centroids(grid: abi.EfvmGrid):
    """Cell centres lo + ((i) + 0.5) * h of the interior (FIELD UniformMesh)."""
    hx = (grid.hi[0] - grid.lo[0]) / grid.nx
    hy = (grid.hi[1] - grid.lo[1]) / grid.ny
    x = grid.lo[0] + (np.arange(grid.nx, dtype=np.float64) + 0.5) * hx
    y = grid.lo[1] + (np.arange(grid.ny, dtype=np.float64) + 0.5) * hy
    return x, y


def vortex_state(v: abi.EfvmVortex, t: float, X, Y):
    """The Shu vortex closure (crates/cfd_solver/tests/isentropic_vortex_muscl_convergence.rs:48-64),
    vectorised, with the optional minimum-image displacement."""
    cx = v.cx0 + v.mean_u * t
    cy = v.cy0 + v.mean_v * t
    dx = X - cx
    dy = Y - cy
    if v.min_image:
        dx = dx - v.len_x * np.round(dx / v.len_x)
        dy = dy - v.len_y * np.round(dy / v.len_y)
    r2 = dx * dx + dy * dy
    f = np.exp(0.5 * (1.0 - r2))
    du = -v.beta / (2.0 * math.pi) * dy * f
    dv = v.beta / (2.0 * math.pi) * dx * f
    dtemp = -(v.gamma - 1.0) * v.beta * v.beta / (8.0 * v.gamma * math.pi ** 2) * np.exp(1.0 - r2)
    temp = 1.0 + dtemp
    rho = temp ** (1.0 / (v.gamma - 1.0))
    p = rho ** v.gamma
    return prim_to_cons(rho, v.mean_u + du, v.mean_v + dv, p, v.gamma)


def vortex_case(n: int, *, periodic: bool, mean=(0.5, 0.5), beta=5.0, centre=(5.0, 5.0), cfl=0.3,
                muscl=False, limiter=abi.LIMITER_MINMOD, precision=abi.PREC_FP64, seam=abi.SEAM_REFERENCE,
                domain=10.0, ny: int | None = None):
    """The isentropic-vortex cases.  periodic=False is the reference's own gate
    (crates/cfd_solver/tests/isentropic_vortex_*convergence.rs: zero-gradient x/y,
    slip z, dz = L/n); periodic=True is the periodic [0,L]^2 benchmark box."""
    ny = ny or n
    side = abi.BC_PERIODIC if periodic else abi.BC_SUPERSONIC_OUTFLOW
    bcs = {abi.XLO: side, abi.XHI: side, abi.YLO: side, abi.YHI: side,
           abi.ZLO: abi.BC_SLIP_WALL, abi.ZHI: abi.BC_SLIP_WALL}
    grid = abi.make_grid(n, ny, lo=(0.0, 0.0, 0.0), hi=(domain, domain * ny / n, domain / n), bcs=bcs)
    params = abi.make_params(cfl=cfl, reconstruction=abi.RECON_MUSCL if muscl else abi.RECON_FIRST_ORDER,
                             limiter=limiter, precision=precision, periodic_seam=seam)
    v = abi.make_vortex(beta=beta, cx0=centre[0], cy0=centre[1], mean_u=mean[0], mean_v=mean[1],
                        length=(domain, domain * ny / n), min_image=periodic)
    x, y = centroids(grid)
    X, Y = np.meshgrid(x, y)
    u = vortex_state(v, 0.0, X, Y)
    return grid, params, u, {"vortex": v}


def prim_to_cons3(rho, u, v, w, p, gamma=1.4):
    """IdealGas::prim_to_cons (crates/cfd_eos/src/lib.rs:55-59) with the z velocity."""
    rho = np.asarray(rho, dtype=np.float64)
    u, v, w, p = (np.broadcast_to(np.asarray(a, dtype=np.float64), rho.shape) for a in (u, v, w, p))
    ke = 0.5 * rho * (u * u + v * v + w * w)
    return np.stack([rho, rho * u, rho * v, rho * w, p / (gamma - 1.0) + ke], -1)


def vortex_tube_case(n: int, nz: int | None = None, *, mean=(1.0, 1.0, 1.0), beta=5.0, centre=(5.0, 5.0),
                     cfl=0.4, muscl=True, limiter=abi.LIMITER_MINMOD, seam=abi.SEAM_REFERENCE, domain=10.0,
                     amp=0.05, viscous=False, mu=1.0e-3):
    """A 3-D periodic box [0,L]^2 x [0, L nz/n]: the isentropic vortex of the 2-D
    benchmark (the reference's closure with the minimum image) along z, carried by
    the mean flow (mean_u, mean_v, mean_w), with the density modulated along z by
    1 + amp sin(2 pi z / Lz) at unchanged pressure and velocity (a contact wave,
    so the z faces carry flux).  Returns the grid, params, the [nz, ny, nx, 5]
    state and the 2-D vortex descriptor."""
    nz = nz or n
    lz = domain * nz / n
    P = abi.BC_PERIODIC
    bcs = {abi.XLO: P, abi.XHI: P, abi.YLO: P, abi.YHI: P, abi.ZLO: P, abi.ZHI: P}
    grid = abi.make_grid(n, n, lo=(0.0, 0.0, 0.0), hi=(domain, domain, lz), bcs=bcs, nz=nz)
    params = abi.make_params(cfl=cfl, reconstruction=abi.RECON_MUSCL if muscl else abi.RECON_FIRST_ORDER,
                             limiter=limiter, periodic_seam=seam, r_gas=1.0,
                             viscous=1 if viscous else 0, viscosity_model=abi.VISC_CONSTANT, mu=mu)
    v = abi.make_vortex(beta=beta, cx0=centre[0], cy0=centre[1], mean_u=mean[0], mean_v=mean[1],
                        length=(domain, domain), min_image=True)
    x, y = centroids(grid)
    X, Y = np.meshgrid(x, y)
    c2 = vortex_state(v, 0.0, X, Y)
    rho2 = c2[..., 0]
    u2, v2 = c2[..., 1] / rho2, c2[..., 2] / rho2
    p2 = (v.gamma - 1.0) * (c2[..., 4] - 0.5 * rho2 * (u2 * u2 + v2 * v2))
    z = (np.arange(nz, dtype=np.float64) + 0.5) * (lz / nz)
    mod = 1.0 + amp * np.sin(2.0 * math.pi * z / lz)
    rho3 = rho2[None] * mod[:, None, None]
    u = prim_to_cons3(rho3, u2[None], v2[None], mean[2], p2[None], v.gamma)
    return grid, params, u, {"vortex": v}


def sphere_drag_case(nx=144, ny=72, nz=72, *, rho=1.0, p=1.0e5, u_inf=56.1, reynolds=20.0, diameter=0.1,
                     cfl=0.3, muscl=False, sponge_x_start=0.5, sponge_sigma=2.0e4, n_markers=2000):
    """Resolved sphere drag at Re = 20 (examples/sphere_drag_validation/main.rs with
    config.toml): box [-0.3,0.9] x [-0.3,0.3]^2, D = 0.1 at the origin (D/dx = 12
    at 144x72x72), subsonic inflow, pressure outlet, symmetry sides, constant mu =
    rho u D / Re, first-order HLLC, RK3, CFL 0.3, uniform-freestream sponge over
    x in [0.5, 0.9] with sigma 2e4, 2000 Fibonacci markers."""
    r_gas = 287.058
    t_inf = p / (rho * r_gas)
    bcs = {abi.XLO: abi.make_bc(abi.BC_SUBSONIC_INFLOW, rho=rho, u=u_inf, v=0.0, w=0.0, t=t_inf),
           abi.XHI: abi.make_bc(abi.BC_PRESSURE_OUTLET, p=p),
           abi.YLO: abi.BC_SYMMETRY, abi.YHI: abi.BC_SYMMETRY, abi.ZLO: abi.BC_SYMMETRY, abi.ZHI: abi.BC_SYMMETRY}
    grid = abi.make_grid(nx, ny, lo=(-0.3, -0.3, -0.3), hi=(0.9, 0.3, 0.3), bcs=bcs, nz=nz)
    mu = rho * u_inf * diameter / reynolds
    params = abi.make_params(cfl=cfl, viscous=1, viscosity_model=abi.VISC_CONSTANT, mu=mu,
                             reconstruction=abi.RECON_MUSCL if muscl else abi.RECON_FIRST_ORDER,
                             sponge=1, sponge_x_start=sponge_x_start, sponge_x_end=0.9, sponge_sigma=sponge_sigma,
                             sponge_u_max=u_inf, sponge_rho=rho, sponge_p=p)
    u = prim_to_cons3(np.full((nz, ny, nx), rho), u_inf, 0.0, 0.0, np.full((nz, ny, nx), p))
    sphere = abi.make_sphere((0.0, 0.0, 0.0), 0.5 * diameter)
    q = 0.5 * rho * u_inf * u_inf * math.pi * (0.5 * diameter) ** 2
    return grid, params, u, {"spheres": [sphere], "freestream": u[0, 0, 0].copy(), "n_markers": n_markers, "q": q}


def cylinder_case(nx=440, ny=82, *, u_mean=50.0, rho=1.0, p=1.0e5, reynolds=20.0, cfl=0.3, muscl=False,
                  limiter=abi.LIMITER_MINMOD, sponge_sigma=1.0e4, sponge_x_start=1.4, precision=abi.PREC_FP64,
                  lz=0.041):
    """The DFG 2D-1 cylinder (examples/cylinder_drag_validation/main.rs:231-316 with
    config.toml).  Defaults are the reference's own passing run: 440x82, first-order
    HLLC, u_mean=50, p=1e5, CFL 0.3, sponge sigma=1e4."""
    L, H, D, cx, cy = 2.2, 0.41, 0.1, 0.2, 0.2
    mu = rho * u_mean * D / reynolds
    u_max = 1.5 * u_mean
    bcs = {abi.XLO: abi.BC_SUPERSONIC_OUTFLOW,
           abi.XHI: abi.make_bc(abi.BC_PRESSURE_OUTLET, p=p),
           abi.YLO: abi.BC_NO_SLIP_WALL, abi.YHI: abi.BC_NO_SLIP_WALL,
           abi.ZLO: abi.BC_SLIP_WALL, abi.ZHI: abi.BC_SLIP_WALL}
    grid = abi.make_grid(nx, ny, lo=(0.0, 0.0, 0.0), hi=(L, H, lz), bcs=bcs)
    params = abi.make_params(
        cfl=cfl, viscous=1, viscosity_model=abi.VISC_CONSTANT, mu=mu,
        reconstruction=abi.RECON_MUSCL if muscl else abi.RECON_FIRST_ORDER, limiter=limiter,
        precision=precision,
        parabolic_inflow=1, inflow_u_max=u_max, inflow_height=H, inflow_rho=rho,
        sponge=1, sponge_x_start=sponge_x_start, sponge_x_end=L, sponge_sigma=sponge_sigma,
        sponge_u_max=u_max, sponge_height=H, sponge_rho=rho, sponge_p=p)
    x, y = centroids(grid)
    X, Y = np.meshgrid(x, y)
    uy = 4.0 * u_max * Y * (H - Y) / (H * H)
    u = prim_to_cons(np.full_like(X, rho), uy, 0.0, np.full_like(X, p))
    freestream = prim_to_cons(np.array(rho), np.array(u_mean), 0.0, np.array(p))
    q = 0.5 * rho * u_mean * u_mean * D * lz
    extras = {"cylinders": [(cx, cy, 0.5 * D)], "freestream": freestream.reshape(5), "q": q, "mu": mu,
              "u_max": u_max}
    return grid, params, u, extras


def cylinder_baseline_case(nx=1100, ny=205, **kw):
    """The benchmark's cylinder: 1100x205 (D/dx=50), MUSCL, peak inflow 0.3
    (mean 0.2), freestream Mach 0.1 on the peak speed (a=3, rho=1,
    p=rho*a^2/gamma), Re=20 on the mean speed, CFL 0.4, sponge rescaled by the
    convective time (sigma*D/U_mean kept at the reference's 20 -> sigma=40)."""
    gamma = 1.4
    a = 3.0
    p = 1.0 * a * a / gamma
    args = dict(u_mean=0.2, rho=1.0, p=p, reynolds=20.0, cfl=0.4, muscl=True, sponge_sigma=40.0)
    args.update(kw)
    return cylinder_case(nx, ny, **args)


def sod_case(n: int, gamma: float = 1.4):
    """crates/cfd_solver/tests/sod_exact_convergence.rs:200-247."""
    bcs = {abi.YLO: abi.BC_SLIP_WALL, abi.YHI: abi.BC_SLIP_WALL, abi.ZLO: abi.BC_SLIP_WALL, abi.ZHI: abi.BC_SLIP_WALL}
    grid = abi.make_grid(n, 1, hi=(1.0, 0.01, 0.01), bcs=bcs)
    params = abi.make_params(cfl=0.4, gamma=gamma)
    x, _ = centroids(grid)
    left = prim_to_cons(np.array(1.0), np.array(0.0), 0.0, np.array(1.0e5), gamma)
    right = prim_to_cons(np.array(0.125), np.array(0.0), 0.0, np.array(1.0e4), gamma)
    u = np.where((x < 0.5)[:, None], left, right)[None, :, :]
    return grid, params, u, {"x": x}


def pulse_case(n: int, cfl=0.45):
    """examples/periodic_advected_pulse/main.rs:62-118 with its config.toml."""
    L = 1.0
    bcs = {abi.XLO: abi.BC_PERIODIC, abi.XHI: abi.BC_PERIODIC, abi.YLO: abi.BC_SLIP_WALL,
           abi.YHI: abi.BC_SLIP_WALL, abi.ZLO: abi.BC_SLIP_WALL, abi.ZHI: abi.BC_SLIP_WALL}
    grid = abi.make_grid(n, 1, hi=(L, L / n, L / n), bcs=bcs)
    params = abi.make_params(cfl=cfl)
    x, _ = centroids(grid)
    u = pulse_state(x, 0.0)[None, :, :]
    return grid, params, u, {"x": x}


def pulse_state(x, t, L=1.0, c0=0.85, sig=0.08, amp=0.2, gamma=1.4, vel=1.0, p=1.0):
    center = (c0 + vel * t) % L
    d = x - center
    d = d - L * np.round(d / L)
    rho = 1.0 + amp * np.exp(-0.5 * (d / sig) ** 2)
    return prim_to_cons(rho, np.full_like(rho, vel), 0.0, np.full_like(rho, p), gamma)


def poiseuille_case(ny=32, nx=3):
    """crates/cfd_solver/tests/poiseuille_channel_validation.rs:124-161 (2-D: the
    reference's nz=1 spanwise cell is the z extent here)."""
    H, rho0, T0, MU, GX = 1.0, 1.0, 300.0, 10.0, 160.0
    p0 = rho0 * R_GAS_AIR * T0
    bcs = {abi.YLO: abi.BC_NO_SLIP_WALL, abi.YHI: abi.BC_NO_SLIP_WALL, abi.ZLO: abi.BC_SLIP_WALL,
           abi.ZHI: abi.BC_SLIP_WALL}
    grid = abi.make_grid(nx, ny, hi=(1.0, H, 1.0), bcs=bcs)
    params = abi.make_params(cfl=0.3, viscous=1, viscosity_model=abi.VISC_CONSTANT, mu=MU, body_force_x=GX)
    u = prim_to_cons(np.full((ny, nx), rho0), np.zeros((ny, nx)), 0.0, np.full((ny, nx), p0))
    return grid, params, u, {"H": H, "mu": MU, "gx": GX, "rho": rho0, "t_final": 0.081}


def restart_pulse_case():
    """The restart test's pulse (crates/cfd_solver/tests/restart.rs:17-55): a
    density and pressure bump moving at 30 m/s through a 24-cell slip-walled box
    of air, first-order HLLC (Thornber), SSP-RK3, CFL 0.4, so both the fields
    and dt change every step."""
    n = 24
    bcs = {side: abi.BC_SLIP_WALL for side in (abi.XLO, abi.XHI, abi.YLO, abi.YHI, abi.ZLO, abi.ZHI)}
    grid = abi.make_grid(n, 1, hi=(1.0, 0.05, 0.05), bcs=bcs)
    params = abi.make_params(cfl=0.4)
    x, _ = centroids(grid)
    bump = np.exp(-(((x - 0.4) / 0.08) ** 2))
    rho = 1.0 + 0.5 * bump
    p = 1e5 * (1.0 + 0.8 * bump)
    u = prim_to_cons(rho, np.full_like(rho, 30.0), 0.0, p)[None, :, :]
    return grid, params, u, {"x": x}


def mpi_pulse_case():
    """The multi-rank check's pulse (tests/periodic_mpi.rs:24-80): 48x12 cells on
    [0,1] x [0,0.25], periodic in x and y, a density pulse starting near the
    high-x side so that it crosses the seam, gamma 1.4, R 1, first-order HLLC
    (Thornber), SSP-RK3, CFL 0.4."""
    bcs = {abi.XLO: abi.BC_PERIODIC, abi.XHI: abi.BC_PERIODIC, abi.YLO: abi.BC_PERIODIC,
           abi.YHI: abi.BC_PERIODIC, abi.ZLO: abi.BC_SLIP_WALL, abi.ZHI: abi.BC_SLIP_WALL}
    grid = abi.make_grid(48, 12, hi=(1.0, 0.25, 1.0 / 48.0), bcs=bcs)
    params = abi.make_params(cfl=0.4, r_gas=1.0)
    x, y = centroids(grid)
    X, _ = np.meshgrid(x, y)
    d = X - 0.9
    d = d - np.round(d)
    rho = 1.0 + 0.2 * np.exp(-0.5 * (d / 0.08) ** 2)
    u = prim_to_cons(rho, np.ones_like(rho), 0.0, np.ones_like(rho))
    return grid, params, u, {"x": X}


def moments(u: np.ndarray, x: np.ndarray, cell_volume: float) -> np.ndarray:
    """[sum rho V, sum rho^2 V, sum rho x V] (tests/periodic_mpi.rs:83-96)."""
    rho = u[..., 0]
    return np.array([np.sum(rho * cell_volume), np.sum(rho * rho * cell_volume), np.sum(rho * x * cell_volume)])


def riemann4_state(x, y, split, states, gamma=1.4):
    """Four constant quadrants around split = (xs, ys); states[q] = (rho, u, v, p)
    for q = 0: x<xs,y<ys; 1: x>=xs,y<ys; 2: x<xs,y>=ys; 3: x>=xs,y>=ys."""
    X, Y = np.meshgrid(x, y)
    q = (X >= split[0]).astype(int) + 2 * (Y >= split[1]).astype(int)
    st = np.asarray(states, dtype=np.float64)
    return prim_to_cons(st[q, 0], st[q, 1], st[q, 2], st[q, 3], gamma)


def batch_cases(n_cases=512, seed=2024, n_min=32, n_max=512, t_vortex=1.0, t_riemann=0.05,
                precision=abi.PREC_FP32_FLUX):
    """The batching workload: n_cases square grids with n log-uniform in
    [n_min, n_max]; even cases are isentropic vortices on the periodic [0,10]^2
    box (beta ~ U[1,5], centre ~ U[3,7]^2, mean flow (1,1)), odd cases
    four-quadrant Riemann problems on [0,1]^2 with zero-gradient (transmissive)
    boundaries (rho, p ~ U[0.1,2], u, v ~ U[-1,1], split point ~ U[0.3,0.7]^2).
    All share MUSCL-minmod + HLLC-Thornber, SSP-RK3, CFL 0.4 and `precision`;
    dz = L/n.  Returns (grids, params, states, t_stop, kinds)."""
    rng = np.random.default_rng(seed)
    params = abi.make_params(cfl=0.4, reconstruction=abi.RECON_MUSCL, limiter=abi.LIMITER_MINMOD, precision=precision)
    grids, states, t_stop, kinds = [], [], [], []
    out = abi.BC_SUPERSONIC_OUTFLOW
    for k in range(n_cases):
        n = int(round(np.exp(rng.uniform(np.log(n_min), np.log(n_max)))))
        if k % 2 == 0:
            beta = float(rng.uniform(1.0, 5.0))
            centre = (float(rng.uniform(3.0, 7.0)), float(rng.uniform(3.0, 7.0)))
            grid, _, u, _ = vortex_case(n, periodic=True, muscl=True, mean=(1.0, 1.0), beta=beta, centre=centre)
            grids.append(grid)
            states.append(u)
            t_stop.append(t_vortex)
            kinds.append("vortex")
        else:
            bcs = {abi.XLO: out, abi.XHI: out, abi.YLO: out, abi.YHI: out,
                   abi.ZLO: abi.BC_SLIP_WALL, abi.ZHI: abi.BC_SLIP_WALL}
            grid = abi.make_grid(n, n, hi=(1.0, 1.0, 1.0 / n), bcs=bcs)
            split = (float(rng.uniform(0.3, 0.7)), float(rng.uniform(0.3, 0.7)))
            quads = [(rng.uniform(0.1, 2.0), rng.uniform(-1.0, 1.0), rng.uniform(-1.0, 1.0), rng.uniform(0.1, 2.0))
                     for _ in range(4)]
            x, y = centroids(grid)
            grids.append(grid)
            states.append(riemann4_state(x, y, split, quads))
            t_stop.append(t_riemann)
            kinds.append("riemann")
    return grids, params, states, np.array(t_stop), kinds
