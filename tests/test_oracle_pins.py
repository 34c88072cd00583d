"""Pin the CPU oracle against the numbers the reference publishes for its own
runs (tests/golden/reference_published.json) and against the reference's
end-to-end App tests (crates/cfd_solver/src/tests.rs).  The oracle reproduces
the published per-run errors to the 7 printed digits, which pins the inferred
FIELD semantics (centroids, face order, ghost handling, CFL with the z term,
the no-clamp stop rule)."""
import json
import math
import os

import numpy as np
import pytest

import exact_riemann as er
from dev_field_efvm_b200 import abi
from dev_field_efvm_b200 import cases
from oracle import pyoracle as po

GOLD = json.load(open(os.path.join(os.path.dirname(__file__), "golden", "reference_published.json")))


def fitted_order(ns, errs):
    x, y = np.log(np.array(ns, float)), np.log(np.array(errs))
    m = len(x)
    return -(m * np.sum(x * y) - x.sum() * y.sum()) / (m * np.sum(x * x) - x.sum() ** 2)


def rel(a, b):
    return abs(a - b) / abs(b)


def same_printed(value, published):
    """The reference prints its errors with 7 significant digits ({:.6e})."""
    return f"{value:.6e}" == f"{published:.6e}"


def vortex_l1(n, muscl=False, limiter=abi.LIMITER_MINMOD):
    grid, params, u, ex = cases.vortex_case(n, periodic=False, muscl=muscl, limiter=limiter)
    c = po.OracleCase(grid, params)
    c.init_vortex(ex["vortex"])  # init_state_system: every raw cell from its centroid
    c.run_until(1.0)
    err = c.density_error(ex["vortex"])[0]
    assert np.all(c.download()[..., 0] > 0)
    return err


def test_vortex_first_order_matches_published_l1():
    g = GOLD["vortex_first_order_l1"]
    errs = [vortex_l1(n) for n in g["n"]]
    for e, ref in zip(errs, g["l1"]):
        assert same_printed(e, ref), (e, ref)
    assert abs(fitted_order(g["n"], errs) - g["fitted_order"]) < 5e-4
    assert errs[-1] < 2.0e-3


def test_periodic_pulse_matches_published_l1_and_mass_drift():
    g = GOLD["periodic_pulse"]
    errs, drifts = [], []
    for n in g["n"]:
        grid, params, u, ex = cases.pulse_case(n)
        c = po.OracleCase(grid, params)
        c.upload(u)
        m0 = c.total_mass()
        info = c.run_until(0.3)
        st = c.download()[0, :, 0]
        exact = cases.pulse_state(ex["x"], info.time)[:, 0]
        errs.append(np.mean(np.abs(st - exact)))
        drifts.append(abs((c.total_mass() - m0) / m0))
    for e, ref in zip(errs, g["l1"]):
        assert same_printed(e, ref), (e, ref)
    assert abs(fitted_order(g["n"], errs) - g["fitted_order"]) < 5e-4
    assert f"{max(drifts):.3e}" == f"{g['max_mass_drift']:.3e}"  # printed with 4 digits
    assert max(drifts) <= 1e-12


def sod_l1(n, gamma=1.4):
    grid, params, u, ex = cases.sod_case(n, gamma)
    c = po.OracleCase(grid, params)
    c.upload(u)
    info = c.run_until(6.0e-4)
    rho = c.download()[0, :, 0]
    ps, us = er.star(1.0, 0.0, 1e5, 0.125, 0.0, 1e4, 1.4)
    exact = np.array([er.density((x - 0.5) / info.time, 1.0, 0.0, 1e5, 0.125, 0.0, 1e4, 1.4, ps, us) for x in ex["x"]])
    return float(np.mean(np.abs(rho - exact))), c.total_mass()


def test_sod_matches_published_l1_and_wrong_gamma_fails():
    g = GOLD["sod_first_order_l1"]
    res = [sod_l1(n) for n in g["n"]]
    for (e, _), ref, n in zip(res, g["l1"], g["n"]):
        assert same_printed(e, ref), (e, ref)
        assert e < 0.25 / math.sqrt(n)
    e_bad, m_bad = sod_l1(100, 1.67)
    assert abs(e_bad - g["wrong_gamma_l1_n100_approx"]) < 5e-4
    assert e_bad > 0.25 / math.sqrt(100)
    for n in (200, 400):
        assert sod_l1(n, 1.67)[0] > 0.25 / math.sqrt(n)


def test_poiseuille_matches_analytic_parabola():
    grid, params, u, ex = cases.poiseuille_case()
    c = po.OracleCase(grid, params)
    c.upload(u)
    # the test drives single substages until t >= T_FINAL
    while c.solver_state().time < ex["t_final"]:
        c.substep()
    st = c.download()
    _, y = cases.centroids(grid)
    un = st[:, 1, 1] / st[:, 1, 0]
    H, mu, gx, rho = ex["H"], ex["mu"], ex["gx"], ex["rho"]
    u_an = lambda m: rho * gx / (2.0 * m) * y * (H - y)
    rel_l2 = lambda m: math.sqrt(np.mean((un - u_an(m)) ** 2)) / (rho * gx / (2.0 * m) * 0.25 * H * H)
    e_true, e_wrong = rel_l2(mu), rel_l2(1.5 * mu)
    assert e_true < GOLD["poiseuille_rel_l2"]["gate"]
    assert abs(e_true - GOLD["poiseuille_rel_l2"]["measured_approx"]) < 0.5e-4
    assert e_wrong > 10 * GOLD["poiseuille_rel_l2"]["gate"]


@pytest.mark.slow
def test_vortex_muscl_mc_is_second_order():
    g = GOLD["vortex_muscl_mc_gate"]
    errs = [vortex_l1(n, muscl=True, limiter=abi.LIMITER_MC) for n in g["n"]]
    orders = [math.log2(errs[k - 1] / errs[k]) for k in range(1, len(errs))]
    assert all(errs[k + 1] < errs[k] for k in range(len(errs) - 1))
    assert fitted_order(g["n"], errs) >= g["min_fitted_order"]
    assert orders[-1] >= g["min_finest_pair_order"]
    assert errs[-1] < g["max_finest_l1"]


# ---- crates/cfd_solver/src/tests.rs (3-D UniformMesh Apps on the oracle) ----
def mesh16x4x4(bcs=None):
    return abi.make_grid(16, 4, nz=4, hi=(1.0, 0.25, 0.25), bcs=bcs)


def uniform_u(grid, prim):
    c = po.prim_to_cons(prim)
    return np.broadcast_to(c, (grid.ny, grid.nx, 5)).copy()


class Raw3D:
    """Upload a 3-D initial condition through the raw array (the oracle's own layout)."""

    def __init__(self, grid, params, init):
        self.c = po.OracleCase(grid, params)
        n = self.c.L.oracle_raw_size(self.c.h)
        raw = np.zeros((n, 5))
        NX, NY = grid.nx + 4, grid.ny + 4
        h = [(grid.hi[a] - grid.lo[a]) / [grid.nx, grid.ny, grid.nz][a] for a in range(3)]
        for idx in range(n):
            i, j, k = idx % NX, (idx // NX) % NY, idx // (NX * NY)
            x = [grid.lo[0] + (i - 2 + 0.5) * h[0], grid.lo[1] + (j - 2 + 0.5) * h[1], grid.lo[2] + (k - 2 + 0.5) * h[2]]
            raw[idx] = init(x)
        self.c.L.oracle_set_raw_state(self.c.h, po._dp(raw))
        self.grid = grid

    def interior(self):
        raw = self.c.raw_state()
        g = self.grid
        NX, NY = g.nx + 4, g.ny + 4
        out = []
        for k in range(g.nz):
            for j in range(g.ny):
                for i in range(g.nx):
                    out.append(raw[(k + 2) * NX * NY + (j + 2) * NX + (i + 2)])
        return np.array(out)

    def mass(self):
        g = self.grid
        vol = np.prod([(g.hi[a] - g.lo[a]) / [g.nx, g.ny, g.nz][a] for a in range(3)])
        return float(np.sum(self.interior()[:, 0] * vol))


def test_uniform_flow_is_preserved():
    grid = mesh16x4x4()
    uu = po.prim_to_cons([1.0, 30.0, 0.0, 0.0, 100000.0, 348.4])
    r = Raw3D(grid, abi.make_params(flux_scheme=abi.FLUX_RUSANOV, integrator=abi.INTEGRATOR_EULER), lambda x: uu)
    for _ in range(25):
        r.c.substep()
    inner = r.interior()
    assert np.all(np.abs(inner[:, 0] - uu[0]) < 1e-9) and np.all(np.abs(inner[:, 1] - uu[1]) < 1e-6)
    assert np.all(np.abs(inner[:, 4] - uu[4]) < 1e-3)
    ss = r.c.solver_state()
    assert ss.step == 25 and np.isfinite(ss.dt) and ss.dt > 0


def test_sod_conserves_mass_and_evolves():
    grid = mesh16x4x4()
    left = po.prim_to_cons([1.0, 0, 0, 0, 100000.0, 348.4])
    right = po.prim_to_cons([0.125, 0, 0, 0, 10000.0, 278.7])
    r = Raw3D(grid, abi.make_params(flux_scheme=abi.FLUX_RUSANOV, integrator=abi.INTEGRATOR_EULER, cfl=0.3),
              lambda x: left if x[0] < 0.5 else right)
    m0 = r.mass()
    mid0 = r.interior()[(2 * 4 + 2) * 16 + 8].copy()
    for _ in range(15):
        r.c.substep()
    assert abs(r.mass() - m0) / m0 < 1e-6
    mid1 = r.interior()[(2 * 4 + 2) * 16 + 8]
    assert np.all(r.interior()[:, 0] > 0)
    assert abs(mid1[1] - mid0[1]) > 1.0


def test_closed_box_conserves_mass_under_slip_walls():
    bcs = {s: abi.BC_SLIP_WALL for s in range(6)}
    grid = mesh16x4x4(bcs)
    center = [0.5, 0.125, 0.125]

    def init(x):
        r2 = sum((x[d] - center[d]) ** 2 for d in range(3))
        p = 3e5 if r2 < 0.15 * 0.15 else 1e5
        return po.prim_to_cons([1.0, 0, 0, 0, p, p / 287.058])

    r = Raw3D(grid, abi.make_params(flux_scheme=abi.FLUX_RUSANOV, integrator=abi.INTEGRATOR_EULER, cfl=0.3), init)
    m0 = r.mass()
    for _ in range(30):
        r.c.substep()
    assert abs(r.mass() - m0) / m0 < 1e-9


def test_viscous_operator_matches_laplacian():
    a = 10.0
    t0 = 100000.0 / 287.058
    grid = abi.make_grid(6, 8, nz=4, hi=(1.0, 1.0, 0.5))

    def run(viscous):
        r = Raw3D(grid, abi.make_params(flux_scheme=abi.FLUX_RUSANOV, integrator=abi.INTEGRATOR_EULER, cfl=0.3,
                                        viscous=1 if viscous else 0),
                  lambda x: po.prim_to_cons([1.0, a * x[1] * x[1], 0.0, 0.0, 100000.0, t0]))
        cell = (2 * 8 + 4) * 6 + 3
        before = r.interior()[cell, 1]
        r.c.substep()
        dt = r.c.solver_state().dt
        return (r.interior()[cell, 1] - before) / dt

    visc = run(True) - run(False)
    expected = po.sutherland(t0) * 2.0 * a
    assert abs(visc - expected) / abs(expected) < 1e-4


def test_colored_parallel_oracle_agrees_with_serial():
    grid, params, u, ex = cases.vortex_case(48, periodic=True, muscl=True, mean=(1.0, 1.0))
    a = po.OracleCase(grid, params)
    b = po.OracleCase(grid, params, parallel=True)
    for c in (a, b):
        c.upload(u)
        c.step(5)
    ua, ub = a.download(), b.download()
    scale = np.max(np.abs(ua), axis=(0, 1)) + 1e-300
    assert np.max(np.abs(ua - ub) / scale) < 1e-13
