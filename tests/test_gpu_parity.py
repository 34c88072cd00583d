"""Parity of the CUDA path (through the C-ABI) with the CPU oracle.

Tolerance: FP64 path within 1e-12 of the oracle per cell after one RK3 step,
relative to max(|oracle|, 1e-3 * max_cells |oracle|) of each conserved
variable (the floor keeps momenta that cross zero meaningful); 1e-10 after
tens of steps.  The CUDA kernels may fuse multiply-adds, so bit equality is not
expected; the integer/geometry parts (solid mask, ghost list, step counts) are
compared exactly.  FP32-flux results are compared with a stated looser bound.
"""
import json
import math
import os

import numpy as np
import pytest

import exact_riemann as er
from dev_field_efvm_b200 import abi
from dev_field_efvm_b200.device import Context, EfvmError
from dev_field_efvm_b200 import cases
from oracle import pyoracle as po

pytestmark = pytest.mark.gpu

GOLD = json.load(open(os.path.join(os.path.dirname(__file__), "golden", "reference_published.json")))
TOL_ONE_STEP = 1e-12
TOL_MANY_STEPS = 1e-10


def rel_err(g, o):
    """max |g - o| / max(|o|, 1e-3 * scale) over cells and variables; the scale of
    rho and rho_e is their max magnitude, that of both momenta max sqrt(rho * rho_e)
    (the momentum unit of the state's total energy, so a component that is only
    round-off, like rho_v in a channel, is judged against the flow, not itself)."""
    mom = float(np.max(np.sqrt(np.abs(o[..., 0] * o[..., 4]))))
    scale = np.array([np.max(np.abs(o[..., 0])), mom, mom, 1.0, np.max(np.abs(o[..., 4]))])
    denom = np.maximum(np.abs(o), 1e-3 * np.maximum(scale, 1e-300))
    return float(np.max(np.abs(g - o) / denom))


def pair(grid, params, u, cyl=None):
    o = po.OracleCase(grid, params)
    d = Context(grid, params)
    if cyl is not None:
        o.set_cylinders(cyl["cylinders"], cyl["freestream"])
        d.set_cylinders(cyl["cylinders"], cyl["freestream"])
    o.upload(u)
    d.upload(u)
    return o, d


def vortex_periodic(n=64, seam=abi.SEAM_REFERENCE, limiter=abi.LIMITER_MINMOD, precision=abi.PREC_FP64):
    return cases.vortex_case(n, periodic=True, muscl=True, limiter=limiter, mean=(1.0, 1.0), cfl=0.4,
                             seam=seam, precision=precision)


@pytest.mark.parametrize("seam", [abi.SEAM_REFERENCE, abi.SEAM_TRUE_PERIODIC])
def test_periodic_vortex_muscl_minmod_one_and_twenty_steps(seam):
    grid, params, u, ex = vortex_periodic(64, seam)
    o, d = pair(grid, params, u)
    assert abs(o.cfl() - d.cfl()) <= 1e-14 * o.cfl()
    o.step(1)
    d.step(1)
    assert rel_err(d.download(), o.download()) < TOL_ONE_STEP
    so, sd = o.solver_state(), d.solver_state()
    assert sd.step == so.step == 1 and abs(sd.time - so.time) <= 1e-15 and abs(sd.dt - so.dt) <= 1e-15 * so.dt
    o.step(19)
    d.step(19)
    assert rel_err(d.download(), o.download()) < TOL_MANY_STEPS


@pytest.mark.parametrize("scheme,muscl,limiter", [
    (abi.FLUX_HLLC, False, abi.LIMITER_MINMOD),
    (abi.FLUX_HLLC, True, abi.LIMITER_MC),
    (abi.FLUX_RUSANOV, True, abi.LIMITER_MINMOD),
    (abi.FLUX_HLLC_TEXTBOOK, True, abi.LIMITER_MC),
])
def test_outflow_vortex_schemes(scheme, muscl, limiter):
    grid, params, u, ex = cases.vortex_case(48, periodic=False, muscl=muscl, limiter=limiter)
    params.flux_scheme = scheme
    o, d = pair(grid, params, u)
    o.step(1)
    d.step(1)
    assert rel_err(d.download(), o.download()) < TOL_ONE_STEP
    o.step(15)
    d.step(15)
    assert rel_err(d.download(), o.download()) < TOL_MANY_STEPS


def test_substep_api_matches_oracle_stage_by_stage():
    grid, params, u, ex = vortex_periodic(40)
    o, d = pair(grid, params, u)
    for k in range(7):  # crosses a step boundary mid-way
        o.substep()
        d.substep()
        assert rel_err(d.download(), o.download()) < TOL_ONE_STEP, k
        assert d.solver_state().rk_stage == o.solver_state().rk_stage


def test_reference_vortex_gate_reproduces_published_l1_on_gpu():
    g = GOLD["vortex_first_order_l1"]
    for n, ref in zip(g["n"][:2], g["l1"][:2]):
        grid, params, u, ex = cases.vortex_case(n, periodic=False)
        d = Context(grid, params)
        d.upload(u)
        info = d.run_until(1.0)
        e = d.density_error(ex["vortex"])[0]
        assert f"{e:.6e}" == f"{ref:.6e}", (n, e, ref)
        o = po.OracleCase(grid, params)
        o.upload(u)
        oi = o.run_until(1.0)
        assert info.steps_done == oi.steps_done


def test_vortex_muscl_mc_second_order_gate_on_gpu():
    """The reference's MUSCL convergence gate (isentropic vortex, outflow, MC
    limiter, N = 40/80/160 to t = 1; crates/cfd_solver/tests/
    isentropic_vortex_muscl_convergence.rs:146-192) on the CUDA path: errors fall,
    the fitted and finest-pair orders reach 1.8, the finest L1 stays under its
    bound, and the two coarser errors agree with the oracle's."""
    g = GOLD["vortex_muscl_mc_gate"]
    errs = []
    for n in g["n"]:
        grid, params, u, ex = cases.vortex_case(n, periodic=False, muscl=True, limiter=abi.LIMITER_MC)
        d = Context(grid, params)
        d.upload(u)
        info = d.run_until(1.0)
        assert np.all(d.download()[..., 0] > 0)
        errs.append(d.density_error(ex["vortex"])[0])
        if n <= 80:
            o = po.OracleCase(grid, params)
            o.upload(u)
            oi = o.run_until(1.0)
            assert info.steps_done == oi.steps_done
            assert abs(errs[-1] - o.density_error(ex["vortex"])[0]) <= 1e-9 * errs[-1]
    x, y = np.log(np.array(g["n"], float)), np.log(np.array(errs))
    m = len(x)
    fitted = -(m * np.sum(x * y) - x.sum() * y.sum()) / (m * np.sum(x * x) - x.sum() ** 2)
    assert all(errs[k + 1] < errs[k] for k in range(len(errs) - 1))
    assert fitted >= g["min_fitted_order"]
    assert math.log2(errs[-2] / errs[-1]) >= g["min_finest_pair_order"]
    assert errs[-1] < g["max_finest_l1"]


def test_sod_and_periodic_pulse_reproduce_published_numbers_on_gpu():
    gs = GOLD["sod_first_order_l1"]
    grid, params, u, ex = cases.sod_case(100)
    d = Context(grid, params)
    d.upload(u)
    info = d.run_until(6.0e-4)
    rho = d.download()[0, :, 0]
    ps, us = er.star(1.0, 0.0, 1e5, 0.125, 0.0, 1e4, 1.4)
    exact = np.array([er.density((x - 0.5) / info.time, 1.0, 0.0, 1e5, 0.125, 0.0, 1e4, 1.4, ps, us) for x in ex["x"]])
    assert f"{np.mean(np.abs(rho - exact)):.6e}" == f"{gs['l1'][0]:.6e}"
    gp = GOLD["periodic_pulse"]
    grid, params, u, ex = cases.pulse_case(40)
    d = Context(grid, params)
    d.upload(u)
    m0 = d.total_mass()
    info = d.run_until(0.3)
    st = d.download()[0, :, 0]
    err = np.mean(np.abs(st - cases.pulse_state(ex["x"], info.time)[:, 0]))
    assert f"{err:.6e}" == f"{gp['l1'][0]:.6e}"
    assert abs(d.total_mass() - m0) / m0 <= 1e-12


@pytest.mark.parametrize("muscl", [False, True])
def test_cylinder_ibm_viscous_parity(muscl):
    grid, params, u, ex = cases.cylinder_case(110, 41, muscl=muscl)
    o, d = pair(grid, params, u, ex)
    assert abs(d.cfl() - o.cfl()) <= 1e-14 * o.cfl()
    o.step(1)
    d.step(1)
    assert np.array_equal(d.solid_mask(), o.mask())
    assert d.ibm_counts() == o.ibm_counts()
    assert rel_err(d.download(), o.download()) < TOL_ONE_STEP
    fo, fd = o.marker_force(), d.marker_force()
    assert np.max(np.abs(fd - fo)) <= 1e-11 * np.max(np.abs(fo))
    wo, wd = o.wall_force(), d.wall_force()
    assert np.max(np.abs(wd - wo)) <= 1e-11 * np.max(np.abs(wo))
    oi, oh = o.step(10, history=True)
    di, dh = d.step(10, history=True)
    assert rel_err(d.download(), o.download()) < TOL_MANY_STEPS
    assert dh.shape == oh.shape == (30, 6)
    assert np.max(np.abs(dh - oh)) <= 1e-10 * np.max(np.abs(oh))


def test_poiseuille_viscous_body_force_parity():
    grid, params, u, ex = cases.poiseuille_case()
    o, d = pair(grid, params, u)
    for _ in range(30):
        o.substep()
        d.substep()
    assert rel_err(d.download(), o.download()) < TOL_MANY_STEPS


def test_fp32_flux_path_tracks_fp64():
    grid, params, u, ex = vortex_periodic(64, precision=abi.PREC_FP32_FLUX)
    o = po.OracleCase(grid, abi.make_params(**{f: getattr(params, f) for f, _ in abi.EfvmParams._fields_
                                                 if f != "precision"}))
    d = Context(grid, params)
    o.upload(u)
    d.upload(u)
    o.step(10)
    d.step(10)
    # FP32 face states and fluxes: ~1e-7 relative per flux, accumulated in FP64
    assert rel_err(d.download(), o.download()) < 5e-5


def test_translation_invariance_at_full_size_true_periodic():
    """Size-independent property at the 4096^2 benchmark size: on a periodic
    box with the conservative seam the step commutes with a shift of the grid
    by whole cells, bit for bit."""
    n = 4096
    grid, params, u, ex = cases.vortex_case(n, periodic=True, muscl=True, mean=(1.0, 1.0), cfl=0.4,
                                            seam=abi.SEAM_TRUE_PERIODIC)
    params.fixed_dt = 2.0e-3
    a = Context(grid, params)
    a.upload(u)
    a.step(2)
    ua = a.download()
    a.close()
    b = Context(grid, params)
    b.upload(np.roll(u, (37, 411), axis=(0, 1)))
    b.step(2)
    ub = b.download()
    assert np.array_equal(np.roll(ua, (37, 411), axis=(0, 1)), ub)


def test_mass_conservation_true_periodic_full_size():
    grid, params, u, ex = cases.vortex_case(1024, periodic=True, muscl=True, mean=(1.0, 1.0), cfl=0.4,
                                            seam=abi.SEAM_TRUE_PERIODIC)
    d = Context(grid, params)
    d.upload(u)
    m0 = d.total_mass()
    d.step(50)
    assert abs(d.total_mass() - m0) / m0 < 1e-13


def test_uniform_flow_stays_uniform_on_cylinder_channel_size():
    grid, params, u, ex = cases.cylinder_baseline_case()
    params.parabolic_inflow = 0
    params.sponge = 0
    params.viscous = 0
    bcs_uniform = cases.prim_to_cons(np.ones((grid.ny, grid.nx)), 0.2, 0.1, np.full((grid.ny, grid.nx), 6.4))
    for s in range(4):
        grid.bc[s] = abi.make_bc(abi.BC_PERIODIC)
    d = Context(grid, params)
    d.upload(bcs_uniform)
    d.step(5)
    out = d.download()
    assert np.max(np.abs(out - bcs_uniform)) <= 1e-13 * np.max(np.abs(bcs_uniform))


def test_nonphysical_state_is_reported():
    """Fault injection on the host: a negative density in the uploaded state."""
    grid, params, u, ex = vortex_periodic(32)
    bad = u.copy()
    bad[5, 7, 0] = -1.0
    d = Context(grid, params)
    d.upload(bad)
    with pytest.raises(EfvmError) as e:
        d.step(2)
    assert e.value.code == abi.ERR_NONPHYSICAL


def test_t_stop_step_count_matches_oracle():
    grid, params, u, ex = cases.vortex_case(40, periodic=False)
    o, d = pair(grid, params, u)
    oi = o.run_until(0.25)
    di = d.run_until(0.25)
    assert oi.steps_done == di.steps_done and di.stopped_at_t_stop == 1
    assert abs(oi.time - di.time) < 1e-13


FIX = np.load(os.path.join(os.path.dirname(__file__), "golden", "oracle_fixtures.npz"))
PINS = json.load(open(os.path.join(os.path.dirname(__file__), "golden", "oracle_pins.json")))


def test_committed_golden_fixtures_on_gpu():
    grid, params, u, ex = vortex_periodic(32)
    d = Context(grid, params)
    d.upload(FIX["vortex32_init"])
    d.step(5)
    assert rel_err(d.download(), FIX["vortex32_periodic_muscl_minmod_5steps"]) < TOL_MANY_STEPS
    grid, params, u, ex = cases.cylinder_case(110, 41, muscl=True)
    d = Context(grid, params)
    d.set_cylinders(ex["cylinders"], ex["freestream"])
    d.upload(FIX["cylinder110x41_init"])
    info, hist = d.step(3, history=True)
    assert np.array_equal(d.solid_mask(), FIX["cylinder110x41_mask"])
    assert rel_err(d.download(), FIX["cylinder110x41_muscl_3steps"]) < TOL_MANY_STEPS
    ref = FIX["cylinder110x41_muscl_3steps_marker_history"]
    assert np.max(np.abs(hist - ref)) <= 1e-10 * np.max(np.abs(ref))


def test_reference_cylinder_drag_is_reproduced_on_gpu():
    """examples/cylinder_drag_validation/config.toml on the GPU: 440x82, first-order
    HLLC, 44,000 substeps; Cd over the last 10 % must print as the reference's
    5.6312, agree with the oracle's full run, and sit on a steady plateau."""
    grid, params, u, ex = cases.cylinder_case()
    d = Context(grid, params)
    d.set_cylinders(ex["cylinders"], ex["freestream"])
    d.upload(u)
    n = 44000
    full, rest = divmod(n, 3)
    info, hist = d.step(full, history=True)
    fx = list(hist[:, 0] + hist[:, 3])
    for _ in range(rest):
        d.substep()
        f = d.marker_force()
        fx.append(f[0] + f[3])
    cd = np.array(fx[int(0.9 * n):]) / ex["q"]
    pin = PINS["cylinder_dfg_2d1_440x82"]
    assert f"{cd.mean():.4f}" == f"{pin['published']:.4f}"
    assert abs(cd.mean() - pin["cd_mean_last_10pct"]) <= 1e-8 * pin["cd_mean_last_10pct"]
    assert (cd.max() - cd.min()) / abs(cd.mean()) <= 0.02
    assert abs(cd.mean() - 5.5795) / 5.5795 <= 0.05
