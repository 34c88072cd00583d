"""GPU parity with the oracle for the options the benchmark cases do not use:
supersonic and subsonic inflow, symmetry, slip and no-slip walls, the pressure
outlet, Sutherland viscosity, the forward-Euler integrator, first-order and
MUSCL reconstruction with every flux, and the FP32-flux form on the viscous
channel.  Tolerances as in test_gpu_parity.py (FP64: 1e-12 after one step,
1e-10 after ten); FP32 fluxes at 1 bar and Mach 0.1: 2e-4."""
from __future__ import annotations

import numpy as np
import pytest

from dev_field_efvm_b200 import abi, cases
from test_gpu_parity import TOL_MANY_STEPS, TOL_ONE_STEP, pair, rel_err

pytestmark = pytest.mark.gpu


def perturbed(grid, rho, u, v, p):
    x, y = cases.centroids(grid)
    X, Y = np.meshgrid(x, y)
    lx, ly = grid.hi[0] - grid.lo[0], grid.hi[1] - grid.lo[1]
    bump = np.exp(-(((X - 0.4 * lx) / (0.15 * lx)) ** 2 + ((Y - 0.5 * ly) / (0.2 * ly)) ** 2))
    return cases.prim_to_cons(rho * (1 + 0.2 * bump), u * (1 + 0.1 * bump), v + 0.05 * u * bump, p * (1 + 0.3 * bump))


def inflow_case(flux, muscl, integrator):
    """Supersonic inflow at x-lo, zero-gradient outflow at x-hi, symmetry below, slip wall above."""
    bcs = {abi.XLO: abi.make_bc(abi.BC_SUPERSONIC_INFLOW, rho=1.4, u=2.0, v=0.1, w=0.0, p=1.0),
           abi.XHI: abi.BC_SUPERSONIC_OUTFLOW, abi.YLO: abi.BC_SYMMETRY, abi.YHI: abi.BC_SLIP_WALL,
           abi.ZLO: abi.BC_SLIP_WALL, abi.ZHI: abi.BC_SLIP_WALL}
    grid = abi.make_grid(48, 24, hi=(2.0, 1.0, 2.0 / 48), bcs=bcs)
    params = abi.make_params(cfl=0.4, r_gas=1.0, flux_scheme=flux, integrator=integrator,
                             reconstruction=abi.RECON_MUSCL if muscl else abi.RECON_FIRST_ORDER)
    return grid, params, perturbed(grid, 1.4, 1.5, 0.0, 1.0)


def subsonic_case(muscl, precision=abi.PREC_FP64):
    """Subsonic inflow at x-lo, pressure outlet at x-hi, no-slip walls, Sutherland air."""
    bcs = {abi.XLO: abi.make_bc(abi.BC_SUBSONIC_INFLOW, rho=1.2, u=40.0, v=0.0, w=0.0, t=300.0),
           abi.XHI: abi.make_bc(abi.BC_PRESSURE_OUTLET, p=1.0e5),
           abi.YLO: abi.BC_NO_SLIP_WALL, abi.YHI: abi.BC_NO_SLIP_WALL,
           abi.ZLO: abi.BC_SLIP_WALL, abi.ZHI: abi.BC_SLIP_WALL}
    grid = abi.make_grid(40, 20, hi=(0.02, 0.01, 0.0005), bcs=bcs)
    params = abi.make_params(cfl=0.4, viscous=1, viscosity_model=abi.VISC_SUTHERLAND, precision=precision,
                             reconstruction=abi.RECON_MUSCL if muscl else abi.RECON_FIRST_ORDER)
    return grid, params, perturbed(grid, 1.2, 40.0, 0.0, 1.0e5)


@pytest.mark.parametrize("flux", [abi.FLUX_HLLC, abi.FLUX_HLLC_TEXTBOOK, abi.FLUX_RUSANOV])
@pytest.mark.parametrize("muscl", [False, True])
@pytest.mark.parametrize("integrator", [abi.INTEGRATOR_RK3, abi.INTEGRATOR_EULER])
def test_inflow_symmetry_slip(flux, muscl, integrator):
    grid, params, u = inflow_case(flux, muscl, integrator)
    o, d = pair(grid, params, u)
    o.step(1)
    d.step(1)
    assert rel_err(d.download(), o.download()) < TOL_ONE_STEP
    o.step(9)
    d.step(9)
    assert rel_err(d.download(), o.download()) < TOL_MANY_STEPS
    assert d.solver_state().step == o.solver_state().step == 10


@pytest.mark.parametrize("muscl", [False, True])
def test_subsonic_inflow_pressure_outlet_sutherland(muscl):
    grid, params, u = subsonic_case(muscl)
    o, d = pair(grid, params, u)
    o.step(1)
    d.step(1)
    assert rel_err(d.download(), o.download()) < TOL_ONE_STEP
    o.step(9)
    d.step(9)
    assert rel_err(d.download(), o.download()) < TOL_MANY_STEPS


def test_fp32_flux_on_the_viscous_channel():
    """Air at 1 bar and Mach 0.1: pressure differences are ~1e-3 of p, so FP32
    face states carry relative errors near 1e-4 of them; the bound is 2e-4."""
    grid, params, u = subsonic_case(True)
    o, _ = pair(grid, params, u)
    _, p32, _ = subsonic_case(True, precision=abi.PREC_FP32_FLUX)
    from dev_field_efvm_b200.device import Context

    d = Context(grid, p32)
    d.upload(u)
    o.step(10)
    d.step(10)
    assert rel_err(d.download(), o.download()) < 2e-4


@pytest.mark.parametrize("nz", [1, 4])
def test_round_off_velocities_in_still_gas(nz):
    """Still gas whose velocities are round-off sized (1e-157, squares below the
    normal range): the low-Mach blend must stay finite and the state must match
    the oracle (the flush-to-zero reciprocal square root once turned these into
    NaN next to a resting immersed disc)."""
    from oracle import pyoracle as po
    from dev_field_efvm_b200.device import Context
    rng = np.random.default_rng(11)
    P = abi.BC_PERIODIC
    grid = abi.make_grid(32, 24, hi=(1.0, 0.75, 0.125 if nz > 1 else 1.0 / 32),
                         bcs={abi.XLO: P, abi.XHI: P, abi.YLO: P, abi.YHI: P,
                              abi.ZLO: P if nz > 1 else abi.BC_SLIP_WALL, abi.ZHI: P if nz > 1 else abi.BC_SLIP_WALL},
                         nz=nz)
    params = abi.make_params(cfl=0.4, reconstruction=abi.RECON_MUSCL)
    shape = (nz, 24, 32) if nz > 1 else (24, 32)
    tiny = 1e-157 * rng.standard_normal((3,) + shape)
    from dev_field_efvm_b200 import cases
    u = cases.prim_to_cons3(np.ones(shape), tiny[0], tiny[1], tiny[2] if nz > 1 else 0.0, np.full(shape, 1.0e5))
    o, d = po.OracleCase(grid, params), Context(grid, params)
    o.upload(u)
    d.upload(u)
    o.step(4)
    d.step(4)
    got, want = d.download(), o.download()
    assert np.isfinite(got).all()
    assert np.max(np.abs(got[..., 0] - want[..., 0])) <= 1e-12
    assert np.max(np.abs(got[..., 4] - want[..., 4])) <= 1e-12 * 2.5e5
