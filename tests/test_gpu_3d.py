"""3-D meshes (nz > 1): the CUDA path through the C-ABI against the CPU oracle,
which is the reference's systems on FIELD's 3-D raw array (x, y and z faces,
both ghost layers on every axis, 7-point viscous stencil).

Tolerances as in test_gpu_parity.py: 1e-12 after one RK3 step, 1e-10 after
ten, relative to max(|oracle|, 1e-3 * scale) per variable, with all three
momenta judged against the momentum unit of the state's energy.  Conservation
and translation invariance are checked bit for bit or to round-off."""
from __future__ import annotations

import math

import numpy as np
import pytest

from dev_field_efvm_b200 import abi, cases
from dev_field_efvm_b200.device import Context, EfvmError
from oracle import pyoracle as po

pytestmark = pytest.mark.gpu

TOL_ONE_STEP = 1e-12
TOL_MANY_STEPS = 1e-10


def rel_err3(g, o):
    mom = float(np.max(np.sqrt(np.abs(o[..., 0] * o[..., 4]))))
    scale = np.array([np.max(np.abs(o[..., 0])), mom, mom, mom, np.max(np.abs(o[..., 4]))])
    denom = np.maximum(np.abs(o), 1e-3 * np.maximum(scale, 1e-300))
    return float(np.max(np.abs(g - o) / denom))


def pair3(grid, params, u):
    o = po.OracleCase(grid, params)
    d = Context(grid, params)
    o.upload(u)
    d.upload(u)
    return o, d


def channel3(muscl, flux=abi.FLUX_HLLC, viscous=True, integrator=abi.INTEGRATOR_RK3):
    """A walled 3-D channel: subsonic inflow at x-lo, pressure outlet at x-hi,
    no-slip walls in y, slip walls in z, Sutherland air, and a 3-D bump in every
    primitive including w."""
    bcs = {abi.XLO: abi.make_bc(abi.BC_SUBSONIC_INFLOW, rho=1.2, u=40.0, v=0.0, w=0.0, t=300.0),
           abi.XHI: abi.make_bc(abi.BC_PRESSURE_OUTLET, p=1.0e5),
           abi.YLO: abi.BC_NO_SLIP_WALL, abi.YHI: abi.BC_NO_SLIP_WALL,
           abi.ZLO: abi.BC_SLIP_WALL, abi.ZHI: abi.BC_SLIP_WALL}
    nx, ny, nz = 40, 18, 10
    grid = abi.make_grid(nx, ny, hi=(0.02, 0.009, 0.005), bcs=bcs, nz=nz)
    params = abi.make_params(cfl=0.4, viscous=1 if viscous else 0, viscosity_model=abi.VISC_SUTHERLAND,
                             flux_scheme=flux, integrator=integrator,
                             reconstruction=abi.RECON_MUSCL if muscl else abi.RECON_FIRST_ORDER)
    x = (np.arange(nx) + 0.5) / nx
    y = (np.arange(ny) + 0.5) / ny
    z = (np.arange(nz) + 0.5) / nz
    Z, Y, X = np.meshgrid(z, y, x, indexing="ij")
    bump = np.exp(-(((X - 0.4) / 0.15) ** 2 + ((Y - 0.5) / 0.2) ** 2 + ((Z - 0.5) / 0.25) ** 2))
    u = cases.prim_to_cons3(1.2 * (1 + 0.2 * bump), 40.0 * (1 + 0.1 * bump), 2.0 * bump, -3.0 * bump,
                            1.0e5 * (1 + 0.3 * bump))
    return grid, params, u


@pytest.mark.parametrize("seam", [abi.SEAM_REFERENCE, abi.SEAM_TRUE_PERIODIC])
def test_vortex_tube_periodic_muscl_hllc(seam):
    grid, params, u, _ = cases.vortex_tube_case(40, 12, seam=seam)
    o, d = pair3(grid, params, u)
    o.step(1)
    d.step(1)
    assert rel_err3(d.download(), o.download()) < TOL_ONE_STEP
    o.step(9)
    d.step(9)
    assert rel_err3(d.download(), o.download()) < TOL_MANY_STEPS
    so, sd = o.solver_state(), d.solver_state()
    assert so.step == sd.step == 10
    assert abs(so.time - sd.time) <= 1e-12 * so.time


@pytest.mark.parametrize("flux", [abi.FLUX_HLLC, abi.FLUX_HLLC_TEXTBOOK, abi.FLUX_RUSANOV])
@pytest.mark.parametrize("muscl", [False, True])
def test_channel_walls_inflow_outlet_viscous(flux, muscl):
    grid, params, u = channel3(muscl, flux)
    o, d = pair3(grid, params, u)
    o.step(1)
    d.step(1)
    assert rel_err3(d.download(), o.download()) < TOL_ONE_STEP
    o.step(9)
    d.step(9)
    assert rel_err3(d.download(), o.download()) < TOL_MANY_STEPS


@pytest.mark.parametrize("nz", [2, 3, 5])
def test_thin_meshes_with_fewer_layers_than_a_block(nz):
    """Meshes whose last (or only) block of stacked layers is partly empty: the
    warps past the last layer keep the block's barriers and write nothing.
    Periodic in z (the wrap then reaches across the whole mesh) and walled."""
    grid, params, u, _ = cases.vortex_tube_case(24, nz, seam=abi.SEAM_TRUE_PERIODIC)
    o, d = pair3(grid, params, u)
    o.step(4)
    d.step(4)
    assert rel_err3(d.download(), o.download()) < TOL_MANY_STEPS
    bcs = {abi.XLO: abi.BC_PERIODIC, abi.XHI: abi.BC_PERIODIC, abi.YLO: abi.BC_PERIODIC,
           abi.YHI: abi.BC_PERIODIC, abi.ZLO: abi.BC_NO_SLIP_WALL, abi.ZHI: abi.BC_SLIP_WALL}
    grid = abi.make_grid(24, 24, lo=(0.0, 0.0, 0.0), hi=(10.0, 10.0, 10.0 * nz / 24), bcs=bcs, nz=nz)
    o, d = pair3(grid, params, u)
    o.step(4)
    d.step(4)
    assert rel_err3(d.download(), o.download()) < TOL_MANY_STEPS


def test_channel_inviscid_euler_integrator_and_mc_limiter():
    grid, params, u = channel3(True, viscous=False, integrator=abi.INTEGRATOR_EULER)
    params.limiter = abi.LIMITER_MC
    o, d = pair3(grid, params, u)
    for _ in range(10):
        o.substep()
        d.substep()
    assert rel_err3(d.download(), o.download()) < TOL_MANY_STEPS


def test_viscous_vortex_tube_and_substeps():
    """The viscous periodic form, advanced stage by stage through efvm_substep."""
    grid, params, u, _ = cases.vortex_tube_case(36, 8, viscous=True, mu=2.0e-3)
    o, d = pair3(grid, params, u)
    for _ in range(6):
        o.substep()
        d.substep()
        assert rel_err3(d.download(), o.download()) < TOL_MANY_STEPS
    assert d.solver_state().step == 2


def test_mass_conservation_true_periodic():
    grid, params, u, _ = cases.vortex_tube_case(64, 32, seam=abi.SEAM_TRUE_PERIODIC)
    d = Context(grid, params)
    d.upload(u)
    m0 = d.total_mass()
    d.step(20)
    assert abs(d.total_mass() - m0) / m0 < 1e-13


def test_translation_invariance_true_periodic():
    """The step commutes with a shift by whole cells in x, y and z, bit for bit:
    a z face on the edge of two blocks' layers is formed by both blocks from
    slopes and states that went through one code path, and a y face on the edge
    of two warps' rows likewise."""
    grid, params, u, _ = cases.vortex_tube_case(96, 40, seam=abi.SEAM_TRUE_PERIODIC)
    params.fixed_dt = 2.0e-3
    shift = (7, 13, 29)  # z, y, x
    a = Context(grid, params)
    a.upload(u)
    a.step(2)
    ua = a.download()
    a.close()
    b = Context(grid, params)
    b.upload(np.roll(u, shift, axis=(0, 1, 2)))
    b.step(2)
    ub = b.download()
    assert np.array_equal(np.roll(ua, shift, axis=(0, 1, 2)), ub)


def test_z_uniform_state_matches_the_2d_path():
    """A state that does not depend on z, with w = 0 on a periodic z axis, evolves
    as the 2-D mesh does (the z fluxes cancel up to round-off in rho_w)."""
    grid2, params, u2, _ = cases.vortex_case(48, periodic=True, muscl=True, mean=(1.0, 1.0), cfl=0.4)
    params.r_gas = 1.0
    grid3 = abi.make_grid(48, 48, lo=(0.0, 0.0, 0.0), hi=(10.0, 10.0, 10.0 * 6 / 48),
                          bcs={s: abi.BC_PERIODIC for s in range(6)}, nz=6)
    params.fixed_dt = 4.0e-3
    d2, d3 = Context(grid2, params), Context(grid3, params)
    d2.upload(u2)
    d3.upload(np.broadcast_to(u2[None], (6,) + u2.shape).copy())
    d2.step(10)
    d3.step(10)
    a, b = d2.download(), d3.download()
    for k in range(6):
        bk = b[k].copy()
        assert np.max(np.abs(bk[..., 3])) <= 1e-12 * np.max(np.abs(a[..., 1]))
        bk[..., 3] = 0.0
        assert rel_err3(bk, a) < 1e-12


def test_two_d_only_entry_points_refuse_a_3d_context():
    grid, params, u, _ = cases.vortex_tube_case(32, 4)
    d = Context(grid, params)
    d.upload(u)
    with pytest.raises(EfvmError):
        d.set_cylinders(np.array([[5.0, 5.0, 1.0]]), [1.0, 1.0, 0.0, 0.0, 1.0 / 0.4])
    import ctypes as C
    buf = np.zeros((4, 32, 32, 5))
    rc = d.L.efvm_upload_state(d.h, buf.ctypes.data_as(C.POINTER(C.c_double)), 5, 5 * 32, 1)
    assert rc == abi.ERR_UNSUPPORTED
    assert b"efvm_upload_state_3d" in d.L.efvm_last_error(d.h)
    # the state survives the refused calls
    d.step(1)
    assert np.isfinite(d.download()).all()
