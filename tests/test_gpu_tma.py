"""The TMA-fed stage kernel (efvm_set_stage_tiling(ctx, EFVM_STAGE_TMA, rows)).

It runs the strip kernel's arithmetic on rows that TMA brings into a
shared-memory ring, so it is held to the same bars as the strip kernel: within
1e-12 of the CPU oracle per cell after one RK3 step and 1e-10 after twenty (FP64),
FP32 face fluxes within 5e-5 of the FP64 oracle after ten steps, the same bits
for any rows per warp, and a step that commutes with a whole-cell shift of a
periodic grid bit for bit.  The kernel's builds per limiter and for fully
periodic grids are each compared with the oracle.  The sizes cover blocks whose last strips are empty
(nx not a multiple of 124), grids narrower than one block, and fewer rows than a
warp marches.  Against the strip form the fields agree to 1e-13.  The autotuner
leaves the state and the clock as it found them.
"""
import numpy as np
import pytest

from dev_field_efvm_b200 import abi, cases
from dev_field_efvm_b200.device import Context
from oracle import pyoracle as po

from test_gpu_parity import TOL_MANY_STEPS, TOL_ONE_STEP, rel_err

pytestmark = pytest.mark.gpu


def tma_context(grid, params, u, rows=0):
    d = Context(grid, params)
    d.set_stage_tiling(abi.STAGE_TMA, rows)
    assert d.stage_tiling()[0] == abi.STAGE_TMA
    d.upload(u)
    return d


@pytest.mark.parametrize("seam", [abi.SEAM_REFERENCE, abi.SEAM_TRUE_PERIODIC])
@pytest.mark.parametrize("n,ny", [(64, 64), (200, 77), (40, 5)])
def test_periodic_vortex_matches_oracle(seam, n, ny):
    grid, params, u, ex = cases.vortex_case(n, periodic=True, muscl=True, mean=(1.0, 1.0), cfl=0.4, seam=seam,
                                            ny=ny)
    o = po.OracleCase(grid, params)
    o.upload(u)
    d = tma_context(grid, params, u)
    o.step(1)
    d.step(1)
    assert rel_err(d.download(), o.download()) < TOL_ONE_STEP
    o.step(19)
    d.step(19)
    assert rel_err(d.download(), o.download()) < TOL_MANY_STEPS
    so, sd = o.solver_state(), d.solver_state()
    assert sd.step == so.step == 20 and abs(sd.time - so.time) <= 1e-13 * so.time


@pytest.mark.parametrize("scheme,muscl,limiter", [
    (abi.FLUX_HLLC, True, abi.LIMITER_MC),
    (abi.FLUX_HLLC, False, abi.LIMITER_MINMOD),
    (abi.FLUX_RUSANOV, True, abi.LIMITER_MINMOD),
])
def test_periodic_builds_per_limiter_and_first_order_match_oracle(scheme, muscl, limiter):
    """The TMA-fed kernel is built per limiter and for fully periodic grids
    (those branches decided at compile time): the MC limiter, first order and
    Rusanov on a periodic grid run those builds, against the oracle."""
    grid, params, u, ex = cases.vortex_case(140, periodic=True, muscl=muscl, limiter=limiter, mean=(1.0, 1.0),
                                            cfl=0.4, ny=53)
    params.flux_scheme = scheme
    o = po.OracleCase(grid, params)
    o.upload(u)
    d = tma_context(grid, params, u)
    o.step(1)
    d.step(1)
    assert rel_err(d.download(), o.download()) < TOL_ONE_STEP
    o.step(9)
    d.step(9)
    assert rel_err(d.download(), o.download()) < TOL_MANY_STEPS


@pytest.mark.parametrize("scheme,muscl,limiter", [
    (abi.FLUX_HLLC, True, abi.LIMITER_MINMOD),
    (abi.FLUX_HLLC, False, abi.LIMITER_MINMOD),
    (abi.FLUX_RUSANOV, True, abi.LIMITER_MC),
    (abi.FLUX_HLLC_TEXTBOOK, True, abi.LIMITER_MC),
])
def test_outflow_vortex_schemes_match_oracle(scheme, muscl, limiter):
    grid, params, u, ex = cases.vortex_case(150, periodic=False, muscl=muscl, limiter=limiter, ny=61)
    params.flux_scheme = scheme
    o = po.OracleCase(grid, params)
    o.upload(u)
    d = tma_context(grid, params, u)
    o.step(1)
    d.step(1)
    assert rel_err(d.download(), o.download()) < TOL_ONE_STEP
    o.step(9)
    d.step(9)
    assert rel_err(d.download(), o.download()) < TOL_MANY_STEPS


def test_fp32_flux_tracks_fp64_oracle():
    grid, params, u, ex = cases.vortex_case(130, periodic=True, muscl=True, mean=(1.0, 1.0), cfl=0.4,
                                            precision=abi.PREC_FP32_FLUX)
    p64 = abi.make_params(**{f: getattr(params, f) for f, _ in abi.EfvmParams._fields_ if f != "precision"})
    o = po.OracleCase(grid, p64)
    o.upload(u)
    d = tma_context(grid, params, u)
    o.step(10)
    d.step(10)
    assert rel_err(d.download(), o.download()) < 5e-5
    s = Context(grid, params)  # the strip form of the same FP32 stage
    s.set_stage_tiling(abi.STAGE_STRIP, 0)
    s.upload(u)
    s.step(10)
    assert rel_err(d.download(), s.download()) < 1e-6


@pytest.mark.parametrize("precision", [abi.PREC_FP64, abi.PREC_FP32_FLUX])
def test_rows_per_warp_change_no_bit(precision):
    grid, params, u, ex = cases.vortex_case(300, periodic=True, muscl=True, mean=(1.0, 1.0), cfl=0.4,
                                            ny=211, precision=precision)
    out = []
    for rows in (2, 7, 64, 0):
        d = tma_context(grid, params, u, rows)
        d.step(3)
        out.append(d.download())
        d.close()
    for x in out[1:]:
        assert np.array_equal(x, out[0])


def test_tma_and_strip_forms_agree():
    grid, params, u, ex = cases.vortex_case(256, periodic=True, muscl=True, mean=(1.0, 1.0), cfl=0.4)
    d = tma_context(grid, params, u)
    s = Context(grid, params)
    s.set_stage_tiling(abi.STAGE_STRIP, 0)
    s.upload(u)
    d.step(5)
    s.step(5)
    assert rel_err(d.download(), s.download()) < 1e-13


def test_translation_invariance_true_periodic():
    n = 1024
    grid, params, u, ex = cases.vortex_case(n, periodic=True, muscl=True, mean=(1.0, 1.0), cfl=0.4,
                                            seam=abi.SEAM_TRUE_PERIODIC)
    params.fixed_dt = 4.0e-3
    a = tma_context(grid, params, u)
    a.step(2)
    ua = a.download()
    a.close()
    b = tma_context(grid, params, np.roll(u, (37, 411), axis=(0, 1)))
    b.step(2)
    assert np.array_equal(np.roll(ua, (37, 411), axis=(0, 1)), b.download())


def test_vortex_4096_one_step_matches_oracle():
    grid, params, u, ex = cases.vortex_case(4096, periodic=True, muscl=True, mean=(1.0, 1.0), cfl=0.4)
    o = po.OracleCase(grid, params, parallel=True)
    o.upload(u)
    d = tma_context(grid, params, u)
    o.step(1)
    d.step(1)
    assert rel_err(d.download(), o.download()) < TOL_ONE_STEP
    o.close()


def test_bodies_and_viscous_cases_run_the_strip_form():
    grid, params, u, ex = cases.cylinder_case(110, 41, muscl=True)
    d = Context(grid, params)
    d.set_stage_tiling(abi.STAGE_TMA, 0)
    d.set_cylinders(ex["cylinders"], ex["freestream"])
    d.upload(u)
    assert d.stage_tiling()[0] == abi.STAGE_STRIP
    o = po.OracleCase(grid, params)
    o.set_cylinders(ex["cylinders"], ex["freestream"])
    o.upload(u)
    d.step(1)
    o.step(1)
    assert rel_err(d.download(), o.download()) < TOL_ONE_STEP


def test_autotune_restores_state_and_clock():
    grid, params, u, ex = cases.vortex_case(512, periodic=True, muscl=True, mean=(1.0, 1.0), cfl=0.4)
    d = Context(grid, params)
    d.upload(u)
    d.step(2)
    before, s_before = d.download(), d.solver_state()
    ms = d.autotune_stage(2)
    assert ms > 0.0
    form, rows, blocks = d.stage_tiling()
    assert form in (abi.STAGE_STRIP, abi.STAGE_TMA) and rows >= 1 and blocks in (5, 6, 7)
    assert np.array_equal(d.download(), before)
    s_after = d.solver_state()
    assert (s_after.step, s_after.time, s_after.dt) == (s_before.step, s_before.time, s_before.dt)
    d.step(3)
    ref = Context(grid, params)
    ref.upload(u)
    ref.step(5)
    assert rel_err(d.download(), ref.download()) < 1e-13


def test_strip_form_at_its_alternate_block_count_matches_oracle():
    """The FP64 inviscid strip form is also built for 7 resident blocks per SM
    (the autotuner's second count); it holds the same 1e-12 bar, and a count no
    form is built for is refused."""
    from dev_field_efvm_b200.device import EfvmError

    grid, params, u, ex = cases.vortex_case(200, periodic=True, muscl=True, mean=(1.0, 1.0), cfl=0.4, ny=77)
    o = po.OracleCase(grid, params)
    o.upload(u)
    d = Context(grid, params)
    d.set_stage_tiling(abi.STAGE_STRIP, 0, 7)
    assert d.stage_tiling()[0] == abi.STAGE_STRIP and d.stage_tiling()[2] == 7
    d.upload(u)
    o.step(1)
    d.step(1)
    assert rel_err(d.download(), o.download()) < TOL_ONE_STEP
    with pytest.raises(EfvmError):
        d.set_stage_tiling(abi.STAGE_STRIP, 0, 5)


def test_ring_wait_that_runs_out_reports_a_timeout():
    """The ring's waits are bounded in time (efvm_set_stage_wait_limit).  With
    the first block's refills withheld (efvm_inject_stage_stall) its warps wait
    for a row that never comes; each wait ends after the limit, the step
    reports EFVM_ERR_TIMEOUT within a few limits, and the GPU stays usable: a
    fresh context on it matches the oracle."""
    import time
    from dev_field_efvm_b200.device import EfvmError

    grid, params, u, ex = cases.vortex_case(256, periodic=True, muscl=True, mean=(1.0, 1.0), cfl=0.4)
    d = tma_context(grid, params, u)
    d.set_stage_wait_limit(0.05)
    d.inject_stage_stall(True)
    t0 = time.perf_counter()
    with pytest.raises(EfvmError) as e:
        d.step(1)
    assert e.value.code == abi.ERR_TIMEOUT
    assert time.perf_counter() - t0 < 10.0
    d.close()
    o = po.OracleCase(grid, params)
    o.upload(u)
    f = tma_context(grid, params, u)
    o.step(1)
    f.step(1)
    assert rel_err(f.download(), o.download()) < TOL_ONE_STEP
