"""Per-cell parity with the CPU oracle at the benchmark's full sizes, the batch
path against the oracle, and forces left pending across calls.

Full sizes: one RK3 step of the 1100x205 cylinder channel (MUSCL + HLLC,
viscous, immersed cylinder, parabolic inlet, sponge) and of the 4096^2 periodic
vortex (reference seam), each against the OpenMP build of the oracle
(the same arithmetic as the serial oracle, faces visited in another order:
the two agree to 1e-13).  Tolerance as in test_gpu_parity.py: 1e-12 per cell
after one step, relative to max(|oracle|, 1e-3 * scale).

Batch: cases of the batching workload (periodic vortices and four-quadrant
Riemann problems with transmissive boundaries) advanced together by
efvm_batch_run and, one by one, by the oracle: 1e-12 after one step and 1e-10
after five in FP64; FP32 face fluxes within 5e-5 of the FP64 oracle.
"""
import numpy as np
import pytest

from dev_field_efvm_b200 import abi, cases
from dev_field_efvm_b200.device import Batch, Context
from oracle import pyoracle as po

from test_gpu_parity import TOL_MANY_STEPS, TOL_ONE_STEP, rel_err

pytestmark = pytest.mark.gpu


def test_cylinder_channel_full_size_one_step_matches_oracle():
    grid, params, u, ex = cases.cylinder_baseline_case()
    assert (grid.nx, grid.ny) == (1100, 205)
    o = po.OracleCase(grid, params, parallel=True)
    d = Context(grid, params)
    for c in (o, d):
        c.set_cylinders(ex["cylinders"], ex["freestream"])
        c.upload(u)
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
    o.close()


def test_vortex_4096_one_step_matches_oracle():
    grid, params, u, ex = cases.vortex_case(4096, periodic=True, muscl=True, mean=(1.0, 1.0), cfl=0.4)
    o = po.OracleCase(grid, params, parallel=True)
    d = Context(grid, params)
    o.upload(u)
    d.upload(u)
    assert abs(d.cfl() - o.cfl()) <= 1e-14 * o.cfl()
    o.step(1)
    d.step(1)
    assert abs(d.solver_state().time - o.solver_state().time) <= 1e-15 * o.solver_state().time
    assert rel_err(d.download(), o.download()) < TOL_ONE_STEP
    o.close()


def batch_subset(precision):
    """Six cases of the batching workload's generator, three of each kind, at
    sizes from 32^2 to 200^2."""
    grids, params, states, t_stop, kinds = cases.batch_cases(n_cases=6, seed=11, n_min=32, n_max=200,
                                                             precision=precision)
    assert kinds.count("riemann") == 3 and kinds.count("vortex") == 3
    return grids, params, states, t_stop, kinds


@pytest.mark.parametrize("steps,tol", [(1, TOL_ONE_STEP), (5, TOL_MANY_STEPS)])
def test_batch_fp64_matches_oracle_per_case(steps, tol):
    grids, params, states, t_stop, kinds = batch_subset(abi.PREC_FP64)
    b = Batch(grids, params)
    for k, u in enumerate(states):
        b.upload(k, u)
    res = b.run(t_stop, max_steps=steps)
    for k, (g, u) in enumerate(zip(grids, states)):
        assert res[k].steps == steps and res[k].nonphysical == 0
        o = po.OracleCase(g, params)
        o.upload(u)
        o.step(steps)
        assert abs(b.solver_state(k).time - o.solver_state().time) <= 1e-14 * o.solver_state().time, (k, kinds[k])
        err = rel_err(b.download(k), o.download())
        assert err < tol, (k, kinds[k], g.nx, err)
        o.close()
    b.close()


def test_batch_fp32_flux_tracks_fp64_oracle():
    grids, params, states, t_stop, kinds = batch_subset(abi.PREC_FP32_FLUX)
    p64 = abi.make_params(**{f: getattr(params, f) for f, _ in abi.EfvmParams._fields_ if f != "precision"})
    b = Batch(grids, params)
    for k, u in enumerate(states):
        b.upload(k, u)
    b.run(t_stop, max_steps=5)
    for k, (g, u) in enumerate(zip(grids, states)):
        o = po.OracleCase(g, p64)
        o.upload(u)
        o.step(5)
        # FP32 face states and fluxes (~1e-7 relative per flux), FP64 accumulation
        assert rel_err(b.download(k), o.download()) < 5e-5, (k, kinds[k])
        o.close()
    b.close()


def test_forces_left_pending_across_calls():
    """efvm_step without a status read leaves the last substage's IBM forces
    pending (they run in the next step's first launch).  Reading the forces, or
    stepping with a history, must first run them: the results equal those of
    synchronous steps, and a history after pending forces has exactly 3 rows
    per step, equal to the oracle's."""
    grid, params, u, ex = cases.cylinder_case(110, 41, muscl=True)

    def ctx():
        d = Context(grid, params)
        d.set_cylinders(ex["cylinders"], ex["freestream"])
        d.upload(u)
        return d

    a, b = ctx(), ctx()
    a.step(4)
    b.step_async(4)
    assert np.array_equal(b.marker_force(), a.marker_force())
    assert np.array_equal(b.wall_force(), a.wall_force())
    assert np.array_equal(b.download(), a.download())
    b.step_async(2)
    _, hb = b.step(3, history=True)
    a.step(2)
    _, ha = a.step(3, history=True)
    assert hb.shape == ha.shape == (9, 6)
    assert np.array_equal(hb, ha)
    o = po.OracleCase(grid, params)
    o.set_cylinders(ex["cylinders"], ex["freestream"])
    o.upload(u)
    o.step(6)
    _, ho = o.step(3, history=True)
    assert np.max(np.abs(hb - ho)) <= 1e-10 * np.max(np.abs(ho))
    assert rel_err(b.download(), o.download()) < TOL_MANY_STEPS
