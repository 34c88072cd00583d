"""Size-independent properties of the newer stage paths at the benchmark's
4096^2 size, where the oracle is too slow for many steps:

* the FP32-flux form (the TMA-fed kernel) conserves mass to FP64 rounding on
  the conservative periodic seam (every face flux is formed once and enters
  both cells' FP64 divergence);
* two row slabs with the halo exchange fused into the stage kernels equal the
  unsplit context bit for bit;
* the stage autotuner on an immersed-body case leaves the state, the clock and
  the marker force as it found them.
"""
import numpy as np
import pytest

from dev_field_efvm_b200 import abi, cases, slab
from dev_field_efvm_b200.device import Context

pytestmark = pytest.mark.gpu


def test_fp32_flux_tma_form_conserves_mass_at_4096():
    grid, params, u, ex = cases.vortex_case(4096, periodic=True, muscl=True, mean=(1.0, 1.0), cfl=0.4,
                                            seam=abi.SEAM_TRUE_PERIODIC, precision=abi.PREC_FP32_FLUX)
    d = Context(grid, params)
    assert d.stage_tiling()[0] == abi.STAGE_TMA
    d.upload(u)
    m0 = d.total_mass()
    d.step(20)
    assert abs(d.total_mass() - m0) / m0 < 1e-13


def test_two_peer_slabs_equal_the_unsplit_context_at_4096():
    grid, params, u, ex = cases.vortex_case(4096, periodic=True, muscl=True, mean=(1.0, 1.0), cfl=0.4)
    ref = Context(grid, params)
    ref.upload(u)
    ref.step(3)
    want, s_ref = ref.download(), ref.solver_state()
    ref.close()
    engines = []
    for r0, n in slab.split_rows(grid.ny, 2):
        e = slab.DeviceSlab(grid, params, r0, n)
        e.ctx.upload(u[r0:r0 + n])
        engines.append(e)
    slab.PeerLocalSlabs(engines, True).step(3)
    got = np.concatenate([e.ctx.download() for e in engines])
    assert engines[0].ctx.solver_state().time == s_ref.time
    assert np.array_equal(got, want)


def test_autotune_on_a_cylinder_restores_state_clock_and_forces():
    grid, params, u, ex = cases.cylinder_case(440, 82, muscl=True)
    d = Context(grid, params)
    d.set_cylinders(ex["cylinders"], ex["freestream"])
    d.upload(u)
    d.step(5)
    before, s0, f0, w0 = d.download(), d.solver_state(), d.marker_force(), d.wall_force()
    assert d.autotune_stage(2) > 0.0
    assert d.stage_tiling()[0] == abi.STAGE_STRIP  # bodies run the strip form
    assert np.array_equal(d.download(), before)
    s1 = d.solver_state()
    assert (s1.step, s1.time, s1.dt) == (s0.step, s0.time, s0.dt)
    assert np.array_equal(d.marker_force(), f0) and np.array_equal(d.wall_force(), w0)
