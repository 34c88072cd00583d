"""Checkpoint / restart parity: a run saved part-way and restored into a fresh
context continues bit for bit (crates/cfd_solver/tests/restart.rs:86-105).

The CPU tests check the algorithm on the oracle (which follows the reference's
substep order) and the checkpoint file round trip; the GPU tests check the
device path, where bit-for-bit continuation also needs deterministic
reductions (CFL maximum, force sums)."""
from __future__ import annotations

import numpy as np
import pytest

from dev_field_efvm_b200 import cases, checkpoint
from oracle import pyoracle


def _fresh_oracle(builder, **kw):
    grid, params, u, ex = builder(**kw)
    c = pyoracle.OracleCase(grid, params)
    if "cylinders" in ex:
        c.set_cylinders(ex["cylinders"], ex["freestream"])
    return c, u, ex


def _check_restart(make_ctx, first: int, second: int):
    """Run `first` steps, snapshot, run `second` more; restore the snapshot into
    a new context and run `second` steps.  Returns both final states."""
    ref, u0 = make_ctx()
    ref.upload(u0)
    ref.step(first)
    snap = checkpoint.snapshot(ref)
    _, hist_ref = ref.step(second, history=True) if hasattr(ref, "marker_force") else (None, None)
    u_ref = ref.download()
    s_ref = ref.solver_state()

    new, _ = make_ctx()
    checkpoint.restore(new, snap)
    _, hist_new = new.step(second, history=True) if hasattr(new, "marker_force") else (None, None)
    u_new = new.download()
    s_new = new.solver_state()
    assert s_new.step == s_ref.step == first + second
    assert np.float64(s_new.time).view(np.uint64) == np.float64(s_ref.time).view(np.uint64)
    assert np.array_equal(u_new, u_ref), "restored fields drifted from the uninterrupted run"
    assert not np.array_equal(u_ref, u0), "the state did not move; the comparison is trivial"
    return u_ref, hist_ref, hist_new


def test_oracle_restart_pulse_bit_for_bit():
    """The reference's own restart case: 12 steps, save, 18 more."""
    def make():
        c, u, _ = _fresh_oracle(cases.restart_pulse_case)
        return c, u
    _check_restart(make, 12, 18)


def test_oracle_restart_cylinder_muscl_viscous_bit_for_bit():
    def make():
        c, u, _ = _fresh_oracle(cases.cylinder_case, nx=110, ny=41, muscl=True)
        return c, u
    _, h_ref, h_new = _check_restart(make, 4, 3)
    assert np.array_equal(h_ref, h_new)


def test_checkpoint_file_round_trip(tmp_path):
    c, u, _ = _fresh_oracle(cases.restart_pulse_case)
    c.upload(u)
    c.step(5)
    path = str(tmp_path / "ckpt.npz")
    checkpoint.save(c, path)
    snap = checkpoint.snapshot(c)
    d, _, _ = _fresh_oracle(cases.restart_pulse_case)
    checkpoint.load(d, path)
    back = checkpoint.snapshot(d)
    for k in snap:
        assert np.array_equal(np.asarray(snap[k]), np.asarray(back[k])), k


def test_checkpoint_refuses_mid_step():
    c, u, _ = _fresh_oracle(cases.restart_pulse_case)
    c.upload(u)
    c.substep()
    with pytest.raises(ValueError):
        checkpoint.snapshot(c)


@pytest.mark.gpu
def test_gpu_restart_pulse_bit_for_bit():
    from dev_field_efvm_b200.device import Context

    def make():
        grid, params, u, _ = cases.restart_pulse_case()
        return Context(grid, params), u
    _check_restart(make, 12, 18)


@pytest.mark.gpu
@pytest.mark.parametrize("precision", ["fp64", "fp32"])
def test_gpu_restart_cylinder_1100x205_bit_for_bit(precision):
    """The benchmark cylinder (IBM, viscous, MUSCL, sponge): fields, clock and
    the per-substage marker force history continue bit for bit."""
    from dev_field_efvm_b200 import abi
    from dev_field_efvm_b200.device import Context

    def make():
        grid, params, u, ex = cases.cylinder_baseline_case()
        if precision == "fp32":
            params.precision = abi.PREC_FP32_FLUX
        ctx = Context(grid, params)
        ctx.set_cylinders(ex["cylinders"], ex["freestream"])
        return ctx, u
    _, h_ref, h_new = _check_restart(make, 40, 25)
    assert np.array_equal(h_ref, h_new)
