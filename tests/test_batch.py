"""Batches of independent cases (efvm_batch_*) against the same cases run one
context at a time: same step counts and clocks, and the same states (the batch
stage kernel runs the single-case strip code over a table of tiles)."""
from __future__ import annotations

import numpy as np
import pytest

from dev_field_efvm_b200 import abi, cases

pytestmark = pytest.mark.gpu


def rel(a, b):
    return float(np.max(np.abs(a - b)) / max(np.max(np.abs(b)), 1e-300))


def small_batch(precision):
    return cases.batch_cases(n_cases=8, seed=7, n_min=32, n_max=128, t_vortex=0.5, t_riemann=0.03,
                             precision=precision)


# FP64: the batch kernel reproduces the single-case kernel to 1e-12 (in practice
# bit for bit).  FP32 fluxes: the two kernels are separate compilations of the
# same code, whose FP32 rounding (multiply-add contraction) may differ; the
# difference stays at FP32 level (state 1e-5, clock 1e-6 relative).
@pytest.mark.parametrize("precision,tol,ttol", [(abi.PREC_FP64, 1e-12, 1e-12), (abi.PREC_FP32_FLUX, 1e-5, 1e-6)])
def test_batch_matches_single_contexts(precision, tol, ttol):
    from dev_field_efvm_b200.device import Batch, Context

    grids, params, states, t_stop, kinds = small_batch(precision)
    b = Batch(grids, params)
    for k, u in enumerate(states):
        b.upload(k, u)
    res = b.run(t_stop, chunk=4)
    exact = 0
    for k, (g, u) in enumerate(zip(grids, states)):
        c = Context(g, params)
        c.upload(u)
        c.run_until(float(t_stop[k]))
        s = c.solver_state()
        assert res[k].finished == 1 and res[k].nonphysical == 0
        assert res[k].steps == s.step, (k, kinds[k], res[k].steps, s.step)
        assert abs(res[k].time - s.time) <= ttol * s.time
        ub, uc = b.download(k), c.download()
        exact += int(np.array_equal(ub, uc))
        assert rel(ub, uc) <= tol, (k, kinds[k], rel(ub, uc))
        c.close()
    print(f"{exact} of {len(grids)} cases bit-identical to their single-context runs")


def test_chunking_does_not_change_results_and_completion_is_ordered():
    from dev_field_efvm_b200.device import Batch

    grids, params, states, t_stop, kinds = small_batch(abi.PREC_FP32_FLUX)
    out = []
    for chunk in (1, 1000):
        b = Batch(grids, params)
        for k, u in enumerate(states):
            b.upload(k, u)
        res = b.run(t_stop, chunk=chunk)
        out.append(([b.download(k) for k in range(len(grids))], res))
        b.close()
    (ua, ra), (ub, rb) = out
    for k in range(len(grids)):
        assert np.array_equal(ua[k], ub[k])
        assert ra[k].steps == rb[k].steps
    # with chunk 1 the table shrinks as cases finish; completion follows step count
    order = np.argsort([r.steps for r in ra])
    comp = np.array([ra[k].completion_ms for k in order])
    assert np.all(comp > 0) and np.all(np.diff(comp) >= -1e-3)


def test_batch_reports_nonphysical_case():
    from dev_field_efvm_b200.device import Batch, EfvmError

    grids, params, states, t_stop, kinds = small_batch(abi.PREC_FP64)
    bad = states[1].copy()
    bad[3, 3, 0] = -1.0
    b = Batch(grids, params)
    for k, u in enumerate(states):
        b.upload(k, bad if k == 1 else u)
    with pytest.raises(EfvmError) as e:
        b.run(t_stop)
    assert e.value.code == abi.ERR_NONPHYSICAL
    s = b.solver_state(0)
    assert s.time >= t_stop[0]  # the other cases ran to their stop time


def test_autotuned_rows_change_no_result():
    """The tuner times steps on the live states and restores them: a tuned
    batch and an untuned one end bit-identical."""
    from dev_field_efvm_b200.device import Batch

    grids, params, states, t_stop, kinds = small_batch(abi.PREC_FP64)
    out = []
    for tune in (True, False):
        b = Batch(grids, params)
        b.set_autotune(tune)
        for k, u in enumerate(states):
            b.upload(k, u)
        res = b.run(t_stop)
        out.append(([b.download(k) for k in range(len(grids))], [r.steps for r in res], b.rows()))
        b.close()
    (ua, sa, rows_tuned), (ub, sb, rows_plain) = out
    assert sa == sb
    for k in range(len(grids)):
        assert np.array_equal(ua[k], ub[k])
    assert any(r in (2, 4, 8) for r in rows_tuned) and rows_plain == [0, 0, 0, 0]


def test_persistent_launch_equals_per_stage_launches_bit_for_bit():
    """One persistent launch per chunk of steps (packed tile queue, per-case
    waits, set-ups inside the launch) against one launch per stage over the same
    table: the same step counts, and the same states and clocks within the
    tolerances of the single-context comparison above (the two kernels are
    separate compilations of the same strip code); the persistent form makes
    fewer launches."""
    from dev_field_efvm_b200.device import Batch

    for precision, tol, ttol in ((abi.PREC_FP64, 1e-12, 1e-12), (abi.PREC_FP32_FLUX, 1e-5, 1e-6)):
        grids, params, states, t_stop, kinds = small_batch(precision)
        out = []
        for persistent in (True, False):
            b = Batch(grids, params)
            b.set_persistent(persistent)
            b.set_autotune(False)
            for k, u in enumerate(states):
                b.upload(k, u)
            n0 = b.launch_count()
            res = b.run(t_stop, chunk=5)
            out.append(([b.download(k) for k in range(len(grids))], [(r.steps, r.time) for r in res],
                        b.launch_count() - n0, max(r.steps for r in res)))
            b.close()
        (ua, ra, la, sa), (ub, rb, lb, sb) = out
        exact = 0
        for k in range(len(grids)):
            assert ra[k][0] == rb[k][0], (precision, k, kinds[k], ra[k], rb[k])
            assert abs(ra[k][1] - rb[k][1]) <= ttol * rb[k][1]
            assert rel(ua[k], ub[k]) <= tol, (precision, k, kinds[k], rel(ua[k], ub[k]))
            exact += int(np.array_equal(ua[k], ub[k]))
        print(f"precision {precision}: {exact} of {len(grids)} cases bit-identical")
        assert la < lb  # the per-stage form launches 4 kernels per step


def test_bounded_wait_runs_out_on_an_injected_stall():
    """Failure detection of the persistent kernel without a device fault: the
    host counts one tile more for one case than the table holds, so that case's
    first stage never completes and the waits of its next stage run out after
    the limit.  The run returns EFVM_ERR_TIMEOUT within a few limits, and the
    batch and the GPU stay usable: the next run completes normally."""
    import time
    from dev_field_efvm_b200.device import Batch, EfvmError

    grids, params, states, t_stop, kinds = small_batch(abi.PREC_FP64)
    b = Batch(grids, params)
    b.set_autotune(False)
    b.set_wait_limit(0.2)
    for k, u in enumerate(states):
        b.upload(k, u)
    b.inject_stall(3)
    t0 = time.perf_counter()
    with pytest.raises(EfvmError) as e:
        b.run(t_stop, max_steps=4, chunk=4)
    assert e.value.code == abi.ERR_TIMEOUT
    assert time.perf_counter() - t0 < 10.0
    for k, u in enumerate(states):
        b.upload(k, u)
    res = b.run(t_stop, chunk=4)
    assert all(r.finished == 1 and r.nonphysical == 0 for r in res)
    b.close()
