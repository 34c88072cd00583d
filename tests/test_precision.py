"""The FP32-flux form tracks all-FP64 on seeded vortices (a short version of
the precision study in dev_field_efvm_b200/precision_study.py): the density
error against the exact solution is the FP64 one to within 1 %, and the
difference between the two density fields is small next to that error (L1 at
most 10 %, Linf at most 25 % of it; near extrema the minmod limiter can switch
branches on an FP32 rounding, which moves single cells by a slope's worth)."""
import pytest

from dev_field_efvm_b200 import precision_study

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("seed", [0, 1])
def test_fp32_flux_matches_fp64_error_on_seeded_vortex(seed):
    r = precision_study.run_seed(256, 1.0, seed)
    print(r)
    f64, f32, d = r["fp64"], r["fp32"], r["fp32_vs_fp64"]
    assert f32["steps"] == f64["steps"]
    assert abs(f32["l1_vs_exact"] - f64["l1_vs_exact"]) <= 0.01 * f64["l1_vs_exact"]
    assert d["l1"] <= 0.10 * f64["l1_vs_exact"]
    assert d["linf"] <= 0.25 * f64["linf_vs_exact"]
