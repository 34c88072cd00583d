"""What the trained correction gains: the network shipped in
dev_field_efvm_b200/models (trained on the GPU by dev_field_efvm_b200.learned
from 2000 fine trajectories) against the plain 64^2 method on held-out seeds of
the vortex family, judged by the density L1 distance to the 256^2 FP64 solution
averaged onto 64^2 after 16 coarse steps."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def test_trained_correction_beats_the_plain_coarse_method_on_held_out_seeds():
    from dev_field_efvm_b200 import learned

    net, dt_c = learned.load_trained()
    seeds = list(range(950000, 950016))  # not used in training or in the recorded evaluation
    summary, per_case = learned.evaluate(net, seeds, dt_c, 16)
    plain, corr = np.array(per_case["plain64"]), np.array(per_case["learned64"])
    print(summary)
    assert np.mean(corr) < 0.8 * np.mean(plain)
    assert np.mean(corr < plain) >= 0.9
    assert summary["fallback_rate"] < 0.01
