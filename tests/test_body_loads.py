"""Per-body marker loads and torque (compute_marker_loadings_per_body,
crates/cfd_ibm/src/lib.rs:509-562) for a channel with two cylinders: the
oracle's per-body sums add up to its MarkerForce, and the GPU matches the oracle."""
import numpy as np
import pytest

from dev_field_efvm_b200 import cases
from oracle import pyoracle

CYLS = [(0.2, 0.2, 0.05), (0.62, 0.17, 0.04)]


def two_cylinder_case():
    grid, params, u, ex = cases.cylinder_case(220, 41)
    ex = dict(ex, cylinders=CYLS)
    return grid, params, u, ex


def test_oracle_body_loads_add_up_to_the_marker_force():
    grid, params, u, ex = two_cylinder_case()
    o = pyoracle.OracleCase(grid, params)
    o.set_cylinders(ex["cylinders"], ex["freestream"])
    o.upload(u)
    o.step(3)
    loads = o.body_loads(2)
    total = loads[:, :6].sum(axis=0)
    mf = o.marker_force()
    assert np.allclose(total, mf, rtol=1e-12, atol=1e-12 * np.max(np.abs(mf)))
    assert np.all(np.abs(loads[:, 6:8]) <= 1e-12 * np.max(np.abs(loads)))  # 2-D: only the z torque
    assert np.all(np.abs(loads[:, 8]) > 0)


@pytest.mark.gpu
def test_gpu_body_loads_match_the_oracle():
    from dev_field_efvm_b200.device import Context

    grid, params, u, ex = two_cylinder_case()
    o = pyoracle.OracleCase(grid, params)
    d = Context(grid, params)
    for c in (o, d):
        c.set_cylinders(ex["cylinders"], ex["freestream"])
        c.upload(u)
        c.step(5)
    got, ref = d.body_loads(2), o.body_loads(2)
    scale = np.max(np.abs(ref), axis=0)
    assert np.all(np.abs(got - ref) <= 1e-10 * np.maximum(scale, 1e-300)), (got, ref)
    assert np.allclose(got[:, :6].sum(axis=0), d.marker_force(), rtol=1e-10, atol=1e-12 * np.max(np.abs(got)))
