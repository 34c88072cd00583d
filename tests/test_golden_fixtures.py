"""The committed oracle fixtures are what the oracle computes today (the oracle
is deterministic, so a regeneration must reproduce them bit for bit)."""
import os

import numpy as np

from dev_field_efvm_b200 import cases
from oracle import pyoracle

FIX = np.load(os.path.join(os.path.dirname(__file__), "golden", "oracle_fixtures.npz"))


def test_vortex_fixture_is_reproduced():
    grid, params, u, ex = cases.vortex_case(32, periodic=True, muscl=True, mean=(1.0, 1.0), cfl=0.4)
    assert np.array_equal(u, FIX["vortex32_init"])
    o = pyoracle.OracleCase(grid, params)
    o.upload(u)
    o.step(5)
    assert np.array_equal(o.download(), FIX["vortex32_periodic_muscl_minmod_5steps"])


def test_cylinder_fixture_is_reproduced():
    grid, params, u, ex = cases.cylinder_case(110, 41, muscl=True)
    o = pyoracle.OracleCase(grid, params)
    o.set_cylinders(ex["cylinders"], ex["freestream"])
    o.upload(u)
    info, hist = o.step(3, history=True)
    assert np.array_equal(o.download(), FIX["cylinder110x41_muscl_3steps"])
    assert np.array_equal(hist, FIX["cylinder110x41_muscl_3steps_marker_history"])
    assert np.array_equal(o.mask(), FIX["cylinder110x41_mask"])
