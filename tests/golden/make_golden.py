"""Regenerate the per-cell golden fixtures of tests/golden/ from the CPU oracle.

    python tests/golden/make_golden.py

The oracle is pinned against the reference's own published runs
(tests/test_oracle_pins.py); these fixtures freeze its output on small cases so
the GPU tests can also compare against committed numbers.  The cylinder drag
entry of oracle_pins.json comes from `python oracle/pin_cylinder.py` (a
16-minute serial run) and is copied here by hand.
"""
import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))

from dev_field_efvm_b200 import abi  # noqa: E402
from dev_field_efvm_b200 import cases
from oracle import pyoracle  # noqa: E402


def main():
    out = {}
    grid, params, u, ex = cases.vortex_case(32, periodic=True, muscl=True, mean=(1.0, 1.0), cfl=0.4)
    o = pyoracle.OracleCase(grid, params)
    o.upload(u)
    o.step(5)
    out["vortex32_periodic_muscl_minmod_5steps"] = o.download()
    out["vortex32_init"] = u
    grid, params, u, ex = cases.cylinder_case(110, 41, muscl=True)
    o = pyoracle.OracleCase(grid, params)
    o.set_cylinders(ex["cylinders"], ex["freestream"])
    o.upload(u)
    info, hist = o.step(3, history=True)
    out["cylinder110x41_muscl_3steps"] = o.download()
    out["cylinder110x41_muscl_3steps_marker_history"] = hist
    out["cylinder110x41_init"] = u
    out["cylinder110x41_mask"] = o.mask()
    np.savez_compressed(os.path.join(HERE, "oracle_fixtures.npz"), **out)
    print("wrote", sorted(out))


if __name__ == "__main__":
    main()
