"""Reproduce the reference's published cylinder drag on the CPU oracle.

examples/cylinder_drag_validation/config.toml (440x82, first-order HLLC, RK3,
CFL 0.3, u_mean=50, p=1e5, Re=20, sponge sigma=1e4, 44,000 substeps, Cd
averaged over the last 10 %) gives Cd = 5.6312 in
examples/make_validation_plots.py:99-108.  This run takes tens of minutes on
one core, so it is a script, not a unit test; its output is recorded in
tests/golden/pins.json by hand after a run.

Usage: python oracle/pin_cylinder.py [--parallel] [--substeps N]
"""
from __future__ import annotations

import argparse
import json
import os
import sys
import time

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(_HERE))

from dev_field_efvm_b200 import cases
from oracle import pyoracle  # noqa: E402


def main() -> None:
    ap = argparse.ArgumentParser()
    ap.add_argument("--parallel", action="store_true")
    ap.add_argument("--substeps", type=int, default=44000)
    ap.add_argument("--average-frac", type=float, default=0.1)
    args = ap.parse_args()
    grid, params, u, ex = cases.cylinder_case()
    c = pyoracle.OracleCase(grid, params, parallel=args.parallel)
    c.set_cylinders(ex["cylinders"], ex["freestream"])
    c.upload(u)
    t0 = time.time()
    n = args.substeps
    full, rest = divmod(n, 3)
    _, hist = c.step(full, history=True)
    fx = list(hist[:, 0] + hist[:, 3])
    for _ in range(rest):
        c.substep()
        f = c.marker_force()
        fx.append(f[0] + f[3])
    fx = np.array(fx)
    avg_start = int((1.0 - args.average_frac) * n)
    cd = fx[avg_start:] / ex["q"]
    out = {
        "substeps": n,
        "cd_mean": float(cd.mean()),
        "cd_ptp_rel": float((cd.max() - cd.min()) / abs(cd.mean())),
        "cd_every_4000": [float(fx[i] / ex["q"]) for i in range(0, n, 4000)],
        "wall_seconds": time.time() - t0,
        "parallel": args.parallel,
    }
    print(json.dumps(out, indent=1))


if __name__ == "__main__":
    main()
