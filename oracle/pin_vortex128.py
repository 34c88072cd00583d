"""Run the small periodic vortex benchmark case on the CPU oracle and print its
density error, for tests/golden/oracle_pins.json.

Case: periodic [0,10]^2, 128^2 cells, gamma 1.4, R 1, rho = p = T = 1 at
infinity, mean flow (1, 1), centre (5, 5), beta 5 (minimum-image exact
solution), MUSCL-minmod + HLLC (Thornber) + SSP-RK3, CFL 0.4, dz = L/n, run to
t >= 10 (examples/isentropic_vortex/main.rs with a periodic box and MUSCL).

Usage: python oracle/pin_vortex128.py [--parallel] [--t-final T]
"""
from __future__ import annotations

import argparse
import json
import os
import sys
import time

_HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(_HERE))

from dev_field_efvm_b200 import cases  # noqa: E402
from oracle import pyoracle  # noqa: E402


def main() -> None:
    ap = argparse.ArgumentParser()
    ap.add_argument("--parallel", action="store_true")
    ap.add_argument("--t-final", type=float, default=10.0)
    args = ap.parse_args()
    grid, params, u, ex = cases.vortex_case(128, periodic=True, muscl=True, mean=(1.0, 1.0), cfl=0.4)
    c = pyoracle.OracleCase(grid, params, parallel=args.parallel)
    c.upload(u)
    t0 = time.time()
    info = c.run_until(args.t_final)
    s = c.solver_state()
    l1, linf = c.density_error(ex["vortex"])
    print(json.dumps({
        "how": "python oracle/pin_vortex128.py" + (" --parallel" if args.parallel else ""),
        "t_final": args.t_final, "steps": int(s.step), "time": s.time,
        "l1": l1, "linf": linf, "wall_seconds": time.time() - t0,
    }, indent=1))


if __name__ == "__main__":
    main()
