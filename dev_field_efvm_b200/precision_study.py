"""Precision study: the FP32-flux form against plain FP64 on the periodic vortex.

    python -m dev_field_efvm_b200.precision_study --n 1024 --t-final 10 --seeds 20 --out study.json

For each seed the isentropic vortex on the periodic [0,10]^2 box gets a vortex
strength beta ~ U[1,5] and a centre ~ U[3,7]^2 (mean flow (1,1), MUSCL-minmod +
HLLC-Thornber, SSP-RK3), and is run twice on the GPU: all-FP64, and with the
reconstruction and fluxes in FP32 (accumulation and state in FP64).  Both runs
use the same fixed dt (CFL 0.4 on the initial state, times 0.95), so they take
the same steps to the same time.  Reported per seed: the density L1 and Linf
error of each run against the exact (minimum-image) solution, and the L1 and
Linf of the FP32 run's density against the FP64 run's.

The exact solution is not periodic: on [0,10]^2 its perturbation at distance 5
is about beta/(2 pi) 5 e^-12 (2.4e-5 for beta 5), so the error against it has a
floor near 1e-6..1e-5 at fine grids; the FP32-vs-FP64 columns are unaffected.
"""
from __future__ import annotations

import argparse
import json
import time

import numpy as np

from . import abi, cases
from .device import Context


def run_seed(n: int, t_final: float, seed: int) -> dict:
    rng = np.random.default_rng(seed)
    beta = float(rng.uniform(1.0, 5.0))
    centre = (float(rng.uniform(3.0, 7.0)), float(rng.uniform(3.0, 7.0)))
    out = {"seed": seed, "beta": beta, "centre": centre}
    grid, params, u, ex = cases.vortex_case(n, periodic=True, muscl=True, mean=(1.0, 1.0), cfl=0.4, beta=beta,
                                            centre=centre)
    probe = Context(grid, params)
    probe.upload(u)
    dt = 0.95 * probe.cfl()
    probe.close()
    steps = int(np.ceil(t_final / dt))
    params.fixed_dt = dt
    rho = {}
    for name, prec in (("fp64", abi.PREC_FP64), ("fp32", abi.PREC_FP32_FLUX)):
        params.precision = prec
        c = Context(grid, params)
        c.upload(u)
        t0 = time.perf_counter()
        c.step(steps)
        s = c.solver_state()
        wall = time.perf_counter() - t0
        l1, linf = c.density_error(ex["vortex"])
        rho[name] = c.download()[..., 0]
        out[name] = {"l1_vs_exact": l1, "linf_vs_exact": linf, "steps": int(s.step), "time": s.time,
                     "wall_s": wall}
        c.close()
    d = np.abs(rho["fp32"] - rho["fp64"])
    out["fp32_vs_fp64"] = {"l1": float(d.mean()), "linf": float(d.max())}
    out["dt"] = dt
    return out


def main() -> None:
    ap = argparse.ArgumentParser()
    ap.add_argument("--n", type=int, default=1024)
    ap.add_argument("--t-final", type=float, default=10.0)
    ap.add_argument("--seeds", type=int, default=20)
    ap.add_argument("--first-seed", type=int, default=0)
    ap.add_argument("--out", default=None)
    args = ap.parse_args()
    rows = []
    for k in range(args.first_seed, args.first_seed + args.seeds):
        r = run_seed(args.n, args.t_final, k)
        rows.append(r)
        print(json.dumps(r), flush=True)
    ratio = [r["fp32"]["l1_vs_exact"] / r["fp64"]["l1_vs_exact"] for r in rows]
    summary = {
        "n": args.n, "t_final": args.t_final, "seeds": args.seeds,
        "l1_ratio_fp32_over_fp64": {"min": min(ratio), "max": max(ratio)},
        "fp32_vs_fp64_l1_max": max(r["fp32_vs_fp64"]["l1"] for r in rows),
        "fp32_vs_fp64_linf_max": max(r["fp32_vs_fp64"]["linf"] for r in rows),
        "speedup_fp32": float(np.mean([r["fp64"]["wall_s"] / r["fp32"]["wall_s"] for r in rows])),
    }
    print(json.dumps({"summary": summary}), flush=True)
    if args.out:
        json.dump({"summary": summary, "runs": rows}, open(args.out, "w"), indent=1)


if __name__ == "__main__":
    main()
