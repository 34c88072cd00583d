"""A few steps of the periodic vortex for profiler captures of the stage kernel.

    python -m dev_field_efvm_b200.stage_probe --n 2048 --precision fp32 --form tma --steps 4

Runs `steps` whole RK3 steps of the benchmark's vortex (periodic [0,10]^2,
MUSCL-minmod + HLLC-Thornber, CFL 0.4) at n x n cells in the chosen precision
and stage-kernel form (auto, strip or tma), with the default rows per warp or
`--rows`.  Each step launches the set-up kernel and three stage kernels, so an
`ncu -k regex:stage_ -s 4 -c 1` capture takes stage 1 of the second step.
"""
from __future__ import annotations

import argparse

from . import abi, cases
from .device import Context

FORMS = {"auto": abi.STAGE_AUTO, "strip": abi.STAGE_STRIP, "tma": abi.STAGE_TMA}


def main() -> None:
    ap = argparse.ArgumentParser()
    ap.add_argument("--n", type=int, default=2048)
    ap.add_argument("--precision", choices=["fp64", "fp32"], default="fp64")
    ap.add_argument("--form", choices=sorted(FORMS), default="auto")
    ap.add_argument("--rows", type=int, default=0)
    ap.add_argument("--steps", type=int, default=4)
    args = ap.parse_args()
    prec = abi.PREC_FP32_FLUX if args.precision == "fp32" else abi.PREC_FP64
    grid, params, u, _ = cases.vortex_case(args.n, periodic=True, muscl=True, mean=(1.0, 1.0), cfl=0.4,
                                           precision=prec)
    with Context(grid, params) as c:
        c.set_stage_tiling(FORMS[args.form], args.rows)
        c.upload(u)
        c.step(args.steps)
        form, rows, _ = c.stage_tiling()
        print(f"{args.steps} steps of the {args.n}^2 vortex, {args.precision}, "
              f"form {'tma' if form == abi.STAGE_TMA else 'strip'}, {rows} rows per warp: "
              f"step {c.solver_state().step}")


if __name__ == "__main__":
    main()
