"""Throughput of the B200 explicit finite-volume step (one JSON line on rank 0).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
                    [--workload vortex4096|cylinder|vortex3d|batch512]

A step is one SSP-RK3 time step (three substages) of the whole case.  The
default workload is the metric's vortex family at its largest single-GPU size:
the isentropic vortex on the periodic [0,10]^2 box at 4096x4096 cells,
MUSCL (minmod) + HLLC-Thornber, SSP-RK3, CFL 0.4, FP64.  The metric is
cell-updates/s (interior cells advanced by one full RK3 step per second).

`value` is the plain FP64 path: device time with the state resident in HBM
(537 MB per state buffer, larger than L2; L2 is also flushed between timed
steps).  `chosen_form` is the FP32-flux form (FP32 reconstruction and face
fluxes, FP64 accumulation) timed the same way, with the L1 and max-norm
density error of both forms against the exact vortex and against each other
after the same number of steps with the same fixed dt, so the line says
whether the two are at equal L1 error.  `e2e` is the same metric through the
C-ABI with host buffers: every step uploads the state from pinned host memory,
steps, and downloads it, on one context (`e2e.value`); `e2e.multi_context`
adds the aggregate of several host threads with one context each, whose
copies overlap one another's kernels.  `roofline` relates the stage kernel's
algorithmic bytes (the RK3 traffic of a cell-update, 256 B, plus the 1 B
solid mask per stage with an immersed body) to its live CUDA-event duration
and the measured HBM copy bandwidth; `fp64` relates the same kernel's FP64
flops (counted by ncu, stored beside the traffic figures) to a measured FP64
GEMM.  `cpu_baseline` times the CPU oracle (the reference's algorithm
restated in C++, OpenMP over the host cores) on a bounded sample of the same
workload, and the serial oracle on one core.

Under torchrun (N > 1) the 4096^2 grid is split into N row slabs, one per
GPU (strong scaling): each stage stores its edge rows straight into the
neighbouring GPUs' ghost rows over CUDA IPC peer mappings, an 8-byte NCCL
all-reduce orders the stages, timing is the max over ranks, and `value`
counts the grid's cells.  `--replicas` restores one replica per GPU (weak
scaling); `--slabs K` runs K slabs on one GPU.
"""
from __future__ import annotations

import argparse
import ctypes as C
import json
import os
import statistics
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "Cell-updates/s on 1 B200: plain FP64 vs chosen form at equal L1 density error"
# Host threads (one context each) in the end-to-end leg.  Measured on the
# cylinder (1100x205, 9 MB each way per step): 3 threads 8.7e8, 4 threads
# 1.05e9, 6 threads 1.10e9 cell-updates/s; the large meshes are bound by the
# host link whatever the count, so they keep 3 and their pinned buffers small.
E2E_THREADS_SMALL, E2E_THREADS_LARGE = 6, 3
UNIT = "cell-updates/s"


def workload(name: str, size: int | None = None):
    from dev_field_efvm_b200 import cases
    from dev_field_efvm_b200 import abi
    if name == "cylinder":
        grid, params, u, ex = cases.cylinder_baseline_case()
        desc = {"workload": "cylinder IBM+viscous channel 2.2x0.41, 1100x205 cells (D/dx=50), "
                            "MUSCL-minmod + HLLC-Thornber, SSP-RK3, CFL 0.4, Re=20, M=0.1, FP64",
                "nx": grid.nx, "ny": grid.ny}
        return grid, params, u, ex, desc
    if name == "vortex4096":
        n = size or 4096
        grid, params, u, ex = cases.vortex_case(n, periodic=True, muscl=True, mean=(1.0, 1.0), cfl=0.4)
        desc = {"workload": f"isentropic vortex, periodic [0,10]^2, {n}x{n} cells, MUSCL-minmod + HLLC-Thornber, "
                            "SSP-RK3, CFL 0.4, FP64", "nx": grid.nx, "ny": grid.ny}
        return grid, params, u, ex, desc
    if name == "vortex3d":
        n = size or 256
        grid, params, u, ex = cases.vortex_tube_case(n, n, seam=abi.SEAM_REFERENCE)
        desc = {"workload": f"3-D isentropic vortex tube, periodic [0,10]^3, {n}x{n}x{n} cells, mean flow (1,1,1), "
                            "density modulated along z, MUSCL-minmod + HLLC-Thornber, SSP-RK3, CFL 0.4, FP64",
                "nx": grid.nx, "ny": grid.ny, "nz": grid.nz}
        return grid, params, u, ex, desc
    raise SystemExit(f"unknown workload {name}")


def measured_peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        d = json.load(open(p))
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def fp64_peaks():
    """FP64 peaks of this GPU in TFLOP/s: measured (a cuBLAS FP64 GEMM, 8192^3,
    2 N^3 flops, best of 5 after 2 warm-ups, CUDA events) and the issue peak at
    the maximum SM clock (64 FP64 FMA lanes per SM x 148 SMs x 2 flops)."""
    import torch
    n = 8192
    a = torch.randn(n, n, dtype=torch.float64, device="cuda")
    b = torch.randn_like(a)
    for _ in range(2):
        torch.matmul(a, b)
    best = float("inf")
    for _ in range(5):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        torch.matmul(a, b)
        e1.record()
        torch.cuda.synchronize()
        best = min(best, e0.elapsed_time(e1) * 1e-3)
    del a, b
    mhz = 1965.0
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        mhz = float(json.load(open(p)).get("sm_max_mhz", mhz))
    return 2.0 * n ** 3 / best / 1e12, 64 * 148 * 2 * mhz * 1e6 / 1e12


class ClockSampler:
    """SM clock and throttle reasons of the local GPU, polled through NVML every
    20 ms while the timed region runs (read-only queries)."""

    REASONS = {"hw_slowdown": 0x8, "hw_thermal_slowdown": 0x40, "sw_thermal_slowdown": 0x20, "sw_power_cap": 0x4}

    def __init__(self, gpu_index: int):
        self.idx = gpu_index
        self.samples, self.reasons, self.smax = [], set(), None
        self._stop = threading.Event()

    def __enter__(self):
        try:
            import pynvml
            pynvml.nvmlInit()
            self.nv = pynvml
            self.h = pynvml.nvmlDeviceGetHandleByIndex(self.idx)
            self.smax = float(pynvml.nvmlDeviceGetMaxClockInfo(self.h, pynvml.NVML_CLOCK_SM))
            self.t = threading.Thread(target=self._poll, daemon=True)
            self.t.start()
        except Exception:
            self.nv = None
        return self

    def _poll(self):
        while not self._stop.is_set():
            try:
                self.samples.append(float(self.nv.nvmlDeviceGetClockInfo(self.h, self.nv.NVML_CLOCK_SM)))
                mask = self.nv.nvmlDeviceGetCurrentClocksEventReasons(self.h)
                for name, bit in self.REASONS.items():
                    if mask & bit:
                        self.reasons.add(name)
            except Exception:
                pass
            time.sleep(0.02)

    def __exit__(self, *exc):
        self._stop.set()
        if self.nv:
            self.t.join(timeout=2)

    def summary(self):
        return {"sm_mhz": statistics.median(self.samples) if self.samples else None, "sm_max_mhz": self.smax,
                "reasons": sorted(self.reasons), "samples": len(self.samples)}


def cpu_baseline(grid, params, u, ex, target_seconds=12.0, one_core_sample=None):
    """The CPU oracle (OpenMP, all host threads) on a bounded number of steps,
    and the serial oracle on one core.  `one_core_sample` = (grid, u, what): a
    smaller grid of the same case for the serial leg when one serial step of the
    full case would take longer than the sample budget (the oracle's work per
    cell does not depend on the grid size)."""
    from oracle import pyoracle
    c = pyoracle.OracleCase(grid, params, parallel=True)
    if "cylinders" in ex:
        c.set_cylinders(ex["cylinders"], ex["freestream"])
    c.upload(u)
    c.step(1)  # first step includes the one-off geometry set-up
    t0 = time.perf_counter()
    c.step(1)
    one = time.perf_counter() - t0
    cells = grid.nx * grid.ny * grid.nz
    cores = pyoracle.lib(True).oracle_num_threads()
    if one > 0.5 * target_seconds:  # a large case: the timed step is the sample
        out = {"value": cells / one, "unit": UNIT, "cores": int(cores), "kind": "port",
               "sample": f"1 RK3 step of the same case after 1 untimed step ({one:.1f} s)"}
    else:
        n = max(1, min(200, int(target_seconds / max(one, 1e-6))))
        t0 = time.perf_counter()
        c.step(n)
        dt = time.perf_counter() - t0
        out = {"value": cells * n / dt, "unit": UNIT, "cores": int(cores), "kind": "port",
               "sample": f"{n} RK3 steps of the same case after 2 untimed steps ({dt:.1f} s)"}
    c.close()
    # the same oracle on one core (the reference itself is serial): a shorter sample
    g1, u1, what = (grid, u, "the same case") if one_core_sample is None else one_core_sample
    cells1 = g1.nx * g1.ny * g1.nz
    s1 = pyoracle.OracleCase(g1, params, parallel=False)
    if "cylinders" in ex:
        s1.set_cylinders(ex["cylinders"], ex["freestream"])
    s1.upload(u1)
    s1.step(1)
    t0 = time.perf_counter()
    s1.step(1)
    one1 = time.perf_counter() - t0
    m = max(1, min(100, int(0.4 * target_seconds / max(one1, 1e-6)))) if one1 < 0.4 * target_seconds else 0
    if m:
        t0 = time.perf_counter()
        s1.step(m)
        one1 = (time.perf_counter() - t0) / m
    out["one_core"] = {"value": cells1 / one1, "unit": UNIT, "cores": 1,
                       "sample": f"{max(m, 1)} RK3 step(s) of {what} after {2 if m else 1} untimed step(s), "
                                 "serial oracle"}
    s1.close()
    return out


def run_reference(args, rank, world, budget_s=90.0):
    """The reference arm: the CPU oracle of the reference's algorithm on all host
    threads, same case and metric.  The timed sample is min(K, what fits in
    about 90 s) whole RK3 steps of the full case, so the arm ends within a few
    minutes for any K; the rate is cell-updates over that sample's time."""
    if rank != 0:
        return
    grid, params, u, ex, desc = workload(args.workload, args.size)
    from oracle import pyoracle
    c = pyoracle.OracleCase(grid, params, parallel=True)
    if "cylinders" in ex:
        c.set_cylinders(ex["cylinders"], ex["freestream"])
    c.upload(u)
    c.step(min(args.warmup, 3))
    t0 = time.perf_counter()
    c.step(1)
    one = time.perf_counter() - t0
    m = max(1, min(args.steps, int(budget_s / max(one, 1e-9))))
    t0 = time.perf_counter()
    c.step(m)
    dt = time.perf_counter() - t0
    value = grid.nx * grid.ny * grid.nz * m / dt
    cores = int(pyoracle.lib(True).oracle_num_threads())
    sample = f"{m} RK3 steps of the full case ({dt:.1f} s) after {min(args.warmup, 3) + 1} untimed steps"
    line = {"impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world,
            "steps": m, "warmup": min(args.warmup, 3) + 1, "ms_per_step": 1e3 * dt / m,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic", "config": dict(desc, parallelism=f"cpu{cores}"),
            "cpu_baseline": {"value": value, "unit": UNIT, "cores": cores, "kind": "port", "sample": sample},
            "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def batch_measurement(args, local):
    """512 independent cases in one batch (n log-uniform in [32, 512]; half
    periodic vortices to t = 1, half four-quadrant Riemann problems to t = 0.05;
    MUSCL-minmod + HLLC-Thornber, FP32 fluxes with FP64 accumulation).  The
    batch runs with the persistent kernel (one launch per chunk of 16 steps over
    the packed tile queue) and, for comparison, with one launch per stage; the
    rate is the batch's total cell-updates over its device time (CUDA events on
    the batch stream around the whole run, host polling gaps included).  The
    sequential leg runs the same cases one context after another and gives the
    per-case completion percentiles the batch is compared with."""
    import torch
    torch.cuda.set_device(local)
    from dev_field_efvm_b200 import cases
    from dev_field_efvm_b200.device import Batch, Context

    grids, params, states, t_stop, kinds = cases.batch_cases()
    cells = np.array([g.nx * g.ny for g in grids], dtype=np.float64)

    def timed_run(persistent):
        warm = Batch(grids, params)
        warm.set_persistent(persistent)
        for k, u in enumerate(states):
            warm.upload(k, u)
        warm.run(t_stop, max_steps=args.warmup)  # also tunes (cached per process)
        warm.close()
        b = Batch(grids, params)
        b.set_persistent(persistent)
        for k, u in enumerate(states):
            b.upload(k, u)
        stream = torch.cuda.ExternalStream(b.stream())
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        n0 = b.launch_count()
        torch.cuda.synchronize()
        with ClockSampler(local) as clocks:
            e0.record(stream)
            res = b.run(t_stop)
            e1.record(stream)
            torch.cuda.synchronize()
        ms = e0.elapsed_time(e1)
        out = {"ms": ms, "launches": b.launch_count() - n0, "res": res, "clocks": clocks.summary(),
               "rows": b.rows(), "blocks_per_sm": b.blocks_per_sm() if persistent else None}
        b.close()
        return out

    per = timed_run(True)
    stg = timed_run(False)
    res = per["res"]
    steps = np.array([r.steps for r in res], dtype=np.float64)
    work = float((cells * steps).sum())
    comp = np.array([r.completion_ms for r in res])
    comp_stage = np.array([r.completion_ms for r in stg["res"]])

    # end to end: host states in, the whole batch run, host states out
    t0 = time.perf_counter()
    b2 = Batch(grids, params)
    for k, u in enumerate(states):
        b2.upload(k, u)
    b2.run(t_stop)
    for k in range(len(grids)):
        b2.download(k)
    e2e_s = time.perf_counter() - t0
    b2.close()
    h2d = int(sum(u.size for u in states) * 8)

    # sequential: one context per case, one after another (shortest first)
    order = np.argsort(cells * steps)
    seq_done = np.zeros(len(grids))
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    for k in order:
        c = Context(grids[k], params)
        c.upload(states[k])
        c.run_until(float(t_stop[k]))
        seq_done[k] = (time.perf_counter() - t0) * 1e3
        c.close()
    seq_s = time.perf_counter() - t0
    return {
        "workload": "512 cases, n log-uniform in [32,512] (23.4 M cells): 256 periodic vortices to t=1, 256 "
                    "four-quadrant Riemann problems to t=0.05; MUSCL-minmod + HLLC-Thornber, SSP-RK3, CFL 0.4, "
                    "FP32 fluxes + FP64 state",
        "cases": len(grids), "cells": int(cells.sum()), "cell_updates": work,
        "value": work / (per["ms"] * 1e-3), "unit": UNIT, "batch_ms": per["ms"], "gpu_launches": int(per["launches"]),
        "kernel": "persistent: one launch per chunk of 16 steps over the packed tile queue",
        "tuned_rows_per_bucket": per["rows"], "tuned_blocks_per_sm": per["blocks_per_sm"],
        "completion_ms_p50": float(np.percentile(comp, 50)), "completion_ms_p99": float(np.percentile(comp, 99)),
        "per_stage_launches": {"value": work / (stg["ms"] * 1e-3), "batch_ms": stg["ms"],
                               "gpu_launches": int(stg["launches"]),
                               "completion_ms_p50": float(np.percentile(comp_stage, 50)),
                               "completion_ms_p99": float(np.percentile(comp_stage, 99))},
        "sequential": {"value": work / seq_s, "seconds": seq_s,
                       "completion_ms_p50": float(np.percentile(seq_done, 50)),
                       "completion_ms_p99": float(np.percentile(seq_done, 99))},
        "e2e": {"value": work / e2e_s, "unit": UNIT, "h2d_bytes": h2d, "d2h_bytes": h2d,
                "note": "host states in, the whole batch run, host states out"},
        "all_finished": bool(all(r.finished for r in res)),
        "clocks": per["clocks"], "steps_max": int(steps.max()),
    }


def run_batch(args, rank, world, local):
    """The batch workload as its own line (each rank runs its own batch: weak
    scaling)."""
    m = batch_measurement(args, local)
    if rank == 0:
        peak, peak_kind = measured_peaks()
        achieved = m["value"] * 256.0 / 1e9
        line = {
            "metric": "total cell-updates/s of a 512-case batch on 1 B200", "value": world * m["value"], "unit": UNIT,
            "n_gpus": world, "steps": m["steps_max"], "warmup": args.warmup,
            "ms_per_step": m["batch_ms"] / m["steps_max"], "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32-flux/f64-state", "data": "synthetic",
            "config": {"workload": m["workload"], "cases": m["cases"], "cells": m["cells"],
                       "cell_updates": m["cell_updates"],
                       "parallelism": f"replicas{world}" if world > 1 else "single",
                       "l2": "inputs larger than L2 (2.2 GB of state)"},
            "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                         "traffic": None, "peak_source": peak_kind,
                         "kernel": "whole batch run (256 algorithmic B per cell-update over the run's device time)"},
            "cpu_baseline": None,
            "e2e": {"value": world * m["e2e"]["value"], "unit": UNIT, "h2d_bytes_per_step": m["e2e"]["h2d_bytes"],
                    "d2h_bytes_per_step": m["e2e"]["d2h_bytes"], "note": "one 'step' here is the whole batch run"},
            "gpu_launches": m["gpu_launches"],
            "clocks": m["clocks"],
            "batch": m,
        }
        print(json.dumps(line), flush=True)


def run_slabs(args, rank, world, local):
    """One grid split into row slabs (strong scaling): one slab per GPU under
    torchrun (DistPeerSlabs: CUDA IPC peers, token all-reduces ordering the
    stages), or `--slabs K` slabs on one GPU (PeerLocalSlabs: stream events).
    Each stage stores its edge rows straight into the neighbours' ghost rows
    (efvm_set_halo_peer), so no pack / send / receive / unpack runs between
    stages.  `value` counts the grid's cells over the max over ranks of the
    device time; e2e uploads every slab from pinned memory, steps, downloads."""
    import datetime
    import torch
    from dev_field_efvm_b200 import abi, slab
    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120), device_id=torch.device("cuda", local))
    grid, params, u, ex, desc = workload(args.workload, args.size)
    cells = grid.nx * grid.ny
    n_slabs = world if world > 1 else args.slabs
    parts = slab.split_rows(grid.ny, n_slabs)
    per_y = grid.bc[abi.YLO].kind == abi.BC_PERIODIC
    mine = [parts[rank]] if world > 1 else parts

    def build():
        engines = []
        for r0, rows in mine:
            e = slab.DeviceSlab(grid, params, r0, rows)
            e.ctx.upload(u[r0:r0 + rows])
            engines.append(e)
        if world > 1:
            return engines, slab.DistPeerSlabs(engines[0], slab.neighbours(rank, world, per_y))
        return engines, slab.PeerLocalSlabs(engines, per_y)

    engines, drv = build()
    drv.step(args.warmup)
    torch.cuda.synchronize()
    if dist:
        dist.barrier()
    n0 = sum(e.ctx.launch_count() for e in engines)
    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in engines]
    with ClockSampler(local) as clocks:
        for (a, _), e in zip(ev, engines):
            a.record(e.stream)
        drv.step(args.steps)
        for (_, b), e in zip(ev, engines):
            b.record(e.stream)
        torch.cuda.synchronize()
    ms = max(a.elapsed_time(b) for a, b in ev)
    launches = sum(e.ctx.launch_count() for e in engines) - n0
    st = engines[0].ctx.solver_state()
    # end to end: every slab's rows up from pinned memory, one step, down again
    host = [torch.from_numpy(np.ascontiguousarray(u[r0:r0 + rows])).pin_memory() for r0, rows in mine]
    n_e2e = max(3, min(args.steps, 10))
    torch.cuda.synchronize()
    if dist:
        dist.barrier()
    t0 = time.perf_counter()
    for _ in range(n_e2e):
        for e, h, (r0, rows) in zip(engines, host, mine):
            e.ctx.upload_ptr(h.data_ptr(), 5, 5 * grid.nx, 1)
        drv.primed = False  # the uploaded rows' ghosts come from one exchange
        drv.step(1)
        for e, h in zip(engines, host):
            e.ctx.download_ptr(h.data_ptr(), 5, 5 * grid.nx, 1)
    torch.cuda.synchronize()
    e2e_s = time.perf_counter() - t0
    if dist:
        t = torch.tensor([ms, e2e_s], dtype=torch.float64, device="cuda")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        ms, e2e_s = float(t[0].item()), float(t[1].item())
        lt = torch.tensor([launches], dtype=torch.int64, device="cuda")
        dist.all_reduce(lt)
        launches = int(lt.item())
        dist.barrier()
        del drv
        dist.destroy_process_group()
    if rank != 0:
        return
    value = cells * args.steps / (ms * 1e-3)
    peak, peak_kind = measured_peaks()
    achieved = cells * 256.0 / (ms / args.steps * 1e-3) / 1e9 / max(world, 1)
    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms / args.steps, "higher_is_better": True, "scaling": "strong",
        "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": dict(desc, parallelism=f"slabs{n_slabs}" + ("" if world > 1 else " on one GPU"),
                       halo="fused into the stage kernels (peer stores into the neighbours' ghost rows)",
                       l2="inputs larger than L2 (537 MB per state buffer)", time=st.time,
                       final_step=int(st.step)),
        "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                     "traffic": None, "peak_source": peak_kind,
                     "kernel": "whole steps per GPU (256 algorithmic B per cell-update over the step time)"},
        "cpu_baseline": None,
        "e2e": {"value": cells * n_e2e / e2e_s, "unit": UNIT, "h2d_bytes_per_step": cells * 5 * 8,
                "d2h_bytes_per_step": cells * 5 * 8, "steps": n_e2e,
                "note": "every slab uploaded from pinned memory, one step, downloaded"},
        "gpu_launches": launches,
        "clocks": clocks.summary(),
    }
    print(json.dumps(line), flush=True)


def with_params(params, **changes):
    from dev_field_efvm_b200 import abi
    p = abi.make_params(**{f: getattr(params, f) for f, _ in abi.EfvmParams._fields_})
    for k, v in changes.items():
        setattr(p, k, type(getattr(p, k))(v))
    return p


def tune(ctx, d3):
    """The library's stage autotuner on the live state (restored afterwards),
    outside every timed region: the tiling it keeps and its device ms/step."""
    from dev_field_efvm_b200 import abi
    if d3:
        return None
    ms = ctx.autotune_stage(5)
    form, rows, blocks = ctx.stage_tiling()
    return {"form": "tma" if form == abi.STAGE_TMA else "strip", "rows_per_warp": rows,
            "blocks_per_sm": blocks, "tuner_ms_per_step": ms}


def hold_stream(n_steps):
    """A sleep kernel on the current stream, long enough for the host to
    enqueue the timed steps behind it: a short step (the cylinder's is ~90 us)
    then never waits on the host between its events, so the events time the
    device.  Outside every timed pair of events."""
    import torch
    if hasattr(torch.cuda, "_sleep"):
        torch.cuda._sleep(int(2.0e6 * max(5.0, 0.2 * n_steps)))  # ~2e6 cycles per ms


def fp32_leg(args, grid, params, u, ex, flush, world, cells):
    """The chosen form on the same case: FP32 reconstruction and fluxes, FP64
    accumulation, device-timed as the FP64 leg."""
    import torch
    from dev_field_efvm_b200 import abi
    from dev_field_efvm_b200.device import Context
    ctx32 = Context(grid, with_params(params, precision=abi.PREC_FP32_FLUX))
    if "cylinders" in ex:
        ctx32.set_cylinders(ex["cylinders"], ex["freestream"])
    ctx32.upload(u)
    ctx32.step(args.warmup)
    tiling32 = tune(ctx32, False)
    s32 = torch.cuda.ExternalStream(ctx32.stream())
    ev32 = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(args.steps)]
    torch.cuda.synchronize()
    with torch.cuda.stream(s32):
        hold_stream(args.steps)
        for a, b in ev32:
            flush.zero_()
            a.record(s32)
            ctx32.step_async(1)
            b.record(s32)
    torch.cuda.synchronize()
    ms32 = sum(a.elapsed_time(b) for a, b in ev32)
    value32 = world * cells * args.steps / (ms32 * 1e-3)
    prof32 = ctx32.profile_steps(max(10, min(args.steps, 50)))
    stage32 = prof32[0] / (3 * max(10, min(args.steps, 50)))
    ctx32.close()
    return value32, ms32, stage32, tiling32


def accuracy_leg(grid, params, u, ex, t_end):
    """Density error of both forms on the vortex: FP64 and FP32-flux contexts
    from the same initial state, the same fixed dt (the CFL dt of the initial
    state) and the same number of steps to t_end; L1 (volume-weighted) and
    max-norm of rho - rho_exact for each, and of rho_fp32 - rho_fp64."""
    from dev_field_efvm_b200 import abi
    from dev_field_efvm_b200.device import Context
    v = ex["vortex"]
    with Context(grid, params) as c:
        c.upload(u)
        dt0 = c.cfl()
    n = max(1, int(round(t_end / dt0)))
    out, rho = {}, {}
    for name, prec in (("fp64", abi.PREC_FP64), ("fp32_flux", abi.PREC_FP32_FLUX)):
        with Context(grid, with_params(params, precision=prec, fixed_dt=dt0)) as c:
            c.upload(u)
            c.step(n)
            l1, linf = c.density_error(v)
            out[name] = {"l1_vs_exact": l1, "linf_vs_exact": linf}
            rho[name] = c.download()[..., 0]
    d = np.abs(rho["fp32_flux"] - rho["fp64"])
    ratio = out["fp32_flux"]["l1_vs_exact"] / out["fp64"]["l1_vs_exact"]
    return {"t": n * dt0, "steps": n, "dt": dt0, "fp64": out["fp64"], "fp32_flux": out["fp32_flux"],
            "fp32_minus_fp64": {"l1": float(d.mean()), "linf": float(d.max())},
            "l1_ratio_fp32_over_fp64": ratio,
            # equal when the FP32 form's error is within 10 % of the plain method's
            "equal_l1": bool(abs(ratio - 1.0) <= 0.10)}


def e2e_leg(grid, params, u, ex, ctx, n_steps, n_threads, dist):
    """End to end through the C-ABI: per step the state goes up from pinned host
    memory (efvm_upload_state), one RK3 step runs (efvm_step, enqueued without
    a status read), and the state comes back (efvm_download_state, which waits
    for the step) with the step's result (marker force with a body, else the
    solver state).  Returns (single-context rate, multi-context rate, threads)."""
    import torch
    from dev_field_efvm_b200.device import Context
    d3 = grid.nz > 1
    cells = grid.nx * grid.ny * grid.nz
    shape = (grid.nz, grid.ny, grid.nx, 5) if d3 else (grid.ny, grid.nx, 5)
    sk = 5 * grid.nx * grid.ny

    def make_host():
        h = torch.empty(shape, dtype=torch.float64, pin_memory=True)
        h.copy_(torch.from_numpy(u))
        return h

    def e2e_loop(c, h, n):
        ptr = h.data_ptr()
        for _ in range(n):
            if d3:
                c.upload_ptr3(ptr, 5, 5 * grid.nx, sk, 1)
                c.step_async(1)
                c.download_ptr3(ptr, 5, 5 * grid.nx, sk, 1)
            else:
                c.upload_ptr(ptr, 5, 5 * grid.nx, 1)
                c.step_async(1)
                c.download_ptr(ptr, 5, 5 * grid.nx, 1)
            if "cylinders" in ex:
                c.marker_force()
            else:
                c.solver_state()

    def timed(ctxs, hosts, n):
        for c, h in zip(ctxs, hosts):  # warm-up: graph capture, staging buffers
            e2e_loop(c, h, 2)
            h.copy_(torch.from_numpy(u))
        torch.cuda.synchronize()
        if dist:
            dist.barrier()
        threads = [threading.Thread(target=e2e_loop, args=(c, h, n)) for c, h in zip(ctxs, hosts)]
        t0 = time.perf_counter()
        for t in threads:
            t.start()
        for t in threads:
            t.join()
        s = time.perf_counter() - t0
        if dist:
            t = torch.tensor([s], dtype=torch.float64, device="cuda")
            dist.all_reduce(t, op=dist.ReduceOp.MAX)
            s = float(t.item())
        return cells * n * len(ctxs) / s

    h0 = make_host()
    single = timed([ctx], [h0], n_steps)
    extra = [Context(grid, params) for _ in range(n_threads - 1)]
    for c in extra:
        if "cylinders" in ex:
            c.set_cylinders(ex["cylinders"], ex["freestream"])
    hosts = [h0] + [make_host() for _ in extra]
    multi = timed([ctx] + extra, hosts, n_steps)
    for c in extra:
        c.close()
    return single, multi


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=200)
    ap.add_argument("--warmup", type=int, default=10)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="vortex4096", choices=["vortex4096", "cylinder", "vortex3d", "batch512"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-accuracy", action="store_true", help="skip the density-error leg (profiler captures)")
    ap.add_argument("--no-batch", action="store_true", help="skip the 512-case batch leg of the default line")
    ap.add_argument("--slabs", type=int, default=1,
                    help="vortex workloads on one GPU: split the grid into this many row slabs with the halo "
                         "exchange fused into the stage kernels")
    ap.add_argument("--replicas", action="store_true",
                    help="under torchrun: one replica of the case per GPU (weak scaling) instead of row slabs")
    ap.add_argument("--size", type=int, default=None,
                    help="vortex workloads only: a smaller n x n (x n) grid of the same case "
                         "(for profiler captures)")
    args = ap.parse_args()
    args.warmup = max(args.warmup, 3)

    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))

    if args.impl == "reference":
        if args.workload == "batch512":
            print(json.dumps({"impl": "reference", "unavailable": "the batch workload has no reference arm here; "
                              "run the default workload"}), flush=True)
            return
        run_reference(args, rank, world)
        return
    if args.workload == "batch512":
        run_batch(args, rank, world, local)
        return
    if args.workload == "vortex4096" and ((world > 1 and not args.replicas) or (world == 1 and args.slabs > 1)):
        run_slabs(args, rank, world, local)
        return

    import torch
    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120), device_id=torch.device("cuda", local))

    from dev_field_efvm_b200 import abi
    from dev_field_efvm_b200.device import Context

    grid, params, u, ex, desc = workload(args.workload, args.size)
    cells = grid.nx * grid.ny * grid.nz
    d3 = grid.nz > 1
    ctx = Context(grid, params)
    if "cylinders" in ex:
        ctx.set_cylinders(ex["cylinders"], ex["freestream"])
    ctx.upload(u)
    stream = torch.cuda.ExternalStream(ctx.stream())
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device="cuda")

    ctx.step(args.warmup)
    tiling = tune(ctx, d3)
    torch.cuda.synchronize()
    if dist:
        dist.barrier()

    # ---- device-timed steps, L2 flushed between steps --------------------
    n0 = ctx.launch_count()
    evs = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(args.steps)]
    with ClockSampler(local) as clocks:
        torch.cuda.synchronize()
        with torch.cuda.stream(stream):
            hold_stream(args.steps)
            for a, b in evs:
                flush.zero_()
                a.record(stream)
                ctx.step_async(1)
                b.record(stream)
        torch.cuda.synchronize()
    launches = ctx.launch_count() - n0
    ms = sum(a.elapsed_time(b) for a, b in evs)
    st = ctx.solver_state()  # synchronising call: reports a non-physical state
    if dist:
        t = torch.tensor([ms], dtype=torch.float64, device="cuda")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        ms = float(t.item())
    value = world * cells * args.steps / (ms * 1e-3)

    # ---- stage-kernel roofline (live CUDA events per kernel class) --------
    n_prof = max(10, min(args.steps, 50))
    prof = ctx.profile_steps(n_prof)
    stage_ms_per_launch = prof[0] / (3 * n_prof)
    mask_bytes = 1 if "cylinders" in ex else 0
    # the RK3 traffic of a cell-update: 8 state reads/writes of 32 B (2-D, 4 planes) or 40 B (3-D, 5 planes)
    bytes_per_cell_update = (320 if d3 else 256) + 3 * mask_bytes
    bytes_per_launch = cells * bytes_per_cell_update / 3.0
    achieved = bytes_per_launch / (stage_ms_per_launch * 1e-3) / 1e9
    peak, peak_kind = measured_peaks()
    traffic = None
    entry = None
    tf = os.path.join(ROOT, "profiles", "stage_kernel_traffic.json")
    if os.path.exists(tf):
        entry = json.load(open(tf)).get(args.workload) if args.size is None else None
        if entry:
            traffic = entry.get("bytes_per_launch")
    roofline = {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                "traffic": traffic, "peak_source": peak_kind,
                "kernel": ("stage3_kernel (fused 3-D MUSCL/HLLC/RK3 substage, x/y/z faces)" if d3
                           else "stage_tma_kernel (fused MUSCL/HLLC/RK3 substage, rows fed by TMA into a "
                                "shared-memory ring)" if tiling and tiling.get("form") == "tma"
                           else "stage_kernel (fused MUSCL/HLLC/RK3 substage)"),
                "bytes_per_cell_update": bytes_per_cell_update, "cells_per_launch": cells,
                "stage_ms_per_launch": stage_ms_per_launch,
                # the three stage launches per step against the graph-timed step above
                # (the per-kernel events of the profile pass wait on the host between
                # stages, so its own whole-step time is not a step of the timed loop)
                "share_of_step": 3 * stage_ms_per_launch / (ms / args.steps)}
    # The same kernel against the FP64 peak: its FP64 flops per cell-update
    # (dadd + dmul + 2 dfma thread instructions of one step's three launches,
    # counted by ncu, per cell) over the same live launch time.
    fp64 = None
    if entry and entry.get("fp64_flops_per_cell_update"):
        fpc = float(entry["fp64_flops_per_cell_update"])
        dgemm, issue = fp64_peaks()
        got = fpc * cells / 3.0 / (stage_ms_per_launch * 1e-3) / 1e12
        fp64 = {"flops_per_cell_update": fpc, "achieved": got, "peak": dgemm, "unit": "TFLOP/s", "frac": got / dgemm,
                "peak_source": "measured: cuBLAS FP64 GEMM 8192^3, best of 5", "issue_peak": issue,
                "issue_frac": got / issue, "issue_peak_source": "64 FP64 FMA lanes/SM x 148 SMs x 2 x max SM clock",
                "counted": entry.get("fp64_how", "")}

    # ---- chosen form: FP32 reconstruction/fluxes, FP64 accumulation -------
    chosen = None
    if not d3:  # 3-D meshes run in FP64 only
        value32, ms32, stage32, tiling32 = fp32_leg(args, grid, params, u, ex, flush, world, cells)
        a32 = bytes_per_launch / (stage32 * 1e-3) / 1e9
        chosen = {"precision": "fp32 reconstruction+flux, fp64 accumulation", "value": value32, "unit": UNIT,
                  "ms_per_step": ms32 / args.steps, "speedup_vs_fp64": value32 / value, "stage_tiling": tiling32,
                  "roofline": {"achieved": a32, "peak": peak, "unit": "GB/s", "frac": a32 / peak,
                               "stage_ms_per_launch": stage32}}
        if "vortex" in ex and not args.no_accuracy:
            # the same horizon in physical time at any grid size: t = 0.25
            chosen["accuracy"] = accuracy_leg(grid, params, u, ex, t_end=0.25)

    # ---- end to end through the C-ABI with pinned host buffers -----------
    n_threads = E2E_THREADS_SMALL if cells < 2_000_000 else E2E_THREADS_LARGE
    n_each = max(3, min(args.steps, 40 if cells < 2_000_000 else 10))
    e2e_single, e2e_multi = e2e_leg(grid, params, u, ex, ctx, n_each, n_threads, dist)
    e2e_single *= world
    e2e_multi *= world

    # ---- the batching configuration (512 cases, FP32 fluxes) --------------
    batch = None
    if world == 1 and args.workload == "vortex4096" and args.size is None and not args.no_batch:
        m = batch_measurement(args, local)
        batch = {k: m[k] for k in ("workload", "value", "unit", "batch_ms", "gpu_launches", "kernel",
                                    "tuned_rows_per_bucket", "tuned_blocks_per_sm", "completion_ms_p50",
                                    "completion_ms_p99", "per_stage_launches", "sequential", "e2e", "all_finished")}

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        sample = None
        if args.workload == "vortex4096" and cells > 2_000_000:
            g1, p1, u1, ex1, _ = workload(args.workload, 1024)
            sample = (g1, u1, "the same vortex at 1024x1024 (the per-cell work does not depend on the size)")
        cpu = cpu_baseline(grid, params, u, ex, one_core_sample=sample)

    if dist:
        dist.barrier()
        dist.destroy_process_group()

    if rank == 0:
        res_bytes = C.sizeof(abi.EfvmSolverState) if "cylinders" not in ex else 48
        line = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms / args.steps, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": dict(desc, parallelism=f"replicas{world}" if world > 1 else "single",
                           l2=("inputs larger than L2 (537 MB per state buffer); L2 also flushed between timed steps "
                               "(256 MB write)") if cells * 32 > 126e6 else
                              "flushed between timed steps (256 MB write)",
                           timing="CUDA events around each step on the context stream; the timed steps are "
                                  "enqueued behind a sleep kernel so no host launch gap falls between events",
                           time=st.time, final_step=int(st.step)),
            "roofline": roofline,
            "stage_tiling": tiling,
            "fp64": fp64,
            "chosen_form": chosen,
            "cpu_baseline": cpu,
            "e2e": {"value": e2e_single, "unit": UNIT, "h2d_bytes_per_step": cells * 5 * 8,
                    "d2h_bytes_per_step": cells * 5 * 8 + res_bytes, "steps": n_each,
                    "note": "one context: per step upload from pinned memory, one RK3 step, download, "
                            + ("marker-force read" if "cylinders" in ex else "solver-state read"),
                    "multi_context": {"value": e2e_multi, "unit": UNIT, "host_threads": n_threads,
                                      "steps_per_thread": n_each,
                                      "note": "one context per host thread, each its own copy of the case; "
                                              "copies of one thread overlap kernels of the others"}},
            "gpu_launches": int(launches),
            "clocks": clocks.summary(),
            "batch512": batch,
        }
        print(json.dumps(line), flush=True)


if __name__ == "__main__":
    main()
