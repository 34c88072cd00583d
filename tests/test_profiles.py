"""The ncu-derived figures that bench.py reports beside its measurement.

bench.py reads the DRAM traffic per stage launch and the FP64 flops per
cell-update of each workload from profiles/stage_kernel_traffic.json.  For the
workloads whose state does not fit in L2, the counted traffic must sit near the
algorithmic bytes of a launch (256/3 B per cell in 2-D, 320/3 B in 3-D): far
above would mean re-reads, far below a capture of the wrong kernel.  Runs on
the CPU.
"""
import json
import os

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def load():
    with open(os.path.join(ROOT, "profiles", "stage_kernel_traffic.json")) as f:
        return json.load(f)


def test_every_bench_workload_has_counted_traffic_and_flops():
    d = load()
    for name in ("vortex4096", "cylinder", "vortex3d"):
        e = d[name]
        assert e["bytes_per_launch"] > 0 and e["fp64_flops_per_cell_update"] > 0, name
        assert "ncu" in e["how"] and "--clock-control none" in e["how"], name


def test_traffic_of_the_large_workloads_is_near_the_algorithmic_bytes():
    d = load()
    for name, cells, bytes_per_cell_update in (("vortex4096", 4096 * 4096, 256), ("vortex3d", 256 ** 3, 320)):
        algorithmic = cells * bytes_per_cell_update / 3.0
        ratio = d[name]["bytes_per_launch"] / algorithmic
        assert 0.85 < ratio < 1.15, (name, ratio)
