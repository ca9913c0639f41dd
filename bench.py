"""Benchmark: cell-steps/s of the CA-water tick on B200, bit-exact engine.

One step = one tick of the dam-break workload (512x128x512 voxels, noise terrain, lake below
y=48, 8-wide channel carved to y=30; the 1000-tick scenario) through the engine's C ABI. The
unit of work is the cell-step: one cell drained and processed by the tick's main loop (the
reference's last_tick_cells, summed), identical for CPU and GPU because results are bit-exact.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

Multi-GPU runs replicas (a single world does not shard): every rank steps its own copy, and
value = all ranks' cell-steps / the slowest rank's device time.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time
from pathlib import Path

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

METRIC = "cell-steps/s on 1 B200 (bit-exact): learned+batched vs plain GPU CA vs fluid.rs CPU"
UNIT = "cell-steps/s"
WORKLOAD = {"workload": "dam-break 512x128x512, noise terrain, lake y<48, 8-wide channel to y=30", "ticks_scenario": 1000}


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=100)
    ap.add_argument("--warmup", type=int, default=10)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", type=int, default=2)
    ap.add_argument("--scale", type=float, default=1.0)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--e2e-steps", type=int, default=20)
    return ap.parse_args()


def peaks():
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        d = json.loads(p.read_text())
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


class Clocks:
    """nvidia-smi samples during the timed region."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
         "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index: int):
        self.index = index
        self.proc = None
        self.lines = []

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--id={self.index}", f"--query-gpu={self.Q}", "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except FileNotFoundError:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def __exit__(self, *a):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self):
        sm, mx, reasons = [], 0.0, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            f = [x.strip() for x in ln.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                mx = max(mx, float(f[2]))
            except ValueError:
                continue
            for n, v in zip(names, f[5:9]):
                if v.lower() == "active":
                    reasons.add(n)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": mx or None, "reasons": sorted(reasons), "samples": len(sm)}


def run_oracle(args, ticks_timed, warm):
    """The CPU restatement of fluid.rs on this host: same workload, same ticks; 1 core."""
    import __graft_entry__ as ge

    vf, orc = ge.load_package(), ge.load_oracle()
    wl = vf.Workload(args.workload, args.scale, 1)
    w = wl.world(0)
    i = w.info
    grid, bricks, ring = w.arrays()
    o = orc.Oracle.from_arrays((i.nx, i.ny, i.nz, i.ring_w), grid, bricks, ring)
    for b in wl.wakes(0):
        o.wake(*map(int, b))
    o.tick(warm)
    c0 = o.stats()["cells"]
    secs = o.time_ticks(ticks_timed)
    cells = o.stats()["cells"] - c0
    return cells / secs, cells, secs


def reference_arm(args):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    v, cells, secs = run_oracle(args, args.steps, args.warmup)
    sample = f"{args.steps} ticks after {args.warmup} warm-up ticks of the workload, oracle port of fluid.rs, 1 thread"
    line = {
        "impl": "reference",
        "metric": METRIC,
        "value": v,
        "unit": UNIT,
        "n_gpus": args.gpus,
        "steps": args.steps,
        "warmup": args.warmup,
        "ms_per_step": 1e3 * secs / max(args.steps, 1),
        "higher_is_better": True,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": "f32",
        "data": "synthetic",
        "config": dict(WORKLOAD, parallelism="replicas"),
        "cpu_baseline": {"value": v, "unit": UNIT, "cores": 1, "kind": "port", "sample": sample},
        "e2e": {"value": v, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


def ours(args):
    import torch
    import torch.distributed as dist

    import __graft_entry__ as ge

    world_size = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    if world_size > 1:
        from datetime import timedelta

        dist.init_process_group("nccl", timeout=timedelta(seconds=300), device_id=torch.device("cuda", local))
    vf = ge.load_package()
    stream = torch.cuda.Stream()  # the engine, the L2 flush and the timing events share it
    torch.cuda.set_stream(stream)
    wl = vf.Workload(args.workload, args.scale, 1)
    world = wl.world(0)
    sim = vf.FluidSim(world, device=local, stream=stream.cuda_stream)
    for b in wl.wakes(0):
        sim.wake(*map(int, b))
    sim.tick(args.warmup)  # W warm-up steps (whole ticks)
    flush = torch.empty(256 << 20, dtype=torch.uint8, device="cuda")  # > 126 MB L2
    s0 = sim.stats()
    evs = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(args.steps)]
    if world_size > 1:
        dist.barrier()
    torch.cuda.synchronize()
    with Clocks(local) as clk:
        for k in range(args.steps):
            flush.zero_()  # L2 flushed between timed steps
            evs[k][0].record(stream)
            sim.tick_async(1)
            evs[k][1].record(stream)
        torch.cuda.synchronize()
    sim.sync()
    if world_size > 1:
        dist.barrier()
    s1 = sim.stats()
    dev_ms = sum(a.elapsed_time(b) for a, b in evs)
    cells = s1.cells_total - s0.cells_total
    lvl = s1.level_cells_total - s0.level_cells_total
    bfs = s1.bfs_visits - s0.bfs_visits
    t = torch.tensor([dev_ms, float(cells)], dtype=torch.float64, device="cuda")
    if world_size > 1:
        tmax = t.clone()
        dist.all_reduce(tmax, op=dist.ReduceOp.MAX)
        tsum = t.clone()
        dist.all_reduce(tsum, op=dist.ReduceOp.SUM)
        dev_ms_all, cells_all = float(tmax[0]), float(tsum[1])
    else:
        dev_ms_all, cells_all = dev_ms, float(cells)
    value = cells_all / (dev_ms_all / 1e3)
    # algorithmic bytes: 10 per cell-step (u8 material + f32 volume read and written), 5 per
    # level-fill cell and per pressure-BFS visit (read)
    alg_bytes = 10.0 * cells + 5.0 * lvl + 5.0 * bfs
    peak, peak_kind = peaks()
    achieved = alg_bytes / (dev_ms / 1e3) / 1e9
    # resident variant: all timed ticks in one persistent launch (state stays in L2)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    sA = sim.stats()
    e0.record(stream)
    sim.tick_async(args.steps)
    e1.record(stream)
    torch.cuda.synchronize()
    sim.sync()
    sB = sim.stats()
    resident = (sB.cells_total - sA.cells_total) / (e0.elapsed_time(e1) / 1e3)
    # end to end through the public API: tick + download of the step's voxel changes + replay
    # into the host world, host wall time
    d2h = 0
    h2d = 0
    sC = sim.stats()
    t0 = time.perf_counter()
    for _ in range(args.e2e_steps):
        sim.tick(1)
        ch = sim.download_changes()
        for x, y, z, m in ch:
            world.set_voxel(int(x), int(y), int(z), int(m))
        d2h += 128 + 16 * len(ch) + 128  # control block after the tick and after the download, changes
        h2d += 4 + 8  # the tick's control word and the download's pending count
    t1 = time.perf_counter()
    sD = sim.stats()
    e2e = (sD.cells_total - sC.cells_total) / (t1 - t0)
    line = {
        "metric": METRIC,
        "value": value,
        "unit": UNIT,
        "n_gpus": world_size,
        "steps": args.steps,
        "warmup": args.warmup,
        "ms_per_step": dev_ms_all / args.steps,
        "higher_is_better": True,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": "f32",
        "data": "synthetic",
        "config": dict(WORKLOAD, parallelism=f"replicas x{world_size}", l2="flushed before every timed step (256 MiB write)",
                       engine="exact sweep, one warp per region"),
        "e2e": {"value": e2e, "unit": UNIT, "h2d_bytes_per_step": h2d // max(args.e2e_steps, 1), "d2h_bytes_per_step": d2h // max(args.e2e_steps, 1),
                "steps": args.e2e_steps, "timer": "host wall clock"},
        "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak, "traffic": None,
                     "peak_kind": peak_kind, "kernel": "k_tick", "alg_bytes_per_step": alg_bytes / args.steps},
        "resident_value": resident,
        "gpu_launches": args.steps,
        "clocks": clk.summary(),
        "cells_per_step": cells / args.steps,
    }
    if rank == 0 and not args.no_cpu_baseline:
        v, c, secs = run_oracle(args, args.steps, args.warmup)
        line["cpu_baseline"] = {"value": v, "unit": UNIT, "cores": 1, "kind": "port",
                                "sample": f"same {args.steps} ticks after {args.warmup} warm-up ticks, oracle port of fluid.rs, 1 thread ({secs:.2f} s)"}
    if rank == 0:
        print(json.dumps(line), flush=True)
    sim.close()
    if world_size > 1:
        dist.destroy_process_group()


def main():
    args = parse()
    if args.impl == "reference":
        reference_arm(args)
    else:
        ours(args)


if __name__ == "__main__":
    main()
