"""Benchmark: cell-steps/s of the CA-water tick on B200, bit-exact engine.

One step = one tick of the dam-break workload (512x128x512 voxels, noise terrain, lake below
y=48, 8-wide channel carved to y=30; the 1000-tick scenario) through the engine's C ABI. The
unit of work is the cell-step: one cell drained and processed by the tick's main loop (the
reference's last_tick_cells, summed), identical for CPU and GPU because results are bit-exact.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
  python bench.py --suite      # every workload: CPU oracle (1 thread, all threads), plain GPU,
                               # batched + CUDA graph, batched + learned proposal; one JSON line each

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
    ap.add_argument("--suite", action="store_true")
    ap.add_argument("--suite-only", default="", help="comma-separated workload ids for --suite")
    ap.add_argument("--no-variants", action="store_true")
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


CPU_SAMPLE_TICKS = 500
# DRAM bytes (read + write) of one k_tick launch of one dam-break tick, from an ncu capture
# (profiles/k_tick_dambreak_full_capture.txt); compare with roofline.alg_bytes_per_step.
TICK_DRAM_BYTES = 636672


def variants(args, vf, wl, torch, stream):
    """The headline workload's timed ticks again through the batched CUDA-graph path and the
    batched + learned-proposal path (fresh sims, same warm-up, same ticks; device time)."""
    from vfwater import proposal, runner

    out = {}
    sims = runner.make_sims(vf, wl, stream.cuda_stream)
    runner.run_batched(vf, wl, sims, 0, args.warmup, torch, stream)
    r = runner.run_batched(vf, wl, sims, args.warmup, args.steps, torch, stream)
    out["batched_graph"] = r.cell_steps_per_s
    for s_ in sims:
        s_.close()
    mlp, info = proposal.train_default(vf, torch)
    sims = runner.make_sims(vf, wl, stream.cuda_stream)
    runner.run_batched(vf, wl, sims, 0, args.warmup, torch, stream)
    lr = runner.run_learned(vf, wl, sims, args.warmup, args.steps, torch, stream, mlp)
    out["batched_graph_learned"] = lr.run.cell_steps_per_s
    out["learned"] = {"recall": lr.recall, "precision": lr.precision, "scored": lr.scored, "staged": lr.staged,
                      "stage_share": lr.stage_seconds / lr.run.seconds if lr.run.seconds else None,
                      "heldout": info["heldout"], "persistence": info["persistence"]}
    for s_ in sims:
        s_.close()
    mlp.close()
    return out


# --suite: (workload id, description, warm-up ticks, timed window of ticks). Every variant runs the
# same window from the same state, so the cell-steps are identical and the rates compare directly.
SUITE = [
    (1, "basin 64^3, 16^3 water block", 0, 300),
    (2, "dam break 512x128x512", 10, 100),
    (3, "64 regions x,z in 32..256, y in 64..128, 1-4 water boxes", 0, 10),
    (4, "ring 9x9 chunks of 128x256x128, sea y<64, 1000 rain emitters", 0, 40),
    (5, "64 regions + sphere carve/fill every 10 ticks", 0, 10),
]


SUITE_TUNE_CANDIDATES = [{"producers": p, "depth": d, "ticks_per_launch": 4} for p in (4, 7) for d in (16, 64)]


def oracle_script(orc, wl, r, warm, ticks):
    """Region r of the workload on the CPU oracle: warm-up, then the timed window with the same
    emitter and edit script as the GPU runs. Returns (cell-steps, seconds, state digest)."""
    w = wl.world(r)
    i = w.info
    grid, bricks, ring = w.arrays()
    o = orc.Oracle.from_arrays((i.nx, i.ny, i.nz, i.ring_w), grid, bricks, ring)
    for b in wl.wakes(r):
        o.wake(*map(int, b))
    em, amt = wl.emitters(r)

    def step(t):
        if wl.emit_every and t % wl.emit_every == 0 and len(em):
            o.emit(em, amt)
        if wl.edit_every and t % wl.edit_every == wl.edit_every - 1:
            ed = wl.edit(r, t)
            if ed is not None:
                o.apply_brush(ed[0], ed[1])
                o.wake(*map(int, ed[2]))
        o.tick()

    for t in range(warm):
        step(t)
    c0 = o.stats()["cells"]
    if not wl.emit_every and not wl.edit_every:
        secs = o.time_ticks(ticks)
    else:
        t0 = time.perf_counter()
        for t in range(warm, warm + ticks):
            step(t)
        secs = time.perf_counter() - t0
    cells = o.stats()["cells"] - c0
    d = o.digest()
    del o
    return cells, secs, d


def cpu_suite_row(orc, wl, warm, ticks, threads):
    """All regions on the oracle with `threads` host threads (one region per task; the oracle
    releases the GIL inside its calls). Returns (cell-steps/s, cell-steps, seconds, digests)."""
    from concurrent.futures import ThreadPoolExecutor

    t0 = time.perf_counter()
    if threads == 1:
        res = [oracle_script(orc, wl, r, warm, ticks) for r in range(wl.regions)]
        secs = sum(x[1] for x in res)  # timed ticks only
    else:
        with ThreadPoolExecutor(threads) as ex:
            res = list(ex.map(lambda r: oracle_script(orc, wl, r, warm, ticks), range(wl.regions)))
        secs = time.perf_counter() - t0  # wall time of the whole pool (includes set-up)
    cells = sum(x[0] for x in res)
    return cells / secs, cells, secs, [x[2] for x in res]


def suite(args):
    """One JSON line per workload: CPU oracle 1 thread / all threads, plain GPU, batched + CUDA
    graph, batched + learned proposal, roofline fraction, recall/precision; states cross-checked."""
    import torch

    import __graft_entry__ as ge

    vf, orc = ge.load_package(), ge.load_oracle()
    from vfwater import autotune, proposal, runner

    torch.cuda.set_device(0)
    stream = torch.cuda.Stream()
    torch.cuda.set_stream(stream)
    peak, peak_kind = peaks()
    threads = os.cpu_count() or 1
    mlp, info = proposal.train_default(vf, torch)
    print(json.dumps({"suite": "proposal training", "samples": info["samples"], "collect_s": info["collect_s"], "train_s": info["train_s"],
                      "loss_first": info["loss_first"], "loss_last": info["loss_last"], "heldout": info["heldout"],
                      "persistence": info["persistence"]}), flush=True)
    only = {int(x) for x in args.suite_only.split(",") if x}
    for wid, desc, warm, ticks in SUITE:
        if only and wid not in only:
            continue
        wl = vf.Workload(wid, 1.0, 1)
        row = {"suite": wid, "workload": desc, "regions": wl.regions, "warmup_ticks": warm, "ticks": ticks, "unit": UNIT}
        # batched runs use the autotuner's knobs for many-region workloads (timed on a short window)
        tune = None
        if wl.regions > 1:
            best, _ = autotune.tune(vf, wid, 1.0, torch, warmup=2, ticks=4, candidates=SUITE_TUNE_CANDIDATES)
            tune = (best["producers"], best["depth"])
            row["tuned"] = best
        # GPU: plain (one region per launch, one tick per launch, host waits each tick)
        sims = runner.make_sims(vf, wl, stream.cuda_stream)
        if warm:
            runner.run_batched(vf, wl, sims, 0, warm, torch, stream)
        s0 = [s.stats() for s in sims]
        with Clocks(0) as clk:
            plain = runner.run_plain(vf, wl, sims, warm, ticks, torch, stream)
        s1 = [s.stats() for s in sims]
        dig_plain = [s.digest() for s in sims]
        lvl = sum(b.level_cells_total - a.level_cells_total for a, b in zip(s0, s1))
        bfs = sum(b.bfs_visits - a.bfs_visits for a, b in zip(s0, s1))
        for s_ in sims:
            s_.close()
        # GPU: batched, whole window as one CUDA graph
        sims = runner.make_sims(vf, wl, stream.cuda_stream, tune=tune)
        if warm:
            runner.run_batched(vf, wl, sims, 0, warm, torch, stream)
        bat = runner.run_batched(vf, wl, sims, warm, ticks, torch, stream)
        dig_bat = [s.digest() for s in sims]
        for s_ in sims:
            s_.close()
        # GPU: batched + learned proposal
        sims = runner.make_sims(vf, wl, stream.cuda_stream, tune=tune)
        if warm:
            runner.run_batched(vf, wl, sims, 0, warm, torch, stream)
        lr = runner.run_learned(vf, wl, sims, warm, ticks, torch, stream, mlp)
        dig_lr = [s.digest() for s in sims]
        for s_ in sims:
            s_.close()
        # CPU oracle
        c1, cells1, secs1, dig_cpu = cpu_suite_row(orc, wl, warm, ticks, 1)
        cn = None
        if wl.regions > 1:
            cn, _, _, _ = cpu_suite_row(orc, wl, warm, ticks, threads)
        same = dig_plain == dig_bat == dig_lr == dig_cpu
        alg = 10.0 * plain.cells + 5.0 * lvl + 5.0 * bfs
        row.update({
            "cell_steps": plain.cells, "bit_exact_all_variants_vs_oracle": same,
            "cpu_1_thread": c1, "cpu_all_threads": cn, "cpu_threads": threads,
            "plain_gpu": plain.cell_steps_per_s, "batched_graph": bat.cell_steps_per_s, "batched_learned": lr.run.cell_steps_per_s,
            "batched_over_plain": bat.cell_steps_per_s / plain.cell_steps_per_s if plain.cell_steps_per_s else None,
            "learned_over_plain": lr.run.cell_steps_per_s / plain.cell_steps_per_s if plain.cell_steps_per_s else None,
            "recall": lr.recall, "precision": lr.precision, "staged_bricks": lr.staged,
            "roofline": {"bound": "hbm", "alg_bytes": alg, "plain_frac": alg / plain.seconds / 1e9 / peak,
                         "batched_frac": alg / bat.seconds / 1e9 / peak, "peak": peak, "peak_kind": peak_kind},
            "clocks_plain": clk.summary(),
        })
        print(json.dumps(row), flush=True)
    mlp.close()


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
    from vfwater import replicas

    dev_ms_all, cells_all = replicas.reduce_rate(dev_ms, float(cells), device=torch.device("cuda", local))
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
        n = sim.sync_world()  # download the tick's voxel changes, replay them through set_voxel
        d2h += 128 + 16 * n + 128  # control block after the tick and after the download, changes
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
        "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak, "traffic": TICK_DRAM_BYTES,
                     "peak_kind": peak_kind, "kernel": "k_tick", "alg_bytes_per_step": alg_bytes / args.steps},
        "resident_value": resident,
        "gpu_launches": args.steps,
        "clocks": clk.summary(),
        "cells_per_step": cells / args.steps,
    }
    if rank == 0 and not args.no_variants:
        line["variants"] = variants(args, vf, wl, torch, stream)
    if rank == 0 and not args.no_cpu_baseline:
        ticks = max(args.steps, CPU_SAMPLE_TICKS)
        runs = [run_oracle(args, ticks, args.warmup) for _ in range(3)]
        v, c, secs = sorted(runs)[1]
        line["cpu_baseline"] = {"value": v, "unit": UNIT, "cores": 1, "kind": "port",
                                "sample": f"ticks {args.warmup}..{args.warmup + ticks} of the workload ({c} cell-steps, {secs:.2f} s), median of 3 runs, oracle port of fluid.rs, 1 thread"}
    if rank == 0:
        print(json.dumps(line), flush=True)
    sim.close()
    if world_size > 1:
        dist.destroy_process_group()


def main():
    args = parse()
    if args.impl == "reference":
        reference_arm(args)
    elif args.suite:
        suite(args)
    else:
        ours(args)


if __name__ == "__main__":
    main()
