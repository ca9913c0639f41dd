"""Benchmark: cell-steps/s of the CA-water tick on B200, bit-exact engine.

Workload: the dam break (512x128x512 voxels, 4-octave noise terrain, lake below y=48, 8-wide
channel carved to y=30; a 1000-tick scenario). One step = one levelling period of the scenario,
10 ticks (FluidSim levels every 10th tick, fluid.rs:652-655), so every step holds the same mix of
sweeps and levelling. The unit of work is the cell-step: one cell drained and processed by a
tick's main loop (the reference's last_tick_cells, summed), identical on CPU and GPU because the
results are bit-exact (the window's end state is checked against the CPU oracle in the run).

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

`--impl reference` times the CPU restatement of fluid.rs (the oracle) on the same window of the
same workload, built from the same inputs (oracle/_build/libvf_inputs.so; the engine's library is
not loaded). The dam break is one world: its sweep is sequential by definition, so the reference
runs on one core. Multi-GPU runs replicas (a world does not shard): every rank steps its own copy,
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
TICKS_PER_STEP = 10
DAM_BREAK = "dam-break 512x128x512, 4-octave noise terrain, lake y<48, 8-wide channel to y=30"
# DRAM bytes (read + write) of one k_tick_par launch of one step (10 dam-break ticks, ticks
# 51..60, cold L2 as after the bench's flush): a one-off ncu capture, summarised in
# profiles/k_tick_par_dambreak_step_dram.txt. Compare with roofline.alg_bytes_per_step.
STEP_DRAM_BYTES = 2570496 + 212480


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20, help="timed steps of 10 ticks")
    ap.add_argument("--warmup", type=int, default=5, help="untimed steps of 10 ticks before them")
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", type=int, default=2)
    ap.add_argument("--scale", type=float, default=1.0)
    ap.add_argument("--engine", type=int, default=1, help="0: one-warp sweep, 1: parallel sweep")
    ap.add_argument("--gate", type=int, default=4 | (1 << 8), help="same-layer gate | lower-layer cone << 8")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-variants", action="store_true")
    ap.add_argument("--variant-ticks", type=int, default=100)
    return ap.parse_args()


def config(args) -> dict:
    """The workload and window both arms time (identical dicts)."""
    name = DAM_BREAK if (args.workload, args.scale) == (2, 1.0) else f"workload {args.workload} at scale {args.scale}"
    w0 = args.warmup * TICKS_PER_STEP
    return {"workload": name, "ticks_scenario": 1000, "ticks_per_step": TICKS_PER_STEP, "timed_ticks": [w0 + 1, w0 + args.steps * TICKS_PER_STEP],
            "l2": "flushed before every timed step (256 MiB write)", "parallelism": "replicas (one world per GPU)"}


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


# ------------------------------------------------------------------------------ CPU oracle
def _oracle_modules():
    import __graft_entry__ as ge

    return ge.load_oracle(), ge.load_oracle_inputs()


def oracle_window(wid: int, scale: float, warm: int, ticks: int, reps: int = 1):
    """Region 0 of workload `wid` on the CPU oracle (1 thread): `warm` ticks, then `ticks` timed
    ticks (the same host-edit script as the engine's runs). Returns the median of `reps` runs as
    (cell-steps/s, cell-steps, seconds, end-state digest)."""
    orc, oin = _oracle_modules()
    inp = oin.Inputs(wid, scale, 1)
    runs = []
    for _ in range(reps):
        o = oin.oracle_for(orc, inp, 0)
        em = inp.emitters(0)
        for t in range(warm):
            oin.script_step(o, inp, 0, t, em)
        c0 = o.stats()["cells"]
        if not inp.emit_every and not inp.edit_every:
            secs = o.time_ticks(ticks)
        else:
            t0 = time.perf_counter()
            for t in range(warm, warm + ticks):
                oin.script_step(o, inp, 0, t, em)
            secs = time.perf_counter() - t0
        cells = o.stats()["cells"] - c0
        runs.append((cells / secs, cells, secs, o.digest()))
        del o
    return sorted(runs)[len(runs) // 2]


def oracle_regions(wid: int, scale: float, ticks: int, threads: int, regions=None):
    """Regions of workload `wid` on the CPU oracle, ticks 0..ticks, `threads` host threads (one
    region per task; the oracle releases the GIL in its calls). Returns (cell-steps/s by wall time
    of the pool, cell-steps, seconds, {region: digest})."""
    from concurrent.futures import ThreadPoolExecutor

    orc, oin = _oracle_modules()
    inp = oin.Inputs(wid, scale, 1)
    regions = list(range(inp.regions)) if regions is None else list(regions)
    built = {r: oin.oracle_for(orc, inp, r) for r in regions}  # built before the clock starts
    emit = {r: inp.emitters(r) for r in regions}

    def run(r):
        o = built[r]
        for t in range(ticks):
            oin.script_step(o, inp, r, t, emit[r])
        return r, o.stats()["cells"], o.digest()

    t0 = time.perf_counter()
    if threads <= 1:
        res = [run(r) for r in regions]
    else:
        with ThreadPoolExecutor(threads) as ex:
            res = list(ex.map(run, regions))
    secs = time.perf_counter() - t0
    cells = sum(c for _, c, _ in res)
    return cells / secs, cells, secs, {r: d for r, _, d in res}


# ------------------------------------------------------------------------------- variants
VARIANTS = [
    (3, "64 regions, x,z in 32..256, y in 64..128, noise terrain, 1-4 water boxes (one persistent launch)"),
    (4, "ring 9x9 chunks of 128x256x128 (1152x256x1152), sea y<64, 1000 rain emitters, 1 level per 4 ticks"),
]
VARIANT_TUNE = [{"engine": 0, "producers": 7, "depth": 64, "ticks_per_launch": 10}, {"engine": 1, "gate": 4, "ticks_per_launch": 10},
                {"engine": 1, "gate": 4 | (1 << 8), "ticks_per_launch": 10}]


def _digests(sims):
    return [s.digest() for s in sims]


def variant_row(vf, torch, stream, wid: int, desc: str, ticks: int, mlp, threads: int) -> dict:
    """Workload `wid` at full size over ticks 0..ticks through the three execution modes (plain,
    batched CUDA graph with autotuned knobs, batched + learned proposal), each checked against the
    CPU oracle's end state, next to the oracle on 1 thread and on all host threads."""
    from vfwater import autotune, runner

    wl = vf.Workload(wid, 1.0, 1)
    row = {"workload": desc, "regions": wl.regions, "ticks": [1, ticks]}
    knobs = None
    if wl.regions > 1:
        knobs, table = autotune.tune(vf, wid, 1.0, torch, warmup=0, ticks=10, candidates=VARIANT_TUNE)
        row["tuned"] = knobs
        row["tune_table"] = [{k: r[k] for k in ("engine", "gate", "producers", "depth", "cell_steps_per_s")} for r in table]
    # plain: one region per launch, one tick per launch, the host waiting for every tick; the
    # regions run one after another, so a sample of them gives the mode's rate
    sample = list(range(0, wl.regions, max(1, wl.regions // 8)))
    sims = runner.make_sims(vf, wl, stream.cuda_stream, regions=sample, tune=knobs)
    plain = runner.run_plain(vf, wl, sims, 0, ticks, torch, stream, regions=sample)
    d_plain = dict(zip(sample, _digests(sims)))
    for s in sims:
        s.close()
    sims = runner.make_sims(vf, wl, stream.cuda_stream, tune=knobs)
    bat = runner.run_batched(vf, wl, sims, 0, ticks, torch, stream)
    d_bat = _digests(sims)
    for s in sims:
        s.close()
    sims = runner.make_sims(vf, wl, stream.cuda_stream, tune=knobs)
    lr = runner.run_learned(vf, wl, sims, 0, ticks, torch, stream, mlp)
    d_lr = _digests(sims)
    for s in sims:
        s.close()
    row.update({"plain": plain.cell_steps_per_s, "batched_graph": bat.cell_steps_per_s, "batched_graph_learned": lr.run.cell_steps_per_s,
                "cell_steps": bat.cells, "batched_over_plain": bat.cell_steps_per_s / plain.cell_steps_per_s,
                "learned_over_batched": lr.run.cell_steps_per_s / bat.cell_steps_per_s,
                "learned": {"recall": lr.recall, "precision": lr.precision, "staged_bricks": lr.staged, "scored": lr.scored,
                            "stage_share": lr.stage_seconds / lr.run.seconds if lr.run.seconds else None}})
    # the CPU oracle: all regions on all host threads (also the end-state check), 1 thread on a
    # sample of up to 4 regions
    v_all, c_all, s_all, d_orc = oracle_regions(wid, 1.0, ticks, threads)
    same = all(d_orc[r] == d_bat[r] == d_lr[r] for r in range(wl.regions)) and all(d_orc[r] == d for r, d in d_plain.items())
    row["plain_regions"] = len(sample)
    sample = list(range(min(4, wl.regions)))
    v1, c1, s1, _ = oracle_regions(wid, 1.0, ticks, 1, regions=sample)
    row["cpu_all_threads"] = {"value": v_all, "unit": UNIT, "cores": threads, "kind": "port", "cell_steps": c_all, "seconds": s_all,
                              "sample": f"all {wl.regions} regions, ticks 1..{ticks}, one region per task, wall time of the pool"}
    row["cpu_1thread"] = {"value": v1, "unit": UNIT, "cores": 1, "kind": "port", "cell_steps": c1, "seconds": s1,
                          "sample": f"regions {sample[0]}..{sample[-1]}, ticks 1..{ticks}, one after another"}
    row["oracle_digest_match"] = bool(same)
    return row


def headline_variants(vf, torch, stream, args, mlp) -> dict:
    """The headline window again through the batched CUDA-graph path and batched + learned."""
    from vfwater import runner

    wl = vf.Workload(args.workload, args.scale, 1)
    w0, nt = args.warmup * TICKS_PER_STEP, args.steps * TICKS_PER_STEP
    knobs = {"engine": args.engine, "gate": args.gate}
    out = {}
    sims = runner.make_sims(vf, wl, stream.cuda_stream, tune=knobs)
    runner.run_batched(vf, wl, sims, 0, w0, torch, stream)
    out["batched_graph"] = runner.run_batched(vf, wl, sims, w0, nt, torch, stream).cell_steps_per_s
    for s in sims:
        s.close()
    sims = runner.make_sims(vf, wl, stream.cuda_stream, tune=knobs)
    runner.run_batched(vf, wl, sims, 0, w0, torch, stream)
    lr = runner.run_learned(vf, wl, sims, w0, nt, torch, stream, mlp)
    out["batched_graph_learned"] = lr.run.cell_steps_per_s
    out["learned"] = {"recall": lr.recall, "precision": lr.precision, "scored": lr.scored, "staged": lr.staged,
                      "stage_share": lr.stage_seconds / lr.run.seconds if lr.run.seconds else None}
    for s in sims:
        s.close()
    return out


# ------------------------------------------------------------------------------------ arms
def reference_arm(args):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    w0, nt = args.warmup * TICKS_PER_STEP, args.steps * TICKS_PER_STEP
    v, cells, secs, _ = oracle_window(args.workload, args.scale, w0, nt)
    sample = (f"ticks {w0 + 1}..{w0 + nt} after {w0} untimed ticks ({cells} cell-steps), the oracle port of fluid.rs on 1 host thread "
              "(one world: the reference's sweep is sequential)")
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
        "config": config(args),
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
    w0, nt = args.warmup * TICKS_PER_STEP, args.steps * TICKS_PER_STEP

    def fresh():
        s = vf.FluidSim(wl.world(0), device=local, stream=stream.cuda_stream)
        s.set_sweep(args.engine, args.gate)
        for b in wl.wakes(0):
            s.wake(*map(int, b))
        s.tick(w0)  # the untimed steps (whole ticks)
        return s

    # ---- device-timed: one launch of 10 ticks per step, inputs resident, L2 flushed before each
    sim = fresh()
    flush = torch.empty(256 << 20, dtype=torch.uint8, device="cuda")  # > 126 MB L2
    s0 = sim.stats()
    evs = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(args.steps)]
    if world_size > 1:
        dist.barrier()
    torch.cuda.synchronize()
    with Clocks(local) as clk:
        for k in range(args.steps):
            flush.zero_()
            evs[k][0].record(stream)
            sim.tick_async(TICKS_PER_STEP)
            evs[k][1].record(stream)
        torch.cuda.synchronize()
    sim.sync()
    if world_size > 1:
        dist.barrier()
    s1 = sim.stats()
    dig = sim.digest()
    sim.close()
    step_ms = [a.elapsed_time(b) for a, b in evs]
    dev_ms = sum(step_ms)
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
    # ---- end to end through the public API, same ticks from the same state: per step the tick
    # call (control word host->device from pinned memory, the launch, the control block back) and
    # the download of the step's voxel changes replayed into the host world; host wall time
    sim = fresh()
    d2h = h2d = 0
    sC = sim.stats()
    if world_size > 1:
        dist.barrier()
    t0 = time.perf_counter()
    for _ in range(args.steps):
        sim.tick(TICKS_PER_STEP)
        n = sim.sync_world()
        d2h += 128 + 16 * n + 128  # control block after the tick and after the download, the changes
        h2d += 4 + 8  # the tick's control word and the download's pending count
    t1 = time.perf_counter()
    sD = sim.stats()
    e2e_same = sim.digest() == dig
    sim.close()
    e2e_secs = torch.tensor([t1 - t0], dtype=torch.float64, device="cuda")
    if world_size > 1:
        dist.all_reduce(e2e_secs, op=dist.ReduceOp.MAX)
    e2e = (sD.cells_total - sC.cells_total) * world_size / float(e2e_secs.item())
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
        "config": config(args),
        "engine": {"engine": args.engine, "gate": args.gate,
                   "sweep": "parallel exact sweep, rows on 16 warps of one CTA" if args.engine else "one-warp exact sweep + 7 prefetching warps"},
        "e2e": {"value": e2e, "unit": UNIT, "h2d_bytes_per_step": h2d // max(args.steps, 1), "d2h_bytes_per_step": d2h // max(args.steps, 1),
                "steps": args.steps, "timer": "host wall clock", "same_ticks_as_value": True, "same_end_state": bool(e2e_same)},
        "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak, "traffic": STEP_DRAM_BYTES,
                     "traffic_source": "one-off ncu capture of one step's k_tick_par launch (dram__bytes read + write)",
                     "peak_kind": peak_kind, "kernel": "k_tick_par" if args.engine else "k_tick", "alg_bytes_per_step": alg_bytes / args.steps},
        "gpu_launches": args.steps,
        "clocks": clk.summary(),
        "cells_per_step": cells / args.steps,
        "step_ms": {"min": min(step_ms), "median": statistics.median(step_ms), "max": max(step_ms)},
    }
    if rank == 0 and not args.no_cpu_baseline:
        v, c, secs, odig = oracle_window(args.workload, args.scale, w0, nt, reps=3)
        line["cpu_baseline"] = {"value": v, "unit": UNIT, "cores": 1, "kind": "port",
                                "sample": f"ticks {w0 + 1}..{w0 + nt} ({c} cell-steps, {secs:.2f} s), median of 3 runs, oracle port of fluid.rs, 1 thread"}
        line["oracle_digest_match"] = odig == dig
    if rank == 0 and not args.no_variants:
        from vfwater import proposal

        mlp, info = proposal.train_default(vf, torch)
        v = headline_variants(vf, torch, stream, args, mlp)
        v["learned"].update({"heldout": info["heldout"], "persistence": info["persistence"]})
        threads = os.cpu_count() or 1
        for wid, desc in VARIANTS:
            v[f"config{wid}"] = variant_row(vf, torch, stream, wid, desc, args.variant_ticks, mlp, threads)
        mlp.close()
        line["variants"] = v
    if rank == 0:
        print(json.dumps(line), flush=True)
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
