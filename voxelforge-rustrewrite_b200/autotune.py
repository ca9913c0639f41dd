"""Autotuner for the tick's launch knobs.

The knobs change how fast a tick runs, never what it computes (every setting is bit-exact):
  * engine    - 0: the one-warp sweep with prefetching warps (256 threads per region);
                1: the parallel sweep, rows of the sorted order on 16 warps (512 threads per region)
  * gate      - engine 1: the pull gate / lower-layer cone radius in cells (the schedule's shape)
  * producers - engine 0: warps that prefetch upcoming cells' footprints into the shared-memory ring
  * depth     - engine 0: how many cells ahead of the sweep they may run (1..64)
  * ticks_per_launch - ticks one persistent launch runs before returning to the host

A candidate is timed on fresh copies of the workload's regions: `warmup` ticks with the default
knobs, then `ticks` timed ticks (CUDA events). The best setting per (GPU, workload id, region
size class) is cached as JSON.
"""
from __future__ import annotations

import json
import os
from pathlib import Path

DEFAULT = {"engine": 1, "gate": 4 | (1 << 8), "producers": 7, "depth": 64, "ticks_per_launch": 10}
CANDIDATES = [dict(DEFAULT, engine=0, producers=p, depth=d) for p in (2, 7) for d in (16, 64)] + [dict(DEFAULT, gate=g) for g in (2, 4, 4 | (1 << 8), 8)]


def apply(sim, knobs: dict):
    """Set a candidate's knobs on one handle (missing keys take DEFAULT's)."""
    k = dict(DEFAULT, **knobs)
    sim.set_sweep(k["engine"], k["gate"])
    sim.set_tuning(k["producers"], k["depth"])
CACHE = Path(os.environ.get("VF_TUNE_CACHE", Path(__file__).resolve().parent / "autotune_cache.json"))


def size_class(cells: int) -> str:
    for lim, name in ((1 << 20, "S"), (1 << 23, "M"), (1 << 26, "L")):
        if cells <= lim:
            return name
    return "XL"


def _key(gpu: str, wid: int, cells: int) -> str:
    return f"{gpu}|w{wid}|{size_class(cells)}"


def load_cache() -> dict:
    try:
        return json.loads(CACHE.read_text())
    except (OSError, ValueError):
        return {}


def save_cache(c: dict):
    CACHE.write_text(json.dumps(c, indent=1, sort_keys=True))


def lookup(gpu: str, wid: int, cells: int) -> dict:
    return load_cache().get(_key(gpu, wid, cells), {}).get("best", DEFAULT)


def tune(vf, wid: int, scale: float, torch, warmup: int = 10, ticks: int = 20, candidates=None, regions=None, seed: int = 1):
    """Time every candidate on the workload; cache and return the best. Returns (best, table)."""
    from . import runner

    candidates = candidates or CANDIDATES
    wl = vf.Workload(wid, scale, seed)
    gpu = torch.cuda.get_device_name()
    stream = torch.cuda.Stream()
    table = []
    for cand in candidates:
        sims = runner.make_sims(vf, wl, stream.cuda_stream, regions=regions)
        batch = vf.Batch(sims)
        batch.tick_async(warmup)
        batch.sync()
        for s in sims:
            apply(s, cand)
        batch.close()
        batch = vf.Batch(sims)  # region table re-read with the new knobs
        c0 = sum(s.stats().cells_total for s in sims)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        left = ticks
        while left > 0:
            n = min(left, dict(DEFAULT, **cand)["ticks_per_launch"])
            batch.tick_async(n)
            left -= n
        e1.record(stream)
        torch.cuda.synchronize()
        batch.sync()
        cells = sum(s.stats().cells_total for s in sims) - c0
        secs = e0.elapsed_time(e1) / 1e3
        table.append(dict(DEFAULT, **cand, cell_steps_per_s=cells / secs if secs else 0.0, cells=cells, seconds=secs))
        batch.close()
        for s in sims:
            s.close()
    best = max(table, key=lambda r: r["cell_steps_per_s"])
    cells_total = wl.resident_cells
    c = load_cache()
    knobs = {k: dict(DEFAULT, **best)[k] for k in DEFAULT}
    c[_key(gpu, wid, cells_total)] = {"best": knobs, "table": table, "scale": scale}
    save_cache(c)
    return knobs, table
