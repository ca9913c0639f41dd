"""Workload runner: the same scripted workload through two execution modes.

* ``plain``   - the baseline GPU CA: one region per launch, one tick per launch, the host waits for
                every tick (what a game loop calling FluidSim::update per frame does).
* ``batched`` - pattern (2): every region of the workload is stepped by one launch (one CTA per
                region, many ticks per launch); host edits between ticks (rain emitters, sphere
                brushes + their wake boxes) are replayed from device buffers, and the whole script is
                captured once as a CUDA graph and replayed.

Both modes run the identical sequence of FluidSim calls, so their states are bit-identical.
The script follows the workloads' definitions: emitters act before every tick t with
t % emit_every == 0, sphere edits before every tick t with t % edit_every == edit_every - 1.
"""
from __future__ import annotations

import time
from dataclasses import dataclass, field

import numpy as np


@dataclass
class RunResult:
    mode: str
    ticks: int
    cells: int
    seconds: float          # device time between the first and the last event of the run
    cell_steps_per_s: float
    per_region_cells: list = field(default_factory=list)


def make_sims(vf, wl, stream_handle: int, regions=None, tune=None):
    """One FluidSim per region (all on one stream), initial wake boxes applied."""
    sims = []
    for r in (range(wl.regions) if regions is None else regions):
        sim = vf.FluidSim(wl.world(r), stream=stream_handle)
        if tune:
            sim.set_tuning(*tune)
        for b in wl.wakes(r):
            sim.wake(*map(int, b))
        sims.append(sim)
    return sims


def _edits_before(wl, t):
    return bool(wl.edit_every) and (t % wl.edit_every) == wl.edit_every - 1


def _emits_before(wl, t):
    return bool(wl.emit_every) and (t % wl.emit_every) == 0


def run_plain(vf, wl, sims, t0: int, ticks: int, torch, stream) -> RunResult:
    """Host-driven baseline: per tick, per region: edits, then one tick with a host sync."""
    regions = list(range(len(sims)))
    emitters = [wl.emitters(r) for r in regions]
    c0 = [s.stats().cells_total for s in sims]
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for t in range(t0, t0 + ticks):
        for r, sim in zip(regions, sims):
            if _emits_before(wl, t) and len(emitters[r][0]):
                sim.emit(emitters[r][0], emitters[r][1])
            if _edits_before(wl, t):
                ed = wl.edit(r, t)
                if ed is not None:
                    cells, m, wake = ed
                    sim.apply_brush(cells, m)
                    sim.wake(*map(int, wake))
            sim.tick(1)
    e1.record(stream)
    torch.cuda.synchronize()
    secs = e0.elapsed_time(e1) / 1e3
    per = [s.stats().cells_total - c for s, c in zip(sims, c0)]
    cells = int(sum(per))
    return RunResult("plain", ticks, cells, secs, cells / secs if secs > 0 else 0.0, per)


class BatchedScript:
    """The workload's ticks t0..t0+ticks as one captured CUDA graph over all regions."""

    def __init__(self, vf, wl, sims, t0: int, ticks: int, torch, stream):
        self.vf, self.wl, self.sims, self.torch, self.stream = vf, wl, sims, torch, stream
        self.t0, self.ticks = t0, ticks
        self.batch = vf.Batch(sims)
        self.bufs = []  # device buffers the graph reads (kept alive)
        regions = list(range(len(sims)))
        # device copies of emitter lists and of every sphere edit in the window
        self.emit = {}
        for r in regions:
            em, amt = wl.emitters(r)
            if len(em):
                b = torch.from_numpy(np.ascontiguousarray(em, np.int32)).to("cuda")
                self.bufs.append(b)
                self.emit[r] = (b, len(em), amt)
        self.edits = {}
        for t in range(t0, t0 + ticks):
            if not _edits_before(wl, t):
                continue
            for r in regions:
                ed = wl.edit(r, t)
                if ed is None:
                    continue
                cells, m, wake = ed
                b = torch.from_numpy(np.ascontiguousarray(cells, np.int32)).to("cuda")
                self.bufs.append(b)
                self.edits[(t, r)] = (b, len(cells), m, wake)
        torch.cuda.synchronize()
        # segments: maximal tick runs without host edits inside
        cuts = [t for t in range(t0, t0 + ticks) if _emits_before(wl, t) or _edits_before(wl, t)]
        bounds = sorted(set([t0] + cuts + [t0 + ticks]))
        self.batch.begin_capture()
        try:
            for a, b_ in zip(bounds[:-1], bounds[1:]):
                self._edits_at(a)
                self.batch.tick_async(b_ - a)
        finally:
            self.batch.end_capture()

    def _edits_at(self, t):
        for r, sim in enumerate(self.sims):
            if _emits_before(self.wl, t) and r in self.emit:
                b, n, amt = self.emit[r]
                sim.emit_device_async(b.data_ptr(), n, amt)
            if (t, r) in self.edits:
                b, n, m, wake = self.edits[(t, r)]
                sim.brush_device_async(b.data_ptr(), n, m)
                sim.wake_async(*map(int, wake))

    def run(self) -> RunResult:
        torch, stream = self.torch, self.stream
        c0 = [s.stats().cells_total for s in self.sims]
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        self.batch.replay()
        e1.record(stream)
        torch.cuda.synchronize()
        self.batch.sync()
        secs = e0.elapsed_time(e1) / 1e3
        per = [s.stats().cells_total - c for s, c in zip(self.sims, c0)]
        cells = int(sum(per))
        return RunResult("batched", self.ticks, cells, secs, cells / secs if secs > 0 else 0.0, per)

    def close(self):
        self.batch.close()


def run_batched(vf, wl, sims, t0: int, ticks: int, torch, stream) -> RunResult:
    s = BatchedScript(vf, wl, sims, t0, ticks, torch, stream)
    try:
        return s.run()
    finally:
        s.close()


def wall(fn):
    t = time.perf_counter()
    r = fn()
    return r, time.perf_counter() - t
