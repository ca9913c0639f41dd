"""Workload runner: the same scripted workload through three execution modes.

* ``plain``   - the baseline GPU CA: one region per launch, one tick per launch, the host waits for
                every tick (what a game loop calling FluidSim::update per frame does).
* ``batched`` - pattern (2): every region of the workload is stepped by one launch (one CTA per
                region, many ticks per launch); host edits between ticks (rain emitters, sphere
                brushes + their wake boxes) are replayed from device buffers, and the whole script is
                captured once as a CUDA graph and replayed.
* ``batched+learned`` - pattern (4) on top of batching: every few ticks the wake-proposal network
                scores every brick and the predicted positives are pre-staged into L2 before the
                batched launch; recall and precision are scored against what the exact scheduler
                drains in the following ticks.

All modes run the identical sequence of FluidSim calls, so their states are bit-identical.
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
    """One FluidSim per region (all on one stream), initial wake boxes applied. `tune`: a dict of
    autotune knobs (engine, gate, producers, depth)."""
    from . import autotune

    sims = []
    for r in (range(wl.regions) if regions is None else regions):
        sim = vf.FluidSim(wl.world(r), stream=stream_handle)
        if tune:
            autotune.apply(sim, tune)
        for b in wl.wakes(r):
            sim.wake(*map(int, b))
        sims.append(sim)
    return sims


def _edits_before(wl, t):
    return bool(wl.edit_every) and (t % wl.edit_every) == wl.edit_every - 1


def _emits_before(wl, t):
    return bool(wl.emit_every) and (t % wl.emit_every) == 0


def run_plain(vf, wl, sims, t0: int, ticks: int, torch, stream, regions=None) -> RunResult:
    """Host-driven baseline: per tick, per region: edits, then one tick with a host sync.
    `regions`: the workload regions the sims hold (default 0..len(sims)-1)."""
    regions = list(range(len(sims))) if regions is None else list(regions)
    emitters = {r: wl.emitters(r) for r in regions}
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


def device_script(wl, nreg: int, t0: int, ticks: int, torch):
    """Device copies of the emitter lists and of every sphere edit in ticks [t0, t0+ticks).
    Returns (emit {region: (buf, n, amount)}, edits {(tick, region): (buf, n, material, wake)},
    buffers to keep alive)."""
    bufs, emit, edits = [], {}, {}
    for r in range(nreg):
        em, amt = wl.emitters(r)
        if len(em):
            b = torch.from_numpy(np.ascontiguousarray(em, np.int32)).to("cuda")
            bufs.append(b)
            emit[r] = (b, len(em), amt)
    for t in range(t0, t0 + ticks):
        if not _edits_before(wl, t):
            continue
        for r in range(nreg):
            ed = wl.edit(r, t)
            if ed is None:
                continue
            cells, m, wake = ed
            b = torch.from_numpy(np.ascontiguousarray(cells, np.int32)).to("cuda")
            bufs.append(b)
            edits[(t, r)] = (b, len(cells), m, wake)
    torch.cuda.synchronize()
    return emit, edits, bufs


def segments(wl, t0: int, ticks: int, every: int = 0):
    """Maximal tick runs without host edits inside (cut also at every `every` ticks from t0)."""
    cuts = [t for t in range(t0, t0 + ticks) if _emits_before(wl, t) or _edits_before(wl, t) or (every and (t - t0) % every == 0)]
    bounds = sorted(set([t0] + cuts + [t0 + ticks]))
    return list(zip(bounds[:-1], bounds[1:]))


def edits_at(wl, sims, emit, edits, t):
    """Enqueue the edits that act before tick t on the sims' streams (device buffers only)."""
    for r, sim in enumerate(sims):
        if _emits_before(wl, t) and r in emit:
            b, n, amt = emit[r]
            sim.emit_device_async(b.data_ptr(), n, amt)
        if (t, r) in edits:
            b, n, m, wake = edits[(t, r)]
            sim.brush_device_async(b.data_ptr(), n, m)
            sim.wake_async(*map(int, wake))


class BatchedScript:
    """The workload's ticks t0..t0+ticks as one captured CUDA graph over all regions."""

    def __init__(self, vf, wl, sims, t0: int, ticks: int, torch, stream):
        self.vf, self.wl, self.sims, self.torch, self.stream = vf, wl, sims, torch, stream
        self.t0, self.ticks = t0, ticks
        self.batch = vf.Batch(sims)
        self.emit, self.edits, self.bufs = device_script(wl, len(sims), t0, ticks, torch)
        self.batch.begin_capture()
        try:
            for a, b_ in segments(wl, t0, ticks):
                self._edits_at(a)
                self.batch.tick_async(b_ - a)
        finally:
            self.batch.end_capture()

    def _edits_at(self, t):
        edits_at(self.wl, self.sims, self.emit, self.edits, t)

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


@dataclass
class LearnedResult:
    run: RunResult
    recall: float
    precision: float
    staged: int          # bricks pre-staged over the run
    scored: int          # (brick, time) pairs with a known outcome
    stage_seconds: float  # device time of features + network + staging inside the run


def run_learned(vf, wl, sims, t0: int, ticks: int, torch, stream, mlp, stage_every: int = 4, threshold: float = 0.5) -> LearnedResult:
    """Batched execution (one launch per tick run over all regions) with the learned wake
    proposal: every `stage_every` ticks each region's bricks are scored by the network and the
    positives' atlas lines are pre-staged into L2 before the ticks run. The exact FIFO still
    decides what runs. Recall/precision are scored against the engine's own wake record
    `proposal.HORIZON` ticks later (outside the timed intervals)."""
    from . import proposal

    horizon = proposal.HORIZON
    batch = vf.Batch(sims)
    emit, edits, bufs = device_script(wl, len(sims), t0, ticks, torch)
    c0 = [s.stats().cells_total for s in sims]
    pending = []  # (tick index, region, probabilities, slots)
    tp = fp = fn = 0
    staged = 0
    dev_ms = 0.0
    stage_ms = 0.0
    try:
        for a, b in segments(wl, t0, ticks, stage_every):
            e0, e1, e2 = (torch.cuda.Event(enable_timing=True) for _ in range(3))
            e0.record(stream)
            edits_at(wl, sims, emit, edits, a)
            if (a - t0) % stage_every == 0:
                for r, sim in enumerate(sims):
                    x, n = proposal.features(sim, torch)
                    if n:
                        p = mlp.forward(x.contiguous(), torch, stream=stream.cuda_stream)
                        staged += proposal.stage(sim, p, threshold)
                        if a + horizon <= t0 + ticks:
                            pending.append((a, r, p, n, sim.stats().tick_no))
            e1.record(stream)
            batch.tick_async(b - a)
            e2.record(stream)
            e2.synchronize()
            batch.sync()
            dev_ms += e0.elapsed_time(e2)
            stage_ms += e0.elapsed_time(e1)
            # score the predictions made `horizon` ticks ago (not timed)
            while pending and pending[0][0] + horizon <= b:
                a0, r, p, n, tick0 = pending.pop(0)
                y = proposal.labels(sims[r], tick0, n, torch)
                pp, tt = p > threshold, y > 0.5
                tp += int((pp & tt).sum())
                fp += int((pp & ~tt).sum())
                fn += int((~pp & tt).sum())
    finally:
        batch.close()
    del bufs
    per = [s.stats().cells_total - c for s, c in zip(sims, c0)]
    cells = int(sum(per))
    secs = dev_ms / 1e3
    run = RunResult("batched+learned", ticks, cells, secs, cells / secs if secs > 0 else 0.0, per)
    rec = tp / (tp + fn) if tp + fn else 1.0
    prec = tp / (tp + fp) if tp + fp else 1.0
    return LearnedResult(run, rec, prec, staged, tp + fp + fn, stage_ms / 1e3)


def wall(fn):
    t = time.perf_counter()
    r = fn()
    return r, time.perf_counter() - t
