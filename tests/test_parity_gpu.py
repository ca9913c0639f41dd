"""Bit-exact parity of the CUDA engine (through the C ABI) against the oracle, after every tick.

Bar: materials and f32 partial volumes bit-identical, FIFO and level-seed list identical in
order, on every tick (src/fluid.rs semantics). Sizes are scaled so the oracle finishes in
seconds; full sizes are covered by the digest tests.
"""
import numpy as np
import pytest

from conftest import assert_same_digest, assert_same_state, oracle_for

pytestmark = pytest.mark.gpu
STONE, WATER = 3, 5


def pair(vf, orc, world):
    o = oracle_for(orc, world)
    sim = vf.FluidSim(world, device=0)
    return sim, o


def test_basin_300_ticks_bit_exact(vf, orc):
    """Workload 1 (64^3 basin): full state + FIFO every tick for 300 ticks."""
    wl = vf.Workload(1)
    sim, o = pair(vf, orc, wl.world(0))
    for box in wl.wakes(0):
        sim.wake(*map(int, box))
        o.wake(*map(int, box))
    for t in range(1, 301):
        ch_g = sim.tick()
        ch_o = o.tick()
        assert ch_g == ch_o, f"changed flag differs at tick {t}"
        if t <= 40 or t % 10 == 0:
            assert_same_state(sim, o, (-1, 0, -1, 66, 65, 66), t)
        else:
            assert_same_digest(sim, o, t)
        assert sim.last_tick_cells() == o.last_tick_cells()
    assert sim.partial_count() == o.partial_count()


def basin(vf):
    w = vf.World(64, 32, 64)
    w.fill_box(0, 0, 0, 63, 3, 63, STONE)
    w.fill_box(0, 4, 0, 63, 31, 0, STONE)
    w.fill_box(0, 4, 63, 63, 31, 63, STONE)
    w.fill_box(0, 4, 0, 0, 31, 63, STONE)
    w.fill_box(63, 4, 0, 63, 31, 63, STONE)
    return w


def test_column_falls_spreads_and_conserves_volume(vf, orc):  # src/fluid.rs:752-771
    w = basin(vf)
    w.fill_box(30, 10, 30, 33, 25, 33, WATER)
    sim, o = pair(vf, orc, w)
    sim.wake(29, 9, 29, 34, 26, 34)
    o.wake(29, 9, 29, 34, 26, 34)
    before = o.total(0, 0, 0, 64, 32, 64)
    for t in range(1, 2001):
        sim.tick()
        o.tick()
        assert_same_digest(sim, o, t)
        if o.idle():
            assert sim.idle()
            break
    assert_same_state(sim, o, (-1, 0, -1, 66, 33, 66))
    m, p = sim.export_box(0, 0, 0, 64, 32, 64)
    vol = np.where(p > 0, p, (m == WATER).astype(np.float32)).astype(np.float64)
    after = vol.sum()
    assert abs(before - after) < 0.05 * before
    assert vol[:, 6:, :].sum() < 1.0
    assert sim.volume(10, 4, 10) > 0.0 or sim.volume(50, 4, 50) > 0.0


def test_displace_moves_water_up(vf, orc):  # src/fluid.rs:773-782
    w = basin(vf)
    w.fill_box(1, 4, 1, 62, 5, 62, WATER)
    sim, o = pair(vf, orc, w)
    sim.displace(20, 4, 20)
    sim.apply_voxel_edits([(20, 4, 20, STONE)])
    o.displace(20, 4, 20)
    o.set_voxel(20, 4, 20, STONE)
    m, _ = sim.export_box(20, 6, 20, 1, 1, 1)
    assert m[0, 0, 0] == WATER
    assert not sim.idle()
    assert_same_state(sim, o, (-1, 0, -1, 66, 33, 66))


def test_hole_under_a_lake_drains_it_level(vf, orc):  # src/fluid.rs:800-817
    w = basin(vf)
    w.fill_box(1, 4, 1, 62, 7, 62, WATER)
    w.fill_box(1, 1, 1, 20, 2, 20, 0)
    w.set_voxel(10, 3, 10, 0)
    sim, o = pair(vf, orc, w)
    sim.wake(9, 2, 9, 11, 5, 11)
    o.wake(9, 2, 9, 11, 5, 11)
    for t in range(1, 401):
        sim.tick()
        o.tick()
        if t % 20 == 0:
            assert_same_digest(sim, o, t)
    assert_same_state(sim, o, (-1, 0, -1, 66, 33, 66), 400)
    assert sim.volume(5, 1, 5) > 0.5
    assert abs(sim.volume(12, 7, 10) - sim.volume(50, 7, 50)) < 0.2


@pytest.mark.parametrize("wid,scale,ticks", [(2, 0.125, 120), (3, 0.05, 80), (4, 0.12, 60), (5, 0.05, 60)])
def test_workloads_scaled_every_tick(vf, orc, wid, scale, ticks):
    """Scaled dam break / regions / ring + rain / regions + sphere edits: digest every tick."""
    wl = vf.Workload(wid, scale, 1)
    for r in range(wl.regions):
        sim, o = pair(vf, orc, wl.world(r))
        for box in wl.wakes(r):
            sim.wake(*map(int, box))
            o.wake(*map(int, box))
        em, amt = wl.emitters(r)
        for t in range(ticks):
            if wl.emit_every and t % wl.emit_every == 0 and len(em):
                sim.emit(em, amt)
                o.emit(em, amt)
            ed = wl.edit(r, t)
            if ed is not None:
                cells, m, wake = ed
                n_g = sim.apply_brush(cells, m)
                n_o = o.apply_brush(cells, m)
                assert n_g == n_o
                sim.wake(*map(int, wake))
                o.wake(*map(int, wake))
            sim.tick()
            o.tick()
            assert_same_digest(sim, o, t + 1)
            assert sim.last_tick_cells() == o.last_tick_cells()
        sim.close()


def test_batched_regions_match_individual_oracles(vf, orc):
    """One launch over many regions (one CTA each) equals each region's own oracle."""
    wl = vf.Workload(3, 0.08, 7)
    sims, oracles = [], []
    for r in range(wl.regions):
        sim, o = pair(vf, orc, wl.world(r))
        for box in wl.wakes(r):
            sim.wake(*map(int, box))
            o.wake(*map(int, box))
        sims.append(sim)
        oracles.append(o)
    for step in range(4):
        vf.batch_tick(sims, 10)
        for o in oracles:
            o.tick(10)
        for r, (s, o) in enumerate(zip(sims, oracles)):
            assert_same_digest(s, o, (step + 1) * 10)


def test_download_changes_keeps_host_world_coherent(vf, orc):
    wl = vf.Workload(1)
    w = wl.world(0)
    sim, o = pair(vf, orc, w)
    for box in wl.wakes(0):
        sim.wake(*map(int, box))
        o.wake(*map(int, box))
    for _ in range(5):
        sim.tick(10)
        o.tick(10)
        sim.sync_world()
    om, _ = o.export_box(0, 0, 0, 64, 64, 64)
    hm = np.array([[[w.get_voxel(x, y, z) for x in range(64)] for y in range(64)] for z in range(64)], np.uint8)
    assert np.array_equal(hm, om)


def test_update_matches_reference_accumulator(vf, orc):
    wl = vf.Workload(1)
    sim, o = pair(vf, orc, wl.world(0))
    for box in wl.wakes(0):
        sim.wake(*map(int, box))
        o.wake(*map(int, box))
    for dt in [0.016, 0.033, 0.1, 0.5, 0.01, 0.2, 0.07, 0.0]:
        sim.update(dt)
        o.update(dt)
        assert sim.stats().tick_no == o.tick_no()
        assert_same_digest(sim, o)


def test_partials_export_and_set_partial(vf, orc):
    wl = vf.Workload(1)
    sim, o = pair(vf, orc, wl.world(0))
    for box in wl.wakes(0):
        sim.wake(*map(int, box))
        o.wake(*map(int, box))
    sim.tick(60)
    o.tick(60)
    xyz, vol = sim.partials()
    assert len(vol) == o.partial_count() == sim.partial_count()
    for (x, y, z), v in zip(xyz[:200], vol[:200]):
        assert np.float32(o.volume(int(x), int(y), int(z))) == v
    # restore into a fresh sim the way saves do (src/app/saves.rs:251-256)
    sim.reset()
    o.reset()
    for (x, y, z), v in zip(xyz, vol):
        sim.set_partial(int(x), int(y), int(z), float(v))
        o.set_partial(int(x), int(y), int(z), float(v))
        sim.wake(int(x), int(y), int(z), int(x), int(y), int(z))
        o.wake(int(x), int(y), int(z), int(x), int(y), int(z))
    for t in range(10):
        sim.tick()
        o.tick()
        assert_same_digest(sim, o, t + 1)


def _oracle_script(wl, oracles, t0, ticks):
    for t in range(t0, t0 + ticks):
        for r, o in enumerate(oracles):
            if wl.emit_every and t % wl.emit_every == 0:
                em, amt = wl.emitters(r)
                if len(em):
                    o.emit(em, amt)
            if wl.edit_every and t % wl.edit_every == wl.edit_every - 1:
                ed = wl.edit(r, t)
                if ed is not None:
                    cells, m, wake = ed
                    o.apply_brush(cells, m)
                    o.wake(*map(int, wake))
            o.tick()


@pytest.mark.parametrize("wid,scale,ticks", [(4, 0.12, 24), (5, 0.05, 40), (3, 0.06, 30)])
def test_batched_graph_script_matches_oracle(vf, orc, wid, scale, ticks):
    """One CUDA graph over all regions (ticks, device-side emitters / brushes / wakes) equals the
    oracle running the same script."""
    import torch

    from vfwater import runner

    stream = torch.cuda.Stream()
    wl = vf.Workload(wid, scale, 3)
    sims = runner.make_sims(vf, wl, stream.cuda_stream)
    oracles = []
    for r in range(wl.regions):
        o = oracle_for(orc, wl.world(r))
        for b in wl.wakes(r):
            o.wake(*map(int, b))
        oracles.append(o)
    res = runner.run_batched(vf, wl, sims, 0, ticks, torch, stream)
    _oracle_script(wl, oracles, 0, ticks)
    assert res.cells == sum(o.stats()["cells"] for o in oracles)
    for s, o in zip(sims, oracles):
        assert_same_digest(s, o, ticks)


def test_plain_and_batched_modes_agree(vf):
    import torch

    from vfwater import runner

    stream = torch.cuda.Stream()
    wl = vf.Workload(5, 0.05, 9)
    a = runner.make_sims(vf, wl, stream.cuda_stream)
    b = runner.make_sims(vf, wl, stream.cuda_stream, tune={"engine": 0, "producers": 2, "depth": 16})
    ra = runner.run_plain(vf, wl, a, 0, 25, torch, stream)
    rb = runner.run_batched(vf, wl, b, 0, 25, torch, stream)
    assert ra.cells == rb.cells
    for x, y in zip(a, b):
        assert x.digest() == y.digest()


def test_download_changes_in_small_batches(vf, orc):
    """Pending changes taken a few at a time: every changed voxel arrives exactly once."""
    import ctypes as C

    wl = vf.Workload(1)
    w = wl.world(0)
    sim, o = pair(vf, orc, w)
    for box in wl.wakes(0):
        sim.wake(*map(int, box))
        o.wake(*map(int, box))
    sim.tick(30)
    o.tick(30)
    seen = {}
    L = vf.lib()
    buf = (vf.Voxel * 97)()
    while True:
        n = C.c_uint64()
        sim._check(L.vf_fluid_download_changes(sim.h, buf, 97, C.byref(n)), "changes")
        got = min(n.value, 97)
        for v in buf[:got]:
            key = (v.x, v.y, v.z)
            assert key not in seen
            seen[key] = v.m
        if n.value <= 97:
            break
    for (x, y, z), m in seen.items():
        w.set_voxel(x, y, z, m)
    om, _ = o.export_box(0, 0, 0, 64, 64, 64)
    hm = np.array([[[w.get_voxel(x, y, z) for x in range(64)] for y in range(64)] for z in range(64)], np.uint8)
    assert np.array_equal(hm, om)


def test_deep_lake_searches_hit_their_budgets(vf, orc):
    """A lake 56 deep drained through a hole in its floor: pressure searches from the bottom
    exhaust the 512-entry budget and the 24 side checks at the start level before they reach the
    surface, and the tick's 4096-pull budget binds. State and counters match every tick."""
    w = vf.World(48, 72, 48)
    w.fill_box(0, 0, 0, 47, 3, 47, 3)          # stone floor
    w.fill_box(0, 4, 0, 47, 71, 1, 3)          # walls
    w.fill_box(0, 4, 46, 47, 71, 47, 3)
    w.fill_box(0, 4, 0, 1, 71, 47, 3)
    w.fill_box(46, 4, 0, 47, 71, 47, 3)
    w.fill_box(2, 4, 2, 45, 59, 45, 5)         # water, 56 deep
    w.fill_box(20, 0, 20, 27, 3, 27, 0)        # a drain hole through the floor
    sim = vf.FluidSim(w)
    o = oracle_for(orc, w)
    for s_ in (sim, o):
        s_.wake(0, 0, 0, 47, 71, 47)
    most = 0
    for t in range(40):
        before = o.stats()["pull_attempts"]
        sim.tick()
        o.tick()
        most = max(most, o.stats()["pull_attempts"] - before)
        assert_same_digest(sim, o, t + 1)
    st = o.stats()
    assert most == 4096  # the per-tick pull budget bound
    assert st["bfs_visits"] > 64 * st["pull_nonempty"] > 0  # long searches (over 100 entries on average)


@pytest.mark.parametrize("global_only", [False, True])
def test_parallel_sweep_search_contexts(vf, orc, global_only):
    """The parallel sweep runs pressure searches on four search contexts in shared memory, or on
    the warp's own context in global memory when those are taken. Bit 21 of the sweep knob sends
    every search to the global ones, so both kinds run the deep lake's long searches; state and
    counters match the oracle every tick."""
    w = vf.World(48, 72, 48)
    w.fill_box(0, 0, 0, 47, 3, 47, 3)
    w.fill_box(0, 4, 0, 47, 71, 1, 3)
    w.fill_box(0, 4, 46, 47, 71, 47, 3)
    w.fill_box(0, 4, 0, 1, 71, 47, 3)
    w.fill_box(46, 4, 0, 47, 71, 47, 3)
    w.fill_box(2, 4, 2, 45, 59, 45, 5)
    w.fill_box(20, 0, 20, 27, 3, 27, 0)
    sim = vf.FluidSim(w)
    sim.set_sweep(1, 4 | (1 << 8) | ((1 << 21) if global_only else 0))
    o = oracle_for(orc, w)
    for s_ in (sim, o):
        s_.wake(0, 0, 0, 47, 71, 47)
    for t in range(25):
        sim.tick()
        o.tick()
        assert_same_digest(sim, o, t + 1)
    assert o.stats()["pull_nonempty"] > 500 and o.stats()["bfs_visits"] > 100000  # many long searches ran
    sim.close()


def test_tuning_knobs_never_change_results(vf, orc):
    """The knobs change speed only: the one-warp engine with extreme prefetch settings and the
    parallel engine with several schedule shapes (gate and cone radii, 8 or 16 warps) all give the
    oracle's state on a batch of regions."""
    import torch

    from vfwater import runner

    wl = vf.Workload(3, 0.1, 4)
    stream = torch.cuda.Stream()
    digests = []
    knobs = [{"engine": 0, "producers": 1, "depth": 1}, {"engine": 0, "producers": 7, "depth": 64}, {"engine": 0, "producers": 3, "depth": 16},
             {"engine": 1, "gate": 2}, {"engine": 1, "gate": 4 | (1 << 8)}, {"engine": 1, "gate": 8 | (4 << 8) | (8 << 16)}]
    for tune in knobs:
        sims = runner.make_sims(vf, wl, stream.cuda_stream, tune=tune)
        runner.run_batched(vf, wl, sims, 0, 12, torch, stream)
        digests.append([s.digest() for s in sims])
        for s in sims:
            s.close()
    assert all(d == digests[0] for d in digests)
    oracles = []
    for r in range(wl.regions):
        o = oracle_for(orc, wl.world(r))
        for b in wl.wakes(r):
            o.wake(*map(int, b))
        o.tick(12)
        oracles.append(o.digest())
    assert digests[0] == oracles


def test_autotuner_times_candidates_and_caches_the_best(vf, tmp_path, monkeypatch):
    import json

    import torch

    from vfwater import autotune

    monkeypatch.setattr(autotune, "CACHE", tmp_path / "tune.json")
    cands = [{"engine": 0, "producers": 2, "depth": 8, "ticks_per_launch": 4}, {"engine": 1, "gate": 2, "ticks_per_launch": 4}]
    best, table = autotune.tune(vf, 3, 0.1, torch, warmup=2, ticks=4, candidates=cands, seed=4)
    assert best in [dict(autotune.DEFAULT, **c) for c in cands]
    assert len(table) == 2 and all(r["cell_steps_per_s"] > 0 for r in table)
    cache = json.loads((tmp_path / "tune.json").read_text())
    (key, entry), = cache.items()
    assert entry["best"] == best and key.endswith("|w3|S")
    assert autotune.lookup(torch.cuda.get_device_name(), 3, vf.Workload(3, 0.1, 4).resident_cells) == best


def test_ring_world_across_negative_coordinates(vf, orc):
    """A ring world whose water straddles x = 0 (chunks -1 and 0): outside() follows the loaded
    chunks, and pressure pulls skip start cells at negative x or z (fluid.rs:519), a quirk the
    engine keeps. State and counters match the oracle every tick."""
    chunk = vf.World(128, 64, 128)
    chunk.fill_box(0, 0, 0, 127, 7, 127, 3)
    ring = vf.World.ring(4, 64)
    ring.ring_paste(chunk, -1, 0)
    ring.ring_paste(chunk, 0, 0)
    ring.fill_box(-20, 8, 40, 19, 30, 59, 5)   # a water block across x = 0
    ring.fill_box(-3, 8, 45, 2, 12, 54, 0)     # a void at its foot, filled by pulls
    sim = vf.FluidSim(ring)
    o = oracle_for(orc, ring)
    for s_ in (sim, o):
        s_.wake(-24, 7, 36, 23, 34, 63)
    for t in range(60):
        sim.tick()
        o.tick()
        assert_same_digest(sim, o, t + 1)
    assert o.stats()["pull_success"] > 0
