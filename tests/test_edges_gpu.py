"""Parity where fluid.rs's order decides the result, the floating origin, and the failure paths.

Each parity case compares the engine (through the C ABI) with the oracle's state, FIFO and
level-seed digests after every tick, and asserts that the cap or branch it is about was reached:
  * the 50,000-cell drain cap (fluid.rs:566-569),
  * a levelling round spread over ticks by the 40,000-cell budget (fluid.rs:489-507),
  * the 4,096 level-seed cap (fluid.rs:312-316),
  * the drain-to-film branch (fluid.rs:456-481),
  * the 400,000-cell layer cap (fluid.rs:431-438),
  * FluidSim::shift by whole ring periods, as the app's floating origin moves (fluid.rs:696-720).
The failure paths make a device wait run out, the brick atlas fill up and an event log overflow,
each ending in an error code with the handle still destroyable and the device still usable.
"""
import numpy as np
import pytest

from conftest import assert_same_digest, oracle_for

pytestmark = pytest.mark.gpu
STONE, WATER = 3, 5


def pair(vf, orc, world, **kw):
    return vf.FluidSim(world, device=0, **kw), oracle_for(orc, world)


def flat_lake(vf, n, ny, top):
    """n x ny x n: stone floor y < 4, full water y in [4, top]."""
    w = vf.World(n, ny, n)
    w.fill_box(0, 0, 0, n - 1, 3, n - 1, STONE)
    w.fill_box(0, 4, 0, n - 1, top, n - 1, WATER)
    return w


def test_drain_cap_binds_on_consecutive_ticks(vf, orc):
    """A woken 512 x 2 x 512 water slab queues 524k cells: ticks drain 50,000 at a time, in FIFO
    order, and the rest waits (fluid.rs:566-569)."""
    w = flat_lake(vf, 512, 16, 5)
    sim, o = pair(vf, orc, w)
    for s in (sim, o):
        s.set_partial(256, 5, 256, 0.25)
        s.wake(0, 4, 0, 511, 6, 511)
    capped = 0
    for t in range(1, 13):
        sim.tick()
        o.tick()
        assert_same_digest(sim, o, t)
        assert sim.last_tick_cells() == o.last_tick_cells()
        capped += sim.last_tick_cells() == 50000
    assert capped >= 8


def three_basins(vf):
    """700 x 16 x 224: water y in [4, 7] in three basins of 230 x 224 (51k surface cells each)
    between stone walls; a 40 x 40 patch of uneven partials at the surface of each."""
    w = vf.World(700, 16, 224)
    w.fill_box(0, 0, 0, 699, 3, 223, STONE)
    w.fill_box(0, 4, 0, 699, 7, 223, WATER)
    for xw in (230, 464):
        w.fill_box(xw, 4, 0, xw + 3, 12, 223, STONE)
    return w


def test_level_round_spreads_over_ticks_and_seed_cap_binds(vf, orc):
    """The dents' refilling seeds more than 4,096 surface cells (the seed set stops there,
    fluid.rs:313); each basin's surface layer spends the 40,000-cell budget, so the round runs
    over three ticks (fluid.rs:492, 503)."""
    sim, o = pair(vf, orc, three_basins(vf))
    for s in (sim, o):
        for x0 in (90, 320, 560):
            for x in range(x0, x0 + 40):
                for z in range(90, 130):
                    s.set_partial(x, 7, z, 0.3 + 0.02 * ((x * 7 + z * 3) % 17))
            s.wake(x0 - 4, 4, 86, x0 + 44, 8, 134)
    open_after = []
    seeds = budget = 0
    for t in range(1, 41):
        sim.tick()
        o.tick()
        assert_same_digest(sim, o, t)
        st = sim.stats()
        assert bool(st.level_round) == o.level_round()
        seeds = max(seeds, st.seed_count)
        budget = max(budget, st.last_level_cells)
        open_after.append(bool(st.level_round))
    assert seeds == 4096
    assert budget >= 40000
    assert any(a and b for a, b in zip(open_after, open_after[1:]))  # open after two consecutive ticks


def test_drain_to_film_branch(vf, orc):
    """The ring world with rain (scaled): thin films drained into the water under them
    (fluid.rs:456-481) on several ticks; state every tick."""
    wl = vf.Workload(4, 0.05, 1)
    sim, o = pair(vf, orc, wl.world(0))
    for box in wl.wakes(0):
        sim.wake(*map(int, box))
        o.wake(*map(int, box))
    em, amt = wl.emitters(0)
    for t in range(60):
        if t % wl.emit_every == 0:
            sim.emit(em, amt)
            o.emit(em, amt)
        sim.tick()
        o.tick()
        assert_same_digest(sim, o, t + 1)
    assert o.stats()["drains"] > 0


def test_layer_cap_binds(vf, orc):
    """A 704 x 704 flat lake (495,616 surface cells) with one dented cell: the refill seeds the
    surface, and its flood fill stops expanding at 400,000 cells (fluid.rs:436-438)."""
    w = flat_lake(vf, 704, 12, 7)
    sim, o = pair(vf, orc, w)
    for s in (sim, o):
        s.set_partial(352, 7, 352, 0.5)
        s.wake(350, 6, 350, 354, 8, 354)
    top = 0
    for t in range(1, 21):
        sim.tick()
        o.tick()
        assert_same_digest(sim, o, t)
        top = max(top, sim.stats().last_level_cells)
    assert 400000 <= top <= 400003 + 40000


def test_shift_by_ring_periods_matches_oracle(vf, orc):
    """The floating origin (window.rs:392-410): the ring world moves by whole ring periods
    (SparseVolume::ring_rebase) and FluidSim::shift re-keys the partials, the FIFO and the seeds
    and restarts the levelling round (fluid.rs:696-720). Ticking on, the engine matches the oracle
    at the shifted coordinates; download_changes reports shifted coordinates to the host world."""
    chunk = vf.World(128, 64, 128)
    chunk.fill_box(0, 0, 0, 127, 7, 127, STONE)
    ring = vf.World.ring(4, 64)
    for cx in (-1, 0):
        ring.ring_paste(chunk, cx, 0)
    ring.fill_box(-20, 8, 40, 19, 30, 59, WATER)
    ring.fill_box(-3, 8, 45, 2, 12, 54, 0)
    sim = vf.FluidSim(ring)
    o = oracle_for(orc, ring)
    for s in (sim, o):
        s.wake(-24, 7, 36, 23, 34, 63)
    period = 4 * 128
    ox = oz = 0
    for t in range(1, 61):
        if t in (17, 41):  # mid-round and at a levelling tick
            dx, dz = (65536, -period) if t == 17 else (-period, 2 * period)
            sim.shift(dx, dz)
            ring.ring_rebase(dx // 128, dz // 128)
            o.ring_rebase(dx // 128, dz // 128)
            o.shift(dx, dz)
            ox += dx
            oz += dz
            assert not o.level_round() and not sim.stats().level_round
        sim.tick()
        o.tick()
        assert_same_digest(sim, o, t)
        sim.sync_world()
    # the host world received the changes at the shifted coordinates
    bad = [(x, y, z) for x in range(-24, 24) for y in range(7, 31) for z in range(36, 64)
           if ring.get_voxel(x - ox, y, z - oz) != o.get_voxel(x - ox, y, z - oz)]
    assert not bad, bad[:4]
    assert o.stats()["pull_success"] > 0


def test_ring_evict_and_paste_on_a_live_handle(vf, orc):
    """Ring streaming without a new handle (SparseVolume::ring_evict / ring_paste,
    sparse_volume.rs:478-537). A chunk holding half of a collapsing water block is evicted mid-flow:
    its cells read as solid, the partial volumes it held are kept per cell as PartialField keeps
    them, and drained cells of the unloaded chunk erase theirs (fluid.rs:586-589). It is pasted
    back (the kept volumes return into its bricks), and later a different chunk replaces the other
    slot's chunk in one paste. State, FIFO, seeds and partial counts match the oracle every tick."""
    chunk = vf.World(128, 64, 128)
    chunk.fill_box(0, 0, 0, 127, 7, 127, STONE)
    hill = vf.World(128, 64, 128)
    hill.fill_box(0, 0, 0, 127, 7, 127, STONE)
    hill.fill_box(100, 8, 30, 127, 20, 70, STONE)
    ring = vf.World.ring(4, 64)
    for cx in (-1, 0):
        ring.ring_paste(chunk, cx, 0)
    ring.fill_box(-20, 8, 40, 19, 30, 59, WATER)
    ring.fill_box(-3, 8, 45, 2, 12, 54, 0)
    sim = vf.FluidSim(ring)
    o = oracle_for(orc, ring)
    for s in (sim, o):
        s.wake(-24, 7, 36, 23, 34, 63)

    def paste(c, cx, cz):
        g, b, _ = c.arrays()
        sim.ring_paste(c, cx, cz)
        o.ring_paste(g, b, c.info.bricks_y, cx, cz)

    kept = 0
    for t in range(1, 91):
        if t == 25:
            sim.ring_evict(0, 0)
            o.ring_evict(0, 0)
            kept = sim.partial_count()
        if t == 50:
            paste(chunk, 0, 0)
        if t == 70:
            paste(hill, -1, 0)  # the slot's chunk (-1, 0) is evicted and replaced
        sim.tick()
        o.tick()
        assert_same_digest(sim, o, t)
        assert sim.partial_count() == o.partial_count(), t
    assert kept > 0
    with pytest.raises(vf.VfError) as e:
        sim.ring_paste(chunk, 1, 0)  # beyond the handle's cell domain
    assert e.value.code == -5
    sim.close()


def test_shift_rejects_other_offsets(vf):
    ring = vf.World.ring(4, 64)
    chunk = vf.World(128, 64, 128)
    ring.ring_paste(chunk, 0, 0)
    sim = vf.FluidSim(ring)
    with pytest.raises(vf.VfError) as e:
        sim.shift(100, 0)
    assert e.value.code == -5  # VF_ERR_RANGE
    sim.close()


# ---------------------------------------------------------------------------- failure paths
@pytest.mark.parametrize("engine", [0, 1])
def test_device_wait_cap_ends_the_tick_with_timeout(vf, engine):
    """With a wait cap of one iteration the first wait of the sweep gives up: the tick returns
    VF_ERR_TIMEOUT, the handle is destroyed cleanly and the device keeps working."""
    wl = vf.Workload(2, 0.125, 1)
    sim = vf.FluidSim(wl.world(0), device=0)
    sim.set_sweep(engine, 4, 1)
    for box in wl.wakes(0):
        sim.wake(*map(int, box))
    with pytest.raises(vf.VfError) as e:
        for _ in range(20):
            sim.tick()
    assert e.value.code == -4  # VF_ERR_TIMEOUT
    sim.close()
    ok = vf.FluidSim(wl.world(0), device=0)
    for box in wl.wakes(0):
        ok.wake(*map(int, box))
    ok.tick(3)
    assert ok.stats().cells_total > 0
    ok.close()


def test_full_brick_atlas_ends_the_tick_with_oom(vf):
    """Every brick of the world is uniform, so the smallest atlas (64 spare bricks) is all there
    is: the collapsing 64 x 24 x 64 block needs more detailed bricks than that, and the tick fails
    with VF_ERR_OOM instead of writing past the atlas."""
    w = vf.World(256, 48, 256)
    w.fill_box(0, 0, 0, 255, 7, 255, STONE)
    w.fill_box(96, 8, 96, 159, 31, 159, WATER)
    w.compact()
    assert w.info.detailed == 0
    sim = vf.FluidSim(w, device=0, atlas_bricks=1)
    sim.wake(90, 8, 90, 165, 33, 165)
    with pytest.raises(vf.VfError) as e:
        for _ in range(200):
            sim.tick()
    assert e.value.code == -2  # VF_ERR_OOM
    sim.close()


def test_event_log_overflow_ends_the_tick_with_oom(vf, orc):
    """Event logs with room for 16 entries: the first busy tick overflows them and fails with
    VF_ERR_OOM; with the full capacities the same tick matches the oracle."""
    wl = vf.Workload(1)
    for caps, fails in (((16, 16, 16), True), ((1 << 22, 1 << 18, 1 << 21), False)):
        sim, o = pair(vf, orc, wl.world(0))
        sim.set_log_caps(*caps)
        for box in wl.wakes(0):
            sim.wake(*map(int, box))
            o.wake(*map(int, box))
        if fails:
            with pytest.raises(vf.VfError) as e:
                sim.tick(5)
            assert e.value.code == -2
        else:
            sim.tick(5)
            o.tick(5)
            assert_same_digest(sim, o, 5)
        sim.close()
