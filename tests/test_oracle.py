"""The oracle against the reference's own tests (src/fluid.rs:723-818,
src/voxel/sparse_volume.rs:639-699), its self-consistency, and the committed golden digests."""
import json
from pathlib import Path

import numpy as np
import pytest

STONE, WATER = 3, 5
GOLDEN = Path(__file__).resolve().parent / "golden"


def basin(orc):
    """A 64x32x64 stone basin: floor at y 0..4, walls 1 thick (src/fluid.rs:730-738)."""
    o = orc.Oracle(64, 32, 64)
    o.fill_box(0, 0, 0, 63, 3, 63, STONE)
    o.fill_box(0, 4, 0, 63, 31, 0, STONE)
    o.fill_box(0, 4, 63, 63, 31, 63, STONE)
    o.fill_box(0, 4, 0, 0, 31, 63, STONE)
    o.fill_box(63, 4, 0, 63, 31, 63, STONE)
    return o


def test_column_falls_spreads_and_conserves_volume(orc):  # src/fluid.rs:752-771
    o = basin(orc)
    o.fill_box(30, 10, 30, 33, 25, 33, WATER)
    o.wake(29, 9, 29, 34, 26, 34)
    before = o.total(0, 0, 0, 64, 32, 64)
    for _ in range(2000):
        o.tick()
        if o.idle():
            break
    after = o.total(0, 0, 0, 64, 32, 64)
    assert abs(before - after) < 0.05 * before, (before, after)
    assert o.total(0, 6, 0, 64, 32, 64) < 1.0
    assert o.volume(10, 4, 10) > 0.0 or o.volume(50, 4, 50) > 0.0


def test_displace_moves_water_up(orc):  # src/fluid.rs:773-782
    o = basin(orc)
    o.fill_box(1, 4, 1, 62, 5, 62, WATER)
    o.displace(20, 4, 20)
    o.set_voxel(20, 4, 20, STONE)
    assert o.get_voxel(20, 6, 20) == WATER
    assert not o.idle()


def test_partial_field_pages(orc):  # src/fluid.rs:784-798
    p = orc.PartialField()
    p.set(-3, 5, 700, 0.25)
    p.set(-4, 5, 700, 0.5)
    assert p.get(-3, 5, 700) == 0.25
    assert len(p) == 2
    p.erase(-3, 5, 700)
    p.erase(-4, 5, 700)
    assert (len(p), p.get(-4, 5, 700)) == (0, 0.0)
    p.set(1, 1, 1, 0.75)
    assert p.entries() == [(1, 1, 1, 0.75)]


def test_hole_under_a_lake_drains_it_level(orc):  # src/fluid.rs:800-817
    o = basin(orc)
    o.fill_box(1, 4, 1, 62, 7, 62, WATER)
    o.fill_box(1, 1, 1, 20, 2, 20, 0)
    o.set_voxel(10, 3, 10, 0)
    o.wake(9, 2, 9, 11, 5, 11)
    o.tick(400)
    assert o.volume(5, 1, 5) > 0.5
    near, far = o.volume(12, 7, 10), o.volume(50, 7, 50)
    assert abs(near - far) < 0.2, (near, far)


def test_set_get_compact(orc):  # src/voxel/sparse_volume.rs:643-658
    o = orc.Oracle(32, 32, 32)
    assert o.get_voxel(3, 4, 5) == 0
    o.set_voxel(3, 4, 5, 7)
    assert o.get_voxel(3, 4, 5) == 7
    L = orc.lib()
    assert L.orc_detailed_bricks(o.h) == 1
    o.set_voxel(3, 4, 5, 0)
    L.orc_compact(o.h)
    assert L.orc_detailed_bricks(o.h) == 0
    assert L.orc_grid_at(o.h, 0, 0, 0) == 0
    o.fill_box(8, 8, 8, 15, 15, 15, 3)
    L.orc_compact(o.h)
    assert L.orc_grid_at(o.h, 1, 1, 1) == 3
    assert o.get_voxel(-1, 0, 0) == 0


def test_oracle_is_deterministic(orc, vf):
    """Two runs on the same input give identical digests every tick (tick() never iterates a
    hash container, src/fluid.rs:564-657)."""
    wl = vf.Workload(1)
    w = wl.world(0)
    from conftest import oracle_for

    a, b = oracle_for(orc, w), oracle_for(orc, w)
    for o in (a, b):
        o.wake(*map(int, wl.wakes(0)[0]))
    for t in range(60):
        a.tick()
        b.tick()
        assert a.digest() == b.digest(), t


def test_update_runs_fixed_ticks(orc):  # src/fluid.rs:662-676
    o = basin(orc)
    o.fill_box(30, 10, 30, 33, 25, 33, WATER)
    o.wake(29, 9, 29, 34, 26, 34)
    o.update(0.07)  # acc 0.07 -> 1 tick, 0.02 left
    assert o.tick_no() == 1
    o.update(0.01)  # 0.03 -> none
    assert o.tick_no() == 1
    o.update(1.0)  # clamp 0.25, cap 0.15 -> 3 ticks
    assert o.tick_no() == 4


@pytest.mark.parametrize("name", ["basin_c1.json"])
def test_oracle_matches_golden_digests(orc, vf, name):
    """The oracle reproduces the committed per-tick digests (regenerate with
    tests/golden/make_golden.py only when the oracle is deliberately changed)."""
    g = json.loads((GOLDEN / name).read_text())
    wl = vf.Workload(g["workload"], g["scale"], g["seed"])
    from conftest import oracle_for

    o = oracle_for(orc, wl.world(0))
    for box in wl.wakes(0):
        o.wake(*map(int, box))
    for t, want in enumerate(g["digests"]):
        o.tick()
        got = list(o.digest()) + [o.last_tick_cells()]
        assert got == want, f"tick {t + 1}"
