"""Shared fixtures. `gpu` marks tests that need a CUDA device (run on the B200 box)."""
import sys
from pathlib import Path

import numpy as np
import pytest

ROOT = Path(__file__).resolve().parents[1]
sys.path.insert(0, str(ROOT))

import __graft_entry__ as ge  # noqa: E402

ge.load_package()  # importable as `vfwater` (and `vfwater.runner`) in every test module


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200, sm_100a)")


@pytest.fixture(scope="session")
def built():
    ge.build()
    return True


@pytest.fixture(scope="session")
def vf(built):
    return ge.load_package()


@pytest.fixture(scope="session")
def orc(built):
    return ge.load_oracle()


def oracle_for(orc, world):
    """An oracle holding a copy of `world` (a product World)."""
    i = world.info
    grid, bricks, ring = world.arrays()
    return orc.Oracle.from_arrays((i.nx, i.ny, i.nz, i.ring_w), grid, bricks, ring)


def assert_same_state(sim, o, box, tick=None):
    """Bit-identical materials + partial volumes over `box` and identical FIFO + seed list."""
    x0, y0, z0, sx, sy, sz = box
    gm, gp = sim.export_box(x0, y0, z0, sx, sy, sz)
    om, op = o.export_box(x0, y0, z0, sx, sy, sz)
    where = f" after tick {tick}" if tick is not None else ""
    if not np.array_equal(gm, om):
        d = np.argwhere(gm != om)[0]
        raise AssertionError(f"material differs{where} at z,y,x={tuple(d)}: gpu {gm[tuple(d)]} oracle {om[tuple(d)]}")
    gb, ob = gp.view(np.uint32), op.view(np.uint32)
    if not np.array_equal(gb, ob):
        d = np.argwhere(gb != ob)[0]
        raise AssertionError(f"partial differs{where} at z,y,x={tuple(d)}: gpu {gp[tuple(d)]!r} oracle {op[tuple(d)]!r}")
    gq, gs = sim.queue()
    oq, os_ = o.queue()
    if not np.array_equal(gq, oq):
        n = min(len(gq), len(oq))
        bad = np.nonzero((gq[:n] != oq[:n]).any(axis=1))[0]
        raise AssertionError(f"FIFO differs{where}: len gpu {len(gq)} oracle {len(oq)}, first diff at {bad[:1]}")
    assert np.array_equal(gs, os_), f"level seeds differ{where}: {len(gs)} vs {len(os_)}"


def assert_same_counters(sim, o, tick=None):
    """The scheduler's counters agree too: drained cells, pull attempts (the 4096 budget), pulls
    that took water, pressure-search queue entries examined (the 512 budget) and level cells."""
    g, s = sim.stats(), o.stats()
    pairs = {
        "cell-steps": (g.cells_total, s["cells"]),
        "pull attempts": (g.pull_attempts, s["pull_attempts"]),
        "pull successes": (g.pull_success, s["pull_success"]),
        "search entries": (g.bfs_visits, s["bfs_visits"]),
        "level cells": (g.level_cells_total, s["level_cells"]),
    }
    bad = {k: v for k, v in pairs.items() if v[0] != v[1]}
    assert not bad, f"counters differ after tick {tick} (gpu, oracle): {bad}"


def assert_same_digest(sim, o, tick=None):
    g = sim.digest()
    d = o.digest()
    assert g == d, f"digest (state, fifo, seeds) differs after tick {tick}: gpu {g} oracle {d}"
    assert_same_counters(sim, o, tick)
