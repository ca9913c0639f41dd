"""The synthetic configurations at full size and full length, against the oracle.

  * config 2: the dam break, 1000 ticks, state/FIFO/seed digests every 50 ticks and at the end;
  * config 3: 64 regions, ticks 1..600 as ONE captured CUDA graph (batched launch), end digests of
    eight regions (all 64 are stepped);
  * config 4: the 1152 x 256 x 1152 ring world with 1000 rain emitters, 2000 ticks, digests every
    100 ticks;
  * config 5: config 3's world with a sphere carved or filled every 10 ticks, 100 ticks batched,
    end digests of eight regions.
The oracle steps the same scripted workload (emitters before ticks t % emit_every == 0, edits before
ticks t % edit_every == edit_every - 1).
"""
from concurrent.futures import ThreadPoolExecutor

import pytest

from conftest import oracle_for

pytestmark = pytest.mark.gpu

CHECKED_REGIONS = (0, 9, 18, 27, 36, 45, 54, 63)


def script(wl, r, t, sim_or_oracle, em):
    if wl.emit_every and t % wl.emit_every == 0 and len(em[0]):
        sim_or_oracle.emit(*em)
    if wl.edit_every and t % wl.edit_every == wl.edit_every - 1:
        ed = wl.edit(r, t)
        if ed is not None:
            sim_or_oracle.apply_brush(ed[0], ed[1])
            sim_or_oracle.wake(*map(int, ed[2]))


def single_world(vf, orc, wid, ticks, every):
    wl = vf.Workload(wid, 1.0, 1)
    sim, o = vf.FluidSim(wl.world(0), device=0), oracle_for(orc, wl.world(0))
    for box in wl.wakes(0):
        sim.wake(*map(int, box))
        o.wake(*map(int, box))
    em = wl.emitters(0)
    for t in range(ticks):
        script(wl, 0, t, sim, em)
        script(wl, 0, t, o, em)
        sim.tick()
        o.tick()
        if (t + 1) % every == 0 or t + 1 == ticks:
            assert sim.digest() == o.digest(), f"workload {wid}: digests differ after tick {t + 1}"
    st = sim.stats()
    assert st.cells_total == o.stats()["cells"]
    assert st.level_cells_total == o.stats()["level_cells"]
    sim.close()


def test_config2_dam_break_1000_ticks(vf, orc):
    single_world(vf, orc, 2, 1000, 50)


def test_config4_ring_world_with_rain_2000_ticks(vf, orc):
    single_world(vf, orc, 4, 2000, 100)


def oracle_digests(orc, wl, regions, ticks):
    def run(r):
        o = oracle_for(orc, wl.world(r))
        for box in wl.wakes(r):
            o.wake(*map(int, box))
        em = wl.emitters(r)
        for t in range(ticks):
            script(wl, r, t, o, em)
            o.tick()
        return o.digest()

    with ThreadPoolExecutor(len(regions)) as ex:
        return dict(zip(regions, ex.map(run, regions)))


@pytest.mark.parametrize("wid,ticks", [(3, 600), (5, 100)])
def test_batched_regions_one_graph(vf, orc, wid, ticks):
    import torch

    from vfwater import runner

    wl = vf.Workload(wid, 1.0, 1)
    stream = torch.cuda.Stream()
    sims = runner.make_sims(vf, wl, stream.cuda_stream)
    script_ = runner.BatchedScript(vf, wl, sims, 0, ticks, torch, stream)
    try:
        res = script_.run()
    finally:
        script_.close()
    assert res.cells > 0
    want = oracle_digests(orc, wl, CHECKED_REGIONS, ticks)
    for r in CHECKED_REGIONS:
        assert sims[r].digest() == want[r], f"workload {wid} region {r}: digests differ after tick {ticks}"
    for s in sims:
        s.close()
