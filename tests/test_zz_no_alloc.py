"""vf_fluid_download_changes_noalloc: the change download for callers that may not allocate device
memory while they run (a frame loop that cannot take an allocation's stall, an engine with a
memory budget fixed at start-up). Its output must equal the allocating entry point's, call after
call. Kept in a file that runs last so a failure here cannot hide any other test."""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

VF_ERR_RANGE = -5
MAXC = 65536  # VF_NOALLOC_MAX_CHANGES


def _noalloc(vf):
    f = vf.lib().vf_fluid_download_changes_noalloc
    f.restype = C.c_int
    f.argtypes = [C.c_void_p, C.POINTER(vf.Voxel), C.c_uint64, C.POINTER(C.c_uint64)]
    return f


def _as_set(buf, count):
    return sorted((v.x, v.y, v.z, v.m) for v in buf[:count])


def _drain(f, sim, vf, cap):
    """Every pending change through `f`, `cap` at a time."""
    out = []
    buf = (vf.Voxel * cap)()
    while True:
        n = C.c_uint64()
        rc = f(sim.h, buf, cap, C.byref(n))
        assert rc == 0, (rc, vf.lib().vf_fluid_last_error(sim.h))
        got = min(n.value, cap)
        out += _as_set(buf, got)
        if n.value <= cap:
            return sorted(out)


def test_noalloc_download_matches_the_allocating_one_twice(vf):
    wl = vf.Workload(1)
    a, b = vf.FluidSim(wl.world(0)), vf.FluidSim(wl.world(0))
    for sim in (a, b):
        for box in wl.wakes(0):
            sim.wake(*map(int, box))
    noalloc = _noalloc(vf)
    existing = vf.lib().vf_fluid_download_changes
    for call in range(2):  # two calls in a row, each after more ticks
        a.tick(25)
        b.tick(25)
        want = _drain(existing, a, vf, 4096)
        got = _drain(noalloc, b, vf, 4096)
        assert len(want) > 0, f"call {call}: no changes to compare"
        assert got == want, f"call {call}: {len(got)} vs {len(want)} changes"
        assert a.digest() == b.digest()
    # small batches leave the rest pending, like the allocating entry point
    a.tick(10)
    b.tick(10)
    assert _drain(noalloc, b, vf, 37) == _drain(existing, a, vf, 37)
    a.close()
    b.close()


def test_noalloc_download_rejects_a_cap_beyond_its_buffer(vf):
    wl = vf.Workload(1)
    sim = vf.FluidSim(wl.world(0))
    buf = (vf.Voxel * 1)()
    n = C.c_uint64()
    rc = _noalloc(vf)(sim.h, buf, MAXC + 1, C.byref(n))
    assert rc == VF_ERR_RANGE
    assert b"exceeds" in vf.lib().vf_fluid_last_error(sim.h)
    # a count-only call (no output buffer) takes any cap, like the allocating entry point
    rc = _noalloc(vf)(sim.h, None, MAXC + 1, C.byref(n))
    assert rc == 0
    sim.close()


def test_noalloc_download_allocates_nothing_at_its_largest_cap(vf):
    """At cap == VF_NOALLOC_MAX_CHANGES, on a handle whose download scratch was never grown, the
    device's free memory is the same before and after every call."""
    import torch

    wl = vf.Workload(1)
    a, b = vf.FluidSim(wl.world(0)), vf.FluidSim(wl.world(0))
    for sim in (a, b):
        for box in wl.wakes(0):
            sim.wake(*map(int, box))
        sim.tick(30)
    want = _drain(vf.lib().vf_fluid_download_changes, a, vf, MAXC)
    torch.cuda.init()
    f = _noalloc(vf)
    f(b.h, None, 0, C.byref(C.c_uint64()))  # first call on the device: looks the array up
    torch.cuda.synchronize()
    free0 = torch.cuda.mem_get_info(0)[0]
    got = _drain(f, b, vf, MAXC)
    torch.cuda.synchronize()
    assert torch.cuda.mem_get_info(0)[0] == free0
    assert got == want and len(got) > 0
    a.close()
    b.close()
