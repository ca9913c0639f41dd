"""The C-ABI library loads and exports every symbol its headers declare (no GPU needed)."""
import ctypes
import re
from pathlib import Path

ROOT = Path(__file__).resolve().parents[1]


def declared_symbols():
    names = set()
    for h in sorted((ROOT / "include").glob("*.h")):
        text = re.sub(r"/\*.*?\*/", "", h.read_text(), flags=re.S)
        for m in re.finditer(r"\b(vf_[a-z0-9_]+)\s*\(", text):
            names.add(m.group(1))
    return names


def test_headers_declare_entry_points():
    names = declared_symbols()
    for n in ("vf_fluid_create", "vf_fluid_tick", "vf_fluid_upload_world", "vf_fluid_download_changes", "vf_world_create"):
        assert n in names


def test_library_exports_every_declared_symbol(built):
    lib = ctypes.CDLL(str(ROOT / "voxelforge-rustrewrite_b200" / "libvf_fluid.so"))
    missing = [n for n in sorted(declared_symbols()) if not hasattr(lib, n)]
    assert not missing, f"declared but not exported: {missing}"


def test_no_device_fails_loudly(vf):
    """Without a usable CUDA device the fluid refuses to run (no CPU fallback)."""
    import torch

    if torch.cuda.is_available():
        return
    w = vf.World(16, 16, 16)
    try:
        vf.FluidSim(w)
    except vf.VfError as e:
        assert e.code == -6
    else:
        raise AssertionError("FluidSim ran without a CUDA device")


def test_world_set_voxels_replays_change_records_in_order(vf):
    """The host write-back: 16-byte change records (x, y, z, material) go through set_voxel in
    order, so a later record for the same voxel wins, and bricks materialise as needed."""
    import ctypes as C

    import numpy as np

    w = vf.World(32, 32, 32)
    recs = np.zeros((4, 4), np.int32)
    recs[:, :3] = [[1, 2, 3], [9, 9, 9], [1, 2, 3], [31, 0, 31]]
    recs[:, 3] = [5, 3, 0, 5]  # the third record overwrites the first
    vf.lib().vf_world_set_voxels(w.h, recs.ctypes.data_as(C.c_void_p), len(recs))
    assert w.get_voxel(1, 2, 3) == 0
    assert w.get_voxel(9, 9, 9) == 3
    assert w.get_voxel(31, 0, 31) == 5
    assert w.get_voxel(0, 0, 0) == 0


def test_ring_paste_and_evict(vf):  # src/voxel/sparse_volume.rs:680-699 (the ring part)
    """The host mirror's ring storage, as the reference's test drives it: a chunk pasted at
    negative chunk coordinates is readable at its absolute position, nowhere else, and gone after
    eviction."""
    chunk = vf.World(128, 64, 128)
    chunk.fill_sphere(64.0, 32.0, 64.0, 10.0, 4)
    chunk.compact()
    ring = vf.World.ring(4, 64)
    ring.ring_paste(chunk, -3, 5)
    assert ring.chunk_loaded(-3, 5)
    assert ring.get_voxel(-3 * 128 + 64, 32, 5 * 128 + 64) == 4
    assert ring.get_voxel(64, 32, 64) == 0
    ring.ring_evict(-3, 5)
    assert not ring.chunk_loaded(-3, 5)
    assert ring.get_voxel(-3 * 128 + 64, 32, 5 * 128 + 64) == 0


def test_world_set_get_compact(vf):  # src/voxel/sparse_volume.rs:643-658, on the product's host mirror
    w = vf.World(32, 32, 32)
    assert w.get_voxel(3, 4, 5) == 0
    w.set_voxel(3, 4, 5, 7)
    assert w.get_voxel(3, 4, 5) == 7
    assert w.info.detailed == 1
    w.set_voxel(3, 4, 5, 0)
    w.compact()
    assert w.info.detailed == 0
    grid, _, _ = w.arrays()
    assert grid[0] == 0
    w.fill_box(8, 8, 8, 15, 15, 15, 3)
    w.compact()
    grid, _, _ = w.arrays()
    assert grid[(1 * 4 + 1) * 4 + 1] == 3  # grid index (z * bricks_y + y) * bricks_x + x of brick (1, 1, 1)
    assert w.get_voxel(-1, 0, 0) == 0


def test_world_matches_oracle_storage_on_every_workload(vf, orc):
    """The host mirror the engine uploads and the oracle's SparseVolume hold the same voxels for
    every synthetic workload (region 0, sampled on a lattice)."""
    import numpy as np

    for wid in (1, 2, 3, 4, 5):
        wl = vf.Workload(wid, 0.25 if wid in (2, 4) else 1.0, 1)
        w = wl.world(0)
        i = w.info
        grid, bricks, ring = w.arrays()
        o = orc.Oracle.from_arrays((i.nx, i.ny, i.nz, i.ring_w), grid, bricks, ring)
        rng = np.random.default_rng(wid)
        span_x = i.nx if not i.ring_w else 3 * 128
        span_z = i.nz if not i.ring_w else 3 * 128
        for x, y, z in zip(rng.integers(-2, span_x + 2, 4000), rng.integers(-2, i.ny + 2, 4000), rng.integers(-2, span_z + 2, 4000)):
            assert w.get_voxel(int(x), int(y), int(z)) == o.get_voxel(int(x), int(y), int(z)), (wid, x, y, z)
