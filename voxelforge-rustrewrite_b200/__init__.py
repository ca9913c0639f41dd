"""Host-side mirror of the reference's fluid interface over the B200 engine's C ABI.

The reference drives its CA water through ``FluidSim`` methods that borrow the world
(src/fluid.rs:230-721). ``FluidSim`` here keeps those names and argument meanings; the world
is a :class:`World` (the reference's ``SparseVolume``, src/voxel/sparse_volume.rs) that the
engine mirrors on the device. Every call goes through ``libvf_fluid.so`` (include/vf_fluid.h,
include/vf_world.h); there is no CPU fallback: if the library or a CUDA device is missing the
calls raise.
"""
from __future__ import annotations

import ctypes as C
import os
from pathlib import Path

import numpy as np

PKG_DIR = Path(__file__).resolve().parent
LIB_PATH = PKG_DIR / "libvf_fluid.so"

WATER = 5
STONE = 3
TICK_HZ = 20.0

_ERRORS = {
    -1: "invalid argument",
    -2: "out of memory / capacity",
    -3: "CUDA error",
    -4: "device wait timed out",
    -5: "coordinate out of range",
    -6: "no CUDA device",
    -7: "invalid state",
}


class VfError(RuntimeError):
    def __init__(self, code: int, what: str, detail: str = ""):
        super().__init__(f"{what}: {_ERRORS.get(code, code)} ({code}) {detail}".strip())
        self.code = code


P = C.c_void_p
I32 = C.c_int32
U64 = C.c_uint64


class WorldInfo(C.Structure):
    _fields_ = [(n, C.c_int32) for n in ("nx", "ny", "nz", "bricks_x", "bricks_y", "bricks_z", "ring_w", "origin_x", "origin_z")] + [
        ("nbricks", C.c_uint64),
        ("detailed", C.c_uint64),
    ]


class WorkloadInfo(C.Structure):
    _fields_ = [(n, C.c_int32) for n in ("id", "regions", "ticks", "emit_every", "edit_every")] + [("resident_cells", C.c_uint64)]


class Stats(C.Structure):
    _fields_ = [
        (n, C.c_uint64)
        for n in (
            "tick_no",
            "last_tick_cells",
            "active_count",
            "partial_count",
            "seed_count",
            "level_round",
            "last_level_cells",
            "memory_bytes",
            "cells_total",
            "pull_attempts",
            "pull_success",
            "bfs_visits",
            "level_cells_total",
            "atlas_used",
            "changes_pending",
        )
    ]


class Desc(C.Structure):
    _fields_ = [("device", C.c_int32), ("stream", C.c_void_p), ("atlas_bricks", C.c_uint64), ("queue_capacity", C.c_uint64)]


class Voxel(C.Structure):
    _fields_ = [("x", C.c_int32), ("y", C.c_int32), ("z", C.c_int32), ("m", C.c_uint8), ("pad", C.c_uint8 * 3)]


_lib = None


def lib():
    """Load libvf_fluid.so (built in-tree by __graft_entry__.build())."""
    global _lib
    if _lib is not None:
        return _lib
    if not LIB_PATH.exists():
        raise VfError(-6, "load", f"{LIB_PATH} is missing: run __graft_entry__.build()")
    L = C.CDLL(str(LIB_PATH))
    sig = {
        "vf_world_create": (C.c_int, [I32, I32, I32, C.POINTER(P)]),
        "vf_world_create_ring": (C.c_int, [I32, I32, C.POINTER(P)]),
        "vf_world_clone": (C.c_int, [P, C.POINTER(P)]),
        "vf_world_destroy": (None, [P]),
        "vf_world_get_info": (C.c_int, [P, C.POINTER(WorldInfo)]),
        "vf_world_get_voxel": (C.c_uint8, [P, I32, I32, I32]),
        "vf_world_set_voxel": (None, [P, I32, I32, I32, C.c_uint8]),
        "vf_world_set_voxels": (None, [P, P, C.c_uint64]),
        "vf_world_fill_box": (None, [P, I32, I32, I32, I32, I32, I32, C.c_uint8]),
        "vf_world_fill_sphere": (None, [P, C.c_float, C.c_float, C.c_float, C.c_float, C.c_uint8]),
        "vf_world_compact": (None, [P]),
        "vf_world_ring_paste": (C.c_int, [P, P, I32, I32]),
        "vf_world_ring_evict": (C.c_int, [P, I32, I32]),
        "vf_world_ring_rebase": (C.c_int, [P, I32, I32]),
        "vf_world_chunk_loaded": (C.c_int, [P, I32, I32]),
        "vf_world_grid": (C.POINTER(C.c_uint32), [P]),
        "vf_world_bricks": (C.POINTER(C.c_uint8), [P]),
        "vf_world_ring_slots": (C.c_int, [P, C.POINTER(C.c_int32)]),
        "vf_world_take_dirty": (C.c_size_t, [P, C.POINTER(C.c_uint32), C.c_size_t]),
        "vf_workload_build": (C.c_int, [I32, C.c_float, U64, C.POINTER(P)]),
        "vf_workload_destroy": (None, [P]),
        "vf_workload_get_info": (C.c_int, [P, C.POINTER(WorkloadInfo)]),
        "vf_workload_world": (P, [P, I32]),
        "vf_workload_wakes": (C.c_size_t, [P, I32, C.POINTER(C.c_int32), C.c_size_t]),
        "vf_workload_emitters": (C.c_size_t, [P, I32, C.POINTER(C.c_int32), C.c_size_t, C.POINTER(C.c_float)]),
        "vf_workload_edit": (C.c_size_t, [P, I32, I32, C.POINTER(C.c_int32), C.c_size_t, C.POINTER(C.c_uint8), C.POINTER(C.c_int32)]),
        "vf_fluid_create": (C.c_int, [C.POINTER(Desc), C.POINTER(P)]),
        "vf_fluid_destroy": (None, [P]),
        "vf_fluid_last_error": (C.c_char_p, [P]),
        "vf_fluid_upload_world": (C.c_int, [P, I32, I32, I32, I32, I32, I32, C.POINTER(C.c_uint32), C.POINTER(C.c_uint8), U64, I32, C.POINTER(C.c_int32)]),
        "vf_fluid_apply_voxel_edits": (C.c_int, [P, C.POINTER(Voxel), U64]),
        "vf_fluid_wake": (C.c_int, [P, I32, I32, I32, I32, I32, I32]),
        "vf_fluid_displace": (C.c_int, [P, I32, I32, I32]),
        "vf_fluid_apply_brush": (C.c_int, [P, C.POINTER(C.c_int32), U64, C.c_uint8, C.POINTER(C.c_uint64)]),
        "vf_fluid_emit": (C.c_int, [P, C.POINTER(C.c_int32), U64, C.c_float]),
        "vf_fluid_set_partial": (C.c_int, [P, I32, I32, I32, C.c_float]),
        "vf_fluid_tick": (C.c_int, [P, I32, C.POINTER(C.c_int32)]),
        "vf_fluid_update": (C.c_int, [P, C.c_float, C.POINTER(C.c_int32)]),
        "vf_fluid_tick_async": (C.c_int, [P, I32]),
        "vf_fluid_sync": (C.c_int, [P]),
        "vf_fluid_stream": (C.c_void_p, [P]),
        "vf_fluid_download_changes": (C.c_int, [P, C.POINTER(Voxel), U64, C.POINTER(C.c_uint64)]),
        "vf_fluid_volume": (C.c_int, [P, I32, I32, I32, C.POINTER(C.c_float)]),
        "vf_fluid_idle": (C.c_int, [P, C.POINTER(C.c_int32)]),
        "vf_fluid_get_stats": (C.c_int, [P, C.POINTER(Stats)]),
        "vf_fluid_export_partials": (C.c_int, [P, C.POINTER(C.c_int32), C.POINTER(C.c_float), U64, C.POINTER(C.c_uint64)]),
        "vf_fluid_shift": (C.c_int, [P, I32, I32]),
        "vf_fluid_ring_evict": (C.c_int, [P, I32, I32]),
        "vf_fluid_ring_paste": (C.c_int, [P, C.POINTER(C.c_uint32), C.POINTER(C.c_uint8), U64, I32, I32, I32]),
        "vf_fluid_reset": (C.c_int, [P]),
        "vf_fluid_snapshot_queue": (
            C.c_int,
            [P, C.POINTER(C.c_int32), U64, C.POINTER(C.c_uint64), C.POINTER(C.c_int32), U64, C.POINTER(C.c_uint64)],
        ),
        "vf_fluid_export_box": (C.c_int, [P, I32, I32, I32, I32, I32, I32, C.POINTER(C.c_uint8), C.POINTER(C.c_float)]),
        "vf_fluid_digest": (C.c_int, [P, C.POINTER(C.c_uint64), C.POINTER(C.c_uint64), C.POINTER(C.c_uint64)]),
        "vf_fluid_batch_tick": (C.c_int, [C.POINTER(P), I32, I32]),
        "vf_fluid_profile": (C.c_int, [P, C.POINTER(C.c_uint64)]),
        "vf_fluid_set_tuning": (C.c_int, [P, I32, I32]),
        "vf_fluid_set_log_caps": (C.c_int, [P, C.c_uint32, C.c_uint32, C.c_uint32]),
        "vf_fluid_set_sweep": (C.c_int, [P, I32, I32, C.c_uint64]),
        "vf_fluid_sweep_profile": (C.c_int, [P, C.POINTER(C.c_uint64)]),
        "vf_fluid_sweep_stats": (C.c_int, [P, C.POINTER(C.c_uint64), C.POINTER(C.c_uint64), C.POINTER(C.c_uint64), C.POINTER(C.c_uint64)]),
        "vf_fluid_emit_device_async": (C.c_int, [P, C.c_void_p, U64, C.c_float]),
        "vf_fluid_brush_device_async": (C.c_int, [P, C.c_void_p, U64, C.c_uint8]),
        "vf_fluid_wake_async": (C.c_int, [P, I32, I32, I32, I32, I32, I32]),
        "vf_batch_create": (C.c_int, [C.POINTER(P), I32, C.POINTER(P)]),
        "vf_batch_destroy": (None, [P]),
        "vf_batch_tick_async": (C.c_int, [P, I32]),
        "vf_batch_sync": (C.c_int, [P]),
        "vf_batch_capture": (C.c_int, [P, I32, I32]),
        "vf_batch_replay": (C.c_int, [P]),
        "vf_batch_begin_capture": (C.c_int, [P]),
        "vf_batch_end_capture": (C.c_int, [P]),
    }
    for name, (res, args) in sig.items():
        f = getattr(L, name)
        f.restype = res
        f.argtypes = args
    _lib = L
    return L


def _i32p(a: np.ndarray):
    return a.ctypes.data_as(C.POINTER(C.c_int32))


# ----------------------------------------------------------------------------------- world
class World:
    """The reference's SparseVolume (src/voxel/sparse_volume.rs:90-637), host side."""

    def __init__(self, nx: int = 0, ny: int = 0, nz: int = 0, *, ring_w: int = 0, _handle=None, _owned=True):
        L = lib()
        self._owned = _owned
        if _handle is not None:
            self.h = P(_handle)
            return
        h = P()
        rc = L.vf_world_create_ring(ring_w, ny, C.byref(h)) if ring_w else L.vf_world_create(nx, ny, nz, C.byref(h))
        if rc:
            raise VfError(rc, "vf_world_create")
        self.h = h

    @classmethod
    def ring(cls, w: int, ny: int) -> "World":
        return cls(0, ny, 0, ring_w=w)

    def clone(self) -> "World":
        h = P()
        rc = lib().vf_world_clone(self.h, C.byref(h))
        if rc:
            raise VfError(rc, "vf_world_clone")
        return World(_handle=h.value)

    def __del__(self):
        if getattr(self, "_owned", False) and getattr(self, "h", None) and _lib is not None:
            _lib.vf_world_destroy(self.h)
            self.h = None

    @property
    def info(self) -> WorldInfo:
        i = WorldInfo()
        lib().vf_world_get_info(self.h, C.byref(i))
        return i

    @property
    def ny(self) -> int:
        return self.info.ny

    def get_voxel(self, x, y, z) -> int:
        return lib().vf_world_get_voxel(self.h, x, y, z)

    def set_voxel(self, x, y, z, m):
        lib().vf_world_set_voxel(self.h, x, y, z, m)

    def fill_box(self, x0, y0, z0, x1, y1, z1, m):
        lib().vf_world_fill_box(self.h, x0, y0, z0, x1, y1, z1, m)

    def fill_sphere(self, cx, cy, cz, r, m):
        lib().vf_world_fill_sphere(self.h, cx, cy, cz, r, m)

    def compact(self):
        lib().vf_world_compact(self.h)

    def ring_paste(self, chunk: "World", cx: int, cz: int):
        rc = lib().vf_world_ring_paste(self.h, chunk.h, cx, cz)
        if rc:
            raise VfError(rc, "ring_paste")

    def ring_evict(self, cx: int, cz: int):
        lib().vf_world_ring_evict(self.h, cx, cz)

    def ring_rebase(self, dcx: int, dcz: int):
        """SparseVolume::ring_rebase: the floating origin moves by (dcx, dcz) chunks."""
        lib().vf_world_ring_rebase(self.h, dcx, dcz)

    def chunk_loaded(self, cx, cz) -> bool:
        return bool(lib().vf_world_chunk_loaded(self.h, cx, cz))

    def arrays(self):
        """(grid u32[nb], bricks u8[nbricks*512], ring slots i32[w*w*3] or None), copied."""
        L = lib()
        i = self.info
        nb = i.bricks_x * i.bricks_y * i.bricks_z
        grid = np.ctypeslib.as_array(L.vf_world_grid(self.h), shape=(nb,)).copy()
        if i.nbricks:
            bricks = np.ctypeslib.as_array(L.vf_world_bricks(self.h), shape=(i.nbricks * 512,)).copy()
        else:
            bricks = np.zeros(512, np.uint8)
        ring = None
        if i.ring_w:
            ring = np.zeros(3 * i.ring_w * i.ring_w, np.int32)
            L.vf_world_ring_slots(self.h, _i32p(ring))
        return grid, bricks, ring

    def take_dirty(self) -> np.ndarray:
        L = lib()
        n = L.vf_world_take_dirty(self.h, None, 0)
        return np.zeros(0, np.uint32) if n == 0 else None  # the list is cleared either way


# -------------------------------------------------------------------------------- workloads
class Workload:
    """A synthetic workload: regions (independent worlds), wake boxes, emitters, edits."""

    def __init__(self, wid: int, scale: float = 1.0, seed: int = 1):
        L = lib()
        h = P()
        rc = L.vf_workload_build(wid, scale, seed, C.byref(h))
        if rc:
            raise VfError(rc, "vf_workload_build")
        self.h = h
        i = WorkloadInfo()
        L.vf_workload_get_info(h, C.byref(i))
        self.id, self.regions, self.ticks = i.id, i.regions, i.ticks
        self.emit_every, self.edit_every, self.resident_cells = i.emit_every, i.edit_every, i.resident_cells

    def __del__(self):
        if getattr(self, "h", None) and _lib is not None:
            _lib.vf_workload_destroy(self.h)
            self.h = None

    def world(self, r: int) -> World:
        """A private copy of region r's initial world."""
        src = World(_handle=lib().vf_workload_world(self.h, r), _owned=False)
        return src.clone()

    def wakes(self, r: int) -> np.ndarray:
        n = lib().vf_workload_wakes(self.h, r, None, 0)
        a = np.zeros(6 * max(n, 1), np.int32)
        lib().vf_workload_wakes(self.h, r, _i32p(a), n)
        return a[: 6 * n].reshape(-1, 6)

    def emitters(self, r: int):
        amt = C.c_float()
        n = lib().vf_workload_emitters(self.h, r, None, 0, C.byref(amt))
        a = np.zeros(3 * max(n, 1), np.int32)
        lib().vf_workload_emitters(self.h, r, _i32p(a), n, C.byref(amt))
        return a[: 3 * n].reshape(-1, 3), amt.value

    def edit(self, r: int, tick: int):
        """(cells (n,3) int32, material, wake box) of the edit before `tick`, or None."""
        L = lib()
        m = C.c_uint8()
        wake = np.zeros(6, np.int32)
        n = L.vf_workload_edit(self.h, r, tick, None, 0, C.byref(m), _i32p(wake))
        if n == 0:
            return None
        a = np.zeros(3 * n, np.int32)
        L.vf_workload_edit(self.h, r, tick, _i32p(a), n, C.byref(m), _i32p(wake))
        return a.reshape(-1, 3), int(m.value), wake


# ------------------------------------------------------------------------------------ fluid
class FluidSim:
    """FluidSim (src/fluid.rs:230-721) on the B200: one handle per simulated world.

    ``FluidSim(world)`` uploads the world mirror (the Rust type borrows the world per call;
    here the world is bound once and kept coherent: voxel changes made by the fluid are
    replayed into ``world`` by :meth:`sync_world`, host edits go through :meth:`apply_voxel_edits`).
    """

    def __init__(self, world: World, device: int = 0, stream: int | None = None, atlas_bricks: int = 0, queue_capacity: int = 0):
        L = lib()
        d = Desc(device, C.c_void_p(stream) if stream else None, atlas_bricks, queue_capacity)
        h = P()
        rc = L.vf_fluid_create(C.byref(d), C.byref(h))
        if rc:
            raise VfError(rc, "vf_fluid_create")
        self.h = h
        self.world = world
        i = world.info
        grid, bricks, ring = world.arrays()
        self._check(
            L.vf_fluid_upload_world(
                h,
                i.nx,
                i.ny,
                i.nz,
                i.bricks_x,
                i.bricks_y,
                i.bricks_z,
                grid.ctypes.data_as(C.POINTER(C.c_uint32)),
                bricks.ctypes.data_as(C.POINTER(C.c_uint8)),
                int(i.nbricks),
                i.ring_w,
                _i32p(ring) if ring is not None else None,
            ),
            "upload_world",
        )

    def _check(self, rc, what):
        if rc:
            raise VfError(rc, what, (lib().vf_fluid_last_error(self.h) or b"").decode())

    def close(self):
        if getattr(self, "h", None) and _lib is not None:
            _lib.vf_fluid_destroy(self.h)
            self.h = None

    __del__ = close

    # ---- the reference's methods
    def tick(self, n: int = 1) -> bool:
        ch = C.c_int32()
        self._check(lib().vf_fluid_tick(self.h, n, C.byref(ch)), "tick")
        return bool(ch.value)

    def set_tuning(self, producers: int, depth: int):
        """Launch knobs of the one-warp sweep (prefetch warps, prefetch distance); results never depend on them."""
        self._check(lib().vf_fluid_set_tuning(self.h, producers, depth), "set_tuning")

    def set_sweep(self, engine: int = 2, gate: int = 4 | (1 << 8), spin_cap: int = 1 << 24):
        """Which sweep runs (0 one warp, 1 all warps of the region's CTA, 2 chosen per call), the parallel sweep's pull
        gate radius and the iteration cap of device waits; results never depend on them."""
        self._check(lib().vf_fluid_set_sweep(self.h, engine, gate, spin_cap), "set_sweep")

    def set_log_caps(self, act: int, seed: int, chg: int):
        """Lower the per-tick event-log capacities (a tick that overflows one fails with VF_ERR_OOM)."""
        self._check(lib().vf_fluid_set_log_caps(self.h, act, seed, chg), "set_log_caps")

    SWEEP_PROFILE = ("prepass", "segments", "rollbacks", "logs", "dep_wait", "start_wait", "footprint", "pulls", "writes", "cells",
                     "row_fetch", "worker_total", "cone_wait", "gate_wait", "searches", "rounds", "search_reads",
                     "source_writes")

    def sweep_profile(self) -> dict:
        """Parallel-sweep SM cycle counters summed over ticks (the per-cell ones also over warps)."""
        a = (C.c_uint64 * 18)()
        self._check(lib().vf_fluid_sweep_profile(self.h, a), "sweep_profile")
        return dict(zip(self.SWEEP_PROFILE, map(int, a)))

    def sweep_stats(self) -> dict:
        """Parallel-sweep counters over all ticks: segments, segments replayed in order, cells replayed."""
        a, b, c = C.c_uint64(), C.c_uint64(), C.c_uint64()
        k = (C.c_uint64 * 3)()
        self._check(lib().vf_fluid_sweep_stats(self.h, C.byref(a), C.byref(b), C.byref(c), k), "sweep_stats")
        return {"segments": a.value, "rollbacks": b.value, "replayed": c.value,
                "conflicts": {"reader_started": k[0], "pull_read": k[1], "new_attempter": k[2]}}

    def emit_device_async(self, dev_xyz_ptr: int, n: int, amount: float):
        self._check(lib().vf_fluid_emit_device_async(self.h, C.c_void_p(dev_xyz_ptr), n, amount), "emit_device_async")

    def brush_device_async(self, dev_xyz_ptr: int, n: int, m: int):
        self._check(lib().vf_fluid_brush_device_async(self.h, C.c_void_p(dev_xyz_ptr), n, m), "brush_device_async")

    def wake_async(self, x0, y0, z0, x1, y1, z1):
        self._check(lib().vf_fluid_wake_async(self.h, x0, y0, z0, x1, y1, z1), "wake_async")

    def tick_async(self, n: int = 1):
        """Enqueue n ticks on the handle's stream without waiting."""
        self._check(lib().vf_fluid_tick_async(self.h, n), "tick_async")

    def sync(self):
        self._check(lib().vf_fluid_sync(self.h), "sync")

    @property
    def stream(self) -> int:
        return lib().vf_fluid_stream(self.h) or 0

    def update(self, dt: float) -> bool:
        ch = C.c_int32()
        self._check(lib().vf_fluid_update(self.h, dt, C.byref(ch)), "update")
        return bool(ch.value)

    def wake(self, x0, y0, z0, x1, y1, z1):
        self._check(lib().vf_fluid_wake(self.h, x0, y0, z0, x1, y1, z1), "wake")

    def displace(self, x, y, z):
        self._check(lib().vf_fluid_displace(self.h, x, y, z), "displace")

    def apply_brush(self, cells: np.ndarray, m: int) -> int:
        cells = np.ascontiguousarray(cells, np.int32)
        n = C.c_uint64()
        self._check(lib().vf_fluid_apply_brush(self.h, _i32p(cells), len(cells), m, C.byref(n)), "apply_brush")
        return n.value

    def emit(self, cells: np.ndarray, amount: float):
        cells = np.ascontiguousarray(cells, np.int32)
        self._check(lib().vf_fluid_emit(self.h, _i32p(cells), len(cells), amount), "emit")

    def set_partial(self, x, y, z, v):
        self._check(lib().vf_fluid_set_partial(self.h, x, y, z, v), "set_partial")

    def volume(self, x, y, z) -> float:
        v = C.c_float()
        self._check(lib().vf_fluid_volume(self.h, x, y, z, C.byref(v)), "volume")
        return v.value

    def idle(self) -> bool:
        v = C.c_int32()
        self._check(lib().vf_fluid_idle(self.h, C.byref(v)), "idle")
        return bool(v.value)

    def stats(self) -> Stats:
        s = Stats()
        self._check(lib().vf_fluid_get_stats(self.h, C.byref(s)), "stats")
        return s

    def active_count(self) -> int:
        return self.stats().active_count

    def partial_count(self) -> int:
        return self.stats().partial_count

    def last_tick_cells(self) -> int:
        return self.stats().last_tick_cells

    PROFILE_PHASES = ("drain", "sort", "sweep", "sweep_wait", "pulls", "act_log", "writes", "seed_commit", "level", "fifo_commit",
                      "chg_commit", "mark_clear", "sweep_top", "sweep_cell", "sweep_tail", "between")

    def profile(self) -> dict:
        """SM cycles per tick phase, summed over all ticks so far."""
        a = (C.c_uint64 * 16)()
        self._check(lib().vf_fluid_profile(self.h, a), "profile")
        return {k: int(v) for k, v in zip(self.PROFILE_PHASES, a) if k != "-"}

    def shift(self, dx, dz):
        self._check(lib().vf_fluid_shift(self.h, dx, dz), "shift")

    def ring_evict(self, cx: int, cz: int):
        """SparseVolume::ring_evict on the device copy of the world; the chunk's partial volumes are
        kept per cell (the host world is evicted by the caller, as the app does)."""
        self._check(lib().vf_fluid_ring_evict(self.h, cx, cz), "ring_evict")

    def ring_paste(self, chunk: "World", cx: int, cz: int):
        """SparseVolume::ring_paste of a 128 x ny x 128 chunk world into the device copy of the world."""
        i = chunk.info
        grid, bricks, _ = chunk.arrays()
        self._check(lib().vf_fluid_ring_paste(self.h, grid.ctypes.data_as(C.POINTER(C.c_uint32)), bricks.ctypes.data_as(C.POINTER(C.c_uint8)),
                                              int(i.nbricks), i.bricks_y, cx, cz), "ring_paste")

    def reset(self):
        self._check(lib().vf_fluid_reset(self.h), "reset")

    def partials(self):
        """Every partial cell: (xyz (n,3) int32, volume (n,) float32), sorted by (z, y, x)."""
        n = C.c_uint64()
        self._check(lib().vf_fluid_export_partials(self.h, None, None, 0, C.byref(n)), "partials")
        cap = n.value
        xyz = np.zeros(3 * max(cap, 1), np.int32)
        vol = np.zeros(max(cap, 1), np.float32)
        self._check(
            lib().vf_fluid_export_partials(self.h, _i32p(xyz), vol.ctypes.data_as(C.POINTER(C.c_float)), cap, C.byref(n)), "partials"
        )
        return xyz[: 3 * cap].reshape(-1, 3), vol[:cap]

    # ---- coherence with the host world
    def apply_voxel_edits(self, edits):
        arr = (Voxel * len(edits))()
        for i, (x, y, z, m) in enumerate(edits):
            arr[i].x, arr[i].y, arr[i].z, arr[i].m = x, y, z, m
        self._check(lib().vf_fluid_apply_voxel_edits(self.h, arr, len(edits)), "apply_voxel_edits")

    def _download_raw(self):
        n = C.c_uint64()
        self._check(lib().vf_fluid_download_changes(self.h, None, 0, C.byref(n)), "changes")
        if n.value == 0:
            return None, 0
        arr = (Voxel * n.value)()
        self._check(lib().vf_fluid_download_changes(self.h, arr, n.value, C.byref(n)), "changes")
        return arr, n.value

    def download_changes(self) -> np.ndarray:
        arr, n = self._download_raw()
        if not n:
            return np.zeros((0, 4), np.int32)
        out = np.frombuffer(arr, dtype=np.int32).reshape(-1, 4).copy()
        out[:, 3] &= 0xFF
        return out

    def sync_world(self) -> int:
        """Replay the fluid's voxel changes into the host world through set_voxel (in C++)."""
        arr, n = self._download_raw()
        if n:
            lib().vf_world_set_voxels(self.world.h, arr, n)
        return n

    # ---- inspection (differential tests)
    def queue(self):
        nq, ns = C.c_uint64(), C.c_uint64()
        self._check(lib().vf_fluid_snapshot_queue(self.h, None, 0, C.byref(nq), None, 0, C.byref(ns)), "snapshot")
        q = np.zeros(3 * max(nq.value, 1), np.int32)
        s = np.zeros(3 * max(ns.value, 1), np.int32)
        self._check(lib().vf_fluid_snapshot_queue(self.h, _i32p(q), nq.value, C.byref(nq), _i32p(s), ns.value, C.byref(ns)), "snapshot")
        return q[: 3 * nq.value].reshape(-1, 3), s[: 3 * ns.value].reshape(-1, 3)

    def export_box(self, x0, y0, z0, sx, sy, sz):
        mat = np.zeros(sx * sy * sz, np.uint8)
        part = np.zeros(sx * sy * sz, np.float32)
        self._check(
            lib().vf_fluid_export_box(
                self.h, x0, y0, z0, sx, sy, sz, mat.ctypes.data_as(C.POINTER(C.c_uint8)), part.ctypes.data_as(C.POINTER(C.c_float))
            ),
            "export_box",
        )
        return mat.reshape(sz, sy, sx), part.reshape(sz, sy, sx)

    def digest(self):
        a, b, c = C.c_uint64(), C.c_uint64(), C.c_uint64()
        self._check(lib().vf_fluid_digest(self.h, C.byref(a), C.byref(b), C.byref(c)), "digest")
        return a.value, b.value, c.value


class Batch:
    """Many independent FluidSims stepped by one launch (one CTA per region), optionally as a
    captured CUDA graph. All sims must share a device; the batch runs on the first sim's stream."""

    def __init__(self, sims):
        self.sims = list(sims)
        arr = (P * len(self.sims))(*[s.h.value for s in self.sims])
        h = P()
        rc = lib().vf_batch_create(arr, len(self.sims), C.byref(h))
        if rc:
            raise VfError(rc, "vf_batch_create", (lib().vf_fluid_last_error(self.sims[0].h) or b"").decode())
        self.h = h

    def _check(self, rc, what):
        if rc:
            raise VfError(rc, what, (lib().vf_fluid_last_error(self.sims[0].h) or b"").decode())

    def tick_async(self, n: int):
        self._check(lib().vf_batch_tick_async(self.h, n), "batch_tick_async")

    def sync(self):
        self._check(lib().vf_batch_sync(self.h), "batch_sync")

    def capture(self, launches: int, ticks_per_launch: int):
        self._check(lib().vf_batch_capture(self.h, launches, ticks_per_launch), "batch_capture")

    def replay(self):
        self._check(lib().vf_batch_replay(self.h), "batch_replay")

    def begin_capture(self):
        self._check(lib().vf_batch_begin_capture(self.h), "batch_begin_capture")

    def end_capture(self):
        self._check(lib().vf_batch_end_capture(self.h), "batch_end_capture")

    def close(self):
        if getattr(self, "h", None) and _lib is not None:
            _lib.vf_batch_destroy(self.h)
            self.h = None

    __del__ = close


def batch_tick(sims, n_ticks: int):
    """Step many independent FluidSims n_ticks times in one launch (one CTA per region)."""
    arr = (P * len(sims))(*[s.h.value for s in sims])
    rc = lib().vf_fluid_batch_tick(arr, len(sims), n_ticks)
    if rc:
        raise VfError(rc, "batch_tick", (lib().vf_fluid_last_error(sims[0].h) or b"").decode())
