"""ORACLE — test infrastructure only.

ctypes binding of the CPU restatement of the reference's CA water (oracle/fluid_oracle.cpp,
restating src/fluid.rs and src/voxel/sparse_volume.rs). Only tests/, __graft_entry__.smoke() and
bench.py's CPU-baseline leg use it, as the checker and as the timed CPU baseline. Parity is
pinned by ports of the reference's own property tests (tests/test_oracle.py); the reference
ships no numeric golden vectors for this path and its Rust crate cannot be built here.
"""
from __future__ import annotations

import ctypes as C
import subprocess
from pathlib import Path

import numpy as np

ORACLE_DIR = Path(__file__).resolve().parent
LIB_PATH = ORACLE_DIR / "_build" / "liboracle.so"

P = C.c_void_p
I32 = C.c_int32
_lib = None


def build() -> Path:
    subprocess.run(["make", "-s", "-C", str(ORACLE_DIR)], check=True)
    return LIB_PATH


def lib():
    global _lib
    if _lib is not None:
        return _lib
    if not LIB_PATH.exists():
        build()
    L = C.CDLL(str(LIB_PATH))
    sig = {
        "orc_create_bounded": (P, [I32, I32, I32]),
        "orc_create_ring": (P, [I32, I32]),
        "orc_destroy": (None, [P]),
        "orc_load_grid": (C.c_int, [P, C.POINTER(C.c_uint32), C.POINTER(C.c_uint8), C.c_uint64, C.POINTER(C.c_int32)]),
        "orc_fill_box": (None, [P, I32, I32, I32, I32, I32, I32, C.c_uint8]),
        "orc_fill_sphere": (None, [P, C.c_float, C.c_float, C.c_float, C.c_float, C.c_uint8]),
        "orc_set_voxel": (None, [P, I32, I32, I32, C.c_uint8]),
        "orc_get_voxel": (C.c_uint8, [P, I32, I32, I32]),
        "orc_compact": (None, [P]),
        "orc_detailed_bricks": (C.c_uint64, [P]),
        "orc_grid_at": (C.c_uint32, [P, I32, I32, I32]),
        "orc_tick": (C.c_int, [P]),
        "orc_ticks": (C.c_int, [P, I32, I32]),
        "orc_update": (C.c_int, [P, C.c_float]),
        "orc_wake": (None, [P, I32, I32, I32, I32, I32, I32]),
        "orc_displace": (None, [P, I32, I32, I32]),
        "orc_emit": (None, [P, C.POINTER(C.c_int32), C.c_uint64, C.c_float]),
        "orc_apply_brush": (C.c_uint64, [P, C.POINTER(C.c_int32), C.c_uint64, C.c_uint8]),
        "orc_volume": (C.c_float, [P, I32, I32, I32]),
        "orc_set_partial": (None, [P, I32, I32, I32, C.c_float]),
        "orc_shift": (None, [P, I32, I32]),
        "orc_ring_rebase": (None, [P, I32, I32]),
        "orc_ring_evict": (None, [P, I32, I32]),
        "orc_ring_paste": (None, [P, C.POINTER(C.c_uint32), C.POINTER(C.c_uint8), C.c_uint64, I32, I32, I32]),
        "orc_reset": (None, [P]),
        "orc_idle": (C.c_int, [P]),
        "orc_active_count": (C.c_uint64, [P]),
        "orc_partial_count": (C.c_uint64, [P]),
        "orc_last_tick_cells": (C.c_uint64, [P]),
        "orc_tick_no": (C.c_uint32, [P]),
        "orc_level_round": (C.c_int, [P]),
        "orc_layer_mark": (C.c_int, [P, I32, I32, I32]),
        "orc_stats": (None, [P, C.POINTER(C.c_uint64)]),
        "orc_queue": (C.c_uint64, [P, C.POINTER(C.c_int32), C.c_uint64]),
        "orc_seeds": (C.c_uint64, [P, C.POINTER(C.c_int32), C.c_uint64]),
        "orc_export_box": (None, [P, I32, I32, I32, I32, I32, I32, C.POINTER(C.c_uint8), C.POINTER(C.c_float)]),
        "orc_state_digest": (C.c_uint64, [P]),
        "orc_queue_digest": (C.c_uint64, [P]),
        "orc_seed_digest": (C.c_uint64, [P]),
        "orc_total_box": (C.c_double, [P, I32, I32, I32, I32, I32, I32]),
        "orc_time_ticks": (C.c_double, [P, I32]),
        "orc_pf_create": (P, []),
        "orc_pf_destroy": (None, [P]),
        "orc_pf_set": (None, [P, I32, I32, I32, C.c_float]),
        "orc_pf_get": (C.c_float, [P, I32, I32, I32]),
        "orc_pf_erase": (None, [P, I32, I32, I32]),
        "orc_pf_len": (C.c_uint64, [P]),
        "orc_pf_entries": (C.c_uint64, [P, C.POINTER(C.c_int32), C.POINTER(C.c_float), C.c_uint64]),
    }
    for name, (res, args) in sig.items():
        f = getattr(L, name)
        f.restype = res
        f.argtypes = args
    _lib = L
    return L


STAT_NAMES = ("cells", "pull_attempts", "pull_nonempty", "pull_success", "bfs_visits", "level_calls", "level_cells", "level_fills", "drains",
              "activations", "ticks")


def _i32p(a):
    return a.ctypes.data_as(C.POINTER(C.c_int32))


class Oracle:
    """One SparseVolume + one FluidSim on the CPU (the reference's pairing)."""

    def __init__(self, nx=0, ny=0, nz=0, ring_w=0):
        L = lib()
        self.h = P(L.orc_create_ring(ring_w, ny) if ring_w else L.orc_create_bounded(nx, ny, nz))
        self.nx, self.ny, self.nz, self.ring_w = nx, ny, nz, ring_w

    @classmethod
    def from_arrays(cls, dims, grid, bricks, ring=None):
        """dims = (nx, ny, nz, ring_w); grid/bricks/ring in the reference's encoding."""
        nx, ny, nz, ring_w = dims
        o = cls(nx, ny, nz, ring_w)
        grid = np.ascontiguousarray(grid, np.uint32)
        bricks = np.ascontiguousarray(bricks, np.uint8)
        lib().orc_load_grid(o.h, grid.ctypes.data_as(C.POINTER(C.c_uint32)), bricks.ctypes.data_as(C.POINTER(C.c_uint8)),
                            bricks.size // 512, _i32p(np.ascontiguousarray(ring, np.int32)) if ring is not None else None)
        return o

    def __del__(self):
        if getattr(self, "h", None) and _lib is not None:
            _lib.orc_destroy(self.h)
            self.h = None

    # world
    def fill_box(self, *a):
        lib().orc_fill_box(self.h, *a)

    def fill_sphere(self, *a):
        lib().orc_fill_sphere(self.h, *a)

    def set_voxel(self, x, y, z, m):
        lib().orc_set_voxel(self.h, x, y, z, m)

    def get_voxel(self, x, y, z):
        return lib().orc_get_voxel(self.h, x, y, z)

    # fluid
    def tick(self, n=1):
        ch = False
        for _ in range(n):
            ch |= bool(lib().orc_tick(self.h))
        return ch

    def update(self, dt):
        return bool(lib().orc_update(self.h, dt))

    def wake(self, x0, y0, z0, x1, y1, z1):
        lib().orc_wake(self.h, x0, y0, z0, x1, y1, z1)

    def displace(self, x, y, z):
        lib().orc_displace(self.h, x, y, z)

    def emit(self, cells, amount):
        cells = np.ascontiguousarray(cells, np.int32)
        lib().orc_emit(self.h, _i32p(cells), len(cells), amount)

    def apply_brush(self, cells, m):
        cells = np.ascontiguousarray(cells, np.int32)
        return lib().orc_apply_brush(self.h, _i32p(cells), len(cells), m)

    def volume(self, x, y, z):
        return lib().orc_volume(self.h, x, y, z)

    def set_partial(self, x, y, z, v):
        lib().orc_set_partial(self.h, x, y, z, v)

    def shift(self, dx, dz):
        lib().orc_shift(self.h, dx, dz)

    def ring_rebase(self, dcx, dcz):
        """SparseVolume::ring_rebase: the floating origin moves by (dcx, dcz) chunks."""
        lib().orc_ring_rebase(self.h, dcx, dcz)

    def ring_evict(self, cx, cz):
        """SparseVolume::ring_evict (the FluidSim keeps its partial entries)."""
        lib().orc_ring_evict(self.h, cx, cz)

    def ring_paste(self, grid, bricks, bricks_y, cx, cz):
        """SparseVolume::ring_paste of a 128 x (bricks_y * 8) x 128 chunk (grid words, bricks)."""
        grid = np.ascontiguousarray(grid, np.uint32)
        bricks = np.ascontiguousarray(bricks, np.uint8)
        lib().orc_ring_paste(self.h, grid.ctypes.data_as(C.POINTER(C.c_uint32)), bricks.ctypes.data_as(C.POINTER(C.c_uint8)),
                             bricks.size // 512, bricks_y, cx, cz)

    def reset(self):
        lib().orc_reset(self.h)

    def idle(self):
        return bool(lib().orc_idle(self.h))

    def active_count(self):
        return lib().orc_active_count(self.h)

    def partial_count(self):
        return lib().orc_partial_count(self.h)

    def last_tick_cells(self):
        return lib().orc_last_tick_cells(self.h)

    def tick_no(self):
        return lib().orc_tick_no(self.h)

    def level_round(self):
        return bool(lib().orc_level_round(self.h))

    def stats(self):
        a = (C.c_uint64 * 11)()
        lib().orc_stats(self.h, a)
        return dict(zip(STAT_NAMES, list(a)))

    def queue(self):
        L = lib()
        n = L.orc_queue(self.h, None, 0)
        q = np.zeros(3 * max(n, 1), np.int32)
        L.orc_queue(self.h, _i32p(q), n)
        m = L.orc_seeds(self.h, None, 0)
        s = np.zeros(3 * max(m, 1), np.int32)
        L.orc_seeds(self.h, _i32p(s), m)
        return q[: 3 * n].reshape(-1, 3), s[: 3 * m].reshape(-1, 3)

    def export_box(self, x0, y0, z0, sx, sy, sz):
        mat = np.zeros(sx * sy * sz, np.uint8)
        part = np.zeros(sx * sy * sz, np.float32)
        lib().orc_export_box(self.h, x0, y0, z0, sx, sy, sz, mat.ctypes.data_as(C.POINTER(C.c_uint8)),
                             part.ctypes.data_as(C.POINTER(C.c_float)))
        return mat.reshape(sz, sy, sx), part.reshape(sz, sy, sx)

    def digest(self):
        L = lib()
        return L.orc_state_digest(self.h), L.orc_queue_digest(self.h), L.orc_seed_digest(self.h)

    def total(self, x0, y0, z0, x1, y1, z1):
        return lib().orc_total_box(self.h, x0, y0, z0, x1, y1, z1)

    def time_ticks(self, n):
        return lib().orc_time_ticks(self.h, n)


class PartialField:
    """The oracle's PartialField (src/fluid.rs:64-180) on its own."""

    def __init__(self):
        self.h = P(lib().orc_pf_create())

    def __del__(self):
        if getattr(self, "h", None) and _lib is not None:
            _lib.orc_pf_destroy(self.h)
            self.h = None

    def set(self, x, y, z, v):
        lib().orc_pf_set(self.h, x, y, z, v)

    def get(self, x, y, z):
        return lib().orc_pf_get(self.h, x, y, z)

    def erase(self, x, y, z):
        lib().orc_pf_erase(self.h, x, y, z)

    def __len__(self):
        return lib().orc_pf_len(self.h)

    def entries(self):
        n = lib().orc_pf_entries(self.h, None, None, 0)
        xyz = np.zeros(3 * max(n, 1), np.int32)
        v = np.zeros(max(n, 1), np.float32)
        lib().orc_pf_entries(self.h, _i32p(xyz), v.ctypes.data_as(C.POINTER(C.c_float)), n)
        return [(int(xyz[3 * i]), int(xyz[3 * i + 1]), int(xyz[3 * i + 2]), float(v[i])) for i in range(n)]
