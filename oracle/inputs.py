"""ORACLE inputs — test infrastructure only.

The synthetic workloads (noise-terrain worlds, wake boxes, rain emitters, sphere edits) built by
oracle/_build/libvf_inputs.so, the workload generator compiled on its own by oracle/Makefile. The
CPU arm of the benchmark and the checker use it to build exactly the inputs the engine gets,
without loading the engine's library.
"""
from __future__ import annotations

import ctypes as C
import subprocess
from pathlib import Path

import numpy as np

ORACLE_DIR = Path(__file__).resolve().parent
LIB_PATH = ORACLE_DIR / "_build" / "libvf_inputs.so"
P = C.c_void_p
I32 = C.c_int32
_lib = None


class _WorldInfo(C.Structure):
    _fields_ = [(n, C.c_int32) for n in ("nx", "ny", "nz", "bricks_x", "bricks_y", "bricks_z", "ring_w", "origin_x", "origin_z")] + [
        ("nbricks", C.c_uint64),
        ("detailed", C.c_uint64),
    ]


class _WorkloadInfo(C.Structure):
    _fields_ = [(n, C.c_int32) for n in ("id", "regions", "ticks", "emit_every", "edit_every")] + [("resident_cells", C.c_uint64)]


def lib():
    global _lib
    if _lib is not None:
        return _lib
    if not LIB_PATH.exists():
        subprocess.run(["make", "-s", "-C", str(ORACLE_DIR)], check=True)
    L = C.CDLL(str(LIB_PATH))
    sig = {
        "vf_workload_build": (C.c_int, [I32, C.c_float, C.c_uint64, C.POINTER(P)]),
        "vf_workload_destroy": (None, [P]),
        "vf_workload_get_info": (C.c_int, [P, C.POINTER(_WorkloadInfo)]),
        "vf_workload_world": (P, [P, I32]),
        "vf_workload_wakes": (C.c_size_t, [P, I32, C.POINTER(I32), C.c_size_t]),
        "vf_workload_emitters": (C.c_size_t, [P, I32, C.POINTER(I32), C.c_size_t, C.POINTER(C.c_float)]),
        "vf_workload_edit": (C.c_size_t, [P, I32, I32, C.POINTER(I32), C.c_size_t, C.POINTER(C.c_uint8), C.POINTER(I32)]),
        "vf_world_get_info": (C.c_int, [P, C.POINTER(_WorldInfo)]),
        "vf_world_grid": (C.POINTER(C.c_uint32), [P]),
        "vf_world_bricks": (C.POINTER(C.c_uint8), [P]),
        "vf_world_ring_slots": (C.c_int, [P, C.POINTER(I32)]),
    }
    for name, (res, args) in sig.items():
        f = getattr(L, name)
        f.restype = res
        f.argtypes = args
    _lib = L
    return L


def _i32p(a):
    return a.ctypes.data_as(C.POINTER(I32))


class Inputs:
    """Workload `wid` at `scale` (seed `seed`): its regions' worlds and host-edit script."""

    def __init__(self, wid: int, scale: float = 1.0, seed: int = 1):
        L = lib()
        h = P()
        rc = L.vf_workload_build(wid, scale, seed, C.byref(h))
        if rc:
            raise RuntimeError(f"vf_workload_build({wid}, {scale}, {seed}) failed: {rc}")
        self.h = h
        i = _WorkloadInfo()
        L.vf_workload_get_info(h, C.byref(i))
        self.id, self.regions, self.ticks = i.id, i.regions, i.ticks
        self.emit_every, self.edit_every = i.emit_every, i.edit_every

    def __del__(self):
        if getattr(self, "h", None) and _lib is not None:
            _lib.vf_workload_destroy(self.h)
            self.h = None

    def arrays(self, r: int):
        """((nx, ny, nz, ring_w), grid u32, bricks u8, ring slots i32 or None) of region r, copied."""
        L = lib()
        w = L.vf_workload_world(self.h, r)
        i = _WorldInfo()
        L.vf_world_get_info(w, C.byref(i))
        nb = i.bricks_x * i.bricks_y * i.bricks_z
        grid = np.ctypeslib.as_array(L.vf_world_grid(w), shape=(nb,)).copy()
        bricks = np.ctypeslib.as_array(L.vf_world_bricks(w), shape=(i.nbricks * 512,)).copy() if i.nbricks else np.zeros(512, np.uint8)
        ring = None
        if i.ring_w:
            ring = np.zeros(3 * i.ring_w * i.ring_w, np.int32)
            L.vf_world_ring_slots(w, _i32p(ring))
        return (i.nx, i.ny, i.nz, i.ring_w), grid, bricks, ring

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
        """(cells (n, 3) int32, material, wake box) of the edit before `tick`, or None."""
        L = lib()
        m = C.c_uint8()
        wake = np.zeros(6, np.int32)
        n = L.vf_workload_edit(self.h, r, tick, None, 0, C.byref(m), _i32p(wake))
        if n == 0:
            return None
        a = np.zeros(3 * n, np.int32)
        L.vf_workload_edit(self.h, r, tick, _i32p(a), n, C.byref(m), _i32p(wake))
        return a.reshape(-1, 3), int(m.value), wake


def oracle_for(orc, inp: Inputs, r: int):
    """An oracle holding region r's initial world with its wake boxes applied."""
    dims, grid, bricks, ring = inp.arrays(r)
    o = orc.Oracle.from_arrays(dims, grid, bricks, ring)
    for b in inp.wakes(r):
        o.wake(*map(int, b))
    return o


def script_step(o, inp: Inputs, r: int, t: int, emitters=None):
    """The host edits that act before tick t (emitters when t % emit_every == 0, a sphere edit when
    t % edit_every == edit_every - 1), then tick t."""
    if inp.emit_every and t % inp.emit_every == 0:
        em, amt = emitters if emitters is not None else inp.emitters(r)
        if len(em):
            o.emit(em, amt)
    if inp.edit_every and t % inp.edit_every == inp.edit_every - 1:
        ed = inp.edit(r, t)
        if ed is not None:
            o.apply_brush(ed[0], ed[1])
            o.wake(*map(int, ed[2]))
    o.tick()
