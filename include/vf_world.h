/* vf_world.h — host-side sparse brick world and the synthetic workloads.
 *
 * vf_world is the host mirror of the reference's SparseVolume (src/voxel/sparse_volume.rs:90-114):
 * a grid of 8^3 bricks, one u32 per brick (0 = empty, 1..255 = uniform material, >= 256 =
 * detailed brick index + 256, voxel index lz*64 + ly*8 + lx), in bounded or ring (toroidal,
 * streaming) mode. It is what a C/C++ caller hands to vf_fluid (vf_fluid.h) and what receives
 * the fluid's voxel changes, exactly as the Rust host's SparseVolume would.
 *
 * All functions are host-only (no GPU needed) and return VF_OK (0) or a negative VF_ERR_* code
 * where they return int.
 */
#ifndef VF_WORLD_H
#define VF_WORLD_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define VF_AIR 0
#define VF_STONE 3
#define VF_WATER 5 /* src/fluid.rs:24, src/voxel/world.rs:46 */

typedef struct vf_world vf_world;

typedef struct vf_world_info {
  int32_t nx, ny, nz;                /* voxel dims (ring: the window span) */
  int32_t bricks_x, bricks_y, bricks_z;
  int32_t ring_w;                    /* 0 = bounded volume */
  int32_t origin_x, origin_z;
  uint64_t nbricks;                  /* detailed bricks allocated (incl. freed ones) */
  uint64_t detailed;                 /* detailed bricks in use */
} vf_world_info;

/* SparseVolume::new (sparse_volume.rs:117-139). */
int vf_world_create(int32_t nx, int32_t ny, int32_t nz, vf_world** out);
/* SparseVolume::ring_init (sparse_volume.rs:177-192); w a power of two. */
int vf_world_create_ring(int32_t w, int32_t ny, vf_world** out);
void vf_world_destroy(vf_world* w);
int vf_world_get_info(const vf_world* w, vf_world_info* out);

/* Voxel access (sparse_volume.rs:228-326). */
uint8_t vf_world_get_voxel(const vf_world* w, int32_t x, int32_t y, int32_t z);
void vf_world_set_voxel(vf_world* w, int32_t x, int32_t y, int32_t z, uint8_t m);
/* Replay n voxel changes through set_voxel, in order: the host side of FluidSim's write-back
 * (src/fluid.rs:327-355 writes materials with SparseVolume::set_voxel). `changes` is an array of
 * n records of 16 bytes as written by vf_fluid_download_changes (int32 x, y, z, uint8 material,
 * 3 bytes padding). */
void vf_world_set_voxels(vf_world* w, const void* changes, uint64_t n);
void vf_world_fill_box(vf_world* w, int32_t x0, int32_t y0, int32_t z0, int32_t x1, int32_t y1, int32_t z1, uint8_t m);
void vf_world_fill_sphere(vf_world* w, float cx, float cy, float cz, float r, uint8_t m);
void vf_world_compact(vf_world* w);
/* Ring paste / evict (sparse_volume.rs:478-537). */
int vf_world_ring_paste(vf_world* ring, const vf_world* chunk, int32_t cx, int32_t cz);
int vf_world_ring_evict(vf_world* ring, int32_t cx, int32_t cz);
/* SparseVolume::ring_rebase (sparse_volume.rs:194-203): the floating origin moves by (dcx, dcz)
 * chunks; every slot's owner moves, the bricks stay. Pair it with vf_fluid_shift(dcx * 128,
 * dcz * 128) on the handles simulating this world. */
int vf_world_ring_rebase(vf_world* ring, int32_t dcx, int32_t dcz);
int vf_world_chunk_loaded(const vf_world* w, int32_t cx, int32_t cz);

/* Raw views of the grid (bricks_x*bricks_y*bricks_z u32), the brick pool (nbricks*512 u8) and
 * the ring slots (ring_w*ring_w triples cx, cz, loaded). Valid until the next mutating call. */
const uint32_t* vf_world_grid(const vf_world* w);
const uint8_t* vf_world_bricks(const vf_world* w);
int vf_world_ring_slots(const vf_world* w, int32_t* out_triples);

/* Grid indices pushed by set_voxel since the last call (sparse_volume.rs:289-291; the
 * renderer's dirty list). Returns the count; copies at most cap. Clears the list. */
size_t vf_world_take_dirty(vf_world* w, uint32_t* out, size_t cap);

/* ---------------------------------------------------------------- synthetic workloads
 * Each workload is one or more regions (independent worlds, each stepped by its own fluid
 * sim) plus a script of host edits between ticks. Workload ids:
 *   1 basin 64^3, 2 dam break 512x128x512, 3 batched regions, 4 ring world + rain emitters,
 *   5 batched regions + sphere edits.
 * `scale` in (0, 1] shrinks the horizontal extents (1 = the full workload) for tests.
 */
typedef struct vf_workload vf_workload;

typedef struct vf_workload_info {
  int32_t id;
  int32_t regions;
  int32_t ticks;            /* ticks the workload runs */
  int32_t emit_every;       /* rain: emit every N ticks (0 = none) */
  int32_t edit_every;       /* sphere edits every N ticks (0 = none) */
  uint64_t resident_cells;  /* sum over regions of addressable cells */
} vf_workload_info;

int vf_workload_build(int32_t id, float scale, uint64_t seed, vf_workload** out);
void vf_workload_destroy(vf_workload* wl);
int vf_workload_get_info(const vf_workload* wl, vf_workload_info* out);
/* The region's initial world (owned by the workload; copy it before mutating). */
const vf_world* vf_workload_world(const vf_workload* wl, int32_t region);
/* Initial wake boxes: n boxes of 6 ints (x0,y0,z0,x1,y1,z1), inclusive. */
size_t vf_workload_wakes(const vf_workload* wl, int32_t region, int32_t* out6, size_t cap);
/* Rain emitter cells of a region (x,y,z triples) and the volume each adds per emission. */
size_t vf_workload_emitters(const vf_workload* wl, int32_t region, int32_t* out3, size_t cap, float* amount);
/* The sphere edit applied to `region` right before tick `tick` (0-based), if any: returns the
 * number of brush cells written to out3 (x,y,z in the reference's fill_sphere order), the
 * brush material in *m (0 = carve) and the wake box (bbox +- 1) in wake6. 0 = no edit. */
size_t vf_workload_edit(const vf_workload* wl, int32_t region, int32_t tick, int32_t* out3, size_t cap, uint8_t* m, int32_t* wake6);

/* Copy a world (deep). */
int vf_world_clone(const vf_world* w, vf_world** out);

#ifdef __cplusplus
}
#endif
#endif
