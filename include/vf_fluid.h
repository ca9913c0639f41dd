/* vf_fluid.h — C ABI of the B200 CA-water engine (drop-in for the reference's FluidSim).
 *
 * The reference's fluid (src/fluid.rs:230-721) is a Rust struct `FluidSim` whose methods borrow
 * the world (`&mut SparseVolume`). This ABI keeps those methods one to one; the world lives on
 * the device as a brick table + atlases mirrored from the host's SparseVolume at
 * vf_fluid_upload_world, and every voxel the fluid changes is handed back to the host by
 * vf_fluid_download_changes so the host replays it through SparseVolume::set_voxel (which
 * feeds the renderer's dirty_grid, src/voxel/sparse_volume.rs:289-291).
 *
 * Conventions follow the reference's own FFI layer (native/ngx_shim.cpp:18-45,
 * src/gfx/dlss/ngx.rs:23-38): `vf_`-prefixed extern "C" functions returning int (0 = OK,
 * negative = error), opaque handles, out-parameters, explicit destroy. A handle is not
 * thread-safe, like the reference's `&mut self`; one handle per CUDA stream.
 *
 * Results are bit-identical to fluid.rs semantics: f32 volumes, f64 level sums, the same FIFO
 * order, 50k-cell cap, pull budget, levelling rounds and seed order.
 */
#ifndef VF_FLUID_H
#define VF_FLUID_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- status codes */
#define VF_OK 0
#define VF_ERR_INVALID (-1)   /* bad argument / handle */
#define VF_ERR_OOM (-2)       /* device or host allocation failed, or a fixed capacity is full */
#define VF_ERR_CUDA (-3)      /* a CUDA call failed (vf_fluid_last_error has the text) */
#define VF_ERR_TIMEOUT (-4)   /* a bounded device-side wait gave up (the sim state is undefined) */
#define VF_ERR_RANGE (-5)     /* a coordinate outside the addressable domain */
#define VF_ERR_NO_DEVICE (-6) /* no CUDA device / the sm_100a image cannot load */
#define VF_ERR_STATE (-7)     /* call not valid in the current state (e.g. tick before upload) */

/* ---- constants of the reference (src/fluid.rs:24-44) */
#define VF_FLUID_WATER 5
#define VF_FLUID_TICK_HZ 20.0f
#define VF_FLUID_MAX_CELLS_PER_TICK 50000
#define VF_FLUID_MAX_PULLS_PER_TICK 4096
#define VF_FLUID_LEVEL_BUDGET 40000
#define VF_FLUID_MAX_LEVEL_SEEDS 4096
#define VF_FLUID_MAX_LEVEL_CELLS 400000

typedef struct vf_fluid vf_fluid;

typedef struct vf_fluid_desc {
  int32_t device;          /* CUDA device ordinal */
  void* stream;            /* cudaStream_t to run on (NULL = the handle creates its own) */
  uint64_t atlas_bricks;   /* capacity of the device brick atlas (0 = sized from the world) */
  uint64_t queue_capacity; /* FIFO capacity in cells (0 = sized from the domain) */
} vf_fluid_desc;

/* A voxel edit or a voxel change: absolute coordinates + material. */
typedef struct vf_voxel {
  int32_t x, y, z;
  uint8_t m;
  uint8_t pad[3];
} vf_voxel;

typedef struct vf_fluid_stats {
  uint64_t tick_no;            /* FluidSim::tick_no */
  uint64_t last_tick_cells;    /* FluidSim::last_tick_cells (src/fluid.rs:271-273) */
  uint64_t active_count;       /* FluidSim::active_count (:262-264) */
  uint64_t partial_count;      /* FluidSim::partial_count (:268-270) */
  uint64_t seed_count;         /* level seeds pending */
  uint64_t level_round;        /* a levelling round is open */
  uint64_t last_level_cells;   /* cells levelled in the last levelling pass */
  uint64_t memory_bytes;       /* device bytes held by this handle (FluidSim::memory_bytes) */
  uint64_t cells_total;        /* sum of last_tick_cells over all ticks */
  uint64_t pull_attempts;      /* pressure pulls attempted, all ticks */
  uint64_t pull_success;       /* pressure pulls that moved water */
  uint64_t bfs_visits;         /* pressure-BFS queue entries examined */
  uint64_t level_cells_total;  /* cells gathered by level flood fills */
  uint64_t atlas_used;         /* device bricks materialised */
  uint64_t changes_pending;    /* voxel changes not yet downloaded */
} vf_fluid_stats;

/* FluidSim::default(). */
int vf_fluid_create(const vf_fluid_desc* desc, vf_fluid** out);
void vf_fluid_destroy(vf_fluid* h);
const char* vf_fluid_last_error(const vf_fluid* h);

/* Mirror the host world onto the device (grid u32 per brick in the reference encoding, bricks
 * 512 bytes each, ring slots as (cx, cz, loaded) triples when ring_w > 0). Replaces any world
 * uploaded before; the fluid state (queue, partials) is kept. */
int vf_fluid_upload_world(vf_fluid* h, int32_t nx, int32_t ny, int32_t nz, int32_t bricks_x, int32_t bricks_y,
                          int32_t bricks_z, const uint32_t* grid, const uint8_t* bricks, uint64_t nbricks,
                          int32_t ring_w, const int32_t* ring_slots);

/* Host voxel writes made outside the fluid (brush, undo, paste) mirrored to the device; call
 * before the next tick. */
int vf_fluid_apply_voxel_edits(vf_fluid* h, const vf_voxel* edits, uint64_t n);

/* FluidSim::wake (src/fluid.rs:358-366), box inclusive. */
int vf_fluid_wake(vf_fluid* h, int32_t x0, int32_t y0, int32_t z0, int32_t x1, int32_t y1, int32_t z1);
/* FluidSim::displace (src/fluid.rs:370-408). */
int vf_fluid_displace(vf_fluid* h, int32_t x, int32_t y, int32_t z);
/* apply_brush with displace as its on_water hook (src/edit/brush.rs:93-111,
 * src/app/scene_edit.rs:231-232): for each cell in order, carve (m = 0) clears solid voxels,
 * place (m != 0) fills air/water voxels, displacing water first. *n_changed = voxels written. */
int vf_fluid_apply_brush(vf_fluid* h, const int32_t* xyz, uint64_t n, uint8_t m, uint64_t* n_changed);
/* Rain emitter (harness edit): for each cell, vol' = min(1, vol + amount) through set_volume,
 * then wake the cell. */
int vf_fluid_emit(vf_fluid* h, const int32_t* xyz, uint64_t n, float amount);
/* FluidSim::set_partial (src/fluid.rs:278-282). */
int vf_fluid_set_partial(vf_fluid* h, int32_t x, int32_t y, int32_t z, float v);

/* FluidSim::tick (src/fluid.rs:564-657), n_ticks times back to back on the device.
 * *changed (optional) = 1 if any voxel changed. */
int vf_fluid_tick(vf_fluid* h, int32_t n_ticks, int32_t* changed);
/* The same ticks, enqueued on the handle's stream without waiting (capturable in a CUDA graph);
 * vf_fluid_sync waits and reports the device status. */
int vf_fluid_tick_async(vf_fluid* h, int32_t n_ticks);
int vf_fluid_sync(vf_fluid* h);
/* The cudaStream_t the handle runs on. */
void* vf_fluid_stream(vf_fluid* h);
/* FluidSim::update (src/fluid.rs:662-676): fixed 20 Hz, at most 3 ticks per call. */
int vf_fluid_update(vf_fluid* h, float dt, int32_t* changed);

/* Voxel changes since the last download (final material per changed voxel, any order).
 * Writes at most cap entries, sets *n to the total pending; entries not copied stay pending. */
int vf_fluid_download_changes(vf_fluid* h, vf_voxel* out, uint64_t cap, uint64_t* n);

/* The same download for callers that must not allocate device memory while they run (no
 * counterpart in the reference, whose fluid lives in host memory). A per-frame game loop cannot
 * take the device-wide stall an allocation may cause, and an engine that fixes every subsystem's
 * memory budget at start-up forbids allocating later; this entry point calls no cudaMalloc,
 * cudaFree or allocating library routine. It gathers through one fixed device array of
 * VF_NOALLOC_MAX_CHANGES changes that each device keeps until the process exits; with out set, cap
 * above that is rejected with VF_ERR_RANGE (a count-only call, out = NULL, takes any cap). The first
 * call on a device looks the array's address up with that device current, then makes the caller's
 * current device current again (make that first call before any stream capture). Every call on a
 * device shares the array and
 * overwrites what the last call left there, so calls whose GPU work overlaps race: serialise them.
 * Same contract as vf_fluid_download_changes otherwise: at most cap entries, *n = total pending,
 * the rest stay pending. */
#define VF_NOALLOC_MAX_CHANGES 65536
int vf_fluid_download_changes_noalloc(vf_fluid* h, vf_voxel* out, uint64_t cap, uint64_t* n);

/* FluidSim::volume (src/fluid.rs:251-260). */
int vf_fluid_volume(vf_fluid* h, int32_t x, int32_t y, int32_t z, float* out);
/* FluidSim::idle (:265-267). */
int vf_fluid_idle(vf_fluid* h, int32_t* out);
int vf_fluid_get_stats(vf_fluid* h, vf_fluid_stats* out);

/* FluidSim::partials().for_each (src/fluid.rs:165-175): every partial cell as (x,y,z) + volume,
 * in ascending (page, local index) order. Writes at most cap, *n = total. */
int vf_fluid_export_partials(vf_fluid* h, int32_t* xyz, float* vol, uint64_t cap, uint64_t* n);
/* FluidSim::shift (src/fluid.rs:696-720): floating origin moved by (dx, dz) voxels. Ring worlds
 * only, by whole ring periods (ring_w * 128 voxels: the only moves src/app/window.rs:393-408 makes,
 * ORIGIN_STEP = 65536); pair it with SparseVolume::ring_rebase / vf_world_ring_rebase on the host.
 * VF_ERR_RANGE otherwise. */
int vf_fluid_shift(vf_fluid* h, int32_t dx, int32_t dz);
/* Ring streaming on a live handle, on the handle's device copy of the world
 * (SparseVolume::ring_evict / ring_paste, src/voxel/sparse_volume.rs:478-537; the host calls the
 * same on its SparseVolume). Evict empties the ring slot holding chunk (cx, cz) (a slot not loaded:
 * nothing) and frees its bricks' atlas slots; the partial volumes its cells held are kept per cell,
 * as FluidSim's PartialField keeps them, and count in vf_fluid_get_stats / export / digests. A
 * drained cell of an unloaded chunk erases its kept entry (fluid.rs:586-589). Paste evicts the
 * slot's chunk, then writes the chunk given as a SparseVolume of 128 x (chunk_bricks_y * 8) x 128
 * voxels (grid in the reference's encoding, 16 x chunk_bricks_y x 16 words; bricks 512 bytes each)
 * into the slot as chunk (cx, cz); kept entries of its cells come back into its bricks. The FIFO,
 * the level seeds and the marks are untouched, as in the reference. The chunk must lie inside the
 * handle's cell domain (the box of the chunks loaded at upload, moved by shifts): VF_ERR_RANGE
 * otherwise; VF_ERR_OOM when the atlas is full. */
int vf_fluid_ring_evict(vf_fluid* h, int32_t cx, int32_t cz);
int vf_fluid_ring_paste(vf_fluid* h, const uint32_t* chunk_grid, const uint8_t* chunk_bricks, uint64_t chunk_nbricks, int32_t chunk_bricks_y,
                        int32_t cx, int32_t cz);
/* FluidSim::reset (src/fluid.rs:318-320): the fluid state only; the world mirror stays, and so
 * do the cumulative counters of vf_fluid_get_stats and vf_fluid_profile. */
int vf_fluid_reset(vf_fluid* h);

/* Differential-test snapshot: the FIFO (x,y,z triples, oldest first) and the level seed list
 * (bottom to top). Writes at most cap of each; *nq / *ns = lengths. */
int vf_fluid_snapshot_queue(vf_fluid* h, int32_t* q_xyz, uint64_t q_cap, uint64_t* nq, int32_t* s_xyz, uint64_t s_cap, uint64_t* ns);
/* Dense export of a box: materials and partial volumes (0 = no partial entry), index
 * ((z-z0)*sy + (y-y0))*sx + (x-x0). */
int vf_fluid_export_box(vf_fluid* h, int32_t x0, int32_t y0, int32_t z0, int32_t sx, int32_t sy, int32_t sz, uint8_t* mat, float* part);
/* Order-independent digests, computed on the device, of the voxel+partial state and of the
 * FIFO and seed list (same definitions as the test oracle's). */
int vf_fluid_digest(vf_fluid* h, uint64_t* state, uint64_t* queue, uint64_t* seeds);

/* Cycle counters per tick phase, summed over all ticks (SM clock of the region's CTA): 0 drain,
 * 1 sort, 2 sweep, 3 sweep waiting on prefetch, 4 pressure pulls, 5 activation logging, 6 voxel
 * writes, 7 seed commit, 8 levelling, 9 FIFO commit, 10 change commit, 11 mark clearing,
 * 15 between ticks. */
int vf_fluid_profile(vf_fluid* h, uint64_t* out16);

/* ---- learned wake proposal (pattern (4)). Rows are atlas slots (materialised bricks).
 * Features: nslots x 32 fp16 into device memory (advances a 4-call history: call once per tick).
 * Labels: 1.0 where the brick's cells were drained in (since_tick, now]. Staging: L2 prefetch of
 * the bricks whose probability >= threshold; it never changes what the fluid computes. */
int vf_fluid_proposal_features(vf_fluid* h, void* dev_x_f16, uint64_t cap_slots, uint64_t* nslots);
int vf_fluid_proposal_labels(vf_fluid* h, uint32_t since_tick, float* dev_y, uint64_t nslots);
int vf_fluid_stage_bricks(vf_fluid* h, const float* dev_prob, uint64_t nslots, float threshold, uint64_t* n_staged);

/* The proposal network: 32 -> 64 -> 64 -> 1 (ReLU, ReLU, sigmoid), fp16 tensor-core forward and
 * backward kernels, fp32 master weights, Adam. All tensors are device pointers; flat fp32
 * parameters: W1[32][64], b1[64], W2[64][64], b2[64], w3[64], b3. */
typedef struct vf_mlp vf_mlp;
int vf_mlp_create(int32_t device, uint64_t seed, vf_mlp** out);
void vf_mlp_destroy(vf_mlp* m);
int vf_mlp_nparams(void);
int vf_mlp_get_params(vf_mlp* m, float* host_out);
int vf_mlp_set_params(vf_mlp* m, const float* host_in);
int vf_mlp_forward(vf_mlp* m, const void* dev_x_f16, uint64_t n, float* dev_prob, void* stream);
int vf_mlp_grads(vf_mlp* m, const void* dev_x_f16, const float* dev_y, uint64_t n, float* host_grads, void* stream);
int vf_mlp_train_step(vf_mlp* m, const void* dev_x_f16, const float* dev_y, uint64_t n, float lr, float* host_loss, void* stream);

/* Launch knobs of the one-warp sweep (the autotuner's search space; results never depend on them):
 * warps prefetching footprints (1..7) and how many cells ahead of the sweep they run (1..64). */
int vf_fluid_set_tuning(vf_fluid* h, int32_t producers, int32_t depth);

/* Which sweep runs FluidSim::tick's cell loop (src/fluid.rs:584-651); results never depend on it.
 * engine 2 (default): chosen per tick call from the last calls' pressure-search entries per drained
 * cell (above 1.5: engine 0, else engine 1; a batch launch uses its first handle's last choice).
 * engine 0: one warp walks the sorted cells (8 warps per region: the sweep and prefetchers).
 * engine 1: all 16 warps of the region's CTA walk rows of the sorted order at once, each
 * cell waiting for the earlier cells it conflicts with; pressure searches read cells as of their own
 * position; a segment whose order the schedule cannot keep is undone and replayed by one warp.
 * gate: bits 0-7 (0..31, default 4) before a pressure search, wait for the earlier cells of its layer
 * within this Chebyshev distance; bits 8-15 (0..31, 0 = the same value, default 1) a cell of a segment with
 * pulls starts only when rows in work on lower layers within that many rows have passed its x plus
 * that distance (fewer replays, less overlap); bits 16-20 (0 = 16, else 8..16) the warps of the
 * region's CTA (for measuring the speed-up against warps); bit 21: pressure searches leave the four
 * search contexts in shared memory unused and run on each warp's context in global memory (the path
 * a search takes when the shared ones are all in use; for tests). spin_cap (> 0, default 2^24): iterations of any device
 * wait (both engines, and the levelling's brick materialisation) before the tick gives up with
 * VF_ERR_TIMEOUT; the kernel then returns and the handle can only be destroyed.
 * No reference counterpart: a device scheduling knob of this library. */
int vf_fluid_set_sweep(vf_fluid* h, int32_t engine, int32_t gate, uint64_t spin_cap);

/* Parallel-sweep counters summed over ticks: budget segments run, segments undone and replayed in
 * sorted order, cells replayed, and (conflicts3, 3 entries, optional) the conflicts that caused the
 * replays: a later reader of a pull's source had started, a later pull had read the source, more
 * cells of a segment attempted a pull than the tick's budget had left (cells that earlier pulls
 * took below full). No reference counterpart (diagnostics). */
int vf_fluid_sweep_stats(vf_fluid* h, uint64_t* segments, uint64_t* rollbacks, uint64_t* replayed, uint64_t* conflicts3);

/* Lower the per-tick event-log capacities (activations, level seeds, voxel changes; each 1 .. its
 * allocated size, 2^22 / 2^18 / 2^21). A tick whose events overflow a log fails with VF_ERR_OOM
 * (the state is then undefined). The allocated sizes hold any tick (at most 50,000 drained cells);
 * lower values serve tests of the overflow path. No reference counterpart. */
int vf_fluid_set_log_caps(vf_fluid* h, uint32_t act, uint32_t seed, uint32_t chg);

/* Parallel-sweep SM cycle counters summed over ticks (18 entries): prepass, segments, rollbacks,
 * event logs; then summed over warps: dependency waits, blocked starts, footprint loads, pulls,
 * writes, cells run, row fetches, worker total, lower-layer (cone) waits, gate waits, pressure
 * searches run, search rounds, cycles in search reads, cycles in source writes. No reference
 * counterpart (diagnostics). */
int vf_fluid_sweep_profile(vf_fluid* h, uint64_t* out18);

/* Non-blocking host edits whose cell lists already live in device memory (x,y,z int32 triples),
 * for scripted runs captured in CUDA graphs: rain emitters, brush edits, wake boxes. */
int vf_fluid_emit_device_async(vf_fluid* h, const int32_t* dev_xyz, uint64_t n, float amount);
int vf_fluid_brush_device_async(vf_fluid* h, const int32_t* dev_xyz, uint64_t n, uint8_t m);
int vf_fluid_wake_async(vf_fluid* h, int32_t x0, int32_t y0, int32_t z0, int32_t x1, int32_t y1, int32_t z1);

/* A batch: many regions stepped by one launch, one CTA per region, on hs[0]'s stream.
 * vf_batch_capture records `launches` launches of `ticks_per_launch` ticks as a CUDA graph that
 * vf_batch_replay relaunches; vf_batch_sync waits and checks every region's status. */
typedef struct vf_batch vf_batch;
int vf_batch_create(vf_fluid* const* hs, int32_t n, vf_batch** out);
void vf_batch_destroy(vf_batch* b);
int vf_batch_tick_async(vf_batch* b, int32_t n_ticks);
int vf_batch_sync(vf_batch* b);
int vf_batch_capture(vf_batch* b, int32_t launches, int32_t ticks_per_launch);
int vf_batch_replay(vf_batch* b);
/* Record everything enqueued on the batch's stream between these two calls (tick launches,
 * device edits, wakes; every handle must run on the batch's stream) as the graph to replay. */
int vf_batch_begin_capture(vf_batch* b);
int vf_batch_end_capture(vf_batch* b);

/* ---- batched regions: pattern (2) of the engine. Every handle is an independent FluidSim
 * (its own world, FIFO, caps); one launch steps all of them n_ticks times, one CTA per region.
 * All handles must live on the same device; the launch runs on hs[0]'s stream. */
int vf_fluid_batch_tick(vf_fluid* const* hs, int32_t n, int32_t n_ticks);

#ifdef __cplusplus
}
#endif
#endif
