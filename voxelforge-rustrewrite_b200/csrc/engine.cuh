// Device data structures and per-cell rules of the CA-water engine (sm_100a).
//
// Semantics restate the reference's FluidSim (src/fluid.rs:230-721); every function cites the
// lines it follows. Layout:
//   * world mirror: grid u32 per 8^3 brick in the reference's encoding (sparse_volume.rs:3-6)
//     where a detailed brick's value is 256 + a slot of the device atlas; the atlas holds
//     materials (u8[512]) and partial volumes (f32[512], 0 = no partial entry, fluid.rs:64-79)
//     per slot, both with the reference's voxel index lz*64 + ly*8 + lx (== PartialField's
//     local index x | y<<3 | z<<6). Uniform bricks stay grid values until the fluid writes them.
//   * scheduler sets (active, level seeds, layer marks, changed voxels) are dense bitmaps over a
//     padded cell domain; the FIFO is a ring of u32 cell ids of that domain.
//
// Floating point: compiled with -fmad=false and no fast-math; f32 where fluid.rs uses f32 and f64
// where it uses f64, so every result is bit-identical to the reference's sequential sweep.
#pragma once
#include <cstdint>

namespace vfe {

constexpr uint8_t WATER = 5;
constexpr float SHOW_AT = 0.5f;
constexpr float HIDE_BELOW = 0.3f;
constexpr float EVAPORATE = 1e-4f;
constexpr float MIN_SPREAD = 0.05f;
constexpr float MIN_FLOW = 1e-4f;
constexpr float SLEEP = 1e-3f;
constexpr uint32_t MAX_CELLS_PER_TICK = 50000;
constexpr uint32_t LEVEL_TICKS = 10;
constexpr uint32_t MAX_LEVEL_CELLS = 400000;
constexpr uint32_t PRESSURE_SEARCH = 512;
constexpr uint32_t MAX_PULLS_PER_TICK = 4096;
constexpr uint32_t LEVEL_BUDGET = 40000;
constexpr uint32_t MAX_LEVEL_SEEDS = 4096;
constexpr uint32_t NOSLOT = 0xFFFFFFFFu;
// Press-BFS queue bound: 5 start cells + 5 pushes per examined entry, 512 entries examined.
constexpr uint32_t PRESS_QCAP = 5 + 5 * PRESSURE_SEARCH + 8;
constexpr uint32_t VIS_CAP = 4096;  // smem visited hash for cells outside the bitmap box (load <= 63%)
// Visited bitmap of a pressure search: a box of 64 x 64 (x, z around the start) x 64 (y from the
// start up) cells, one bit each; cells outside it use the hash.
constexpr int VB_SIDE = 64;
constexpr uint32_t VB_WORDS = VB_SIDE * VB_SIDE * VB_SIDE / 32;

// status codes written to Ctl::status by device code (mirrors VF_ERR_*)
constexpr int ST_OK = 0;
constexpr int ST_OOM = -2;
constexpr int ST_TIMEOUT = -4;
constexpr int ST_RANGE = -5;

struct Ctl {
  unsigned long long qhead, qtail;  // FIFO positions (monotonic)
  unsigned long long cells_total, pull_attempts, pull_success, bfs_visits, level_cells_total, activations;
  long long partial_count;
  unsigned long long nchg;          // changed voxels pending download
  unsigned int tick_no, level_round, nseeds, atlas_used;
  unsigned int last_cells, last_level_cells, changed, mark_ntiles;
  int status;
  unsigned int err_info;
  unsigned int seg_epoch;           // parallel sweep: segments begun so far (tags versions and reads)
  unsigned int ptn;                 // parallel sweep: cells listed in Region::ptlist this tick
  unsigned int pxn;                 // parallel sweep: positions listed in Region::pxlist this tick
  unsigned int att_ratio;           // parallel sweep: pull attempts per possible attempter of the
                                    // last tick's completed segments, x 65536 (0: none yet)
  unsigned int ndetached;           // ring worlds: partial entries kept for evicted chunks (detbits set)
  // parallel sweep diagnostics, summed over ticks: budget segments run, segments rolled back and
  // replayed in order by one warp, cells replayed
  unsigned long long par_segments, par_rollbacks, par_replayed;
  // conflicts by kind: a later reader of a pull's source had started, a later pull had read the
  // source, more cells of a segment attempted a pull than the budget had left
  unsigned long long par_conflicts[4];
  // parallel sweep cycle counters: 0 prepass, 1 segments (workers), 2 rollbacks, 3 event logs;
  // summed over warps: 4 dependency waits, 5 start (blocked), 6 footprint loads, 7 pulls (gate and
  // search), 8 writes, 9 cells run, 10 between cells (row fetch), 11 worker total
  unsigned long long pprof[18];  // + 12 cone waits, 13 gate waits, 14 searches, 15 rounds, 16 reads, 17 source writes
  // SM cycles spent per tick phase, summed over ticks (clock64 on the SM running the region):
  // 0 drain, 1 sort, 2 sweep, 3 sweep waits for prefetch, 4 pressure pulls, 5 activation logs,
  // 6 writes, 7 seed commit, 8 levelling, 9 activation commit, 10 change commit, 11 mark clear
#ifdef VF_FINE_PROFILE
  unsigned long long prof[32];  // + per-call counters of the fine-profiling build
#else
  unsigned long long prof[16];
#endif
};
constexpr int NPROF = 16;

// Per drained cell of the parallel sweep (global memory, indexed by sorted position). The old
// footprint values serve readers that must see the state before this cell (multi-version reads)
// and the rollback of a segment; the event fields are committed in sorted order at the tick's end.
struct __align__(16) CellRec {
  float opart[7];          // footprint partials when the cell started (self, below, up, +x, -x, +z, -z)
  unsigned char omat[7];   // footprint materials when the cell started
  unsigned char wmask;     // footprint cells the cell's flow wrote
  unsigned char cmask;     // cells whose material changed: footprint bits 0..6, bit 7 the pull source
  unsigned char amask;     // activation slots in program order (0 source, 1 self after the pull,
                           // 2 below, 3..6 sides, 7 self)
  unsigned char flags;     // RF_*
  signed char pdelta;      // partial-entry count delta
  unsigned src;            // pull source cell id
  float src_opart;         // the source's partial before the pull wrote it
  unsigned char src_omat;  // and its material
  unsigned char pad0;
  unsigned short entries;  // pressure-search queue entries examined
  unsigned tk_main;        // execution ticket of the flow's writes (segment-wide order of writes)
  unsigned tk_src;         // execution ticket of the pull's source write
};
constexpr unsigned RF_ATTEMPT = 1u, RF_SUCCESS = 2u, RF_CHANGED = 4u, RF_SEED_SELF = 8u, RF_SEED_SRC = 16u, RF_SRCW = 32u;

// A pull's write of its source cell, kept for readers earlier in sorted order that read the cell
// after the write (open addressing by cell id; a slot belongs to the segment whose epoch it holds).
struct __align__(16) PullTarget {
  unsigned epoch;   // segment epoch owning the slot (claimed by CAS)
  unsigned ready;   // == epoch once the fields below are written
  unsigned id;      // source cell id
  unsigned writer;  // sorted position of the pulling cell
  float opart;      // the source's partial before the write
  unsigned omat;    // the source's material before the write
  unsigned pad[2];
};
constexpr unsigned PTREG_CAP = 16384;  // > 4 x the pulls one segment can make

struct Region {
  // ---- geometry (voxel dims, brick dims, ring width; padded scheduler domain)
  int nx, ny, nz, bx, by, bz, ring_w;
  int px0, pz0, PX, PY, PZ;  // domain: x in [px0, px0+PX), y in [0, PY), z in [pz0, pz0+PZ)
  unsigned mx, my, mz;       // ceil(2^32 / PX), ceil(2^32 / PY), ceil(2^32 / PZ): see udiv
  int TX, TZ;                // layer-mark tiles (64x64) per row / column
  unsigned int ncells;       // PX*PY*PZ
  // ---- world mirror
  unsigned int* grid;        // bx*by*bz
  unsigned char* amat;       // atlas materials [atlas_cap][512]
  float* avol;               // atlas partial volumes [atlas_cap][512]
  unsigned int atlas_cap;
  int* ring;                 // ring_w*ring_w triples (cx, cz, loaded)
  // ---- scheduler
  unsigned int* active;      // ncells bits
  unsigned int* seedbits;    // ncells bits
  unsigned int* marks;       // tiles * 128 words
  unsigned int* mark_list;   // touched tiles
  unsigned int* mark_tflag;  // per tile: listed in mark_list
  unsigned int* chgbits;     // ncells bits
  unsigned int* chg;         // changed ids (chg_cap)
  unsigned int chg_cap;
  unsigned int* queue;       // FIFO ring
  unsigned long long qmask;  // capacity - 1 (power of two)
  unsigned int* cells;       // drained cells (sort keys), MAX_CELLS_PER_TICK
  unsigned int* cells_tmp;
  unsigned int* seeds;       // MAX_LEVEL_SEEDS
  unsigned int* lvl_id;      // MAX_LEVEL_CELLS + 8
  float* lvl_vol;
  // ---- per-tick event logs (program order), committed in parallel at the tick's end
  unsigned int* ev_act;      // activation events: cell ids
  unsigned int* ev_seed;     // level-seed events
  unsigned int* ev_chg;      // voxel-material writes
  unsigned int ev_act_cap, ev_seed_cap, ev_chg_cap;
  unsigned int* stamp;       // ncells: first event index per cell during a commit (0xFFFFFFFF idle)
  unsigned int* last_woken;  // atlas_cap: last tick a cell of the slot's brick was drained (0 = never)
  // ---- parallel sweep (per tick; `stamp` doubles as the cell -> sorted position map)
  CellRec* rec;          // MAX_CELLS_PER_TICK
  unsigned* rowstart;    // MAX_CELLS_PER_TICK + 1: first sorted position of each row (y, z)
  unsigned* rowof;       // MAX_CELLS_PER_TICK: row of each cell, bit 31 may attempt a pull, bit 30 solid
  unsigned* rowprog;     // MAX_CELLS_PER_TICK: cells of the row finished
  unsigned* pcnt;        // MAX_CELLS_PER_TICK + 1: exclusive prefix count of possible attempts
  unsigned* zrow;        // PY * PZ: row of (y, z) this tick, NOSLOT otherwise
  unsigned* preader;     // ncells: latest pull read (segment epoch << 16 | position + 1)
  unsigned* ptbits;      // ncells bits: a pull wrote the cell this tick
  unsigned* ptlist;      // MAX_PULLS_PER_TICK + 64 cells whose ptbits are set
  PullTarget* ptreg;     // PTREG_CAP
  unsigned* pextra;      // MAX_CELLS_PER_TICK bits: later cells a pull took below 1 - 1e-4 (not counted in pcnt)
  unsigned* pxlist;      // MAX_CELLS_PER_TICK: the positions whose pextra bit is set
  unsigned* rb;          // ncells: earliest writer during a segment's rollback (0xFFFFFFFF idle)
  unsigned* deps;        // MAX_CELLS_PER_TICK * 16: earlier conflicting cells of each cell (10 used)
  unsigned* detbits;     // ring worlds: ncells bits, the cell's partial entry is kept for an evicted chunk
  struct PullCtx* pcg;   // one pressure-search context per sweep warp (used when the shared pool is empty)
  Ctl* ctl;
};

// ---------------------------------------------------------------- reference key (fluid.rs:46-62)
__host__ __device__ inline unsigned long long ref_key(int x, int y, int z) {
  auto f = [](int v) { return (unsigned long long)(((unsigned)v + (1u << 20)) & 0x1FFFFFu); };
  return f(x) | f(y) << 21 | f(z) << 42;
}

__host__ __device__ inline unsigned long long fmix64(unsigned long long k) {
  k ^= k >> 33;
  k *= 0xff51afd7ed558ccdULL;
  k ^= k >> 33;
  k *= 0xc4ceb9fe1a85ec53ULL;
  k ^= k >> 33;
  return k;
}

// ------------------------------------------------------------------------ domain ids
// n / d for n < 2^31 and d >= 2, with m = ceil(2^32 / d): umulhi(n, m) is n / d or one more (its
// error is below n / 2^32 < 1/2), and one compare corrects it. Cell ids and sort keys are below 2^31.
__host__ __device__ inline unsigned udiv(unsigned n, unsigned d, unsigned m) {
#ifdef __CUDA_ARCH__
  unsigned q = __umulhi(n, m);
  if (q * d > n) --q;
  return q;
#else
  (void)m;
  return n / d;
#endif
}
__host__ inline unsigned udiv_magic(unsigned d) { return (unsigned)(((1ull << 32) + d - 1ull) / d); }

__host__ __device__ inline bool in_dom(const Region& R, int x, int y, int z) {
  return (unsigned)(x - R.px0) < (unsigned)R.PX && (unsigned)y < (unsigned)R.PY && (unsigned)(z - R.pz0) < (unsigned)R.PZ;
}
__host__ __device__ inline unsigned dom_id(const Region& R, int x, int y, int z) {
  return ((unsigned)(z - R.pz0) * (unsigned)R.PY + (unsigned)y) * (unsigned)R.PX + (unsigned)(x - R.px0);
}
__host__ __device__ inline void dom_xyz(const Region& R, unsigned id, int& x, int& y, int& z) {
  unsigned t = udiv(id, (unsigned)R.PX, R.mx);
  x = (int)(id - t * (unsigned)R.PX) + R.px0;
  unsigned zz = udiv(t, (unsigned)R.PY, R.my);
  y = (int)(t - zz * (unsigned)R.PY);
  z = (int)zz + R.pz0;
}
// Sort key realising the reference's order (fluid.rs:575-580): (y, z, x), or (y, -z, -x) when
// the tick number is odd. Unique per cell, < ncells.
__host__ __device__ inline unsigned sort_key(const Region& R, unsigned id, bool flip) {
  int x, y, z;
  dom_xyz(R, id, x, y, z);
  unsigned xr = (unsigned)(x - R.px0), zr = (unsigned)(z - R.pz0);
  if (flip) {
    xr = (unsigned)R.PX - 1u - xr;
    zr = (unsigned)R.PZ - 1u - zr;
  }
  return ((unsigned)y * (unsigned)R.PZ + zr) * (unsigned)R.PX + xr;
}
__host__ __device__ inline unsigned key_to_id(const Region& R, unsigned key, bool flip) {
  unsigned t = udiv(key, (unsigned)R.PX, R.mx);
  unsigned xr = key - t * (unsigned)R.PX;
  unsigned y = udiv(t, (unsigned)R.PZ, R.mz);
  unsigned zr = t - y * (unsigned)R.PZ;
  if (flip) {
    xr = (unsigned)R.PX - 1u - xr;
    zr = (unsigned)R.PZ - 1u - zr;
  }
  return (zr * (unsigned)R.PY + y) * (unsigned)R.PX + xr;
}

// ------------------------------------------------------------------ world access
// SparseVolume::grid_index (sparse_volume.rs:142-148).
__host__ __device__ inline unsigned grid_index(const Region& R, int ix, int iy, int iz) {
  if (R.ring_w) {
    ix &= R.bx - 1;
    iz &= R.bz - 1;
  }
  return ((unsigned)iz * (unsigned)R.by + (unsigned)iy) * (unsigned)R.bx + (unsigned)ix;
}

// One cell as the rules see it.
struct __align__(16) CD {
  float part;       // partial volume (0 = none)
  unsigned slot;    // atlas slot of the brick, NOSLOT when the brick is a uniform grid value
  unsigned gi;      // grid index
  unsigned char mat;
  bool out;         // fluid.rs `outside` (:212-217)
};

__device__ inline bool cd_solid(const CD& c) { return c.out || (c.mat != 0 && c.mat != WATER); }  // fluid.rs:220-226
__device__ inline float cd_volume(const CD& c) {  // fluid.rs:251-260
  if (c.out) return 0.0f;
  if (c.part > 0.0f) return c.part;
  return c.mat == WATER ? 1.0f : 0.0f;
}

}  // namespace vfe
