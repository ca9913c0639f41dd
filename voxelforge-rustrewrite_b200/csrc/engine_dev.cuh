// Warp-cooperative device implementation of the reference's fluid tick (src/fluid.rs:292-657).
//
// One warp owns one region's sweep: it walks the drained cells in the reference's sorted order,
// so every cell sees exactly the state the sequential Rust loop would show it. Parallelism inside
// a cell comes from the 32 lanes: the 7-cell footprint, the writes into self, below and sides,
// six pressure-search queue entries (5 neighbours each) and the 12 cells of four level-fill
// membership tests go in one round each; activations, seeds and changed voxels are logged in
// program order with ballots and committed by the whole CTA at the tick's end; bricks are
// materialised cooperatively. Batching across regions runs one CTA per region (k_tick in
// kernels.cuh).
#pragma once
#include "engine.cuh"

namespace vfe {

constexpr unsigned FULLMASK = 0xFFFFFFFFu;

// Per-call cycle counters inside a cell (pressure search, writes, activation log) cost issue
// slots on the sweep's critical path; they are compiled in only with VF_FINE_PROFILE.
#ifdef VF_FINE_PROFILE
__device__ __forceinline__ long long fine_clock() { return clock64(); }
#else
__device__ __forceinline__ long long fine_clock() { return 0; }
#endif

__device__ __forceinline__ unsigned lane_id() { return threadIdx.x & 31u; }
__device__ __forceinline__ unsigned lanemask_lt() {
  unsigned m;
  asm("mov.u32 %0, %%lanemask_lt;" : "=r"(m));
  return m;
}

// f32 constant 1.0 - 1e-4 folded in f32 (fluid.rs:323, :337, :513, :594).
__device__ __forceinline__ float full_level() { return __fsub_rn(1.0f, 1e-4f); }

// ---------------------------------------------------------------------------- world reads
__device__ __forceinline__ bool chunk_loaded(const Region& R, const int* ring, int cx, int cz) {  // sparse_volume.rs:164-170
  int m = R.ring_w - 1;
  int i = ((cz & m) * R.ring_w + (cx & m)) * 3;
  return ring[i + 2] != 0 && ring[i] == cx && ring[i + 1] == cz;
}

__device__ __forceinline__ bool outside(const Region& R, const int* ring, int x, int y, int z) {  // fluid.rs:212-217
  if (y < 0 || y >= R.ny) return true;
  if (R.ring_w) return !chunk_loaded(R, ring, x >> 7, z >> 7);
  return x < 0 || z < 0 || x >= R.nx || z >= R.nz;
}

__device__ __forceinline__ unsigned local_index(int x, int y, int z) { return ((unsigned)(z & 7) << 6) | ((unsigned)(y & 7) << 3) | (unsigned)(x & 7); }

__device__ __forceinline__ CD load_cell(const Region& R, const int* ring, int x, int y, int z) {
  CD c;
  c.part = 0.0f;
  c.slot = NOSLOT;
  c.gi = 0;
  c.mat = 0;
  c.out = outside(R, ring, x, y, z);
  if (c.out) return c;
  c.gi = grid_index(R, x >> 3, y >> 3, z >> 3);
  unsigned g = R.grid[c.gi];
  if (g < 256u) {
    c.mat = (unsigned char)g;
    return c;
  }
  c.slot = g - 256u;
  size_t o = (size_t)c.slot * 512u + local_index(x, y, z);
  c.mat = R.amat[o];
  c.part = R.avol[o];
  return c;
}

__device__ __forceinline__ CD shfl_cd(const CD& c, int src) {
  CD r;
  r.part = __shfl_sync(FULLMASK, c.part, src);
  r.slot = __shfl_sync(FULLMASK, c.slot, src);
  r.gi = __shfl_sync(FULLMASK, c.gi, src);
  unsigned p = __shfl_sync(FULLMASK, (unsigned)c.mat | ((unsigned)c.out << 8), src);
  r.mat = (unsigned char)(p & 255u);
  r.out = (p >> 8) != 0;
  return r;
}

// Warp-uniform state of one region's sweep.
struct WS {
  unsigned long long qhead, qtail;
  unsigned long long activations, pull_attempts, pull_success, bfs_visits, level_cells_total;
  long long pdelta;        // partial_count delta (lane-local, reduced at the end)
  unsigned nseeds;
  unsigned pulls;          // this tick's pull attempts (fluid.rs:583)
  unsigned llc;            // last_level_cells
  unsigned ndrain;         // layers drained to a film (fluid.rs:456-481) since the handle's start
  unsigned epoch;          // press-BFS visited epoch
  bool level_round;
  bool changed;
  // Inside a tick the scheduler side effects are logged in program order and committed in
  // parallel at the tick's end (deferred); host edits apply them at once.
  bool deferred;
  unsigned nact, nseed, nchg;  // event-log cursors (deferred mode)
  // store-forwarding table of the prefetching sweep (null outside it) and the sequence number
  // (sorted index + 1) of the cell the sweep is processing
  struct FwdEntry* fwd;
  unsigned seq;
  // grid words the sweep has read or published (null outside the sweep): GCACHE entries of
  // grid index << 32 | grid word, one 64-bit store each so that an entry is never torn
  unsigned long long* gc;
  unsigned long long t_wait, t_pull, t_act, t_write, t_top, t_pc, t_tail;  // cycle counters (profiling)
#ifdef VF_FINE_PROFILE
  unsigned long long f_pre, f_plan, f_seed, n_pc, n_quiet, n_rounds, f_bload, f_bexp, f_match, f_vis;
#endif
};

// Store forwarding for the prefetching sweep: a direct-mapped table of the sweep's latest writes.
// An entry holds the cell id (tag), the writer's sequence number (sorted index + 1) and the
// written material, partial volume and atlas slot. A prefetched footprint cell fetched when
// `c0` cells were finished is current unless its entry's sequence is above c0; then the entry
// supplies the value if its tag is the cell, and otherwise (another cell wrote over the entry)
// the sweep re-reads the cell from memory, which holds every write of the sweep.
constexpr unsigned FWD_SIZE = 4096;
struct __align__(16) FwdEntry {
  unsigned tag;   // cell id
  unsigned meta;  // writer sequence (low 16 bits) | material << 16
  float part;
  unsigned slot;
};
static_assert(MAX_CELLS_PER_TICK < 65536u, "writer sequence numbers must fit 16 bits");

// Index of a cell in the table: low bits of x, z and y, so that the cells written by the last
// few dozen cells of the sweep (one neighbourhood of rows and layers) rarely share an entry.
__device__ __forceinline__ unsigned fwd_index(int x, int y, int z) {
  return ((unsigned)x & 127u) | (((unsigned)z & 7u) << 7) | (((unsigned)y & 3u) << 10);
}

__device__ __forceinline__ void fwd_insert(WS& W, unsigned id, int x, int y, int z, const CD& c) {
  FwdEntry e;
  e.tag = id;
  e.meta = W.seq | ((unsigned)c.mat << 16);
  e.part = c.part;
  e.slot = c.slot;
  W.fwd[fwd_index(x, y, z)] = e;
}

constexpr unsigned EMPTY_ID = 0xFFFFFFFFu;

// Neighbour loads done ahead of a pressure search by the prefetching warps while they wait.
// The search writes nothing, so a neighbour loaded at any time during it is current. The search
// publishes its queue; a helper claims up to six queued entries at a time. A claim is one CAS on
// `state`, which packs the search's epoch (bits 40-63), the next unclaimed entry (bits 20-39)
// and the helpers in flight (bits 0-19). The helper loads the entries' five neighbours into the
// ring slot (entry % HRING), then tags the slot (epoch << 32 | entry). The search uses a slot only
// when its tag names the current search and entry, and loads the cell itself otherwise, so it
// never waits for a helper. Before a new search begins, the old one closes its state and waits
// (bounded) until no helper is in flight, so no helper of an old search writes a slot again.
constexpr unsigned HRING = 64;
struct SearchHelp {
  CD nb[HRING][5];                // neighbours (up, +x, -x, +z, -z) of entry q at slot q % HRING
  unsigned long long tag[HRING];  // epoch << 32 | q once nb[q % HRING] is complete
  unsigned long long state;       // epoch << 40 | next entry << 20 | helpers in flight
  unsigned qlen;                  // entries queued so far (published after they are written)
  unsigned done;                  // entries the search has examined (their slots are free)
};
__host__ __device__ constexpr unsigned long long help_state(unsigned epoch, unsigned next, unsigned inflight) {
  return ((unsigned long long)(epoch & 0xFFFFFFu) << 40) | ((unsigned long long)next << 20) | inflight;
}

struct Smem {
  unsigned long long* vis;  // VIS_CAP entries (epoch << 32 | id)
  const int* ring;
  int4* pq;                 // PRESS_QCAP queued cells: x, y, z and the volume (bits) seen when queued
  unsigned* vb;             // VB_WORDS: visited bitmap of the search box (all zero between searches)
  unsigned* vtl;            // PRESS_QCAP: bitmap words the current search set (cleared at its end)
  SearchHelp* help;         // neighbour loads ahead of the search (null: none)
  unsigned* abort;          // the one-warp sweep's stop flag (null outside it)
  unsigned long long spin_cap;  // iterations before a wait on the helpers gives up (ST_TIMEOUT)
};

__device__ __forceinline__ void set_status(const Region& R, int st, unsigned info) {
  if (atomicCAS(&R.ctl->status, 0, st) == 0) R.ctl->err_info = info;
}

// ---------------------------------------------------------------------- materialisation
// Bricks that are uniform grid values get an atlas slot before their first write (the
// reference's SparseVolume::materialize, sparse_volume.rs:250-266; partial pages, fluid.rs:108-128).
// Lanes with `need` name a grid index; one leader per distinct index allocates, the warp fills.
constexpr unsigned GCACHE = 1024;  // grid-word cache entries of the sweep (direct-mapped by grid index)

__device__ void materialize_lanes(const Region& R, bool need, unsigned gi, unsigned& slot, unsigned long long* gc = nullptr) {
  const unsigned lane = lane_id();
  unsigned key = need ? gi : (0xFFFFFFFFu - lane);
  unsigned peers = __match_any_sync(FULLMASK, key);
  bool leader = need && !(peers & lanemask_lt());
  unsigned lead_mask = __ballot_sync(FULLMASK, leader);
  if (!lead_mask) return;
  unsigned s = NOSLOT;
  unsigned g = 0;
  if (leader) {
    g = R.grid[gi];
    if (g >= 256u) {
      s = g - 256u;
    } else {
      s = atomicAdd(&R.ctl->atlas_used, 1u);
      if (s >= R.atlas_cap) {
        set_status(R, ST_OOM, 1);
        s = NOSLOT;
      }
    }
  }
  // cooperative fill of each new slot
  for (unsigned m = lead_mask; m; m &= m - 1) {
    int l = __ffs(m) - 1;
    unsigned sl = __shfl_sync(FULLMASK, s, l);
    unsigned gv = __shfl_sync(FULLMASK, g, l);
    if (sl != NOSLOT && gv < 256u) {
      unsigned fill = gv & 255u;
      fill |= fill << 8;
      fill |= fill << 16;
      uint4 f4 = make_uint4(fill, fill, fill, fill);
      reinterpret_cast<uint4*>(R.amat + (size_t)sl * 512u)[lane] = f4;
      uint4 z4 = make_uint4(0, 0, 0, 0);
      uint4* vv = reinterpret_cast<uint4*>(R.avol + (size_t)sl * 512u);
#pragma unroll
      for (int k = 0; k < 4; ++k) vv[lane + 32 * k] = z4;
    }
  }
  __syncwarp();
  // publish the slot after its fill (release): prefetching warps read the grid word first and
  // then the atlas, with a fence in between
  __threadfence_block();
  if (leader && s != NOSLOT && g < 256u) {
    *(volatile unsigned*)(R.grid + gi) = 256u + s;
    unsigned long long* e = gc ? gc + (gi & (GCACHE - 1u)) : nullptr;
    if (e && (unsigned)(*e >> 32) == gi) *e = ((unsigned long long)gi << 32) | (256u + s);
  }
  int src = need ? (__ffs(peers) - 1) : (int)lane;
  unsigned s2 = __shfl_sync(FULLMASK, s, src);
  if (need) slot = s2;
  __syncwarp();
}

// --------------------------------------------------------------------------- writes
__device__ __forceinline__ void record_change(const Region& R, unsigned id) {
  unsigned old = atomicOr(&R.chgbits[id >> 5], 1u << (id & 31));
  if (!(old & (1u << (id & 31)))) {
    unsigned long long i = atomicAdd(&R.ctl->nchg, 1ull);
    if (i < R.chg_cap) R.chg[i] = id;
    else set_status(R, ST_OOM, 2);
  }
}

// Material write; the change is recorded at once (host edits) or logged by the caller (ticks,
// where `deferred` is set and the caller appends the cell to the change log).
__device__ __forceinline__ void write_mat(const Region& R, CD& c, unsigned l, unsigned id, unsigned char m, bool deferred = false) {
  if (c.slot == NOSLOT) return;  // materialisation failed (status already set)
  R.amat[(size_t)c.slot * 512u + l] = m;
  c.mat = m;
  if (!deferred) record_change(R, id);
}

__device__ __forceinline__ void erase_part(const Region& R, CD& c, unsigned l, long long& pdelta) {
  if (c.slot != NOSLOT && c.part > 0.0f) {
    R.avol[(size_t)c.slot * 512u + l] = 0.0f;
    c.part = 0.0f;
    pdelta -= 1;
  }
}

// Does set_volume(c, vol) write into the brick (so a uniform brick needs a slot first)?
__device__ __forceinline__ bool set_volume_needs_slot(const CD& c, float vol) {
  if (c.slot != NOSLOT) return false;
  bool is_water = c.mat == WATER;
  if (vol <= 1e-6f) return is_water;
  if (vol >= full_level()) return !is_water;
  return true;
}

// FluidSim::set_volume (fluid.rs:327-355) on one lane's cell; c.slot must be valid when
// set_volume_needs_slot said so. Returns "the voxel changed". Written as selects: the snapping
// (<= 1e-6 -> 0, >= 1-1e-4 -> full), the partial entry and the show/hide hysteresis each decide a
// value, and the stores are predicated.
__device__ __forceinline__ bool set_volume_lane(const Region& R, CD& c, int x, int y, int z, unsigned id, float vol, long long& pdelta,
                                                bool deferred = false) {
  const unsigned l = local_index(x, y, z);
  const bool is_water = c.mat == WATER;
  const bool has = c.slot != NOSLOT;  // false only when materialisation failed (status set)
  const bool low = vol <= 1e-6f;
  const bool high = !low && vol >= full_level();
  const bool mid = !low && !high;
  const bool had = has && c.part > 0.0f;
  const float npart = mid ? vol : 0.0f;
  const unsigned char nmat = low ? (unsigned char)0
                           : high ? (unsigned char)WATER
                           : (is_water && vol < HIDE_BELOW) ? (unsigned char)0
                           : (!is_water && vol >= SHOW_AT) ? (unsigned char)WATER
                           : c.mat;
  const bool wpart = has && (mid || had);
  const bool wmat = has && nmat != c.mat;
  const bool ch = mid ? wmat : nmat != c.mat;
  pdelta += (mid && has && !had) ? 1 : 0;
  pdelta -= (!mid && had) ? 1 : 0;
  if (wpart) R.avol[(size_t)c.slot * 512u + l] = npart;
  if (wmat) R.amat[(size_t)c.slot * 512u + l] = nmat;
  if (has) c.part = npart;
  if (wmat) c.mat = nmat;
  if (wmat && !deferred) record_change(R, id);
  return ch;
}

// Append per-lane events (lane order) to a log; returns the new cursor.
__device__ __forceinline__ unsigned log_append(const Region& R, unsigned* log, unsigned cap, unsigned cur, bool v, unsigned id, unsigned site) {
  unsigned b = __ballot_sync(FULLMASK, v);
  if (v) {
    unsigned pos = cur + (unsigned)__popc(b & lanemask_lt());
    if (pos < cap) log[pos] = id;
    else set_status(R, ST_OOM, site);
  }
  return cur + (unsigned)__popc(b);
}

// Warp: lanes with `w` write `vol` into their cell through set_volume. Returns whether any
// voxel changed.
__device__ bool warp_set_volume(const Region& R, WS& W, bool w, CD& c, int x, int y, int z, float vol) {
  const long long t0 = fine_clock();
  bool need = w && set_volume_needs_slot(c, vol);
  if (__any_sync(FULLMASK, need)) materialize_lanes(R, need, c.gi, c.slot, W.gc);
  bool ch = false;
  const unsigned id = (w && in_dom(R, x, y, z)) ? dom_id(R, x, y, z) : 0u;
  if (w) {
    ch = set_volume_lane(R, c, x, y, z, id, vol, W.pdelta, W.deferred);
    if (W.fwd) fwd_insert(W, id, x, y, z, c);
  }
  if (W.deferred) W.nchg = log_append(R, R.ev_chg, R.ev_chg_cap, W.nchg, ch, id, 9);
  __syncwarp();
  W.t_write += fine_clock() - t0;
  return __any_sync(FULLMASK, ch);
}

// ---------------------------------------------------------------------------- activation
// An ordered activation list: each entry is a single cell (FluidSim::activate, fluid.rs:292-300)
// or a wake_around centre (7 cells in the order self,+x,-x,+y,-y,+z,-z; fluid.rs:302-310).
// One cell's activations occupy fixed slots in program order (fluid.rs:584-650): 0 the pull
// source (single), 1 wake_around(self) after a pull, 2 wake_around(below) after a fall, 3..6
// wake_around(side) for +x,-x,+z,-z, 7 wake_around(self) at the end. Kept in registers.
struct ActList {
  int cx, cy, cz;  // the cell
  int sx, sy, sz;  // the pull source
  unsigned mask;
  __device__ __forceinline__ void reset(int x, int y, int z) {
    cx = x; cy = y; cz = z; mask = 0;
    sx = sy = sz = 0;
  }
  __device__ __forceinline__ void source(int a, int b, int c) {
    sx = a; sy = b; sz = c; mask |= 1u;
  }
  __device__ __forceinline__ void slot(int g) { mask |= 1u << g; }
  // slot g's centre and kind (1 or 7)
  __device__ __forceinline__ int get(int g, int& x, int& y, int& z) const {
    const bool src = g == 0;
    x = src ? sx : cx + (g == 3) - (g == 4);
    y = src ? sy : cy - (g == 2);
    z = src ? sz : cz + (g == 5) - (g == 6);
    return src ? 1 : 7;
  }
};

// Push cells (one per lane, lane order = program order) that are not active yet.
__device__ __forceinline__ void activate_round(const Region& R, WS& W, bool valid, int x, int y, int z) {
  const unsigned lane = lane_id();
  unsigned id = 0;
  if (valid) {
    if (y < 0) valid = false;  // fluid.rs:293-295
    else if (!in_dom(R, x, y, z)) {
      set_status(R, ST_RANGE, 3);
      valid = false;
    } else {
      id = dom_id(R, x, y, z);
    }
  }
  unsigned peers = __match_any_sync(FULLMASK, valid ? id : (0xFFFFFFFFu - lane));
  bool first = valid && !(peers & lanemask_lt());
  if (W.deferred) {  // inside a tick: log in program order, the tick's end commits
    W.nact = log_append(R, R.ev_act, R.ev_act_cap, W.nact, first, id, 10);
    __syncwarp();
    return;
  }
  bool isnew = false;
  if (first) isnew = !((R.active[id >> 5] >> (id & 31)) & 1u);
  unsigned nb = __ballot_sync(FULLMASK, isnew);
  if (isnew) {
    unsigned long long pos = W.qtail + (unsigned long long)__popc(nb & lanemask_lt());
    R.queue[pos & R.qmask] = id;
    atomicOr(&R.active[id >> 5], 1u << (id & 31));
  }
  W.qtail += (unsigned long long)__popc(nb);
  W.activations += (unsigned long long)__popc(nb);
  __syncwarp();
}

// Activation-log word: the cell id, bit 31 set for a wake_around centre (7 cells).
constexpr unsigned ACT_AROUND = 0x80000000u;

__device__ void flush_acts(const Region& R, WS& W, const ActList& A) {
  if (A.mask == 0) return;
  const long long t0 = fine_clock();
  const unsigned lane = lane_id();
  if (W.deferred) {  // one log word per call, in program order (expanded by the commit)
    bool v = lane < 8 && ((A.mask >> lane) & 1u);
    unsigned word = 0;
    if (v) {
      int x, y, z;
      int kind = A.get((int)lane, x, y, z);
      if (!in_dom(R, x, y, z) || y < 0) {
        set_status(R, ST_RANGE, 13);
        v = false;
      } else {
        word = dom_id(R, x, y, z) | (kind == 7 ? ACT_AROUND : 0u);
      }
    }
    W.nact = log_append(R, R.ev_act, R.ev_act_cap, W.nact, v, word, 10);
    W.t_act += fine_clock() - t0;
    return;  // the log is read only by the commit, after a CTA barrier
  }
  // immediate mode: expand the slots into single cells, 32 per round
  int total = 0;
  for (int g = 0; g < 8; ++g)
    if ((A.mask >> g) & 1u) total += g == 0 ? 1 : 7;
  for (int base = 0; base < total; base += 32) {
    int t = base + (int)lane;
    bool valid = t < total;
    int x = 0, y = 0, z = 0;
    if (valid) {
      int acc = 0;
      for (int g = 0; g < 8; ++g) {
        if (!((A.mask >> g) & 1u)) continue;
        int k = A.get(g, x, y, z);
        if (t < acc + k) {
          int o = t - acc;
          if (k == 7) {
            // self, +x, -x, +y, -y, +z, -z
            x += (o == 1) - (o == 2);
            y += (o == 3) - (o == 4);
            z += (o == 5) - (o == 6);
          }
          break;
        }
        acc += k;
      }
    }
    activate_round(R, W, valid, x, y, z);
  }
  if (W.qtail - W.qhead > R.qmask + 1ull) set_status(R, ST_OOM, 4);
  W.t_act += fine_clock() - t0;
}

// FluidSim::seed_level (fluid.rs:312-316); warp-uniform call.
__device__ __forceinline__ void seed_level(const Region& R, WS& W, int x, int y, int z) {
  if (W.level_round) return;
  unsigned id = dom_id(R, x, y, z);
  if (W.deferred) {  // the cap and the set membership are applied in order by the commit
    W.nseed = log_append(R, R.ev_seed, R.ev_seed_cap, W.nseed, lane_id() == 0, id, 11);
    return;  // the log is read only by the commit, after a CTA barrier
  }
  if (W.nseeds >= MAX_LEVEL_SEEDS) return;
  unsigned ins = 0;
  if (lane_id() == 0) {
    unsigned old = atomicOr(&R.seedbits[id >> 5], 1u << (id & 31));
    ins = !(old & (1u << (id & 31)));
    if (ins) R.seeds[W.nseeds] = id;
  }
  ins = __shfl_sync(FULLMASK, ins, 0);
  W.nseeds += ins;
  __syncwarp();
}

// ------------------------------------------------------------------- pressure BFS
__device__ __forceinline__ bool vis_insert(unsigned long long* vis, unsigned id, unsigned epoch) {
  unsigned h = (id * 2654435761u) & (VIS_CAP - 1u);
  unsigned long long want = ((unsigned long long)epoch << 32) | id;
  unsigned long long cur = vis[h];
  while (true) {
    if ((unsigned)(cur >> 32) != epoch) {
      unsigned long long old = atomicCAS(&vis[h], cur, want);
      if (old == cur) return true;
      cur = old;
      continue;
    }
    if ((unsigned)cur == id) return false;
    h = (h + 1u) & (VIS_CAP - 1u);
    cur = vis[h];
  }
}

// load_cell for the sweep's pressure search: the grid word comes from the sweep's cache when it
// holds it (only the sweep warp publishes grid words during a sweep, and it updates the cache).
__device__ __forceinline__ CD load_cell_gc(const Region& R, const WS& W, const int* ring, int x, int y, int z) {
  if (!W.gc) return load_cell(R, ring, x, y, z);
  CD c;
  c.part = 0.0f;
  c.slot = NOSLOT;
  c.gi = 0;
  c.mat = 0;
  c.out = outside(R, ring, x, y, z);
  if (c.out) return c;
  c.gi = grid_index(R, x >> 3, y >> 3, z >> 3);
  const unsigned h = c.gi & (GCACHE - 1u);
  const unsigned long long e = W.gc[h];
  unsigned g;
  if ((unsigned)(e >> 32) == c.gi) {
    g = (unsigned)e;
  } else {
    g = R.grid[c.gi];
    W.gc[h] = ((unsigned long long)c.gi << 32) | g;
  }
  if (g < 256u) {
    c.mat = (unsigned char)g;
    return c;
  }
  c.slot = g - 256u;
  size_t o = (size_t)c.slot * 512u + local_index(x, y, z);
  c.mat = R.amat[o];
  c.part = R.avol[o];
  return c;
}

// Visited test-and-insert of a pressure search started at (x0, y0, z0), warp-collective: lanes
// with `want` insert their cell (distinct cells; at most one lane per cell). Cells in the bitmap
// box take one atomicOr; the lane that finds its word empty adds the word to the touched list,
// which the search's end clears. Cells outside the box use the epoch-tagged hash. Returns "new".
__device__ __forceinline__ bool visit(const Smem& S, unsigned epoch, unsigned& ntouch, int x0, int y0, int z0, bool want, int a, int b, int c,
                                      unsigned id) {
  const unsigned lx = (unsigned)(a - x0 + VB_SIDE / 2), ly = (unsigned)(b - y0), lz = (unsigned)(c - z0 + VB_SIDE / 2);
  const bool inbox = want && lx < (unsigned)VB_SIDE && ly < (unsigned)VB_SIDE && lz < (unsigned)VB_SIDE;
  bool isnew = false, first = false;
  unsigned word = 0;
  if (inbox) {
    const unsigned bit = (ly * VB_SIDE + lz) * VB_SIDE + lx;
    const unsigned m = 1u << (bit & 31u);
    word = bit >> 5;
    const unsigned old = atomicOr(&S.vb[word], m);
    first = old == 0u;
    isnew = !(old & m);
  } else if (want) {
    isnew = vis_insert(S.vis, id, epoch);
  }
  const unsigned fm = __ballot_sync(FULLMASK, first);
  if (first) S.vtl[ntouch + (unsigned)__popc(fm & lanemask_lt())] = word;
  ntouch += (unsigned)__popc(fm);
  return isnew;
}

// D of pressure_pull (fluid.rs:512): up, +x, -x, +z, -z.
__device__ __forceinline__ void dir5(int d, int& dx, int& dy, int& dz) {
  dx = (d == 1) - (d == 2);
  dy = (d == 0);
  dz = (d == 3) - (d == 4);
}

// Queue entries a pressure search examines per round: lane 5j+d loads neighbour d of entry j.
constexpr unsigned PB = 6;

// FluidSim::pressure_pull (fluid.rs:511-561), warp-cooperative. fp[2..6] = up,+x,-x,+z,-z.
// Appends the source's activation to A and seeds it. Returns the volume taken.
//
// The search examines PB queue entries per round (their 5 neighbours in one load round) and
// keeps the reference's queue order exactly: the search writes nothing until it ends, so an
// entry's volume is the one seen when it was queued; the first entry (in queue order) that is a
// surface cell above the start wins, and entries after it in the round are dropped; otherwise
// the round's expansions are appended in entry-major, direction order, with the side-step
// budget counted in that order and duplicates inside the round left to their first occurrence.
__device__ float pressure_pull(const Region& R, WS& W, Smem& S, ActList& A, int x, int y, int z, float need, const CD* fp) {
  const unsigned lane = lane_id();
  const float FULL = full_level();
  // start cells: full up/side neighbours (fluid.rs:518-525); none -> the search examines nothing
  bool ok = false;
  unsigned nid = 0;
  float nvol = 0.0f;
  if (lane < 5) {
    int dx, dy, dz;
    dir5((int)lane, dx, dy, dz);
    int a = x + dx, b = y + dy, c = z + dz;
    // constant-index selects keep fp in registers (a lane-dependent index would spill it)
    const CD cd = lane == 0 ? fp[2] : lane == 1 ? fp[3] : lane == 2 ? fp[4] : lane == 3 ? fp[5] : fp[6];
    ok = a >= 0 && c >= 0 && !cd_solid(cd) && cd_volume(cd) >= FULL;
    if (ok) {
      nid = dom_id(R, a, b, c);
      nvol = cd_volume(cd);
    }
  }
  unsigned bm = __ballot_sync(FULLMASK, ok);
  unsigned qlen = (unsigned)__popc(bm);
  if (qlen == 0) return 0.0f;
  W.epoch += 1u;
  if (W.epoch == 0u) {  // wrapped: clear
    for (unsigned i = lane; i < VIS_CAP; i += 32) S.vis[i] = 0ull;
    __syncwarp();
    W.epoch = 1u;
  }
  unsigned ntouch = 0;
  visit(S, W.epoch, ntouch, x, y, z, lane == 0, x, y, z, dom_id(R, x, y, z));
  __syncwarp();
  {
    int dx = 0, dy = 0, dz = 0;
    if (lane < 5) dir5((int)lane, dx, dy, dz);
    if (ok) {
      const unsigned pos = (unsigned)__popc(bm & lanemask_lt());
      S.pq[pos] = make_int4(x + dx, y + dy, z + dz, __float_as_int(nvol));
    }
    visit(S, W.epoch, ntouch, x, y, z, ok, x + dx, y + dy, z + dz, nid);
  }
  __syncwarp();
  const unsigned hep = W.epoch & 0xFFFFFFu;
  if (S.help && hep <= 1u) {  // the 24-bit search epoch wrapped: no old tag may match again
    for (unsigned t = lane; t < HRING; t += 32u) S.help->tag[t] = ~0ull;
    __syncwarp();
  }
  SearchHelp* const H = hep ? S.help : nullptr;  // epoch 0 marks a closed search: run alone
  if (H) {  // open the search to helpers (the previous one closed with none in flight)
    if (lane == 0) {
      *(volatile unsigned*)&H->qlen = qlen;
      *(volatile unsigned*)&H->done = 0u;
    }
    __syncwarp();
    __threadfence_block();
    if (lane == 0) *(volatile unsigned long long*)&H->state = help_state(hep, 0u, 0u);
  }
  const unsigned j = lane / 5u, d = lane - 5u * (lane / 5u);
  unsigned side = 0, i = 0;
  float got = 0.0f;
  while (i < qlen && i < PRESSURE_SEARCH) {
#ifdef VF_FINE_PROFILE
    const long long b0 = clock64();
#endif
    const unsigned k = min(PB, min(qlen - i, PRESSURE_SEARCH - i));
    const bool act = j < k;
    int a = 0, b = 0, c = 0, na = 0, nb = 0, nc = 0;
    float here = 0.0f;
    CD cd = CD{0.0f, NOSLOT, 0u, 0, true};
    if (act) {
      const int4 e = S.pq[i + j];
      a = e.x;
      b = e.y;
      c = e.z;
      here = __int_as_float(e.w);
      int dx, dy, dz;
      dir5((int)d, dx, dy, dz);
      na = a + dx;
      nb = b + dy;
      nc = c + dz;
      bool have = false;
      if (H) {
        const unsigned q = i + j;
        const unsigned long long tg = *(volatile unsigned long long*)&H->tag[q % HRING];
        if (tg == (((unsigned long long)hep << 32) | q)) {
          __threadfence_block();
          cd = H->nb[q % HRING][d];
          have = true;
        }
      }
      if (!have) cd = load_cell_gc(R, W, S.ring, na, nb, nc);
    }
    // surface test of each entry on its up neighbour (fluid.rs:534-535)
    const bool win = act && d == 0u && (b + 1 >= R.ny || cd_solid(cd) || cd_volume(cd) <= 0.0f) && b > y && here > 0.0f;
    const unsigned wm = __ballot_sync(FULLMASK, win);
#ifdef VF_FINE_PROFILE
    const long long b1 = clock64();
    W.f_bload += b1 - b0;
#endif
    if (wm) {
      const int wl = __ffs(wm) - 1;
      const int wa = __shfl_sync(FULLMASK, a, wl), wb = __shfl_sync(FULLMASK, b, wl), wc = __shfl_sync(FULLMASK, c, wl);
      const float wh = __shfl_sync(FULLMASK, here, wl);
      const float take = fminf(need, wh);
      const float nv = __fsub_rn(wh, take);
      CD c0 = CD{0.0f, NOSLOT, 0u, 0, true};
      if (lane == 0) c0 = load_cell(R, S.ring, wa, wb, wc);
      W.changed |= warp_set_volume(R, W, lane == 0, c0, wa, wb, wc, nv);
      A.source(wa, wb, wc);
      seed_level(R, W, wa, wb, wc);
      got = take;
      i += (unsigned)wl / 5u + 1u;
      break;
    }
    // expansions (fluid.rs:541-556)
    bool cand = act && !(na < 0 || nc < 0 || nb >= R.ny || cd_solid(cd) || cd_volume(cd) <= 0.0f);
    const bool sc = cand && d >= 1u && nb == y;
    const unsigned sm = __ballot_sync(FULLMASK, sc);
    if (sc && side + (unsigned)__popc(sm & lanemask_lt()) + 1u > 24u) cand = false;
    side += (unsigned)__popc(sm);
    const unsigned id = cand ? dom_id(R, na, nb, nc) : (0xFFFFFFFFu - lane);
#ifdef VF_FINE_PROFILE
    const long long b2 = clock64();
#endif
    const unsigned peers = __match_any_sync(FULLMASK, id);
#ifdef VF_FINE_PROFILE
    const long long b3 = clock64();
    W.f_match += b3 - b2;
#endif
    const bool isnew = visit(S, W.epoch, ntouch, x, y, z, cand && !(peers & lanemask_lt()), na, nb, nc, id);
#ifdef VF_FINE_PROFILE
    __syncwarp();
    W.f_vis += clock64() - b3;
#endif
    const unsigned nm = __ballot_sync(FULLMASK, isnew);
    if (isnew) {
      const unsigned pos = qlen + (unsigned)__popc(nm & lanemask_lt());
      if (pos < PRESS_QCAP) S.pq[pos] = make_int4(na, nb, nc, __float_as_int(cd_volume(cd)));
    }
    qlen += (unsigned)__popc(nm);
    i += k;
    if (H) {  // the round's entries are examined and the new ones queued: publish both
      __syncwarp();
      __threadfence_block();
      if (lane == 0) {
        *(volatile unsigned*)&H->qlen = qlen;
        *(volatile unsigned*)&H->done = i;
      }
    }
#ifdef VF_FINE_PROFILE
    W.n_rounds += 1;
    W.f_bexp += clock64() - b1;
#endif
    __syncwarp();
  }
  if (H) {  // close the search to new claims, then let the helpers in flight finish
    unsigned ok2 = 1u;
    if (lane == 0) {
      unsigned long long st = *(volatile unsigned long long*)&H->state;
      while (true) {  // clear the entry field: no claim can match it any more
        const unsigned long long want = help_state(0u, 0u, (unsigned)(st & 0xFFFFFu));
        const unsigned long long old = atomicCAS(&H->state, st, want);
        if (old == st) break;
        st = old;
      }
      unsigned long long spins = 0;
      while ((*(volatile unsigned long long*)&H->state & 0xFFFFFull) != 0ull) {
        if (++spins > S.spin_cap) {
          ok2 = 0u;
          break;
        }
        __nanosleep(20);
      }
      if (!ok2) {  // the sweep stops: no new search may reuse the ring while a helper runs
        set_status(R, ST_TIMEOUT, 21);
        if (S.abort) *(volatile unsigned*)S.abort = 1u;
      }
      __threadfence_block();
    }
    __syncwarp();
  }
  // leave the bitmap all zero for the next search
  __syncwarp();
  for (unsigned t = lane; t < ntouch; t += 32u) S.vb[S.vtl[t]] = 0u;
  __syncwarp();
  W.bfs_visits += i;
  return got;
}

// A prefetching warp with nothing to prefetch helps the running pressure search (SearchHelp).
// Warp-collective; bounded work. Returns whether it loaded anything.
__device__ bool help_search(const Region& R, const int* ring, SearchHelp* H, const int4* pq) {
  const unsigned lane = lane_id();
  unsigned c = 0, take = 0, ep = 0;
  if (lane == 0) {
    unsigned long long st = *(volatile unsigned long long*)&H->state;
    for (int tries = 0; tries < 4; ++tries) {
      ep = (unsigned)(st >> 40);
      const unsigned next = (unsigned)((st >> 20) & 0xFFFFFu), inflight = (unsigned)(st & 0xFFFFFu);
      if (ep == 0u) break;
      __threadfence_block();
      const unsigned ql = *(volatile unsigned*)&H->qlen, dn = *(volatile unsigned*)&H->done;
      const unsigned lim = min(min(ql, dn + HRING), (unsigned)PRESSURE_SEARCH);
      if (next < dn) {  // entries the search already passed: skip ahead
        const unsigned long long old = atomicCAS(&H->state, st, help_state(ep, dn, inflight));
        st = old == st ? help_state(ep, dn, inflight) : old;
        continue;
      }
      if (next >= lim) break;
      const unsigned t = min(PB, lim - next);
      const unsigned long long want = help_state(ep, next + t, inflight + 1u);
      const unsigned long long old = atomicCAS(&H->state, st, want);
      if (old == st) {
        c = next;
        take = t;
        break;
      }
      st = old;
    }
  }
  take = __shfl_sync(FULLMASK, take, 0);
  if (!take) return false;
  c = __shfl_sync(FULLMASK, c, 0);
  ep = __shfl_sync(FULLMASK, ep, 0);
  __threadfence_block();
  const unsigned j = lane / 5u, d = lane - 5u * (lane / 5u);
  if (j < take) {
    const int4 e = pq[c + j];
    int dx, dy, dz;
    dir5((int)d, dx, dy, dz);
    H->nb[(c + j) % HRING][d] = load_cell(R, ring, e.x + dx, e.y + dy, e.z + dz);
  }
  __syncwarp();
  __threadfence_block();
  if (lane < take) *(volatile unsigned long long*)&H->tag[(c + lane) % HRING] = ((unsigned long long)ep << 32) | (c + lane);
  __syncwarp();
  __threadfence_block();
  if (lane == 0) atomicAdd(&H->state, ~0ull);  // one helper fewer in flight (the field is >= 1)
  return true;
}

// --------------------------------------------------------------------------- one cell
// The body of FluidSim::tick's loop (fluid.rs:584-650) for the cell (x, y, z).
// The flow part of a cell's update (fluid.rs:606-650 after the pressure pull) from its footprint
// and its volume `vol` (> 0) at that point: 1. fall into the free capacity below, 2. share with
// lower sides when supported, 3. evaporate crumbs. Written as selects: every side's flow depends
// only on `here` (the volume after the fall) and that side's volume, so the four decisions are
// independent; only the running volume subtracts them in side order.
struct CellPlan {
  float vol;          // the cell's volume afterwards (before the write-back test)
  float below_new;    // the cell below's new volume when w_below
  float side_new[4];  // +x, -x, +z, -z new volumes when their bit of wside is set
  bool w_below;
  unsigned wside;     // bit i: side i is written
  unsigned amask;     // activation slots 2 (below) and 3..6 (sides)
};

__device__ __forceinline__ CellPlan plan_flow(const CD* fp, float vol) {
  const float FULL = full_level();
  CellPlan P;
  const bool below_solid = cd_solid(fp[1]);
  const float bv = cd_volume(fp[1]);
  const float ff = fminf(vol, __fsub_rn(1.0f, bv));
  P.w_below = !below_solid && ff > 1e-6f;
  P.below_new = __fadd_rn(bv, ff);
  vol = P.w_below ? __fsub_rn(vol, ff) : vol;
  const float below_after = P.w_below ? (P.below_new >= FULL ? 1.0f : P.below_new) : bv;
  const bool spread = vol > MIN_SPREAD && (below_solid || below_after >= FULL);
  const float here = vol;
  P.wside = 0u;
  P.amask = P.w_below ? (1u << 2) : 0u;
#pragma unroll
  for (int i = 0; i < 4; ++i) {
    const bool open = !cd_solid(fp[3 + i]);
    const float nv = open ? cd_volume(fp[3 + i]) : 0.0f;
    const float f = __fmul_rn(__fsub_rn(here, nv), 0.2f);
    const bool ok = spread && open && !(nv >= here) && !(f < MIN_FLOW) && !(__fsub_rn(here, f) < MIN_SPREAD * 0.5f);
    P.side_new[i] = __fadd_rn(nv, f);
    P.wside |= ok ? (1u << i) : 0u;
    vol = ok ? __fsub_rn(vol, f) : vol;
    P.amask |= (ok && f > SLEEP) ? (1u << (3 + i)) : 0u;
  }
  P.vol = vol < EVAPORATE ? 0.0f : vol;
  return P;
}

// Does the pressure pull of a cell at (x, y, z) have a start cell (a full up/side neighbour with
// x, z >= 0; fluid.rs:518-525)? Without one the pull examines nothing and takes nothing.
__device__ __forceinline__ bool pull_has_start(const CD* fp, int x, int z) {
  const float FULL = full_level();
  bool any = false;
#pragma unroll
  for (int d = 0; d < 5; ++d) {
    const CD& c = fp[2 + d];  // up, +x, -x, +z, -z (the pull's direction order)
    const int a = x + (d == 1) - (d == 2), cc = z + (d == 3) - (d == 4);
    any |= a >= 0 && cc >= 0 && !cd_solid(c) && cd_volume(c) >= FULL;
  }
  return any;
}

// Quiet-cell classification for the sweep's prefetchers. Bit 0: processing the cell with this
// footprint writes nothing, activates nothing and seeds nothing (a solid cell without a partial
// entry; or a cell whose pull, if it attempts one, has no start cell and whose flow plan changes
// no volume by more than 1e-7); bit 1: the cell attempts a pull (counted against the tick's
// budget). Everything else goes through process_cell.
constexpr unsigned QUIET = 1u, QUIET_PULL = 2u;
__device__ __forceinline__ unsigned classify_quiet(const CD* fp, int x, int z) {
  if (cd_solid(fp[0])) return (fp[0].slot != NOSLOT && fp[0].part > 0.0f) ? 0u : QUIET;
  const float v0 = cd_volume(fp[0]);
  const bool attempt = v0 < full_level();
  if (attempt && pull_has_start(fp, x, z)) return 0u;
  const unsigned pbit = attempt ? QUIET_PULL : 0u;
  if (v0 <= 0.0f) return QUIET | pbit;
  const CellPlan P = plan_flow(fp, v0);
  const float dv = fabsf(__fsub_rn(P.vol, v0));
  const bool quiet = !P.w_below && P.wside == 0u && !(dv > 1e-7f);
  return quiet ? (QUIET | pbit) : 0u;
}

// fp: the footprint (0 self, 1 below, 2 up, 3 +x, 4 -x, 5 +z, 6 -z) as prefetched and
// store-forwarded by the sweep, the same on every lane; lanes 0..6 also hold their own cell
// (`mine`, at fx, fy, fz).
__device__ void process_cell(const Region& R, WS& W, Smem& S, int x, int y, int z, int fx, int fy, int fz, const CD (&fp)[7], CD mine) {
#ifdef VF_FINE_PROFILE
  const long long f0 = clock64();
  W.n_pc += 1;
#endif
  const unsigned lane = lane_id();
  const float FULL = full_level();
  if (cd_solid(fp[0])) {  // fluid.rs:586-589
    if (lane == 0) erase_part(R, mine, local_index(x, y, z), W.pdelta);
    __syncwarp();
    return;
  }
  ActList A;
  A.reset(x, y, z);
  float vol = cd_volume(fp[0]);
  const float v0 = vol;
#ifdef VF_FINE_PROFILE
  W.f_pre += clock64() - f0;
#endif
  // 0. pressure (fluid.rs:594-601)
  if (vol < FULL && W.pulls < MAX_PULLS_PER_TICK) {
    const long long tp = fine_clock();
    float got = pressure_pull(R, W, S, A, x, y, z, __fsub_rn(1.0f, vol), fp);
    W.t_pull += fine_clock() - tp;
    W.pulls += 1;
    W.pull_attempts += 1;
    if (got > 0.0f) {
      W.pull_success += 1;
      vol = __fadd_rn(vol, got);
      A.slot(1);
    }
  }
  if (vol <= 0.0f) {  // fluid.rs:602-604
    flush_acts(R, W, A);
    return;
  }
#ifdef VF_FINE_PROFILE
  const long long f1 = clock64();
#endif
  const CellPlan P = plan_flow(fp, vol);
  vol = P.vol;
#ifdef VF_FINE_PROFILE
  W.f_plan += clock64() - f1;
#endif
  A.mask |= P.amask;
  const bool w_below = P.w_below;
  const float below_new = P.below_new;
  bool w_side[4];
  float side_new[4];
#pragma unroll
  for (int i = 0; i < 4; ++i) {
    w_side[i] = (P.wside >> i) & 1u;
    side_new[i] = P.side_new[i];
  }
  // 3. evaporate, write back, sleep test (fluid.rs:641-650)
  const float dv = fabsf(__fsub_rn(vol, v0));
  const bool w_self = dv > 1e-7f;
  // parallel writes into distinct cells: lane 0 self, 1 below, 3..6 sides
  bool w = false;
  float wv = 0.0f;
  if (lane == 0) {
    w = w_self;
    wv = vol;
  } else if (lane == 1) {
    w = w_below;
    wv = below_new;
  } else if (lane == 3) {
    w = w_side[0];
    wv = side_new[0];
  } else if (lane == 4) {
    w = w_side[1];
    wv = side_new[1];
  } else if (lane == 5) {
    w = w_side[2];
    wv = side_new[2];
  } else if (lane == 6) {
    w = w_side[3];
    wv = side_new[3];
  }
  if (__any_sync(FULLMASK, w)) W.changed |= warp_set_volume(R, W, w, mine, fx, fy, fz, wv);
  if (dv > SLEEP) {
#ifdef VF_FINE_PROFILE
    const long long f2 = clock64();
#endif
    A.slot(7);
    seed_level(R, W, x, y, z);
#ifdef VF_FINE_PROFILE
    W.f_seed += clock64() - f2;
#endif
  }
  flush_acts(R, W, A);
}

// ------------------------------------------------------------------------ level fill
// LayerMarks::test_and_set (fluid.rs:194-200): one bit per cell in 64x64 tiles per layer; the
// tiles touched during a levelling round are listed so the round's end clears only those.
__device__ __forceinline__ bool mark_tas(const Region& R, int x, int y, int z) {
  if (!in_dom(R, x, y, z)) {  // cannot happen for neighbours of addressable cells; never write out of range
    set_status(R, ST_RANGE, 8);
    return true;
  }
  unsigned xr = (unsigned)(x - R.px0), zr = (unsigned)(z - R.pz0);
  unsigned tile = ((zr >> 6) * (unsigned)R.PY + (unsigned)y) * (unsigned)R.TX + (xr >> 6);
  unsigned bit = ((zr & 63u) << 6) | (xr & 63u);
  unsigned old = atomicOr(&R.marks[(size_t)tile * 128u + (bit >> 5)], 1u << (bit & 31));
  if (R.mark_tflag[tile] == 0u && atomicExch(&R.mark_tflag[tile], 1u) == 0u) {
    unsigned k = atomicAdd(&R.ctl->mark_ntiles, 1u);
    R.mark_list[k] = tile;
  }
  return (old >> (bit & 31)) & 1u;
}

// LayerMarks::test_and_set of a cell known to be unmarked, in two halves so that the caller's other
// loads overlap them: mark_begin sets the bit (no result wanted) and reads the tile's listed flag,
// mark_end lists the tile if nobody has.
__device__ __forceinline__ unsigned mark_begin(const Region& R, int x, int y, int z, unsigned& tile) {
  const unsigned xr = (unsigned)(x - R.px0), zr = (unsigned)(z - R.pz0);
  tile = ((zr >> 6) * (unsigned)R.PY + (unsigned)y) * (unsigned)R.TX + (xr >> 6);
  const unsigned bit = ((zr & 63u) << 6) | (xr & 63u);
  atomicOr(&R.marks[(size_t)tile * 128u + (bit >> 5)], 1u << (bit & 31));
  return __ldcg(R.mark_tflag + tile);  // set by atomics (in L2): read past L1
}
__device__ __forceinline__ void mark_end(const Region& R, unsigned tile, unsigned listed) {
  if (listed == 0u && atomicExch(&R.mark_tflag[tile], 1u) == 0u) {
    const unsigned k = atomicAdd(&R.ctl->mark_ntiles, 1u);
    R.mark_list[k] = tile;
  }
}

__device__ __forceinline__ void side4(int d, int& dx, int& dz) {  // SIDES (fluid.rs:228)
  dx = (d == 0) - (d == 1);
  dz = (d == 2) - (d == 3);
}

// FluidSim::level_layer's membership test (fluid.rs:413-415) of (x, y, z): !solid && vol > 0 &&
// supported && vol(above) <= 0. Returns the cell's volume through *v.
__device__ __forceinline__ bool level_member(const Region& R, const int* ring, int x, int y, int z, float* v) {
  const float FULL = full_level();
  const CD c = load_cell(R, ring, x, y, z);
  *v = cd_volume(c);
  if (cd_solid(c) || !(*v > 0.0f)) return false;
  const CD b = load_cell(R, ring, x, y - 1, z);
  if (!(cd_solid(b) || cd_volume(b) >= FULL)) return false;
  const CD a = load_cell(R, ring, x, y + 1, z);
  return cd_volume(a) <= 0.0f;
}

// The flood fill of FluidSim::level_layer (fluid.rs:425-446) continued by one warp from queue
// entry i of len (R.lvl_id / R.lvl_vol): entries are examined in order, each testing its four
// sides once (LayerMarks) and appending the members. Stops early, with i < len, when `hand` or
// more entries wait (the CTA takes the layer over from there). Returns the length.
__device__ unsigned level_bfs_warp(const Region& R, Smem& S, unsigned& i, unsigned len, unsigned hand) {
  const unsigned lane = lane_id();
  const float FULL = full_level();
  while (i < len) {
    if (len >= MAX_LEVEL_CELLS) {  // the rest is only summed (fluid.rs:436-438)
      i = len;
      break;
    }
    if (len - i >= hand) break;
    unsigned cid = R.lvl_id[i];
    ++i;
    int x, y, z;
    dom_xyz(R, cid, x, y, z);
    // lanes 0..11: side d = lane/3, j = lane%3 (0 the neighbour, 1 below it, 2 above it)
    int d = (int)lane / 3, j = (int)lane % 3;
    int dx = 0, dz = 0;
    if (lane < 12) side4(d, dx, dz);
    int nx = x + dx, nz = z + dz;
    bool skip = lane >= 12 || (R.ring_w == 0 && (nx < 0 || nz < 0));
    unsigned tas = 0;
    if (!skip && j == 0) tas = mark_tas(R, nx, y, nz);
    CD c = CD{0.0f, NOSLOT, 0u, 0, true};
    if (!skip) c = load_cell(R, S.ring, nx, y + (j == 1 ? -1 : (j == 2 ? 1 : 0)), nz);
    // gather the three cells of each side at its j==0 lane
    float v = cd_volume(c);
    bool sol = cd_solid(c);
    float v1 = __shfl_down_sync(FULLMASK, v, 1), v2 = __shfl_down_sync(FULLMASK, v, 2);
    bool s1 = __shfl_down_sync(FULLMASK, (unsigned)sol, 1) != 0u;
    bool push = !skip && j == 0 && !tas && !sol && v > 0.0f && (s1 || v1 >= FULL) && v2 <= 0.0f;
    unsigned pm = __ballot_sync(FULLMASK, push);
    if (push) {
      unsigned pos = len + (unsigned)__popc(pm & lanemask_lt());
      R.lvl_id[pos] = dom_id(R, nx, y, nz);
      R.lvl_vol[pos] = v;
    }
    len += (unsigned)__popc(pm);
    __syncwarp();
  }
  return len;
}

// The sum and range of the gathered volumes in queue order (fluid.rs:431-434), one lane adding in
// f64 in order; the result is broadcast to the warp.
__device__ void level_sum_warp(const Region& R, unsigned len, double& sum, float& lo, float& hi) {
  double s = 0.0;
  float l = 2.0f, h = -1.0f;
  if (lane_id() == 0) {
    for (unsigned i = 0; i < len; ++i) {
      const float v = R.lvl_vol[i];
      s = __dadd_rn(s, (double)v);
      l = fminf(l, v);
      h = fmaxf(h, v);
    }
  }
  sum = __shfl_sync(FULLMASK, s, 0);
  lo = __shfl_sync(FULLMASK, l, 0);
  hi = __shfl_sync(FULLMASK, h, 0);
}

// What FluidSim::level_layer does with a gathered layer (fluid.rs:446-485), one warp: count the
// cells, then level to the average or drain the film. Returns "a voxel changed".
__device__ bool level_finish(const Region& R, WS& W, Smem& S, unsigned len, double sum, float lo, float hi);

// FluidSim::level_layer (fluid.rs:412-486), one warp. Cells are gathered in the exact BFS order of
// the reference and summed in that order in f64. A layer whose flood fill grows to `hand` waiting
// entries is handed over: returns true with the queue state in qi / qlen, nothing levelled yet.
__device__ bool level_layer(const Region& R, WS& W, Smem& S, int sx, int sy, int sz, unsigned hand, unsigned& qi,
                            unsigned& qlen) {
  const unsigned lane = lane_id();
  unsigned was = 0;
  if (lane == 0) was = mark_tas(R, sx, sy, sz);
  was = __shfl_sync(FULLMASK, was, 0);
  if (was) return false;
  float v0 = 0.0f;
  const bool member = level_member(R, S.ring, sx, sy, sz, &v0);
  if (!member) return false;
  if (lane == 0) {
    R.lvl_id[0] = dom_id(R, sx, sy, sz);
    R.lvl_vol[0] = v0;
  }
  __syncwarp();
  unsigned i = 0;
  const unsigned len = level_bfs_warp(R, S, i, 1u, hand);
  if (i < len) {
    qi = i;
    qlen = len;
    return true;
  }
  double sum;
  float lo, hi;
  level_sum_warp(R, len, sum, lo, hi);
  W.changed |= level_finish(R, W, S, len, sum, lo, hi);
  return false;
}

__device__ bool level_finish(const Region& R, WS& W, Smem& S, unsigned len, double sum, float lo, float hi) {
  const unsigned lane = lane_id();
  W.llc += len;
  W.level_cells_total += len;
  bool changed = false;
  if (len >= 2 && __fsub_rn(hi, lo) >= SLEEP) {
    const float avg = __double2float_rn(__ddiv_rn(sum, (double)len));
    if (avg >= MIN_SPREAD) {  // fluid.rs:449-455
      for (unsigned b0 = 0; b0 < len; b0 += 32) {
        unsigned k = b0 + lane;
        bool wv = false;
        int x = 0, y = 0, z = 0;
        CD c = CD{0.0f, NOSLOT, 0u, 0, true};
        if (k < len) {
          dom_xyz(R, R.lvl_id[k], x, y, z);
          c = load_cell(R, S.ring, x, y, z);
          wv = fabsf(__fsub_rn(cd_volume(c), avg)) > 1e-6f;
        }
        changed |= warp_set_volume(R, W, wv, c, x, y, z, avg);
      }
    } else {  // drain into the water under the film (fluid.rs:456-481)
      W.ndrain += 1;
      double left = sum;
      bool stop = false;
      for (unsigned b0 = 0; b0 < len && !stop; b0 += 32) {
        unsigned k = b0 + lane;
        int x = 0, y = 0, z = 0;
        CD c = CD{0.0f, NOSLOT, 0u, 0, true};
        bool ok = false;
        if (k < len) {
          dom_xyz(R, R.lvl_id[k], x, y, z);
          if (y != 0) {
            c = load_cell(R, S.ring, x, y - 1, z);
            ok = !cd_solid(c);
          }
        }
        float bel = cd_volume(c);
        // sequential in cell order: take = min(left, 1 - below)
        bool wv = false;
        float nvv = 0.0f;
        unsigned n_here = min(32u, len - b0);
        for (unsigned t = 0; t < n_here; ++t) {
          bool okt = __shfl_sync(FULLMASK, ok, t);
          float bt = __shfl_sync(FULLMASK, bel, t);
          if (!okt) continue;
          float take = __double2float_rn(fmin(left, (double)__fsub_rn(1.0f, bt)));
          if (take <= 0.0f) continue;
          if (lane == t) {
            wv = true;
            nvv = __fadd_rn(bt, take);
          }
          left = __dsub_rn(left, (double)take);
          if (left <= 1e-6) {
            stop = true;
            break;
          }
        }
        changed |= warp_set_volume(R, W, wv, c, x, y - 1, z, nvv);
        // activations in cell order (fluid.rs:472)
        unsigned am = __ballot_sync(FULLMASK, wv);
        for (unsigned m = am; m; m &= m - 1) {
          int l = __ffs(m) - 1;
          int ax = __shfl_sync(FULLMASK, x, l), ay = __shfl_sync(FULLMASK, y, l), az = __shfl_sync(FULLMASK, z, l);
          activate_round(R, W, lane == 0, ax, ay - 1, az);
        }
      }
      const float rest = __double2float_rn(__ddiv_rn(left, (double)len));
      const float rv = rest < EVAPORATE ? 0.0f : rest;
      for (unsigned b0 = 0; b0 < len; b0 += 32) {
        unsigned k = b0 + lane;
        int x = 0, y = 0, z = 0;
        CD c = CD{0.0f, NOSLOT, 0u, 0, true};
        bool wv = k < len;
        if (wv) {
          dom_xyz(R, R.lvl_id[k], x, y, z);
          c = load_cell(R, S.ring, x, y, z);
        }
        changed |= warp_set_volume(R, W, wv, c, x, y, z, rv);
      }
    }
  }
  return changed;
}

}  // namespace vfe
