// Parallel exact sweep: the body of FluidSim::tick (src/fluid.rs:584-651) run by all warps of a
// region's CTA, with results bit-identical to the reference's sequential loop.
//
// Sequential semantics are kept by ordering every pair of conflicting operations as the sorted
// order does, or by reading the version the sorted order would show:
//   * Static conflicts. A cell reads and writes {self, below, +-x, +-z} and reads up (the pull's
//     start test). Two cells conflict iff they are on one layer within manhattan distance 2, on
//     adjacent layers within distance 1, or two layers apart in one column. Each cell waits for
//     the earlier drained cells at those positions (found through the position map `stamp`).
//   * Rows. The drained cells of one (y, z) are a row; a warp takes whole rows in sorted order
//     and walks them in order, so a row's own chain needs no waits.
//   * Pull budget (fluid.rs:594, 4096 attempts per tick). Cells that can attempt a pull are known
//     before the sweep up to one case that is checked at run time: a cell full at the tick's start
//     only drops below 1 - 1e-4 when a pull takes from it, and pulls take only from surface cells.
//     The sweep runs in segments of sorted order with a CTA barrier between them. A segment is
//     sized from the attempts expected per possible attempter (measured on earlier segments and
//     ticks); its attempts are counted when it ends, and one that made more than the budget had
//     left is undone and run again up to its room-th attempt. Once that end is known, one segment
//     runs the rest of the tick: attempts before it, none after it.
//   * Pressure searches read cells as of their own sorted position. Earlier writers of a cell on
//     the pulling layer are waited for; later writers that already wrote are read through their
//     records of the values they replaced (multi-version reads); a pull's source write is held
//     back until no later cell has read the source (readers that have not started are blocked,
//     one that has started is a conflict). Every pull read is stamped per cell so that an earlier
//     pull writing a cell a later pull already read is detected.
//   * Conflicts that ordering cannot prevent (a pull writing where a later cell has already
//     looked) stop the segment: its writes are undone from the records (the first write of each
//     location by execution ticket) and it runs again up to the conflicting pull, so the late
//     reader falls outside it; a position split too often is replayed in sorted order by one warp.
//     Every result is therefore the sequential one; conflicts cost time only.
// All waits are bounded (Tune::spin_cap) and end in ST_TIMEOUT.
#pragma once
#include "engine_dev.cuh"

namespace vfe {

constexpr unsigned GRID_LOCKED = 0xFFFFFFFFu;  // grid word while a warp materialises the brick
constexpr unsigned PQ_CAP = PRESSURE_SEARCH;   // queue entries a search can examine (fluid.rs:530)
constexpr unsigned PV_CAP = 1024;              // visited-set slots of one search (<= 549 cells)
constexpr unsigned CS_STARTED = 0xF0u, CS_WRITING = 0xF1u, CS_DONE = 0xF2u, CS_BLOCKMAX = 0xEFu;
constexpr int GATE_MAX = 31;
constexpr int MAX_WARPS = 16;  // warps of a CTA running the parallel sweep

enum ParMode { PM_PULL = 0, PM_NOPULL = 1, PM_SEQ = 2 };

// A pressure search's queue and visited set (one per warp).
struct PullCtx {
  unsigned qxz[PQ_CAP];       // queued cells: (x - px0) | (z - pz0) << 16
  unsigned short qy[PQ_CAP];  // their y
  float qv[PQ_CAP];           // their volume as of the pulling cell
  unsigned vis[PV_CAP];       // visited cell ids (EMPTY_ID = free)
};

// Pressure searches in flight at once are few (a search is ~4% of a worker warp's time on the dam
// break), so shared memory holds a small pool of search contexts; a warp that finds the pool empty
// runs its search on its own context in global memory (Region::pcg) and never waits. Keeping the
// pool small leaves the SM's L1 most of its 256 KB for the footprint loads.
constexpr int NPC_SMEM = 4;
struct ParSmem {
  unsigned state[(MAX_CELLS_PER_TICK + 3) / 4];  // one byte per drained cell: blockers / CS_*
  PullCtx pc[NPC_SMEM];
  unsigned pc_free;  // bit c: shared search context c is free
  unsigned next_task, task_end, abort, viol;
  unsigned viol_pos;  // smallest sorted position of a pull that met a conflict
  unsigned ticket;    // execution order of write groups in the segment (rollback restores the first)
  // the row each warp works on: y << 48 | (z - pz0) << 32 | sorted x of its next cell (x - px0, or
  // mirrored on odd ticks); WROW_IDLE when the warp holds no row
  unsigned long long wrow[MAX_WARPS];
};
constexpr unsigned long long WROW_IDLE = ~0ull;

__device__ __forceinline__ unsigned sorted_xr(const Region& R, int x, bool flip) {
  const unsigned xr = (unsigned)(x - R.px0);
  return flip ? (unsigned)R.PX - 1u - xr : xr;
}



// Per-warp cycle counters of the parallel sweep (lane 0), added to Ctl::pprof per segment.
struct ParProf {
  unsigned long long dep, start, load, pull, write, cells, cone, gate, npull, rounds, tread, tpw;
};

// Per-segment constants, the same on every warp.
struct ParTick {
  unsigned seg_start, seg_end, epoch;
  unsigned pull_end;  // cells from here on make no attempt: the tick's budget is spent before them
  int gate;  // same-layer radius waited for before a pressure search
  int cone;  // lower-layer radius a cell waits for before it starts
  bool flip;
  unsigned long long spin_cap;
};

__device__ __forceinline__ unsigned vld(const unsigned* p) { return *(volatile const unsigned*)p; }
// A global word that only this CTA's threads write (grid words, row progress, pull stamps and
// registries): a relaxed load at CTA scope. It is coherent with the CTA's stores and atomics, as
// volatile is, but may be served by the SM's L1 instead of a round trip to L2.
__device__ __forceinline__ unsigned gld(const unsigned* p) {
  unsigned v;
  asm volatile("ld.relaxed.cta.global.u32 %0, [%1];" : "=r"(v) : "l"(__cvta_generic_to_global(p)));
  return v;
}
__device__ __forceinline__ void vst(unsigned* p, unsigned v) { *(volatile unsigned*)p = v; }

// Back-off of a polling loop after n polls: a few polls at full rate, then sleeps growing from 32 ns
// to about 1 us, so waiting warps leave the issue slots to the warps that work.
__device__ __forceinline__ void backoff(unsigned long long n) {
  if (n > 4) __nanosleep(min(32u << (unsigned)min((n - 4) >> 2, 5ull), 1024u));
}

// ------------------------------------------------------------------------- cell states (shared)
__device__ __forceinline__ unsigned cs_get(const unsigned* st, unsigned i) { return (vld(&st[i >> 2]) >> ((i & 3u) * 8u)) & 0xFFu; }
// The owner's steps STARTED -> WRITING -> DONE: a byte add (the byte is >= 0xF0, no carry).
__device__ __forceinline__ void cs_advance(unsigned* st, unsigned i) { atomicAdd(&st[i >> 2], 1u << ((i & 3u) * 8u)); }
// IDLE -> STARTED; false while a pull blocks the cell.
__device__ __forceinline__ bool cs_try_start(unsigned* st, unsigned i) {
  const unsigned sh = (i & 3u) * 8u;
  unsigned w = vld(&st[i >> 2]);
  while (((w >> sh) & 0xFFu) == 0u) {
    const unsigned old = atomicCAS(&st[i >> 2], w, w | (CS_STARTED << sh));
    if (old == w) return true;
    w = old;
  }
  return false;
}
// One more blocker on a cell that has not started; false if it has.
__device__ __forceinline__ bool cs_block(unsigned* st, unsigned i) {
  const unsigned sh = (i & 3u) * 8u;
  unsigned w = vld(&st[i >> 2]);
  while (((w >> sh) & 0xFFu) < CS_BLOCKMAX) {
    const unsigned old = atomicCAS(&st[i >> 2], w, w + (1u << sh));
    if (old == w) return true;
    w = old;
  }
  return false;
}
__device__ __forceinline__ void cs_unblock(unsigned* st, unsigned i) { atomicSub(&st[i >> 2], 1u << ((i & 3u) * 8u)); }

__device__ __forceinline__ void par_timeout(const Region& R, ParSmem& ps, unsigned site) {
  set_status(R, ST_TIMEOUT, site);
  vst(&ps.abort, 1u);
}

// Bounded wait for cell j to finish; false on abort or timeout.
__device__ __forceinline__ bool wait_done(const Region& R, ParSmem& ps, const ParTick& T, unsigned j, unsigned site) {
  unsigned long long spins = 0;
  while (cs_get(ps.state, j) != CS_DONE) {
    if (vld(&ps.abort)) return false;
    if (++spins > T.spin_cap) {
      par_timeout(R, ps, site);
      return false;
    }
    backoff(spins);
  }
  return true;
}

// Before a cell of a pull segment starts: wait while a row on a lower layer within `d` rows of z,
// held by another warp, has not passed x + d (in sorted order). A pull's source lies above the
// pulling cell, so cells above a row still in work would otherwise read sources before the pulls
// that write them. Rows are taken in sorted order, so every lower-layer row is finished or held.
// Returns false on abort or timeout.
__device__ bool cone_wait(const Region& R, ParSmem& ps, const ParTick& T, unsigned me, int y, int z, unsigned xs, int d) {
  const unsigned lane = lane_id();
  const unsigned zr = (unsigned)(z - R.pz0);
  unsigned long long spins = 0;
  while (true) {
    bool held = false;
    if (lane < (unsigned)MAX_WARPS && lane != me) {
      const unsigned long long w = *(volatile unsigned long long*)&ps.wrow[lane];
      if (w != WROW_IDLE) {
        const int wy = (int)(w >> 48), wz = (int)((w >> 32) & 0xFFFFu);
        const unsigned wx = (unsigned)(w & 0xFFFFFFFFu);
        held = wy < y && abs(wz - (int)zr) <= d && wx <= xs + (unsigned)d;
      }
    }
    if (!__any_sync(FULLMASK, held)) return true;
    if (vld(&ps.abort)) return false;
    if (++spins > T.spin_cap) {
      if (lane == 0) par_timeout(R, ps, 44);
      __syncwarp();
      return false;
    }
    backoff(spins);
  }
}

// ---------------------------------------------------------------------------- world access
// load_cell for warps running side by side: the grid word is read volatile (a brick another warp
// is materialising reads GRID_LOCKED until its slot is filled and published) with a fence before
// the atlas reads.
__device__ __forceinline__ CD load_cell_par(const Region& R, const int* ring, int x, int y, int z, unsigned long long cap) {
  CD c;
  c.part = 0.0f;
  c.slot = NOSLOT;
  c.gi = 0;
  c.mat = 0;
  c.out = outside(R, ring, x, y, z);
  if (c.out) return c;
  c.gi = grid_index(R, x >> 3, y >> 3, z >> 3);
  unsigned g = gld(R.grid + c.gi);
  unsigned long long spins = 0;
  while (g == GRID_LOCKED) {
    if (++spins > cap) {
      set_status(R, ST_TIMEOUT, 30);
      c.out = true;
      return c;
    }
    backoff(spins);
    g = gld(R.grid + c.gi);
  }
  __threadfence_block();
  if (g < 256u) {
    c.mat = (unsigned char)g;
    return c;
  }
  c.slot = g - 256u;
  const size_t o = (size_t)c.slot * 512u + local_index(x, y, z);
  c.mat = R.amat[o];
  c.part = R.avol[o];
  return c;
}

// load_cell_par with a one-entry cache of the lane's last grid word: a detailed brick's word (slot)
// never changes during a sweep, so along a row the brick lookup is skipped for the cells that
// stay in the brick of the previous cell. Uniform words are always re-read (a warp may
// materialise the brick).
__device__ __forceinline__ CD load_cell_cached(const Region& R, const int* ring, int x, int y, int z, unsigned long long cap, unsigned& cgi,
                                               unsigned& cg) {
  CD c;
  c.part = 0.0f;
  c.slot = NOSLOT;
  c.gi = 0;
  c.mat = 0;
  c.out = outside(R, ring, x, y, z);
  if (c.out) return c;
  c.gi = grid_index(R, x >> 3, y >> 3, z >> 3);
  unsigned g;
  if (c.gi == cgi && cg >= 256u && cg != GRID_LOCKED) {
    g = cg;
  } else {
    g = gld(R.grid + c.gi);
    unsigned long long spins = 0;
    while (g == GRID_LOCKED) {
      if (++spins > cap) {
        set_status(R, ST_TIMEOUT, 30);
        c.out = true;
        return c;
      }
      backoff(spins);
      g = gld(R.grid + c.gi);
    }
    __threadfence_block();
    cgi = c.gi;
    cg = g;
  }
  if (g < 256u) {
    c.mat = (unsigned char)g;
    return c;
  }
  c.slot = g - 256u;
  const size_t o = (size_t)c.slot * 512u + local_index(x, y, z);
  c.mat = R.amat[o];
  c.part = R.avol[o];
  return c;
}

// Atlas slots for the bricks lanes with `need` are about to write (sparse_volume.rs:250-266).
// The first warp to take a brick's grid word (CAS to GRID_LOCKED) allocates and fills the slot and
// publishes it; the others read the published slot.
__device__ void materialize_par(const Region& R, bool need, unsigned gi, unsigned& slot, unsigned long long cap) {
  const unsigned lane = lane_id();
  const unsigned key = need ? gi : (0xFFFFFFFFu - lane);
  const unsigned peers = __match_any_sync(FULLMASK, key);
  const bool leader = need && !(peers & lanemask_lt());
  unsigned s = NOSLOT, g = 0;
  bool fill = false;
  if (leader) {
    unsigned long long spins = 0;
    g = gld(R.grid + gi);
    while (true) {
      if (g == GRID_LOCKED) {
        if (++spins > cap) {
          set_status(R, ST_TIMEOUT, 31);
          break;
        }
        backoff(spins);
        g = gld(R.grid + gi);
        continue;
      }
      if (g >= 256u) {
        s = g - 256u;
        break;
      }
      const unsigned old = atomicCAS(R.grid + gi, g, GRID_LOCKED);
      if (old != g) {
        g = old;
        continue;
      }
      s = atomicAdd(&R.ctl->atlas_used, 1u);
      if (s >= R.atlas_cap) {
        set_status(R, ST_OOM, 1);
        atomicExch(R.grid + gi, g);
        s = NOSLOT;
      } else {
        fill = true;
      }
      break;
    }
  }
  for (unsigned m = __ballot_sync(FULLMASK, fill); m; m &= m - 1) {
    const int l = __ffs(m) - 1;
    const unsigned sl = __shfl_sync(FULLMASK, s, l);
    unsigned fv = __shfl_sync(FULLMASK, g, l) & 255u;
    fv |= fv << 8;
    fv |= fv << 16;
    reinterpret_cast<uint4*>(R.amat + (size_t)sl * 512u)[lane] = make_uint4(fv, fv, fv, fv);
    uint4* vv = reinterpret_cast<uint4*>(R.avol + (size_t)sl * 512u);
#pragma unroll
    for (int k = 0; k < 4; ++k) vv[lane + 32 * k] = make_uint4(0, 0, 0, 0);
  }
  __syncwarp();
  __threadfence_block();
  if (fill) atomicExch(R.grid + gi, 256u + s);
  const int src = need ? (__ffs(peers) - 1) : (int)lane;
  const unsigned s2 = __shfl_sync(FULLMASK, s, src);
  if (need) slot = s2;
  __syncwarp();
}

// FluidSim::set_volume (fluid.rs:327-355) split into the decision and the stores, so a cell can
// publish what it will write before writing it.
struct SVPlan {
  float npart;
  unsigned char nmat;
  bool wpart, wmat, ch;
  int dp;
};
__device__ __forceinline__ SVPlan sv_plan(const CD& c, float vol) {
  SVPlan p;
  const bool is_water = c.mat == WATER;
  const bool has = c.slot != NOSLOT;
  const bool low = vol <= 1e-6f;
  const bool high = !low && vol >= full_level();
  const bool mid = !low && !high;
  const bool had = has && c.part > 0.0f;
  p.npart = mid ? vol : 0.0f;
  p.nmat = low ? (unsigned char)0
         : high ? (unsigned char)WATER
         : (is_water && vol < HIDE_BELOW) ? (unsigned char)0
         : (!is_water && vol >= SHOW_AT) ? (unsigned char)WATER
         : c.mat;
  p.wpart = has && (mid || had);
  p.wmat = has && p.nmat != c.mat;
  p.ch = mid ? p.wmat : p.nmat != c.mat;
  p.dp = ((mid && has && !had) ? 1 : 0) - ((!mid && had) ? 1 : 0);
  return p;
}
__device__ __forceinline__ void sv_apply(const Region& R, const CD& c, int x, int y, int z, const SVPlan& p) {
  const size_t o = (size_t)c.slot * 512u + local_index(x, y, z);
  if (p.wpart) R.avol[o] = p.npart;
  if (p.wmat) R.amat[o] = p.nmat;
}

// Footprint slot offsets: 0 self, 1 below, 2 up, 3 +x, 4 -x, 5 +z, 6 -z.
__device__ __forceinline__ void fp_off(int l, int& ox, int& oy, int& oz) {
  ox = (l == 3) - (l == 4);
  oy = (l == 2) - (l == 1);
  oz = (l == 5) - (l == 6);
}

__device__ __forceinline__ unsigned rank_at(const Region& R, int x, int y, int z) {
  if (!in_dom(R, x, y, z)) return NOSLOT;
  return R.stamp[dom_id(R, x, y, z)];
}

// ----------------------------------------------------------------- pull-written versions
__device__ void ptreg_insert(const Region& R, unsigned epoch, unsigned id, unsigned writer, float opart, unsigned omat) {
  unsigned h = (id * 2654435761u) & (PTREG_CAP - 1u);
  for (unsigned n = 0; n < 2u * PTREG_CAP; ++n) {
    PullTarget* e = R.ptreg + h;
    const unsigned ep = gld(&e->epoch);
    if (ep != epoch) {
      if (atomicCAS(&e->epoch, ep, epoch) == ep) {
        e->id = id;
        e->writer = writer;
        e->opart = opart;
        e->omat = omat;
        __threadfence_block();
        vst(&e->ready, epoch);
        return;
      }
      continue;
    }
    h = (h + 1u) & (PTREG_CAP - 1u);
  }
  set_status(R, ST_OOM, 32);
}

// The earliest pull write of cell `id` by a cell after position k in this segment: its writer
// (NOSLOT if none) and the values it replaced.
__device__ unsigned ptreg_after(const Region& R, ParSmem& ps, const ParTick& T, unsigned id, unsigned k, float& opart, unsigned& omat) {
  unsigned best = NOSLOT;
  unsigned h = (id * 2654435761u) & (PTREG_CAP - 1u);
  for (unsigned n = 0; n < PTREG_CAP; ++n) {
    const PullTarget* e = R.ptreg + h;
    if (gld(&e->epoch) != T.epoch) break;
    unsigned long long spins = 0;
    while (gld(&e->ready) != T.epoch) {
      if (++spins > T.spin_cap) {
        par_timeout(R, ps, 33);
        return best;
      }
    }
    __threadfence_block();
    if (e->id == id && e->writer > k && e->writer < best) {
      best = e->writer;
      opart = e->opart;
      omat = e->omat;
    }
    h = (h + 1u) & (PTREG_CAP - 1u);
  }
  return best;
}

// A cell (a, b, c) as the pressure search of the cell at sorted position k must see it
// (fluid.rs:531-547 read volume / solid): earlier writers on the pulling layer are waited for
// (those within the gate are done already), later writers that wrote it supply the value they
// replaced. The read is stamped for the detection of earlier pulls writing it later. Returns false
// on abort.
__device__ bool read_mvcc(const Region& R, ParSmem& ps, const int* ring, const ParTick& T, unsigned k, int kx, int ky, int kz, int a, int b,
                          int c, CD& out) {
  out = CD{0.0f, NOSLOT, 0u, 0, true};
  if (outside(R, ring, a, b, c)) return true;
  const unsigned id = dom_id(R, a, b, c);
  // Issued together: the cell's writers among the drained cells (footprint slots 0, 1, 3..6 cover
  // it; up is read only), its grid word, and the stamp of this read (made before the value is
  // read: an earlier pull writes, then checks the stamp, so either it sees this stamp - a
  // conflict - or this read sees its write).
  unsigned jr[6];
#pragma unroll
  for (int q = 0; q < 6; ++q) {
    const int fl = q < 2 ? q : q + 1;
    int ox, oy, oz;
    fp_off(fl, ox, oy, oz);
    jr[q] = rank_at(R, a - ox, b - oy, c - oz);
  }
  out.out = false;
  out.gi = grid_index(R, a >> 3, b >> 3, c >> 3);
  unsigned g = gld(R.grid + out.gi);
  atomicMax(R.preader + id, ((T.epoch & 0xFFFFu) << 16) | (k + 1u));
  if (b == ky) {
    // earlier writers on the pulling layer must be done (those within the gate are already)
    const bool gated = T.gate > 0 && abs(a - kx) < T.gate && abs(c - kz) < T.gate;
    if (!gated) {
#pragma unroll
      for (int q = 0; q < 6; ++q)
        if (jr[q] != NOSLOT && jr[q] < k && jr[q] >= T.seg_start && !wait_done(R, ps, T, jr[q], 34)) return false;
      g = gld(R.grid + out.gi);  // a writer waited for may have materialised the brick
    }
  }
  unsigned long long spins = 0;
  while (g == GRID_LOCKED) {
    if (++spins > T.spin_cap) {
      set_status(R, ST_TIMEOUT, 30);
      return false;
    }
    backoff(spins);
    g = gld(R.grid + out.gi);
  }
  __threadfence_block();  // one CTA runs the region: CTA scope orders every party
  if (g < 256u) {
    out.mat = (unsigned char)g;
  } else {
    out.slot = g - 256u;
    const size_t o = (size_t)out.slot * 512u + local_index(a, b, c);
    out.mat = R.amat[o];
    out.part = R.avol[o];
  }
  __threadfence_block();
  const unsigned ptw = gld(&R.ptbits[id >> 5]);
  unsigned best = NOSLOT;
  float bp = 0.0f;
  unsigned bm = 0;
#pragma unroll
  for (int q = 0; q < 6; ++q) {
    const unsigned j = jr[q];
    if (j == NOSLOT || j <= k || j >= T.seg_end || j >= best) continue;
    if (cs_get(ps.state, j) < CS_WRITING) continue;
    __threadfence_block();
    const int fl = q < 2 ? q : q + 1;
    const CellRec& rc = R.rec[j];
    if ((rc.wmask >> fl) & 1u) {
      best = j;
      bp = rc.opart[fl];
      bm = rc.omat[fl];
    }
  }
  if ((ptw >> (id & 31u)) & 1u) {
    float op = 0.0f;
    unsigned om = 0;
    const unsigned w = ptreg_after(R, ps, T, id, k, op, om);
    if (w < best) {
      best = w;
      bp = op;
      bm = om;
    }
  }
  if (best != NOSLOT) {
    out.part = bp;
    out.mat = (unsigned char)bm;
  }
  return true;
}

__device__ __forceinline__ bool vis_insert_par(unsigned* vis, unsigned id) {
  unsigned h = (id * 2654435761u) >> 22;  // 10 bits
  for (unsigned n = 0; n < PV_CAP; ++n) {
    const unsigned old = atomicCAS(&vis[h], EMPTY_ID, id);
    if (old == EMPTY_ID) return true;
    if (old == id) return false;
    h = (h + 1u) & (PV_CAP - 1u);
  }
  return false;
}

// Outputs of a cell that its record carries.
struct CellOut {
  unsigned flags, amask, cmask, src, entries;
  int pdelta;
};

// The pull's write of its source (fluid.rs:536-540). Warp-collective. In PM_PULL mode it first
// waits for an earlier cell below the source (its start test reads the source), blocks the later
// cells that read the source and have not started, and checks that no later cell has read it; a
// later reader that started already, or a possible-attempt set that the write would break, is a
// conflict (returns false and the segment is replayed).
__device__ bool pull_write(const Region& R, ParSmem& ps, const int* ring, const ParTick& T, int mode, unsigned k, int wa, int wb, int wc,
                           float nvv, CellOut& co) {
  const unsigned lane = lane_id();
  const unsigned sid = dom_id(R, wa, wb, wc);
  unsigned jr = NOSLOT;
  bool blk = false;
  if (mode == PM_PULL) {
    // readers of the source among the drained cells: itself, below, above, +-x, +-z
    if (lane < 7) {
      const int ox = (lane == 3) - (lane == 4), oy = (lane == 2) - (lane == 1), oz = (lane == 5) - (lane == 6);
      jr = rank_at(R, wa + ox, wb + oy, wc + oz);
    }
    bool bad = false;
    if (lane == 1 && jr != NOSLOT && jr < k && jr >= T.seg_start && !wait_done(R, ps, T, jr, 35)) bad = true;
    if (__any_sync(FULLMASK, bad)) return false;
    unsigned kind = 0;
    if (lane < 7 && jr != NOSLOT && jr > k && jr < T.seg_end) {
      if (cs_block(ps.state, jr)) blk = true;
      else kind = 1;
    }
    if (lane == 0 && jr != NOSLOT && jr >= T.seg_end && nvv < full_level() && !(R.rowof[jr] >> 31)) {
      // a drained source taken below 1 - 1e-4 attempts a pull when its turn comes; one in a later
      // segment that was not counted as a possible attempter is counted when that segment is
      // sized (in this segment the attempt count is checked when the segment ends)
      if (!(atomicOr(R.pextra + (jr >> 5), 1u << (jr & 31u)) & (1u << (jr & 31u)))) {
        const unsigned q = atomicAdd(&R.ctl->pxn, 1u);
        if (q < MAX_CELLS_PER_TICK) R.pxlist[q] = jr;
      }
    }
    if (kind) {
      atomicAdd(&R.ctl->par_conflicts[kind - 1u], 1ull);
      atomicMin(&ps.viol_pos, k);
    }
    if (__any_sync(FULLMASK, kind != 0u)) {
      if (blk) cs_unblock(ps.state, jr);
      __syncwarp();
      return false;
    }
  }
  // Pull writes of one source are made one at a time (a lock on the source's rollback word, idle
  // during the sweep), so their tickets and recorded old values follow the order of the writes.
  bool locked = true;
  if (mode == PM_PULL && lane == 0) {
    unsigned long long spins = 0;
    while (atomicCAS(R.rb + sid, 0xFFFFFFFFu, k) != 0xFFFFFFFFu) {
      if (++spins > T.spin_cap) {
        par_timeout(R, ps, 43);
        locked = false;
        break;
      }
      backoff(spins);
    }
    __threadfence_block();  // one CTA runs the region: CTA scope orders every party
  }
  if (!__shfl_sync(FULLMASK, locked ? 1u : 0u, 0)) {
    if (blk) cs_unblock(ps.state, jr);
    __syncwarp();
    return false;
  }
  CD c = CD{0.0f, NOSLOT, 0u, 0, true};
  if (lane == 0) c = load_cell_par(R, ring, wa, wb, wc, T.spin_cap);
  const bool need = lane == 0 && c.slot == NOSLOT && set_volume_needs_slot(c, nvv);
  if (__any_sync(FULLMASK, need)) materialize_par(R, need, c.gi, c.slot, T.spin_cap);
  if (lane == 0) {
    CellRec* rc = R.rec + k;
    rc->src = sid;
    rc->src_opart = c.part;
    rc->src_omat = c.mat;
    rc->tk_src = atomicAdd(&ps.ticket, 1u);
    rc->flags = RF_SRCW;
    if (mode == PM_PULL) {
      ptreg_insert(R, T.epoch, sid, k, c.part, c.mat);
      const unsigned old = atomicOr(R.ptbits + (sid >> 5), 1u << (sid & 31u));
      if (!(old & (1u << (sid & 31u)))) {
        const unsigned p = atomicAdd(&R.ctl->ptn, 1u);
        if (p < MAX_PULLS_PER_TICK + 64u) R.ptlist[p] = sid;
        else set_status(R, ST_OOM, 36);
      }
    }
    __threadfence_block();
    const SVPlan p = sv_plan(c, nvv);
    if (c.slot != NOSLOT) sv_apply(R, c, wa, wb, wc, p);
    co.cmask |= p.ch ? 0x80u : 0u;
    co.flags |= RF_SRCW | (p.ch ? RF_CHANGED : 0u);
    co.pdelta += p.dp;
    co.src = sid;
  }
  __syncwarp();
  __threadfence_block();  // one CTA runs the region: CTA scope orders every party
  // a later pull that stamped its read of the source before this write saw the old value: a
  // conflict (the write is undone with the segment: the record holds the old value)
  bool late = false;
  if (mode == PM_PULL && lane == 0) {
    const unsigned v = gld(R.preader + sid);
    if ((v >> 16) == (T.epoch & 0xFFFFu) && (v & 0xFFFFu) > k + 1u) {
      late = true;
      atomicAdd(&R.ctl->par_conflicts[1], 1ull);
      atomicMin(&ps.viol_pos, k);
    }
    __threadfence_block();  // one CTA runs the region: CTA scope orders every party
    atomicExch(R.rb + sid, 0xFFFFFFFFu);
  }
  if (blk) cs_unblock(ps.state, jr);
  if (__any_sync(FULLMASK, late)) return false;
  co.cmask = __shfl_sync(FULLMASK, co.cmask, 0);
  co.flags = __shfl_sync(FULLMASK, co.flags, 0);
  co.pdelta = __shfl_sync(FULLMASK, co.pdelta, 0);
  co.src = __shfl_sync(FULLMASK, co.src, 0);
  __syncwarp();
  return true;
}

// FluidSim::pressure_pull (fluid.rs:511-561) for the cell at sorted position k, warp-cooperative:
// six queue entries per round, one neighbour per lane, the reference's queue order kept exactly
// (first surface entry in queue order wins; expansions entry-major in direction order; the 24 side
// checks at the start level counted in that order; duplicates of a round to their first
// occurrence). Entries past the 512th are never examined, so appends stop once 512 are queued.
// Returns the volume taken; *ok = false on a conflict or abort.
__device__ float pull_par(const Region& R, ParSmem& ps, PullCtx& pc, const int* ring, const ParTick& T, int mode, unsigned k, int x, int y,
                          int z, float need, const CD* fp, CellOut& co, bool& ok, ParProf& pf) {
  const unsigned lane = lane_id();
  const float FULL = full_level();
  ok = true;
  bool st = false;
  float svol = 0.0f;
  int sa = 0, sb = 0, sc = 0;
  if (lane < 5) {
    int dx, dy, dz;
    dir5((int)lane, dx, dy, dz);
    sa = x + dx;
    sb = y + dy;
    sc = z + dz;
    const CD cd = lane == 0 ? fp[2] : lane == 1 ? fp[3] : lane == 2 ? fp[4] : lane == 3 ? fp[5] : fp[6];
    st = sa >= 0 && sc >= 0 && !cd_solid(cd) && cd_volume(cd) >= FULL;
    svol = cd_volume(cd);
  }
  const unsigned bm = __ballot_sync(FULLMASK, st);
  unsigned qlen = (unsigned)__popc(bm);
  if (qlen == 0) return 0.0f;
  if (lane == 0) vis_insert_par(pc.vis, dom_id(R, x, y, z));
  if (st) {
    const unsigned pos = (unsigned)__popc(bm & lanemask_lt());
    pc.qxz[pos] = (unsigned)(sa - R.px0) | ((unsigned)(sc - R.pz0) << 16);
    pc.qy[pos] = (unsigned short)sb;
    pc.qv[pos] = svol;
    vis_insert_par(pc.vis, dom_id(R, sa, sb, sc));
  }
  __syncwarp();
  const unsigned j = lane / 5u, d = lane - 5u * (lane / 5u);
  unsigned side = 0, i = 0;
  float got = 0.0f;
  while (i < qlen && i < PRESSURE_SEARCH) {
    const unsigned kk = min(PB, min(qlen - i, PRESSURE_SEARCH - i));
    const bool act = j < kk;
    int a = 0, b = 0, c = 0, na = 0, nb = 0, nc = 0;
    float here = 0.0f;
    bool rd = false;
    if (act) {
      const unsigned q = i + j;
      const unsigned xz = pc.qxz[q];
      a = (int)(xz & 0xFFFFu) + R.px0;
      c = (int)(xz >> 16) + R.pz0;
      b = (int)pc.qy[q];
      here = pc.qv[q];
      int dx, dy, dz;
      dir5((int)d, dx, dy, dz);
      na = a + dx;
      nb = b + dy;
      nc = c + dz;
      rd = d == 0 ? nb < R.ny : (na >= 0 && nc >= 0);
    }
    CD cd = CD{0.0f, NOSLOT, 0u, 0, true};
    bool rok = true;
    const long long r0 = clock64();
    if (rd) {
      if (mode == PM_SEQ) cd = load_cell_par(R, ring, na, nb, nc, T.spin_cap);
      else rok = read_mvcc(R, ps, ring, T, k, x, y, z, na, nb, nc, cd);
    }
    const bool allok = __all_sync(FULLMASK, rok);
    pf.tread += (unsigned long long)(clock64() - r0);
    pf.rounds += 1;
    if (!allok) {
      ok = false;
      break;
    }
    // surface test of each entry on its up neighbour (fluid.rs:534-535)
    const bool win = act && d == 0u && (nb >= R.ny || cd_solid(cd) || cd_volume(cd) <= 0.0f) && b > y && here > 0.0f;
    const unsigned wm = __ballot_sync(FULLMASK, win);
    if (wm) {
      const int wl = __ffs(wm) - 1;
      const int wa = __shfl_sync(FULLMASK, a, wl), wb = __shfl_sync(FULLMASK, b, wl), wc = __shfl_sync(FULLMASK, c, wl);
      const float wh = __shfl_sync(FULLMASK, here, wl);
      i += (unsigned)wl / 5u + 1u;
      const float take = fminf(need, wh);
      const long long w0 = clock64();
      const bool wok = pull_write(R, ps, ring, T, mode, k, wa, wb, wc, __fsub_rn(wh, take), co);
      pf.tpw += (unsigned long long)(clock64() - w0);
      if (!wok) {
        ok = false;
        break;
      }
      co.amask |= 1u;
      co.flags |= RF_SEED_SRC;
      got = take;
      break;
    }
    if (qlen < PQ_CAP) {
      // expansions (fluid.rs:541-556)
      bool cand = rd && !(nb >= R.ny || cd_solid(cd) || cd_volume(cd) <= 0.0f);
      const bool scnt = cand && d >= 1u && nb == y;
      const unsigned sm = __ballot_sync(FULLMASK, scnt);
      if (scnt && side + (unsigned)__popc(sm & lanemask_lt()) + 1u > 24u) cand = false;
      side += (unsigned)__popc(sm);
      const unsigned id = cand ? dom_id(R, na, nb, nc) : (0xFFFFFFFFu - lane);
      const unsigned peers = __match_any_sync(FULLMASK, id);
      const bool isnew = cand && !(peers & lanemask_lt()) && vis_insert_par(pc.vis, id);
      const unsigned nm = __ballot_sync(FULLMASK, isnew);
      if (isnew) {
        const unsigned pos = qlen + (unsigned)__popc(nm & lanemask_lt());
        if (pos < PQ_CAP) {
          pc.qxz[pos] = (unsigned)(na - R.px0) | ((unsigned)(nc - R.pz0) << 16);
          pc.qy[pos] = (unsigned short)nb;
          pc.qv[pos] = cd_volume(cd);
        }
      }
      qlen += (unsigned)__popc(nm);
    }
    i += kk;
    __syncwarp();
  }
  co.entries = i;
  __syncwarp();
  for (unsigned t = lane; t < PV_CAP; t += 32u) pc.vis[t] = EMPTY_ID;
  __syncwarp();
  return got;
}

// Before a pressure search on layer y, wait for every earlier cell of the layer within Chebyshev
// distance `gate` (earlier rows, through their finished-cell counts): the search's reads there and
// the sources of earlier pulls there are then final. Returns false on abort.
__device__ bool gate_wait(const Region& R, ParSmem& ps, const ParTick& T, int x, int y, int z) {
  const unsigned lane = lane_id();
  unsigned r = NOSLOT, needc = 0;
  if ((int)lane < T.gate) {
    const int zz = T.flip ? z + 1 + (int)lane : z - 1 - (int)lane;
    const int zr = zz - R.pz0;
    if (zr >= 0 && zr < R.PZ) {
      r = R.zrow[(size_t)y * (unsigned)R.PZ + (unsigned)zr];
      if (r != NOSLOT) {
        int xr = T.flip ? (R.PX - 1 - (x - T.gate - R.px0)) : (x + T.gate - R.px0);
        xr = min(xr, R.PX - 1);
        if (xr >= 0) {
          const unsigned zs = T.flip ? (unsigned)(R.PZ - 1 - zr) : (unsigned)zr;
          const unsigned kmax = ((unsigned)y * (unsigned)R.PZ + zs) * (unsigned)R.PX + (unsigned)xr;
          const unsigned a = R.rowstart[r];
          unsigned lo = a, hi = R.rowstart[r + 1];
          while (lo < hi) {
            const unsigned m = (lo + hi) >> 1;
            if (R.cells[m] <= kmax) lo = m + 1u;
            else hi = m;
          }
          needc = lo - a;
        }
      }
    }
  }
  bool pend = r != NOSLOT && needc > 0u;
  unsigned long long spins = 0;
  while (true) {
    pend = pend && gld(R.rowprog + r) < needc;
    if (!__any_sync(FULLMASK, pend)) return true;
    if (vld(&ps.abort)) return false;
    if (++spins > T.spin_cap) {
      if (lane == 0) par_timeout(R, ps, 37);
      __syncwarp();
      return false;
    }
    backoff(spins);
  }
}

// One drained cell (fluid.rs:584-651) at sorted position i, warp-collective. PM_PULL / PM_NOPULL:
// running beside other warps (waits, blocking, multi-version pull reads); PM_SEQ: one warp replaying
// a segment in order, attempts counted in `seq_pulls`. Returns false when the segment stops.
// pcw: the warp's search context in global memory (used when the shared pool is empty);
// jr: this lane's entry of the cell's earlier conflicting cells (ParDeps, lanes 0..9); cgi / cg:
// the lane's grid-word cache (load_cell_cached); row / rstart: the cell's row and its first sorted
// position (row NOSLOT: looked up); key: the cell's sort key (R.cells[i], loaded ahead by the caller).
__device__ bool process_cell_par(const Region& R, ParSmem& ps, PullCtx& pcw, const int* ring, const ParTick& T, int mode, unsigned i,
                                 unsigned& seq_pulls, ParProf& pf, unsigned jr, unsigned& cgi, unsigned& cg, unsigned row,
                                 unsigned rstart, unsigned key) {
  const unsigned lane = lane_id();
  long long c0 = clock64();
  const float FULL = full_level();
  const unsigned cid = key_to_id(R, key, T.flip);
  int x, y, z;
  dom_xyz(R, cid, x, y, z);
  // ---- earlier conflicting cells: earlier rows of the layer, the layer below, two below
  if (mode != PM_SEQ) {
    bool pend = (lane < 9u || (lane == 9u && mode == PM_PULL)) && jr != NOSLOT && jr >= T.seg_start;
    unsigned long long spins = 0;
    while (true) {
      pend = pend && cs_get(ps.state, jr) != CS_DONE;
      if (!__any_sync(FULLMASK, pend)) break;
      if (vld(&ps.abort)) return false;
      if (++spins > T.spin_cap) {
        if (lane == 0) par_timeout(R, ps, 38);
        __syncwarp();
        return false;
      }
      backoff(spins);
    }
    const long long c1 = clock64();
    pf.dep += (unsigned long long)(c1 - c0);
    c0 = c1;
    if (mode == PM_PULL && T.cone > 0 && !cone_wait(R, ps, T, threadIdx.x >> 5, y, z, sorted_xr(R, x, T.flip), T.cone)) return false;
    {
      const long long c1 = clock64();
      pf.cone += (unsigned long long)(c1 - c0);
      c0 = c1;
    }
    // start: pulls may hold the cell until they have written a source it reads
    bool ok = true;
    if (lane == 0) {
      if (mode == PM_PULL) {
        unsigned long long spins = 0;
        while (!cs_try_start(ps.state, i)) {
          if (vld(&ps.abort)) {
            ok = false;
            break;
          }
          if (++spins > T.spin_cap) {
            par_timeout(R, ps, 39);
            ok = false;
            break;
          }
          backoff(spins);
        }
      } else {
        atomicAdd(&ps.state[i >> 2], CS_STARTED << ((i & 3u) * 8u));
      }
    }
    if (!__shfl_sync(FULLMASK, ok ? 1u : 0u, 0)) return false;
    __threadfence_block();
    const long long c2 = clock64();
    pf.start += (unsigned long long)(c2 - c0);
    c0 = c2;
  }
  CellRec* rc = R.rec + i;
  // ---- footprint (lane l = slot l)
  int ox = 0, oy = 0, oz = 0;
  fp_off((int)lane, ox, oy, oz);
  CD mine = CD{0.0f, NOSLOT, 0u, 0, true};
  if (lane < 7u) {
    mine = load_cell_cached(R, ring, x + ox, y + oy, z + oz, T.spin_cap, cgi, cg);
    rc->opart[lane] = mine.part;
    rc->omat[lane] = mine.mat;
  }
  if (lane == 0) rc->flags = 0;
  // every lane gets what the rules read of the footprint, cd_solid and cd_volume: one ballot of
  // the solid cells and the 7 volumes (a solid cell's volume is never read). The atlas slot, grid
  // index, material and partial entry stay with the lane that loaded the cell (`mine`).
  CD fp[7];
  {
    const unsigned solid = __ballot_sync(FULLMASK, cd_solid(mine));
    const float lv = cd_volume(mine);
#pragma unroll
    for (int l = 0; l < 7; ++l) {
      const float v = __shfl_sync(FULLMASK, lv, l);
      const bool so = (solid >> l) & 1u;
      fp[l] = CD{so ? 0.0f : v, NOSLOT, 0u, (unsigned char)0, so};  // cd_solid = so, cd_volume = v
    }
  }
  {
    const long long c1 = clock64();
    pf.load += (unsigned long long)(c1 - c0);
    c0 = c1;
  }
  CellOut co{0u, 0u, 0u, 0u, 0u, 0};
  bool w = false;
  float wv = 0.0f;
  bool live = true;
  if (cd_solid(fp[0])) {
    // fluid.rs:586-589: a solid cell's partial entry is erased
    w = lane == 0 && mine.slot != NOSLOT && mine.part > 0.0f;
    live = false;
  }
  float vol = cd_volume(fp[0]);
  const float v0 = vol;
  if (live) {
    bool attempt = false;
    // in a segment with pulls, cells from T.pull_end on come after the budget's last attempt
    if (vol < FULL) attempt = (mode == PM_PULL && i < T.pull_end) || (mode == PM_SEQ && seq_pulls < MAX_PULLS_PER_TICK);
    if (attempt) {
      co.flags |= RF_ATTEMPT;
      if (mode == PM_SEQ) seq_pulls += 1;
      if (pull_has_start(fp, x, z)) {
        if (mode == PM_PULL && T.gate > 0 && !gate_wait(R, ps, T, x, y, z)) return false;
        {
          const long long c1 = clock64();
          pf.gate += (unsigned long long)(c1 - c0);
          pf.npull += 1;
          c0 = c1;
        }
        bool ok = true;
        // a search context: a free one of the shared pool, else the warp's own in global memory
        int pcs = -1;
        if (lane == 0) {
          unsigned m = vld(&ps.pc_free);
          for (int tries = 0; m && tries < 2 * NPC_SMEM; ++tries) {
            const int b = __ffs(m) - 1;
            const unsigned old = atomicAnd(&ps.pc_free, ~(1u << b));
            if (old & (1u << b)) {
              pcs = b;
              break;
            }
            m = old & ~(1u << b);
          }
        }
        pcs = __shfl_sync(FULLMASK, pcs, 0);
        // a shared context passes between warps: the last user's emptied visited set is released
        // before its free bit (fence, then atomicOr) and acquired after it (atomicAnd, then fence)
        if (pcs >= 0) __threadfence_block();
        PullCtx& pc = pcs >= 0 ? ps.pc[pcs] : pcw;
        const float got = pull_par(R, ps, pc, ring, T, mode, i, x, y, z, __fsub_rn(1.0f, vol), fp, co, ok, pf);
        if (pcs >= 0) {
          __threadfence_block();
          if (lane == 0) atomicOr(&ps.pc_free, 1u << pcs);
        }
        if (!ok) {
          if (lane == 0 && !vld(&ps.abort)) {
            vst(&ps.viol, 1u);
            vst(&ps.abort, 1u);
          }
          return false;
        }
        if (got > 0.0f) {
          co.flags |= RF_SUCCESS;
          vol = __fadd_rn(vol, got);
          co.amask |= 2u;
        }
        const long long c1 = clock64();
        pf.pull += (unsigned long long)(c1 - c0);
        c0 = c1;
      }
    }
    if (vol > 0.0f) {  // fluid.rs:602-604
      const CellPlan P = plan_flow(fp, vol);
      vol = P.vol;
      co.amask |= P.amask;
      const float dv = fabsf(__fsub_rn(vol, v0));
      if (lane == 0) {
        w = dv > 1e-7f;
        wv = vol;
      } else if (lane == 1) {
        w = P.w_below;
        wv = P.below_new;
      } else if (lane >= 3u && lane < 7u) {
        w = (P.wside >> (lane - 3u)) & 1u;
        wv = P.side_new[lane - 3u];
      }
      if (dv > SLEEP) {
        co.amask |= 0x80u;
        co.flags |= RF_SEED_SELF;
      }
    }
  }
  // ---- publish the record, then write (readers of old versions use the record)
  const bool needm = w && live && set_volume_needs_slot(mine, wv);
  if (__any_sync(FULLMASK, needm)) materialize_par(R, needm, mine.gi, mine.slot, T.spin_cap);
  SVPlan p{};
  if (w) {
    if (live) {
      p = sv_plan(mine, wv);
    } else {  // PartialField::erase of a solid cell
      p.npart = 0.0f;
      p.nmat = mine.mat;
      p.wpart = true;
      p.wmat = false;
      p.ch = false;
      p.dp = -1;
    }
  }
  const unsigned wmask = __ballot_sync(FULLMASK, w) & 0x7Fu;
  const unsigned chm = __ballot_sync(FULLMASK, w && p.ch) & 0x7Fu;
  // partial-entry count change: each lane's is -1, 0 or +1
  const int pd = __popc(__ballot_sync(FULLMASK, w && p.dp > 0)) - __popc(__ballot_sync(FULLMASK, w && p.dp < 0));
  if (lane == 0) {
    co.cmask |= chm;
    co.pdelta += pd;
    if (chm) co.flags |= RF_CHANGED;
    rc->wmask = (unsigned char)wmask;
    rc->cmask = (unsigned char)co.cmask;
    rc->amask = (unsigned char)co.amask;
    rc->flags = (unsigned char)co.flags;
    rc->pdelta = (signed char)co.pdelta;
    rc->src = co.src;
    rc->entries = (unsigned short)co.entries;
    rc->tk_main = atomicAdd(&ps.ticket, 1u);
  }
  __syncwarp();
  __threadfence_block();
  const unsigned sh = (i & 3u) * 8u;
  if (lane == 0) {
    if (mode != PM_SEQ) cs_advance(ps.state, i);
    else ps.state[i >> 2] = (ps.state[i >> 2] & ~(0xFFu << sh)) | (CS_WRITING << sh);
  }
  __syncwarp();
  if (w && mine.slot != NOSLOT) sv_apply(R, mine, x + ox, y + oy, z + oz, p);
  __syncwarp();
  __threadfence_block();
  if (lane == 0) {
    if (row == NOSLOT) {
      row = R.rowof[i] & 0x3FFFFFFFu;
      rstart = R.rowstart[row];
    }
    vst(R.rowprog + row, i - rstart + 1u);
    if (mode != PM_SEQ) cs_advance(ps.state, i);
    else ps.state[i >> 2] = (ps.state[i >> 2] & ~(0xFFu << sh)) | (CS_DONE << sh);
  }
  __syncwarp();
  pf.write += (unsigned long long)(clock64() - c0);
  pf.cells += 1;
  return true;
}

// Location and execution ticket of write slot l (0..6 footprint, 7 pull source) of the cell at
// sorted position i; false if the cell did not make that write. Valid once the cell stopped (no warp
// runs in the segment).
__device__ __forceinline__ bool rb_write(const Region& R, const ParSmem& ps, unsigned i, unsigned cid, unsigned l, unsigned& loc,
                                         unsigned& tk) {
  const unsigned st = cs_get(ps.state, i);
  if (st < CS_STARTED) return false;
  const CellRec& rc = R.rec[i];
  if (l == 7u) {
    if (!(rc.flags & RF_SRCW)) return false;
    loc = rc.src;
    tk = rc.tk_src;
    return true;
  }
  if (st < CS_WRITING || !((rc.wmask >> l) & 1u)) return false;
  tk = rc.tk_main;
  const unsigned px = (unsigned)R.PX, pxy = px * (unsigned)R.PY;
  switch (l) {
    case 0: loc = cid; break;
    case 1: loc = cid - px; break;
    case 3: loc = cid + 1u; break;
    case 4: loc = cid - 1u; break;
    case 5: loc = cid + pxy; break;
    default: loc = cid - pxy; break;  // 6 (slot 2, up, is never written)
  }
  return true;
}

// Offset of the l-th (0..9) position whose earlier drained cell a cell conflicts with: earlier rows
// of its layer (x-1, x, x+1 one row back, x two rows back, mirrored on odd ticks), the five cells of
// the layer below under its plus footprint, and the cell two below (whose start test reads the cell
// this one falls into).
__device__ __forceinline__ void dep_offset(unsigned l, bool flip, int& dx, int& dy, int& dz) {
  dx = dy = dz = 0;
  if (l < 4u) {
    const int s = flip ? 1 : -1;
    dz = l == 3u ? 2 * s : s;
    dx = l == 0u ? -1 : (l == 2u ? 1 : 0);
  } else if (l < 9u) {
    const unsigned q = l - 4u;
    dy = -1;
    dx = (q == 1u) - (q == 2u);
    dz = (q == 3u) - (q == 4u);
  } else {
    dy = -2;  // 9
  }
}

// Undo the writes of segment [a, b), CTA-wide: every cell written in the segment gets back the
// value replaced by its first write in execution order (tickets), which is its value at the
// segment's start. `rb` (one word per domain cell, all 0xFFFFFFFF between calls) finds that write.
// All threads call; no warp may be running in the segment.
__device__ void rollback_segment(const Region& R, ParSmem& ps, const int* ring, unsigned a, unsigned b, bool flip) {
  const unsigned nt = blockDim.x;
  for (int phase = 0; phase < 3; ++phase) {
    for (unsigned t = threadIdx.x; t < (b - a) * 8u; t += nt) {
      const unsigned i = a + t / 8u, l = t % 8u;
      if (l == 2u) continue;
      const unsigned cid = key_to_id(R, R.cells[i], flip);
      unsigned loc, tk;
      if (!rb_write(R, ps, i, cid, l, loc, tk)) continue;
      if (phase == 0) {
        atomicMin(R.rb + loc, tk);
      } else if (phase == 1) {
        if (__ldcg(R.rb + loc) != tk) continue;  // set by atomics (in L2): read past L1
        int x, y, z;
        dom_xyz(R, loc, x, y, z);
        const CD c = load_cell(R, ring, x, y, z);
        if (c.slot == NOSLOT) continue;
        const CellRec& rc = R.rec[i];
        const size_t o = (size_t)c.slot * 512u + local_index(x, y, z);
        R.amat[o] = l == 7u ? rc.src_omat : rc.omat[l];
        R.avol[o] = l == 7u ? rc.src_opart : rc.opart[l];
      } else {
        R.rb[loc] = 0xFFFFFFFFu;
      }
    }
    __syncthreads();
  }
}

}  // namespace vfe
