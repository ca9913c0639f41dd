// Kernels of the CA-water engine: the tick (drain -> sort -> sweep -> levelling) for one or many
// regions, host-edit kernels (wake, displace, brush, emitters, set_partial) and inspection
// kernels (digests, dense export, change download).
#pragma once
#include <cuda_fp16.h>

#include "engine_dev.cuh"
#include "sweep_par.cuh"

namespace vfe {

// blockDim-derived thread / warp counts of the running CTA
#define NT_ ((unsigned)blockDim.x)
#define NW_ ((unsigned)(blockDim.x >> 5))

// Launch shapes: the one-warp sweep runs 8 warps per region (the sweep plus prefetchers), the
// parallel sweep MAX_WARPS (row workers). CTA-wide helpers below use the launched block size;
// shared arrays are sized for the larger shape.
constexpr int TICK_THREADS = 256;
constexpr int TICK_WARPS = TICK_THREADS / 32;
constexpr int PAR_THREADS = MAX_WARPS * 32;
constexpr int PEXPOSE = 3;            // water cells over a full cell that pulls may empty in one tick
constexpr unsigned PAR_MAX_SPLITS = 6;  // conflicts at one position before it runs in order

// ---------------------------------------------------------------- CTA radix sort (LSD, 8 bit)
// Stable within each warp's contiguous chunk; chunks in order -> stable overall. Sorts n unique
// keys in place (tmp is scratch). hist: NW_*256 u32 of shared memory.
__device__ void cta_radix_sort(unsigned* keys, unsigned* tmp, unsigned n, unsigned* hist, unsigned* sred) {
  const unsigned tid = threadIdx.x, lane = tid & 31u, warp = tid >> 5;
  if (n <= 1) return;
  // key range -> number of passes
  unsigned mn = 0xFFFFFFFFu, mx = 0;
  for (unsigned i = tid; i < n; i += NT_) {
    unsigned k = keys[i];
    mn = min(mn, k);
    mx = max(mx, k);
  }
  for (int o = 16; o; o >>= 1) {
    mn = min(mn, __shfl_xor_sync(FULLMASK, mn, o));
    mx = max(mx, __shfl_xor_sync(FULLMASK, mx, o));
  }
  if (lane == 0) {
    sred[warp] = mn;
    sred[NW_ + warp] = mx;
  }
  __syncthreads();
  if (tid == 0) {
    unsigned a = 0xFFFFFFFFu, b = 0;
    for (int w = 0; w < NW_; ++w) {
      a = min(a, sred[w]);
      b = max(b, sred[NW_ + w]);
    }
    sred[2 * NW_] = a;
    sred[2 * NW_ + 1] = b;
  }
  __syncthreads();
  const unsigned kmin = sred[2 * NW_], range = sred[2 * NW_ + 1] - kmin;
  __syncthreads();
  const int bits = range ? 32 - __clz(range) : 0;
  const int passes = (bits + 7) / 8;
  const unsigned chunk = (n + NW_ - 1) / NW_;
  const unsigned b0 = min(n, warp * chunk), b1 = min(n, b0 + chunk);
  unsigned* src = keys;
  unsigned* dst = tmp;
  for (int p = 0; p < passes; ++p) {
    const int sh = 8 * p;
    for (unsigned i = tid; i < NW_ * 256; i += NT_) hist[i] = 0;
    __syncthreads();
    for (unsigned i = b0 + lane; i < b1; i += 32) atomicAdd(&hist[warp * 256 + (((src[i] - kmin) >> sh) & 255u)], 1u);
    __syncthreads();
    // offsets: digit-major, warp-minor
    if (tid < 256) {
      unsigned s = 0;
      for (int w = 0; w < NW_; ++w) s += hist[w * 256 + tid];
      sred[tid] = s;
    }
    __syncthreads();
    if (tid < 32) {
      // exclusive scan of 256 digit totals by one warp (8 per lane)
      unsigned v[8], t = 0;
      for (int k = 0; k < 8; ++k) {
        v[k] = sred[lane * 8 + k];
        t += v[k];
      }
      unsigned incl = t;
      for (int o = 1; o < 32; o <<= 1) {
        unsigned u = __shfl_up_sync(FULLMASK, incl, o);
        if (lane >= (unsigned)o) incl += u;
      }
      unsigned run = incl - t;
      for (int k = 0; k < 8; ++k) {
        sred[256 + lane * 8 + k] = run;
        run += v[k];
      }
    }
    __syncthreads();
    if (tid < 256) {
      unsigned run = sred[256 + tid];
      for (int w = 0; w < NW_; ++w) {
        unsigned c = hist[w * 256 + tid];
        hist[w * 256 + tid] = run;
        run += c;
      }
    }
    __syncthreads();
    for (unsigned base = b0; base < b1; base += 32) {
      unsigned i = base + lane;
      bool valid = i < b1;
      unsigned k = valid ? src[i] : 0u;
      unsigned d = valid ? (((k - kmin) >> sh) & 255u) : (256u + lane);
      unsigned peers = __match_any_sync(FULLMASK, d);
      unsigned rank = __popc(peers & lanemask_lt());
      unsigned pos = 0;
      if (valid) pos = hist[warp * 256 + d] + rank;
      __syncwarp();
      if (valid) {
        dst[pos] = k;
        if (rank == 0) hist[warp * 256 + d] += __popc(peers);
      }
      __syncwarp();
    }
    __syncthreads();
    unsigned* t = src;
    src = dst;
    dst = t;
  }
  if (src != keys) {
    for (unsigned i = tid; i < n; i += NT_) keys[i] = src[i];
    __syncthreads();
  }
}

// ----------------------------------------------------------------------------- the tick
constexpr int PF_RING = 64;                      // prefetched footprints in flight

// Launch-time knobs of the tick (results do not depend on them): which sweep runs, the one-warp
// sweep's producer warps and prefetch distance (chosen by the autotuner), the parallel sweep's
// pull gate radius and the iteration cap of device waits.
struct Tune {
  int producers;  // one-warp sweep: 1 .. TICK_WARPS-1 prefetching warps
  int depth;      // one-warp sweep: 1 .. PF_RING cells ahead
  int engine;     // 0 one-warp sweep (TICK_THREADS per region), 1 parallel sweep (PAR_THREADS)
  int gate;       // parallel sweep: bits 0-7 gate radius, 8-15 cone radius (0..GATE_MAX), 16-20 warps (0: MAX_WARPS), 21 global search contexts only
  unsigned long long spin_cap;  // iterations before a wait gives up (ST_TIMEOUT)
};

// Shared memory of the one-warp sweep: prefetch ring, store forwarding and search structures.
struct SeqSmem {
  int4 pq[PRESS_QCAP];
  unsigned long long vis[VIS_CAP];
  unsigned vb[VB_WORDS];        // pressure-search visited bitmap (zero between searches)
  unsigned vtl[PRESS_QCAP];     // bitmap words touched by the current search
  CD pf[PF_RING][7];            // prefetched footprints (self, below, up, +x, -x, +z, -z)
  unsigned pf_ready[PF_RING];   // the cell index whose footprint a slot holds
  int pxyz[PF_RING][4];         // the cell's coordinates and domain id
  unsigned pf_c0[PF_RING];      // cells the sweep had finished when the slot's footprint was fetched
  unsigned pf_quiet[PF_RING];   // classify_quiet of the fetched footprint
  FwdEntry fwd[FWD_SIZE];       // the sweep's latest writes (store forwarding)
  unsigned long long gc[GCACHE];  // grid-word cache of the sweep's pressure searches
  SearchHelp help;              // neighbour loads by idle prefetchers ahead of a search
  unsigned consumed;            // cells the sweep has finished
  unsigned abort;               // a wait gave up: every warp leaves the sweep
};

struct TickSmem {
  unsigned hist[MAX_WARPS * 256];
  unsigned sred[2 * 256 + 64];
  int ring[3 * 16 * 16];
  unsigned scan[MAX_WARPS + 1];
  union {
    SeqSmem s;  // one-warp sweep
    ParSmem p;  // parallel sweep
  } u;
};

__device__ void load_ws(const Region& R, WS& W) {
  const Ctl& c = *R.ctl;
  W.qhead = c.qhead;
  W.qtail = c.qtail;
  W.activations = 0;
  W.pull_attempts = 0;
  W.pull_success = 0;
  W.bfs_visits = 0;
  W.level_cells_total = 0;
  W.pdelta = 0;
  W.nseeds = c.nseeds;
  W.pulls = 0;
  W.llc = c.last_level_cells;
  W.ndrain = 0;
  W.epoch = 1;
  W.level_round = c.level_round != 0;
  W.changed = false;
  W.deferred = false;
  W.nact = W.nseed = W.nchg = 0;
  W.fwd = nullptr;
  W.seq = 0;
  W.gc = nullptr;
  W.t_wait = W.t_pull = W.t_act = W.t_write = W.t_top = W.t_pc = W.t_tail = 0;
#ifdef VF_FINE_PROFILE
  W.f_pre = W.f_plan = W.f_seed = W.n_pc = W.n_quiet = W.n_rounds = W.f_bload = W.f_bexp = W.f_match = W.f_vis = 0;
#endif
}

// Load a cell for the prefetch ring: the grid word is read with a fence after it, pairing with
// the sweep's fenced publication of freshly materialised bricks.
__device__ __forceinline__ CD load_cell_acq(const Region& R, const int* ring, int x, int y, int z) {
  CD c;
  c.part = 0.0f;
  c.slot = NOSLOT;
  c.gi = 0;
  c.mat = 0;
  c.out = outside(R, ring, x, y, z);
  if (c.out) return c;
  c.gi = grid_index(R, x >> 3, y >> 3, z >> 3);
  unsigned g = *(volatile const unsigned*)(R.grid + c.gi);
  __threadfence_block();
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

// ----------------------------------------------------------------- CTA-wide ordered commits
// Exclusive prefix of per-thread flags over the CTA (in thread order). Returns this thread's
// offset; *total gets the CTA total. All threads must call.
__device__ unsigned cta_scan(TickSmem& sm, bool f, unsigned* total) {
  const unsigned lane = threadIdx.x & 31u, warp = threadIdx.x >> 5;
  unsigned b = __ballot_sync(FULLMASK, f);
  if (lane == 0) sm.scan[warp] = __popc(b);
  __syncthreads();
  unsigned before = 0, all = 0;
  for (int w = 0; w < NW_; ++w) {
    unsigned c = sm.scan[w];
    if ((unsigned)w < warp) before += c;
    all += c;
  }
  __syncthreads();
  *total = all;
  return before + __popc(b & lanemask_lt());
}

// First occurrence of each cell id in an event log (stamp = lowest event index).
__device__ void stamp_first(const Region& R, const unsigned* ev, unsigned n) {
  for (unsigned i = threadIdx.x; i < n; i += NT_) atomicMin(&R.stamp[ev[i]], i);
  __syncthreads();
}
__device__ void stamp_clear(const Region& R, const unsigned* ev, unsigned n) {
  __syncthreads();
  for (unsigned i = threadIdx.x; i < n; i += NT_) R.stamp[ev[i]] = 0xFFFFFFFFu;
  __syncthreads();
}

// The sweep's FluidSim::activate calls in program order (fluid.rs:292-300): a cell joins the
// FIFO at its first activation if it was not active already.
// Exclusive prefix of per-thread counts over the CTA (thread order); *total = the CTA sum.
__device__ unsigned cta_scan_count(TickSmem& sm, unsigned c, unsigned* total) {
  const unsigned lane = threadIdx.x & 31u, warp = threadIdx.x >> 5;
  unsigned incl = c;
  for (int o = 1; o < 32; o <<= 1) {
    unsigned u = __shfl_up_sync(FULLMASK, incl, o);
    if (lane >= (unsigned)o) incl += u;
  }
  if (lane == 31) sm.scan[warp] = incl;
  __syncthreads();
  unsigned before = 0, all = 0;
  for (int w = 0; w < NW_; ++w) {
    unsigned s = sm.scan[w];
    if ((unsigned)w < warp) before += s;
    all += s;
  }
  __syncthreads();
  *total = all;
  return before + incl - c;
}

// Cell o of an activation-log word: a single cell, or wake_around's order self, +x, -x, +y, -y,
// +z, -z (fluid.rs:302-310). Returns false for cells activate() ignores (y < 0).
__device__ __forceinline__ bool act_cell(const Region& R, unsigned word, int o, unsigned& id) {
  const unsigned c = word & ~ACT_AROUND;
  if (!(word & ACT_AROUND)) {
    id = c;
    return o == 0;
  }
  const unsigned px = (unsigned)R.PX, pxy = px * (unsigned)R.PY;
  switch (o) {
    case 0: id = c; return true;
    case 1: id = c + 1u; return true;
    case 2: id = c - 1u; return true;
    case 3: id = c + px; return true;
    case 4: {  // y - 1 < 0
      id = c - px;
      const unsigned t = udiv(c, px, R.mx);
      return t != udiv(t, (unsigned)R.PY, R.my) * (unsigned)R.PY;
    }
    case 5: id = c + pxy; return true;
    default: id = c - pxy; return true;
  }
}

// The tick's FluidSim::activate calls in program order (fluid.rs:292-300): a cell joins the
// FIFO at its first activation if it was not active already. Log word i covers activation
// indices 8i..8i+6, which keeps program order for the first-occurrence stamps.
__device__ void commit_acts(const Region& R, TickSmem& sm, unsigned n, unsigned long long& qtail, unsigned long long qhead) {
  for (unsigned i = threadIdx.x; i < n; i += NT_) {
    unsigned w = R.ev_act[i], id;
    for (int o = 0; o < 7; ++o)
      if (act_cell(R, w, o, id)) atomicMin(&R.stamp[id], i * 8u + (unsigned)o);
  }
  __syncthreads();
  __shared__ unsigned long long s_tail;
  if (threadIdx.x == 0) s_tail = qtail;
  __syncthreads();
  for (unsigned base = 0; base < n; base += NT_) {
    const unsigned i = base + threadIdx.x;
    unsigned newmask = 0, w = 0;
    if (i < n) {
      w = R.ev_act[i];
      // the word's cells, then all their stamps and active words in flight together
      unsigned ids[7], st[7], ac[7];
      bool ok[7];
#pragma unroll
      for (int o = 0; o < 7; ++o) ok[o] = act_cell(R, w, o, ids[o]);
#pragma unroll
      for (int o = 0; o < 7; ++o) {
        st[o] = ok[o] ? R.stamp[ids[o]] : 0xFFFFFFFFu;
        ac[o] = ok[o] ? R.active[ids[o] >> 5] : 0u;
      }
#pragma unroll
      for (int o = 0; o < 7; ++o)
        if (ok[o] && st[o] == i * 8u + (unsigned)o && !((ac[o] >> (ids[o] & 31u)) & 1u)) newmask |= 1u << o;
    }
    unsigned total;
    unsigned off = cta_scan_count(sm, __popc(newmask), &total);
    for (int o = 0; o < 7; ++o) {
      if (!(newmask & (1u << o))) continue;
      unsigned id;
      act_cell(R, w, o, id);
      R.queue[(s_tail + off) & R.qmask] = id;
      atomicOr(&R.active[id >> 5], 1u << (id & 31));
      ++off;
    }
    __syncthreads();
    if (threadIdx.x == 0) s_tail += total;
    __syncthreads();
  }
  qtail = s_tail;
  if (threadIdx.x == 0 && s_tail - qhead > R.qmask + 1ull) set_status(R, ST_OOM, 12);
  __syncthreads();
  for (unsigned i = threadIdx.x; i < n; i += NT_) {
    unsigned w = R.ev_act[i], id;
    for (int o = 0; o < 7; ++o)
      if (act_cell(R, w, o, id)) R.stamp[id] = 0xFFFFFFFFu;
  }
  __syncthreads();
}

// FluidSim::seed_level calls in order (fluid.rs:312-316): first insertion of a cell not yet a
// seed, while the set holds fewer than MAX_LEVEL_SEEDS.
__device__ void commit_seeds(const Region& R, TickSmem& sm, unsigned n, unsigned& nseeds) {
  stamp_first(R, R.ev_seed, n);
  __shared__ unsigned s_ns;
  if (threadIdx.x == 0) s_ns = nseeds;
  __syncthreads();
  for (unsigned base = 0; base < n; base += NT_) {
    unsigned i = base + threadIdx.x;
    bool isnew = false;
    unsigned id = 0;
    if (i < n) {
      id = R.ev_seed[i];
      isnew = R.stamp[id] == i && !((R.seedbits[id >> 5] >> (id & 31)) & 1u);
    }
    unsigned total;
    unsigned off = cta_scan(sm, isnew, &total);
    unsigned pos = s_ns + off;
    if (isnew && pos < MAX_LEVEL_SEEDS) {
      R.seeds[pos] = id;
      atomicOr(&R.seedbits[id >> 5], 1u << (id & 31));
    }
    __syncthreads();
    if (threadIdx.x == 0) s_ns = min(MAX_LEVEL_SEEDS, s_ns + total);
    __syncthreads();
  }
  nseeds = s_ns;
  stamp_clear(R, R.ev_seed, n);
}

// Voxel changes for the host (order irrelevant; the host sorts and dedups its dirty list).
__device__ void commit_chgs(const Region& R, unsigned n) {
  for (unsigned i = threadIdx.x; i < n; i += NT_) record_change(R, R.ev_chg[i]);
  __syncthreads();
}

// ------------------------------------------------------------------------ the sweep
// Warp 0 walks the sorted cells (the reference's order); warps 1.. prefetch footprints of the
// cells ahead into a shared-memory ring, each stamped with the number of cells the sweep had
// finished when it was fetched. Values the sweep wrote after a fetch come from the
// store-forwarding table (or, when the table cannot tell, from memory).
__device__ void sweep(const Region& R, TickSmem& sm, WS& sW, const int* ring, unsigned n, bool flip, Tune tune) {
  const unsigned tid = threadIdx.x, lane = tid & 31u, warp = tid >> 5;
  if (tid == 0) {
    sm.u.s.consumed = 0;
    sm.u.s.abort = 0;
  }
  for (unsigned i = tid; i < PF_RING; i += NT_) sm.u.s.pf_ready[i] = 0xFFFFFFFFu;
  for (unsigned i = tid; i < FWD_SIZE; i += NT_) sm.u.s.fwd[i].meta = 0u;
  for (unsigned i = tid; i < GCACHE; i += NT_) sm.u.s.gc[i] = ~0ull;
  __syncthreads();
  if (warp == 0) {
    WS W = sW;
    W.fwd = sm.u.s.fwd;
    W.gc = sm.u.s.gc;
    Smem S{sm.u.s.vis, ring, sm.u.s.pq, sm.u.s.vb, sm.u.s.vtl, &sm.u.s.help, &sm.u.s.abort, tune.spin_cap};
    const unsigned pxy = (unsigned)R.PX * (unsigned)R.PY;
    // footprint offsets (self, below, up, +x, -x, +z, -z) of this lane, in cells and in ids
    const int ox = (lane == 3) - (lane == 4), oy = (lane == 2) - (lane == 1), oz = (lane == 5) - (lane == 6);
    const unsigned oid = (unsigned)ox + (unsigned)oy * (unsigned)R.PX + (unsigned)oz * pxy;
    for (unsigned r = 0; r < n; ++r) {
      const unsigned slot = r % PF_RING;
      // wait (bounded) for the footprint of cell r; every lane reads the same word
      const long long tw = fine_clock();
      unsigned long long spins = 0;
      while (*(volatile unsigned*)&sm.u.s.pf_ready[slot] != r) {
        if (++spins > tune.spin_cap) break;
        __nanosleep(20);
      }
      if (spins > tune.spin_cap) {
        if (lane == 0) {
          set_status(R, ST_TIMEOUT, 20);
          *(volatile unsigned*)&sm.u.s.abort = 1u;
        }
        break;
      }
      __threadfence_block();
      W.t_wait += fine_clock() - tw;
      const int x = sm.u.s.pxyz[slot][0], y = sm.u.s.pxyz[slot][1], z = sm.u.s.pxyz[slot][2];
      const unsigned cid = (unsigned)sm.u.s.pxyz[slot][3];
      const unsigned c0 = sm.u.s.pf_c0[slot];
      const unsigned quiet = sm.u.s.pf_quiet[slot];
      // footprint cells the sweep wrote since the fetch: from the forwarding table, or from
      // memory when another cell's write took the cell's table entry
      bool touched = false;
      if (lane < 7) {
        CD mine = sm.u.s.pf[slot][lane];
        const int fx = x + ox, fy = y + oy, fz = z + oz;
        const FwdEntry e = sm.u.s.fwd[fwd_index(fx, fy, fz)];
        if (!mine.out && (e.meta & 0xFFFFu) > c0) {
          touched = true;
          if (e.tag == cid + oid) {
            mine.mat = (unsigned char)(e.meta >> 16);
            mine.part = e.part;
            mine.slot = e.slot;
          } else {
            mine = load_cell(R, ring, fx, fy, fz);
          }
          sm.u.s.pf[slot][lane] = mine;
        }
      }
      const bool stale = __any_sync(FULLMASK, touched);
      __syncwarp();
      const long long t1 = fine_clock();
      W.t_top += t1 - tw;
      W.seq = r + 1u;
      if (!stale && (quiet & QUIET)) {
        // nothing to write, activate or seed (classified by the prefetcher on this footprint):
        // only the pull budget counts the attempt
        if ((quiet & QUIET_PULL) && W.pulls < MAX_PULLS_PER_TICK) {
          W.pulls += 1;
          W.pull_attempts += 1;
        }
#ifdef VF_FINE_PROFILE
        W.n_quiet += 1;
#endif
      } else {
        CD fp[7];
#pragma unroll
        for (int j = 0; j < 7; ++j) fp[j] = sm.u.s.pf[slot][j];
        const CD mine = lane < 7 ? sm.u.s.pf[slot][lane] : CD{0.0f, NOSLOT, 0u, 0, true};
        process_cell(R, W, S, x, y, z, x + ox, y + oy, z + oz, fp, mine);
      }
      __syncwarp();
      const long long t2 = fine_clock();
      W.t_pc += t2 - t1;
      __threadfence_block();
      if (lane == 0) *(volatile unsigned*)&sm.u.s.consumed = r + 1u;
      W.t_tail += fine_clock() - t2;
    }
    W.fwd = nullptr;
    W.gc = nullptr;
    long long pd = W.pdelta;  // lane-local partial-count deltas
    for (int o = 16; o; o >>= 1) pd += __shfl_xor_sync(FULLMASK, pd, o);
    W.pdelta = pd;
    if (lane == 0) {
      sW = W;
      Ctl& c = *R.ctl;
      c.prof[3] += W.t_wait;
      c.prof[4] += W.t_pull;
      c.prof[5] += W.t_act;
      c.prof[6] += W.t_write;
      c.prof[12] += W.t_top;
      c.prof[13] += W.t_pc;
      c.prof[14] += W.t_tail;
      sW.t_wait = sW.t_pull = sW.t_act = sW.t_write = sW.t_top = sW.t_pc = sW.t_tail = 0;
#ifdef VF_FINE_PROFILE
      c.prof[16] += W.f_pre;
      c.prof[17] += W.f_plan;
      c.prof[18] += W.f_seed;
      c.prof[19] += W.n_pc;
      c.prof[20] += W.n_quiet;
      c.prof[21] += W.n_rounds;
      c.prof[22] += W.f_bload;
      c.prof[23] += W.f_bexp;
      c.prof[24] += W.f_match;
      c.prof[25] += W.f_vis;
      sW.f_pre = sW.f_plan = sW.f_seed = sW.n_pc = sW.n_quiet = sW.n_rounds = sW.f_bload = sW.f_bexp = sW.f_match = sW.f_vis = 0;
#endif
    }
    __syncwarp();
  } else if (warp <= (unsigned)tune.producers) {
    // producers: warp p prefetches cells p-1, p-1+NP, ...
    const unsigned NP = (unsigned)tune.producers;
    const unsigned depth = (unsigned)tune.depth;
    for (unsigned r = warp - 1; r < n; r += NP) {
      // wait (bounded) until the ring slot of cell r is free; every lane reads the same words
      unsigned long long spins = 0;
      unsigned c0;
      bool ok = true;
      while ((c0 = *(volatile unsigned*)&sm.u.s.consumed) + depth <= r) {
        if (*(volatile unsigned*)&sm.u.s.abort || ++spins > tune.spin_cap) {
          ok = false;
          break;
        }
        // nothing to prefetch yet: load neighbours for a running pressure search, else yield
        // issue slots to the sweep warp
        if (!help_search(R, ring, &sm.u.s.help, sm.u.s.pq)) __nanosleep(200);
      }
      if (!ok) break;
      __threadfence_block();
      int x, y, z;
      const unsigned cid = key_to_id(R, R.cells[r], flip);
      dom_xyz(R, cid, x, y, z);
      const unsigned s = r % PF_RING;
      if (lane < 7) {
        int fx = x + (lane == 3) - (lane == 4), fy = y - (lane == 1) + (lane == 2), fz = z + (lane == 5) - (lane == 6);
        sm.u.s.pf[s][lane] = load_cell_acq(R, ring, fx, fy, fz);
      } else if (lane == 7) {
        sm.u.s.pxyz[s][0] = x;
        sm.u.s.pxyz[s][1] = y;
        sm.u.s.pxyz[s][2] = z;
        sm.u.s.pxyz[s][3] = (int)cid;
        sm.u.s.pf_c0[s] = c0;
      }
      __syncwarp();
      CD fq[7];
#pragma unroll
      for (int j = 0; j < 7; ++j) fq[j] = sm.u.s.pf[s][j];
      const unsigned q = classify_quiet(fq, x, z);
      if (lane == 0) sm.u.s.pf_quiet[s] = q;
      __syncwarp();
      __threadfence_block();
      if (lane == 0) *(volatile unsigned*)&sm.u.s.pf_ready[s] = r;
    }
  }
  __syncthreads();
}
// ------------------------------------------------------------------- the parallel sweep
// Segment end for `room` more attempts from `pos` (one thread): the largest e <= n with at most
// `room` cells in [pos, e) that may attempt a pull. `extra` cells at or after pos, taken below full
// by earlier pulls of the tick although not counted in pcnt, are charged up front.
__device__ unsigned seg_end_for(const Region& R, unsigned pos, unsigned n, unsigned room, unsigned extra, float ratio, float factor) {
  if (extra >= room) return pos + 1u;
  // sized for `factor` times the attempts expected at `ratio` per possible attempter; a segment
  // that overshoots the budget is undone and cut at its room-th attempt (exact either way)
  unsigned span = room - extra;
  if (span > 32u && ratio * (1.0f / factor) < 1.0f) span = (unsigned)fminf(4.0e9f, factor * (float)span / ratio);
  const unsigned lim = R.pcnt[pos] + span;
  unsigned lo = pos + 1u, hi = n;  // answer in [pos + 1, n]
  while (lo < hi) {
    const unsigned m = (lo + hi + 1u) >> 1;
    if (R.pcnt[m] <= lim) lo = m;
    else hi = m - 1u;
  }
  return lo;
}

// Sum of a per-thread value over the CTA (all threads call).
__device__ unsigned long long cta_sum(TickSmem& sm, unsigned long long v) {
  for (int o = 16; o; o >>= 1) v += __shfl_xor_sync(FULLMASK, v, o);
  __shared__ unsigned long long s_part[MAX_WARPS];
  if ((threadIdx.x & 31u) == 0) s_part[threadIdx.x >> 5] = v;
  __syncthreads();
  unsigned long long t = 0;
  for (unsigned w = 0; w < NW_; ++w) t += s_part[w];
  __syncthreads();
  return t;
}

// The sweep of one tick by every warp of the CTA (sweep_par.cuh describes the schedule). On return
// the tick's activation, seed and change logs hold the sweep's events in program order and sW its
// counters, exactly as the one-warp sweep leaves them.
__device__ __noinline__ void sweep_parallel(const Region& R, TickSmem& sm, WS& sW, const int* ring, unsigned n, bool flip, Tune tune) {
  ParSmem& ps = sm.u.p;
  const unsigned tid = threadIdx.x, lane = tid & 31u, warp = tid >> 5;
  const float FULL = full_level();
  long long tp0 = clock64();
  auto plap = [&](int k) {
    if (tid == 0) {
      const long long now = clock64();
      R.ctl->pprof[k] += (unsigned long long)(now - tp0);
      tp0 = now;
    }
  };
  ParProf pf{0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0};
  unsigned long long w_fetch = 0, w_total = 0;
  // ---- positions, rows and the cells that may attempt a pull (fluid.rs:594)
  __shared__ unsigned s_rows, s_pc;
  if (tid == 0) {
    s_rows = 0;
    s_pc = 0;
  }
  __syncthreads();
  for (unsigned base = 0; base < n; base += NT_) {
    const unsigned i = base + tid;
    const bool valid = i < n;
    unsigned rowflag = 0, P = 0, S = 0;
    int x = 0, y = 0, z = 0;
    if (valid) {
      const unsigned key = R.cells[i];
      const unsigned cid = key_to_id(R, key, flip);
      R.stamp[cid] = i;
      rowflag = (i == 0u || udiv(key, (unsigned)R.PX, R.mx) != udiv(R.cells[i - 1u], (unsigned)R.PX, R.mx)) ? 1u : 0u;
      dom_xyz(R, cid, x, y, z);
      // the cell and the PEXPOSE + 1 cells over it, loads issued together
      CD col[PEXPOSE + 2];
#pragma unroll
      for (int d = 0; d <= PEXPOSE + 1; ++d) col[d] = load_cell(R, ring, x, y + d, z);
      const CD c = col[0];
      S = cd_solid(c) ? 1u : 0u;
      if (!S) {
        // A cell attempts only below 1 - 1e-4. One full at the tick's start gets there only as a
        // pull's source, which must be a surface cell (up solid, outside or empty) when the pull
        // runs; a cell under water becomes one after pulls empty the cells above it, one pull per
        // cell. Cells with at most PEXPOSE water cells over them are counted; a deeper exposure
        // in one tick is caught when the pull runs (a conflict).
        P = cd_volume(c) < FULL ? 1u : 0u;
#pragma unroll
        for (int d = 1; d <= PEXPOSE + 1; ++d)
          if (!P && (cd_solid(col[d]) || cd_volume(col[d]) <= 0.0f)) P = 1u;
      }
    }
    unsigned trow, tp;
    const unsigned orow = cta_scan_count(sm, rowflag, &trow);
    const unsigned op = cta_scan_count(sm, P, &tp);
    const unsigned rows0 = s_rows, pc0 = s_pc;
    if (valid) {
      const unsigned row = rows0 + orow + rowflag - 1u;
      R.rowof[i] = row | (P << 31) | (S << 30);
      R.pcnt[i] = pc0 + op;
      if (rowflag) {
        R.rowstart[row] = i;
        R.rowprog[row] = 0u;
        R.zrow[(size_t)y * (unsigned)R.PZ + (unsigned)(z - R.pz0)] = row;
      }
    }
    __syncthreads();
    if (tid == 0) {
      s_rows += trow;
      s_pc += tp;
    }
    __syncthreads();
  }
  if (tid == 0) {
    R.rowstart[s_rows] = n;
    R.pcnt[n] = s_pc;
    R.ctl->ptn = 0u;
  }
  // earlier conflicting cells of every cell (the position map is complete now)
  for (unsigned i = tid; i < n; i += NT_) {  // one cell per thread: ten position loads in flight
    const unsigned cid = key_to_id(R, R.cells[i], flip);
    int x, y, z;
    dom_xyz(R, cid, x, y, z);
    unsigned d[16];
#pragma unroll
    for (unsigned l = 0; l < 10u; ++l) {
      int dx, dy, dz;
      dep_offset(l, flip, dx, dy, dz);
      const unsigned r = rank_at(R, x + dx, y + dy, z + dz);
      d[l] = r < i ? r : NOSLOT;
    }
#pragma unroll
    for (unsigned l = 10u; l < 16u; ++l) d[l] = NOSLOT;
    uint4* o = reinterpret_cast<uint4*>(R.deps + (size_t)i * 16u);
#pragma unroll
    for (int q = 0; q < 4; ++q) o[q] = make_uint4(d[4 * q], d[4 * q + 1], d[4 * q + 2], d[4 * q + 3]);
  }
  for (unsigned w = tid; w < (n + 3u) / 4u; w += NT_) ps.state[w] = 0u;
  for (unsigned w = tid; w < (n + 31u) / 32u; w += NT_) R.pextra[w] = 0u;
  if (tid == 0) R.ctl->pxn = 0u;
  for (unsigned t = tid; t < NPC_SMEM * PV_CAP; t += NT_) ps.pc[t / PV_CAP].vis[t % PV_CAP] = EMPTY_ID;
  if (tid == 0) ps.pc_free = ((tune.gate >> 21) & 1) ? 0u : (1u << NPC_SMEM) - 1u;  // bit 21: global contexts only
  __syncthreads();
  plap(0);
  // ---- budget segments
  __shared__ unsigned s_pos, s_c, s_end, s_mode, s_epoch, s_go, s_cap, s_split;
  if (tid == 0) {
    s_pos = 0;
    s_c = 0;
    s_cap = n;    // a segment split by a conflict ends here
    s_split = 0;  // splits of the current position so far
  }
  __syncthreads();
  const int gate = max(0, min(tune.gate & 0xFF, GATE_MAX));
  const int cone = (tune.gate >> 8) & 0xFF ? min((tune.gate >> 8) & 0xFF, GATE_MAX) : gate;
  __shared__ unsigned s_extra;
  // attempts per possible attempter over this tick's completed pull segments (the last tick's to
  // start with), for sizing the next segment
  __shared__ unsigned long long s_att_acc, s_p_acc;
  __shared__ unsigned s_pull_end, s_nseg;
  if (tid == 0) {
    s_att_acc = 0ull;
    s_p_acc = 0ull;
    s_pull_end = n;  // known once a segment overshot the budget: its room-th attempt's cell + 1
    s_nseg = 0;
  }
  while (true) {
    // cells at or after the position that earlier pulls took below full (not counted in pcnt)
    {
      const unsigned nx = min(__ldcg(&R.ctl->pxn), MAX_CELLS_PER_TICK);
      unsigned long long c = 0;
      for (unsigned q = tid; q < nx; q += NT_) c += __ldcg(R.pxlist + q) >= s_pos ? 1u : 0u;
      c = cta_sum(sm, c);
      if (tid == 0) s_extra = (unsigned)c;
    }
    if (tid == 0) {
      const unsigned pos = s_pos;
      s_go = pos < n ? 1u : 0u;
      if (s_go) {
        if (s_c >= MAX_PULLS_PER_TICK) {
          s_end = n;
          s_mode = PM_NOPULL;
        } else {
          float ratio = 1.0f;
          if (s_p_acc >= 256ull) ratio = (float)s_att_acc / (float)s_p_acc;
          else if (R.ctl->att_ratio) ratio = (float)R.ctl->att_ratio * (1.0f / 65536.0f);
          ratio = fminf(1.0f, fmaxf(ratio, 0.125f));
          // the tick's first segment stops short of the expected budget end; later ones reach past
          // it, so that an overshoot finds the exact end, after which one segment runs the rest
          // with pulls up to that end and none after it
          if (s_pull_end < n) s_end = n;
          else s_end = seg_end_for(R, pos, n, MAX_PULLS_PER_TICK - s_c, s_extra, ratio, s_nseg == 0u ? 0.9f : 1.25f);
          s_mode = PM_PULL;
        }
        s_end = min(s_end, max(s_cap, pos + 1u));
        // a position split too often runs its (short) segment in order on one warp
        if (s_split >= PAR_MAX_SPLITS) s_mode = PM_SEQ;
        unsigned ep = R.ctl->seg_epoch + 1u;
        if ((ep & 0xFFFFu) == 0u) ep += 1u;  // epoch 0 marks free version slots and unstamped reads
        R.ctl->seg_epoch = ep;
        s_epoch = ep;
        ps.next_task = R.rowof[pos] & 0x3FFFFFFFu;
        ps.task_end = R.rowof[s_end - 1u] & 0x3FFFFFFFu;
        ps.abort = 0u;
        ps.viol = 0u;
        ps.viol_pos = 0xFFFFFFFFu;
        ps.ticket = 0u;
        for (int w = 0; w < MAX_WARPS; ++w) ps.wrow[w] = WROW_IDLE;
        R.ctl->par_segments += 1ull;
      }
    }
    __syncthreads();
    if (!s_go) break;
    ParTick T;
    T.seg_start = s_pos;
    T.seg_end = s_end;
    T.pull_end = s_pull_end;
    T.epoch = s_epoch;
    T.gate = gate;
    T.cone = cone;
    T.flip = flip;
    T.spin_cap = tune.spin_cap;
    const int mode = (int)s_mode;
    unsigned seq_pulls = 0;
    if (mode == PM_SEQ) {
      // one warp, in sorted order, the budget counted exactly
      if (warp == 0) {
        unsigned sp = s_c;
        unsigned cgi = 0xFFFFFFFFu, cg = 0u;
        for (unsigned i = T.seg_start; i < T.seg_end; ++i) process_cell_par(R, ps, R.pcg[0], ring, T, PM_SEQ, i, sp, pf, NOSLOT, cgi, cg, NOSLOT, 0u, R.cells[i]);
        if (lane == 0) R.ctl->par_replayed += T.seg_end - T.seg_start;
      }
      __syncthreads();
      if (vld((const unsigned*)&R.ctl->status) != 0u) return;
    } else {
      // ---- row workers
      const long long w0 = clock64();
      while (true) {
        const long long f0 = clock64();
        unsigned t = 0;
        if (lane == 0) t = atomicAdd(&ps.next_task, 1u);
        t = __shfl_sync(FULLMASK, t, 0);
        if (t > ps.task_end) break;
        const unsigned rs = R.rowstart[t];
        const unsigned a = max(rs, T.seg_start), b = min(R.rowstart[t + 1u], T.seg_end);
        // publish the row and its next cell for cone_wait (key / PX = y * PZ + sorted z)
        const unsigned ka = R.cells[a];
        const unsigned yz = udiv(ka, (unsigned)R.PX, R.mx), yy = udiv(yz, (unsigned)R.PZ, R.mz), zs = yz - yy * (unsigned)R.PZ;
        const unsigned zr = flip ? (unsigned)R.PZ - 1u - zs : zs;
        const unsigned long long rowtag = ((unsigned long long)yy << 48) | ((unsigned long long)zr << 32);
        w_fetch += (unsigned long long)(clock64() - f0);
        bool ok = true;
        unsigned cgi = 0xFFFFFFFFu, cg = 0u;
        unsigned jr_next = R.deps[a * 16u + (lane & 15u)];
        unsigned key_next = ka;
        for (unsigned i = a; i < b && ok; ++i) {
          const unsigned jr = jr_next, key = key_next;
          if (i + 1u < b) {  // used by the next cell
            jr_next = R.deps[(i + 1u) * 16u + (lane & 15u)];
            key_next = R.cells[i + 1u];
          }
          if (lane == 0) *(volatile unsigned long long*)&ps.wrow[warp] = rowtag | (key - yz * (unsigned)R.PX);
          ok = process_cell_par(R, ps, R.pcg[warp], ring, T, mode, i, seq_pulls, pf, jr, cgi, cg, t, rs, key);
        }
        if (lane == 0) *(volatile unsigned long long*)&ps.wrow[warp] = WROW_IDLE;
        if (!ok || vld(&ps.abort)) break;
      }
      w_total += (unsigned long long)(clock64() - w0);
      __syncthreads();
      plap(1);
      if (vld((const unsigned*)&R.ctl->status) != 0u) return;  // a wait or a capacity ran out: the tick fails
      if (ps.viol) {
        // a conflict the schedule could not order at pull position k: undo the segment and run it
        // again up to k + 1 (the late reader is then outside it), the rest afterwards
        rollback_segment(R, ps, ring, T.seg_start, T.seg_end, flip);
        for (unsigned i = T.seg_start + tid; i < T.seg_end; i += NT_) atomicAnd(&ps.state[i >> 2], ~(0xFFu << ((i & 3u) * 8u)));
        const unsigned r0 = R.rowof[T.seg_start] & 0x3FFFFFFFu, r1 = R.rowof[T.seg_end - 1u] & 0x3FFFFFFFu;
        for (unsigned r = r0 + tid; r <= r1; r += NT_) {
          const unsigned st = R.rowstart[r];
          R.rowprog[r] = T.seg_start > st ? T.seg_start - st : 0u;
        }
        __syncthreads();
        plap(2);
        if (tid == 0) {
          R.ctl->par_rollbacks += 1ull;
          s_cap = min(ps.viol_pos, T.seg_end - 1u) + 1u;
          s_split += 1u;
        }
        __syncthreads();
        continue;
      }
    }
    // ---- attempts made in the segment (exact: every cell of it has finished)
    unsigned long long att = 0;
    for (unsigned i = T.seg_start + tid; i < T.seg_end; i += NT_) att += (R.rec[i].flags & RF_ATTEMPT) ? 1u : 0u;
    att = cta_sum(sm, att);
    const unsigned room = MAX_PULLS_PER_TICK - min(s_c, MAX_PULLS_PER_TICK);
    if (mode == PM_PULL && att > room) {
      // more cells attempted than the budget left (cells that pulls took below full beyond the
      // counted ones): the cells up to the room-th attempt were right. Undo the segment and run it
      // again up to that cell; the rest follows with the budget spent.
      __shared__ unsigned s_cut;
      if (tid == 0) s_cut = T.seg_end;
      __syncthreads();
      unsigned run = 0;
      for (unsigned base = T.seg_start; base < T.seg_end; base += NT_) {
        const unsigned i = base + tid;
        const unsigned f = (i < T.seg_end && (R.rec[i].flags & RF_ATTEMPT)) ? 1u : 0u;
        unsigned tot;
        const unsigned off = cta_scan_count(sm, f, &tot);
        if (f && run + off + 1u == room) s_cut = i + 1u;
        run += tot;
        __syncthreads();
        if (run >= room) break;
      }
      rollback_segment(R, ps, ring, T.seg_start, T.seg_end, flip);
      for (unsigned i = T.seg_start + tid; i < T.seg_end; i += NT_) atomicAnd(&ps.state[i >> 2], ~(0xFFu << ((i & 3u) * 8u)));
      const unsigned r0 = R.rowof[T.seg_start] & 0x3FFFFFFFu, r1 = R.rowof[T.seg_end - 1u] & 0x3FFFFFFFu;
      for (unsigned r = r0 + tid; r <= r1; r += NT_) {
        const unsigned st = R.rowstart[r];
        R.rowprog[r] = T.seg_start > st ? T.seg_start - st : 0u;
      }
      __syncthreads();
      if (tid == 0) {
        R.ctl->par_rollbacks += 1ull;
        R.ctl->par_conflicts[2] += 1ull;
        s_pull_end = s_cut;
        s_cap = n;
      }
      __syncthreads();
      continue;
    }
    if (tid == 0) {
      if (mode == PM_PULL) {
        s_att_acc += att;
        s_p_acc += R.pcnt[min(T.seg_end, T.pull_end)] - R.pcnt[T.seg_start];
        s_nseg += 1u;
      }
      s_c += (unsigned)att;
      s_pos = T.seg_end;
      s_cap = n;
      s_split = 0;
    }
    __syncthreads();
  }
  if (tid == 0 && s_p_acc >= 256ull) R.ctl->att_ratio = (unsigned)(65536.0 * (double)s_att_acc / (double)s_p_acc);
  if (lane == 0) {
    unsigned long long* q = R.ctl->pprof;
    atomicAdd(q + 4, pf.dep);
    atomicAdd(q + 5, pf.start);
    atomicAdd(q + 6, pf.load);
    atomicAdd(q + 7, pf.pull);
    atomicAdd(q + 8, pf.write);
    atomicAdd(q + 9, pf.cells);
    atomicAdd(q + 10, w_fetch);
    atomicAdd(q + 11, w_total);
    atomicAdd(q + 12, pf.cone);
    atomicAdd(q + 13, pf.gate);
    atomicAdd(q + 14, pf.npull);
    atomicAdd(q + 15, pf.rounds);
    atomicAdd(q + 16, pf.tread);
    atomicAdd(q + 17, pf.tpw);
  }
  tp0 = clock64();
  // ---- per-tick maps back to idle: positions, rows, pull-written cells
  for (unsigned i = tid; i < n; i += NT_) {
    const unsigned key = R.cells[i];
    const unsigned cid = key_to_id(R, key, flip);
    R.stamp[cid] = 0xFFFFFFFFu;
    if (i == 0u || udiv(key, (unsigned)R.PX, R.mx) != udiv(R.cells[i - 1u], (unsigned)R.PX, R.mx)) {
      int x, y, z;
      dom_xyz(R, cid, x, y, z);
      R.zrow[(size_t)y * (unsigned)R.PZ + (unsigned)(z - R.pz0)] = NOSLOT;
    }
  }
  {
    const unsigned np = min(R.ctl->ptn, MAX_PULLS_PER_TICK + 64u);
    for (unsigned t = tid; t < np; t += NT_) {
      const unsigned id = R.ptlist[t];
      atomicAnd(R.ptbits + (id >> 5), ~(1u << (id & 31u)));
    }
  }
  // ---- the records in sorted order -> the tick's event logs (program order) and counters
  __shared__ unsigned s_na, s_ns, s_nc;
  if (tid == 0) {
    s_na = 0;
    s_ns = 0;
    s_nc = 0;
  }
  __syncthreads();
  const unsigned pxy = (unsigned)R.PX * (unsigned)R.PY;
  const bool lr = sW.level_round;
  unsigned long long c_att = 0, c_succ = 0, c_ent = 0, c_chg = 0, c_pd = 0;
  for (unsigned base = 0; base < n; base += NT_) {
    const unsigned i = base + tid;
    unsigned am = 0, fl = 0, cm = 0, src = 0, cid = 0;
    if (i < n) {
      const CellRec& rc = R.rec[i];
      am = rc.amask;
      fl = rc.flags;
      cm = rc.cmask;
      src = rc.src;
      cid = key_to_id(R, R.cells[i], flip);
      c_att += (fl & RF_ATTEMPT) ? 1u : 0u;
      c_succ += (fl & RF_SUCCESS) ? 1u : 0u;
      c_ent += rc.entries;
      c_pd += (unsigned long long)(long long)rc.pdelta;
      c_chg |= (fl & RF_CHANGED) ? 1u : 0u;
    }
    const unsigned ns = lr ? 0u : (((fl & RF_SEED_SRC) ? 1u : 0u) + ((fl & RF_SEED_SELF) ? 1u : 0u));
    unsigned ta, ts, tc;
    const unsigned oa = cta_scan_count(sm, (unsigned)__popc(am), &ta);
    const unsigned os = cta_scan_count(sm, ns, &ts);
    const unsigned oc = cta_scan_count(sm, (unsigned)__popc(cm), &tc);
    if (i < n) {
      // activations: slot 0 the source (one cell), slots 1..7 wake_around centres
      unsigned pa = s_na + oa;
      for (int g = 0; g < 8; ++g) {
        if (!((am >> g) & 1u)) continue;
        unsigned w;
        switch (g) {
          case 0: w = src; break;
          case 2: w = (cid - (unsigned)R.PX) | ACT_AROUND; break;
          case 3: w = (cid + 1u) | ACT_AROUND; break;
          case 4: w = (cid - 1u) | ACT_AROUND; break;
          case 5: w = (cid + pxy) | ACT_AROUND; break;
          case 6: w = (cid - pxy) | ACT_AROUND; break;
          default: w = cid | ACT_AROUND; break;  // 1 and 7: the cell itself
        }
        if (pa < R.ev_act_cap) R.ev_act[pa] = w;
        else set_status(R, ST_OOM, 40);
        ++pa;
      }
      unsigned psd = s_ns + os;
      if (ns) {
        if (fl & RF_SEED_SRC) {
          if (psd < R.ev_seed_cap) R.ev_seed[psd] = src;
          else set_status(R, ST_OOM, 41);
          ++psd;
        }
        if (fl & RF_SEED_SELF) {
          if (psd < R.ev_seed_cap) R.ev_seed[psd] = cid;
          else set_status(R, ST_OOM, 41);
        }
      }
      unsigned pc = s_nc + oc;
      for (int l = 0; l < 8; ++l) {
        if (!((cm >> l) & 1u)) continue;
        unsigned id;
        switch (l) {
          case 0: id = cid; break;
          case 1: id = cid - (unsigned)R.PX; break;
          case 2: id = cid + (unsigned)R.PX; break;
          case 3: id = cid + 1u; break;
          case 4: id = cid - 1u; break;
          case 5: id = cid + pxy; break;
          case 6: id = cid - pxy; break;
          default: id = src; break;
        }
        if (pc < R.ev_chg_cap) R.ev_chg[pc] = id;
        else set_status(R, ST_OOM, 42);
        ++pc;
      }
    }
    __syncthreads();
    if (tid == 0) {
      s_na += ta;
      s_ns += ts;
      s_nc += tc;
    }
    __syncthreads();
  }
  c_att = cta_sum(sm, c_att);
  c_succ = cta_sum(sm, c_succ);
  c_ent = cta_sum(sm, c_ent);
  c_chg = cta_sum(sm, c_chg);
  c_pd = cta_sum(sm, c_pd);
  if (tid == 0) {
    sW.nact = s_na;
    sW.nseed = s_ns;
    sW.nchg = s_nc;
    sW.pull_attempts = c_att;
    sW.pull_success = c_succ;
    sW.bfs_visits = c_ent;
    sW.pdelta = (long long)c_pd;
    sW.changed = c_chg != 0;
  }
  __syncthreads();
  plap(3);
}

// ------------------------------------------------------------------ levelling, all warps
// LayerMarks probe without setting (mark_tas's tile and bit); cells outside the domain read as
// marked, as mark_tas treats them. Marks are set by atomics (in L2): read past L1.
__device__ __forceinline__ bool mark_test(const Region& R, int x, int y, int z) {
  if (!in_dom(R, x, y, z)) return true;
  const unsigned xr = (unsigned)(x - R.px0), zr = (unsigned)(z - R.pz0);
  const unsigned tile = ((zr >> 6) * (unsigned)R.PY + (unsigned)y) * (unsigned)R.TX + (xr >> 6);
  const unsigned bit = ((zr & 63u) << 6) | (xr & 63u);
  return (__ldcg(R.marks + (size_t)tile * 128u + (bit >> 5)) >> (bit & 31u)) & 1u;
}

// Exclusive prefix of a per-thread 64-bit value over the CTA (thread order); *total = the sum.
__device__ unsigned long long cta_scan_u64(unsigned long long v, unsigned long long* total) {
  __shared__ unsigned long long s_w[MAX_WARPS];
  const unsigned lane = threadIdx.x & 31u, warp = threadIdx.x >> 5;
  unsigned long long incl = v;
  for (int o = 1; o < 32; o <<= 1) {
    const unsigned long long u = __shfl_up_sync(FULLMASK, incl, o);
    if (lane >= (unsigned)o) incl += u;
  }
  if (lane == 31u) s_w[warp] = incl;
  __syncthreads();
  unsigned long long before = 0, all = 0;
  for (unsigned w = 0; w < NW_; ++w) {
    const unsigned long long t = s_w[w];
    if (w < warp) before += t;
    all += t;
  }
  __syncthreads();
  *total = all;
  return before + incl - v;
}

// The flood fill of FluidSim::level_layer (fluid.rs:425-446) continued from queue entry qs of qe,
// batch by batch over the CTA. The batch is every waiting entry; entry p's side d is tried in the
// reference's order p-major, d-minor: its rank 4(p - qs) + d claims the cell (the lowest rank is
// the reference's first test, which sets the mark; the others find it set), and the members are
// appended in rank order, so the queue is the reference's queue. A batch that could carry the
// queue to MAX_LEVEL_CELLS (where the reference stops expanding part-way) finishes on one warp.
// Returns the final length.
__device__ __noinline__ unsigned level_bfs_cta(const Region& R, TickSmem& sm, Smem& S, unsigned qs, unsigned qe) {
  __shared__ unsigned s_run, s_len;
  const unsigned tid = threadIdx.x;
  while (qs < qe) {
    const unsigned F = qe - qs;
    if ((unsigned long long)qe + 4ull * F >= MAX_LEVEL_CELLS) {
      if (tid < 32u) {
        unsigned i = qs;
        const unsigned len = level_bfs_warp(R, S, i, qe, 0xFFFFFFFFu);
        if (tid == 0) s_len = len;
      }
      __syncthreads();
      return s_len;
    }
    // claims
    for (unsigned t = tid; t < 4u * F; t += NT_) {
      int x, y, z, dx, dz;
      dom_xyz(R, R.lvl_id[qs + t / 4u], x, y, z);
      side4((int)(t & 3u), dx, dz);
      const int nx = x + dx, nz = z + dz;
      if (R.ring_w == 0 && (nx < 0 || nz < 0)) continue;
      if (!in_dom(R, nx, y, nz)) {  // cannot happen for neighbours of addressable cells
        set_status(R, ST_RANGE, 8);
        continue;
      }
      if (mark_test(R, nx, y, nz)) continue;
      atomicMin(R.rb + dom_id(R, nx, y, nz), t);
    }
    if (tid == 0) s_run = 0;
    __syncthreads();
    // the winners set the mark, test and append, in rank order
    for (unsigned base = 0; base < 4u * F; base += NT_) {
      const unsigned t = base + tid;
      unsigned f = 0, nid = 0;
      float v = 0.0f;
      if (t < 4u * F) {
        int x, y, z, dx, dz;
        dom_xyz(R, R.lvl_id[qs + t / 4u], x, y, z);
        side4((int)(t & 3u), dx, dz);
        const int nx = x + dx, nz = z + dz;
        if (!(R.ring_w == 0 && (nx < 0 || nz < 0)) && in_dom(R, nx, y, nz)) {
          nid = dom_id(R, nx, y, nz);
          if (__ldcg(R.rb + nid) == t) {  // set by atomics (in L2): read past L1
            R.rb[nid] = 0xFFFFFFFFu;
            unsigned tile;
            const unsigned listed = mark_begin(R, nx, y, nz, tile);  // unmarked: it won the claim
            f = level_member(R, S.ring, nx, y, nz, &v) ? 1u : 0u;
            mark_end(R, tile, listed);
          }
        }
      }
      unsigned tot;
      const unsigned off = cta_scan_count(sm, f, &tot);
      if (f) {
        R.lvl_id[qe + s_run + off] = nid;
        R.lvl_vol[qe + s_run + off] = v;
      }
      __syncthreads();
      if (tid == 0) s_run += tot;
      __syncthreads();
    }
    qs = qe;
    qe += s_run;
    __syncthreads();
  }
  return qe;
}

// A layer whose one-warp flood fill has this many entries waiting continues over the CTA.
constexpr unsigned LEVEL_HAND = 16;

// Minimum and maximum of a float over the CTA.
__device__ void cta_minmax(float& lo, float& hi) {
  __shared__ float s_lo[MAX_WARPS], s_hi[MAX_WARPS];
  for (int o = 16; o; o >>= 1) {
    lo = fminf(lo, __shfl_xor_sync(FULLMASK, lo, o));
    hi = fmaxf(hi, __shfl_xor_sync(FULLMASK, hi, o));
  }
  if ((threadIdx.x & 31u) == 0) {
    s_lo[threadIdx.x >> 5] = lo;
    s_hi[threadIdx.x >> 5] = hi;
  }
  __syncthreads();
  for (unsigned w = 0; w < NW_; ++w) {
    lo = fminf(lo, s_lo[w]);
    hi = fmaxf(hi, s_hi[w]);
  }
  __syncthreads();
}

// What FluidSim::level_layer does with a gathered layer of len cells (fluid.rs:430-485), over the
// CTA. The f64 sum in queue order is formed exactly whenever every partial sum is representable:
// all volumes are multiples of 2^L (L from the smallest, lo) and every partial sum is below
// len * hi < 2^H, so H - L <= 53 makes each f64 addition exact and the integer sum of v / 2^L is
// the reference's sum, in any order. Otherwise one thread adds in queue order. Levelling to the
// average writes each cell once, in parallel, the change log in cell order; the drain branch
// (`left` runs through the cells in order) and layers left as they are go to warp 0's
// level_finish.
__device__ __noinline__ void level_finish_cta(const Region& R, TickSmem& sm, WS& sW, Smem& S, unsigned len, unsigned long long cap) {
  __shared__ double s_sum;
  const unsigned tid = threadIdx.x;
  float lo = 2.0f, hi = -1.0f;
  for (unsigned k = tid; k < len; k += NT_) {
    const float v = R.lvl_vol[k];
    lo = fminf(lo, v);
    hi = fmaxf(hi, v);
  }
  cta_minmax(lo, hi);
  int el, eh;
  frexpf(lo, &el);
  frexp((double)len * (double)hi, &eh);
  const int L = el - 24;  // lo = m 2^el, m in [0.5, 1): its last mantissa bit is 2^(el - 24)
  double sum;
  if (lo >= 1.17549435e-38f && eh - L <= 53) {
    unsigned long long q = 0;
    for (unsigned k = tid; k < len; k += NT_) q += (unsigned long long)ldexp((double)R.lvl_vol[k], -L);
    sum = ldexp((double)cta_sum(sm, q), L);
  } else {
    if (tid == 0) {
      double a = 0.0;
      for (unsigned k = 0; k < len; ++k) a = __dadd_rn(a, (double)R.lvl_vol[k]);
      s_sum = a;
    }
    __syncthreads();
    sum = s_sum;
    __syncthreads();
  }
  const bool spread = len >= 2 && __fsub_rn(hi, lo) >= SLEEP;
  const float avg = spread ? __double2float_rn(__ddiv_rn(sum, (double)len)) : 0.0f;
  if (!spread || avg < MIN_SPREAD) {
    if (tid < 32u) {
      WS W = sW;
      W.pdelta = 0;
      const bool ch = level_finish(R, W, S, len, sum, lo, hi);
      long long pd = W.pdelta;
      for (int o = 16; o; o >>= 1) pd += __shfl_xor_sync(FULLMASK, pd, o);
      if (tid == 0) {
        W.pdelta = sW.pdelta + pd;
        W.changed |= ch;
        sW = W;
      }
      __syncwarp();
    }
    __syncthreads();
    return;
  }
  long long pd = 0;
  for (unsigned base = 0; base < len; base += NT_) {
    const unsigned k = base + tid;
    bool wv = false;
    int x = 0, y = 0, z = 0;
    unsigned id = 0;
    CD c = CD{0.0f, NOSLOT, 0u, 0, true};
    if (k < len) {
      id = R.lvl_id[k];
      dom_xyz(R, id, x, y, z);
      c = load_cell_par(R, S.ring, x, y, z, cap);
      wv = fabsf(__fsub_rn(cd_volume(c), avg)) > 1e-6f;
    }
    const bool need = wv && set_volume_needs_slot(c, avg);
    if (__any_sync(FULLMASK, need)) materialize_par(R, need, c.gi, c.slot, cap);
    bool ch = false;
    if (wv) {
      const SVPlan p = sv_plan(c, avg);
      if (c.slot != NOSLOT) sv_apply(R, c, x, y, z, p);
      ch = p.ch;
      pd += p.dp;
    }
    unsigned tot;
    const unsigned off = cta_scan(sm, ch, &tot);
    if (ch) {
      const unsigned pos = sW.nchg + off;
      if (pos < R.ev_chg_cap) R.ev_chg[pos] = id;
      else set_status(R, ST_OOM, 9);
    }
    __syncthreads();
    if (tid == 0) {
      sW.nchg += tot;
      if (tot) sW.changed = true;
    }
    __syncthreads();
  }
  const long long dp = (long long)cta_sum(sm, (unsigned long long)pd);
  if (tid == 0) {
    sW.pdelta += dp;
    sW.llc += len;
    sW.level_cells_total += len;
  }
  __syncthreads();
}

// FluidSim::level_surfaces (fluid.rs:489-507) from sW.llc on, over the CTA, in batches of up to one
// seed per thread (LIFO order = thread order). Every thread walks its seed up to the top water cell
// (fluid.rs:496-499) and tests the start: a start that is marked, repeats an earlier start of the
// batch, or is not a layer member needs no flood fill. Levelling a layer to its average changes no
// cell's solidity, its "vol > 0" or "supported", so these tests stay true while the batch's
// earlier layers are levelled; a drained layer (which can change them) ends the batch. The
// remaining starts, the candidates, are levelled in order (warp 0, handing grown layers to the
// CTA), each marked at its turn as the reference does; the budget (fluid.rs:492) ends the batch
// after the candidate that spends it. The popped seeds leave the seed set and their starts are
// marked (a start that is not a member is marked, and skipped by every later flood fill, either
// way). sW.level_round is updated at the end.
__device__ __noinline__ void level_round_cta(const Region& R, TickSmem& sm, WS& sW, Smem& S, unsigned long long cap) {
  __shared__ unsigned s_ns, s_stop, s_brk, s_pend, s_qi, s_ql, s_cur;
  const unsigned tid = threadIdx.x;
  unsigned* b_start = sm.hist;          // the batch's starts (domain ids), by seed
  unsigned* b_cand = sm.hist + NT_;     // candidate seeds in order
  while (true) {
    if (tid == 0) s_ns = (sW.llc < LEVEL_BUDGET) ? sW.nseeds : 0u;
    __syncthreads();
    const unsigned ns = s_ns;
    if (ns == 0u) break;
    const unsigned B = min(ns, NT_);
    // ---- starts and their tests, one seed per thread
    unsigned sid = 0;
    int x = 0, y = 0, z = 0;
    if (tid < B) {
      dom_xyz(R, R.seeds[ns - 1u - tid], x, y, z);
      while (true) {  // four cells of the column per step
        bool up[4];
#pragma unroll
        for (int q = 0; q < 4; ++q) {
          const int yy = y + 1 + q;
          up[q] = false;
          if (yy < R.ny) {
            const CD c = load_cell(R, S.ring, x, yy, z);
            up[q] = !cd_solid(c) && cd_volume(c) > 0.0f;
          }
        }
        const int steps = !up[0] ? 0 : !up[1] ? 1 : !up[2] ? 2 : !up[3] ? 3 : 4;
        y += steps;
        if (steps < 4) break;
      }
      sid = dom_id(R, x, y, z);
      b_start[tid] = sid;
      atomicMin(R.rb + sid, tid);
    }
    __syncthreads();
    const bool first = tid < B && __ldcg(R.rb + sid) == tid;  // set by atomics (in L2): read past L1
    __syncthreads();
    unsigned cand = 0, single = 0;
    if (first) {
      R.rb[sid] = 0xFFFFFFFFu;
      float v;
      cand = (!mark_test(R, x, y, z) && level_member(R, S.ring, x, y, z, &v)) ? 1u : 0u;
      // a start none of whose sides is an unmarked member is a layer of one cell: no flood fill
      // (marks only grow and membership holds through the batch, so this stays true)
      if (cand) {
        single = 1u;
        for (int d = 0; d < 4 && single; ++d) {
          int dx, dz;
          side4(d, dx, dz);
          const int nx = x + dx, nz = z + dz;
          if (R.ring_w == 0 && (nx < 0 || nz < 0)) continue;
          if (!mark_test(R, nx, y, nz) && level_member(R, S.ring, nx, y, nz, &v)) single = 0u;
        }
      }
    }
    unsigned nc;
    const unsigned off = cta_scan_count(sm, cand, &nc);
    if (cand) b_cand[off] = tid | (single << 31);
    if (tid == 0) {
      s_stop = B;
      s_brk = 0;
      s_cur = 0;  // the next candidate to level
    }
    __syncthreads();
    // ---- the candidates in order. One-cell layers only count (fluid.rs:446, len < 2); a start
    // that an earlier layer's flood fill marked is skipped, as its test_and_set would return
    // (entry bits: 31 one cell, 30 marked since the batch began, 0-29 the seed)
    while (true) {
      if (tid == 0) {
        unsigned c = s_cur;
        while (c < nc && (b_cand[c] >> 30)) {
          if (b_cand[c] >> 31) {
            sW.llc += 1u;
            sW.level_cells_total += 1u;
            if (sW.llc >= LEVEL_BUDGET) {
              s_stop = (b_cand[c] & 0x3FFFFFFFu) + 1u;
              s_brk = 1u;
            }
          }
          ++c;
          if (s_brk) break;
        }
        s_cur = c;
      }
      __syncthreads();
      if (s_brk || s_cur >= nc) break;
      const unsigned cur = s_cur;
      const unsigned j = b_cand[cur];
      if (tid < 32u) {
        WS W = sW;
        W.pdelta = 0;
        int cx, cy, cz;
        dom_xyz(R, b_start[j], cx, cy, cz);
        unsigned qi = 0, ql = 0;
        const bool pend = level_layer(R, W, S, cx, cy, cz, LEVEL_HAND, qi, ql);
        long long pd = W.pdelta;
        for (int o = 16; o; o >>= 1) pd += __shfl_xor_sync(FULLMASK, pd, o);
        if (tid == 0) {
          W.pdelta = sW.pdelta + pd;
          sW = W;
          s_pend = pend ? 1u : 0u;
          s_qi = qi;
          s_ql = ql;
        }
        __syncwarp();
      }
      __syncthreads();
      if (s_pend) {
        const unsigned len = level_bfs_cta(R, sm, S, s_qi, s_ql);
        level_finish_cta(R, sm, sW, S, len, cap);
      }
      // the later candidates this layer's flood fill marked
      for (unsigned c = cur + 1u + tid; c < nc; c += NT_) {
        const unsigned e = b_cand[c];
        if (e >> 30) continue;
        int cx, cy, cz;
        dom_xyz(R, b_start[e], cx, cy, cz);
        if (mark_test(R, cx, cy, cz)) b_cand[c] = e | (1u << 30);
      }
      if (tid == 0) {
        if (sW.llc >= LEVEL_BUDGET || sW.ndrain != 0u) {
          s_stop = j + 1u;
          s_brk = 1u;
        }
        s_cur += 1u;
      }
      __syncthreads();
      if (s_brk) break;
    }
    // ---- the popped seeds: out of the seed set, starts marked (and the sides a one-cell layer's
    // flood fill tested)
    const unsigned stop = s_stop;
    if (tid < stop) {
      const unsigned k = R.seeds[ns - 1u - tid];
      atomicAnd(&R.seedbits[k >> 5], ~(1u << (k & 31u)));
      int sx, sy, sz;
      dom_xyz(R, b_start[tid], sx, sy, sz);
      mark_tas(R, sx, sy, sz);
      if (single) {
        for (int d = 0; d < 4; ++d) {
          int dx, dz;
          side4(d, dx, dz);
          const int nx = sx + dx, nz = sz + dz;
          if (R.ring_w == 0 && (nx < 0 || nz < 0)) continue;
          if (in_dom(R, nx, sy, nz)) mark_tas(R, nx, sy, nz);
        }
      }
    }
    __syncthreads();
    if (tid == 0) {
      sW.nseeds = ns - stop;
      sW.ndrain = 0u;
    }
    __syncthreads();
  }
  if (tid == 0) sW.level_round = sW.nseeds != 0u;
  __syncthreads();
}

// FluidSim::tick (fluid.rs:564-657) for region R, n_ticks times. All threads of the CTA enter.
// Per tick: drain the FIFO head and sort it (CTA), the sweep (warp 0, prefetched by the other
// warps), the seed log's commit, levelling (warp 0), then the activation and change logs'
// commits (CTA). The logs keep program order, so the committed FIFO and seed list are exactly
// the reference's.
__device__ void run_ticks(const Region& R, TickSmem& sm, int n_ticks, Tune tune) {
  const unsigned tid = threadIdx.x, warp = tid >> 5;
  const int* ring = R.ring;
  if (R.ring_w && R.ring_w <= 16) {
    for (int i = tid; i < 3 * R.ring_w * R.ring_w; i += NT_) sm.ring[i] = R.ring[i];
    ring = sm.ring;
  }
  const bool par = tune.engine != 0;
  if (!par) {
    for (unsigned i = tid; i < VIS_CAP; i += NT_) sm.u.s.vis[i] = 0ull;
    for (unsigned i = tid; i < VB_WORDS; i += NT_) sm.u.s.vb[i] = 0u;
    for (unsigned i = tid; i < HRING; i += NT_) sm.u.s.help.tag[i] = ~0ull;
    if (tid == 0) {
      sm.u.s.help.state = 0ull;
      sm.u.s.help.qlen = sm.u.s.help.done = 0u;
    }
  }
  __shared__ unsigned s_n, s_flip, s_clear, s_abort, s_nseeds, s_lv;
  __shared__ unsigned long long s_qtail;
  __shared__ WS sW;
  if (tid == 0) {
    load_ws(R, sW);
    sW.deferred = true;
    s_abort = R.ctl->status != 0;
    s_clear = 0;
  }
  __syncthreads();
  long long tp = clock64();
  auto lap = [&](int k) {
    if (tid == 0) {
      long long now = clock64();
      R.ctl->prof[k] += (unsigned long long)(now - tp);
      tp = now;
    }
  };
  for (int t = 0; t < n_ticks; ++t) {
    if (s_abort) break;
    lap(15);
    // ---- drain the FIFO head (fluid.rs:565-572)
    if (tid == 0) {
      unsigned tick = R.ctl->tick_no + 1u;
      R.ctl->tick_no = tick;
      unsigned long long len = sW.qtail - sW.qhead;
      s_n = (unsigned)min(len, (unsigned long long)MAX_CELLS_PER_TICK);
      s_flip = tick & 1u;
    }
    __syncthreads();
    const unsigned n = s_n;
    const bool flip = s_flip != 0;
    const unsigned long long qh = sW.qhead;
    const unsigned tick_now = R.ctl->tick_no;
    for (unsigned i = tid; i < n; i += NT_) {
      unsigned id = R.queue[(qh + i) & R.qmask];
      atomicAnd(&R.active[id >> 5], ~(1u << (id & 31)));
      R.cells[i] = sort_key(R, id, flip);
      // wake history of materialised bricks (training labels of the wake proposal)
      int x, y, z;
      dom_xyz(R, id, x, y, z);
      if (!outside(R, ring, x, y, z)) {
        unsigned g = R.grid[grid_index(R, x >> 3, y >> 3, z >> 3)];
        if (g >= 256u) R.last_woken[g - 256u] = tick_now;
      }
    }
    __syncthreads();
    if (tid == 0) {
      sW.qhead = qh + n;
      sW.pulls = 0;
      sW.changed = false;
      sW.activations = sW.pull_attempts = sW.pull_success = sW.bfs_visits = sW.level_cells_total = 0;
      sW.pdelta = 0;
      sW.nact = sW.nseed = sW.nchg = 0;
    }
    __syncthreads();
    // ---- ring worlds: a drained cell of an evicted chunk is solid (outside), and the sweep erases its
    // partial entry (fluid.rs:586-589); entries kept for evicted chunks are erased here, which nothing
    // in the tick can tell apart (an outside cell's volume reads 0)
    if (R.detbits && vld(&R.ctl->ndetached) != 0u) {
      unsigned long long er = 0;
      for (unsigned i = tid; i < n; i += NT_) {
        const unsigned id = R.queue[(qh + i) & R.qmask];
        int x, y, z;
        dom_xyz(R, id, x, y, z);
        if (!outside(R, ring, x, y, z)) continue;
        const unsigned bit = 1u << (id & 31u);
        if (atomicAnd(R.detbits + (id >> 5), ~bit) & bit) ++er;
      }
      er = cta_sum(sm, er);
      if (tid == 0) {
        R.ctl->partial_count -= (long long)er;
        R.ctl->ndetached -= (unsigned)er;
      }
      __syncthreads();
    }
    lap(0);
    // ---- sort (fluid.rs:575-580)
    cta_radix_sort(R.cells, R.cells_tmp, n, sm.hist, sm.sred);
    __syncthreads();
    lap(1);
    // ---- the sweep (fluid.rs:584-651)
    if (par) sweep_parallel(R, sm, sW, ring, n, flip, tune);
    else sweep(R, sm, sW, ring, n, flip, tune);
    lap(2);
    if (par ? vld((const unsigned*)&R.ctl->status) != 0u : sm.u.s.abort != 0u) {
      if (tid == 0) s_abort = 1;
      __syncthreads();
      break;
    }
    // ---- level seeds logged by the sweep (fluid.rs:312-316)
    if (tid == 0) s_nseeds = sW.nseeds;
    __syncthreads();
    unsigned nseeds = s_nseeds;
    commit_seeds(R, sm, min(sW.nseed, R.ev_seed_cap), nseeds);
    if (tid == 0) sW.nseeds = nseeds;
    __syncthreads();
    lap(7);
    // ---- levelling (fluid.rs:652-655)
    if (tid == 0) s_lv = (sW.level_round || (R.ctl->tick_no % LEVEL_TICKS) == 0u) ? 1u : 0u;
    __syncthreads();
    if (s_lv) {
      Smem S{sm.u.s.vis, ring, sm.u.s.pq, sm.u.s.vb, sm.u.s.vtl, nullptr, nullptr, tune.spin_cap};
      if (tid == 0) sW.llc = 0;
      __syncthreads();
      level_round_cta(R, sm, sW, S, tune.spin_cap);
      if (tid == 0) s_clear = sW.level_round ? 0u : 1u;
    }
    __syncthreads();
    lap(8);
    // ---- FIFO appends and voxel changes logged during the tick
    if (tid == 0) s_qtail = sW.qtail;
    __syncthreads();
    unsigned long long qt = s_qtail;
    commit_acts(R, sm, min(sW.nact, R.ev_act_cap), qt, sW.qhead);
    lap(9);
    commit_chgs(R, min(sW.nchg, R.ev_chg_cap));
    lap(10);
    if (tid == 0) {
      Ctl& c = *R.ctl;
      c.activations += qt - s_qtail;
      sW.qtail = qt;
      c.last_cells = n;
      c.cells_total += n;
      c.pull_attempts += sW.pull_attempts;
      c.pull_success += sW.pull_success;
      c.bfs_visits += sW.bfs_visits;
      c.level_cells_total += sW.level_cells_total;
      c.partial_count += sW.pdelta;
      c.last_level_cells = sW.llc;
      c.nseeds = sW.nseeds;
      c.level_round = sW.level_round ? 1u : 0u;
      if (sW.changed) c.changed = 1u;
      c.qhead = sW.qhead;
      c.qtail = sW.qtail;
      s_abort = c.status != 0;
    }
    __syncthreads();
    // ---- end of a levelling round: clear the marks it touched (fluid.rs:503-505)
    if (s_clear) {
      const unsigned nt = R.ctl->mark_ntiles;
      for (unsigned k = warp; k < nt; k += NW_) {
        unsigned tile = R.mark_list[k];
        for (unsigned w = lane_id(); w < 128; w += 32) R.marks[(size_t)tile * 128u + w] = 0u;
        if (lane_id() == 0) R.mark_tflag[tile] = 0u;
      }
      __syncthreads();
      if (tid == 0) {
        R.ctl->mark_ntiles = 0;
        s_clear = 0;
      }
      __syncthreads();
    }
    lap(11);
  }
}

// One CTA per region. k_tick runs the one-warp sweep (TICK_THREADS per CTA), k_tick_par the
// parallel sweep (PAR_THREADS per CTA).
__global__ void __launch_bounds__(TICK_THREADS, 1) k_tick(Region* regs, int nreg, int n_ticks, Tune tune) {
  extern __shared__ __align__(16) unsigned char smraw[];
  TickSmem& sm = *reinterpret_cast<TickSmem*>(smraw);
  tune.engine = 0;
  __shared__ Region s_reg;  // the region's constants, as in k_tick_par
  for (int r = blockIdx.x; r < nreg; r += gridDim.x) {
    if (threadIdx.x == 0) s_reg = regs[r];
    __syncthreads();
    run_ticks(s_reg, sm, n_ticks, tune);
    __syncthreads();
  }
}

__global__ void __launch_bounds__(PAR_THREADS, 1) k_tick_par(Region* regs, int nreg, int n_ticks, Tune tune) {
  extern __shared__ __align__(16) unsigned char smraw[];
  TickSmem& sm = *reinterpret_cast<TickSmem*>(smraw);
  tune.engine = 1;
  // The region's constants (sizes, array bases) are read on every cell of the sweep: a copy in
  // shared memory keeps them off the L1, which the sweep's records and atlas lines stream through.
  __shared__ Region s_reg;
  for (int r = blockIdx.x; r < nreg; r += gridDim.x) {
    if (threadIdx.x == 0) s_reg = regs[r];
    __syncthreads();
    run_ticks(s_reg, sm, n_ticks, tune);
    __syncthreads();
  }
}

// -------------------------------------------------------------------------- host edits
// Activate a box in z, y, x order (FluidSim::wake, fluid.rs:358-366). One CTA; ordered by a
// CTA-wide exclusive scan per chunk of cells.
__global__ void __launch_bounds__(1024) k_wake_box(Region R, int x0, int y0, int z0, int x1, int y1, int z1) {
  __shared__ unsigned warp_cnt[32];
  __shared__ unsigned long long s_tail;
  const unsigned tid = threadIdx.x, lane = tid & 31u, warp = tid >> 5;
  if (tid == 0) s_tail = R.ctl->qtail;
  __syncthreads();
  const long long sx = (long long)x1 - x0 + 1, sy = (long long)y1 - y0 + 1, sz = (long long)z1 - z0 + 1;
  if (sx <= 0 || sy <= 0 || sz <= 0) return;
  const long long total = sx * sy * sz;
  for (long long base = 0; base < total; base += 1024) {
    long long t = base + tid;
    bool isnew = false;
    unsigned id = 0;
    if (t < total) {
      long long xx = t % sx, rest = t / sx;
      int x = x0 + (int)xx, y = y0 + (int)(rest % sy), z = z0 + (int)(rest / sy);
      if (y >= 0) {
        if (!in_dom(R, x, y, z)) {
          if (atomicCAS(&R.ctl->status, 0, ST_RANGE) == 0) R.ctl->err_info = 5;
        } else {
          id = dom_id(R, x, y, z);
          isnew = !((R.active[id >> 5] >> (id & 31)) & 1u);
        }
      }
    }
    unsigned b = __ballot_sync(FULLMASK, isnew);
    if (lane == 0) warp_cnt[warp] = __popc(b);
    __syncthreads();
    unsigned before = 0, all = 0;
    for (int w = 0; w < 32; ++w) {
      unsigned c = warp_cnt[w];
      if ((unsigned)w < warp) before += c;
      all += c;
    }
    if (isnew) {
      unsigned long long pos = s_tail + before + __popc(b & lanemask_lt());
      R.queue[pos & R.qmask] = id;
      atomicOr(&R.active[id >> 5], 1u << (id & 31));
    }
    __syncthreads();
    if (tid == 0) {
      s_tail += all;
      R.ctl->activations += all;
    }
    __syncthreads();
  }
  if (tid == 0) {
    R.ctl->qtail = s_tail;
    if (s_tail - R.ctl->qhead > R.qmask + 1ull) atomicCAS(&R.ctl->status, 0, ST_OOM);
  }
}

// A single warp running sequential host edits with the tick's device rules.
struct EditSmem {
  unsigned pq[8];
  unsigned long long vis[8];
  int ring[3 * 16 * 16];
};

__device__ const int* edit_ring(const Region& R, int* smring) {
  if (R.ring_w && R.ring_w <= 16) {
    for (int i = lane_id(); i < 3 * R.ring_w * R.ring_w; i += 32) smring[i] = R.ring[i];
    __syncwarp();
    return smring;
  }
  return R.ring;
}

__device__ void commit_ws(const Region& R, WS& W) {
  long long pd = W.pdelta;
  for (int o = 16; o; o >>= 1) pd += __shfl_xor_sync(FULLMASK, pd, o);
  if (lane_id() == 0) {
    Ctl& c = *R.ctl;
    c.partial_count += pd;
    c.qtail = W.qtail;
    c.activations += W.activations;
    c.nseeds = W.nseeds;
    if (W.changed) c.changed = 1u;
  }
  __syncwarp();
}

__device__ void wake_box_warp(const Region& R, WS& W, int x0, int y0, int z0, int x1, int y1, int z1) {
  // small boxes (displace's 3^3): z, y, x order, 32 cells per round
  int sx = x1 - x0 + 1, sy = y1 - y0 + 1, sz = z1 - z0 + 1;
  int total = sx * sy * sz;
  for (int base = 0; base < total; base += 32) {
    int t = base + (int)lane_id();
    bool v = t < total;
    int x = 0, y = 0, z = 0;
    if (v) {
      x = x0 + t % sx;
      y = y0 + (t / sx) % sy;
      z = z0 + t / (sx * sy);
    }
    activate_round(R, W, v, x, y, z);
  }
}

// FluidSim::displace (fluid.rs:370-408), warp-uniform.
__device__ void displace_warp(const Region& R, WS& W, const int* ring, int x, int y, int z) {
  const unsigned lane = lane_id();
  CD c = load_cell(R, ring, x, y, z);  // all lanes same cell
  float amount = cd_volume(c);
  if (lane == 0) erase_part(R, c, local_index(x, y, z), W.pdelta);
  __syncwarp();
  wake_box_warp(R, W, x - 1, y - 1, z - 1, x + 1, y + 1, z + 1);
  if (amount <= 0.0f) return;
  int yy = y + 1;
  while (yy < R.ny && amount > 1e-6f) {
    CD u = load_cell(R, ring, x, yy, z);
    if (cd_solid(u)) break;
    float cur = cd_volume(u);
    float take = fminf(amount, __fsub_rn(1.0f, cur));
    if (take > 0.0f) {
      W.changed |= warp_set_volume(R, W, lane == 0, u, x, yy, z, __fadd_rn(cur, take));
      amount = __fsub_rn(amount, take);
      activate_round(R, W, lane == 0, x, yy, z);
    }
    yy += 1;
  }
  for (int d = 0; d < 4; ++d) {
    if (amount <= 1e-6f) break;
    int dx, dz;
    side4(d, dx, dz);
    int nx = x + dx, nz = z + dz;
    CD s = load_cell(R, ring, nx, y, nz);
    if (cd_solid(s)) continue;
    float cur = cd_volume(s);
    float take = fminf(amount, __fsub_rn(1.0f, cur));
    if (take > 0.0f) {
      W.changed |= warp_set_volume(R, W, lane == 0, s, nx, y, nz, __fadd_rn(cur, take));
      amount = __fsub_rn(amount, take);
      activate_round(R, W, lane == 0, nx, y, nz);
    }
  }
}

__device__ void set_voxel_warp(const Region& R, const int* ring, int x, int y, int z, unsigned char m) {
  // SparseVolume::set_voxel (sparse_volume.rs:268-293) on the device mirror, lane 0.
  const unsigned lane = lane_id();
  CD c = load_cell(R, ring, x, y, z);
  if (c.out) return;  // set_voxel ignores cells that are not inside
  bool need = lane == 0 && c.slot == NOSLOT && c.mat != m;
  materialize_lanes(R, need, c.gi, c.slot);
  if (lane == 0 && c.mat != m && c.slot != NOSLOT) {
    R.amat[(size_t)c.slot * 512u + local_index(x, y, z)] = m;
    record_change(R, dom_id(R, x, y, z));
  }
  __syncwarp();
}

enum EditKind { ED_DISPLACE = 1, ED_BRUSH = 2, ED_EMIT = 3, ED_SET_PARTIAL = 4, ED_VOXELS = 5 };

// kind/args: ED_DISPLACE: xyz[0..3]; ED_BRUSH: n cells, m; ED_EMIT: n cells, amount;
// ED_SET_PARTIAL: xyz[0..3], amount; ED_VOXELS: n (x,y,z,m) quads.
__global__ void __launch_bounds__(32) k_edit(Region R, int kind, const int* xyz, unsigned long long n, int m, float amount,
                                             unsigned long long* out_count) {
  __shared__ EditSmem es;
  const unsigned lane = lane_id();
  const int* ring = edit_ring(R, es.ring);
  WS W;
  load_ws(R, W);
  unsigned long long cnt = 0;
  if (kind == ED_DISPLACE) {
    displace_warp(R, W, ring, xyz[0], xyz[1], xyz[2]);
  } else if (kind == ED_BRUSH) {
    // apply_brush (src/edit/brush.rs:93-111) with displace as on_water
    for (unsigned long long i = 0; i < n; ++i) {
      int x = xyz[3 * i], y = xyz[3 * i + 1], z = xyz[3 * i + 2];
      CD c = load_cell(R, ring, x, y, z);
      if (c.out) continue;  // in_brush_world (brush.rs:82-87)
      bool empty = c.mat == 0 || c.mat == WATER;
      if ((m == 0) == empty) continue;
      if (c.mat == WATER) displace_warp(R, W, ring, x, y, z);
      set_voxel_warp(R, ring, x, y, z, (unsigned char)m);
      ++cnt;
    }
  } else if (kind == ED_EMIT) {
    for (unsigned long long i = 0; i < n; ++i) {
      int x = xyz[3 * i], y = xyz[3 * i + 1], z = xyz[3 * i + 2];
      CD c = load_cell(R, ring, x, y, z);
      if (cd_solid(c)) continue;
      float nv = fminf(1.0f, __fadd_rn(cd_volume(c), amount));
      W.changed |= warp_set_volume(R, W, lane == 0, c, x, y, z, nv);
      activate_round(R, W, lane == 0, x, y, z);
    }
  } else if (kind == ED_SET_PARTIAL) {
    // FluidSim::set_partial (fluid.rs:278-282): PartialField::set only, voxel untouched
    int x = xyz[0], y = xyz[1], z = xyz[2];
    if (amount > 0.0f && amount < 1.0f) {
      CD c = load_cell(R, ring, x, y, z);
      if (c.out) {
        if (lane == 0 && atomicCAS(&R.ctl->status, 0, ST_RANGE) == 0) R.ctl->err_info = 6;
      } else {
        bool need = lane == 0 && c.slot == NOSLOT;
        materialize_lanes(R, need, c.gi, c.slot);
        if (lane == 0 && c.slot != NOSLOT) {
          if (!(c.part > 0.0f)) W.pdelta += 1;
          R.avol[(size_t)c.slot * 512u + local_index(x, y, z)] = amount;
        }
      }
    }
  } else if (kind == ED_VOXELS) {
    for (unsigned long long i = 0; i < n; ++i) {
      int x = xyz[4 * i], y = xyz[4 * i + 1], z = xyz[4 * i + 2];
      set_voxel_warp(R, ring, x, y, z, (unsigned char)xyz[4 * i + 3]);
    }
  }
  if (W.qtail - W.qhead > R.qmask + 1ull) set_status(R, ST_OOM, 7);
  commit_ws(R, W);
  if (lane == 0 && out_count) *out_count = cnt;
}

// ------------------------------------------------------------------------- inspection
__device__ __forceinline__ unsigned long long cell_hash(int x, int y, int z, unsigned m, unsigned vb) {
  return fmix64(ref_key(x, y, z) * 0x9E3779B97F4A7C15ULL + (((unsigned long long)m << 32) | vb));
}

// Sum over cells with (material, partial bits) != (0, 0) of cell_hash; one thread per voxel.
__global__ void k_state_digest(Region R, unsigned long long* out) {
  const unsigned long long nb = (unsigned long long)R.bx * R.by * R.bz;
  unsigned long long acc = 0;
  for (unsigned long long t = blockIdx.x * (unsigned long long)blockDim.x + threadIdx.x; t < nb * 512ull;
       t += (unsigned long long)gridDim.x * blockDim.x) {
    unsigned long long gi = t >> 9;
    unsigned l = (unsigned)(t & 511u);
    int bx = (int)(gi % R.bx), by = (int)((gi / R.bx) % R.by), bz = (int)(gi / ((unsigned long long)R.bx * R.by));
    int ax = bx, az = bz;
    if (R.ring_w) {
      const int* s = R.ring + 3 * ((bz / 16) * R.ring_w + (bx / 16));
      if (!s[2]) continue;
      ax = s[0] * 16 + bx % 16;
      az = s[1] * 16 + bz % 16;
    }
    int x = ax * 8 + (int)(l & 7u), y = by * 8 + (int)((l >> 3) & 7u), z = az * 8 + (int)(l >> 6);
    if (y >= R.ny) continue;
    unsigned g = R.grid[gi];
    unsigned m;
    float p = 0.0f;
    if (g < 256u) {
      m = g;
    } else {
      // atlas local index == voxel index here (x|y<<3|z<<6 with l's bit layout)
      m = R.amat[(size_t)(g - 256u) * 512u + l];
      p = R.avol[(size_t)(g - 256u) * 512u + l];
    }
    unsigned vb = __float_as_uint(p);
    if (m == 0 && vb == 0) continue;
    acc += cell_hash(x, y, z, m, vb);
  }
  for (int o = 16; o; o >>= 1) acc += __shfl_xor_sync(FULLMASK, acc, o);
  if ((threadIdx.x & 31u) == 0) atomicAdd(out, acc);
}

// Partial entries kept for evicted ring chunks (x, y, z, volume bits, cell id per entry) whose cell
// still has its detbits bit: hashed like cells outside the loaded chunks (material 0).
__global__ void k_detached_digest(Region R, const int4* ent, const unsigned* ids, unsigned n, unsigned long long* out) {
  unsigned long long acc = 0;
  for (unsigned i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const unsigned id = ids[i];
    if (!((R.detbits[id >> 5] >> (id & 31u)) & 1u)) continue;
    const int4 e = ent[i];
    acc += cell_hash(e.x, e.y, e.z, 0u, (unsigned)e.w);
  }
  for (int o = 16; o; o >>= 1) acc += __shfl_xor_sync(FULLMASK, acc, o);
  if ((threadIdx.x & 31u) == 0) atomicAdd(out, acc);
}

// Ring paste/evict helpers: gather the partial volumes of atlas slots; write whole bricks (materials
// and volumes) into slots; set, clear or read bits of cells.
__global__ void k_gather_vol(const float* avol, const unsigned* slots, unsigned n, float* out) {
  for (unsigned t = blockIdx.x * blockDim.x + threadIdx.x; t < n * 512u; t += gridDim.x * blockDim.x)
    out[t] = avol[(size_t)slots[t >> 9] * 512u + (t & 511u)];
}
__global__ void k_scatter_bricks(unsigned char* amat, float* avol, const unsigned* slots, unsigned n, const unsigned char* mats,
                                 const float* vols) {
  for (unsigned t = blockIdx.x * blockDim.x + threadIdx.x; t < n * 512u; t += gridDim.x * blockDim.x) {
    const size_t o = (size_t)slots[t >> 9] * 512u + (t & 511u);
    amat[o] = mats[t];
    avol[o] = vols[t];
  }
}
// op 0: clear, 1: set, 2: read into out
__global__ void k_cell_bits(unsigned* bits, const unsigned* ids, unsigned n, int op, unsigned* out) {
  for (unsigned i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const unsigned id = ids[i], bit = 1u << (id & 31u);
    if (op == 0) atomicAnd(bits + (id >> 5), ~bit);
    else if (op == 1) atomicOr(bits + (id >> 5), bit);
    else out[i] = (bits[id >> 5] & bit) ? 1u : 0u;
  }
}

// Order-dependent digest of a list of domain ids: sum fmix64(ref_key * golden + position).
__global__ void k_list_digest(Region R, const unsigned* ids, unsigned long long n, unsigned long long head, unsigned long long mask,
                              unsigned long long* out) {
  unsigned long long acc = 0;
  for (unsigned long long i = blockIdx.x * (unsigned long long)blockDim.x + threadIdx.x; i < n; i += (unsigned long long)gridDim.x * blockDim.x) {
    unsigned id = ids[(head + i) & mask];
    int x, y, z;
    dom_xyz(R, id, x, y, z);
    acc += fmix64(ref_key(x, y, z) * 0x9E3779B97F4A7C15ULL + i);
  }
  for (int o = 16; o; o >>= 1) acc += __shfl_xor_sync(FULLMASK, acc, o);
  if ((threadIdx.x & 31u) == 0) atomicAdd(out, acc);
}

__global__ void k_export_box(Region R, int x0, int y0, int z0, int sx, int sy, int sz, unsigned char* mat, float* part) {
  const unsigned long long total = (unsigned long long)sx * sy * sz;
  for (unsigned long long t = blockIdx.x * (unsigned long long)blockDim.x + threadIdx.x; t < total; t += (unsigned long long)gridDim.x * blockDim.x) {
    int x = x0 + (int)(t % sx), y = y0 + (int)((t / sx) % sy), z = z0 + (int)(t / ((unsigned long long)sx * sy));
    CD c = load_cell(R, R.ring, x, y, z);
    // get_voxel reads 0 outside (sparse_volume.rs:238-241); partials of outside cells are none
    if (mat) mat[t] = c.out ? 0 : c.mat;
    if (part) part[t] = c.out ? 0.0f : c.part;
  }
}

// Gather pending voxel changes (final material) for the host and clear their bits.
struct Voxel {
  int x, y, z;
  unsigned char m, pad[3];
};
__global__ void k_gather_changes(Region R, unsigned long long n, Voxel* out) {
  for (unsigned long long i = blockIdx.x * (unsigned long long)blockDim.x + threadIdx.x; i < n; i += (unsigned long long)gridDim.x * blockDim.x) {
    unsigned id = R.chg[i];
    int x, y, z;
    dom_xyz(R, id, x, y, z);
    CD c = load_cell(R, R.ring, x, y, z);
    Voxel v;
    v.x = x;
    v.y = y;
    v.z = z;
    v.m = c.mat;
    v.pad[0] = v.pad[1] = v.pad[2] = 0;
    out[i] = v;
    atomicAnd(&R.chgbits[id >> 5], ~(1u << (id & 31)));
  }
}

// Partial entries of every atlas slot, compacted (ascending slot, voxel index order).
__global__ void k_export_partials(Region R, unsigned nslots, int* xyz, float* vol, unsigned long long cap, unsigned long long* count,
                                  const int* slot_brick /* slot -> grid index */) {
  for (unsigned long long t = blockIdx.x * (unsigned long long)blockDim.x + threadIdx.x; t < (unsigned long long)nslots * 512ull;
       t += (unsigned long long)gridDim.x * blockDim.x) {
    unsigned s = (unsigned)(t >> 9), l = (unsigned)(t & 511u);
    float p = R.avol[t];
    if (!(p > 0.0f)) continue;
    int gi = slot_brick[s];
    if (gi < 0) continue;
    int bx = gi % R.bx, by = (gi / R.bx) % R.by, bz = gi / (R.bx * R.by);
    int ax = bx, az = bz;
    if (R.ring_w) {
      const int* rs = R.ring + 3 * ((bz / 16) * R.ring_w + (bx / 16));
      ax = rs[0] * 16 + bx % 16;
      az = rs[1] * 16 + bz % 16;
    }
    unsigned long long k = atomicAdd(count, 1ull);
    if (k < cap) {
      xyz[3 * k] = ax * 8 + (int)(l & 7u);
      xyz[3 * k + 1] = by * 8 + (int)((l >> 3) & 7u);
      xyz[3 * k + 2] = az * 8 + (int)(l >> 6);
      vol[k] = p;
    }
  }
}

__global__ void k_slot_map(Region R, int* slot_brick, unsigned nslots) {
  const unsigned long long nb = (unsigned long long)R.bx * R.by * R.bz;
  for (unsigned long long gi = blockIdx.x * (unsigned long long)blockDim.x + threadIdx.x; gi < nb; gi += (unsigned long long)gridDim.x * blockDim.x) {
    unsigned g = R.grid[gi];
    if (g >= 256u && g - 256u < nslots) slot_brick[g - 256u] = (int)gi;
  }
}

}  // namespace vfe

namespace vfe {

// ------------------------------------------------------------------ wake-proposal features
// Per materialised brick (atlas slot): aggregates of its 512 cells.
struct SlotAggr {
  float wsum, wmax;
  unsigned npart, nwater, nsolid, nactive, ntop;
  int gi;  // grid index, -1 for a slot no brick uses
};

__global__ void k_slot_aggr(Region R, const int* slot_gi, unsigned nslots, SlotAggr* out) {
  __shared__ float s_sum[4], s_max[4];
  __shared__ unsigned s_cnt[4][5];
  const unsigned tid = threadIdx.x, lane = tid & 31u, warp = tid >> 5;  // 128 threads
  for (unsigned s = blockIdx.x; s < nslots; s += gridDim.x) {
    const int gi = slot_gi[s];
    float sum = 0.f, mx = 0.f;
    unsigned c[5] = {0, 0, 0, 0, 0};
    if (gi >= 0) {
      int bx = gi % R.bx, by = (gi / R.bx) % R.by, bz = gi / (R.bx * R.by);
      if (R.ring_w) {
        const int* rs = R.ring + 3 * ((bz / 16) * R.ring_w + (bx / 16));
        bx = rs[0] * 16 + bx % 16;
        bz = rs[1] * 16 + bz % 16;
      }
      for (unsigned l = tid; l < 512u; l += 128u) {
        const size_t o = (size_t)s * 512u + l;
        const unsigned m = R.amat[o];
        const float p = R.avol[o];
        const float v = p > 0.f ? p : (m == WATER ? 1.f : 0.f);
        sum += v;
        mx = fmaxf(mx, v);
        c[0] += p > 0.f;
        c[1] += m == WATER;
        c[2] += (m != 0u && m != WATER);
        const int x = bx * 8 + (int)(l & 7u), y = by * 8 + (int)((l >> 3) & 7u), z = bz * 8 + (int)(l >> 6);
        if (in_dom(R, x, y, z)) {
          unsigned id = dom_id(R, x, y, z);
          c[3] += (R.active[id >> 5] >> (id & 31)) & 1u;
        }
        if (v > 0.f && ((l >> 3) & 7u) < 7u) {  // water with air above (within the brick)
          const unsigned m2 = R.amat[o + 8];
          const float p2 = R.avol[o + 8];
          c[4] += (m2 == 0u && !(p2 > 0.f));
        }
      }
    }
    for (int off = 16; off; off >>= 1) {
      sum += __shfl_xor_sync(FULLMASK, sum, off);
      mx = fmaxf(mx, __shfl_xor_sync(FULLMASK, mx, off));
      for (int k = 0; k < 5; ++k) c[k] += __shfl_xor_sync(FULLMASK, c[k], off);
    }
    if (lane == 0) {
      s_sum[warp] = sum;
      s_max[warp] = mx;
      for (int k = 0; k < 5; ++k) s_cnt[warp][k] = c[k];
    }
    __syncthreads();
    if (tid == 0) {
      SlotAggr a;
      a.wsum = s_sum[0] + s_sum[1] + s_sum[2] + s_sum[3];
      a.wmax = fmaxf(fmaxf(s_max[0], s_max[1]), fmaxf(s_max[2], s_max[3]));
      unsigned t[5];
      for (int k = 0; k < 5; ++k) t[k] = s_cnt[0][k] + s_cnt[1][k] + s_cnt[2][k] + s_cnt[3][k];
      a.npart = t[0];
      a.nwater = t[1];
      a.nsolid = t[2];
      a.nactive = t[3];
      a.ntop = t[4];
      a.gi = gi;
      out[s] = a;
    }
    __syncthreads();
  }
}

// Aggregate of the face neighbour (dx,dy,dz) of grid cell gi: its slot's, or the uniform value's.
__device__ __forceinline__ void neighbour_aggr(const Region& R, const SlotAggr* aggr, int gi, int dx, int dy, int dz, float& wsum,
                                               float& act, int& nslot) {
  int bx = gi % R.bx + dx, by = (gi / R.bx) % R.by + dy, bz = gi / (R.bx * R.by) + dz;
  wsum = 0.f;
  act = 0.f;
  nslot = -1;
  if (by < 0 || by >= R.by) return;
  if (!R.ring_w && (bx < 0 || bz < 0 || bx >= R.bx || bz >= R.bz)) return;
  unsigned g = R.grid[grid_index(R, bx, by, bz)];
  if (g >= 256u) {
    nslot = (int)(g - 256u);
    wsum = aggr[nslot].wsum;
    act = (float)aggr[nslot].nactive;
  } else if (g == WATER) {
    wsum = 512.f;
  }
}

// Features (32 fp16 per slot): water sum, max level, partial/water/solid/active counts, exposed
// surface, the six face neighbours' water sums and active counts, water-sum changes over the last
// four calls (own and the faces': the flux proxy), wake recency, height, bias.
__global__ void k_slot_features(Region R, const SlotAggr* aggr, unsigned nslots, const float* hist, unsigned hpos, unsigned tick,
                                __half* X) {
  for (unsigned s = blockIdx.x * blockDim.x + threadIdx.x; s < nslots; s += gridDim.x * blockDim.x) {
    float f[32];
    for (int k = 0; k < 32; ++k) f[k] = 0.f;
    const SlotAggr a = aggr[s];
    if (a.gi >= 0) {
      const float old = hist[(size_t)s * 4 + ((hpos + 1) & 3u)];
      f[0] = a.wsum / 512.f;
      f[1] = a.wmax;
      f[2] = a.npart / 512.f;
      f[3] = a.nwater / 512.f;
      f[4] = a.nsolid / 512.f;
      f[5] = a.nactive / 512.f;
      f[6] = a.ntop / 64.f;
      const int D[6][3] = {{1, 0, 0}, {-1, 0, 0}, {0, 1, 0}, {0, -1, 0}, {0, 0, 1}, {0, 0, -1}};
      for (int k = 0; k < 6; ++k) {
        float w, ac;
        int ns;
        neighbour_aggr(R, aggr, a.gi, D[k][0], D[k][1], D[k][2], w, ac, ns);
        f[7 + k] = w / 512.f;
        f[13 + k] = ac / 512.f;
        f[20 + k] = ns >= 0 ? (w - hist[(size_t)ns * 4 + ((hpos + 1) & 3u)]) / 64.f : 0.f;
      }
      f[19] = (a.wsum - old) / 64.f;
      const unsigned lw = R.last_woken[s];
      const unsigned age = lw ? tick - lw : 0xFFFFFFFFu;
      f[26] = age <= 1u ? 1.f : 0.f;
      f[27] = age <= 4u ? 1.f : 0.f;
      f[28] = lw ? 1.f / (1.f + (float)age) : 0.f;
      f[29] = (float)(((a.gi / R.bx) % R.by) * 8) / (float)R.ny;
      f[30] = 1.f;
      f[31] = a.nactive ? 1.f : 0.f;
    }
    __half2* out = reinterpret_cast<__half2*>(X + (size_t)s * 32);
    for (int k = 0; k < 16; ++k) out[k] = __floats2half2_rn(f[2 * k], f[2 * k + 1]);
  }
}

__global__ void k_slot_hist(const SlotAggr* aggr, unsigned nslots, float* hist, unsigned hpos) {
  for (unsigned s = blockIdx.x * blockDim.x + threadIdx.x; s < nslots; s += gridDim.x * blockDim.x)
    hist[(size_t)s * 4 + (hpos & 3u)] = aggr[s].gi >= 0 ? aggr[s].wsum : 0.f;
}

// Label: a cell of the slot's brick was drained in ticks (since, now].
__global__ void k_slot_labels(Region R, unsigned nslots, unsigned since, unsigned now, float* y) {
  for (unsigned s = blockIdx.x * blockDim.x + threadIdx.x; s < nslots; s += gridDim.x * blockDim.x) {
    const unsigned lw = R.last_woken[s];
    y[s] = (lw > since && lw <= now) ? 1.f : 0.f;
  }
}

// Pre-stage the bricks the proposal expects to wake: their material and volume lines into L2.
__global__ void k_stage(Region R, unsigned nslots, const float* prob, float thr, unsigned* staged) {
  for (unsigned s = blockIdx.x * blockDim.x + threadIdx.x; s < nslots; s += gridDim.x * blockDim.x) {
    if (!(prob[s] >= thr)) continue;
    const char* m = reinterpret_cast<const char*>(R.amat + (size_t)s * 512u);
    const char* v = reinterpret_cast<const char*>(R.avol + (size_t)s * 512u);
    for (int k = 0; k < 4; ++k) asm volatile("prefetch.global.L2 [%0];" ::"l"(m + 128 * k));
    for (int k = 0; k < 16; ++k) asm volatile("prefetch.global.L2 [%0];" ::"l"(v + 128 * k));
    atomicAdd(staged, 1u);
  }
}

}  // namespace vfe
