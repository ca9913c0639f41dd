// Kernels of the CA-water engine: the tick (drain -> sort -> sweep -> levelling) for one or many
// regions, host-edit kernels (wake, displace, brush, emitters, set_partial) and inspection
// kernels (digests, dense export, change download).
#pragma once
#include "engine_dev.cuh"

namespace vfe {

constexpr int TICK_THREADS = 512;
constexpr int TICK_WARPS = TICK_THREADS / 32;

// ---------------------------------------------------------------- CTA radix sort (LSD, 8 bit)
// Stable within each warp's contiguous chunk; chunks in order -> stable overall. Sorts n unique
// keys in place (tmp is scratch). hist: TICK_WARPS*256 u32 of shared memory.
__device__ void cta_radix_sort(unsigned* keys, unsigned* tmp, unsigned n, unsigned* hist, unsigned* sred) {
  const unsigned tid = threadIdx.x, lane = tid & 31u, warp = tid >> 5;
  if (n <= 1) return;
  // key range -> number of passes
  unsigned mn = 0xFFFFFFFFu, mx = 0;
  for (unsigned i = tid; i < n; i += TICK_THREADS) {
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
    sred[TICK_WARPS + warp] = mx;
  }
  __syncthreads();
  if (tid == 0) {
    unsigned a = 0xFFFFFFFFu, b = 0;
    for (int w = 0; w < TICK_WARPS; ++w) {
      a = min(a, sred[w]);
      b = max(b, sred[TICK_WARPS + w]);
    }
    sred[2 * TICK_WARPS] = a;
    sred[2 * TICK_WARPS + 1] = b;
  }
  __syncthreads();
  const unsigned kmin = sred[2 * TICK_WARPS], range = sred[2 * TICK_WARPS + 1] - kmin;
  __syncthreads();
  const int bits = range ? 32 - __clz(range) : 0;
  const int passes = (bits + 7) / 8;
  const unsigned chunk = (n + TICK_WARPS - 1) / TICK_WARPS;
  const unsigned b0 = min(n, warp * chunk), b1 = min(n, b0 + chunk);
  unsigned* src = keys;
  unsigned* dst = tmp;
  for (int p = 0; p < passes; ++p) {
    const int sh = 8 * p;
    for (unsigned i = tid; i < TICK_WARPS * 256; i += TICK_THREADS) hist[i] = 0;
    __syncthreads();
    for (unsigned i = b0 + lane; i < b1; i += 32) atomicAdd(&hist[warp * 256 + (((src[i] - kmin) >> sh) & 255u)], 1u);
    __syncthreads();
    // offsets: digit-major, warp-minor
    if (tid < 256) {
      unsigned s = 0;
      for (int w = 0; w < TICK_WARPS; ++w) s += hist[w * 256 + tid];
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
      for (int w = 0; w < TICK_WARPS; ++w) {
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
    for (unsigned i = tid; i < n; i += TICK_THREADS) keys[i] = src[i];
    __syncthreads();
  }
}

// ----------------------------------------------------------------------------- the tick
struct TickSmem {
  unsigned hist[TICK_WARPS * 256];
  unsigned sred[2 * 256 + 64];
  unsigned pq[PRESS_QCAP];
  unsigned long long vis[VIS_CAP];
  int ring[3 * 16 * 16];
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
  W.epoch = 1;
  W.level_round = c.level_round != 0;
  W.changed = false;
}

// FluidSim::tick (fluid.rs:564-657) for region R, n_ticks times. All threads of the CTA enter.
__device__ void run_ticks(const Region& R, TickSmem& sm, int n_ticks) {
  const unsigned tid = threadIdx.x, warp = tid >> 5;
  // ring table to shared memory when small
  const int* ring = R.ring;
  if (R.ring_w && R.ring_w <= 16) {
    for (int i = tid; i < 3 * R.ring_w * R.ring_w; i += TICK_THREADS) sm.ring[i] = R.ring[i];
    ring = sm.ring;
  }
  for (unsigned i = tid; i < VIS_CAP; i += TICK_THREADS) sm.vis[i] = 0ull;
  __shared__ unsigned s_n, s_flip, s_clear, s_abort;
  __shared__ WS sW;
  if (tid == 0) {
    load_ws(R, sW);
    s_abort = R.ctl->status != 0;
  }
  __syncthreads();
  for (int t = 0; t < n_ticks; ++t) {
    if (s_abort) break;
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
    for (unsigned i = tid; i < n; i += TICK_THREADS) {
      unsigned id = R.queue[(qh + i) & R.qmask];
      atomicAnd(&R.active[id >> 5], ~(1u << (id & 31)));
      R.cells[i] = sort_key(R, id, flip);
    }
    __syncthreads();
    if (tid == 0) sW.qhead = qh + n;
    __syncthreads();
    // ---- sort (fluid.rs:575-580)
    cta_radix_sort(R.cells, R.cells_tmp, n, sm.hist, sm.sred);
    // ---- the sweep (fluid.rs:584-651), one warp, reference order
    if (warp == 0) {
      WS W = sW;
      W.pulls = 0;
      W.changed = false;
      W.activations = W.pull_attempts = W.pull_success = W.bfs_visits = W.level_cells_total = 0;
      W.pdelta = 0;
      Smem S{sm.vis, sm.pq, ring};
      for (unsigned r = 0; r < n; ++r) {
        unsigned id = key_to_id(R, R.cells[r], flip);
        int x, y, z;
        dom_xyz(R, id, x, y, z);
        process_cell(R, W, S, x, y, z);
      }
      // ---- levelling (fluid.rs:652-655)
      unsigned clear = 0;
      if (W.level_round || (R.ctl->tick_no % LEVEL_TICKS) == 0u) clear = level_surfaces(R, W, S) ? 1u : 0u;
      // partial_count delta: reduce across lanes
      long long pd = W.pdelta;
      for (int o = 16; o; o >>= 1) pd += __shfl_xor_sync(FULLMASK, pd, o);
      if (lane_id() == 0) {
        Ctl& c = *R.ctl;
        c.last_cells = n;
        c.cells_total += n;
        c.pull_attempts += W.pull_attempts;
        c.pull_success += W.pull_success;
        c.bfs_visits += W.bfs_visits;
        c.level_cells_total += W.level_cells_total;
        c.activations += W.activations;
        c.partial_count += pd;
        c.last_level_cells = W.llc;
        c.nseeds = W.nseeds;
        c.level_round = W.level_round ? 1u : 0u;
        if (W.changed) c.changed = 1u;
        c.qhead = W.qhead;
        c.qtail = W.qtail;
        W.pdelta = 0;
        sW = W;
        sW.pdelta = 0;
        s_clear = clear;
        s_abort = c.status != 0;
      }
      __syncwarp();
    }
    __syncthreads();
    // ---- end of a levelling round: clear the marks it touched (fluid.rs:503-505)
    if (s_clear) {
      const unsigned nt = R.ctl->mark_ntiles;
      for (unsigned k = warp; k < nt; k += TICK_WARPS) {
        unsigned tile = R.mark_list[k];
        for (unsigned w = lane_id(); w < 128; w += 32) R.marks[(size_t)tile * 128u + w] = 0u;
        if (lane_id() == 0) R.mark_tflag[tile] = 0u;
      }
      __syncthreads();
      if (tid == 0) R.ctl->mark_ntiles = 0;
      __syncthreads();
    }
  }
}

__global__ void __launch_bounds__(TICK_THREADS, 1) k_tick(Region* regs, int nreg, int n_ticks) {
  extern __shared__ __align__(16) unsigned char smraw[];
  TickSmem& sm = *reinterpret_cast<TickSmem*>(smraw);
  for (int r = blockIdx.x; r < nreg; r += gridDim.x) {
    run_ticks(regs[r], sm, n_ticks);
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
