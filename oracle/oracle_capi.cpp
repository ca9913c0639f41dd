// ORACLE — test infrastructure only. A C ABI over the CPU restatement (fluid_oracle.hpp) so
// tests and the CPU-baseline leg of bench.py can drive it through ctypes. One handle = one
// SparseVolume + one FluidSim, the pairing every reference call site uses
// (src/app/window.rs:856-858, src/app/shot.rs:161-175).
#include <chrono>
#include <cstring>
#include <vector>

#include "fluid_oracle.hpp"

using namespace orc;

struct orc_handle {
  SparseVolume v;
  FluidSim s;
};

static inline uint64_t cell_hash(int32_t x, int32_t y, int32_t z, uint8_t m, uint32_t vb) {
  return fmix64(key(x, y, z) * 0x9E3779B97F4A7C15ULL + (((uint64_t)m << 32) | vb));
}

extern "C" {

orc_handle* orc_create_bounded(int32_t nx, int32_t ny, int32_t nz) {
  auto* h = new orc_handle();
  h->v = SparseVolume(nx, ny, nz);
  return h;
}

orc_handle* orc_create_ring(int32_t w, int32_t ny) {
  auto* h = new orc_handle();
  h->v = SparseVolume(8, 8, 8);
  h->v.ring_init(w, ny);
  return h;
}

void orc_destroy(orc_handle* h) { delete h; }

// Load a brick grid in the reference's encoding (0 empty, 1..255 uniform, >=256 detailed: index
// into `bricks`, 512 bytes each, index lz*64+ly*8+lx) into the handle's volume. Ring slots, when
// the volume is a ring: (cx, cz, loaded) triples, ring_w*ring_w of them.
int orc_load_grid(orc_handle* h, const uint32_t* grid, const uint8_t* bricks, uint64_t nbricks, const int32_t* ring_slots) {
  SparseVolume& v = h->v;
  v.grid.assign(grid, grid + v.grid.size());
  v.bricks.resize(nbricks);
  for (uint64_t i = 0; i < nbricks; ++i) std::memcpy(v.bricks[i].data(), bricks + i * 512, 512);
  v.free_bricks.clear();
  v.dirty_grid.clear();
  if (v.ring_w && ring_slots) {
    for (int i = 0; i < v.ring_w * v.ring_w; ++i) {
      v.ring_slots[i].cx = ring_slots[3 * i];
      v.ring_slots[i].cz = ring_slots[3 * i + 1];
      v.ring_slots[i].loaded = ring_slots[3 * i + 2] != 0;
      v.ring_slots[i].modified = false;
    }
  }
  return 0;
}

void orc_fill_box(orc_handle* h, int32_t x0, int32_t y0, int32_t z0, int32_t x1, int32_t y1, int32_t z1, uint8_t m) {
  h->v.fill_box(x0, y0, z0, x1, y1, z1, m);
}
void orc_fill_sphere(orc_handle* h, float cx, float cy, float cz, float r, uint8_t m) { h->v.fill_sphere(cx, cy, cz, r, m); }
void orc_set_voxel(orc_handle* h, int32_t x, int32_t y, int32_t z, uint8_t m) { h->v.set_voxel(x, y, z, m); }
uint8_t orc_get_voxel(orc_handle* h, int32_t x, int32_t y, int32_t z) { return h->v.get_voxel(x, y, z); }
void orc_compact(orc_handle* h) { h->v.compact(); }
uint64_t orc_detailed_bricks(orc_handle* h) { return h->v.detailed_bricks(); }
uint32_t orc_grid_at(orc_handle* h, int32_t bx, int32_t by, int32_t bz) { return h->v.grid[h->v.grid_index(bx, by, bz)]; }

int orc_tick(orc_handle* h) { return h->s.tick(h->v) ? 1 : 0; }
int orc_ticks(orc_handle* h, int32_t n, int32_t stop_when_idle) {
  int any = 0;
  for (int32_t i = 0; i < n; ++i) {
    any |= h->s.tick(h->v) ? 1 : 0;
    if (stop_when_idle && h->s.idle()) break;
  }
  return any;
}
int orc_update(orc_handle* h, float dt) { return h->s.update(h->v, dt) ? 1 : 0; }
void orc_wake(orc_handle* h, int32_t x0, int32_t y0, int32_t z0, int32_t x1, int32_t y1, int32_t z1) { h->s.wake(x0, y0, z0, x1, y1, z1); }
void orc_displace(orc_handle* h, int32_t x, int32_t y, int32_t z) { h->s.displace(h->v, x, y, z); }
void orc_emit(orc_handle* h, const int32_t* xyz, uint64_t n, float amount) {
  for (uint64_t i = 0; i < n; ++i) h->s.emit(h->v, xyz[3 * i], xyz[3 * i + 1], xyz[3 * i + 2], amount);
}
uint64_t orc_apply_brush(orc_handle* h, const int32_t* xyz, uint64_t n, uint8_t m) { return h->s.apply_brush(h->v, xyz, n, m); }
float orc_volume(orc_handle* h, int32_t x, int32_t y, int32_t z) { return h->s.volume(h->v, x, y, z); }
void orc_set_partial(orc_handle* h, int32_t x, int32_t y, int32_t z, float val) { h->s.set_partial(x, y, z, val); }
void orc_shift(orc_handle* h, int32_t dx, int32_t dz) { h->s.shift(dx, dz); }
void orc_ring_rebase(orc_handle* h, int32_t dcx, int32_t dcz) { h->v.ring_rebase(dcx, dcz); }
void orc_ring_evict(orc_handle* h, int32_t cx, int32_t cz) { h->v.ring_evict(cx, cz); }
// ring_paste of a 128 x (bricks_y * 8) x 128 chunk given as grid words and bricks
void orc_ring_paste(orc_handle* h, const uint32_t* grid, const uint8_t* bricks, uint64_t nbricks, int32_t bricks_y, int32_t cx, int32_t cz) {
  SparseVolume c(128, bricks_y * 8, 128);
  c.grid.assign(grid, grid + c.grid.size());
  c.bricks.resize(nbricks);
  for (uint64_t i = 0; i < nbricks; ++i) std::memcpy(c.bricks[i].data(), bricks + i * 512, 512);
  h->v.ring_paste(c, cx, cz);
}
void orc_reset(orc_handle* h) { h->s.reset(); }
int orc_idle(orc_handle* h) { return h->s.idle() ? 1 : 0; }
uint64_t orc_active_count(orc_handle* h) { return h->s.active_count(); }
uint64_t orc_partial_count(orc_handle* h) { return h->s.partial_count(); }
uint64_t orc_last_tick_cells(orc_handle* h) { return h->s.last_tick_cells(); }
uint32_t orc_tick_no(orc_handle* h) { return h->s.tick_no(); }
int orc_level_round(orc_handle* h) { return h->s.level_round() ? 1 : 0; }
int orc_layer_mark(orc_handle* h, int32_t x, int32_t y, int32_t z) { return h->s.layer_mark(x, y, z) ? 1 : 0; }

// Stats: cells, pull_attempts, pull_nonempty, pull_success, bfs_visits, level_calls,
// level_cells, level_fills, drains, activations, ticks.
void orc_stats(orc_handle* h, uint64_t* out) {
  const Stats& s = h->s.stats;
  uint64_t a[11] = {s.cells, s.pull_attempts, s.pull_nonempty, s.pull_success, s.bfs_visits, s.level_calls,
                    s.level_cells, s.level_fills, s.drains, s.activations, s.ticks};
  std::memcpy(out, a, sizeof(a));
}

// FIFO keys in order, as (x, y, z) triples. Returns the length (writes at most cap entries).
uint64_t orc_queue(orc_handle* h, int32_t* out, uint64_t cap) {
  const auto& q = h->s.queue();
  uint64_t n = 0;
  for (uint64_t k : q) {
    if (n < cap) unkey(k, out[3 * n], out[3 * n + 1], out[3 * n + 2]);
    ++n;
  }
  return n;
}
uint64_t orc_seeds(orc_handle* h, int32_t* out, uint64_t cap) {
  const auto& q = h->s.seed_list();
  uint64_t n = 0;
  for (uint64_t k : q) {
    if (n < cap) unkey(k, out[3 * n], out[3 * n + 1], out[3 * n + 2]);
    ++n;
  }
  return n;
}

// Dense export of a box [x0, x0+sx) x [y0, y0+sy) x [z0, z0+sz): materials and partial volumes
// (0 where the cell has no partial entry), index ((z-z0)*sy + (y-y0))*sx + (x-x0).
void orc_export_box(orc_handle* h, int32_t x0, int32_t y0, int32_t z0, int32_t sx, int32_t sy, int32_t sz, uint8_t* mat, float* part) {
  for (int32_t z = 0; z < sz; ++z)
    for (int32_t y = 0; y < sy; ++y)
      for (int32_t x = 0; x < sx; ++x) {
        size_t i = ((size_t)z * sy + y) * sx + x;
        if (mat) mat[i] = h->v.get_voxel(x0 + x, y0 + y, z0 + z);
        if (part) part[i] = h->s.partials().get(x0 + x, y0 + y, z0 + z);
      }
}

// Order-independent state digest: sum over every cell whose (material, partial bits) is not
// (0, 0) of fmix64(key(x,y,z) * golden + (material << 32 | partial bits)). Cells are visited
// over the brick grid (bounded: the volume; ring: loaded chunks) plus every partial entry.
uint64_t orc_state_digest(orc_handle* h) {
  SparseVolume& v = h->v;
  uint64_t d = 0;
  std::vector<uint8_t> seen;
  for (int32_t bz = 0; bz < v.bricks_z; ++bz)
    for (int32_t by = 0; by < v.bricks_y; ++by)
      for (int32_t bx = 0; bx < v.bricks_x; ++bx) {
        size_t gi = v.grid_index(bx, by, bz);
        int32_t ax = bx, az = bz;
        if (v.ring_w) {
          const RingSlot& s = v.ring_slots[(size_t)(bz / RING_CHUNK_B) * v.ring_w + (bx / RING_CHUNK_B)];
          if (!s.loaded) continue;
          ax = s.cx * RING_CHUNK_B + bx % RING_CHUNK_B;
          az = s.cz * RING_CHUNK_B + bz % RING_CHUNK_B;
        }
        uint32_t g = v.grid[gi];
        for (int l = 0; l < 512; ++l) {
          int32_t x = ax * 8 + (l & 7), y = by * 8 + ((l >> 3) & 7), z = az * 8 + (l >> 6);
          if (y >= v.ny) continue;
          uint8_t m = g < 256 ? (uint8_t)g : v.bricks[g - 256][(z & 7) * 64 + (y & 7) * 8 + (x & 7)];
          float p = h->s.partials().get(x, y, z);
          uint32_t vb;
          std::memcpy(&vb, &p, 4);
          if (m == 0 && vb == 0) continue;
          d += cell_hash(x, y, z, m, vb);
        }
      }
  // partial entries outside the addressable volume (never produced by tick; kept for safety)
  h->s.partials().for_each([&](int32_t x, int32_t y, int32_t z, float p) {
    if (v.inside(x, y, z)) return;
    uint32_t vb;
    std::memcpy(&vb, &p, 4);
    d += cell_hash(x, y, z, 0, vb);
  });
  return d;
}

// Order-dependent digest of the FIFO: sum of fmix64(key * golden + position).
uint64_t orc_queue_digest(orc_handle* h) {
  uint64_t d = 0, i = 0;
  for (uint64_t k : h->s.queue()) d += fmix64(k * 0x9E3779B97F4A7C15ULL + (i++));
  return d;
}
uint64_t orc_seed_digest(orc_handle* h) {
  uint64_t d = 0, i = 0;
  for (uint64_t k : h->s.seed_list()) d += fmix64(k * 0x9E3779B97F4A7C15ULL + (i++));
  return d;
}

// Total volume in f64, cells visited in the reference test's order (z, y, x) over a box
// (src/fluid.rs:740-750).
double orc_total_box(orc_handle* h, int32_t x0, int32_t y0, int32_t z0, int32_t x1, int32_t y1, int32_t z1) {
  double t = 0.0;
  for (int32_t z = z0; z < z1; ++z)
    for (int32_t y = y0; y < y1; ++y)
      for (int32_t x = x0; x < x1; ++x) t += (double)h->s.volume(h->v, x, y, z);
  return t;
}

// PartialField on its own (src/fluid.rs:64-180), for the reference's page test (:784-798).
PartialField* orc_pf_create() { return new PartialField(); }
void orc_pf_destroy(PartialField* p) { delete p; }
void orc_pf_set(PartialField* p, int32_t x, int32_t y, int32_t z, float v) { p->set(x, y, z, v); }
float orc_pf_get(PartialField* p, int32_t x, int32_t y, int32_t z) { return p->get(x, y, z); }
void orc_pf_erase(PartialField* p, int32_t x, int32_t y, int32_t z) { p->erase(x, y, z); }
uint64_t orc_pf_len(PartialField* p) { return p->len(); }
uint64_t orc_pf_entries(PartialField* p, int32_t* xyz, float* v, uint64_t cap) {
  uint64_t n = 0;
  p->for_each([&](int32_t x, int32_t y, int32_t z, float val) {
    if (n < cap) {
      xyz[3 * n] = x;
      xyz[3 * n + 1] = y;
      xyz[3 * n + 2] = z;
      v[n] = val;
    }
    ++n;
  });
  return n;
}

// Time n ticks with steady_clock; returns seconds. (CPU baseline leg.)
double orc_time_ticks(orc_handle* h, int32_t n) {
  auto t0 = std::chrono::steady_clock::now();
  for (int32_t i = 0; i < n; ++i) h->s.tick(h->v);
  auto t1 = std::chrono::steady_clock::now();
  return std::chrono::duration<double>(t1 - t0).count();
}

}  // extern "C"
