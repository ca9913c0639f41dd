// Host-side sparse brick world (SparseVolume mirror) and the synthetic workloads.
#include "world.hpp"

#include <algorithm>
#include <cmath>
#include <cstring>
#include <memory>
#include <new>

#include "../../include/vf_world.h"
#include "../../include/vf_fluid.h"

namespace vfw {

World::World(int32_t nx_, int32_t ny_, int32_t nz_) {  // sparse_volume.rs:117-139
  nx = nx_;
  ny = ny_;
  nz = nz_;
  bricks_x = (nx + BRICK - 1) / BRICK;
  bricks_y = (ny + BRICK - 1) / BRICK;
  bricks_z = (nz + BRICK - 1) / BRICK;
  grid.assign((size_t)bricks_x * bricks_y * bricks_z, 0);
}

void World::ring_init(int32_t w, int32_t ny_) {  // sparse_volume.rs:177-192
  ring_w = w;
  nx = w * RING_CHUNK_B * BRICK;
  nz = nx;
  ny = ny_;
  bricks_x = w * RING_CHUNK_B;
  bricks_z = bricks_x;
  bricks_y = (ny + BRICK - 1) / BRICK;
  grid.assign((size_t)bricks_x * bricks_y * bricks_z, 0);
  bricks.clear();
  free_bricks.clear();
  dirty_grid.clear();
  ring_slots.assign((size_t)w * w, RingSlot{});
}

size_t World::alloc_brick() {
  if (!free_bricks.empty()) {
    size_t i = free_bricks.back();
    free_bricks.pop_back();
    return i;
  }
  bricks.emplace_back();
  return bricks.size() - 1;
}

size_t World::materialize(size_t gi, uint8_t fill) {  // sparse_volume.rs:250-266
  size_t idx = alloc_brick();
  bricks[idx].fill(fill);
  grid[gi] = 256 + (uint32_t)idx;
  return idx;
}

void World::mark_modified(size_t gi) {  // sparse_volume.rs:218-225
  if (ring_w == 0) return;
  size_t bxy = (size_t)bricks_x * bricks_y;
  size_t i = ((gi / bxy) / RING_CHUNK_B) * ring_w + (gi % bricks_x) / RING_CHUNK_B;
  ring_slots[i].modified = true;
}

void World::set_voxel(int32_t x, int32_t y, int32_t z, uint8_t m) {  // sparse_volume.rs:268-293
  if (!inside(x, y, z)) return;
  size_t gi = grid_index(x >> 3, y >> 3, z >> 3);
  uint32_t v = grid[gi];
  size_t bi;
  if (v < 256) {
    if ((uint8_t)v == m) return;
    bi = materialize(gi, (uint8_t)v);
  } else {
    bi = v - 256;
  }
  uint8_t& slot = bricks[bi][(z & 7) * 64 + (y & 7) * 8 + (x & 7)];
  if (slot == m) return;
  slot = m;
  if (track_dirty) dirty_grid.push_back((uint32_t)gi);
  mark_modified(gi);
}

void World::fill_box(int32_t x0, int32_t y0, int32_t z0, int32_t x1, int32_t y1, int32_t z1, uint8_t m) {
  for (int32_t z = z0; z <= z1; ++z)
    for (int32_t y = y0; y <= y1; ++y)
      for (int32_t x = x0; x <= x1; ++x) set_voxel(x, y, z, m);
}

// The cells fill_sphere visits, in its loop order (sparse_volume.rs:295-316).
template <class F>
static void sphere_cells(float cx, float cy, float cz, float r, F f) {
  int32_t x0 = (int32_t)std::floor(cx - r), x1 = (int32_t)std::ceil(cx + r);
  int32_t y0 = (int32_t)std::floor(cy - r), y1 = (int32_t)std::ceil(cy + r);
  int32_t z0 = (int32_t)std::floor(cz - r), z1 = (int32_t)std::ceil(cz + r);
  float r2 = r * r;
  for (int32_t z = z0; z <= z1; ++z) {
    float dz = (float)z + 0.5f - cz;
    for (int32_t y = y0; y <= y1; ++y) {
      float dy = (float)y + 0.5f - cy;
      float rem = r2 - dz * dz - dy * dy;
      if (rem < 0.0f) continue;
      for (int32_t x = x0; x <= x1; ++x) {
        float dx = (float)x + 0.5f - cx;
        if (dx * dx <= rem) f(x, y, z);
      }
    }
  }
}

void World::fill_sphere(float cx, float cy, float cz, float r, uint8_t m) {
  sphere_cells(cx, cy, cz, r, [&](int32_t x, int32_t y, int32_t z) { set_voxel(x, y, z, m); });
}

void World::compact() {  // sparse_volume.rs:339-350
  for (size_t gi = 0; gi < grid.size(); ++gi) {
    uint32_t v = grid[gi];
    if (v < 256) continue;
    const auto& b = bricks[v - 256];
    if (std::all_of(b.begin(), b.end(), [&](uint8_t c) { return c == b[0]; })) {
      grid[gi] = b[0];
      free_bricks.push_back(v - 256);
    }
  }
}

void World::ring_paste(const World& src, int32_t cx, int32_t cz) {  // sparse_volume.rs:478-510
  RingSlot s = ring_slots[ring_slot_index(cx, cz)];
  if (s.loaded) ring_evict(s.cx, s.cz);
  int32_t bx0 = cx * RING_CHUNK_B, bz0 = cz * RING_CHUNK_B;
  for (int32_t bz = 0; bz < std::min(RING_CHUNK_B, src.bricks_z); ++bz)
    for (int32_t by = 0; by < std::min(bricks_y, src.bricks_y); ++by)
      for (int32_t bx = 0; bx < std::min(RING_CHUNK_B, src.bricks_x); ++bx) {
        uint32_t v = src.grid[src.grid_index(bx, by, bz)];
        size_t gi = grid_index(bx0 + bx, by, bz0 + bz);
        if (v < 256) {
          grid[gi] = v;
          continue;
        }
        size_t idx = alloc_brick();
        bricks[idx] = src.bricks[v - 256];
        grid[gi] = 256 + (uint32_t)idx;
      }
  ring_slots[ring_slot_index(cx, cz)] = RingSlot{cx, cz, true, false};
}

void World::ring_evict(int32_t cx, int32_t cz) {  // sparse_volume.rs:513-537
  RingSlot s = ring_slots[ring_slot_index(cx, cz)];
  if (!s.loaded) return;
  int32_t bx0 = s.cx * RING_CHUNK_B, bz0 = s.cz * RING_CHUNK_B;
  for (int32_t bz = 0; bz < RING_CHUNK_B; ++bz)
    for (int32_t by = 0; by < bricks_y; ++by)
      for (int32_t bx = 0; bx < RING_CHUNK_B; ++bx) {
        size_t gi = grid_index(bx0 + bx, by, bz0 + bz);
        uint32_t v = grid[gi];
        if (v >= 256) free_bricks.push_back(v - 256);
        grid[gi] = 0;
      }
  ring_slots[ring_slot_index(cx, cz)] = RingSlot{};
}

// ------------------------------------------------------------------ noise (worldgen/mod.rs)
uint32_t hash2(int32_t x, int32_t y, uint32_t seed) {  // worldgen/mod.rs:31-39
  uint32_t h = seed;
  h ^= (uint32_t)x * 0x8da6b343u;
  h ^= (uint32_t)y * 0xd8163841u;
  h = (h ^ (h >> 13)) * 0x9e3779b1u;
  return h ^ (h >> 16);
}

static inline float rand01(uint32_t h) { return (float)(h & 0xffffff) / 16777216.0f; }  // :42-44

float value_noise(float x, float y, uint32_t seed) {  // worldgen/mod.rs:45-56
  int32_t xi = (int32_t)std::floor(x), yi = (int32_t)std::floor(y);
  float fx = x - (float)xi, fy = y - (float)yi;
  float sx = fx * fx * (3.0f - 2.0f * fx), sy = fy * fy * (3.0f - 2.0f * fy);
  float v00 = rand01(hash2(xi, yi, seed));
  float v10 = rand01(hash2(xi + 1, yi, seed));
  float v01 = rand01(hash2(xi, yi + 1, seed));
  float v11 = rand01(hash2(xi + 1, yi + 1, seed));
  float a = v00 + (v10 - v00) * sx;
  float b = v01 + (v11 - v01) * sx;
  return a + (b - a) * sy;
}

float fbm(float x, float y, uint32_t seed, int octaves) {  // worldgen/mod.rs:58-66
  float sum = 0.0f, amp = 0.5f, freq = 1.0f;
  for (int i = 0; i < octaves; ++i) {
    sum += amp * value_noise(x * freq, y * freq, seed + (uint32_t)i * 101u);
    amp *= 0.5f;
    freq *= 2.0f;
  }
  return sum;
}

}  // namespace vfw

using namespace vfw;

// ======================================================================== workloads
namespace {

struct Rng {  // splitmix64
  uint64_t s;
  explicit Rng(uint64_t seed) : s(seed) {}
  uint64_t next() {
    uint64_t z = (s += 0x9E3779B97F4A7C15ULL);
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ULL;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBULL;
    return z ^ (z >> 31);
  }
  int32_t uniform(int32_t lo, int32_t hi) { return lo + (int32_t)(next() % (uint64_t)(hi - lo + 1)); }  // inclusive
};

// Build a world brick by brick from a voxel function (uniform bricks stay grid values, like
// the reference's compacted worlds).
template <class F>
void build_bricks(World& w, int32_t ox, int32_t oz, int32_t bx0, int32_t bz0, int32_t nbx, int32_t nbz, F vox) {
  std::array<uint8_t, 512> tmp;
  for (int32_t bz = 0; bz < nbz; ++bz)
    for (int32_t by = 0; by < w.bricks_y; ++by)
      for (int32_t bx = 0; bx < nbx; ++bx) {
        for (int l = 0; l < 512; ++l) {
          int32_t x = ox + bx * 8 + (l & 7), y = by * 8 + ((l >> 3) & 7), z = oz + bz * 8 + (l >> 6);
          tmp[l] = y < w.ny ? vox(x, y, z) : 0;
        }
        size_t gi = w.grid_index(bx0 + bx, by, bz0 + bz);
        if (std::all_of(tmp.begin(), tmp.end(), [&](uint8_t c) { return c == tmp[0]; })) {
          w.grid[gi] = tmp[0];
        } else {
          size_t idx = w.alloc_brick();
          w.bricks[idx] = tmp;
          w.grid[gi] = 256 + (uint32_t)idx;
        }
      }
}

struct Region {
  std::unique_ptr<World> world;
  std::vector<std::array<int32_t, 6>> wakes;
  std::vector<std::array<int32_t, 3>> emitters;
  uint64_t edit_seed = 0;
  int32_t sx = 0, sy = 0, sz = 0;
};

static int32_t round8(float v) { return std::max(8, ((int32_t)std::lround(v) + 7) / 8 * 8); }

}  // namespace

struct vf_world {
  World w;
};

struct vf_workload {
  int32_t id = 0;
  int32_t ticks = 0;
  int32_t emit_every = 0;
  int32_t edit_every = 0;
  float emit_amount = 1.0f;
  std::vector<Region> regions;
  std::vector<std::unique_ptr<vf_world>> handles;
};

namespace {

// Workload 1: 64^3 basin. Stone floor y<4; 2-voxel walls enclose x,z in [8,56) (walls at
// [6,8) and [56,58) from y=4 to the top); a 16^3 block of full water at x,z in [24,40),
// y in [40,56), woken with a 1-voxel margin.
void build_basin(vf_workload& wl) {
  Region r;
  r.world = std::make_unique<World>(64, 64, 64);
  World& w = *r.world;
  w.fill_box(0, 0, 0, 63, 3, 63, STONE);
  w.fill_box(6, 4, 6, 7, 63, 57, STONE);
  w.fill_box(56, 4, 6, 57, 63, 57, STONE);
  w.fill_box(6, 4, 6, 57, 63, 7, STONE);
  w.fill_box(6, 4, 56, 57, 63, 57, STONE);
  w.fill_box(24, 40, 24, 39, 55, 39, WATER);
  w.compact();
  w.dirty_grid.clear();
  r.wakes.push_back({23, 39, 23, 40, 56, 40});
  r.sx = r.sz = r.sy = 64;
  wl.ticks = 300;
  wl.regions.push_back(std::move(r));
}

// Workload 2: dam break on terrain, 512x128x512 (x/z scaled by `scale`). Height
// h = 20 + floor(80 * fbm4(x/128, z/128, seed 1)); stone below h; every air cell with y < 48
// is water; an 8-wide channel (z in [c, c+8) at the middle of z, all x) carves solid voxels
// with y >= 30 into air; the channel box +-1 is woken.
void build_dambreak(vf_workload& wl, float scale) {
  Region r;
  int32_t n = round8(512 * scale);
  r.world = std::make_unique<World>(n, 128, n);
  World& w = *r.world;
  int32_t c0 = n / 2 - 4;
  std::vector<int32_t> h((size_t)n * n);
  for (int32_t z = 0; z < n; ++z)
    for (int32_t x = 0; x < n; ++x) h[(size_t)z * n + x] = 20 + (int32_t)std::floor(80.0f * fbm((float)x / 128.0f, (float)z / 128.0f, 1u, 4));
  build_bricks(w, 0, 0, 0, 0, w.bricks_x, w.bricks_z, [&](int32_t x, int32_t y, int32_t z) -> uint8_t {
    int32_t hh = h[(size_t)z * n + x];
    bool chan = z >= c0 && z < c0 + 8;
    if (y < hh) return (chan && y >= 30) ? 0 : STONE;
    return y < 48 ? WATER : 0;
  });
  r.wakes.push_back({-1, 29, c0 - 1, n, 128, c0 + 8});
  r.sx = r.sz = n;
  r.sy = 128;
  wl.ticks = 1000;
  wl.regions.push_back(std::move(r));
}

// Workloads 3/5: independent regions. Region i: x/z sides uniform in {32..256 step 8}, height
// in {64..128 step 8} (sides scaled by `scale` for tests); terrain
// h = floor(sy*20/128) + floor(sy*80/128 * fbm4(x/128, z/128, seed i+1)); 1-4 water cubes of
// side 8..32 dropped into air over the terrain, each woken with a 1-voxel margin.
void build_regions(vf_workload& wl, float scale, uint64_t seed, int32_t nreg) {
  Rng rng(seed * 0x100000001B3ULL + 3);
  for (int32_t ri = 0; ri < nreg; ++ri) {
    Region r;
    int32_t sx = 32 + 8 * rng.uniform(0, 28), sz = 32 + 8 * rng.uniform(0, 28), sy = 64 + 8 * rng.uniform(0, 8);
    sx = std::max(16, round8(sx * scale));
    sz = std::max(16, round8(sz * scale));
    if (scale < 1.0f) sy = std::max(32, round8(sy * std::sqrt(scale)));
    r.world = std::make_unique<World>(sx, sy, sz);
    World& w = *r.world;
    std::vector<int32_t> h((size_t)sx * sz);
    int32_t base = sy * 20 / 128;
    float amp = (float)sy * 80.0f / 128.0f;
    for (int32_t z = 0; z < sz; ++z)
      for (int32_t x = 0; x < sx; ++x)
        h[(size_t)z * sx + x] = base + (int32_t)std::floor(amp * fbm((float)x / 128.0f, (float)z / 128.0f, (uint32_t)ri + 1u, 4));
    build_bricks(w, 0, 0, 0, 0, w.bricks_x, w.bricks_z, [&](int32_t x, int32_t y, int32_t z) -> uint8_t {
      return y < h[(size_t)z * sx + x] ? STONE : 0;
    });
    int32_t nbox = rng.uniform(1, 4);
    for (int32_t b = 0; b < nbox; ++b) {
      int32_t d = std::min({rng.uniform(8, 32), sx, sz});
      int32_t x0 = rng.uniform(0, sx - d), z0 = rng.uniform(0, sz - d);
      int32_t hmax = 0;
      for (int32_t z = z0; z < z0 + d; ++z)
        for (int32_t x = x0; x < x0 + d; ++x) hmax = std::max(hmax, h[(size_t)z * sx + x]);
      int32_t y0 = hmax + rng.uniform(0, 8);
      int32_t y1 = std::min(sy - 1, y0 + d - 1);
      if (y0 > y1) continue;
      for (int32_t z = z0; z < z0 + d; ++z)
        for (int32_t y = y0; y <= y1; ++y)
          for (int32_t x = x0; x < x0 + d; ++x)
            if (w.get_voxel(x, y, z) == 0) w.set_voxel(x, y, z, WATER);
      r.wakes.push_back({x0 - 1, y0 - 1, z0 - 1, x0 + d, y1 + 1, z0 + d});
    }
    w.compact();
    w.dirty_grid.clear();
    r.sx = sx;
    r.sy = sy;
    r.sz = sz;
    r.edit_seed = rng.next();
    wl.regions.push_back(std::move(r));
  }
  wl.ticks = 600;
}

// Workload 4: ring world. ring_init(16, 256); 9x9 chunks (chunk coords 0..8, scaled down for
// tests) of 128x256x128 each; h = 40 + floor(120 * fbm4(X/256, Z/256, seed 4)); sea fills air
// with y < 64. 1000 rain emitters (x,z uniform over the loaded area, y = first cell above the
// column's top solid or water voxel) each add 1.0 every 4 ticks.
void build_ring(vf_workload& wl, float scale, uint64_t seed) {
  Region r;
  int32_t nch = std::max(1, (int32_t)std::lround(9.0f * scale));
  r.world = std::make_unique<World>(8, 8, 8);
  World& w = *r.world;
  w.ring_init(16, 256);
  const int32_t CH = RING_CHUNK_B * BRICK;  // 128
  auto height = [](int32_t x, int32_t z) { return 40 + (int32_t)std::floor(120.0f * fbm((float)x / 256.0f, (float)z / 256.0f, 4u, 4)); };
  for (int32_t cz = 0; cz < nch; ++cz)
    for (int32_t cx = 0; cx < nch; ++cx) {
      World chunk(CH, 256, CH);
      std::vector<int32_t> h((size_t)CH * CH);
      for (int32_t z = 0; z < CH; ++z)
        for (int32_t x = 0; x < CH; ++x) h[(size_t)z * CH + x] = height(cx * CH + x, cz * CH + z);
      build_bricks(chunk, 0, 0, 0, 0, chunk.bricks_x, chunk.bricks_z, [&](int32_t x, int32_t y, int32_t z) -> uint8_t {
        int32_t hh = h[(size_t)z * CH + x];
        if (y < hh) return STONE;
        return y < 64 ? WATER : 0;
      });
      w.ring_paste(chunk, cx, cz);
    }
  Rng rng(seed * 0x9E3779B97F4A7C15ULL + 4);
  int32_t span = nch * CH;
  int32_t nem = std::max(8, (int32_t)std::lround(1000.0f * scale * scale));
  for (int32_t i = 0; i < nem; ++i) {
    int32_t x = rng.uniform(0, span - 1), z = rng.uniform(0, span - 1);
    int32_t y = std::max(height(x, z), 64);
    if (y >= 256) y = 255;
    r.emitters.push_back({x, y, z});
  }
  r.sx = r.sz = span;
  r.sy = 256;
  wl.ticks = 2000;
  wl.emit_every = 4;
  wl.emit_amount = 1.0f;
  wl.regions.push_back(std::move(r));
}

}  // namespace

// ======================================================================== C ABI
extern "C" {

int vf_world_create(int32_t nx, int32_t ny, int32_t nz, vf_world** out) {
  if (!out || nx <= 0 || ny <= 0 || nz <= 0) return VF_ERR_INVALID;
  auto* h = new (std::nothrow) vf_world();
  if (!h) return VF_ERR_OOM;
  h->w = World(nx, ny, nz);
  *out = h;
  return VF_OK;
}

int vf_world_create_ring(int32_t w, int32_t ny, vf_world** out) {
  if (!out || w <= 0 || (w & (w - 1)) != 0 || ny <= 0) return VF_ERR_INVALID;
  auto* h = new (std::nothrow) vf_world();
  if (!h) return VF_ERR_OOM;
  h->w.ring_init(w, ny);
  *out = h;
  return VF_OK;
}

int vf_world_clone(const vf_world* w, vf_world** out) {
  if (!w || !out) return VF_ERR_INVALID;
  auto* h = new (std::nothrow) vf_world(*w);
  if (!h) return VF_ERR_OOM;
  *out = h;
  return VF_OK;
}

void vf_world_destroy(vf_world* w) { delete w; }

int vf_world_get_info(const vf_world* w, vf_world_info* o) {
  if (!w || !o) return VF_ERR_INVALID;
  const World& v = w->w;
  o->nx = v.nx;
  o->ny = v.ny;
  o->nz = v.nz;
  o->bricks_x = v.bricks_x;
  o->bricks_y = v.bricks_y;
  o->bricks_z = v.bricks_z;
  o->ring_w = v.ring_w;
  o->origin_x = v.origin_x;
  o->origin_z = v.origin_z;
  o->nbricks = v.bricks.size();
  o->detailed = v.detailed();
  return VF_OK;
}

uint8_t vf_world_get_voxel(const vf_world* w, int32_t x, int32_t y, int32_t z) { return w->w.get_voxel(x, y, z); }
void vf_world_set_voxel(vf_world* w, int32_t x, int32_t y, int32_t z, uint8_t m) { w->w.set_voxel(x, y, z, m); }
void vf_world_set_voxels(vf_world* w, const void* changes, uint64_t n) {
  if (!w || !changes) return;
  const unsigned char* p = static_cast<const unsigned char*>(changes);
  for (uint64_t i = 0; i < n; ++i, p += 16) {
    int32_t xyz[3];
    std::memcpy(xyz, p, 12);
    w->w.set_voxel(xyz[0], xyz[1], xyz[2], p[12]);
  }
}
void vf_world_fill_box(vf_world* w, int32_t x0, int32_t y0, int32_t z0, int32_t x1, int32_t y1, int32_t z1, uint8_t m) {
  w->w.fill_box(x0, y0, z0, x1, y1, z1, m);
}
void vf_world_fill_sphere(vf_world* w, float cx, float cy, float cz, float r, uint8_t m) { w->w.fill_sphere(cx, cy, cz, r, m); }
void vf_world_compact(vf_world* w) { w->w.compact(); }
int vf_world_ring_paste(vf_world* ring, const vf_world* chunk, int32_t cx, int32_t cz) {
  if (!ring || !chunk || ring->w.ring_w == 0) return VF_ERR_INVALID;
  ring->w.ring_paste(chunk->w, cx, cz);
  return VF_OK;
}
int vf_world_ring_evict(vf_world* ring, int32_t cx, int32_t cz) {
  if (!ring || ring->w.ring_w == 0) return VF_ERR_INVALID;
  ring->w.ring_evict(cx, cz);
  return VF_OK;
}
int vf_world_ring_rebase(vf_world* ring, int32_t dcx, int32_t dcz) {  // sparse_volume.rs:194-203
  if (!ring || ring->w.ring_w == 0) return VF_ERR_INVALID;
  for (RingSlot& s : ring->w.ring_slots) {
    s.cx -= dcx;
    s.cz -= dcz;
  }
  ring->w.origin_x += dcx * 128;
  ring->w.origin_z += dcz * 128;
  return VF_OK;
}
int vf_world_chunk_loaded(const vf_world* w, int32_t cx, int32_t cz) { return w->w.chunk_loaded(cx, cz) ? 1 : 0; }
const uint32_t* vf_world_grid(const vf_world* w) { return w->w.grid.data(); }
const uint8_t* vf_world_bricks(const vf_world* w) { return w->w.bricks.empty() ? nullptr : w->w.bricks[0].data(); }
int vf_world_ring_slots(const vf_world* w, int32_t* out) {
  const World& v = w->w;
  if (!out) return v.ring_w * v.ring_w;
  for (size_t i = 0; i < v.ring_slots.size(); ++i) {
    out[3 * i] = v.ring_slots[i].cx;
    out[3 * i + 1] = v.ring_slots[i].cz;
    out[3 * i + 2] = v.ring_slots[i].loaded ? 1 : 0;
  }
  return (int)v.ring_slots.size();
}
size_t vf_world_take_dirty(vf_world* w, uint32_t* out, size_t cap) {
  size_t n = w->w.dirty_grid.size();
  if (out) std::memcpy(out, w->w.dirty_grid.data(), std::min(n, cap) * sizeof(uint32_t));
  w->w.dirty_grid.clear();
  return n;
}

int vf_workload_build(int32_t id, float scale, uint64_t seed, vf_workload** out) {
  if (!out || !(scale > 0.0f && scale <= 1.0f)) return VF_ERR_INVALID;
  auto wl = std::make_unique<vf_workload>();
  wl->id = id;
  switch (id) {
    case 1: build_basin(*wl); break;
    case 2: build_dambreak(*wl, scale); break;
    case 3: build_regions(*wl, scale, seed, scale >= 1.0f ? 64 : std::max(2, (int32_t)std::lround(64 * scale))); break;
    case 4: build_ring(*wl, scale, seed); break;
    case 5:
      build_regions(*wl, scale, seed, scale >= 1.0f ? 64 : std::max(2, (int32_t)std::lround(64 * scale)));
      wl->edit_every = 10;
      break;
    default: return VF_ERR_INVALID;
  }
  for (auto& r : wl->regions) {
    r.world->dirty_grid.clear();
    auto h = std::make_unique<vf_world>();
    h->w = *r.world;
    wl->handles.push_back(std::move(h));
  }
  *out = wl.release();
  return VF_OK;
}

void vf_workload_destroy(vf_workload* wl) { delete wl; }

int vf_workload_get_info(const vf_workload* wl, vf_workload_info* o) {
  if (!wl || !o) return VF_ERR_INVALID;
  o->id = wl->id;
  o->regions = (int32_t)wl->regions.size();
  o->ticks = wl->ticks;
  o->emit_every = wl->emit_every;
  o->edit_every = wl->edit_every;
  uint64_t cells = 0;
  for (auto& r : wl->regions) cells += (uint64_t)r.sx * r.sy * r.sz;
  o->resident_cells = cells;
  return VF_OK;
}

const vf_world* vf_workload_world(const vf_workload* wl, int32_t region) {
  if (!wl || region < 0 || region >= (int32_t)wl->handles.size()) return nullptr;
  return wl->handles[region].get();
}

size_t vf_workload_wakes(const vf_workload* wl, int32_t region, int32_t* out6, size_t cap) {
  const auto& w = wl->regions[region].wakes;
  for (size_t i = 0; i < w.size() && i < cap; ++i) std::memcpy(out6 + 6 * i, w[i].data(), 6 * sizeof(int32_t));
  return w.size();
}

size_t vf_workload_emitters(const vf_workload* wl, int32_t region, int32_t* out3, size_t cap, float* amount) {
  const auto& e = wl->regions[region].emitters;
  if (amount) *amount = wl->emit_amount;
  for (size_t i = 0; i < e.size() && i < cap; ++i) std::memcpy(out3 + 3 * i, e[i].data(), 3 * sizeof(int32_t));
  return e.size();
}

// Sphere edit of workload 5: before every tick t (0-based) with t % 10 == 9 each region gets one
// sphere, radius uniform in {4..16}, centre uniform over the region, carve or fill with equal odds.
size_t vf_workload_edit(const vf_workload* wl, int32_t region, int32_t tick, int32_t* out3, size_t cap, uint8_t* m, int32_t* wake6) {
  if (!wl || wl->edit_every <= 0 || (tick % wl->edit_every) != wl->edit_every - 1) return 0;
  const Region& r = wl->regions[region];
  Rng rng(r.edit_seed ^ ((uint64_t)tick * 0xD1B54A32D192ED03ULL));
  float rad = (float)rng.uniform(4, 16);
  float cx = (float)rng.uniform(0, r.sx - 1) + 0.5f, cy = (float)rng.uniform(0, r.sy - 1) + 0.5f, cz = (float)rng.uniform(0, r.sz - 1) + 0.5f;
  bool carve = (rng.next() & 1) != 0;
  size_t n = 0;
  sphere_cells(cx, cy, cz, rad, [&](int32_t x, int32_t y, int32_t z) {
    if (n < cap && out3) {
      out3[3 * n] = x;
      out3[3 * n + 1] = y;
      out3[3 * n + 2] = z;
    }
    ++n;
  });
  if (m) *m = carve ? 0 : STONE;
  if (wake6) {
    wake6[0] = (int32_t)std::floor(cx - rad) - 1;
    wake6[1] = (int32_t)std::floor(cy - rad) - 1;
    wake6[2] = (int32_t)std::floor(cz - rad) - 1;
    wake6[3] = (int32_t)std::ceil(cx + rad) + 1;
    wake6[4] = (int32_t)std::ceil(cy + rad) + 1;
    wake6[5] = (int32_t)std::ceil(cz + rad) + 1;
  }
  return n;
}

}  // extern "C"
