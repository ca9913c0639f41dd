// ORACLE — test infrastructure only (see fluid_oracle.hpp). Each function cites the reference
// lines it restates.
#include "fluid_oracle.hpp"

#include <algorithm>
#include <cmath>
#include <cstring>

namespace orc {

// ============================================================ SparseVolume (sparse_volume.rs)

SparseVolume::SparseVolume(int32_t nx_, int32_t ny_, int32_t nz_) {  // :117-139
  nx = nx_;
  ny = ny_;
  nz = nz_;
  bricks_x = (nx + BRICK - 1) / BRICK;
  bricks_y = (ny + BRICK - 1) / BRICK;
  bricks_z = (nz + BRICK - 1) / BRICK;
  grid.assign((size_t)bricks_x * bricks_y * bricks_z, 0);
}

size_t SparseVolume::grid_index(int32_t ix, int32_t iy, int32_t iz) const {  // :142-148
  if (ring_w != 0) {
    ix &= bricks_x - 1;
    iz &= bricks_z - 1;
  }
  return ((size_t)(uint32_t)iz * (size_t)bricks_y + (size_t)(uint32_t)iy) * (size_t)bricks_x + (size_t)(uint32_t)ix;
}

size_t SparseVolume::ring_slot_index(int32_t cx, int32_t cz) const {  // :152-155
  int32_t m = ring_w - 1;
  return (size_t)(cz & m) * (size_t)ring_w + (size_t)(cx & m);
}

bool SparseVolume::chunk_loaded(int32_t cx, int32_t cz) const {  // :164-170
  if (ring_w == 0) return true;
  const RingSlot& s = ring_slots[ring_slot_index(cx, cz)];
  return s.loaded && s.cx == cx && s.cz == cz;
}

// The floating origin moves by (dcx, dcz) chunks: every slot's owner moves, the bricks stay.
void SparseVolume::ring_rebase(int32_t dcx, int32_t dcz) {  // :194-203
  for (auto& s : ring_slots) {
    s.cx -= dcx;
    s.cz -= dcz;
  }
  origin_x += dcx * RING_CHUNK_B * BRICK;
  origin_z += dcz * RING_CHUNK_B * BRICK;
}

bool SparseVolume::loaded_at(int32_t x, int32_t z) const {  // :173-175
  return ring_w == 0 || chunk_loaded(x >> 7, z >> 7);
}

void SparseVolume::ring_init(int32_t w, int32_t ny_) {  // :177-192
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

void SparseVolume::mark_modified(size_t gi) {  // :218-225
  if (ring_w == 0) return;
  size_t bxy = (size_t)bricks_x * bricks_y;
  size_t i = ((gi / bxy) / RING_CHUNK_B) * ring_w + (gi % bricks_x) / RING_CHUNK_B;
  ring_slots[i].modified = true;
}

bool SparseVolume::inside(int32_t x, int32_t y, int32_t z) const {  // :229-235
  if (ring_w != 0) return (uint32_t)y < (uint32_t)ny && chunk_loaded(x >> 7, z >> 7);
  return (uint32_t)x < (uint32_t)nx && (uint32_t)y < (uint32_t)ny && (uint32_t)z < (uint32_t)nz;
}

uint8_t SparseVolume::get_voxel(int32_t x, int32_t y, int32_t z) const {  // :238-247
  if (!inside(x, y, z)) return 0;
  uint32_t v = grid[grid_index(x >> 3, y >> 3, z >> 3)];
  if (v < 256) return (uint8_t)v;
  return bricks[v - 256][(z & 7) * 64 + (y & 7) * 8 + (x & 7)];
}

size_t SparseVolume::materialize(size_t gi, uint8_t fill) {  // :250-266
  size_t idx;
  if (!free_bricks.empty()) {
    idx = free_bricks.back();
    free_bricks.pop_back();
    bricks[idx].fill(fill);
  } else {
    bricks.emplace_back();
    bricks.back().fill(fill);
    idx = bricks.size() - 1;
  }
  grid[gi] = 256 + (uint32_t)idx;
  return idx;
}

void SparseVolume::set_voxel(int32_t x, int32_t y, int32_t z, uint8_t m) {  // :268-293
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

void SparseVolume::fill_sphere(float cx, float cy, float cz, float r, uint8_t m) {  // :295-316
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
        if (dx * dx <= rem) set_voxel(x, y, z, m);
      }
    }
  }
}

void SparseVolume::fill_box(int32_t x0, int32_t y0, int32_t z0, int32_t x1, int32_t y1, int32_t z1, uint8_t m) {  // :318-326
  for (int32_t z = z0; z <= z1; ++z)
    for (int32_t y = y0; y <= y1; ++y)
      for (int32_t x = x0; x <= x1; ++x) set_voxel(x, y, z, m);
}

void SparseVolume::compact() {  // :339-350
  for (size_t gi = 0; gi < grid.size(); ++gi) {
    uint32_t v = grid[gi];
    if (v < 256) continue;
    const auto& b = bricks[v - 256];
    bool uni = std::all_of(b.begin(), b.end(), [&](uint8_t c) { return c == b[0]; });
    if (uni) {
      grid[gi] = b[0];
      free_bricks.push_back(v - 256);
    }
  }
}

void SparseVolume::ring_paste(const SparseVolume& src, int32_t cx, int32_t cz) {  // :478-510
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
        size_t idx;
        if (!free_bricks.empty()) {
          idx = free_bricks.back();
          free_bricks.pop_back();
          bricks[idx] = src.bricks[v - 256];
        } else {
          bricks.push_back(src.bricks[v - 256]);
          idx = bricks.size() - 1;
        }
        grid[gi] = 256 + (uint32_t)idx;
      }
  ring_slots[ring_slot_index(cx, cz)] = RingSlot{cx, cz, true, false};
}

void SparseVolume::ring_evict(int32_t cx, int32_t cz) {  // :513-537
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

// ====================================================================== PartialField (:64-180)

static inline uint64_t page_key(int32_t x, int32_t y, int32_t z) { return key(x >> 3, y >> 3, z >> 3); }  // :83-85
static inline size_t local_index(int32_t x, int32_t y, int32_t z) { return (size_t)((x & 7) | (y & 7) << 3 | (z & 7) << 6); }  // :87-89

int64_t PartialField::page(uint64_t k) const {  // :91-101 (one-entry last-page cache)
  uint32_t i;
  if (last_k_ == k) {
    i = last_i_;
  } else {
    uint32_t* p = index_.find(k);
    i = p ? *p + 1 : 0;
    last_k_ = k;
    last_i_ = i;
  }
  return i != 0 ? (int64_t)(i - 1) : -1;
}

float PartialField::get(int32_t x, int32_t y, int32_t z) const {  // :103-105
  int64_t p = page(page_key(x, y, z));
  return p < 0 ? 0.0f : pages_[p].v[local_index(x, y, z)];
}

void PartialField::set(int32_t x, int32_t y, int32_t z, float v) {  // :108-136
  uint64_t k = page_key(x, y, z);
  int64_t p = page(k);
  if (p < 0) {
    uint32_t i;
    if (!free_.empty()) {
      i = free_.back();
      free_.pop_back();
      std::memset(&pages_[i], 0, sizeof(Page));
    } else {
      pages_.emplace_back();
      std::memset(&pages_.back(), 0, sizeof(Page));
      i = (uint32_t)pages_.size() - 1;
    }
    index_.insert(k, i);
    last_k_ = k;
    last_i_ = i + 1;
    p = i;
  }
  Page& page = pages_[p];
  float& c = page.v[local_index(x, y, z)];
  if (c <= 0.0f) {
    page.count += 1;
    count_ += 1;
  }
  c = v;
}

void PartialField::erase(int32_t x, int32_t y, int32_t z) {  // :138-154
  uint64_t k = page_key(x, y, z);
  int64_t p = page(k);
  if (p < 0) return;
  Page& page = pages_[p];
  float& c = page.v[local_index(x, y, z)];
  if (c <= 0.0f) return;
  c = 0.0f;
  count_ -= 1;
  page.count -= 1;
  if (page.count == 0) {
    index_.erase(k);
    free_.push_back((uint32_t)p);
    last_k_ = ~0ULL;
    last_i_ = 0;
  }
}

void PartialField::clear() {  // :160-162
  index_.clear();
  pages_.clear();
  free_.clear();
  last_k_ = ~0ULL;
  last_i_ = 0;
  count_ = 0;
}

// ======================================================================= LayerMarks (:182-207)

bool LayerMarks::test(int32_t x, int32_t y, int32_t z) const {
  uint64_t tk = field(x >> 6) | field(y) << 21 | field(z >> 6) << 42;
  auto* slot = tiles_.find(tk);
  if (!slot || !*slot) return false;
  return ((**slot)[(size_t)(z & 63)] >> (x & 63)) & 1ULL;
}

bool LayerMarks::test_and_set(int32_t x, int32_t y, int32_t z) {  // :194-200
  uint64_t tk = field(x >> 6) | field(y) << 21 | field(z >> 6) << 42;  // :190-192
  auto* slot = tiles_.find(tk);
  if (!slot) slot = tiles_.insert(tk, std::make_shared<std::array<uint64_t, 64>>()).first;
  if (!*slot) *slot = std::make_shared<std::array<uint64_t, 64>>();
  auto& t = **slot;
  size_t w = (size_t)(z & 63);
  uint64_t b = 1ULL << (x & 63);
  bool was = (t[w] & b) != 0;
  t[w] |= b;
  return was;
}

// ========================================================================= FluidSim (:230-721)

static constexpr float SHOW_AT = 0.5f;
static constexpr float HIDE_BELOW = 0.3f;
static constexpr float EVAPORATE = 1e-4f;
static constexpr float MIN_SPREAD = 0.05f;
static constexpr float MIN_FLOW = 1e-4f;
static constexpr float SLEEP = 1e-3f;
static constexpr float TICK_HZ = 20.0f;
static constexpr size_t MAX_CELLS_PER_TICK = 50000;
static constexpr uint32_t LEVEL_TICKS = 10;
static constexpr size_t MAX_LEVEL_CELLS = 400000;
static constexpr size_t PRESSURE_SEARCH = 512;
static constexpr size_t MAX_PULLS_PER_TICK = 4096;
static constexpr size_t LEVEL_BUDGET = 40000;
static constexpr size_t MAX_LEVEL_SEEDS = 4096;
// `1.0 - 1e-4` with f32 operands, folded in f32 as Rust does.
static const float FULL = 1.0f - 1e-4f;

static const int32_t SIDES[4][2] = {{1, 0}, {-1, 0}, {0, 1}, {0, -1}};  // :228

static inline bool outside(const SparseVolume& v, int32_t x, int32_t y, int32_t z) {  // :212-217
  if (y < 0 || y >= v.ny) return true;
  if (v.ring_w != 0) return !v.loaded_at(x, z);
  return x < 0 || z < 0 || x >= v.nx || z >= v.nz;
}

static inline bool solid(const SparseVolume& v, int32_t x, int32_t y, int32_t z) {  // :220-226
  if (outside(v, x, y, z)) return true;
  uint8_t m = v.get_voxel(x, y, z);
  return m != 0 && m != WATER;
}

float FluidSim::volume(const SparseVolume& v, int32_t x, int32_t y, int32_t z) const {  // :251-260
  if (outside(v, x, y, z)) return 0.0f;
  float p = partial_.get(x, y, z);
  if (p > 0.0f) return p;
  return v.get_voxel(x, y, z) == WATER ? 1.0f : 0.0f;
}

void FluidSim::set_partial(int32_t x, int32_t y, int32_t z, float v) {  // :278-282
  if (v > 0.0f && v < 1.0f) partial_.set(x, y, z, v);
}

void FluidSim::activate(int32_t x, int32_t y, int32_t z) {  // :292-300
  if (y < 0) return;
  uint64_t k = key(x, y, z);
  if (active_.insert(k)) {
    queue_.push_back(k);
    stats.activations++;
  }
}

void FluidSim::wake_around(int32_t x, int32_t y, int32_t z) {  // :302-310
  activate(x, y, z);
  activate(x + 1, y, z);
  activate(x - 1, y, z);
  activate(x, y + 1, z);
  activate(x, y - 1, z);
  activate(x, y, z + 1);
  activate(x, y, z - 1);
}

void FluidSim::seed_level(uint64_t k) {  // :312-316
  if (!level_round_ && level_seeds_.size() < MAX_LEVEL_SEEDS && level_seeds_.insert(k)) level_seed_list_.push_back(k);
}

void FluidSim::reset() {  // :318-320
  Stats s = stats;
  *this = FluidSim();
  stats = s;
}

bool FluidSim::supported(const SparseVolume& v, int32_t x, int32_t y, int32_t z) const {  // :322-324
  return solid(v, x, y - 1, z) || volume(v, x, y - 1, z) >= FULL;
}

bool FluidSim::set_volume(SparseVolume& v, int32_t x, int32_t y, int32_t z, float vol) {  // :327-355
  bool is_water = v.get_voxel(x, y, z) == WATER;
  if (vol <= 1e-6f) {
    partial_.erase(x, y, z);
    if (is_water) {
      v.set_voxel(x, y, z, 0);
      return true;
    }
    return false;
  }
  if (vol >= FULL) {
    partial_.erase(x, y, z);
    if (!is_water) {
      v.set_voxel(x, y, z, WATER);
      return true;
    }
    return false;
  }
  partial_.set(x, y, z, vol);
  if (is_water && vol < HIDE_BELOW) {
    v.set_voxel(x, y, z, 0);
    return true;
  }
  if (!is_water && vol >= SHOW_AT) {
    v.set_voxel(x, y, z, WATER);
    return true;
  }
  return false;
}

void FluidSim::wake(int32_t x0, int32_t y0, int32_t z0, int32_t x1, int32_t y1, int32_t z1) {  // :358-366
  for (int32_t z = z0; z <= z1; ++z)
    for (int32_t y = y0; y <= y1; ++y)
      for (int32_t x = x0; x <= x1; ++x) activate(x, y, z);
}

void FluidSim::displace(SparseVolume& v, int32_t x, int32_t y, int32_t z) {  // :370-408
  float amount = volume(v, x, y, z);
  partial_.erase(x, y, z);
  wake(x - 1, y - 1, z - 1, x + 1, y + 1, z + 1);
  if (amount <= 0.0f) return;
  int32_t yy = y + 1;
  while (yy < v.ny && amount > 1e-6f) {
    if (solid(v, x, yy, z)) break;
    float cur = volume(v, x, yy, z);
    float take = std::min(amount, 1.0f - cur);
    if (take > 0.0f) {
      set_volume(v, x, yy, z, cur + take);
      amount -= take;
      activate(x, yy, z);
    }
    yy += 1;
  }
  for (auto& s : SIDES) {
    if (amount <= 1e-6f) break;
    int32_t nx = x + s[0], nz = z + s[1];
    if (solid(v, nx, y, nz)) continue;
    float cur = volume(v, nx, y, nz);
    float take = std::min(amount, 1.0f - cur);
    if (take > 0.0f) {
      set_volume(v, nx, y, nz, cur + take);
      amount -= take;
      activate(nx, y, nz);
    }
  }
}

void FluidSim::emit(SparseVolume& v, int32_t x, int32_t y, int32_t z, float amount) {
  if (solid(v, x, y, z)) return;
  float cur = volume(v, x, y, z);
  float nv = std::min(1.0f, cur + amount);
  set_volume(v, x, y, z, nv);
  wake(x, y, z, x, y, z);
}

bool FluidSim::level_layer(SparseVolume& v, int32_t sx, int32_t sy, int32_t sz) {  // :412-486
  auto member = [&](int32_t x, int32_t y, int32_t z) {
    return !solid(v, x, y, z) && volume(v, x, y, z) > 0.0f && supported(v, x, y, z) && volume(v, x, y + 1, z) <= 0.0f;
  };
  stats.level_calls++;
  if (level_visited_.test_and_set(sx, sy, sz) || !member(sx, sy, sz)) return false;
  std::vector<uint64_t> cells;
  cells.swap(level_cells_);
  cells.clear();
  cells.push_back(key(sx, sy, sz));
  double sum = 0.0;
  float lo = 2.0f, hi = -1.0f;
  size_t i = 0;
  while (i < cells.size()) {
    int32_t x, y, z;
    unkey(cells[i], x, y, z);
    i += 1;
    float vol = volume(v, x, y, z);
    sum += (double)vol;
    lo = std::min(lo, vol);
    hi = std::max(hi, vol);
    if (cells.size() >= MAX_LEVEL_CELLS) continue;
    for (auto& s : SIDES) {
      int32_t nx = x + s[0], nz = z + s[1];
      if (v.ring_w == 0 && (nx < 0 || nz < 0)) continue;
      if (level_visited_.test_and_set(nx, y, nz) || !member(nx, y, nz)) continue;
      cells.push_back(key(nx, y, nz));
    }
  }
  last_level_cells_ += cells.size();
  stats.level_cells += cells.size();
  stats.level_fills++;
  bool changed = false;
  if (cells.size() >= 2 && hi - lo >= SLEEP) {
    float avg = (float)(sum / (double)cells.size());
    if (avg >= MIN_SPREAD) {
      for (uint64_t k : cells) {
        int32_t x, y, z;
        unkey(k, x, y, z);
        if (std::fabs(volume(v, x, y, z) - avg) > 1e-6f) changed |= set_volume(v, x, y, z, avg);
      }
    } else {
      stats.drains++;
      double left = sum;
      for (uint64_t k : cells) {
        int32_t x, y, z;
        unkey(k, x, y, z);
        if (y == 0 || solid(v, x, y - 1, z)) continue;
        float below = volume(v, x, y - 1, z);
        float take = (float)std::min(left, (double)(1.0f - below));
        if (take <= 0.0f) continue;
        changed |= set_volume(v, x, y - 1, z, below + take);
        left -= (double)take;
        activate(x, y - 1, z);
        if (left <= 1e-6) break;
      }
      float rest = (float)(left / (double)cells.size());
      for (uint64_t k : cells) {
        int32_t x, y, z;
        unkey(k, x, y, z);
        changed |= set_volume(v, x, y, z, rest < EVAPORATE ? 0.0f : rest);
      }
    }
  }
  level_cells_.swap(cells);
  return changed;
}

bool FluidSim::level_surfaces(SparseVolume& v) {  // :489-507
  last_level_cells_ = 0;
  bool changed = false;
  while (last_level_cells_ < LEVEL_BUDGET) {
    if (level_seed_list_.empty()) break;
    uint64_t k = level_seed_list_.back();
    level_seed_list_.pop_back();
    level_seeds_.remove(k);
    int32_t x, y, z;
    unkey(k, x, y, z);
    while (y + 1 < v.ny && !solid(v, x, y + 1, z) && volume(v, x, y + 1, z) > 0.0f) y += 1;
    changed |= level_layer(v, x, y, z);
  }
  level_round_ = !level_seed_list_.empty();
  if (!level_round_) level_visited_.clear();
  return changed;
}

float FluidSim::pressure_pull(SparseVolume& v, int32_t x, int32_t y, int32_t z, float need) {  // :511-561
  static const int32_t D[5][3] = {{0, 1, 0}, {1, 0, 0}, {-1, 0, 0}, {0, 0, 1}, {0, 0, -1}};
  auto full = [&](int32_t a, int32_t b, int32_t c) { return !solid(v, a, b, c) && volume(v, a, b, c) >= FULL; };
  std::vector<uint64_t> queue;
  queue.swap(press_queue_);
  queue.clear();
  press_visited_.clear();
  press_visited_.insert(key(x, y, z));
  for (auto& d : D) {
    int32_t a = x + d[0], b = y + d[1], c = z + d[2];
    if (a < 0 || c < 0 || !full(a, b, c)) continue;
    queue.push_back(key(a, b, c));
    press_visited_.insert(key(a, b, c));
  }
  if (!queue.empty()) stats.pull_nonempty++;
  int side_at_start = 0;
  float got = 0.0f;
  size_t i = 0;
  while (i < queue.size() && i < PRESSURE_SEARCH) {
    int32_t a, b, c;
    unkey(queue[i], a, b, c);
    i += 1;
    float here = volume(v, a, b, c);
    bool top = b + 1 >= v.ny || solid(v, a, b + 1, c) || volume(v, a, b + 1, c) <= 0.0f;
    if (top && b > y && here > 0.0f) {
      float take = std::min(need, here);
      set_volume(v, a, b, c, here - take);
      activate(a, b, c);
      seed_level(key(a, b, c));
      got = take;
      break;
    }
    for (auto& d : D) {
      int32_t na = a + d[0], nb = b + d[1], nc = c + d[2];
      if (na < 0 || nc < 0 || nb >= v.ny || solid(v, na, nb, nc) || volume(v, na, nb, nc) <= 0.0f) continue;
      if (nb == y && d[1] == 0) {
        side_at_start += 1;
        if (side_at_start > 24) continue;
      }
      if (!press_visited_.insert(key(na, nb, nc))) continue;
      queue.push_back(key(na, nb, nc));
    }
  }
  stats.bfs_visits += i;
  press_queue_.swap(queue);
  return got;
}

bool FluidSim::tick(SparseVolume& v) {  // :564-657
  tick_no_ += 1;
  stats.ticks++;
  size_t n = std::min(queue_.size(), MAX_CELLS_PER_TICK);
  std::vector<uint64_t> cells(queue_.begin(), queue_.begin() + (ptrdiff_t)n);
  queue_.erase(queue_.begin(), queue_.begin() + (ptrdiff_t)n);
  for (uint64_t k : cells) active_.remove(k);
  bool flip = (tick_no_ & 1) != 0;
  // Sort by (y, z, x), or (y, -z, -x) on odd ticks. Keys are unique, so the order is total.
  std::vector<std::pair<std::array<int32_t, 3>, uint64_t>> sk(n);
  for (size_t i = 0; i < n; ++i) {
    int32_t x, y, z;
    unkey(cells[i], x, y, z);
    if (flip) {
      x = -x;
      z = -z;
    }
    sk[i] = {{y, z, x}, cells[i]};
  }
  std::sort(sk.begin(), sk.end(), [](const auto& a, const auto& b) { return a.first < b.first; });
  for (size_t i = 0; i < n; ++i) cells[i] = sk[i].second;
  last_cells_ = cells.size();
  stats.cells += cells.size();
  bool changed = false;
  size_t pulls = 0;
  for (uint64_t k : cells) {
    int32_t x, y, z;
    unkey(k, x, y, z);
    if (solid(v, x, y, z)) {
      partial_.erase(x, y, z);
      continue;
    }
    float vol = volume(v, x, y, z);
    float v0 = vol;
    if (vol < FULL && pulls < MAX_PULLS_PER_TICK) {
      float got = pressure_pull(v, x, y, z, 1.0f - vol);
      pulls += 1;
      stats.pull_attempts++;
      if (got > 0.0f) {
        stats.pull_success++;
        vol += got;
        wake_around(x, y, z);
      }
    }
    if (vol <= 0.0f) continue;
    if (!solid(v, x, y - 1, z)) {
      float below = volume(v, x, y - 1, z);
      float f = std::min(vol, 1.0f - below);
      if (f > 1e-6f) {
        changed |= set_volume(v, x, y - 1, z, below + f);
        vol -= f;
        wake_around(x, y - 1, z);
      }
    }
    if (vol > MIN_SPREAD && supported(v, x, y, z)) {
      float nv[4] = {0, 0, 0, 0};
      bool open[4] = {false, false, false, false};
      for (int i = 0; i < 4; ++i) {
        open[i] = !solid(v, x + SIDES[i][0], y, z + SIDES[i][1]);
        nv[i] = open[i] ? volume(v, x + SIDES[i][0], y, z + SIDES[i][1]) : 0.0f;
      }
      float here = vol;
      for (int i = 0; i < 4; ++i) {
        if (!open[i] || nv[i] >= here) continue;
        float f = (here - nv[i]) * 0.2f;
        if (f < MIN_FLOW || here - f < MIN_SPREAD * 0.5f) continue;
        changed |= set_volume(v, x + SIDES[i][0], y, z + SIDES[i][1], nv[i] + f);
        vol -= f;
        if (f > SLEEP) wake_around(x + SIDES[i][0], y, z + SIDES[i][1]);
      }
    }
    if (vol < EVAPORATE) vol = 0.0f;
    if (std::fabs(vol - v0) > 1e-7f) changed |= set_volume(v, x, y, z, vol);
    if (std::fabs(vol - v0) > SLEEP) {
      wake_around(x, y, z);
      seed_level(k);
    }
  }
  if (level_round_ || tick_no_ % LEVEL_TICKS == 0) {
    changed |= level_surfaces(v);
    // shrink_tables (:679-692) only trims capacities: no effect on results.
  }
  return changed;
}

bool FluidSim::update(SparseVolume& v, float dt) {  // :662-676
  if (idle()) {
    acc_ = 0.0f;
    return false;
  }
  acc_ = std::min(acc_ + std::min(dt, 0.25f), 3.0f / TICK_HZ);
  bool changed = false;
  int n = 0;
  while (acc_ >= 1.0f / TICK_HZ && n < 3) {
    acc_ -= 1.0f / TICK_HZ;
    changed |= tick(v);
    n += 1;
  }
  return changed;
}

void FluidSim::shift(int32_t dx, int32_t dz) {  // :696-720
  struct C { int32_t x, y, z; float v; };
  std::vector<C> cells;
  cells.reserve(partial_.len());
  partial_.for_each([&](int32_t x, int32_t y, int32_t z, float val) { cells.push_back({x - dx, y, z - dz, val}); });
  partial_.clear();
  for (auto& c : cells) partial_.set(c.x, c.y, c.z, c.v);
  auto mv = [&](uint64_t k) {
    int32_t x, y, z;
    unkey(k, x, y, z);
    return key(x - dx, y, z - dz);
  };
  U64Set na;
  active_.for_each([&](uint64_t k) { na.insert(mv(k)); });
  active_ = na;
  for (auto& k : level_seed_list_) k = mv(k);
  level_seeds_.clear();
  for (auto k : level_seed_list_) level_seeds_.insert(k);
  for (auto& k : queue_) k = mv(k);
  level_visited_.clear();
  level_cells_.clear();
  press_queue_.clear();
  press_visited_.clear();
  level_round_ = false;
}

size_t FluidSim::apply_brush(SparseVolume& v, const int32_t* xyz, size_t n, uint8_t m) {  // brush.rs:93-111
  size_t changed = 0;
  for (size_t i = 0; i < n; ++i) {
    int32_t x = xyz[3 * i], y = xyz[3 * i + 1], z = xyz[3 * i + 2];
    if (!v.inside(x, y, z)) continue;  // in_brush_world: the voxel must be addressable
    uint8_t cur = v.get_voxel(x, y, z);
    bool empty = cur == 0 || cur == WATER;
    if ((m == 0) == empty) continue;
    if (cur == WATER) displace(v, x, y, z);
    v.set_voxel(x, y, z, m);
    changed++;
  }
  return changed;
}

}  // namespace orc
