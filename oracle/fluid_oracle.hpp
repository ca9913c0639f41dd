// ORACLE — test infrastructure only. Not part of the product and never linked into it.
//
// A CPU restatement of the reference's CA water and the storage it steps:
//   * src/fluid.rs:18-721        (constants, key packing, PartialField, LayerMarks, FluidSim)
//   * src/voxel/sparse_volume.rs (bounded + ring storage, get/set_voxel, fill_box/fill_sphere,
//                                 compact, ring_paste/ring_evict)
//   * src/hash.rs:9-30           (fmix64 hashing of u64 keys; performance only)
//
// Only tests/, __graft_entry__.smoke() and bench.py's cpu_baseline leg use it, as the checker
// of the CUDA path and as the timed CPU baseline.
//
// Parity pin: the reference has no numeric golden vectors for this path and its Rust crate
// cannot be built here (no cargo/rustc). The restatement is pinned by a line-by-line review
// against fluid.rs and by ports of the reference's own property tests (src/fluid.rs:723-818,
// src/voxel/sparse_volume.rs:639-699); bit-level parity with fluid.rs itself is therefore
// "parity unpinned" by reference outputs.
//
// Floating point: f32 for volumes, f64 exactly where fluid.rs uses f64; built with
// -ffp-contract=off and no fast-math so every operation rounds as Rust's does.
#pragma once
#include <cstdint>
#include <cstddef>
#include <deque>
#include <vector>
#include <array>
#include <memory>

namespace orc {

// ---------------------------------------------------------------- hashing (src/hash.rs:21-29)
inline uint64_t fmix64(uint64_t k) {
  k ^= k >> 33;
  k *= 0xff51afd7ed558ccdULL;
  k ^= k >> 33;
  k *= 0xc4ceb9fe1a85ec53ULL;
  k ^= k >> 33;
  return k;
}

// Open-addressing u64 set / map (linear probing, backward-shift delete). Stands in for the
// reference's VoxSet / VoxMap (std HashSet/HashMap with the fmix64 hasher). Only membership
// and lookup are semantic; tick() never iterates these containers (src/fluid.rs:564-657).
template <class V>
class U64Map {
 public:
  static constexpr uint64_t EMPTY = ~0ULL;
  U64Map() { rehash(16); }
  size_t size() const { return n_; }
  bool empty() const { return n_ == 0; }
  void clear() { std::fill(keys_.begin(), keys_.end(), EMPTY); n_ = 0; }
  const V* find(uint64_t k) const { return const_cast<U64Map*>(this)->find(k); }
  V* find(uint64_t k) {
    size_t m = keys_.size() - 1, i = fmix64(k) & m;
    while (true) {
      if (keys_[i] == k) return &vals_[i];
      if (keys_[i] == EMPTY) return nullptr;
      i = (i + 1) & m;
    }
  }
  // Returns (slot value pointer, inserted?)
  std::pair<V*, bool> insert(uint64_t k, const V& v) {
    if ((n_ + 1) * 8 > keys_.size() * 7) rehash(keys_.size() * 2);
    size_t m = keys_.size() - 1, i = fmix64(k) & m;
    while (true) {
      if (keys_[i] == k) return {&vals_[i], false};
      if (keys_[i] == EMPTY) {
        keys_[i] = k;
        vals_[i] = v;
        ++n_;
        return {&vals_[i], true};
      }
      i = (i + 1) & m;
    }
  }
  bool erase(uint64_t k) {
    size_t m = keys_.size() - 1, i = fmix64(k) & m;
    while (true) {
      if (keys_[i] == EMPTY) return false;
      if (keys_[i] == k) break;
      i = (i + 1) & m;
    }
    // backward-shift deletion
    size_t j = i;
    while (true) {
      j = (j + 1) & m;
      if (keys_[j] == EMPTY) break;
      size_t h = fmix64(keys_[j]) & m;
      // can keys_[j] move to i? (h not cyclically in (i, j])
      bool move = (i <= j) ? (h <= i || h > j) : (h <= i && h > j);
      if (move) {
        keys_[i] = keys_[j];
        vals_[i] = std::move(vals_[j]);
        i = j;
      }
    }
    keys_[i] = EMPTY;
    vals_[i] = V();
    --n_;
    return true;
  }
  template <class F>
  void for_each(F f) const {
    for (size_t i = 0; i < keys_.size(); ++i)
      if (keys_[i] != EMPTY) f(keys_[i], vals_[i]);
  }
  size_t capacity() const { return keys_.size(); }

 private:
  void rehash(size_t cap) {
    std::vector<uint64_t> ok;
    std::vector<V> ov;
    ok.swap(keys_);
    ov.swap(vals_);
    keys_.assign(cap, EMPTY);
    vals_.resize(cap);
    n_ = 0;
    for (size_t i = 0; i < ok.size(); ++i)
      if (ok[i] != EMPTY) insert(ok[i], std::move(ov[i]));
  }
  std::vector<uint64_t> keys_;
  std::vector<V> vals_;
  size_t n_ = 0;
};

struct Unit {};
class U64Set {
 public:
  bool insert(uint64_t k) { return m_.insert(k, Unit{}).second; }
  bool remove(uint64_t k) { return m_.erase(k); }
  bool contains(uint64_t k) { return m_.find(k) != nullptr; }
  size_t size() const { return m_.size(); }
  bool empty() const { return m_.empty(); }
  void clear() { m_.clear(); }
  template <class F>
  void for_each(F f) const { m_.for_each([&](uint64_t k, const Unit&) { f(k); }); }

 private:
  U64Map<Unit> m_;
};

// ------------------------------------------------------ sparse volume (src/voxel/sparse_volume.rs)
constexpr int BRICK = 8;
constexpr int RING_CHUNK_B = 16;

struct RingSlot {
  int32_t cx = 0, cz = 0;
  bool loaded = false, modified = false;
};

struct SparseVolume {
  int32_t nx = 0, ny = 0, nz = 0;
  int32_t bricks_x = 0, bricks_y = 0, bricks_z = 0;
  std::vector<uint32_t> grid;
  std::vector<std::array<uint8_t, 512>> bricks;
  std::vector<uint32_t> dirty_grid;
  bool track_dirty = true;
  int32_t ring_w = 0;
  std::vector<RingSlot> ring_slots;
  int32_t origin_x = 0, origin_z = 0;
  std::vector<uint32_t> free_bricks;

  SparseVolume() = default;
  SparseVolume(int32_t nx, int32_t ny, int32_t nz);                   // :117-139
  size_t grid_index(int32_t ix, int32_t iy, int32_t iz) const;       // :142-148
  size_t ring_slot_index(int32_t cx, int32_t cz) const;              // :152-155
  bool chunk_loaded(int32_t cx, int32_t cz) const;                   // :164-170
  bool loaded_at(int32_t x, int32_t z) const;                        // :173-175
  void ring_init(int32_t w, int32_t ny);                             // :177-192
  void ring_rebase(int32_t dcx, int32_t dcz);                        // :194-203
  bool inside(int32_t x, int32_t y, int32_t z) const;                // :229-235
  uint8_t get_voxel(int32_t x, int32_t y, int32_t z) const;          // :238-247
  size_t materialize(size_t gi, uint8_t fill);                       // :250-266
  void set_voxel(int32_t x, int32_t y, int32_t z, uint8_t m);        // :268-293
  void fill_sphere(float cx, float cy, float cz, float r, uint8_t m);  // :295-316
  void fill_box(int32_t x0, int32_t y0, int32_t z0, int32_t x1, int32_t y1, int32_t z1, uint8_t m);  // :318-326
  void compact();                                                     // :339-350
  void ring_paste(const SparseVolume& src, int32_t cx, int32_t cz);  // :478-510
  void ring_evict(int32_t cx, int32_t cz);                           // :513-537
  size_t detailed_bricks() const { return bricks.size() - free_bricks.size(); }
  void mark_modified(size_t gi);                                      // :218-225
};

// ------------------------------------------------------------------- fluid (src/fluid.rs)
constexpr uint8_t WATER = 5;

struct Page {
  float v[512];
  uint32_t count;
};

// src/fluid.rs:64-180
class PartialField {
 public:
  float get(int32_t x, int32_t y, int32_t z) const;
  void set(int32_t x, int32_t y, int32_t z, float v);
  void erase(int32_t x, int32_t y, int32_t z);
  size_t len() const { return count_; }
  void clear();
  // f(x, y, z, v) for every entry: pages in index-table order, cells in local order.
  template <class F>
  void for_each(F f) const;
  size_t pages() const { return index_.size(); }

 private:
  int64_t page(uint64_t k) const;
  mutable U64Map<uint32_t> index_;
  std::vector<Page> pages_;
  std::vector<uint32_t> free_;
  mutable uint64_t last_k_ = ~0ULL;
  mutable uint32_t last_i_ = 0;
  size_t count_ = 0;
};

// src/fluid.rs:182-207
class LayerMarks {
 public:
  bool test_and_set(int32_t x, int32_t y, int32_t z);
  bool test(int32_t x, int32_t y, int32_t z) const;  // read-only probe (inspection only)
  void clear() { tiles_.clear(); }
  size_t tiles() const { return tiles_.size(); }

 private:
  U64Map<std::shared_ptr<std::array<uint64_t, 64>>> tiles_;
};

// Counters for the measurement plan (no effect on results).
struct Stats {
  uint64_t cells = 0;          // cells drained and processed (fluid.rs last_cells, summed)
  uint64_t pull_attempts = 0;  // pressure_pull calls (counted toward MAX_PULLS_PER_TICK)
  uint64_t pull_nonempty = 0;  // pulls whose BFS queue got at least one start cell
  uint64_t pull_success = 0;   // pulls that took water
  uint64_t bfs_visits = 0;     // BFS queue entries examined by pulls
  uint64_t level_calls = 0;    // level_layer calls
  uint64_t level_cells = 0;    // cells gathered by level_layer flood fills
  uint64_t level_fills = 0;    // level_layer calls that gathered >= 1 cell
  uint64_t drains = 0;         // film drains (avg < MIN_SPREAD branch)
  uint64_t activations = 0;    // FIFO pushes
  uint64_t ticks = 0;
};

class FluidSim {
 public:
  float volume(const SparseVolume& v, int32_t x, int32_t y, int32_t z) const;  // :251-260
  size_t active_count() const { return active_.size(); }
  bool idle() const { return active_.empty() && level_seeds_.empty(); }
  size_t partial_count() const { return partial_.len(); }
  size_t last_tick_cells() const { return last_cells_; }
  const PartialField& partials() const { return partial_; }
  void set_partial(int32_t x, int32_t y, int32_t z, float v);                   // :278-282
  void reset();
  void wake(int32_t x0, int32_t y0, int32_t z0, int32_t x1, int32_t y1, int32_t z1);  // :358-366
  void displace(SparseVolume& v, int32_t x, int32_t y, int32_t z);              // :370-408
  bool tick(SparseVolume& v);                                                   // :564-657
  bool update(SparseVolume& v, float dt);                                       // :662-676
  void shift(int32_t dx, int32_t dz);                                           // :696-720
  // Harness edit used by the rain-emitter workload: vol' = min(1, vol + amount) written
  // through set_volume, then the cell is woken (the reference has no emitter API).
  void emit(SparseVolume& v, int32_t x, int32_t y, int32_t z, float amount);

  // Inspection for differential tests.
  const std::deque<uint64_t>& queue() const { return queue_; }
  const std::vector<uint64_t>& seed_list() const { return level_seed_list_; }
  uint32_t tick_no() const { return tick_no_; }
  bool level_round() const { return level_round_; }
  size_t last_level_cells() const { return last_level_cells_; }
  float acc() const { return acc_; }
  bool layer_mark(int32_t x, int32_t y, int32_t z) const { return level_visited_.test(x, y, z); }
  // Harness edit: the reference's apply_brush (src/edit/brush.rs:93-111) with displace as the
  // on_water hook (src/app/scene_edit.rs:231-232), over an explicit cell list.
  size_t apply_brush(SparseVolume& v, const int32_t* xyz, size_t n, uint8_t m);
  Stats stats;

 private:
  void activate(int32_t x, int32_t y, int32_t z);
  void wake_around(int32_t x, int32_t y, int32_t z);
  void seed_level(uint64_t k);
  bool supported(const SparseVolume& v, int32_t x, int32_t y, int32_t z) const;
  bool set_volume(SparseVolume& v, int32_t x, int32_t y, int32_t z, float vol);
  bool level_layer(SparseVolume& v, int32_t sx, int32_t sy, int32_t sz);
  bool level_surfaces(SparseVolume& v);
  float pressure_pull(SparseVolume& v, int32_t x, int32_t y, int32_t z, float need);

  PartialField partial_;
  U64Set active_;
  std::deque<uint64_t> queue_;
  U64Set level_seeds_;
  std::vector<uint64_t> level_seed_list_;
  LayerMarks level_visited_;
  std::vector<uint64_t> level_cells_;
  std::vector<uint64_t> press_queue_;
  U64Set press_visited_;
  float acc_ = 0.0f;
  size_t last_cells_ = 0;
  size_t last_level_cells_ = 0;
  bool level_round_ = false;
  uint32_t tick_no_ = 0;
};

// key packing (src/fluid.rs:46-62)
inline uint64_t field(int32_t v) { return (uint64_t)(((uint32_t)v + (1u << 20)) & 0x1FFFFFu); }
inline int32_t field_value(uint64_t f) { return (int32_t)(f & 0x1FFFFF) - (1 << 20); }
inline uint64_t key(int32_t x, int32_t y, int32_t z) { return field(x) | field(y) << 21 | field(z) << 42; }
inline void unkey(uint64_t k, int32_t& x, int32_t& y, int32_t& z) {
  x = field_value(k);
  y = field_value(k >> 21);
  z = field_value(k >> 42);
}

template <class F>
void PartialField::for_each(F f) const {
  index_.for_each([&](uint64_t k, uint32_t i) {
    int32_t px, py, pz;
    unkey(k, px, py, pz);
    for (int j = 0; j < 512; ++j) {
      float v = pages_[i].v[j];
      if (v > 0.0f) f(px * 8 + (j & 7), py * 8 + ((j >> 3) & 7), pz * 8 + (j >> 6), v);
    }
  });
}

}  // namespace orc
