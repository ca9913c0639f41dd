// Host-side sparse brick world: the product's restatement of the reference's SparseVolume
// (src/voxel/sparse_volume.rs:90-537), used as the host mirror the fluid reads at upload and
// writes back into. Layout and encodings are kept identical to the reference because they are
// the drop-in boundary: grid u32 per brick (0 empty, 1..255 uniform, >= 256 detailed index +
// 256), brick voxel index lz*64 + ly*8 + lx, ring chunks of 16x16 brick columns.
#pragma once
#include <array>
#include <cstdint>
#include <vector>

namespace vfw {

constexpr int BRICK = 8;
constexpr int RING_CHUNK_B = 16;
constexpr uint8_t WATER = 5;
constexpr uint8_t STONE = 3;

struct RingSlot {
  int32_t cx = 0, cz = 0;
  bool loaded = false, modified = false;
};

struct World {
  int32_t nx = 0, ny = 0, nz = 0;
  int32_t bricks_x = 0, bricks_y = 0, bricks_z = 0;
  std::vector<uint32_t> grid;
  std::vector<std::array<uint8_t, 512>> bricks;
  std::vector<uint32_t> free_bricks;
  std::vector<uint32_t> dirty_grid;
  bool track_dirty = true;
  int32_t ring_w = 0;
  std::vector<RingSlot> ring_slots;
  int32_t origin_x = 0, origin_z = 0;

  World() = default;
  World(int32_t nx, int32_t ny, int32_t nz);
  void ring_init(int32_t w, int32_t ny);
  size_t grid_index(int32_t ix, int32_t iy, int32_t iz) const {
    if (ring_w != 0) {
      ix &= bricks_x - 1;
      iz &= bricks_z - 1;
    }
    return ((size_t)(uint32_t)iz * (size_t)bricks_y + (size_t)(uint32_t)iy) * (size_t)bricks_x + (size_t)(uint32_t)ix;
  }
  size_t ring_slot_index(int32_t cx, int32_t cz) const {
    int32_t m = ring_w - 1;
    return (size_t)(cz & m) * (size_t)ring_w + (size_t)(cx & m);
  }
  bool chunk_loaded(int32_t cx, int32_t cz) const {
    if (ring_w == 0) return true;
    const RingSlot& s = ring_slots[ring_slot_index(cx, cz)];
    return s.loaded && s.cx == cx && s.cz == cz;
  }
  bool inside(int32_t x, int32_t y, int32_t z) const {
    if (ring_w != 0) return (uint32_t)y < (uint32_t)ny && chunk_loaded(x >> 7, z >> 7);
    return (uint32_t)x < (uint32_t)nx && (uint32_t)y < (uint32_t)ny && (uint32_t)z < (uint32_t)nz;
  }
  uint8_t get_voxel(int32_t x, int32_t y, int32_t z) const {
    if (!inside(x, y, z)) return 0;
    uint32_t v = grid[grid_index(x >> 3, y >> 3, z >> 3)];
    if (v < 256) return (uint8_t)v;
    return bricks[v - 256][(z & 7) * 64 + (y & 7) * 8 + (x & 7)];
  }
  size_t materialize(size_t gi, uint8_t fill);
  size_t alloc_brick();
  void set_voxel(int32_t x, int32_t y, int32_t z, uint8_t m);
  void fill_box(int32_t x0, int32_t y0, int32_t z0, int32_t x1, int32_t y1, int32_t z1, uint8_t m);
  void fill_sphere(float cx, float cy, float cz, float r, uint8_t m);
  void compact();
  void ring_paste(const World& src, int32_t cx, int32_t cz);
  void ring_evict(int32_t cx, int32_t cz);
  void mark_modified(size_t gi);
  size_t detailed() const { return bricks.size() - free_bricks.size(); }
};

// Noise of the reference's world generator (src/worldgen/mod.rs:31-56), f32 throughout.
uint32_t hash2(int32_t x, int32_t y, uint32_t seed);
float value_noise(float x, float y, uint32_t seed);
// Octave sum like the reference's fbm (src/worldgen/mod.rs:58-66) with a chosen octave count:
// amplitude 0.5 halving, frequency doubling, octave seed = seed + i*101.
float fbm(float x, float y, uint32_t seed, int octaves);

}  // namespace vfw
