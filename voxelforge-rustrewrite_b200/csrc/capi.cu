// Host side of the C ABI (include/vf_fluid.h): device memory layout, uploads, launches,
// downloads. The reference's FluidSim methods map one to one onto vf_fluid_* calls.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdio>
#include <cstring>
#include <string>
#include <tuple>
#include <mutex>
#include <vector>

#include "../../include/vf_fluid.h"
#include "kernels.cuh"

using namespace vfe;

// A partial entry of a cell in an evicted ring chunk: the reference's PartialField keys entries by
// cell, not by brick, so they outlive the chunk's bricks (and return with a paste).
struct DetachedPartial {
  int32_t x, y, z;
  float v;
  uint32_t id;  // domain cell id
};

struct vf_fluid {
  int device = 0;
  cudaStream_t stream = nullptr;
  bool own_stream = false;
  Region R{};
  Region* dR = nullptr;
  Ctl* hctl = nullptr;  // pinned mirror
  unsigned* hzero = nullptr;  // pinned control word copied in by every tick
  bool uploaded = false;
  std::string err;
  std::vector<void*> dev_allocs;
  uint64_t want_atlas = 0, want_queue = 0;
  int pad = 32;
  float acc = 0.0f;  // FluidSim::acc (fluid.rs:243), host-side like the reference's
  // download scratch
  void* scratch = nullptr;
  size_t scratch_bytes = 0;
  // tick launch shape
  int smem_bytes = 0;
  Tune tune{TICK_WARPS - 1, PF_RING, 1, 4 | (1 << 8), 1ull << 24};
  // wake proposal state (allocated on first use)
  int* slot_gi = nullptr;
  SlotAggr* aggr = nullptr;
  float* whist = nullptr;
  unsigned* staged = nullptr;
  unsigned hpos = 0;
  // ring streaming on a live handle: entries kept for evicted chunks, atlas slots they freed
  std::vector<DetachedPartial> det;
  std::vector<unsigned> free_slots;
  // engine chosen per launch from the last launches' pressure-search entries per cell-step
  bool auto_engine = true;
  uint64_t auto_cells = 0, auto_bfs = 0;
};

// A set of regions stepped together: one CTA per region in one launch (pattern (2)).
struct vf_batch {
  std::vector<vf_fluid*> hs;
  Region* dregs = nullptr;
  cudaStream_t stream = nullptr;
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t exec = nullptr;
};

namespace {

// Makes `dev` current for a scope and gives the caller back the device it had current.
struct DeviceScope {
  int prev = -1;
  cudaError_t err = cudaSuccess;
  explicit DeviceScope(int dev) {
    if (cudaGetDevice(&prev) != cudaSuccess) prev = -1;
    err = cudaSetDevice(dev);
  }
  ~DeviceScope() {
    if (prev >= 0) cudaSetDevice(prev);
  }
};

// The tick kernel of the handle's engine for `nreg` regions: one CTA per region.
// The parallel sweep uses only the parallel member of TickSmem's union: its launch asks for that
// much shared memory, which leaves the rest of the SM's 256 KB to L1.
constexpr int PAR_SMEM_BYTES = (int)((offsetof(TickSmem, u) + sizeof(ParSmem) + 127) / 128 * 128);
static_assert(PAR_SMEM_BYTES <= (int)sizeof(TickSmem), "parallel sweep shared memory");

cudaError_t launch_tick(const Tune& t, Region* regs, int nreg, int n_ticks, int smem, cudaStream_t st) {
  if (t.engine) {
    const int warps = (t.gate >> 16) & 0x1F;
    k_tick_par<<<(unsigned)nreg, warps ? 32 * warps : PAR_THREADS, PAR_SMEM_BYTES, st>>>(regs, nreg, n_ticks, t);
  }
  else k_tick<<<(unsigned)nreg, TICK_THREADS, smem, st>>>(regs, nreg, n_ticks, t);
  return cudaGetLastError();
}

int fail(vf_fluid* h, int code, const std::string& msg) {
  if (h) h->err = msg;
  return code;
}

#define CK(call)                                                                              \
  do {                                                                                        \
    cudaError_t e_ = (call);                                                                  \
    if (e_ != cudaSuccess) return fail(h, VF_ERR_CUDA, std::string(#call) + ": " + cudaGetErrorString(e_)); \
  } while (0)

template <class T>
int dalloc(vf_fluid* h, T** p, size_t count, bool zero = true) {
  size_t bytes = std::max<size_t>(count * sizeof(T), 16);
  cudaError_t e = cudaMalloc((void**)p, bytes);
  if (e != cudaSuccess) return fail(h, VF_ERR_OOM, std::string("cudaMalloc: ") + cudaGetErrorString(e));
  h->dev_allocs.push_back(*p);
  if (zero) {
    e = cudaMemsetAsync(*p, 0, bytes, h->stream);
    if (e != cudaSuccess) return fail(h, VF_ERR_CUDA, cudaGetErrorString(e));
  }
  return VF_OK;
}

void free_world(vf_fluid* h) {
  if (h->stream) cudaStreamSynchronize(h->stream);
  for (void* p : h->dev_allocs) cudaFree(p);
  h->dev_allocs.clear();
  h->dR = nullptr;
  h->scratch = nullptr;
  h->scratch_bytes = 0;
  h->uploaded = false;
}

int ensure_scratch(vf_fluid* h, size_t bytes) {
  if (h->scratch_bytes >= bytes) return VF_OK;
  if (h->scratch) {
    cudaStreamSynchronize(h->stream);
    cudaFree(h->scratch);
    auto it = std::find(h->dev_allocs.begin(), h->dev_allocs.end(), h->scratch);
    if (it != h->dev_allocs.end()) h->dev_allocs.erase(it);
  }
  size_t b = std::max<size_t>(bytes, 1 << 20);
  cudaError_t e = cudaMalloc(&h->scratch, b);
  if (e != cudaSuccess) {
    h->scratch = nullptr;
    h->scratch_bytes = 0;
    return fail(h, VF_ERR_OOM, "scratch alloc");
  }
  h->dev_allocs.push_back(h->scratch);
  h->scratch_bytes = b;
  return VF_OK;
}

int sync_ctl(vf_fluid* h) {
  CK(cudaMemcpyAsync(h->hctl, h->R.ctl, sizeof(Ctl), cudaMemcpyDeviceToHost, h->stream));
  CK(cudaStreamSynchronize(h->stream));
  if (h->hctl->status != 0) {
    char b[128];
    snprintf(b, sizeof b, "device status %d (site %u)", h->hctl->status, h->hctl->err_info);
    return fail(h, h->hctl->status, b);
  }
  return VF_OK;
}

// Offsets into the scratch buffer are kept 16-byte aligned (8-byte device atomics live there).
size_t align16(size_t v) { return (v + 15) & ~(size_t)15; }

// live[k] = 1 when the k-th entry kept for an evicted ring chunk still exists (a drained cell of an
// unloaded chunk erases it).
int detached_live(vf_fluid* h, std::vector<uint8_t>& live) {
  const size_t nd = h->det.size();
  live.assign(nd, 0);
  if (!nd) return VF_OK;
  int rc;
  if ((rc = ensure_scratch(h, nd * 8 + 64))) return rc;
  unsigned* dids = (unsigned*)h->scratch;
  unsigned* dout = dids + align16(nd * 4) / 4;
  std::vector<unsigned> ids(nd), out(nd);
  for (size_t k = 0; k < nd; ++k) ids[k] = h->det[k].id;
  CK(cudaMemcpyAsync(dids, ids.data(), nd * 4, cudaMemcpyHostToDevice, h->stream));
  k_cell_bits<<<(unsigned)std::min<size_t>((nd + 255) / 256, 1024), 256, 0, h->stream>>>(h->R.detbits, dids, (unsigned)nd, 2, dout);
  CK(cudaGetLastError());
  CK(cudaMemcpyAsync(out.data(), dout, nd * 4, cudaMemcpyDeviceToHost, h->stream));
  CK(cudaStreamSynchronize(h->stream));
  for (size_t k = 0; k < nd; ++k) live[k] = out[k] ? 1 : 0;
  return VF_OK;
}

// Set (op 1) or clear (op 0) the detbits of `ids`.
int detached_bits(vf_fluid* h, const std::vector<unsigned>& ids, int op) {
  if (ids.empty()) return VF_OK;
  int rc;
  if ((rc = ensure_scratch(h, ids.size() * 4 + 64))) return rc;
  CK(cudaMemcpyAsync(h->scratch, ids.data(), ids.size() * 4, cudaMemcpyHostToDevice, h->stream));
  k_cell_bits<<<(unsigned)std::min<size_t>((ids.size() + 255) / 256, 1024), 256, 0, h->stream>>>(h->R.detbits, (unsigned*)h->scratch,
                                                                                                 (unsigned)ids.size(), op, nullptr);
  CK(cudaGetLastError());
  CK(cudaStreamSynchronize(h->stream));
  return VF_OK;
}

// The device's count of kept entries after a change of `delta` (the ticks' erasures included).
int detached_count(vf_fluid* h, long long delta) {
  if ((h->hctl->ndetached + delta) > 0xFFFFFFFFll) return fail(h, VF_ERR_OOM, "too many kept partial entries");
  const unsigned v = (unsigned)((long long)h->hctl->ndetached + delta);
  h->hctl->ndetached = v;
  CK(cudaMemcpy(&h->R.ctl->ndetached, &v, 4, cudaMemcpyHostToDevice));
  return VF_OK;
}

// SparseVolume::ring_evict (sparse_volume.rs:513-537) of ring slot `si` on the device: the slot's
// bricks become empty and their atlas slots free; the partial volumes they held are kept per cell,
// as the reference's PartialField keeps them. `ring` is the device ring table, updated here.
int ring_evict_slot(vf_fluid* h, int si, std::vector<int32_t>& ring) {
  const Region& R = h->R;
  if (!ring[3 * si + 2]) return VF_OK;
  const int w = R.ring_w, ocx = ring[3 * si], ocz = ring[3 * si + 1];
  const int bx0 = (si % w) * 16, bz0 = (si / w) * 16;
  const uint64_t nb = (uint64_t)R.bx * R.by * R.bz;
  std::vector<uint32_t> grid(nb);
  CK(cudaMemcpy(grid.data(), R.grid, nb * 4, cudaMemcpyDeviceToHost));
  std::vector<unsigned> slots;
  std::vector<uint64_t> gis;
  for (int bz = 0; bz < 16; ++bz)
    for (int by = 0; by < R.by; ++by)
      for (int bx = 0; bx < 16; ++bx) {
        const uint64_t gi = ((uint64_t)(bz0 + bz) * R.by + by) * R.bx + (bx0 + bx);
        if (grid[gi] >= 256u) {
          slots.push_back(grid[gi] - 256u);
          gis.push_back(gi);
        }
        grid[gi] = 0u;
      }
  int rc;
  if (!slots.empty()) {
    const size_t n = slots.size();
    if ((rc = ensure_scratch(h, align16(n * 4) + n * 2048 + 64))) return rc;
    unsigned* dslots = (unsigned*)h->scratch;
    float* dvol = (float*)((char*)h->scratch + align16(n * 4));
    std::vector<float> vols(n * 512);
    CK(cudaMemcpyAsync(dslots, slots.data(), n * 4, cudaMemcpyHostToDevice, h->stream));
    k_gather_vol<<<(unsigned)std::min<size_t>((n * 512 + 255) / 256, 8192), 256, 0, h->stream>>>(R.avol, dslots, (unsigned)n, dvol);
    CK(cudaGetLastError());
    CK(cudaMemcpyAsync(vols.data(), dvol, n * 2048, cudaMemcpyDeviceToHost, h->stream));
    CK(cudaStreamSynchronize(h->stream));
    std::vector<unsigned> ids;
    for (size_t k = 0; k < n; ++k) {
      const uint64_t gi = gis[k];
      const int bx = (int)(gi % R.bx), by = (int)((gi / R.bx) % R.by), bz = (int)(gi / ((uint64_t)R.bx * R.by));
      for (int l = 0; l < 512; ++l) {
        const float v = vols[k * 512 + l];
        if (!(v > 0.0f)) continue;
        const int x = ocx * 128 + (bx % 16) * 8 + (l & 7), y = by * 8 + ((l >> 3) & 7), z = ocz * 128 + (bz % 16) * 8 + (l >> 6);
        if (!in_dom(R, x, y, z)) continue;
        const unsigned id = dom_id(R, x, y, z);
        h->det.push_back({x, y, z, v, id});
        ids.push_back(id);
      }
      h->free_slots.push_back(slots[k]);
    }
    if ((rc = detached_bits(h, ids, 1))) return rc;
    if ((rc = detached_count(h, (long long)ids.size()))) return rc;
  }
  CK(cudaMemcpy(R.grid, grid.data(), nb * 4, cudaMemcpyHostToDevice));
  ring[3 * si + 2] = 0;
  CK(cudaMemcpy(R.ring, ring.data(), ring.size() * 4, cudaMemcpyHostToDevice));
  return VF_OK;
}

uint64_t next_pow2(uint64_t v) {
  uint64_t p = 1;
  while (p < v) p <<= 1;
  return p;
}

int check(vf_fluid* h) {
  if (!h) return VF_ERR_INVALID;
  if (!h->uploaded) return fail(h, VF_ERR_STATE, "no world uploaded");
  return VF_OK;
}

}  // namespace

extern "C" {

int vf_fluid_create(const vf_fluid_desc* desc, vf_fluid** out) {
  if (!out) return VF_ERR_INVALID;
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) return VF_ERR_NO_DEVICE;
  auto* h = new vf_fluid();
  h->device = desc ? desc->device : 0;
  if (h->device < 0 || h->device >= ndev) {
    delete h;
    return VF_ERR_INVALID;
  }
  DeviceScope scope(h->device);
  if (scope.err != cudaSuccess) {
    delete h;
    return VF_ERR_NO_DEVICE;
  }
  if (desc && desc->stream) {
    h->stream = (cudaStream_t)desc->stream;
  } else {
    if (cudaStreamCreateWithFlags(&h->stream, cudaStreamNonBlocking) != cudaSuccess) {
      delete h;
      return VF_ERR_CUDA;
    }
    h->own_stream = true;
  }
  if (desc) {
    h->want_atlas = desc->atlas_bricks;
    h->want_queue = desc->queue_capacity;
  }
  if (cudaMallocHost(&h->hctl, sizeof(Ctl)) != cudaSuccess) {
    delete h;
    return VF_ERR_OOM;
  }
  std::memset(h->hctl, 0, sizeof(Ctl));
  if (cudaMallocHost(&h->hzero, 16) != cudaSuccess) {
    cudaFreeHost(h->hctl);
    delete h;
    return VF_ERR_OOM;
  }
  // the tick kernel's image must load (sm_100a only): probe its attributes
  cudaFuncAttributes fa;
  if (cudaFuncGetAttributes(&fa, k_tick) != cudaSuccess) {
    cudaFreeHost(h->hctl);
    delete h;
    return VF_ERR_NO_DEVICE;
  }
  h->smem_bytes = (int)sizeof(TickSmem);
  cudaFuncSetAttribute(k_tick, cudaFuncAttributeMaxDynamicSharedMemorySize, h->smem_bytes);
  cudaFuncSetAttribute(k_tick_par, cudaFuncAttributeMaxDynamicSharedMemorySize, PAR_SMEM_BYTES);
  *out = h;
  return VF_OK;
}

void vf_fluid_destroy(vf_fluid* h) {
  if (!h) return;
  DeviceScope scope(h->device);
  free_world(h);
  if (h->hctl) cudaFreeHost(h->hctl);
  if (h->hzero) cudaFreeHost(h->hzero);
  if (h->own_stream && h->stream) cudaStreamDestroy(h->stream);
  delete h;
}

const char* vf_fluid_last_error(const vf_fluid* h) { return h ? h->err.c_str() : "null handle"; }

int vf_fluid_upload_world(vf_fluid* h, int32_t nx, int32_t ny, int32_t nz, int32_t bricks_x, int32_t bricks_y, int32_t bricks_z,
                          const uint32_t* grid, const uint8_t* bricks, uint64_t nbricks, int32_t ring_w, const int32_t* ring_slots) {
  if (!h || !grid || nx <= 0 || ny <= 0 || nz <= 0 || bricks_x <= 0 || bricks_y <= 0 || bricks_z <= 0) return VF_ERR_INVALID;
  if (ring_w && (!ring_slots || (ring_w & (ring_w - 1)))) return VF_ERR_INVALID;
  DeviceScope scope(h->device);
  if (scope.err != cudaSuccess) return VF_ERR_CUDA;
  if (h->uploaded) return fail(h, VF_ERR_STATE, "world already uploaded: create a new handle or use apply_voxel_edits");
  Region R{};
  R.nx = nx;
  R.ny = ny;
  R.nz = nz;
  R.bx = bricks_x;
  R.by = bricks_y;
  R.bz = bricks_z;
  R.ring_w = ring_w;
  const int P = h->pad;
  if (!ring_w) {
    R.px0 = -P;
    R.pz0 = -P;
    R.PX = nx + 2 * P;
    R.PZ = nz + 2 * P;
  } else {
    // bounding box of the loaded chunks (absolute chunk coords)
    int cx0 = 1 << 30, cx1 = -(1 << 30), cz0 = 1 << 30, cz1 = -(1 << 30);
    for (int i = 0; i < ring_w * ring_w; ++i)
      if (ring_slots[3 * i + 2]) {
        cx0 = std::min(cx0, ring_slots[3 * i]);
        cx1 = std::max(cx1, ring_slots[3 * i]);
        cz0 = std::min(cz0, ring_slots[3 * i + 1]);
        cz1 = std::max(cz1, ring_slots[3 * i + 1]);
      }
    if (cx0 > cx1) cx0 = cx1 = cz0 = cz1 = 0;
    R.px0 = cx0 * 128 - P;
    R.pz0 = cz0 * 128 - P;
    R.PX = (cx1 - cx0 + 1) * 128 + 2 * P;
    R.PZ = (cz1 - cz0 + 1) * 128 + 2 * P;
  }
  R.PY = ny + P;
  R.mx = udiv_magic((unsigned)R.PX);
  R.my = udiv_magic((unsigned)R.PY);
  R.mz = udiv_magic((unsigned)R.PZ);
  uint64_t ncells = (uint64_t)R.PX * R.PY * R.PZ;
  if (ncells >= 0x7FFFFFF0ull) return fail(h, VF_ERR_RANGE, "domain too large for 31-bit cell ids");
  R.ncells = (unsigned)ncells;
  R.TX = (R.PX + 63) / 64;
  R.TZ = (R.PZ + 63) / 64;
  const uint64_t nb = (uint64_t)bricks_x * bricks_y * bricks_z;
  // device grid: detailed host bricks get atlas slots in grid order
  std::vector<uint32_t> dgrid(nb);
  uint64_t nd = 0, nfree_uniform = 0;
  for (uint64_t gi = 0; gi < nb; ++gi) {
    uint32_t v = grid[gi];
    if (v >= 256) {
      if (v - 256 >= nbricks || !bricks) return fail(h, VF_ERR_INVALID, "grid names a brick out of range");
      dgrid[gi] = 256 + (uint32_t)nd++;
    } else {
      dgrid[gi] = v;
      if (v == 0 || v == VF_FLUID_WATER) ++nfree_uniform;
    }
  }
  uint64_t cap = h->want_atlas ? h->want_atlas : nd + nfree_uniform + 1024;
  cap = std::max<uint64_t>(cap, nd + 64);
  if (cap > 0xFFFFFF00ull - 256) return fail(h, VF_ERR_RANGE, "atlas too large");
  R.atlas_cap = (unsigned)cap;
  int rc;
  if ((rc = dalloc(h, &R.grid, nb, false))) return rc;
  if ((rc = dalloc(h, &R.amat, cap * 512, false))) return rc;
  if ((rc = dalloc(h, &R.avol, cap * 512, false))) return rc;
  CK(cudaMemsetAsync(R.avol, 0, nd * 512 * sizeof(float) + 16, h->stream));
  CK(cudaMemcpyAsync(R.grid, dgrid.data(), nb * 4, cudaMemcpyHostToDevice, h->stream));
  {
    std::vector<uint8_t> tmp(std::max<uint64_t>(nd, 1) * 512);
    uint64_t k = 0;
    for (uint64_t gi = 0; gi < nb; ++gi)
      if (grid[gi] >= 256) std::memcpy(&tmp[(k++) * 512], bricks + (uint64_t)(grid[gi] - 256) * 512, 512);
    CK(cudaMemcpyAsync(R.amat, tmp.data(), nd * 512, cudaMemcpyHostToDevice, h->stream));
    CK(cudaStreamSynchronize(h->stream));
  }
  if ((rc = dalloc(h, &R.ring, std::max(1, 3 * ring_w * ring_w)))) return rc;
  if (ring_w) CK(cudaMemcpyAsync(R.ring, ring_slots, 3 * ring_w * ring_w * 4, cudaMemcpyHostToDevice, h->stream));
  const uint64_t words = (ncells + 31) / 32;
  if ((rc = dalloc(h, &R.active, words))) return rc;
  if ((rc = dalloc(h, &R.seedbits, words))) return rc;
  if ((rc = dalloc(h, &R.chgbits, words))) return rc;
  const uint64_t tiles = (uint64_t)R.TX * R.PY * R.TZ;
  if ((rc = dalloc(h, &R.marks, tiles * 128))) return rc;
  if ((rc = dalloc(h, &R.mark_list, tiles))) return rc;
  if ((rc = dalloc(h, &R.mark_tflag, tiles))) return rc;
  // per-tick event logs: <= 50 activations and 7 writes per swept cell, plus levelling's
  R.ev_act_cap = 1u << 22;
  R.ev_seed_cap = 1u << 18;
  R.ev_chg_cap = 1u << 21;
  if ((rc = dalloc(h, &R.ev_act, R.ev_act_cap, false))) return rc;
  if ((rc = dalloc(h, &R.ev_seed, R.ev_seed_cap, false))) return rc;
  if ((rc = dalloc(h, &R.ev_chg, R.ev_chg_cap, false))) return rc;
  if ((rc = dalloc(h, &R.stamp, ncells, false))) return rc;
  if ((rc = dalloc(h, &R.last_woken, cap))) return rc;
  CK(cudaMemsetAsync(R.stamp, 0xFF, ncells * 4, h->stream));
  // parallel sweep: per-cell records, rows, pull stamps and versions
  if ((rc = dalloc(h, &R.rec, MAX_CELLS_PER_TICK))) return rc;
  if ((rc = dalloc(h, &R.rowstart, MAX_CELLS_PER_TICK + 1))) return rc;
  if ((rc = dalloc(h, &R.rowof, MAX_CELLS_PER_TICK))) return rc;
  if ((rc = dalloc(h, &R.rowprog, MAX_CELLS_PER_TICK))) return rc;
  if ((rc = dalloc(h, &R.pcnt, MAX_CELLS_PER_TICK + 1))) return rc;
  if ((rc = dalloc(h, &R.zrow, (uint64_t)R.PY * R.PZ, false))) return rc;
  CK(cudaMemsetAsync(R.zrow, 0xFF, (uint64_t)R.PY * R.PZ * 4, h->stream));
  if ((rc = dalloc(h, &R.preader, ncells))) return rc;
  if ((rc = dalloc(h, &R.ptbits, words))) return rc;
  if ((rc = dalloc(h, &R.ptlist, MAX_PULLS_PER_TICK + 64))) return rc;
  if ((rc = dalloc(h, &R.ptreg, PTREG_CAP))) return rc;
  if ((rc = dalloc(h, &R.pextra, (MAX_CELLS_PER_TICK + 31) / 32))) return rc;
  if ((rc = dalloc(h, &R.pxlist, MAX_CELLS_PER_TICK))) return rc;
  if ((rc = dalloc(h, &R.rb, ncells, false))) return rc;
  if (ring_w && (rc = dalloc(h, &R.detbits, words))) return rc;
  if ((rc = dalloc(h, &R.deps, (uint64_t)MAX_CELLS_PER_TICK * 16, false))) return rc;
  // the warps' search contexts in global memory: visited sets empty (every search empties its own
  // before it returns)
  if ((rc = dalloc(h, &R.pcg, MAX_WARPS, false))) return rc;
  static_assert(EMPTY_ID == 0xFFFFFFFFu, "a visited-set slot of 0xFF bytes is free");
  CK(cudaMemsetAsync(R.pcg, 0xFF, MAX_WARPS * sizeof(PullCtx), h->stream));
  CK(cudaMemsetAsync(R.rb, 0xFF, ncells * 4, h->stream));
  // the parallel sweep packs search-queue coordinates in 16 bits per axis
  if (R.PX >= 65536 || R.PZ >= 65536 || R.PY >= 65536) h->tune.engine = 0;
  R.chg_cap = 1u << 22;
  if ((rc = dalloc(h, &R.chg, R.chg_cap, false))) return rc;
  uint64_t qcap = next_pow2(std::max<uint64_t>({h->want_queue, std::min<uint64_t>(ncells, 1ull << 22), 1ull << 16}));
  R.qmask = qcap - 1;
  if ((rc = dalloc(h, &R.queue, qcap, false))) return rc;
  if ((rc = dalloc(h, &R.cells, MAX_CELLS_PER_TICK, false))) return rc;
  if ((rc = dalloc(h, &R.cells_tmp, MAX_CELLS_PER_TICK, false))) return rc;
  if ((rc = dalloc(h, &R.seeds, MAX_LEVEL_SEEDS, false))) return rc;
  if ((rc = dalloc(h, &R.lvl_id, MAX_LEVEL_CELLS + 8, false))) return rc;
  if ((rc = dalloc(h, &R.lvl_vol, MAX_LEVEL_CELLS + 8, false))) return rc;
  if ((rc = dalloc(h, &R.ctl, 1))) return rc;
  std::memset(h->hctl, 0, sizeof(Ctl));
  h->hctl->atlas_used = (unsigned)nd;
  CK(cudaMemcpyAsync(R.ctl, h->hctl, sizeof(Ctl), cudaMemcpyHostToDevice, h->stream));
  if ((rc = dalloc(h, &h->dR, 1, false))) return rc;
  CK(cudaMemcpyAsync(h->dR, &R, sizeof(Region), cudaMemcpyHostToDevice, h->stream));
  CK(cudaStreamSynchronize(h->stream));
  h->R = R;
  h->uploaded = true;
  h->acc = 0.0f;
  return VF_OK;
}

int vf_fluid_apply_voxel_edits(vf_fluid* h, const vf_voxel* edits, uint64_t n) {
  int rc = check(h);
  if (rc) return rc;
  DeviceScope scope(h->device);  // the caller's current device is given back on return
  if (!n) return VF_OK;
  if (!edits) return VF_ERR_INVALID;
  if ((rc = ensure_scratch(h, n * 16))) return rc;
  std::vector<int> q(4 * n);
  for (uint64_t i = 0; i < n; ++i) {
    q[4 * i] = edits[i].x;
    q[4 * i + 1] = edits[i].y;
    q[4 * i + 2] = edits[i].z;
    q[4 * i + 3] = edits[i].m;
  }
  CK(cudaMemcpyAsync(h->scratch, q.data(), n * 16, cudaMemcpyHostToDevice, h->stream));
  k_edit<<<1, 32, 0, h->stream>>>(h->R, ED_VOXELS, (const int*)h->scratch, n, 0, 0.0f, nullptr);
  CK(cudaGetLastError());
  return sync_ctl(h);
}

int vf_fluid_wake(vf_fluid* h, int32_t x0, int32_t y0, int32_t z0, int32_t x1, int32_t y1, int32_t z1) {
  int rc = check(h);
  if (rc) return rc;
  DeviceScope scope(h->device);  // the caller's current device is given back on return
  if (x1 < x0 || y1 < y0 || z1 < z0) return VF_OK;  // empty box: the reference's loops do nothing
  y0 = std::max(y0, 0);                            // activate ignores y < 0 (fluid.rs:293)
  if (y1 < y0) return VF_OK;
  if (!in_dom(h->R, x0, y0, z0) || !in_dom(h->R, x1, y1, z1)) return fail(h, VF_ERR_RANGE, "wake box outside the padded domain");
  k_wake_box<<<1, 1024, 0, h->stream>>>(h->R, x0, y0, z0, x1, y1, z1);
  CK(cudaGetLastError());
  return sync_ctl(h);
}

static int run_edit(vf_fluid* h, int kind, const int32_t* xyz, uint64_t n, int m, float amount, uint64_t* out_count, size_t ints_per) {
  int rc = check(h);
  if (rc) return rc;
  const size_t data = align16(n * ints_per * 4);
  if ((rc = ensure_scratch(h, data + 64))) return rc;
  if (n) CK(cudaMemcpyAsync(h->scratch, xyz, n * ints_per * 4, cudaMemcpyHostToDevice, h->stream));
  unsigned long long* dcount = (unsigned long long*)((char*)h->scratch + data);
  k_edit<<<1, 32, 0, h->stream>>>(h->R, kind, (const int*)h->scratch, n, m, amount, out_count ? dcount : nullptr);
  CK(cudaGetLastError());
  if (out_count) {
    unsigned long long c = 0;
    CK(cudaMemcpyAsync(&c, dcount, 8, cudaMemcpyDeviceToHost, h->stream));
    rc = sync_ctl(h);
    *out_count = c;
    return rc;
  }
  return sync_ctl(h);
}

int vf_fluid_displace(vf_fluid* h, int32_t x, int32_t y, int32_t z) {
  int32_t p[3] = {x, y, z};
  return run_edit(h, ED_DISPLACE, p, 1, 0, 0.0f, nullptr, 3);
}

int vf_fluid_apply_brush(vf_fluid* h, const int32_t* xyz, uint64_t n, uint8_t m, uint64_t* n_changed) {
  if (n && !xyz) return VF_ERR_INVALID;
  uint64_t c = 0;
  int rc = run_edit(h, ED_BRUSH, xyz, n, m, 0.0f, &c, 3);
  if (n_changed) *n_changed = c;
  return rc;
}

int vf_fluid_emit(vf_fluid* h, const int32_t* xyz, uint64_t n, float amount) {
  if (n && !xyz) return VF_ERR_INVALID;
  return run_edit(h, ED_EMIT, xyz, n, 0, amount, nullptr, 3);
}

int vf_fluid_set_partial(vf_fluid* h, int32_t x, int32_t y, int32_t z, float v) {
  int32_t p[3] = {x, y, z};
  return run_edit(h, ED_SET_PARTIAL, p, 1, 0, v, nullptr, 3);
}

int vf_fluid_tick_async(vf_fluid* h, int32_t n_ticks) {
  int rc = check(h);
  if (rc) return rc;
  DeviceScope scope(h->device);  // the caller's current device is given back on return
  if (n_ticks < 0) return VF_ERR_INVALID;
  // the step's control input (reset of the "changed" flag) goes host -> device from pinned memory
  h->hzero[0] = 0u;
  CK(cudaMemcpyAsync(&h->R.ctl->changed, h->hzero, sizeof(unsigned), cudaMemcpyHostToDevice, h->stream));
  if (n_ticks > 0) {
    if (h->auto_engine) {
      // pull-heavy water (deep lakes, many pressure searches per cell) runs faster on the one-warp
      // sweep; everything else on the parallel sweep. Counters as of the last synchronisation.
      const uint64_t dc = h->hctl->cells_total - h->auto_cells, db = h->hctl->bfs_visits - h->auto_bfs;
      const bool wide_ok = h->R.PX < 65536 && h->R.PZ < 65536 && h->R.PY < 65536;
      if (dc > 0) h->tune.engine = (wide_ok && 2 * db <= 3 * dc) ? 1 : 0;
      h->auto_cells = h->hctl->cells_total;
      h->auto_bfs = h->hctl->bfs_visits;
    }
    CK(launch_tick(h->tune, h->dR, 1, n_ticks, h->smem_bytes, h->stream));
  }
  return VF_OK;
}

int vf_fluid_tick(vf_fluid* h, int32_t n_ticks, int32_t* changed) {
  int rc = vf_fluid_tick_async(h, n_ticks);
  if (rc) return rc;
  rc = sync_ctl(h);
  if (changed) *changed = h->hctl->changed ? 1 : 0;
  return rc;
}

int vf_fluid_sync(vf_fluid* h) {
  int rc = check(h);
  if (rc) return rc;
  DeviceScope scope(h->device);  // the caller's current device is given back on return
  return sync_ctl(h);
}

void* vf_fluid_stream(vf_fluid* h) { return h ? (void*)h->stream : nullptr; }

int vf_fluid_idle(vf_fluid* h, int32_t* out) {
  int rc = check(h);
  if (rc) return rc;
  DeviceScope scope(h->device);  // the caller's current device is given back on return
  if ((rc = sync_ctl(h))) return rc;
  if (out) *out = (h->hctl->qtail == h->hctl->qhead && h->hctl->nseeds == 0) ? 1 : 0;  // fluid.rs:265-267
  return VF_OK;
}

int vf_fluid_update(vf_fluid* h, float dt, int32_t* changed) {  // fluid.rs:662-676
  int32_t idle = 0;
  int rc = vf_fluid_idle(h, &idle);
  if (rc) return rc;
  if (changed) *changed = 0;
  if (idle) {
    h->acc = 0.0f;
    return VF_OK;
  }
  const float step = 1.0f / VF_FLUID_TICK_HZ;
  h->acc = std::min(h->acc + std::min(dt, 0.25f), 3.0f / VF_FLUID_TICK_HZ);
  int n = 0;
  while (h->acc >= step && n < 3) {
    h->acc -= step;
    n += 1;
  }
  if (n == 0) return VF_OK;
  return vf_fluid_tick(h, n, changed);
}

int vf_fluid_download_changes(vf_fluid* h, vf_voxel* out, uint64_t cap, uint64_t* n) {
  int rc = check(h);
  if (rc) return rc;
  if ((rc = sync_ctl(h))) return rc;
  uint64_t total = std::min<uint64_t>(h->hctl->nchg, h->R.chg_cap);
  if (n) *n = total;
  uint64_t take = std::min(total, cap);
  if (!take || !out) return VF_OK;
  const size_t vox_bytes = align16(take * sizeof(Voxel));
  if ((rc = ensure_scratch(h, vox_bytes + (total - take) * 4))) return rc;
  k_gather_changes<<<(unsigned)std::min<uint64_t>((take + 255) / 256, 4096), 256, 0, h->stream>>>(h->R, take, (Voxel*)h->scratch);
  CK(cudaGetLastError());
  CK(cudaMemcpyAsync(out, h->scratch, take * sizeof(Voxel), cudaMemcpyDeviceToHost, h->stream));
  if (take < total) {
    // keep the rest pending: move it to the front of the list through the scratch buffer (the
    // source and destination ranges may overlap)
    unsigned* tmp = (unsigned*)((char*)h->scratch + vox_bytes);
    CK(cudaMemcpyAsync(tmp, h->R.chg + take, (total - take) * 4, cudaMemcpyDeviceToDevice, h->stream));
    CK(cudaMemcpyAsync(h->R.chg, tmp, (total - take) * 4, cudaMemcpyDeviceToDevice, h->stream));
  }
  unsigned long long left = total - take;
  CK(cudaMemcpyAsync(&h->R.ctl->nchg, &left, 8, cudaMemcpyHostToDevice, h->stream));
  return sync_ctl(h);
}

// ------------------------------------------------------- allocation-free change download
// Some callers must not allocate device memory while they run: a game's per-frame loop cannot
// afford the device-wide stall that cudaMalloc/cudaFree may cause, and an engine that hands a
// fixed memory budget to its subsystems at start-up forbids allocations after that. For them,
// vf_fluid_download_changes_noalloc gathers into this fixed array instead of the handle's
// growable scratch buffer. The array is VF_NOALLOC_MAX_CHANGES entries (1 MiB) on every device
// that loads the library, held until the process exits, and shared by every call on that device:
// each call overwrites what the previous one left there, so calls whose work overlaps on the GPU
// (for example from two host threads or two streams at once) race and must be serialised.
static __device__ __align__(256) Voxel g_noalloc_changes[VF_NOALLOC_MAX_CHANGES];

namespace {
constexpr int NOALLOC_MAX_DEVICES = 64;
std::mutex g_noalloc_mu;
Voxel* g_noalloc_ptr[NOALLOC_MAX_DEVICES] = {};

// The device address of the array, looked up once per device with that device current.
int noalloc_buffer(vf_fluid* h, Voxel** out) {
  if (h->device < 0 || h->device >= NOALLOC_MAX_DEVICES) return fail(h, VF_ERR_INVALID, "device ordinal out of range");
  std::lock_guard<std::mutex> lock(g_noalloc_mu);
  if (!g_noalloc_ptr[h->device]) {
    DeviceScope scope(h->device);  // the caller's current device is given back on return
    CK(scope.err);
    void* p = nullptr;
    cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_changes);
    if (e != cudaSuccess || !p) return fail(h, VF_ERR_CUDA, std::string("cudaGetSymbolAddress: ") + cudaGetErrorString(e));
    g_noalloc_ptr[h->device] = (Voxel*)p;
  }
  *out = g_noalloc_ptr[h->device];
  return VF_OK;
}
}  // namespace

// Takes the last `take` pending changes (the list's order carries no meaning), writes their final
// material into `out`, clears their pending bits and shortens the list, so nothing needs moving.
__global__ void k_gather_changes_tail(Region R, unsigned long long total, unsigned long long take, Voxel* out) {
  const unsigned long long first = total - take;
  for (unsigned long long i = blockIdx.x * (unsigned long long)blockDim.x + threadIdx.x; i < take; i += (unsigned long long)gridDim.x * blockDim.x) {
    unsigned id = R.chg[first + i];
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
  if (blockIdx.x == 0 && threadIdx.x == 0) R.ctl->nchg = first;
}

int vf_fluid_download_changes_noalloc(vf_fluid* h, vf_voxel* out, uint64_t cap, uint64_t* n) {
  int rc = check(h);
  if (rc) return rc;
  DeviceScope scope(h->device);  // the caller's current device is given back on return
  if (out && cap > VF_NOALLOC_MAX_CHANGES) {
    char b[160];
    snprintf(b, sizeof b, "download_changes_noalloc: cap %llu exceeds its fixed buffer of %d changes per call",
             (unsigned long long)cap, VF_NOALLOC_MAX_CHANGES);
    return fail(h, VF_ERR_RANGE, b);
  }
  Voxel* buf = nullptr;
  if ((rc = noalloc_buffer(h, &buf))) return rc;
  if ((rc = sync_ctl(h))) return rc;
  const uint64_t total = std::min<uint64_t>(h->hctl->nchg, h->R.chg_cap);
  if (n) *n = total;
  const uint64_t take = std::min(total, cap);
  if (!take || !out) return VF_OK;
  k_gather_changes_tail<<<(unsigned)std::min<uint64_t>((take + 255) / 256, 256), 256, 0, h->stream>>>(h->R, total, take, buf);
  CK(cudaGetLastError());
  CK(cudaMemcpyAsync(out, buf, take * sizeof(Voxel), cudaMemcpyDeviceToHost, h->stream));
  return sync_ctl(h);
}

int vf_fluid_volume(vf_fluid* h, int32_t x, int32_t y, int32_t z, float* out) {
  int rc = check(h);
  if (rc) return rc;
  DeviceScope scope(h->device);  // the caller's current device is given back on return
  if (!out) return VF_ERR_INVALID;
  if ((rc = ensure_scratch(h, 64))) return rc;
  k_export_box<<<1, 32, 0, h->stream>>>(h->R, x, y, z, 1, 1, 1, (unsigned char*)h->scratch, (float*)((char*)h->scratch + 16));
  CK(cudaGetLastError());
  unsigned char m = 0;
  float p = 0.0f;
  CK(cudaMemcpyAsync(&m, h->scratch, 1, cudaMemcpyDeviceToHost, h->stream));
  CK(cudaMemcpyAsync(&p, (char*)h->scratch + 16, 4, cudaMemcpyDeviceToHost, h->stream));
  CK(cudaStreamSynchronize(h->stream));
  // FluidSim::volume (fluid.rs:251-260); outside cells export as material 0, partial 0
  *out = p > 0.0f ? p : (m == VF_FLUID_WATER ? 1.0f : 0.0f);
  return VF_OK;
}

int vf_fluid_get_stats(vf_fluid* h, vf_fluid_stats* o) {
  int rc = check(h);
  if (rc) return rc;
  DeviceScope scope(h->device);  // the caller's current device is given back on return
  if (!o) return VF_ERR_INVALID;
  if ((rc = sync_ctl(h))) return rc;
  const Ctl& c = *h->hctl;
  std::memset(o, 0, sizeof(*o));
  o->tick_no = c.tick_no;
  o->last_tick_cells = c.last_cells;
  o->active_count = c.qtail - c.qhead;
  o->partial_count = (uint64_t)c.partial_count;
  o->seed_count = c.nseeds;
  o->level_round = c.level_round;
  o->last_level_cells = c.last_level_cells;
  size_t bytes = 0;
  {
    const Region& R = h->R;
    uint64_t words = ((uint64_t)R.ncells + 31) / 32;
    uint64_t tiles = (uint64_t)R.TX * R.PY * R.TZ;
    bytes += (uint64_t)R.bx * R.by * R.bz * 4 + (uint64_t)R.atlas_cap * 512 * 5 + words * 4 * 3 + tiles * (512 + 8) +
             (uint64_t)R.chg_cap * 4 + (R.qmask + 1) * 4 + (uint64_t)MAX_CELLS_PER_TICK * 8 + MAX_LEVEL_SEEDS * 4 +
             (uint64_t)(MAX_LEVEL_CELLS + 8) * 8;
  }
  o->memory_bytes = bytes;
  o->cells_total = c.cells_total;
  o->pull_attempts = c.pull_attempts;
  o->pull_success = c.pull_success;
  o->bfs_visits = c.bfs_visits;
  o->level_cells_total = c.level_cells_total;
  o->atlas_used = c.atlas_used;
  o->changes_pending = c.nchg;
  return VF_OK;
}

int vf_fluid_export_partials(vf_fluid* h, int32_t* xyz, float* vol, uint64_t cap, uint64_t* n) {
  int rc = check(h);
  if (rc) return rc;
  DeviceScope scope(h->device);  // the caller's current device is given back on return
  if ((rc = sync_ctl(h))) return rc;
  unsigned nslots = std::min(h->hctl->atlas_used, h->R.atlas_cap);
  const size_t o_count = align16((size_t)nslots * 4), o_xyz = o_count + 64, o_vol = o_xyz + align16(cap * 12);
  if ((rc = ensure_scratch(h, o_vol + align16(cap * 4) + 16))) return rc;
  int* slot_brick = (int*)h->scratch;
  unsigned long long* dcount = (unsigned long long*)((char*)h->scratch + o_count);
  int* dxyz = (int*)((char*)h->scratch + o_xyz);
  float* dvol = (float*)((char*)h->scratch + o_vol);
  CK(cudaMemsetAsync(slot_brick, 0xFF, (size_t)nslots * 4 + 8, h->stream));
  CK(cudaMemsetAsync(dcount, 0, 8, h->stream));
  uint64_t nb = (uint64_t)h->R.bx * h->R.by * h->R.bz;
  k_slot_map<<<(unsigned)std::min<uint64_t>((nb + 255) / 256, 8192), 256, 0, h->stream>>>(h->R, slot_brick, nslots);
  if (nslots)
    k_export_partials<<<(unsigned)std::min<uint64_t>(((uint64_t)nslots * 512 + 255) / 256, 16384), 256, 0, h->stream>>>(h->R, nslots, dxyz, dvol,
                                                                                                                         cap, dcount, slot_brick);
  CK(cudaGetLastError());
  unsigned long long cnt = 0;
  CK(cudaMemcpyAsync(&cnt, dcount, 8, cudaMemcpyDeviceToHost, h->stream));
  CK(cudaStreamSynchronize(h->stream));
  uint64_t take = std::min<uint64_t>(cnt, cap);
  if (take && xyz) CK(cudaMemcpy(xyz, dxyz, take * 12, cudaMemcpyDeviceToHost));
  if (take && vol) CK(cudaMemcpy(vol, dvol, take * 4, cudaMemcpyDeviceToHost));
  // entries kept for evicted ring chunks
  std::vector<uint8_t> live;
  if ((rc = detached_live(h, live))) return rc;
  for (size_t k = 0; k < h->det.size(); ++k) {
    if (!live[k]) continue;
    if (take < cap) {
      if (xyz) {
        xyz[3 * take] = h->det[k].x;
        xyz[3 * take + 1] = h->det[k].y;
        xyz[3 * take + 2] = h->det[k].z;
      }
      if (vol) vol[take] = h->det[k].v;
      ++take;
    }
    ++cnt;
  }
  if (n) *n = cnt;
  // canonical order: by (x, y, z) ascending? keep (slot, voxel) order but make it deterministic
  if (take && xyz && vol) {
    std::vector<uint64_t> idx(take);
    for (uint64_t i = 0; i < take; ++i) idx[i] = i;
    std::sort(idx.begin(), idx.end(), [&](uint64_t a, uint64_t b) {
      return std::make_tuple(xyz[3 * a + 2], xyz[3 * a + 1], xyz[3 * a]) < std::make_tuple(xyz[3 * b + 2], xyz[3 * b + 1], xyz[3 * b]);
    });
    std::vector<int32_t> x2(take * 3);
    std::vector<float> v2(take);
    for (uint64_t i = 0; i < take; ++i) {
      std::memcpy(&x2[3 * i], &xyz[3 * idx[i]], 12);
      v2[i] = vol[idx[i]];
    }
    std::memcpy(xyz, x2.data(), take * 12);
    std::memcpy(vol, v2.data(), take * 4);
  }
  return VF_OK;
}

int vf_fluid_shift(vf_fluid* h, int32_t dx, int32_t dz) {  // fluid.rs:696-720
  int rc = check(h);
  if (rc) return rc;
  DeviceScope scope(h->device);  // the caller's current device is given back on return
  // Ring worlds move their origin by whole ring periods (sparse_volume.rs:194-203): the brick
  // slots then stay where they are, only coordinates change. Cell ids are relative to the padded
  // domain's origin, so moving the origin re-keys the FIFO, seeds and partials at once.
  const Region& R = h->R;
  if (!R.ring_w || (dx % (R.ring_w * 128)) != 0 || (dz % (R.ring_w * 128)) != 0)
    return fail(h, VF_ERR_RANGE, "shift supports ring worlds moved by whole ring periods");
  if ((rc = sync_ctl(h))) return rc;
  h->R.px0 -= dx;
  h->R.pz0 -= dz;
  // the ring slots' owners move with the origin (the host rebases its SparseVolume alike)
  std::vector<int32_t> ring(3 * R.ring_w * R.ring_w);
  CK(cudaMemcpy(ring.data(), R.ring, ring.size() * 4, cudaMemcpyDeviceToHost));
  for (size_t i = 0; i < ring.size(); i += 3) {
    ring[i] -= dx / 128;
    ring[i + 1] -= dz / 128;
  }
  CK(cudaMemcpy(R.ring, ring.data(), ring.size() * 4, cudaMemcpyHostToDevice));
  for (DetachedPartial& e : h->det) {  // PartialField re-keyed (fluid.rs:697-701); ids are domain-relative
    e.x -= dx;
    e.z -= dz;
  }
  // the levelling round starts over (fluid.rs:715-719)
  const unsigned nt = h->hctl->mark_ntiles;
  if (nt) {
    const uint64_t tiles = (uint64_t)R.TX * R.PY * R.TZ;
    CK(cudaMemsetAsync(R.marks, 0, tiles * 128 * 4, h->stream));
    CK(cudaMemsetAsync(R.mark_tflag, 0, tiles * 4, h->stream));
  }
  unsigned zero = 0;
  CK(cudaMemcpyAsync(&R.ctl->mark_ntiles, &zero, 4, cudaMemcpyHostToDevice, h->stream));
  CK(cudaMemcpyAsync(&R.ctl->level_round, &zero, 4, cudaMemcpyHostToDevice, h->stream));
  CK(cudaMemcpyAsync(h->dR, &h->R, sizeof(Region), cudaMemcpyHostToDevice, h->stream));
  return sync_ctl(h);
}

int vf_fluid_ring_evict(vf_fluid* h, int32_t cx, int32_t cz) {  // sparse_volume.rs:513-537
  int rc = check(h);
  if (rc) return rc;
  if (!h->R.ring_w) return fail(h, VF_ERR_INVALID, "not a ring world");
  DeviceScope scope(h->device);
  if (scope.err != cudaSuccess) return VF_ERR_CUDA;
  if ((rc = sync_ctl(h))) return rc;
  const int w = h->R.ring_w;
  std::vector<int32_t> ring(3 * w * w);
  CK(cudaMemcpy(ring.data(), h->R.ring, ring.size() * 4, cudaMemcpyDeviceToHost));
  return ring_evict_slot(h, (cz & (w - 1)) * w + (cx & (w - 1)), ring);
}

int vf_fluid_ring_paste(vf_fluid* h, const uint32_t* chunk_grid, const uint8_t* chunk_bricks, uint64_t chunk_nbricks, int32_t chunk_bricks_y,
                        int32_t cx, int32_t cz) {  // sparse_volume.rs:478-510
  int rc = check(h);
  if (rc) return rc;
  Region& R = h->R;
  if (!R.ring_w || !chunk_grid || chunk_bricks_y <= 0) return fail(h, VF_ERR_INVALID, "ring paste: not a ring world or no chunk");
  if ((int64_t)cx * 128 < R.px0 || (int64_t)cx * 128 + 128 > (int64_t)R.px0 + R.PX || (int64_t)cz * 128 < R.pz0 ||
      (int64_t)cz * 128 + 128 > (int64_t)R.pz0 + R.PZ)
    return fail(h, VF_ERR_RANGE, "ring paste: the chunk lies outside the handle's cell domain (the chunks loaded at upload, after shifts)");
  DeviceScope scope(h->device);
  if (scope.err != cudaSuccess) return VF_ERR_CUDA;
  if ((rc = sync_ctl(h))) return rc;
  const int w = R.ring_w, si = (cz & (w - 1)) * w + (cx & (w - 1));
  std::vector<int32_t> ring(3 * w * w);
  CK(cudaMemcpy(ring.data(), R.ring, ring.size() * 4, cudaMemcpyDeviceToHost));
  if ((rc = ring_evict_slot(h, si, ring))) return rc;  // whatever the slot held
  // kept entries of this chunk's cells that no tick erased come back with it
  std::vector<uint8_t> live;
  if ((rc = detached_live(h, live))) return rc;
  std::vector<DetachedPartial> keep;
  std::vector<std::vector<std::pair<int, float>>> brick_parts(16 * 16 * (size_t)R.by);
  std::vector<unsigned> back;
  for (size_t k = 0; k < h->det.size(); ++k) {
    if (!live[k]) continue;  // erased while its chunk was away
    const DetachedPartial& e = h->det[k];
    if ((e.x >> 7) != cx || (e.z >> 7) != cz || e.y / 8 >= std::min(R.by, chunk_bricks_y)) {
      keep.push_back(e);
      continue;
    }
    const int bx = (e.x & 127) >> 3, by = e.y >> 3, bz = (e.z & 127) >> 3;
    brick_parts[((size_t)bz * R.by + by) * 16 + bx].push_back({(e.z & 7) * 64 + (e.y & 7) * 8 + (e.x & 7), e.v});
    back.push_back(e.id);
  }
  const uint64_t nb = (uint64_t)R.bx * R.by * R.bz;
  std::vector<uint32_t> grid(nb);
  CK(cudaMemcpy(grid.data(), R.grid, nb * 4, cudaMemcpyDeviceToHost));
  const int bx0 = (si % w) * 16, bz0 = (si / w) * 16;
  std::vector<unsigned> slots;
  std::vector<uint8_t> mats;
  std::vector<float> vols;
  unsigned used = h->hctl->atlas_used;
  for (int bz = 0; bz < 16; ++bz)
    for (int by = 0; by < std::min(R.by, chunk_bricks_y); ++by)
      for (int bx = 0; bx < 16; ++bx) {
        const uint32_t g = chunk_grid[((size_t)bz * chunk_bricks_y + by) * 16 + bx];
        if (g >= 256u && (g - 256u >= chunk_nbricks || !chunk_bricks)) return fail(h, VF_ERR_INVALID, "ring paste: grid names a brick out of range");
        const auto& parts = brick_parts[((size_t)bz * R.by + by) * 16 + bx];
        const uint64_t gi = ((uint64_t)(bz0 + bz) * R.by + by) * R.bx + (bx0 + bx);
        if (g < 256u && parts.empty()) {
          grid[gi] = g;
          continue;
        }
        unsigned slot;
        if (!h->free_slots.empty()) {
          slot = h->free_slots.back();
          h->free_slots.pop_back();
        } else {
          if (used >= R.atlas_cap) return fail(h, VF_ERR_OOM, "ring paste: brick atlas full");
          slot = used++;
        }
        slots.push_back(slot);
        const size_t o = mats.size();
        mats.resize(o + 512);
        vols.resize(o + 512, 0.0f);
        if (g < 256u) std::memset(&mats[o], (int)g, 512);
        else std::memcpy(&mats[o], chunk_bricks + (size_t)(g - 256u) * 512, 512);
        for (const auto& pr : parts) vols[o + pr.first] = pr.second;
        grid[gi] = 256u + slot;
      }
  if (!slots.empty()) {
    const size_t n = slots.size();
    if ((rc = ensure_scratch(h, align16(n * 4) + n * 512 + n * 2048 + 64))) return rc;
    unsigned* dslots = (unsigned*)h->scratch;
    uint8_t* dm = (uint8_t*)h->scratch + align16(n * 4);
    float* dv = (float*)(dm + n * 512);
    CK(cudaMemcpyAsync(dslots, slots.data(), n * 4, cudaMemcpyHostToDevice, h->stream));
    CK(cudaMemcpyAsync(dm, mats.data(), n * 512, cudaMemcpyHostToDevice, h->stream));
    CK(cudaMemcpyAsync(dv, vols.data(), n * 2048, cudaMemcpyHostToDevice, h->stream));
    k_scatter_bricks<<<(unsigned)std::min<size_t>((n * 512 + 255) / 256, 8192), 256, 0, h->stream>>>(R.amat, R.avol, dslots, (unsigned)n, dm, dv);
    CK(cudaGetLastError());
    CK(cudaStreamSynchronize(h->stream));
  }
  if (used != h->hctl->atlas_used) {
    h->hctl->atlas_used = used;
    CK(cudaMemcpy(&R.ctl->atlas_used, &used, 4, cudaMemcpyHostToDevice));
  }
  CK(cudaMemcpy(R.grid, grid.data(), nb * 4, cudaMemcpyHostToDevice));
  ring[3 * si] = cx;
  ring[3 * si + 1] = cz;
  ring[3 * si + 2] = 1;
  CK(cudaMemcpy(R.ring, ring.data(), ring.size() * 4, cudaMemcpyHostToDevice));
  // the returned entries live in the atlas again; erased ones are gone for good
  if ((rc = detached_bits(h, back, 0))) return rc;
  if ((rc = detached_count(h, -(long long)back.size()))) return rc;
  h->det.swap(keep);
  return VF_OK;
}

int vf_fluid_reset(vf_fluid* h) {  // fluid.rs:318-320: the fluid's tables only
  int rc = check(h);
  if (rc) return rc;
  DeviceScope scope(h->device);  // the caller's current device is given back on return
  const Region& R = h->R;
  if ((rc = sync_ctl(h))) return rc;
  unsigned used = h->hctl->atlas_used;
  CK(cudaMemsetAsync(R.avol, 0, (size_t)used * 512 * 4, h->stream));
  uint64_t words = ((uint64_t)R.ncells + 31) / 32;
  CK(cudaMemsetAsync(R.active, 0, words * 4, h->stream));
  CK(cudaMemsetAsync(R.seedbits, 0, words * 4, h->stream));
  const uint64_t tiles = (uint64_t)R.TX * R.PY * R.TZ;
  CK(cudaMemsetAsync(R.marks, 0, tiles * 128 * 4, h->stream));
  CK(cudaMemsetAsync(R.mark_tflag, 0, tiles * 4, h->stream));
  // per-tick maps a failed tick may have left set (cell positions, rows, pull-written cells)
  CK(cudaMemsetAsync(R.stamp, 0xFF, (size_t)R.ncells * 4, h->stream));
  CK(cudaMemsetAsync(R.zrow, 0xFF, (size_t)R.PY * R.PZ * 4, h->stream));
  CK(cudaMemsetAsync(R.ptbits, 0, words * 4, h->stream));
  if (R.detbits) CK(cudaMemsetAsync(R.detbits, 0, words * 4, h->stream));  // kept entries go with the rest
  h->det.clear();
  Ctl c = *h->hctl;
  Ctl z{};
  z.atlas_used = c.atlas_used;
  z.nchg = c.nchg;  // voxel changes still owed to the host
  // the cumulative counters and phase cycles are diagnostics, not fluid state: they run on
  z.cells_total = c.cells_total;
  z.pull_attempts = c.pull_attempts;
  z.pull_success = c.pull_success;
  z.bfs_visits = c.bfs_visits;
  z.level_cells_total = c.level_cells_total;
  z.activations = c.activations;
  z.seg_epoch = c.seg_epoch;
  z.par_segments = c.par_segments;
  z.par_rollbacks = c.par_rollbacks;
  z.par_replayed = c.par_replayed;
  std::memcpy(z.par_conflicts, c.par_conflicts, sizeof(z.par_conflicts));
  std::memcpy(z.pprof, c.pprof, sizeof(z.pprof));
  std::memcpy(z.prof, c.prof, sizeof(z.prof));
  CK(cudaMemcpyAsync(R.ctl, &z, sizeof(Ctl), cudaMemcpyHostToDevice, h->stream));
  h->acc = 0.0f;
  return sync_ctl(h);
}

int vf_fluid_snapshot_queue(vf_fluid* h, int32_t* q_xyz, uint64_t q_cap, uint64_t* nq, int32_t* s_xyz, uint64_t s_cap, uint64_t* ns) {
  int rc = check(h);
  if (rc) return rc;
  DeviceScope scope(h->device);  // the caller's current device is given back on return
  if ((rc = sync_ctl(h))) return rc;
  const Region& R = h->R;
  uint64_t len = h->hctl->qtail - h->hctl->qhead;
  if (nq) *nq = len;
  uint64_t take = std::min(len, q_cap);
  if (take && q_xyz) {
    std::vector<uint32_t> ids(take);
    uint64_t cap = R.qmask + 1, head = h->hctl->qhead & R.qmask;
    uint64_t first = std::min(take, cap - head);
    CK(cudaMemcpy(ids.data(), R.queue + head, first * 4, cudaMemcpyDeviceToHost));
    if (take > first) CK(cudaMemcpy(ids.data() + first, R.queue, (take - first) * 4, cudaMemcpyDeviceToHost));
    for (uint64_t i = 0; i < take; ++i) dom_xyz(R, ids[i], q_xyz[3 * i], q_xyz[3 * i + 1], q_xyz[3 * i + 2]);
  }
  uint64_t sl = h->hctl->nseeds;
  if (ns) *ns = sl;
  uint64_t st = std::min(sl, s_cap);
  if (st && s_xyz) {
    std::vector<uint32_t> ids(st);
    CK(cudaMemcpy(ids.data(), R.seeds, st * 4, cudaMemcpyDeviceToHost));
    for (uint64_t i = 0; i < st; ++i) dom_xyz(R, ids[i], s_xyz[3 * i], s_xyz[3 * i + 1], s_xyz[3 * i + 2]);
  }
  return VF_OK;
}

int vf_fluid_export_box(vf_fluid* h, int32_t x0, int32_t y0, int32_t z0, int32_t sx, int32_t sy, int32_t sz, uint8_t* mat, float* part) {
  int rc = check(h);
  if (rc) return rc;
  DeviceScope scope(h->device);  // the caller's current device is given back on return
  if (sx <= 0 || sy <= 0 || sz <= 0) return VF_ERR_INVALID;
  uint64_t n = (uint64_t)sx * sy * sz;
  if ((rc = ensure_scratch(h, n * 5 + 64))) return rc;
  unsigned char* dm = (unsigned char*)h->scratch;
  float* dp = (float*)((char*)h->scratch + ((n + 15) / 16) * 16);
  k_export_box<<<(unsigned)std::min<uint64_t>((n + 255) / 256, 16384), 256, 0, h->stream>>>(h->R, x0, y0, z0, sx, sy, sz, dm, dp);
  CK(cudaGetLastError());
  if (mat) CK(cudaMemcpyAsync(mat, dm, n, cudaMemcpyDeviceToHost, h->stream));
  if (part) CK(cudaMemcpyAsync(part, dp, n * 4, cudaMemcpyDeviceToHost, h->stream));
  CK(cudaStreamSynchronize(h->stream));
  return VF_OK;
}

int vf_fluid_digest(vf_fluid* h, uint64_t* state, uint64_t* queue, uint64_t* seeds) {
  int rc = check(h);
  if (rc) return rc;
  DeviceScope scope(h->device);  // the caller's current device is given back on return
  if ((rc = sync_ctl(h))) return rc;
  if ((rc = ensure_scratch(h, 64 + h->det.size() * 20 + 32))) return rc;
  unsigned long long* d = (unsigned long long*)h->scratch;
  CK(cudaMemsetAsync(d, 0, 24, h->stream));
  const Region& R = h->R;
  uint64_t nvox = (uint64_t)R.bx * R.by * R.bz * 512;
  k_state_digest<<<(unsigned)std::min<uint64_t>((nvox + 255) / 256, 16384), 256, 0, h->stream>>>(R, d);
  uint64_t ql = h->hctl->qtail - h->hctl->qhead;
  if (ql) k_list_digest<<<(unsigned)std::min<uint64_t>((ql + 255) / 256, 4096), 256, 0, h->stream>>>(R, R.queue, ql, h->hctl->qhead, R.qmask, d + 1);
  uint64_t sl = h->hctl->nseeds;
  if (sl) k_list_digest<<<(unsigned)((sl + 255) / 256), 256, 0, h->stream>>>(R, R.seeds, sl, 0, 0xFFFFFFFFFFFFFFFFull, d + 2);
  if (!h->det.empty()) {  // entries kept for evicted ring chunks, hashed as cells outside the loaded chunks
    const size_t nd = h->det.size();
    std::vector<int4> ent(nd);
    std::vector<unsigned> ids(nd);
    for (size_t k = 0; k < nd; ++k) {
      unsigned vb;
      std::memcpy(&vb, &h->det[k].v, 4);
      ent[k] = make_int4(h->det[k].x, h->det[k].y, h->det[k].z, (int)vb);
      ids[k] = h->det[k].id;
    }
    int4* dent = (int4*)((char*)h->scratch + 64);
    unsigned* dids = (unsigned*)((char*)h->scratch + 64 + nd * 16);
    CK(cudaMemcpyAsync(dent, ent.data(), nd * 16, cudaMemcpyHostToDevice, h->stream));
    CK(cudaMemcpyAsync(dids, ids.data(), nd * 4, cudaMemcpyHostToDevice, h->stream));
    k_detached_digest<<<(unsigned)std::min<size_t>((nd + 255) / 256, 1024), 256, 0, h->stream>>>(R, dent, dids, (unsigned)nd, d);
    CK(cudaStreamSynchronize(h->stream));
  }
  CK(cudaGetLastError());
  unsigned long long out[3];
  CK(cudaMemcpyAsync(out, d, 24, cudaMemcpyDeviceToHost, h->stream));
  CK(cudaStreamSynchronize(h->stream));
  if (state) *state = out[0];
  if (queue) *queue = out[1];
  if (seeds) *seeds = out[2];
  return VF_OK;
}

int vf_fluid_profile(vf_fluid* h, uint64_t* out16) {
  int rc = check(h);
  if (rc) return rc;
  DeviceScope scope(h->device);  // the caller's current device is given back on return
  if ((rc = sync_ctl(h))) return rc;
  if (out16) std::memcpy(out16, h->hctl->prof, 16 * sizeof(uint64_t));
  return VF_OK;
}

#ifdef VF_FINE_PROFILE
// Fine-profiling builds only: all 32 counters (the 16 phases and the per-call counters).
extern "C" int vf_fluid_profile_fine(vf_fluid* h, uint64_t* out32) {
  int rc = check(h);
  if (rc) return rc;
  if ((rc = sync_ctl(h))) return rc;
  if (out32) std::memcpy(out32, h->hctl->prof, 32 * sizeof(uint64_t));
  return VF_OK;
}
#endif

// ---------------------------------------------------------------- learned wake proposal
static int proposal_buffers(vf_fluid* h) {
  if (h->slot_gi) return VF_OK;
  const unsigned cap = h->R.atlas_cap;
  int rc;
  if ((rc = dalloc(h, &h->slot_gi, cap, false))) return rc;
  if ((rc = dalloc(h, &h->aggr, cap, false))) return rc;
  if ((rc = dalloc(h, &h->whist, (size_t)cap * 4))) return rc;
  if ((rc = dalloc(h, &h->staged, 4))) return rc;
  return VF_OK;
}

// Features of every materialised brick at the current state: dev_x gets nslots x 32 fp16
// (row s = atlas slot s). Each call also advances the 4-call water-sum history used for the
// flux features, so call it once per tick while the proposal runs.
int vf_fluid_proposal_features(vf_fluid* h, void* dev_x, uint64_t cap_slots, uint64_t* nslots) {
  int rc = check(h);
  if (rc) return rc;
  DeviceScope scope(h->device);  // the caller's current device is given back on return
  if ((rc = proposal_buffers(h))) return rc;
  if ((rc = sync_ctl(h))) return rc;
  const unsigned n = std::min(h->hctl->atlas_used, h->R.atlas_cap);
  if (nslots) *nslots = n;
  if (!dev_x || cap_slots < n || !n) return dev_x && cap_slots < n ? VF_ERR_INVALID : VF_OK;
  const uint64_t nb = (uint64_t)h->R.bx * h->R.by * h->R.bz;
  CK(cudaMemsetAsync(h->slot_gi, 0xFF, (size_t)n * 4, h->stream));
  k_slot_map<<<(unsigned)std::min<uint64_t>((nb + 255) / 256, 8192), 256, 0, h->stream>>>(h->R, h->slot_gi, n);
  k_slot_aggr<<<std::min(n, 16384u), 128, 0, h->stream>>>(h->R, h->slot_gi, n, h->aggr);
  k_slot_features<<<(n + 255) / 256, 256, 0, h->stream>>>(h->R, h->aggr, n, h->whist, h->hpos, h->hctl->tick_no, (__half*)dev_x);
  k_slot_hist<<<(n + 255) / 256, 256, 0, h->stream>>>(h->aggr, n, h->whist, h->hpos);
  h->hpos += 1;
  CK(cudaGetLastError());
  return VF_OK;
}

// Labels for features taken at tick `since`: 1 where the brick woke in (since, now].
int vf_fluid_proposal_labels(vf_fluid* h, uint32_t since_tick, float* dev_y, uint64_t nslots) {
  int rc = check(h);
  if (rc) return rc;
  DeviceScope scope(h->device);  // the caller's current device is given back on return
  if ((rc = sync_ctl(h))) return rc;
  if (!nslots) return VF_OK;
  if (!dev_y) return VF_ERR_INVALID;
  const unsigned n = (unsigned)std::min<uint64_t>(nslots, h->R.atlas_cap);
  k_slot_labels<<<(n + 255) / 256, 256, 0, h->stream>>>(h->R, n, since_tick, h->hctl->tick_no, dev_y);
  CK(cudaGetLastError());
  return VF_OK;
}

// Pre-stage (L2 prefetch) the bricks whose wake probability is >= threshold; the exact FIFO still
// decides what runs. *n_staged (optional) = bricks staged.
int vf_fluid_stage_bricks(vf_fluid* h, const float* dev_prob, uint64_t nslots, float threshold, uint64_t* n_staged) {
  int rc = check(h);
  if (rc) return rc;
  DeviceScope scope(h->device);  // the caller's current device is given back on return
  if ((rc = proposal_buffers(h))) return rc;
  if (!nslots) return VF_OK;
  const unsigned n = (unsigned)std::min<uint64_t>(nslots, h->R.atlas_cap);
  CK(cudaMemsetAsync(h->staged, 0, 4, h->stream));
  k_stage<<<(n + 255) / 256, 256, 0, h->stream>>>(h->R, n, dev_prob, threshold, h->staged);
  CK(cudaGetLastError());
  if (n_staged) {
    unsigned c = 0;
    CK(cudaMemcpyAsync(&c, h->staged, 4, cudaMemcpyDeviceToHost, h->stream));
    CK(cudaStreamSynchronize(h->stream));
    *n_staged = c;
  }
  return VF_OK;
}

int vf_fluid_set_tuning(vf_fluid* h, int32_t producers, int32_t depth) {
  if (!h || producers < 1 || producers > TICK_WARPS - 1 || depth < 1 || depth > PF_RING) return VF_ERR_INVALID;
  h->tune.producers = producers;
  h->tune.depth = depth;
  return VF_OK;
}

int vf_fluid_set_sweep(vf_fluid* h, int32_t engine, int32_t gate, uint64_t spin_cap) {
  const int warps = (gate >> 16) & 0x1F;
  if (!h || engine < 0 || engine > 2 || gate < 0 || (gate & 0xFF) > GATE_MAX || ((gate >> 8) & 0xFF) > GATE_MAX || (gate >> 22) ||
      (warps != 0 && (warps < 8 || warps > MAX_WARPS)) || spin_cap == 0)
    return VF_ERR_INVALID;
  if (engine == 1 && h->uploaded && (h->R.PX >= 65536 || h->R.PZ >= 65536 || h->R.PY >= 65536))
    return fail(h, VF_ERR_RANGE, "the parallel sweep needs domain sides below 65536");
  h->auto_engine = engine == 2;
  if (engine != 2) h->tune.engine = engine;
  h->tune.gate = gate;
  h->tune.spin_cap = spin_cap;
  return VF_OK;
}

int vf_fluid_set_log_caps(vf_fluid* h, uint32_t act, uint32_t seed, uint32_t chg) {
  int rc = check(h);
  if (rc) return rc;
  if (act < 1 || act > (1u << 22) || seed < 1 || seed > (1u << 18) || chg < 1 || chg > (1u << 21)) return VF_ERR_INVALID;
  DeviceScope scope(h->device);
  if (scope.err != cudaSuccess) return VF_ERR_CUDA;
  if ((rc = sync_ctl(h))) return rc;
  h->R.ev_act_cap = act;
  h->R.ev_seed_cap = seed;
  h->R.ev_chg_cap = chg;
  CK(cudaMemcpyAsync(h->dR, &h->R, sizeof(Region), cudaMemcpyHostToDevice, h->stream));
  return sync_ctl(h);
}

int vf_fluid_sweep_profile(vf_fluid* h, uint64_t* out18) {
  int rc = check(h);
  if (rc) return rc;
  DeviceScope scope(h->device);  // the caller's current device is given back on return
  if ((rc = sync_ctl(h))) return rc;
  if (out18) std::memcpy(out18, h->hctl->pprof, 18 * sizeof(uint64_t));
  return VF_OK;
}

int vf_fluid_sweep_stats(vf_fluid* h, uint64_t* segments, uint64_t* rollbacks, uint64_t* replayed, uint64_t* conflicts3) {
  int rc = check(h);
  if (rc) return rc;
  DeviceScope scope(h->device);  // the caller's current device is given back on return
  if ((rc = sync_ctl(h))) return rc;
  if (segments) *segments = h->hctl->par_segments;
  if (rollbacks) *rollbacks = h->hctl->par_rollbacks;
  if (replayed) *replayed = h->hctl->par_replayed;
  if (conflicts3)
    for (int i = 0; i < 3; ++i) conflicts3[i] = h->hctl->par_conflicts[i];
  return VF_OK;
}

// Host edits that take their cell list from DEVICE memory and do not wait: capturable in a
// CUDA graph together with vf_batch_tick_async / vf_fluid_tick_async.
int vf_fluid_emit_device_async(vf_fluid* h, const int32_t* dev_xyz, uint64_t n, float amount) {
  int rc = check(h);
  if (rc) return rc;
  DeviceScope scope(h->device);  // the caller's current device is given back on return
  k_edit<<<1, 32, 0, h->stream>>>(h->R, ED_EMIT, dev_xyz, n, 0, amount, nullptr);
  CK(cudaGetLastError());
  return VF_OK;
}

int vf_fluid_brush_device_async(vf_fluid* h, const int32_t* dev_xyz, uint64_t n, uint8_t m) {
  int rc = check(h);
  if (rc) return rc;
  DeviceScope scope(h->device);  // the caller's current device is given back on return
  k_edit<<<1, 32, 0, h->stream>>>(h->R, ED_BRUSH, dev_xyz, n, m, 0.0f, nullptr);
  CK(cudaGetLastError());
  return VF_OK;
}

int vf_fluid_wake_async(vf_fluid* h, int32_t x0, int32_t y0, int32_t z0, int32_t x1, int32_t y1, int32_t z1) {
  int rc = check(h);
  if (rc) return rc;
  DeviceScope scope(h->device);  // the caller's current device is given back on return
  if (x1 < x0 || y1 < y0 || z1 < z0) return VF_OK;
  y0 = std::max(y0, 0);
  if (y1 < y0) return VF_OK;
  if (!in_dom(h->R, x0, y0, z0) || !in_dom(h->R, x1, y1, z1)) return fail(h, VF_ERR_RANGE, "wake box outside the padded domain");
  k_wake_box<<<1, 1024, 0, h->stream>>>(h->R, x0, y0, z0, x1, y1, z1);
  CK(cudaGetLastError());
  return VF_OK;
}

int vf_batch_create(vf_fluid* const* hs, int32_t n, vf_batch** out) {
  if (!hs || n <= 0 || !out) return VF_ERR_INVALID;
  vf_fluid* h = hs[0];
  for (int i = 0; i < n; ++i) {
    int rc = check(hs[i]);
    if (rc) return rc;
    if (hs[i]->device != h->device) return fail(h, VF_ERR_INVALID, "batched handles must share a device");
  }
  DeviceScope scope(h->device);
  auto* b = new vf_batch();
  b->hs.assign(hs, hs + n);
  b->stream = h->stream;
  std::vector<Region> regs(n);
  for (int i = 0; i < n; ++i) regs[i] = hs[i]->R;
  if (cudaMalloc(&b->dregs, sizeof(Region) * n) != cudaSuccess) {
    delete b;
    return VF_ERR_OOM;
  }
  if (cudaMemcpy(b->dregs, regs.data(), sizeof(Region) * n, cudaMemcpyHostToDevice) != cudaSuccess) {
    cudaFree(b->dregs);
    delete b;
    return VF_ERR_CUDA;
  }
  *out = b;
  return VF_OK;
}

void vf_batch_destroy(vf_batch* b) {
  if (!b) return;
  DeviceScope scope(b->hs[0]->device);
  if (b->exec) cudaGraphExecDestroy(b->exec);
  if (b->graph) cudaGraphDestroy(b->graph);
  if (b->dregs) cudaFree(b->dregs);
  delete b;
}

int vf_batch_tick_async(vf_batch* b, int32_t n_ticks) {
  if (!b || n_ticks < 0) return VF_ERR_INVALID;
  vf_fluid* h = b->hs[0];
  DeviceScope scope(h->device);
  if (n_ticks) {
    CK(launch_tick(h->tune, b->dregs, (int)b->hs.size(), n_ticks, h->smem_bytes, b->stream));
  }
  return VF_OK;
}

int vf_batch_sync(vf_batch* b) {
  if (!b) return VF_ERR_INVALID;
  vf_fluid* h = b->hs[0];
  DeviceScope scope(h->device);
  CK(cudaStreamSynchronize(b->stream));
  for (vf_fluid* x : b->hs) {
    int rc = sync_ctl(x);
    if (rc) return rc;
  }
  return VF_OK;
}

// Capture `launches` back-to-back launches of `ticks_per_launch` ticks each into a CUDA graph.
int vf_batch_capture(vf_batch* b, int32_t launches, int32_t ticks_per_launch) {
  if (!b || launches <= 0 || ticks_per_launch <= 0) return VF_ERR_INVALID;
  vf_fluid* h = b->hs[0];
  DeviceScope scope(h->device);
  if (b->exec) {
    cudaGraphExecDestroy(b->exec);
    b->exec = nullptr;
  }
  if (b->graph) {
    cudaGraphDestroy(b->graph);
    b->graph = nullptr;
  }
  CK(cudaStreamBeginCapture(b->stream, cudaStreamCaptureModeThreadLocal));
  for (int i = 0; i < launches; ++i)
    launch_tick(h->tune, b->dregs, (int)b->hs.size(), ticks_per_launch, h->smem_bytes, b->stream);
  cudaError_t e = cudaStreamEndCapture(b->stream, &b->graph);
  if (e != cudaSuccess) return fail(h, VF_ERR_CUDA, std::string("capture: ") + cudaGetErrorString(e));
  CK(cudaGraphInstantiate(&b->exec, b->graph, 0));
  return VF_OK;
}

// Record everything enqueued on the batch's stream between these calls (tick launches, device
// edits, wakes of the batch's handles) as one CUDA graph for vf_batch_replay.
int vf_batch_begin_capture(vf_batch* b) {
  if (!b) return VF_ERR_INVALID;
  vf_fluid* h = b->hs[0];
  DeviceScope scope(h->device);
  for (vf_fluid* x : b->hs)
    if (x->stream != b->stream) return fail(h, VF_ERR_INVALID, "capture needs every handle on the batch's stream");
  if (b->exec) {
    cudaGraphExecDestroy(b->exec);
    b->exec = nullptr;
  }
  if (b->graph) {
    cudaGraphDestroy(b->graph);
    b->graph = nullptr;
  }
  CK(cudaStreamBeginCapture(b->stream, cudaStreamCaptureModeThreadLocal));
  return VF_OK;
}

int vf_batch_end_capture(vf_batch* b) {
  if (!b) return VF_ERR_INVALID;
  vf_fluid* h = b->hs[0];
  DeviceScope scope(h->device);
  cudaError_t e = cudaStreamEndCapture(b->stream, &b->graph);
  if (e != cudaSuccess) return fail(h, VF_ERR_CUDA, std::string("capture: ") + cudaGetErrorString(e));
  CK(cudaGraphInstantiate(&b->exec, b->graph, 0));
  return VF_OK;
}

int vf_batch_replay(vf_batch* b) {
  if (!b || !b->exec) return VF_ERR_STATE;
  vf_fluid* h = b->hs[0];
  DeviceScope scope(h->device);
  CK(cudaGraphLaunch(b->exec, b->stream));
  return VF_OK;
}

// ------------------------------------------------------------------------ batched regions
int vf_fluid_batch_tick(vf_fluid* const* hs, int32_t n, int32_t n_ticks) {
  if (!hs || n <= 0 || n_ticks < 0) return VF_ERR_INVALID;
  vf_fluid* h = hs[0];
  for (int i = 0; i < n; ++i) {
    int rc = check(hs[i]);
    if (rc) return rc;
    if (hs[i]->device != h->device) return fail(h, VF_ERR_INVALID, "batched handles must share a device");
  }
  DeviceScope scope(h->device);
  std::vector<Region> regs(n);
  for (int i = 0; i < n; ++i) regs[i] = hs[i]->R;
  int rc;
  if ((rc = ensure_scratch(h, sizeof(Region) * n))) return rc;
  CK(cudaMemcpyAsync(h->scratch, regs.data(), sizeof(Region) * n, cudaMemcpyHostToDevice, h->stream));
  for (int i = 0; i < n; ++i) CK(cudaMemsetAsync(&regs[i].ctl->changed, 0, 4, h->stream));
  if (n_ticks) {
    CK(launch_tick(h->tune, (Region*)h->scratch, n, n_ticks, h->smem_bytes, h->stream));
  }
  CK(cudaStreamSynchronize(h->stream));
  for (int i = 0; i < n; ++i) {
    if ((rc = sync_ctl(hs[i]))) return rc;
  }
  return VF_OK;
}

}  // extern "C"
