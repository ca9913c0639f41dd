// Learned wake proposal: a 32 -> 64 -> 64 -> 1 MLP (ReLU, ReLU, sigmoid) over per-brick
// features, with hand-written fp16 tensor-core forward and backward kernels (mma.sync m16n8k16,
// f16 operands, f32 accumulation), a BCE loss and an Adam step. fp32 master weights; the fp16
// operand copies are refreshed after every step.
//
// The network only proposes which bricks to stage ahead of the exact scheduler; it never decides
// what the fluid computes.
#include <cuda_fp16.h>
#include <cuda_runtime.h>

#include <cmath>
#include <cstdint>
#include <cstring>
#include <vector>

#include "../../include/vf_fluid.h"

namespace vfm {

constexpr int IN = 32, H = 64;
// flat fp32 parameter layout: W1[IN][H] (input-major), b1[H], W2[H][H] (input-major), b2[H],
// w3[H], b3[1]
constexpr int OFF_W1 = 0, OFF_B1 = OFF_W1 + IN * H, OFF_W2 = OFF_B1 + H, OFF_B2 = OFF_W2 + H * H, OFF_W3 = OFF_B2 + H,
              OFF_B3 = OFF_W3 + H, NPARAM = OFF_B3 + 1;
constexpr int WARPS = 4;  // 16-row tiles per CTA = WARPS

struct Dev {
  float* p;       // parameters (fp32 master)
  float* g;       // gradients (fp32)
  float* m;       // Adam first moment
  float* v;       // Adam second moment
  __half* w1t;    // [H][IN]  output-major: B operand of X.W1
  __half* w2t;    // [H][H]   output-major: B operand of H1.W2
  __half* w2n;    // [H][H]   input-major: B operand of dH2.W2^T
  float* loss;    // scratch scalar
};

__device__ __forceinline__ void mma16816(float* c, const unsigned* a, const unsigned* b) {
  asm volatile(
      "mma.sync.aligned.m16n8k16.row.col.f32.f16.f16.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, {%0,%1,%2,%3};\n"
      : "+f"(c[0]), "+f"(c[1]), "+f"(c[2]), "+f"(c[3])
      : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b[0]), "r"(b[1]));
}

__device__ __forceinline__ unsigned pack2(float lo, float hi) {
  __half2 h = __floats2half2_rn(lo, hi);
  return *reinterpret_cast<unsigned*>(&h);
}
__device__ __forceinline__ unsigned ld2(const __half* p) { return *reinterpret_cast<const unsigned*>(p); }

// Per-warp forward of 16 rows. Fragment conventions of m16n8k16: g = lane/4, t = lane%4; an A
// fragment holds (row g | g+8) x (cols 2t,2t+1 | 2t+8,2t+9) of a 16x16 tile; an accumulator tile
// (16x8) holds rows g, g+8 x cols 2t, 2t+1; a B fragment holds k = 2t,2t+1 (+8) of column g.
struct Fwd {
  float h1[8][4];  // relu(X W1 + b1): 8 n-tiles of 8 columns
  float h2[8][4];  // relu(H1 W2 + b2)
  float z[2];      // logits of rows g and g+8
};

__device__ void forward_tile(const Dev& d, const __half* X, int row0, int n, Fwd& f) {
  const int lane = threadIdx.x & 31, g = lane >> 2, t = lane & 3;
  const int r0 = row0 + g, r1 = row0 + g + 8;
  // A fragments of X (16 x 32): two k-steps
  unsigned a[2][4];
#pragma unroll
  for (int kk = 0; kk < 2; ++kk) {
    const int c = kk * 16 + 2 * t;
    a[kk][0] = r0 < n ? ld2(X + (size_t)r0 * IN + c) : 0u;
    a[kk][1] = r1 < n ? ld2(X + (size_t)r1 * IN + c) : 0u;
    a[kk][2] = r0 < n ? ld2(X + (size_t)r0 * IN + c + 8) : 0u;
    a[kk][3] = r1 < n ? ld2(X + (size_t)r1 * IN + c + 8) : 0u;
  }
#pragma unroll
  for (int j = 0; j < 8; ++j) {
    float c[4] = {0.f, 0.f, 0.f, 0.f};
#pragma unroll
    for (int kk = 0; kk < 2; ++kk) {
      unsigned b[2];
      const __half* col = d.w1t + (size_t)(8 * j + g) * IN + kk * 16 + 2 * t;
      b[0] = ld2(col);
      b[1] = ld2(col + 8);
      mma16816(c, a[kk], b);
    }
    const float bb0 = d.p[OFF_B1 + 8 * j + 2 * t], bb1 = d.p[OFF_B1 + 8 * j + 2 * t + 1];
    f.h1[j][0] = fmaxf(c[0] + bb0, 0.f);
    f.h1[j][1] = fmaxf(c[1] + bb1, 0.f);
    f.h1[j][2] = fmaxf(c[2] + bb0, 0.f);
    f.h1[j][3] = fmaxf(c[3] + bb1, 0.f);
  }
  // layer 2: A fragments straight from the layer-1 accumulators (k-step kk = tiles 2kk, 2kk+1)
  unsigned a2[4][4];
#pragma unroll
  for (int kk = 0; kk < 4; ++kk) {
    a2[kk][0] = pack2(f.h1[2 * kk][0], f.h1[2 * kk][1]);
    a2[kk][1] = pack2(f.h1[2 * kk][2], f.h1[2 * kk][3]);
    a2[kk][2] = pack2(f.h1[2 * kk + 1][0], f.h1[2 * kk + 1][1]);
    a2[kk][3] = pack2(f.h1[2 * kk + 1][2], f.h1[2 * kk + 1][3]);
  }
#pragma unroll
  for (int j = 0; j < 8; ++j) {
    float c[4] = {0.f, 0.f, 0.f, 0.f};
#pragma unroll
    for (int kk = 0; kk < 4; ++kk) {
      unsigned b[2];
      const __half* col = d.w2t + (size_t)(8 * j + g) * H + kk * 16 + 2 * t;
      b[0] = ld2(col);
      b[1] = ld2(col + 8);
      mma16816(c, a2[kk], b);
    }
    const float bb0 = d.p[OFF_B2 + 8 * j + 2 * t], bb1 = d.p[OFF_B2 + 8 * j + 2 * t + 1];
    f.h2[j][0] = fmaxf(c[0] + bb0, 0.f);
    f.h2[j][1] = fmaxf(c[1] + bb1, 0.f);
    f.h2[j][2] = fmaxf(c[2] + bb0, 0.f);
    f.h2[j][3] = fmaxf(c[3] + bb1, 0.f);
  }
  // layer 3: 64 -> 1 dot products, reduced over the 4 threads of a row group
  float z0 = 0.f, z1 = 0.f;
#pragma unroll
  for (int j = 0; j < 8; ++j) {
    const float w0 = d.p[OFF_W3 + 8 * j + 2 * t], w1 = d.p[OFF_W3 + 8 * j + 2 * t + 1];
    z0 += f.h2[j][0] * w0 + f.h2[j][1] * w1;
    z1 += f.h2[j][2] * w0 + f.h2[j][3] * w1;
  }
  z0 += __shfl_xor_sync(0xFFFFFFFFu, z0, 1);
  z0 += __shfl_xor_sync(0xFFFFFFFFu, z0, 2);
  z1 += __shfl_xor_sync(0xFFFFFFFFu, z1, 1);
  z1 += __shfl_xor_sync(0xFFFFFFFFu, z1, 2);
  f.z[0] = z0 + d.p[OFF_B3];
  f.z[1] = z1 + d.p[OFF_B3];
}

__device__ __forceinline__ float sigmoidf_(float z) { return 1.0f / (1.0f + expf(-z)); }

__global__ void k_forward(Dev d, const __half* X, int n, float* prob) {
  const int tile = blockIdx.x * WARPS + (threadIdx.x >> 5);
  const int row0 = tile * 16;
  if (row0 >= n) return;
  Fwd f;
  forward_tile(d, X, row0, n, f);
  const int lane = threadIdx.x & 31, g = lane >> 2, t = lane & 3;
  if (t == 0) {
    if (row0 + g < n) prob[row0 + g] = sigmoidf_(f.z[0]);
    if (row0 + g + 8 < n) prob[row0 + g + 8] = sigmoidf_(f.z[1]);
  }
}

// Backward of mean BCE-with-logits; gradients accumulate into d.g (fp32). Each warp: 16 rows.
__global__ void k_backward(Dev d, const __half* X, const float* y, int n, float inv_n) {
  __shared__ __half sh_h1[WARPS][16][H];   // H1 tile (row-major) for dW2
  __shared__ __half sh_d2[WARPS][16][H];   // dZ2 tile for dW2, then dZ1 for dW1
  __shared__ float sg[NPARAM];
  const int w = threadIdx.x >> 5, lane = threadIdx.x & 31, g = lane >> 2, t = lane & 3;
  for (int i = threadIdx.x; i < NPARAM; i += blockDim.x) sg[i] = 0.f;
  __syncthreads();
  const int tile = blockIdx.x * WARPS + w;
  const int row0 = tile * 16;
  if (row0 < n) {
    Fwd f;
    forward_tile(d, X, row0, n, f);
    const int r0 = row0 + g, r1 = row0 + g + 8;
    const float dz0 = r0 < n ? (sigmoidf_(f.z[0]) - y[r0]) * inv_n : 0.f;
    const float dz1 = r1 < n ? (sigmoidf_(f.z[1]) - y[r1]) * inv_n : 0.f;
    if (t == 0) atomicAdd(&sg[OFF_B3], dz0 + dz1);
    // dw3, dZ2 = dz w3 (relu')
    float d2[8][4];
#pragma unroll
    for (int j = 0; j < 8; ++j) {
      const int c0 = 8 * j + 2 * t;
      const float w0 = d.p[OFF_W3 + c0], w1 = d.p[OFF_W3 + c0 + 1];
      float gw0 = f.h2[j][0] * dz0 + f.h2[j][2] * dz1;
      float gw1 = f.h2[j][1] * dz0 + f.h2[j][3] * dz1;
      // sum over the 8 row groups (lanes with equal t)
#pragma unroll
      for (int o = 4; o < 32; o <<= 1) {
        gw0 += __shfl_xor_sync(0xFFFFFFFFu, gw0, o);
        gw1 += __shfl_xor_sync(0xFFFFFFFFu, gw1, o);
      }
      if (g == 0) {
        atomicAdd(&sg[OFF_W3 + c0], gw0);
        atomicAdd(&sg[OFF_W3 + c0 + 1], gw1);
      }
      d2[j][0] = f.h2[j][0] > 0.f ? dz0 * w0 : 0.f;
      d2[j][1] = f.h2[j][1] > 0.f ? dz0 * w1 : 0.f;
      d2[j][2] = f.h2[j][2] > 0.f ? dz1 * w0 : 0.f;
      d2[j][3] = f.h2[j][3] > 0.f ? dz1 * w1 : 0.f;
      // db2
      float s0 = d2[j][0] + d2[j][2], s1 = d2[j][1] + d2[j][3];
#pragma unroll
      for (int o = 4; o < 32; o <<= 1) {
        s0 += __shfl_xor_sync(0xFFFFFFFFu, s0, o);
        s1 += __shfl_xor_sync(0xFFFFFFFFu, s1, o);
      }
      if (g == 0) {
        atomicAdd(&sg[OFF_B2 + c0], s0);
        atomicAdd(&sg[OFF_B2 + c0 + 1], s1);
      }
      sh_h1[w][g][c0] = __float2half_rn(f.h1[j][0]);
      sh_h1[w][g][c0 + 1] = __float2half_rn(f.h1[j][1]);
      sh_h1[w][g + 8][c0] = __float2half_rn(f.h1[j][2]);
      sh_h1[w][g + 8][c0 + 1] = __float2half_rn(f.h1[j][3]);
      sh_d2[w][g][c0] = __float2half_rn(d2[j][0]);
      sh_d2[w][g][c0 + 1] = __float2half_rn(d2[j][1]);
      sh_d2[w][g + 8][c0] = __float2half_rn(d2[j][2]);
      sh_d2[w][g + 8][c0 + 1] = __float2half_rn(d2[j][3]);
    }
    __syncwarp();
    // dW2[i][j] = sum_r H1[r][i] dZ2[r][j]: M = 64 (i), N = 64 (j), K = 16 (r)
#pragma unroll
    for (int mi = 0; mi < 4; ++mi) {
      unsigned a[4];  // A[i][r] = H1[r][i]
      const int i0 = 16 * mi + g;
      auto h = [&](int r, int i) { return sh_h1[w][r][i]; };
      __half2 p;
      p = __halves2half2(h(2 * t, i0), h(2 * t + 1, i0));
      a[0] = *reinterpret_cast<unsigned*>(&p);
      p = __halves2half2(h(2 * t, i0 + 8), h(2 * t + 1, i0 + 8));
      a[1] = *reinterpret_cast<unsigned*>(&p);
      p = __halves2half2(h(2 * t + 8, i0), h(2 * t + 9, i0));
      a[2] = *reinterpret_cast<unsigned*>(&p);
      p = __halves2half2(h(2 * t + 8, i0 + 8), h(2 * t + 9, i0 + 8));
      a[3] = *reinterpret_cast<unsigned*>(&p);
#pragma unroll
      for (int nj = 0; nj < 8; ++nj) {
        unsigned b[2];  // B[r][j] = dZ2[r][j], column j = 8nj + g
        const int jc = 8 * nj + g;
        __half2 q = __halves2half2(sh_d2[w][2 * t][jc], sh_d2[w][2 * t + 1][jc]);
        b[0] = *reinterpret_cast<unsigned*>(&q);
        q = __halves2half2(sh_d2[w][2 * t + 8][jc], sh_d2[w][2 * t + 9][jc]);
        b[1] = *reinterpret_cast<unsigned*>(&q);
        float c[4] = {0.f, 0.f, 0.f, 0.f};
        mma16816(c, a, b);
        const int ci = 16 * mi + g, cj = 8 * nj + 2 * t;
        atomicAdd(&sg[OFF_W2 + ci * H + cj], c[0]);
        atomicAdd(&sg[OFF_W2 + ci * H + cj + 1], c[1]);
        atomicAdd(&sg[OFF_W2 + (ci + 8) * H + cj], c[2]);
        atomicAdd(&sg[OFF_W2 + (ci + 8) * H + cj + 1], c[3]);
      }
    }
    __syncwarp();  // the dZ2 tile is reused for dZ1 below
    // dH1 = dZ2 W2^T (relu'): M = 16, N = 64 (i), K = 64 (j); A from the dZ2 accumulators
    unsigned ad[4][4];
#pragma unroll
    for (int kk = 0; kk < 4; ++kk) {
      ad[kk][0] = pack2(d2[2 * kk][0], d2[2 * kk][1]);
      ad[kk][1] = pack2(d2[2 * kk][2], d2[2 * kk][3]);
      ad[kk][2] = pack2(d2[2 * kk + 1][0], d2[2 * kk + 1][1]);
      ad[kk][3] = pack2(d2[2 * kk + 1][2], d2[2 * kk + 1][3]);
    }
    float d1[8][4];
#pragma unroll
    for (int j = 0; j < 8; ++j) {
      float c[4] = {0.f, 0.f, 0.f, 0.f};
#pragma unroll
      for (int kk = 0; kk < 4; ++kk) {
        unsigned b[2];  // B[k=j'][n=i] = W2[i][j'] (input-major copy), column i = 8j + g
        const __half* col = d.w2n + (size_t)(8 * j + g) * H + kk * 16 + 2 * t;
        b[0] = ld2(col);
        b[1] = ld2(col + 8);
        mma16816(c, ad[kk], b);
      }
      const int c0 = 8 * j + 2 * t;
      d1[j][0] = f.h1[j][0] > 0.f ? c[0] : 0.f;
      d1[j][1] = f.h1[j][1] > 0.f ? c[1] : 0.f;
      d1[j][2] = f.h1[j][2] > 0.f ? c[2] : 0.f;
      d1[j][3] = f.h1[j][3] > 0.f ? c[3] : 0.f;
      float s0 = d1[j][0] + d1[j][2], s1 = d1[j][1] + d1[j][3];
#pragma unroll
      for (int o = 4; o < 32; o <<= 1) {
        s0 += __shfl_xor_sync(0xFFFFFFFFu, s0, o);
        s1 += __shfl_xor_sync(0xFFFFFFFFu, s1, o);
      }
      if (g == 0) {
        atomicAdd(&sg[OFF_B1 + c0], s0);
        atomicAdd(&sg[OFF_B1 + c0 + 1], s1);
      }
      sh_d2[w][g][c0] = __float2half_rn(d1[j][0]);
      sh_d2[w][g][c0 + 1] = __float2half_rn(d1[j][1]);
      sh_d2[w][g + 8][c0] = __float2half_rn(d1[j][2]);
      sh_d2[w][g + 8][c0 + 1] = __float2half_rn(d1[j][3]);
    }
    __syncwarp();
    // dW1[i][j] = sum_r X[r][i] dZ1[r][j]: M = 32 (i), N = 64 (j), K = 16 (r)
#pragma unroll
    for (int mi = 0; mi < 2; ++mi) {
      unsigned a[4];  // A[i][r] = X[r][i]
      const int i0 = 16 * mi + g;
      auto xv = [&](int r, int i) { return (row0 + r < n) ? X[(size_t)(row0 + r) * IN + i] : __float2half_rn(0.f); };
      __half2 p;
      p = __halves2half2(xv(2 * t, i0), xv(2 * t + 1, i0));
      a[0] = *reinterpret_cast<unsigned*>(&p);
      p = __halves2half2(xv(2 * t, i0 + 8), xv(2 * t + 1, i0 + 8));
      a[1] = *reinterpret_cast<unsigned*>(&p);
      p = __halves2half2(xv(2 * t + 8, i0), xv(2 * t + 9, i0));
      a[2] = *reinterpret_cast<unsigned*>(&p);
      p = __halves2half2(xv(2 * t + 8, i0 + 8), xv(2 * t + 9, i0 + 8));
      a[3] = *reinterpret_cast<unsigned*>(&p);
#pragma unroll
      for (int nj = 0; nj < 8; ++nj) {
        unsigned b[2];
        const int jc = 8 * nj + g;
        __half2 q = __halves2half2(sh_d2[w][2 * t][jc], sh_d2[w][2 * t + 1][jc]);
        b[0] = *reinterpret_cast<unsigned*>(&q);
        q = __halves2half2(sh_d2[w][2 * t + 8][jc], sh_d2[w][2 * t + 9][jc]);
        b[1] = *reinterpret_cast<unsigned*>(&q);
        float c[4] = {0.f, 0.f, 0.f, 0.f};
        mma16816(c, a, b);
        const int ci = 16 * mi + g, cj = 8 * nj + 2 * t;
        atomicAdd(&sg[OFF_W1 + ci * H + cj], c[0]);
        atomicAdd(&sg[OFF_W1 + ci * H + cj + 1], c[1]);
        atomicAdd(&sg[OFF_W1 + (ci + 8) * H + cj], c[2]);
        atomicAdd(&sg[OFF_W1 + (ci + 8) * H + cj + 1], c[3]);
      }
    }
  }
  __syncthreads();
  for (int i = threadIdx.x; i < NPARAM; i += blockDim.x)
    if (sg[i] != 0.f) atomicAdd(&d.g[i], sg[i]);
}

// mean BCE-with-logits over n rows (for monitoring)
__global__ void k_loss(Dev d, const __half* X, const float* y, int n, float inv_n) {
  const int tile = blockIdx.x * WARPS + (threadIdx.x >> 5);
  const int row0 = tile * 16;
  if (row0 >= n) return;
  Fwd f;
  forward_tile(d, X, row0, n, f);
  const int lane = threadIdx.x & 31, g = lane >> 2, t = lane & 3;
  float l = 0.f;
  if (t == 0) {
    for (int k = 0; k < 2; ++k) {
      int r = row0 + g + 8 * k;
      if (r < n) {
        float z = f.z[k];
        l += fmaxf(z, 0.f) - z * y[r] + log1pf(expf(-fabsf(z)));
      }
    }
  }
  for (int o = 16; o; o >>= 1) l += __shfl_xor_sync(0xFFFFFFFFu, l, o);
  if (lane == 0) atomicAdd(d.loss, l * inv_n);
}

// Adam on the fp32 master weights, then refresh the fp16 operand copies.
__global__ void k_adam(Dev d, float lr, float b1, float b2, float eps, float c1, float c2) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < NPARAM; i += gridDim.x * blockDim.x) {
    float gi = d.g[i];
    float m = b1 * d.m[i] + (1.f - b1) * gi;
    float v = b2 * d.v[i] + (1.f - b2) * gi * gi;
    d.m[i] = m;
    d.v[i] = v;
    d.p[i] -= lr * (m / c1) / (sqrtf(v / c2) + eps);
    d.g[i] = 0.f;
  }
}

__global__ void k_refresh(Dev d) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < H * H + IN * H; i += gridDim.x * blockDim.x) {
    if (i < IN * H) {  // W1[in][out] -> w1t[out][in]
      int in = i / H, out = i % H;
      d.w1t[out * IN + in] = __float2half_rn(d.p[OFF_W1 + i]);
    } else {
      int k = i - IN * H, in = k / H, out = k % H;
      d.w2t[out * H + in] = __float2half_rn(d.p[OFF_W2 + k]);
      d.w2n[in * H + out] = __float2half_rn(d.p[OFF_W2 + k]);
    }
  }
}

}  // namespace vfm

using namespace vfm;

struct vf_mlp {
  int device = 0;
  Dev d{};
  int step = 0;
  std::vector<void*> allocs;
};

namespace {
template <class T>
bool alloc(vf_mlp* h, T** p, size_t n) {
  if (cudaMalloc((void**)p, sizeof(T) * n) != cudaSuccess) return false;
  h->allocs.push_back(*p);
  cudaMemset(*p, 0, sizeof(T) * n);
  return true;
}
unsigned blocks_for(uint64_t n) { return (unsigned)((n + 16 * WARPS - 1) / (16 * WARPS)); }
}  // namespace

extern "C" {

int vf_mlp_create(int32_t device, uint64_t seed, vf_mlp** out) {
  if (!out) return VF_ERR_INVALID;
  if (cudaSetDevice(device) != cudaSuccess) return VF_ERR_NO_DEVICE;
  auto* h = new vf_mlp();
  h->device = device;
  if (!alloc(h, &h->d.p, NPARAM) || !alloc(h, &h->d.g, NPARAM) || !alloc(h, &h->d.m, NPARAM) || !alloc(h, &h->d.v, NPARAM) ||
      !alloc(h, &h->d.w1t, H * IN) || !alloc(h, &h->d.w2t, H * H) || !alloc(h, &h->d.w2n, H * H) || !alloc(h, &h->d.loss, 1)) {
    for (void* p : h->allocs) cudaFree(p);
    delete h;
    return VF_ERR_OOM;
  }
  // He-uniform init from a splitmix64 stream (host), biases 0
  std::vector<float> p(NPARAM, 0.f);
  uint64_t s = seed * 0x9E3779B97F4A7C15ULL + 1;
  auto rnd = [&]() {
    uint64_t z = (s += 0x9E3779B97F4A7C15ULL);
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ULL;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBULL;
    z ^= z >> 31;
    return (float)((z >> 11) * (1.0 / 9007199254740992.0)) * 2.f - 1.f;
  };
  const float a1 = std::sqrt(6.f / IN), a2 = std::sqrt(6.f / H), a3 = std::sqrt(3.f / H);
  for (int i = 0; i < IN * H; ++i) p[OFF_W1 + i] = a1 * rnd();
  for (int i = 0; i < H * H; ++i) p[OFF_W2 + i] = a2 * rnd();
  for (int i = 0; i < H; ++i) p[OFF_W3 + i] = a3 * rnd();
  cudaMemcpy(h->d.p, p.data(), NPARAM * 4, cudaMemcpyHostToDevice);
  k_refresh<<<32, 256>>>(h->d);
  if (cudaDeviceSynchronize() != cudaSuccess) {
    for (void* q : h->allocs) cudaFree(q);
    delete h;
    return VF_ERR_CUDA;
  }
  *out = h;
  return VF_OK;
}

void vf_mlp_destroy(vf_mlp* h) {
  if (!h) return;
  for (void* p : h->allocs) cudaFree(p);
  delete h;
}

int vf_mlp_nparams(void) { return NPARAM; }

int vf_mlp_get_params(vf_mlp* h, float* out) {
  if (!h || !out) return VF_ERR_INVALID;
  return cudaMemcpy(out, h->d.p, NPARAM * 4, cudaMemcpyDeviceToHost) == cudaSuccess ? VF_OK : VF_ERR_CUDA;
}

int vf_mlp_set_params(vf_mlp* h, const float* in) {
  if (!h || !in) return VF_ERR_INVALID;
  if (cudaMemcpy(h->d.p, in, NPARAM * 4, cudaMemcpyHostToDevice) != cudaSuccess) return VF_ERR_CUDA;
  k_refresh<<<32, 256>>>(h->d);
  return cudaDeviceSynchronize() == cudaSuccess ? VF_OK : VF_ERR_CUDA;
}

// probabilities for n feature rows (x: n x 32 fp16, device), out: n fp32 (device)
int vf_mlp_forward(vf_mlp* h, const void* dev_x, uint64_t n, float* dev_prob, void* stream) {
  if (!h || (!dev_x && n)) return VF_ERR_INVALID;
  if (!n) return VF_OK;
  k_forward<<<blocks_for(n), 32 * WARPS, 0, (cudaStream_t)stream>>>(h->d, (const __half*)dev_x, (int)n, dev_prob);
  return cudaGetLastError() == cudaSuccess ? VF_OK : VF_ERR_CUDA;
}

// gradients of the mean BCE over n rows into the flat fp32 host array grads (NPARAM), no update
int vf_mlp_grads(vf_mlp* h, const void* dev_x, const float* dev_y, uint64_t n, float* grads, void* stream) {
  if (!h || !dev_x || !dev_y || !n || !grads) return VF_ERR_INVALID;
  cudaStream_t st = (cudaStream_t)stream;
  cudaMemsetAsync(h->d.g, 0, NPARAM * 4, st);
  k_backward<<<blocks_for(n), 32 * WARPS, 0, st>>>(h->d, (const __half*)dev_x, dev_y, (int)n, 1.0f / (float)n);
  if (cudaMemcpyAsync(grads, h->d.g, NPARAM * 4, cudaMemcpyDeviceToHost, st) != cudaSuccess) return VF_ERR_CUDA;
  if (cudaStreamSynchronize(st) != cudaSuccess) return VF_ERR_CUDA;
  cudaMemsetAsync(h->d.g, 0, NPARAM * 4, st);
  return cudaStreamSynchronize(st) == cudaSuccess ? VF_OK : VF_ERR_CUDA;
}

// one Adam step on a minibatch (device arrays); *loss (host, optional) = the batch's mean BCE
// before the step
int vf_mlp_train_step(vf_mlp* h, const void* dev_x, const float* dev_y, uint64_t n, float lr, float* loss, void* stream) {
  if (!h || !dev_x || !dev_y || !n) return VF_ERR_INVALID;
  cudaStream_t st = (cudaStream_t)stream;
  if (loss) {
    cudaMemsetAsync(h->d.loss, 0, 4, st);
    k_loss<<<blocks_for(n), 32 * WARPS, 0, st>>>(h->d, (const __half*)dev_x, dev_y, (int)n, 1.0f / (float)n);
  }
  k_backward<<<blocks_for(n), 32 * WARPS, 0, st>>>(h->d, (const __half*)dev_x, dev_y, (int)n, 1.0f / (float)n);
  h->step += 1;
  const float b1 = 0.9f, b2 = 0.999f;
  const float c1 = 1.f - std::pow(b1, (float)h->step), c2 = 1.f - std::pow(b2, (float)h->step);
  k_adam<<<(NPARAM + 255) / 256, 256, 0, st>>>(h->d, lr, b1, b2, 1e-8f, c1, c2);
  k_refresh<<<32, 256, 0, st>>>(h->d);
  if (loss) {
    if (cudaMemcpyAsync(loss, h->d.loss, 4, cudaMemcpyDeviceToHost, st) != cudaSuccess) return VF_ERR_CUDA;
    if (cudaStreamSynchronize(st) != cudaSuccess) return VF_ERR_CUDA;
  }
  return cudaGetLastError() == cudaSuccess ? VF_OK : VF_ERR_CUDA;
}

}  // extern "C"
