// Learned tile scheduler: per-tile features and in-kernel CNN inference.
//
// After every exact global relabel the persistent solve summarises each
// active tile in 10 features (log2 of the excess sum, active voxel count and
// an 8-bin height histogram; inactive tiles are all zero), runs a small CNN
// over the tile grid (three bias-free 3x3x3 convolutions with 16 channels and
// ReLU, then a linear head) and stores, per tile, a priority logit and a
// pulse budget in [1, 32].  The sweeps then give each tile its own budget
// instead of the fixed pulse count and defer low-priority tiles during the
// first half of the relabel cycle.  Neither changes which pushes and relabels
// are valid, only their order, so the flow and the cut sets are those of the
// plain schedule.
//
// Numerics: BF16 weights and activations, FP32 accumulation.  Because the
// convolutions have no bias, an all-zero neighbourhood gives an exact zero:
// only the active tiles dilated by 3, 2 and 1 tiles need features, conv 1 and
// conv 2 outputs, and conv 3 + head outputs respectively (DevPool::smask), so
// the cost follows the active region, not the grid.
#pragma once
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include "cgc_device.cuh"

namespace cgc {

constexpr int SCHED_C = 16;                        // channels (features padded to 16)
constexpr int SCHED_NF = 10;                       // real input features
constexpr int SCHED_TAPS = 27;                     // 3x3x3
constexpr int SCHED_WCONV = SCHED_TAPS * SCHED_C * SCHED_C;  // per layer, [tap][cin][cout]
constexpr int SCHED_NHEAD = 2 * SCHED_C + 2;      // head weights [2][16] + bias [2] (fp32)

// height histogram bin of a voxel: 1, 2, 3-4, 5-8, 9-16, 17-32, 33+, INF
__device__ __forceinline__ int height_bin(int h) {
  if (h >= INF) return 7;
  if (h <= 1) return 0;
  if (h == 2) return 1;
  if (h <= 4) return 2;
  if (h <= 8) return 3;
  if (h <= 16) return 4;
  if (h <= 32) return 5;
  return 6;
}

struct SchedShared {
  int unused;
};

// region masks of DevPool::smask (bit k = needed by layer stage k)
enum SchedMask { SM_ACTIVE = 1, SM_L3 = 2, SM_L2 = 4, SM_L1 = 8, SM_FEAT = 16 };

struct TileCoord {
  int base, TX, TY, TZ, tx, ty, tz;
};

__device__ __forceinline__ TileCoord tile_coord(const DevPool& P, int t) {
  const InstGeo G = P.geo[P.tinst[t]];
  const int lt = t - G.tile_base;
  return {G.tile_base, G.TX, G.TY, G.TZ, lt % G.TX, (lt / G.TX) % G.TY, lt / (G.TX * G.TY)};
}

// neighbour at tap k (offset (k%3-1, k/3%3-1, k/9-1)) inside the instance, or -1
__device__ __forceinline__ int tap_tile(const TileCoord& c, int k) {
  const int x = c.tx + k % 3 - 1, y = c.ty + (k / 3) % 3 - 1, z = c.tz + k / 9 - 1;
  if (x < 0 || y < 0 || z < 0 || x >= c.TX || y >= c.TY || z >= c.TZ) return -1;
  return c.base + x + c.TX * (y + c.TY * z);
}

// Features of active tile t by one warp (16 coalesced passes over its voxels).
__device__ inline void sched_features_warp(const DevPool& P, const int t, __nv_bfloat16* out) {
  const int lane = threadIdx.x & 31;
  unsigned long long ex = 0;
  int act = 0, bins[8] = {0, 0, 0, 0, 0, 0, 0, 0};
  for (int i = lane; i < TV; i += 32) {
    const int64_t g = (int64_t)t * TV + i;
    const int e = __ldcg(P.e + g), h = __ldcg(P.h + g);
    if (e > 0 && h < INF) { ++act; ex += (unsigned long long)e; }
    const int b = height_bin(h);
#pragma unroll
    for (int k = 0; k < 8; ++k) bins[k] += (b == k);
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) ex += __shfl_down_sync(0xffffffffu, ex, o);
  act = __reduce_add_sync(0xffffffffu, act);
#pragma unroll
  for (int k = 0; k < 8; ++k) bins[k] = __reduce_add_sync(0xffffffffu, bins[k]);
  const float ex0 = __shfl_sync(0xffffffffu, log2f(1.0f + (float)ex) * (1.0f / 24.0f), 0);
  if (lane < SCHED_C) {
    float v = 0.f;
    if (lane == 0) v = ex0;
    else if (lane == 1) v = (float)act * (1.0f / 512.0f);
    else if (lane < SCHED_NF) {
#pragma unroll
      for (int k = 0; k < 8; ++k)
        if (lane == 2 + k) v = (float)bins[k] * (1.0f / 512.0f);
    }
    out[(int64_t)t * SCHED_C + lane] = __float2bfloat16(v);
  }
}

// One dilation step of the region mask: bit `to` is set where a neighbour
// (3x3x3) has bit `from`.  Thread per tile.
__device__ __forceinline__ void sched_dilate(const DevPool& P, int t, unsigned from, unsigned to) {
  if (t >= P.T) return;
  const TileCoord c = tile_coord(P, t);
  bool hit = false;
  for (int k = 0; k < SCHED_TAPS && !hit; ++k) {
    const int n = tap_tile(c, k);
    if (n >= 0 && (__ldcg(P.smask + n) & from)) hit = true;
  }
  if (hit) atomicOr(reinterpret_cast<unsigned*>(P.smask + (t & ~3)), to << (8 * (t & 3)));
}

// One 3x3x3 convolution output of tile t by one warp: lane co = lane & 15
// accumulates output channel co over half of the 27 taps; the halves are
// summed with a shuffle.  Returns the ReLU'd value in every lane (channel
// lane & 15).
__device__ __forceinline__ float sched_conv_tile(const DevPool& P, int t, const __nv_bfloat16* in,
                                                 const __nv_bfloat16* __restrict__ W) {
  const int lane = threadIdx.x & 31;
  const int co = lane & 15, half = lane >> 4;
  const TileCoord c = tile_coord(P, t);
  float acc = 0.f;
  const int k0 = half ? 14 : 0, k1 = half ? SCHED_TAPS : 14;
  for (int k = k0; k < k1; ++k) {
    const int n = tap_tile(c, k);
    if (n < 0) continue;
    const uint4* src = reinterpret_cast<const uint4*>(in + (int64_t)n * SCHED_C);
    const uint4 a = __ldcg(src), b = __ldcg(src + 1);
    if ((a.x | a.y | a.z | a.w | b.x | b.y | b.z | b.w) == 0u) continue;  // exact zero contribution
    const __nv_bfloat16* v0 = reinterpret_cast<const __nv_bfloat16*>(&a);
    const __nv_bfloat16* v1 = reinterpret_cast<const __nv_bfloat16*>(&b);
    const __nv_bfloat16* w = W + (k * SCHED_C) * SCHED_C + co;
#pragma unroll
    for (int ci = 0; ci < 8; ++ci) acc = fmaf(__bfloat162float(v0[ci]), __bfloat162float(w[ci * SCHED_C]), acc);
#pragma unroll
    for (int ci = 0; ci < 8; ++ci) acc = fmaf(__bfloat162float(v1[ci]), __bfloat162float(w[(8 + ci) * SCHED_C]), acc);
  }
  acc += __shfl_xor_sync(0xffffffffu, acc, 16);
  return fmaxf(acc, 0.f);
}

// Layer `layer` of the CNN for the tiles of its region (warp-strided over all
// tiles, skipping tiles outside the region).  Layers 0 and 1 write
// activations; layer 2 applies the head and writes budget and priority.
__device__ inline void sched_layer(const DevPool& P, int layer, int warp_global, int nwarps) {
  const __nv_bfloat16* in = layer == 0 ? P.sfeat : (layer == 1 ? P.sact0 : P.sact1);
  __nv_bfloat16* out = layer == 0 ? P.sact0 : P.sact1;
  const __nv_bfloat16* W = P.swconv + (int64_t)layer * SCHED_WCONV;
  const unsigned need = layer == 0 ? SM_L1 : (layer == 1 ? SM_L2 : SM_L3);
  const int lane = threadIdx.x & 31;
  for (int t = warp_global; t < P.T; t += nwarps) {
    if (!(__ldcg(P.smask + t) & need)) continue;
    const float v = sched_conv_tile(P, t, in, W);
    if (layer < 2) {
      if (lane < SCHED_C) out[(int64_t)t * SCHED_C + lane] = __float2bfloat16(v);
    } else {
      // the head reads the conv3 output rounded to BF16 like the stored layers
      const float vb = __bfloat162float(__float2bfloat16(v));
      float p0 = (lane < SCHED_C) ? vb * P.swhead[lane] : 0.f;
      float p1 = (lane < SCHED_C) ? vb * P.swhead[SCHED_C + lane] : 0.f;
#pragma unroll
      for (int o = 8; o > 0; o >>= 1) {
        p0 += __shfl_down_sync(0xffffffffu, p0, o);
        p1 += __shfl_down_sync(0xffffffffu, p1, o);
      }
      if (lane == 0) {
        p0 += P.swhead[2 * SCHED_C];
        p1 += P.swhead[2 * SCHED_C + 1];
        const float s = 1.0f / (1.0f + __expf(-p1));
        int b = 1 + (int)(31.0f * s + 0.5f);
        b = b < 1 ? 1 : (b > 32 ? 32 : b);
        P.sbudget[t] = (uint8_t)b;
        P.sprio[t] = p0 >= 0.f ? 1 : 0;
      }
    }
  }
}

}  // namespace cgc
