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
// Numerics: BF16 weights and activations, FP32 accumulation, on the tensor
// cores (mma.sync m16n8k16).  The convolutions have no bias, so an all-zero
// neighbourhood gives an exact zero: taps whose rows are all zero are skipped,
// and the cost follows the active region.
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
  float pool[16];  // cadence: sum of the last layer's outputs over this CTA's active tiles
  int count;       // and the number of those tiles
};

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

// Features of active tile t by one warp (16 coalesced passes over its voxels)
// into out[t] and, if given, into trace row out2.
__device__ inline void sched_features_warp(const DevPool& P, const int t, __nv_bfloat16* out,
                                           __nv_bfloat16* out2 = nullptr) {
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
    if (out2) out2[lane] = __float2bfloat16(v);
  }
}

// ---------------------------------------------------------------------------
// Convolutions on the tensor cores.  One warp computes a 3x3x3 convolution
// (16 -> 16 channels) of 16 consecutive tiles as 27 K-steps of
// mma.sync.m16n8k16 (BF16 A and B, FP32 accumulation): per tap, the rows of A
// are the 16 tiles' neighbours at that tap (16 input channels = K), B is the
// tap's 16x16 weight matrix, split into two halves of 8 output channels (N).
// Fragment layout of m16n8k16 (g = lane / 4, q = lane % 4): A registers
// {row g, cols 2q..2q+1}, {row g+8, cols 2q..}, {row g, cols 2q+8..},
// {row g+8, cols 2q+8..}; B registers {k = 2q..2q+1, n = g}, {k = 2q+8.., n = g};
// C/D {row g, cols 2q, 2q+1}, {row g+8, cols 2q, 2q+1}.  A channel pair
// 2q..2q+1 of a tile is one 32-bit word of its BF16 row, so every A register
// is one load.  The weights are stored in fragment order (SchedFrag) so a warp
// reads a tap's B fragments as one coalesced 256-byte line per half.

// B fragments of one layer: [tap][half][lane] -> {reg 0, reg 1}
constexpr int SCHED_FRAG = SCHED_TAPS * 2 * 32;  // uint2 per layer

__device__ __forceinline__ void mma_bf16_16816(float (&d)[4], uint32_t a0, uint32_t a1, uint32_t a2, uint32_t a3,
                                               uint32_t b0, uint32_t b1) {
  asm volatile(
      "mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, "
      "{%0,%1,%2,%3};\n"
      : "+f"(d[0]), "+f"(d[1]), "+f"(d[2]), "+f"(d[3])
      : "r"(a0), "r"(a1), "r"(a2), "r"(a3), "r"(b0), "r"(b1));
}

__device__ __forceinline__ uint32_t pack_bf16x2(float lo, float hi) {
  const __nv_bfloat162 v = __floats2bfloat162_rn(lo, hi);
  return *reinterpret_cast<const uint32_t*>(&v);
}

// acc[h][0..1]: row g, channels 8h + 2q, +1; acc[h][2..3]: row g + 8.  `tap(row, k)`
// gives the neighbour tile of row 0..15 at tap k (-1: none, a zero row); `in`
// holds 8 words (16 BF16 channels) per tile.  The loop has no warp vote, so
// the loads of consecutive taps are in flight together.
template <typename Tap>
__device__ __forceinline__ void conv_rows16(const uint32_t* __restrict__ in, const uint2* __restrict__ wf, Tap&& tap,
                                            float (&acc)[2][4]) {
  const int lane = threadIdx.x & 31, g = lane >> 2, q = lane & 3;
#pragma unroll
  for (int h = 0; h < 2; ++h)
#pragma unroll
    for (int i = 0; i < 4; ++i) acc[h][i] = 0.f;
#pragma unroll 3
  for (int k = 0; k < SCHED_TAPS; ++k) {
    const int na = tap(g, k), nb = tap(g + 8, k);
    const uint32_t a0 = na >= 0 ? __ldcg(in + (int64_t)na * 8 + q) : 0u;
    const uint32_t a1 = nb >= 0 ? __ldcg(in + (int64_t)nb * 8 + q) : 0u;
    const uint32_t a2 = na >= 0 ? __ldcg(in + (int64_t)na * 8 + 4 + q) : 0u;
    const uint32_t a3 = nb >= 0 ? __ldcg(in + (int64_t)nb * 8 + 4 + q) : 0u;
    const uint2 w0 = __ldg(wf + (k * 2) * 32 + lane), w1 = __ldg(wf + (k * 2 + 1) * 32 + lane);
    mma_bf16_16816(acc[0], a0, a1, a2, a3, w0.x, w0.y);
    mma_bf16_16816(acc[1], a0, a1, a2, a3, w1.x, w1.y);
  }
}

// Tile spaces the layers run over: the tiles of a solver pool (instances of
// any extents) and stacks of D^3 grids (training and the standalone
// inference).  coord(t) caches what tap(coord, k) needs.
struct PoolSpace {
  const DevPool* P;
  __device__ int count() const { return P->T; }
  __device__ TileCoord coord(int t) const { return tile_coord(*P, t); }
  __device__ int tap(const TileCoord& c, int k) const { return tap_tile(c, k); }
};
struct GridCoord {
  int base, x, y, z;
};
struct GridSpace {
  int grids, D;
  __device__ int count() const { return grids * D * D * D; }
  __device__ GridCoord coord(int t) const {
    const int D3 = D * D * D, r = t % D3;
    return {t - r, r % D, (r / D) % D, r / (D * D)};
  }
  __device__ int tap(const GridCoord& c, int k) const {
    const int x = c.x + k % 3 - 1, y = c.y + (k / 3) % 3 - 1, z = c.z + k / 9 - 1;
    if (x < 0 || y < 0 || z < 0 || x >= D || y >= D || z >= D) return -1;
    return c.base + x + D * (y + D * z);
  }
};

// Buffers of one layer: BF16 rows of 16 channels as 8 words per tile.
struct SchedIO {
  const uint32_t* in;
  uint32_t* out;         // layers 0 and 1
  const uint2* wf;       // this layer's B fragments
  const float* wh;       // head (layer 2)
  uint8_t* budget;       // layer 2: pulse budget per tile
  uint8_t* prio;         // layer 2: priority per tile
  const uint8_t* act;    // layer 2 with a cadence pool: active tiles
  float* logits;         // layer 2, optional: the head's two logits per tile
};

// Budget (1..32) and priority of a tile from the head's two logits.
__device__ __forceinline__ void sched_emit(const SchedIO& io, int t, float p0, float p1) {
  p0 += io.wh[2 * SCHED_C];
  p1 += io.wh[2 * SCHED_C + 1];
  if (io.logits) {
    io.logits[2 * (int64_t)t] = p0;
    io.logits[2 * (int64_t)t + 1] = p1;
  }
  const float s = 1.0f / (1.0f + __expf(-p1));
  int b = 1 + (int)(31.0f * s + 0.5f);
  b = b < 1 ? 1 : (b > 32 ? 32 : b);
  io.budget[t] = (uint8_t)b;
  io.prio[t] = p0 >= 0.f ? 1 : 0;
}

// Layer `layer` (0..2) of the CNN over every tile of the space, 16 tiles per
// warp step.  Layers 0 and 1 store their ReLU'd BF16 outputs; layer 2 applies
// the head (budget and priority of every tile) and, with `pool`, adds the
// BF16 outputs of the active tiles to the CTA's cadence pool.
template <typename Space>
__device__ inline void sched_layer(const Space& sp, int layer, const SchedIO& io, int warp_global, int nwarps,
                                   SchedShared* pool) {
  const int lane = threadIdx.x & 31, g = lane >> 2, q = lane & 3;
  const int T = sp.count();
  const int nchunks = (T + 15) >> 4;
  for (int c = warp_global; c < nchunks; c += nwarps) {
    const int t0 = c << 4;
    const int ta = t0 + g, tb = t0 + g + 8;
    const bool va = ta < T, vb = tb < T;
    const auto ca = sp.coord(va ? ta : 0), cb = sp.coord(vb ? tb : 0);
    float acc[2][4];
    conv_rows16(io.in, io.wf, [&](int row, int k) {
      return row < 8 ? (va ? sp.tap(ca, k) : -1) : (vb ? sp.tap(cb, k) : -1);
    }, acc);
    float o[2][4];
#pragma unroll
    for (int h = 0; h < 2; ++h)
#pragma unroll
      for (int i = 0; i < 4; ++i) o[h][i] = __bfloat162float(__float2bfloat16(fmaxf(acc[h][i], 0.f)));
    if (layer < 2) {
#pragma unroll
      for (int h = 0; h < 2; ++h) {
        if (va) io.out[(int64_t)ta * 8 + 4 * h + q] = pack_bf16x2(o[h][0], o[h][1]);
        if (vb) io.out[(int64_t)tb * 8 + 4 * h + q] = pack_bf16x2(o[h][2], o[h][3]);
      }
      continue;
    }
    // head: this lane holds channels 2q, 2q+1, 8+2q, 9+2q of rows ta and tb;
    // the quad (lanes 4g..4g+3) holds all 16
    const float* wh = io.wh;
    const int c0 = 2 * q, c1 = 2 * q + 1, c2 = 8 + 2 * q, c3 = 9 + 2 * q;
    float pa0 = o[0][0] * wh[c0] + o[0][1] * wh[c1] + o[1][0] * wh[c2] + o[1][1] * wh[c3];
    float pa1 = o[0][0] * wh[SCHED_C + c0] + o[0][1] * wh[SCHED_C + c1] + o[1][0] * wh[SCHED_C + c2] +
                o[1][1] * wh[SCHED_C + c3];
    float pb0 = o[0][2] * wh[c0] + o[0][3] * wh[c1] + o[1][2] * wh[c2] + o[1][3] * wh[c3];
    float pb1 = o[0][2] * wh[SCHED_C + c0] + o[0][3] * wh[SCHED_C + c1] + o[1][2] * wh[SCHED_C + c2] +
                o[1][3] * wh[SCHED_C + c3];
#pragma unroll
    for (int m = 1; m <= 2; m <<= 1) {
      pa0 += __shfl_xor_sync(0xffffffffu, pa0, m);
      pa1 += __shfl_xor_sync(0xffffffffu, pa1, m);
      pb0 += __shfl_xor_sync(0xffffffffu, pb0, m);
      pb1 += __shfl_xor_sync(0xffffffffu, pb1, m);
    }
    if (q == 0) {
      if (va) sched_emit(io, ta, pa0, pa1);
      if (vb) sched_emit(io, tb, pb0, pb1);
    }
    if (pool) {
      // channel sums over the chunk's active rows: reduce over g (lanes q, q+4, ...)
      const bool aa = va && __ldcg(io.act + ta), ab = vb && __ldcg(io.act + tb);
      float s4[4];
#pragma unroll
      for (int i = 0; i < 2; ++i) {
        s4[i] = (aa ? o[0][i] : 0.f) + (ab ? o[0][2 + i] : 0.f);
        s4[2 + i] = (aa ? o[1][i] : 0.f) + (ab ? o[1][2 + i] : 0.f);
      }
#pragma unroll
      for (int m = 4; m <= 16; m <<= 1)
#pragma unroll
        for (int i = 0; i < 4; ++i) s4[i] += __shfl_xor_sync(0xffffffffu, s4[i], m);
      const int n = __popc(__ballot_sync(0xffffffffu, q == 0 && aa)) + __popc(__ballot_sync(0xffffffffu, q == 0 && ab));
      if (g == 0) {
        atomicAdd(&pool->pool[c0], s4[0]);
        atomicAdd(&pool->pool[c1], s4[1]);
        atomicAdd(&pool->pool[c2], s4[2]);
        atomicAdd(&pool->pool[c3], s4[3]);
      }
      if (lane == 0 && n) atomicAdd(&pool->count, n);
    }
  }
}

// The layer's buffers in a solver pool.
__device__ __forceinline__ SchedIO pool_io(const DevPool& P, int layer) {
  SchedIO io;
  io.in = reinterpret_cast<const uint32_t*>(layer == 0 ? P.sfeat : (layer == 1 ? P.sact0 : P.sact1));
  io.out = reinterpret_cast<uint32_t*>(layer == 0 ? P.sact0 : P.sact1);
  io.wf = P.swfrag + (int64_t)layer * SCHED_FRAG;
  io.wh = P.swhead;
  io.budget = P.sbudget;
  io.prio = P.sprio;
  io.act = P.act;
  io.logits = nullptr;
  return io;
}

}  // namespace cgc
