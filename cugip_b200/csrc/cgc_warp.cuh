// Warp-per-tile routines: the seeding passes over all tiles
// (bfs_init_tile_w, reach_init_tile_w), which need no block barrier, so a CTA
// seeds 16 tiles at a time, and the warp-per-tile BFS visit (bfs_tile_w) used
// by rounds with many tiles per CTA (SolveParams::bfs_warp_min).
//
// One warp owns one 8x8x8 tile: lane l owns the 16 voxels l + 32k
// (k = 0..15), i.e. x = l&7, y = ((l>>3)&3) + 4(k&1), z = k>>1.  The BFS
// visit keeps the tile's heights (with the one-voxel halo) and residual masks
// in the warp's 4.6 KB slice of shared memory and relaxes in place
// (Gauss-Seidel), which converges to the same fixed point as the 512-thread
// visit in fewer steps, with __syncwarp instead of block barriers.
#pragma once
#include "cgc_kernels.cuh"

namespace cgc {

constexpr unsigned FULL = 0xffffffffu;

struct WarpBfsSmem {
  int h[HALO];
  unsigned char m[TV];
};

__device__ __forceinline__ int wv_index(int lane, int k) { return lane + 32 * k; }
__device__ __forceinline__ int wv_x(int lane) { return lane & 7; }
__device__ __forceinline__ int wv_y(int lane, int k) { return ((lane >> 3) & 3) | ((k & 1) << 2); }
__device__ __forceinline__ int wv_z(int k) { return k >> 1; }


// halo heights of tile t into sh (INF outside the grid): 384 entries, 12 per lane
__device__ __forceinline__ void warp_load_halo_heights(const DevPool& P, int t, int* sh, int lane) {
#pragma unroll 4
  for (int m = 0; m < 12; ++m) {
    for_halo_entry(lane + 32 * m, [&](int f, int hi, int src) {
      const int nt = __ldcg(P.nbr + f * P.T + t);
      sh[hi] = (nt >= 0 && CGC_IN_BOUNDS(P, nt, P.T)) ? __ldcg(P.h + (int64_t)nt * TV + src) : INF;
    });
  }
}

// ---------------------------------------------------------------------------
// BFS seed for tile t: h = 1 where the sink residual is positive, INF
// elsewhere; the tile's seed summary (face bits, any seed, all seeds) goes to
// tflag for the second seeding step (bfs_seed_tile / bfs_queue_tile).
// A tile whose voxels were all found unable to reach the sink stays so (dead
// vertices neither receive nor send flow, and all their residual neighbours
// are dead), so it keeps INF and is never visited again; heights are 0 before
// the first relabel of a solve.  A tile whose voxels are all seeds is final
// at h = 1 and is never visited.
__device__ inline void bfs_init_tile_w(const DevPool& P, const int t) {
  if (!CGC_IN_BOUNDS(P, t, P.T)) return;  // uniform over the warp
  const int lane = threadIdx.x & 31;
  const int64_t base = (int64_t)t * TV;
  bool dead = true, all_seed = true, any_excess = false;
  unsigned flags = 0;
  unsigned rms[16];
#pragma unroll
  for (int k = 0; k < 16; ++k) {
    const int i = wv_index(lane, k);
    rms[k] = __ldcg(P.rmask + base + i);
    dead = dead && __ldcg(P.h + base + i) == INF;
  }
  // a tile whose voxels were all found unable to reach the sink stays so
  dead = __all_sync(FULL, dead);
  if (dead) {
    if (lane == 0) { P.tflag[t] = TF_DEAD; P.act[t] = 0; }
    return;
  }
#pragma unroll
  for (int k = 0; k < 16; ++k) {
    const int i = wv_index(lane, k);
    const bool seed = (rms[k] & 64u) != 0;
    P.h[base + i] = seed ? 1 : INF;
    if (seed) flags |= (face_bits(wv_x(lane), wv_y(lane, k), wv_z(k)) << 1) | TF_HAS_SEED;
    all_seed = all_seed && seed;
    any_excess = any_excess || (rms[k] & 128u) != 0;
  }
  flags = __reduce_or_sync(FULL, flags);
  all_seed = __all_sync(FULL, all_seed);
  any_excess = __any_sync(FULL, any_excess);
  if (lane == 0) {
    P.tflag[t] = (uint16_t)(flags | (all_seed ? TF_ALL_SEED : 0));
    P.act[t] = (uint8_t)((all_seed && any_excess) ? 1 : 0);
  }
}

__device__ inline void bfs_tile_w(const DevPool& P, const int t, WarpBfsSmem& S, const uint32_t id_next,
                                  int32_t* list_next, int32_t* cnt_next) {
  if (!CGC_IN_BOUNDS(P, t, P.T)) return;      // uniform over the warp
  if (__ldcg(P.tflag + t) & TF_DEAD) return;  // uniform over the warp
  const int lane = threadIdx.x & 31;
  const int64_t base = (int64_t)t * TV;
  const int x = wv_x(lane);
  int h0[16];
#pragma unroll
  for (int k = 0; k < 16; ++k) {
    const int i = wv_index(lane, k);
    h0[k] = __ldcg(P.h + base + i);
    S.m[i] = __ldcg(P.rmask + base + i);
    S.h[halo_index(x, wv_y(lane, k), wv_z(k))] = h0[k];
  }
  warp_load_halo_heights(P, t, S.h, lane);
  __syncwarp();
  for (int it = 0; it < 1200; ++it) {
    bool ch = false;
#pragma unroll
    for (int k = 0; k < 16; ++k) {
      const int i = wv_index(lane, k);
      const int hi = halo_index(x, wv_y(lane, k), wv_z(k));
      const unsigned m = S.m[i];
      const int cur = S.h[hi];
      int mn = cur;
#pragma unroll
      for (int d = 0; d < 6; ++d)
        if ((m >> d) & 1u) mn = min(mn, S.h[hi + hoff(d)] + 1);
      if (mn < cur) { S.h[hi] = mn; ch = true; }
    }
    __syncwarp();
    if (!__any_sync(FULL, ch)) break;
  }
  unsigned faces = 0;
  bool act = false;
#pragma unroll
  for (int k = 0; k < 16; ++k) {
    const int i = wv_index(lane, k);
    const int y = wv_y(lane, k), z = wv_z(k);
    const int h = S.h[halo_index(x, y, z)];
    if (h < h0[k]) {
      P.h[base + i] = h;
      faces |= face_bits(x, y, z);
    }
    act = act || ((S.m[i] & 128u) && h < INF);
  }
  faces = __reduce_or_sync(FULL, faces);
  act = __any_sync(FULL, act);
  if (lane == 0) {
    P.act[t] = (uint8_t)(act ? 1 : 0);  // heights only drop in later visits: the last visit's value is final
    atomicAdd(P.stats + S_TILES_BFS, 1ull);
  }
  if (lane < 6 && ((faces >> lane) & 1)) {
    const int nt = __ldcg(P.nbr + lane * P.T + t);
    if (nt >= 0) queue_tile(P, P.stamp_bfs, nt, id_next, list_next, cnt_next);
  }
  __syncwarp();
}

// ---------------------------------------------------------------------------
// Reachability seed for tile t: the voxels holding excess; the tile is queued
// if it has one, and so is every face neighbour next to one.
__device__ inline void reach_init_tile_w(const DevPool& P, const int t, const uint32_t id0, int32_t* list0,
                                         int32_t* cnt0) {
  if (!CGC_IN_BOUNDS(P, t, P.T)) return;  // uniform over the warp
  const int lane = threadIdx.x & 31;
  const int64_t base = (int64_t)t * TV;
  // A seed only spreads along its residual edges: the tile needs a visit if
  // some seed has one inside the tile (bit 6), and the neighbour across face
  // f if a seed on that face has one through it (bit f; that neighbour's
  // visit reads the seed and the edge from its halo).  A seed without
  // residual edges -- in a maximum flow, typically an isolated excess voxel
  // whose out-edges are saturated -- is its own closure.
  unsigned flags = 0;
#pragma unroll
  for (int k = 0; k < 16; ++k) {
    const int i = wv_index(lane, k);
    const unsigned m = __ldcg(P.rmask + base + i);
    const bool seed = (m & 128u) != 0;
    P.reach[base + i] = seed ? 1 : 0;
    if (seed) {
      const unsigned fb = (unsigned)face_bits(wv_x(lane), wv_y(lane, k), wv_z(k));
      flags |= (m & fb & 63u) | ((m & ~fb & 63u) ? 64u : 0u);
    }
  }
  flags = __reduce_or_sync(FULL, flags);
  if (lane == 0 && (flags & 64u)) queue_tile(P, P.stamp_bfs, t, id0, list0, cnt0);
  if (lane < 6 && ((flags >> lane) & 1)) {
    const int nt = __ldcg(P.nbr + lane * P.T + t);
    if (nt >= 0) queue_tile(P, P.stamp_bfs, nt, id0, list0, cnt0);
  }
}

}  // namespace cgc
