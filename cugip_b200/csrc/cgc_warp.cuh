// Warp-per-tile variants of the tile routines.  The seeding passes over all
// tiles (bfs_init_tile_w, reach_init_tile_w) are also what the 512-thread
// kernels use: a warp per tile needs no block barrier, so a CTA seeds 16
// tiles at a time.
//
// One warp owns one 8x8x8 tile: lane l owns the 16 voxels l + 32k
// (k = 0..15), i.e. x = l&7, y = ((l>>3)&3) + 4(k&1), z = k>>1.  The tile's
// excess, sink residual, out-residuals and heights (with the one-voxel halo)
// live in the warp's 20 KB slice of shared memory, so every step needs only
// __syncwarp instead of a 16-warp block barrier, and an SM holds about ten
// tiles at a time instead of three.
//
// Push step: labels are fixed while pushes run, so two voxels never push to
// each other; a push adds to the receiver's excess with a shared-memory atomic
// and to its reverse residual with a plain add (single writer), and a voxel
// subtracts what it pushed with an atomic at the end, so excess that arrives
// during the step can be pushed on (a valid push of available excess).
// Relabel step: a voxel with excess and no admissible edge takes
// 1 + min over its residual neighbours; neighbours relabel concurrently, but
// labels only grow, so reading an old or a new neighbour label both keep the
// labelling valid.  Bellman-Ford steps (region relabel, BFS, reachability)
// update in place (Gauss-Seidel), which converges to the same fixed point in
// fewer steps.
#pragma once
#include "cgc_kernels.cuh"

namespace cgc {

constexpr unsigned FULL = 0xffffffffu;

struct WarpSweepSmem {
  int h[HALO];
  int e[TV];
  int rT[TV];
  int r[6][TV];
  int acc[6][64];  // flow pushed out of the tile per face entry (halo order of for_halo_entry)
};
struct WarpBfsSmem {
  int h[HALO];
  unsigned char m[TV];
};
struct WarpReachSmem {
  unsigned char rc[HALO];
  unsigned char m[HALO];
};
union WarpSmem {
  WarpSweepSmem sw;
  WarpBfsSmem bfs;
  WarpReachSmem rc;
};
constexpr size_t kWarpSmemBytes = sizeof(WarpSmem) * WARP_CTA_WARPS;
static_assert(kWarpSmemBytes <= 227 * 1024, "warp-per-tile CTA exceeds the shared memory of an SM");

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
      sh[hi] = (nt >= 0) ? __ldcg(P.h + (int64_t)nt * TV + src) : INF;
    });
  }
}

// ---------------------------------------------------------------------------
template <bool APPEND>
__device__ inline void sweep_tile_w(const DevPool& P, const int t, const int L, const int R, WarpSweepSmem& S,
                                    const uint32_t id_next, int32_t* list_next, int32_t* cnt_next,
                                    const uint32_t id_self, int32_t* list_self, int32_t* cnt_self,
                                    const SweepExtra ex) {
  const int lane = threadIdx.x & 31;
  const int64_t base = (int64_t)t * TV;
  const int64_t Np = P.Np;
  const int x = wv_x(lane);
  int hv[16];
#pragma unroll
  for (int k = 0; k < 16; ++k) {
    const int i = wv_index(lane, k);
    const int64_t g = base + i;
    S.e[i] = __ldcg(P.e + g);
    S.rT[i] = __ldcg(P.rT + g);
#pragma unroll
    for (int d = 0; d < 6; ++d) S.r[d][i] = __ldcg(P.r + d * Np + g);
    hv[k] = __ldcg(P.h + g);
    S.h[halo_index(x, wv_y(lane, k), wv_z(k))] = hv[k];
  }
  warp_load_halo_heights(P, t, S.h, lane);
#pragma unroll
  for (int m = 0; m < 12; ++m) (&S.acc[0][0])[lane + 32 * m] = 0;
  const int inst = __ldcg(P.tinst + t);
  const int hdead = P.geo[inst].hdead;
  __syncwarp();

  long long sink = 0;
  int pulses = 0, lastout = 0, faces = 0;
  bool any = true;
  for (int round = 0;; ++round) {
    if (R > 0) {
      // region relabel: exact in-tile distance to the sink or the frozen halo,
      // then h = max(h, d) (see the block version for why this is valid)
#pragma unroll
      for (int k = 0; k < 16; ++k) {
        const int i = wv_index(lane, k);
        S.h[halo_index(x, wv_y(lane, k), wv_z(k))] = S.rT[i] > 0 ? 1 : INF;
      }
      __syncwarp();
      for (int it = 0; it < 600; ++it) {
        bool ch = false;
#pragma unroll
        for (int k = 0; k < 16; ++k) {
          const int i = wv_index(lane, k);
          const int hi = halo_index(x, wv_y(lane, k), wv_z(k));
          const int cur = S.h[hi];
          int mn = cur;
#pragma unroll
          for (int d = 0; d < 6; ++d)
            if (S.r[d][i] > 0) mn = min(mn, S.h[hi + hoff(d)] + 1);
          if (mn < cur) { S.h[hi] = mn; ch = true; }
        }
        __syncwarp();
        if (!__any_sync(FULL, ch)) break;
      }
#pragma unroll
      for (int k = 0; k < 16; ++k) {
        const int hi = halo_index(x, wv_y(lane, k), wv_z(k));
        int hn = max(hv[k], S.h[hi]);
        if (hn >= hdead) hn = INF;
        hv[k] = hn;
        S.h[hi] = hn;
      }
      __syncwarp();
    }
    for (int p = 0; p < L; ++p) {
      bool moved = false;
      // push step (labels fixed)
#pragma unroll
      for (int k = 0; k < 16; ++k) {
        const int i = wv_index(lane, k);
        const int h = hv[k];
        int e = S.e[i];
        if (e <= 0 || h >= INF) continue;
        const int e0 = e;
        const int y = wv_y(lane, k), z = wv_z(k);
        const int hi = halo_index(x, y, z);
        const int rt = S.rT[i];
        if (rt > 0 && h == 1) {
          const int dl = min(e, rt);
          S.rT[i] = rt - dl;
          e -= dl;
          sink += dl;
          moved = true;
        }
#pragma unroll
        for (int d = 0; d < 6; ++d) {
          if (e <= 0) break;
          const int rr = S.r[d][i];
          if (rr > 0 && S.h[hi + hoff(d)] == h - 1) {
            const int dl = min(e, rr);
            S.r[d][i] = rr - dl;
            e -= dl;
            if (inside(d, x, y, z)) {
              const int iu = i + loff(d);
              atomicAdd(&S.e[iu], dl);
              S.r[d ^ 1][iu] += dl;
            } else {
              S.acc[d][face_entry(d, x, y, z)] += dl;  // single writer: this voxel
              moved = true;
            }
          }
        }
        if (e != e0) atomicSub(&S.e[i], e0 - e);
      }
      if (moved) lastout = pulses + 1;
      __syncwarp();
      // relabel step
      bool act = false;
#pragma unroll
      for (int k = 0; k < 16; ++k) {
        const int i = wv_index(lane, k);
        const int h = hv[k];
        if (S.e[i] <= 0 || h >= INF) continue;
        const int hi = halo_index(x, wv_y(lane, k), wv_z(k));
        const int rt = S.rT[i];
        bool adm = (rt > 0 && h == 1);
        int mn = rt > 0 ? 0 : INF;
#pragma unroll
        for (int d = 0; d < 6; ++d) {
          if (S.r[d][i] > 0) {
            const int hn = S.h[hi + hoff(d)];
            adm = adm || hn == h - 1;
            mn = min(mn, hn);
          }
        }
        if (!adm) {
          int hnew = mn >= INF ? INF : mn + 1;
          if (hnew >= hdead) hnew = INF;
          hv[k] = hnew;
          S.h[hi] = hnew;
        }
        act = act || hv[k] < INF;
      }
      ++pulses;
      __syncwarp();
      any = __any_sync(FULL, act);
      if (!any) break;
    }
    if (!any || round + 1 >= max(R, 1)) break;
  }

  // write back
  bool still = false;
#pragma unroll
  for (int k = 0; k < 16; ++k) {
    const int i = wv_index(lane, k);
    const int64_t g = base + i;
    const int e = S.e[i], rT = S.rT[i];
    P.e[g] = e;
    P.h[g] = hv[k];
    P.rT[g] = rT;
    unsigned m = ((rT > 0) ? 64u : 0u) | ((e > 0) ? 128u : 0u);
#pragma unroll
    for (int d = 0; d < 6; ++d) {
      const int rr = S.r[d][i];
      P.r[d * Np + g] = rr;
      m |= (rr > 0 ? 1u : 0u) << d;
    }
    P.rmask[g] = (uint8_t)m;
    still = still || (e > 0 && hv[k] < INF);
  }
  // flow that left the tile: excess and reverse residual of the neighbour
  __syncwarp();
#pragma unroll 4
  for (int m = 0; m < 12; ++m) {
    for_halo_entry(lane + 32 * m, [&](int f, int hi, int src) {
      const int a = (&S.acc[0][0])[lane + 32 * m];
      if (a > 0) {
        const int nt = __ldcg(P.nbr + f * P.T + t);
        if (nt < 0) { raise_error(P, CGC_ERR_OVERFLOW); return; }  // capacity leaving the grid
        const int64_t ng = (int64_t)nt * TV + src;
        atomicAdd(P.e + ng, a);
        atomicAdd(P.r + (f ^ 1) * Np + ng, a);
        atomicOr((unsigned*)(P.rmask + (ng & ~(int64_t)3)), (128u | (1u << (f ^ 1))) << (8 * (int)(ng & 3)));
        faces |= 1 << f;
      }
    });
  }
  still = __any_sync(FULL, still);
  faces = __reduce_or_sync(FULL, (unsigned)faces);
  lastout = __reduce_max_sync(FULL, (unsigned)lastout);
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) sink += __shfl_down_sync(FULL, sink, o);
  if (lane == 0) {
    P.act[t] = (uint8_t)(still ? 1 : 0);
    if (sink) {
      atomicAdd(P.flow + inst, (unsigned long long)sink);
      if (ex.sink_tiles) atomicAdd(ex.sink_tiles, 1);
      if (ex.tr_sink) ex.tr_sink[t] = 1;
    }
    if (ex.tr_pulses && ex.tr_pulses[t] == 0) ex.tr_pulses[t] = (uint8_t)(lastout > 0 ? min(lastout, 254) : 255);
    atomicAdd(P.stats + S_TILES_SWEPT, 1ull);
    atomicAdd(P.stats + S_PULSES, (unsigned long long)pulses);
    if (APPEND && still) {
      if (atomicExch(P.stamp_sw + t, id_self) != id_self) list_self[atomicAdd(cnt_self, 1)] = t;
    }
  }
  if (lane < 6 && ((faces >> lane) & 1)) {
    const int nt = __ldcg(P.nbr + lane * P.T + t);
    P.act[nt] = 1;
    if (APPEND) {
      if (atomicExch(P.stamp_sw + nt, id_next) != id_next) list_next[atomicAdd(cnt_next, 1)] = nt;
    }
  }
  __syncwarp();
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
    if (act) P.act[t] = 1;  // only ever set during a BFS (bfs_init_tile_w clears it)
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
                                         int32_t* cnt0, const WorkQueue* wq = nullptr) {
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
  if (lane == 0 && (flags & 64u)) enqueue(P, P.stamp_bfs, t, id0, list0, cnt0, wq);
  if (lane < 6 && ((flags >> lane) & 1)) {
    const int nt = __ldcg(P.nbr + lane * P.T + t);
    if (nt >= 0) enqueue(P, P.stamp_bfs, nt, id0, list0, cnt0, wq);
  }
}

__device__ inline void reach_tile_w(const DevPool& P, const int t, WarpReachSmem& S, const uint32_t id_next,
                                    int32_t* list_next, int32_t* cnt_next) {
  const int lane = threadIdx.x & 31;
  const int64_t base = (int64_t)t * TV;
  const int x = wv_x(lane);
  unsigned char rc0[16];
#pragma unroll
  for (int k = 0; k < 16; ++k) {
    const int i = wv_index(lane, k);
    const int hi = halo_index(x, wv_y(lane, k), wv_z(k));
    rc0[k] = __ldcg(P.reach + base + i);
    S.rc[hi] = rc0[k];
    S.m[hi] = __ldcg(P.rmask + base + i);
  }
#pragma unroll 4
  for (int mm = 0; mm < 12; ++mm) {
    for_halo_entry(lane + 32 * mm, [&](int f, int hh, int src) {
      const int nt = __ldcg(P.nbr + f * P.T + t);
      unsigned char rv = 0, mv = 0;
      if (nt >= 0) {
        rv = __ldcg(P.reach + (int64_t)nt * TV + src);
        mv = __ldcg(P.rmask + (int64_t)nt * TV + src);
      }
      S.rc[hh] = rv;
      S.m[hh] = mv;
    });
  }
  __syncwarp();
  for (int it = 0; it < 1200; ++it) {
    bool ch = false;
#pragma unroll
    for (int k = 0; k < 16; ++k) {
      const int hi = halo_index(x, wv_y(lane, k), wv_z(k));
      if (S.rc[hi]) continue;
      bool r = false;
#pragma unroll
      for (int d = 0; d < 6; ++d) {
        const int u = hi + hoff(d);
        r = r || (S.rc[u] && ((S.m[u] >> (d ^ 1)) & 1u));
      }
      if (r) { S.rc[hi] = 1; ch = true; }
    }
    __syncwarp();
    if (!__any_sync(FULL, ch)) break;
  }
  unsigned faces = 0;
#pragma unroll
  for (int k = 0; k < 16; ++k) {
    const int i = wv_index(lane, k);
    const int y = wv_y(lane, k), z = wv_z(k);
    if (S.rc[halo_index(x, y, z)] && !rc0[k]) {
      P.reach[base + i] = 1;
      faces |= face_bits(x, y, z);
    }
  }
  faces = __reduce_or_sync(FULL, faces);
  if (lane < 6 && ((faces >> lane) & 1)) {
    const int nt = __ldcg(P.nbr + lane * P.T + t);
    if (nt >= 0) queue_tile(P, P.stamp_bfs, nt, id_next, list_next, cnt_next);
  }
  __syncwarp();
}

}  // namespace cgc
