// Kernels and host driver of the grid push-relabel engine, plus the C ABI.
//
// The host driver replaces MinCut::compute / MinimalGraphCutComputation::run
// (include/cugip/advanced_operations/detail/graph_cut_implementation.hpp:122-198,
// 286-308): preflow initialisation, then {exact global relabel; K sweep pairs}
// until a global relabel finds no active voxel, then the cut sets.  With
// `persistent` (the default) the whole loop runs inside one cooperative
// launch whose phases are separated by a grid barrier with a bounded wait, so
// no host round trip happens per BFS level or push level (the reference
// synchronises and copies a counter back for every level,
// detail/graph_cut_relabeling.hpp:962-984, detail/graph_cut_push.hpp:395-459).
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdio>
#include <cstring>
#include <atomic>
#include <functional>
#include <memory>
#include <mutex>
#include <new>
#include <string>
#include <vector>

#include "cgc.h"
#include "cgc_internal.h"
#include "cgc_kernels.cuh"
#include "cgc_sched.cuh"
#include "cgc_warp.cuh"
#include "cgc_sync.cuh"
#include "cgc_pool.h"

namespace cgc {

static thread_local std::string g_last_error;
std::atomic<long long> g_launches{0};
void note_launch() { g_launches.fetch_add(1, std::memory_order_relaxed); }

int fail(int code, const std::string& msg) {
  g_last_error = msg;
  return code;
}
int ok() {
  g_last_error.clear();
  return CGC_OK;
}


// ===========================================================================
// kernels
// ===========================================================================

// Copies the linear (x-fastest) t-link arrays of one instance into the
// blocked e (= capS for now) and rT (= capT) planes.
__global__ void __launch_bounds__(512) k_put_tlinks(DevPool P, int inst, const int32_t* __restrict__ capS,
                                                    const int32_t* __restrict__ capT) {
  const InstGeo G = P.geo[inst];
  const int lt = blockIdx.x;
  const int tx = lt % G.TX, ty = (lt / G.TX) % G.TY, tz = lt / (G.TX * G.TY);
  const int l = threadIdx.x;
  const int x = tx * 8 + (l & 7), y = ty * 8 + ((l >> 3) & 7), z = tz * 8 + (l >> 6);
  const int64_t g = (int64_t)(G.tile_base + lt) * TV + l;
  int s = 0, c = 0;
  if (x < G.X && y < G.Y && z < G.Z) {
    const int64_t v = x + (int64_t)G.X * (y + (int64_t)G.Y * z);
    s = capS[v]; c = capT[v];
    if (s < 0 || c < 0) raise_error(P, CGC_ERR_ARG);
  }
  P.e[g] = s;
  P.rT[g] = c;
}

// Copies the n-links of one axis: r[+a][v] = fwd[v], r[-a][v+e_a] = bwd[v].
__global__ void __launch_bounds__(512) k_put_nlinks(DevPool P, int inst, int axis, const int32_t* __restrict__ fwd,
                                                    const int32_t* __restrict__ bwd) {
  const InstGeo G = P.geo[inst];
  const int lt = blockIdx.x;
  const int tx = lt % G.TX, ty = (lt / G.TX) % G.TY, tz = lt / (G.TX * G.TY);
  const int l = threadIdx.x;
  const int x = tx * 8 + (l & 7), y = ty * 8 + ((l >> 3) & 7), z = tz * 8 + (l >> 6);
  const int64_t g = (int64_t)(G.tile_base + lt) * TV + l;
  int f = 0, b = 0;
  if (x < G.X && y < G.Y && z < G.Z) {
    const int c = axis == 0 ? x : axis == 1 ? y : z;
    const int ext = axis == 0 ? G.X : axis == 1 ? G.Y : G.Z;
    const int64_t stride = axis == 0 ? 1 : axis == 1 ? (int64_t)G.X : (int64_t)G.X * G.Y;
    const int64_t v = x + (int64_t)G.X * (y + (int64_t)G.Y * z);
    if (fwd && c + 1 < ext) f = fwd[v];
    if (bwd && c > 0) b = bwd[v - stride];
    if (f < 0 || b < 0) raise_error(P, CGC_ERR_ARG);
  }
  P.r[(2 * axis) * P.Np + g] = f;
  P.r[(2 * axis + 1) * P.Np + g] = b;
}

// Preflow initialisation (replaces initResidualsKernel and
// pushThroughTLinksFromSourceKernel, graph_cut_implementation.hpp:28-40,
// graph_cut_push.hpp:11-24): the t-links of a voxel cancel,
// m = min(capS, capT) goes straight from the source to the sink, the rest of
// capS becomes excess.  Also checks that no excess or residual can exceed
// int32 and builds the residual bit mask.  The kernel is bound by load
// latency: the face neighbours are read first (the same six values for the
// whole tile), then all fourteen per-voxel loads are issued at once, with the
// index of a missing neighbour clamped to the voxel itself and the value
// masked afterwards.
__global__ void __launch_bounds__(512) k_prepare(DevPool P) {
  __shared__ long long red[16];
  const int t = blockIdx.x;
  const int l = threadIdx.x;
  const int x = l & 7, y = (l >> 3) & 7, z = l >> 6;
  const int64_t g = (int64_t)t * TV + l;
  const int64_t Np = P.Np;
  int nbt[6];
#pragma unroll
  for (int d = 0; d < 6; ++d) nbt[d] = __ldg(P.nbr + d * P.T + t);
  const int s = P.e[g], c = P.rT[g];
  int rv[6], bk[6];
  bool has[6];
#pragma unroll
  for (int d = 0; d < 6; ++d) {
    const bool in = inside(d, x, y, z);
    has[d] = in || nbt[d] >= 0;
    const int64_t ng = in ? g + loff(d) : (has[d] ? (int64_t)nbt[d] * TV + l + xoff(d) : g);
    rv[d] = P.r[d * Np + g];
    bk[d] = P.r[(d ^ 1) * Np + ng];
  }
  const int mcap = min(s, c);
  const int e = s - mcap, rT = c - mcap;
  long long inflow = e;
  unsigned m = (rT > 0 ? 64u : 0u) | (e > 0 ? 128u : 0u);
  bool bad = false;
#pragma unroll
  for (int d = 0; d < 6; ++d) {
    const long long back = has[d] ? (long long)bk[d] : 0ll;
    if (!has[d] && rv[d] != 0) bad = true;  // capacity towards the outside of the grid
    inflow += back;
    if ((long long)rv[d] + back > 2147483647ll) bad = true;
    m |= (rv[d] > 0 ? 1u : 0u) << d;
  }
  if (inflow > 2147483647ll) bad = true;
  if (bad) raise_error(P, CGC_ERR_OVERFLOW);
  P.e[g] = e;
  P.rT[g] = rT;
  P.h[g] = 0;  // no label yet (INF would read as "dead" to the first global relabel)
  P.rmask[g] = (uint8_t)m;
  P.reach[g] = 0;
  const long long tot = block_sum64((long long)mcap, red);
  if (l == 0) {
    P.act[t] = 0;
    if (tot) atomicAdd(P.flow + P.tinst[t], (unsigned long long)tot);
  }
}

// Fused upload + preflow of a single instance whose 8 input planes (capS,
// capT, fwd x/y/z, bwd x/y/z; null = zero) are passed by value, so a queued
// solve reads exactly the planes of its own set_* calls (put_tile4).
struct InputPlanes { const int32_t* p[8]; };
__global__ void __launch_bounds__(128) k_put_one(DevPool P, InputPlanes in) {
  put_tile4(P, blockIdx.x, in.p);
}

// Cut sets as mask / background bytes from the 1/0 bytes of one buffer
// (16 bytes per thread where src and dst allow it).
__global__ void k_mask_remap(const uint8_t* __restrict__ src, uint8_t* __restrict__ dst, int64_t n, uint8_t mask,
                             uint8_t bg) {
  const bool vec = ((reinterpret_cast<uintptr_t>(src) | reinterpret_cast<uintptr_t>(dst)) & 15u) == 0;
  const int64_t stride = (int64_t)gridDim.x * blockDim.x;
  const int64_t i0 = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (vec) {
    const int64_t n16 = n / 16;
    for (int64_t i = i0; i < n16; i += stride) {
      uint4 v = reinterpret_cast<const uint4*>(src)[i];
      unsigned* w = reinterpret_cast<unsigned*>(&v);
#pragma unroll
      for (int k = 0; k < 4; ++k) {
        unsigned o = 0;
#pragma unroll
        for (int b = 0; b < 4; ++b) o |= (unsigned)(((w[k] >> (8 * b)) & 1u) ? mask : bg) << (8 * b);
        w[k] = o;
      }
      reinterpret_cast<uint4*>(dst)[i] = v;
    }
    for (int64_t i = n16 * 16 + i0; i < n; i += stride) dst[i] = src[i] ? mask : bg;
  } else {
    for (int64_t i = i0; i < n; i += stride) dst[i] = src[i] ? mask : bg;
  }
}

// Host-driven schedule: one launch per sweep / BFS round.
__global__ void __launch_bounds__(512, 2) k_sweep_list(DevPool P, const int32_t* list, const int32_t* cnt, int L, int R) {
  __shared__ SweepShared S;
  const int n = *cnt;
  for (int i = blockIdx.x; i < n; i += gridDim.x) sweep_tile<false>(P, list[i], L, R, S, 0, nullptr, nullptr, 0, nullptr, nullptr);
}

__global__ void k_compact(DevPool P, int parity, int32_t* list, int32_t* cnt) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  const bool pred = t < P.T && P.act[t] && P.tpar[t] == parity;
  warp_append(P, pred, t, list, cnt);
}

__global__ void __launch_bounds__(512) k_bfs_init(DevPool P) {
  const int nw = gridDim.x * (blockDim.x >> 5);
  for (int t = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5); t < P.T; t += nw) bfs_init_tile_w(P, t);
}

__global__ void k_bfs_queue(DevPool P, uint32_t id0, int32_t* list0, int32_t* cnt0) {
  bfs_queue_tile(P, blockIdx.x * blockDim.x + threadIdx.x, id0, list0, cnt0);
}

__global__ void __launch_bounds__(512, 2) k_bfs_round(DevPool P, const int32_t* list, const int32_t* cnt, uint32_t id_next,
                                                      int32_t* list_next, int32_t* cnt_next) {
  __shared__ BfsShared S;
  const int n = *cnt;
  for (int i = blockIdx.x; i < n; i += gridDim.x) bfs_tile(P, list[i], S, id_next, list_next, cnt_next);
}

__global__ void __launch_bounds__(512) k_reach_init(DevPool P, uint32_t id0, int32_t* list0, int32_t* cnt0) {
  const int nw = gridDim.x * (blockDim.x >> 5);
  for (int t = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5); t < P.T; t += nw)
    reach_init_tile_w(P, t, id0, list0, cnt0);
}

__global__ void __launch_bounds__(512, 2) k_reach_round(DevPool P, const int32_t* list, const int32_t* cnt, uint32_t id_next,
                                                        int32_t* list_next, int32_t* cnt_next) {
  __shared__ ReachShared S;
  const int n = *cnt;
  for (int i = blockIdx.x; i < n; i += gridDim.x) reach_tile(P, list[i], S, id_next, list_next, cnt_next);
}

// ---------------------------------------------------------------------------
// Grid-wide barrier of the persistent solve (bounded waits, cgc_sync.cuh).
__device__ __forceinline__ bool grid_sync(const DevPool& P, uint64_t limit_ns) {
  return grid_barrier(P.bar, P.err, limit_ns);
}

__device__ __forceinline__ int ld_cnt(const int32_t* p) { return *(volatile const int32_t*)p; }


// Learned-scheduler stage at the start of a relabel cycle: the features of
// every tile (zero for inactive ones; recorded when tracing), then the three
// convolution layers on the tensor cores, the last one with the head (budgets
// and priorities).  The active tiles are the entries of the cycle's first
// lists (la: na entries, lb: nb).  Four grid barriers.  Returns false when a
// barrier failed.
__device__ __forceinline__ bool sched_stage(const DevPool& P, const SolveParams& prm, int cycle, bool learned,
                                            bool tracing, const int32_t* la, int na, const int32_t* lb, int nb) {
  const int G = gridDim.x, b = blockIdx.x, tid = threadIdx.x;
  const int gw = b * (blockDim.x >> 5) + (tid >> 5), nw = G * (blockDim.x >> 5);
  // zeros for the inactive tiles, a thread per tile
  for (int t = b * blockDim.x + tid; t < P.T; t += G * blockDim.x) {
    const int64_t r = (int64_t)cycle * P.T + t;  // trace row
    if (tracing) { P.tpulses[r] = 0; P.tsink[r] = 0; }
    if (__ldcg(P.act + t)) continue;
    uint4* f = reinterpret_cast<uint4*>(P.sfeat + (int64_t)t * SCHED_C);
    f[0] = make_uint4(0, 0, 0, 0);
    f[1] = make_uint4(0, 0, 0, 0);
    if (tracing) {
      uint4* tf = reinterpret_cast<uint4*>(P.tfeat + r * SCHED_C);
      tf[0] = make_uint4(0, 0, 0, 0);
      tf[1] = make_uint4(0, 0, 0, 0);
    }
  }
  // features of the active tiles, a warp per list entry
  for (int i = gw; i < na + nb; i += nw) {
    const int t = __ldcg(i < na ? la + i : lb + (i - na));
    sched_features_warp(P, t, P.sfeat, tracing ? P.tfeat + ((int64_t)cycle * P.T + t) * SCHED_C : nullptr);
  }
  if (!grid_sync(P, prm.limit_ns)) return false;
  if (!learned) return true;
  const PoolSpace sp{&P};
  for (int layer = 0; layer < 3; ++layer) {
    sched_layer(sp, layer, pool_io(P, layer), gw, nw, nullptr);
    if (!grid_sync(P, prm.limit_ns)) return false;
  }
  return true;
}

// BFS rounds with many tiles run a warp per tile on the first BFS_WARPS warps
// of each CTA (one WarpBfsSmem slice each).
constexpr int BFS_WARPS = 8;

union SolveShared {
  SweepShared sw;
  BfsShared bfs;
  WarpBfsSmem wbfs[BFS_WARPS];
  ReachShared rc;
  SchedShared sched;
};

// The whole solve in one cooperative launch; a CTA of 512 threads is the unit
// that visits a tile.
template <bool BFSW = false>
__device__ __forceinline__ void solve_body(const DevPool& P, const SolveParams& prm, SolveShared& S) {
  const int G = gridDim.x, b = blockIdx.x, tid = threadIdx.x;
  const bool leader = tid == 0;
  // warps of the grid, for the passes that visit every tile with a warp
  const int gw = b * (int)(blockDim.x >> 5) + (tid >> 5), nw = G * (int)(blockDim.x >> 5);
  // Hands out the n entries of a round.  The first entry of CTA b is entry b;
  // later ones come from the round's counter (C_TAKE0 + round % 3, the next
  // round's slot is cleared meanwhile) through an atomic issued when the
  // current visit starts and read when it ends, so visits of uneven cost
  // spread over the CTAs.
  __shared__ int s_next;
  int round_no = 0;
  auto for_entries = [&](int n, auto&& visit) {
    if (!CGC_IN_BOUNDS(P, n, P.T + 1)) n = P.T;  // a list holds at most T entries
    int32_t* take = P.cnt + C_TAKE0 + round_no % 3;
    if (b == 0 && tid == 0) P.cnt[C_TAKE0 + (round_no + 1) % 3] = 0;
    ++round_no;
    int i = b;
    while (i < n) {
      int nx = 0;
      if (tid == 0) nx = atomicAdd(take, 1);
      visit(i);
      if (tid == 0) s_next = G + nx;
      __syncthreads();
      i = s_next;
      __syncthreads();
    }
  };
  int32_t* const bl[3] = {P.lists, P.lists + P.T, P.lists + 2 * P.T};
  int32_t* const sl[4] = {P.lists + 3 * P.T, P.lists + 4 * P.T, P.lists + 5 * P.T, P.lists + 6 * P.T};
  int32_t* const bc = P.cnt + C_BFS0;
  int32_t* const sc = P.cnt + C_SW0;
  uint32_t bfs_id = 1;
  int64_t s = 0;        // sweep index; sweep s uses list s&3 and stamp id s+1
  int64_t sweeps = 0;
  long long rounds = 0, relabels = 0;
  unsigned long long ns_bfs = 0, ns_sweep = 0, ns_reach = 0, ns_sched = 0;
  int traced = 0;
  uint64_t tmark = globaltimer_ns();
  const uint64_t t_launch = tmark;
  int ntrace = 0;
  // block 0 records one phase step (after the barrier that ended it)
  auto record = [&](unsigned long long kind, long long index, int tiles) {
    if (b == 0 && tid == 0 && P.trace && ntrace < TRACE_CAP) {
      P.trace[2 * ntrace] = (kind << 56) | ((unsigned long long)(index & 0xffffffffll) << 24) | (unsigned)(tiles & 0xffffff);
      P.trace[2 * ntrace + 1] = globaltimer_ns() - t_launch;
      ++ntrace;
    }
  };
  auto lap = [&](unsigned long long& acc) {
    const uint64_t now = globaltimer_ns();
    acc += now - tmark;
    tmark = now;
  };
  // Tile rounds of one relabel pass: round 0 visits the entries of list0
  // (count *cnt0), round k > 0 the tiles round k - 1 queued in bl[k % 3]
  // (bc[1], bc[2] zero on entry).  inval: invalidation visits, otherwise BFS
  // visits.  False when a grid barrier gave up.
  auto relabel_rounds = [&](int32_t* list0, int32_t* cnt0, bool inval) -> bool {
    int k = 0;
    for (;;) {
      int32_t* const lst = k == 0 ? list0 : bl[k % 3];
      int n = ld_cnt(k == 0 ? cnt0 : bc + k % 3);
      if (n == 0) break;
      if (!CGC_IN_BOUNDS(P, n, P.T + 1)) n = P.T;  // a list holds at most T entries
      if (b == 0 && tid == 0) bc[(k + 2) % 3] = 0;
      if (inval) {
        const uint32_t id_inc = (uint32_t)(relabels + 1);
        for_entries(n, [&](int i) {
          inval_tile(P, __ldcg(lst + i), S.bfs, bfs_id + k + 1, bl[(k + 1) % 3], bc + (k + 1) % 3, id_inc, sl[0],
                     P.cnt + C_INC);
        });
      } else if (BFSW && n / G >= prm.bfs_warp_min) {
        // Throughput-bound round: a warp per tile (no block barriers, a
        // tile's relaxation costs one warp's issue slots instead of 16),
        // entries handed out like for_entries, per warp.
        int32_t* take = P.cnt + C_TAKE0 + round_no % 3;
        if (b == 0 && tid == 0) P.cnt[C_TAKE0 + (round_no + 1) % 3] = 0;
        ++round_no;
        const int wid = tid >> 5;
        if (wid < BFS_WARPS) {
          int i = b * BFS_WARPS + wid;
          while (i < n) {
            int nx = 0;
            if ((tid & 31) == 0) nx = atomicAdd(take, 1);
            bfs_tile_w(P, __ldcg(lst + i), S.wbfs[wid], bfs_id + k + 1, bl[(k + 1) % 3], bc + (k + 1) % 3);
            i = G * BFS_WARPS + __shfl_sync(0xffffffffu, nx, 0);
          }
        }
      } else {
        for_entries(n, [&](int i) {
          bfs_tile(P, __ldcg(lst + i), S.bfs, bfs_id + k + 1, bl[(k + 1) % 3], bc + (k + 1) % 3);
        });
      }
      ++k;
      if (!grid_sync(P, prm.limit_ns)) return false;
      record(TR_BFS_ROUND, rounds + k, n);
    }
    bfs_id += k + 1;
    rounds += k;
    return true;
  };
  uint32_t c0 = 0;  // sweep stamps above c0 were written during the current cycle
  for (;;) {
    // ------------------------------------------------ exact global relabel
    // The first relabel of a solve is a full BFS from the sink; later ones
    // are incremental when the pool has the stamps for it.
    const bool inc = prm.incremental && relabels > 0 && P.stamp_inc != nullptr;
    if (b == 0 && tid == 0) {
      bc[0] = bc[1] = bc[2] = 0;
      sc[0] = sc[1] = sc[2] = sc[3] = 0;
      P.cnt[C_SINKT0] = P.cnt[C_SINKT0 + 1] = P.cnt[C_SINKT0 + 2] = 0;
      P.cnt[C_TAKE0] = P.cnt[C_TAKE0 + 1] = P.cnt[C_TAKE0 + 2] = 0;
      P.cnt[C_INC] = 0;
    }
    round_no = 0;
    if (!grid_sync(P, prm.limit_ns)) return;
    if (!inc) {
      for (int t = gw; t < P.T; t += nw) bfs_init_tile_w(P, t);  // a warp per tile in both shapes
      if (!grid_sync(P, prm.limit_ns)) return;
      for (int t0 = b * blockDim.x; t0 < P.T; t0 += G * blockDim.x) bfs_queue_tile(P, t0 + tid, bfs_id, bl[0], bc + 0);
      if (!grid_sync(P, prm.limit_ns)) return;
      if (!relabel_rounds(bl[0], bc + 0, false)) return;
    } else {
      // invalidation from the tiles the last cycle queued, then BFS rounds
      // from the tiles with dropped voxels (listed in sl[0], free until the
      // sweep lists are rebuilt below)
      for (int t0 = b * blockDim.x; t0 < P.T; t0 += G * blockDim.x)
        inval_queue_tile(P, t0 + tid, c0, prm.exclusive != 0, bfs_id, bl[0], bc + 0);
      if (!grid_sync(P, prm.limit_ns)) return;
      if (!relabel_rounds(bl[0], bc + 0, true)) return;
      if (b == 0 && tid == 0) bc[0] = bc[1] = bc[2] = 0;
      if (!grid_sync(P, prm.limit_ns)) return;
      if (!relabel_rounds(sl[0], P.cnt + C_INC, false)) return;
    }
    ++relabels;
    lap(ns_bfs);
    // ------------------------------------------------ active tiles -> parity lists
    s += 2;  // fresh stamp ids for the lists built here
    c0 = (uint32_t)s;
    for (int t0 = b * blockDim.x + (tid & ~31); t0 < P.T; t0 += G * blockDim.x) {  // warp-aggregated appends
      const int t = t0 + (tid & 31);
      const bool a = t < P.T && __ldcg(P.act + t);
      const int par = a ? __ldcg(P.tpar + t) : 0;
      if (prm.exclusive) {  // one list: the whole active set is queued for sweep s
        if (a) P.stamp_sw[(s & 1) * P.T + t] = (uint32_t)(s + 1);
        warp_append(P, a, t, sl[s & 3], sc + (s & 3));
      } else {              // one list per parity, for sweeps s and s + 1
        if (a) P.stamp_sw[t] = (uint32_t)(s + par + 1);
        warp_append(P, a && par == 0, t, sl[s & 3], sc + (s & 3));
        warp_append(P, a && par == 1, t, sl[(s + 1) & 3], sc + ((s + 1) & 3));
      }
    }
    if (!grid_sync(P, prm.limit_ns)) return;
    const int nact = ld_cnt(sc + (s & 3)) + ld_cnt(sc + ((s + 1) & 3));
    record(TR_RELABEL_DONE, relabels, nact);
    if (b == 0 && tid == 0 && P.trace && ntrace < TRACE_CAP) {  // flow at this relabel (after the barrier)
      unsigned long long f = 0;
      for (int i = 0; i < P.ninst; ++i) f += __ldcg(P.flow + i);
      P.trace[2 * ntrace] = ((unsigned long long)TR_FLOW << 56) | ((unsigned long long)(relabels & 0xffffffffll) << 24);
      P.trace[2 * ntrace + 1] = f;
      ++ntrace;
    }
    if (nact == 0) break;
    if (sweeps >= prm.max_sweeps) {
      if (b == 0 && tid == 0) raise_error(P, CGC_ERR_NOT_CONVERGED);
      break;
    }
    // ------------------------------------------------ learned scheduler
    const int cycle = (int)relabels - 1;
    const bool tracing = prm.trace_cycles > cycle;
    if (tracing) traced = cycle + 1;
    // Priorities (deferral) only pay off while active tiles outnumber the
    // CTAs: with fewer, a sweep lasts one tile visit whatever the order.
    // Budgets can still shorten that visit, so learned = 3 runs the stage in
    // every cycle, with each tile's budget capped at the schedule's L (a
    // budget may only end a visit early).
    const bool throughput = nact > 2 * G;
    const bool learned = prm.learned && (throughput || prm.learned == 3);
    if (learned || tracing) {
      if (!sched_stage(P, prm, cycle, learned, tracing, sl[s & 3], ld_cnt(sc + (s & 3)), sl[(s + 1) & 3],
                       prm.exclusive ? 0 : ld_cnt(sc + ((s + 1) & 3))))
        return;
      lap(ns_sched);
    }
    // ------------------------------------------------ sweeps
    SweepExtra ex;
    if (tracing) {
      ex.tr_pulses = P.tpulses + (int64_t)cycle * P.T;
      ex.tr_sink = P.tsink + (int64_t)cycle * P.T;
    }
    int idle = 0;  // consecutive sweeps in which no tile delivered flow to the sink
    for (int j = 0; j < 2 * prm.K; ++j, ++s) {
      const int n = ld_cnt(sc + (s & 3));
      if (n == 0 && (prm.exclusive || ld_cnt(sc + ((s + 1) & 3)) == 0)) break;
      if (b == 0 && tid == 0) {
        sc[(s + 3) & 3] = 0;
        P.cnt[C_SINKT0 + (int)((s + 1) % 3)] = 0;
      }
      ex.sink_tiles = P.cnt + C_SINKT0 + (int)(s % 3);
      // the learned scheduler defers low-priority tiles during the first half
      // of the cycle; every active tile is swept in the second half
      const bool may_defer = learned && throughput && (prm.learned == 1 || prm.learned == 3) && j < prm.K;
      // Parity sweeps: sweep s uses stamp id s + 1; a visited tile queues the
      // tiles it pushed into for sweep s + 1 and itself, of the same parity,
      // for sweep s + 2.  Exclusive sweeps: every queued tile runs unless it
      // has the other parity than s and a face neighbour is queued for sweep
      // s, so the tiles that run form an independent set (no two share a
      // face) and the halo heights and cross-face pushes are exact as under
      // the parity schedule; everything is queued for sweep s + 1, with the
      // stamps in half (s+1)&1 of stamp_sw, so half s&1 -- this sweep's list --
      // does not change during the sweep.
      uint32_t* const stamp_q = prm.exclusive ? P.stamp_sw + ((s + 1) & 1) * P.T : P.stamp_sw;
      const uint32_t id_self = (uint32_t)(prm.exclusive ? s + 2 : s + 3);
      int32_t* const list_self = sl[(prm.exclusive ? s + 1 : s + 2) & 3];
      int32_t* const cnt_self = sc + ((prm.exclusive ? s + 1 : s + 2) & 3);
      for_entries(n, [&](int i) {
        const int t = __ldcg(sl[s & 3] + i);
        if (may_defer && !__ldcg(P.sprio + t)) {
          if (leader && atomicExch(stamp_q + t, id_self) != id_self) list_self[atomicAdd(cnt_self, 1)] = t;
          return;
        }
        if (prm.exclusive && (int)__ldcg(P.tpar + t) != (int)(s & 1)) {  // uniform over the block
          bool queued_nb = false;
          if (tid < 6) {
            const int nb = __ldcg(P.nbr + tid * P.T + t);
            queued_nb = nb >= 0 && __ldcg(P.stamp_sw + (s & 1) * P.T + nb) == (uint32_t)(s + 1);
          }
          if (__syncthreads_or(queued_nb)) {  // wait one sweep
            if (leader) queue_tile(P, stamp_q, t, (uint32_t)(s + 2), sl[(s + 1) & 3], sc + ((s + 1) & 3));
            return;
          }
        }
        const int L = !learned ? prm.L
                      : prm.learned == 3 ? min((int)__ldcg(P.sbudget + t), prm.L) : (int)__ldcg(P.sbudget + t);
        sweep_tile<true>(P, t, L, prm.R, S.sw, (uint32_t)(s + 2), sl[(s + 1) & 3], sc + ((s + 1) & 3), id_self,
                         list_self, cnt_self, ex, stamp_q);
      });
      ++sweeps;
      if (!grid_sync(P, prm.limit_ns)) return;
      record(TR_SWEEP, sweeps, n);
      // Early relabel: after stall consecutive non-empty sweeps of each parity
      // delivered no flow to the sink.  Empty sweeps do not count, so every
      // cycle performs at least one push or relabel; labels never decrease
      // (an exact relabel only raises valid labels), so the solve still ends.
      if (n > 0) idle = ld_cnt(P.cnt + C_SINKT0 + (int)(s % 3)) ? 0 : idle + 1;
      if (prm.stall > 0 && idle >= 2 * prm.stall) { ++s; break; }
    }
    lap(ns_sweep);
  }
  lap(ns_bfs);
  // ------------------------------------------------ source-side reachability
  if (b == 0 && tid == 0) {
    bc[0] = bc[1] = bc[2] = 0;
    P.cnt[C_TAKE0] = P.cnt[C_TAKE0 + 1] = P.cnt[C_TAKE0 + 2] = 0;
  }
  round_no = 0;
  if (!grid_sync(P, prm.limit_ns)) return;
  for (int t = gw; t < P.T; t += nw) reach_init_tile_w(P, t, bfs_id, bl[0], bc + 0);
  if (!grid_sync(P, prm.limit_ns)) return;
  int k = 0;
  for (;;) {
    const int n = ld_cnt(bc + k % 3);
    if (n == 0) break;
    if (b == 0 && tid == 0) bc[(k + 2) % 3] = 0;
    for_entries(n, [&](int i) {
      reach_tile(P, __ldcg(bl[k % 3] + i), S.rc, bfs_id + k + 1, bl[(k + 1) % 3], bc + (k + 1) % 3);
    });
    ++k;
    if (!grid_sync(P, prm.limit_ns)) return;
    record(TR_REACH_ROUND, k, n);
  }
  if (b == 0 && tid == 0) {
    P.stats[S_SWEEPS] = (unsigned long long)sweeps;
    P.stats[S_RELABELS] = (unsigned long long)relabels;
    P.stats[S_ROUNDS] = (unsigned long long)rounds;
    lap(ns_reach);
    P.stats[S_NS_BFS] = ns_bfs;
    P.stats[S_NS_SWEEP] = ns_sweep;
    P.stats[S_NS_REACH] = ns_reach;
    P.stats[S_TRACE_N] = (unsigned long long)ntrace;
    P.stats[S_TRACE_CYC] = (unsigned long long)traced;
    P.stats[S_NS_SCHED] = ns_sched;
  }
}

// Cooperative launches of this library on one device run one after another.
// Each waits on the device (an event, no host synchronisation) for the
// previous one to end: two grid-barrier kernels in flight on different
// streams could each hold part of the SMs and wait for their missing CTAs,
// until their bounded barriers gave up.  Launches into a stream under capture
// are not ordered (a CUDA graph is replayed on its own).
static std::mutex g_coop_mu;
static cudaEvent_t g_coop_last[64] = {};

int coop_launch_ordered(int device, cudaStream_t stream, const std::function<int()>& launch) {
  cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
  CGC_CUDA(cudaStreamIsCapturing(stream, &cs));
  if (cs != cudaStreamCaptureStatusNone || device < 0 || device >= 64) return launch();
  std::lock_guard<std::mutex> lock(g_coop_mu);
  cudaEvent_t& last = g_coop_last[device];
  if (!last) CGC_CUDA(cudaEventCreateWithFlags(&last, cudaEventDisableTiming));
  CGC_CUDA(cudaStreamWaitEvent(stream, last, 0));  // a no-op before the first record
  if (int rc = launch()) return rc;
  CGC_CUDA(cudaEventRecord(last, stream));
  return CGC_OK;
}

int launch_solve(Pool& p, const cgc_options& o, const DevPool& d, const SolveParams& prm, cudaStream_t stream) {
  cudaLaunchConfig_t cfg = {};
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeCooperative;
  attr[0].val.cooperative = 1;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  cfg.stream = stream;
  const bool three = o.ctas_per_sm == 3, four = o.ctas_per_sm == 4;
  cfg.gridDim = dim3(four ? p.coop_blocks4 : three ? p.coop_blocks3 : p.coop_blocks);
  cfg.blockDim = dim3(512);
  cfg.dynamicSmemBytes = 0;
  const bool bw = prm.bfs_warp_min > 0;
  int rc = coop_launch_ordered(p.device, stream, [&]() -> int {
    if (four) CGC_CUDA(cudaLaunchKernelEx(&cfg, bw ? k_solve4w : k_solve4, d, prm));
    else if (three) CGC_CUDA(cudaLaunchKernelEx(&cfg, bw ? k_solve3w : k_solve3, d, prm));
    else CGC_CUDA(cudaLaunchKernelEx(&cfg, k_solve, d, prm));
    return CGC_OK;
  });
  if (rc) return rc;
  note_launch();
  return ok();
}

// The solve kernel at 2 CTAs per SM (64 registers), at 3 (40 registers, a
// few spills) and at 4 (2048 threads, 32 registers).
__global__ void __launch_bounds__(512, 2) k_solve(DevPool P, SolveParams prm) {
  __shared__ SolveShared S;
  solve_body(P, prm, S);
}
__global__ void __launch_bounds__(512, 3) k_solve3(DevPool P, SolveParams prm) {
  __shared__ SolveShared S;
  solve_body(P, prm, S);
}
__global__ void __launch_bounds__(512, 4) k_solve4(DevPool P, SolveParams prm) {
  __shared__ SolveShared S;
  solve_body(P, prm, S);
}
// The same with warp-per-tile BFS rounds (SolveParams::bfs_warp_min); separate
// kernels, so that the others do not carry that code's registers.
__global__ void __launch_bounds__(512, 3) k_solve3w(DevPool P, SolveParams prm) {
  __shared__ SolveShared S;
  solve_body<true>(P, prm, S);
}
__global__ void __launch_bounds__(512, 4) k_solve4w(DevPool P, SolveParams prm) {
  __shared__ SolveShared S;
  solve_body<true>(P, prm, S);
}

// Output kernels (linear layout of one instance).  k_segments, a thread per
// voxel, serves the allocation-free entry point; grids and batches use
// k_segments_lin / k_seg_all (four voxels per thread).
__global__ void k_segments(DevPool P, int inst, int which, uint8_t* out, uint8_t mask, uint8_t bg) {
  const InstGeo G = P.geo[inst];
  const int64_t N = (int64_t)G.X * G.Y * G.Z;
  for (int64_t v = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; v < N; v += (int64_t)gridDim.x * blockDim.x) {
    const int x = (int)(v % G.X), y = (int)((v / G.X) % G.Y), z = (int)(v / ((int64_t)G.X * G.Y));
    const int64_t t = G.tile_base + (x >> 3) + G.TX * ((y >> 3) + G.TY * (z >> 3));
    const int64_t g = t * TV + (x & 7) + 8 * (y & 7) + 64 * (z & 7);
    const bool in = which == CGC_SEG_SINK_REACH ? (P.h[g] < INF) : (P.reach[g] != 0);
    out[v] = in ? mask : bg;
  }
}

// The same in linear voxel order, four voxels per thread (seg_gather4 /
// seg_store4).
__global__ void __launch_bounds__(256) k_segments_lin(DevPool P, int inst, int which, uint8_t* out, uint8_t mask,
                                                      uint8_t bg) {
  const InstGeo G = P.geo[inst];
  const int64_t N = (int64_t)G.X * G.Y * G.Z;
  for (int64_t v0 = 4 * ((int64_t)blockIdx.x * blockDim.x + threadIdx.x); v0 < N;
       v0 += 4 * (int64_t)gridDim.x * blockDim.x) {
    unsigned bits = 0;
    if (which == CGC_SEG_SINK_REACH) seg_gather4(P, G, v0, N, &bits, nullptr);
    else seg_gather4(P, G, v0, N, nullptr, &bits);
    seg_store4(out, v0, N, bits, mask, bg);
  }
}

__global__ void k_unpermute(DevPool P, int inst, const int32_t* plane, int32_t* out) {
  const InstGeo G = P.geo[inst];
  const int64_t N = (int64_t)G.X * G.Y * G.Z;
  for (int64_t v = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; v < N; v += (int64_t)gridDim.x * blockDim.x) {
    const int x = (int)(v % G.X), y = (int)((v / G.X) % G.Y), z = (int)(v / ((int64_t)G.X * G.Y));
    const int64_t t = G.tile_base + (x >> 3) + G.TX * ((y >> 3) + G.TY * (z >> 3));
    out[v] = plane[t * TV + (x & 7) + 8 * (y & 7) + 64 * (z & 7)];
  }
}

// ===========================================================================
// host side
// ===========================================================================

int check_device_error(Pool& p, const char* where) {
  int32_t err = 0;
  CGC_CUDA(cudaMemcpyAsync(&err, p.dp.err, sizeof(int32_t), cudaMemcpyDeviceToHost, p.stream));
  CGC_CUDA(cudaStreamSynchronize(p.stream));
  if (err == 0) return CGC_OK;
#ifdef CGC_BOUNDS_CHECK
  if (err == CGC_ERR_ARG) {
    unsigned long long at = 0;
    CGC_CUDA(cudaMemcpyAsync(&at, p.dp.stats + S_BOUND_AT, 8, cudaMemcpyDeviceToHost, p.stream));
    CGC_CUDA(cudaStreamSynchronize(p.stream));
    return fail(err, std::string(where) + ": index out of range (bounds-checked build): " +
                         std::to_string((long long)at) + ", or a negative capacity");
  }
#endif
  const char* what = err == CGC_ERR_OVERFLOW ? "capacities may overflow int32 excess/residuals (or a capacity points outside the grid)"
                   : err == CGC_ERR_ARG ? "negative capacity"
                   : err == CGC_ERR_TIMEOUT ? "a device-side wait timed out"
                   : err == CGC_ERR_NOT_CONVERGED ? "max_sweeps reached before convergence"
                   : "device error";
  return fail(err, std::string(where) + ": " + what);
}

int pool_create(int32_t count, const int32_t* ext, void* stream, Pool** out) {
  if (!out || count <= 0 || !ext) return fail(CGC_ERR_ARG, "create: bad arguments");
  std::unique_ptr<Pool> p(new (std::nothrow) Pool());
  if (!p) return fail(CGC_ERR_OOM, "create: host allocation");
  CGC_CUDA(cudaGetDevice(&p->device));
  p->stream = (cudaStream_t)stream;
  p->ninst = count;
  int64_t T = 0;
  for (int i = 0; i < count; ++i) {
    const int32_t X = ext[3 * i], Y = ext[3 * i + 1], Z = ext[3 * i + 2];
    if (X <= 0 || Y <= 0 || Z <= 0) return fail(CGC_ERR_ARG, "create: extents must be positive");
    InstGeo G{};
    G.X = X; G.Y = Y; G.Z = Z;
    G.TX = (X + 7) / 8; G.TY = (Y + 7) / 8; G.TZ = (Z + 7) / 8;
    G.tile_base = (int32_t)T;
    const int64_t n = (int64_t)X * Y * Z;
    if (n + 1 >= (int64_t)INF) return fail(CGC_ERR_ARG, "create: instance too large for int32 heights");
    G.hdead = (int32_t)(n + 1);  // a distance to the sink is at most n (a path through every voxel)
    T += (int64_t)G.TX * G.TY * G.TZ;
    if (T > (int64_t)1 << 30) return fail(CGC_ERR_ARG, "create: too many tiles");
    p->maxN = std::max(p->maxN, n);
    p->geo.push_back(G);
  }
  p->T = (int32_t)T;
  p->Np = T * TV;
  p->uploaded.assign(count, 0u);
  p->flows.assign(count, 0);

  // one device allocation for all state (planes first, 256-byte aligned pieces)
  const int64_t Np = p->Np;
  auto al = [](int64_t b) { return (b + 255) & ~(int64_t)255; };
  int64_t off = 0;
  const int64_t o_e = off; off += al(Np * 4);
  const int64_t o_h = off; off += al(Np * 4);
  const int64_t o_rT = off; off += al(Np * 4);
  const int64_t o_r = off; off += al(6 * Np * 4);
  const int64_t o_rm = off; off += al(Np);
  const int64_t o_rc = off; off += al(Np);
  const int64_t o_nbr = off; off += al(6 * T * 4);
  const int64_t o_ti = off; off += al(T * 4);
  const int64_t o_tp = off; off += al(T);
  const int64_t o_act = off; off += al(T);
  const int64_t o_tf = off; off += al(T * 2);
  const int64_t o_sb = off; off += al(T * 4);
  const int64_t o_ss = off; off += al(2 * T * 4);
  const int64_t o_si = off; off += al(T * 4);
  const int64_t o_li = off; off += al(7 * T * 4);
  const int64_t o_cnt = off; off += al(C_NCOUNTERS * 4);
  const int64_t o_fl = off; off += al((int64_t)count * 8);
  const int64_t o_geo = off; off += al((int64_t)count * sizeof(InstGeo));
  const int64_t o_st = off; off += al(S_NSTATS * 8);
  const int64_t o_err = off; off += al(4);
  const int64_t o_bar = off; off += al(8);
  const int64_t o_tr = off; off += al(2 * TRACE_CAP * 8);
  CGC_CUDA(cudaMalloc(&p->dbuf, off));
  CGC_CUDA(cudaMemsetAsync(p->dbuf, 0, off, p->stream));
  char* base = (char*)p->dbuf;
  DevPool& d = p->dp;
  d.T = p->T; d.ninst = count; d.Np = Np;
  d.e = (int32_t*)(base + o_e); d.h = (int32_t*)(base + o_h); d.rT = (int32_t*)(base + o_rT);
  d.r = (int32_t*)(base + o_r); d.rmask = (uint8_t*)(base + o_rm); d.reach = (uint8_t*)(base + o_rc);
  d.nbr = (int32_t*)(base + o_nbr); d.tinst = (int32_t*)(base + o_ti); d.tpar = (uint8_t*)(base + o_tp);
  d.act = (uint8_t*)(base + o_act); d.tflag = (uint16_t*)(base + o_tf); d.stamp_bfs = (uint32_t*)(base + o_sb); d.stamp_sw = (uint32_t*)(base + o_ss);
  d.stamp_inc = (uint32_t*)(base + o_si);
  d.lists = (int32_t*)(base + o_li); d.cnt = (int32_t*)(base + o_cnt);
  d.flow = (unsigned long long*)(base + o_fl); d.geo = (InstGeo*)(base + o_geo);
  d.stats = (unsigned long long*)(base + o_st); d.err = (int32_t*)(base + o_err); d.bar = (uint32_t*)(base + o_bar);
  d.trace = (unsigned long long*)(base + o_tr);

  // tile tables
  std::vector<int32_t> nbr(6 * (size_t)T, -1), ti((size_t)T);
  std::vector<uint8_t> tp((size_t)T);
  for (int i = 0; i < count; ++i) {
    const InstGeo& G = p->geo[i];
    for (int tz = 0; tz < G.TZ; ++tz)
      for (int ty = 0; ty < G.TY; ++ty)
        for (int tx = 0; tx < G.TX; ++tx) {
          const int64_t t = G.tile_base + tx + (int64_t)G.TX * (ty + (int64_t)G.TY * tz);
          ti[t] = i;
          tp[t] = (uint8_t)((tx + ty + tz) & 1);
          auto id = [&](int a, int b2, int c) -> int32_t {
            if (a < 0 || b2 < 0 || c < 0 || a >= G.TX || b2 >= G.TY || c >= G.TZ) return -1;
            return (int32_t)(G.tile_base + a + (int64_t)G.TX * (b2 + (int64_t)G.TY * c));
          };
          nbr[PX * T + t] = id(tx + 1, ty, tz); nbr[MX * T + t] = id(tx - 1, ty, tz);
          nbr[PY * T + t] = id(tx, ty + 1, tz); nbr[MY * T + t] = id(tx, ty - 1, tz);
          nbr[PZ * T + t] = id(tx, ty, tz + 1); nbr[MZ * T + t] = id(tx, ty, tz - 1);
        }
  }
  CGC_CUDA(cudaMemcpyAsync((void*)d.nbr, nbr.data(), nbr.size() * 4, cudaMemcpyHostToDevice, p->stream));
  CGC_CUDA(cudaMemcpyAsync((void*)d.tinst, ti.data(), ti.size() * 4, cudaMemcpyHostToDevice, p->stream));
  CGC_CUDA(cudaMemcpyAsync((void*)d.tpar, tp.data(), tp.size(), cudaMemcpyHostToDevice, p->stream));
  CGC_CUDA(cudaMemcpyAsync((void*)d.geo, p->geo.data(), p->geo.size() * sizeof(InstGeo), cudaMemcpyHostToDevice, p->stream));
  p->voff.resize(count);
  for (int i = 0; i < count; ++i) {  // offsets of multiples of 4: 16-byte aligned plane rows
    p->voff[i] = p->sumN;
    p->sumN += ((int64_t)p->geo[i].X * p->geo[i].Y * p->geo[i].Z + 3) & ~(int64_t)3;
  }
  p->host_in.assign(8 * (size_t)count, nullptr);
  CGC_CUDA(cudaMallocHost(&p->pinned_cnt, 64 * 4));
  CGC_CUDA(cudaEventCreateWithFlags(&p->inputs_read, cudaEventDisableTiming));
  for (auto& e : p->ev) CGC_CUDA(cudaEventCreate(&e));

  cudaDeviceProp prop;
  CGC_CUDA(cudaGetDeviceProperties(&prop, p->device));
  p->sms = prop.multiProcessorCount;
  int occ = 0;
  CGC_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, k_solve, 512, 0));
  p->coop_blocks = std::max(1, occ) * p->sms;
  int occ3 = 0;
  CGC_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ3, k_solve3, 512, 0));
  p->coop_blocks3 = std::max(1, occ3) * p->sms;
  int occ4 = 0, occ3w = 0, occ4w = 0;
  CGC_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ4, k_solve4, 512, 0));
  CGC_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ3w, k_solve3w, 512, 0));
  CGC_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ4w, k_solve4w, 512, 0));
  p->coop_blocks4 = std::max(1, std::min(occ4, occ4w)) * p->sms;
  p->coop_blocks3 = std::min(p->coop_blocks3, std::max(1, occ3w) * p->sms);
  int occ2 = 0;
  CGC_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ2, k_sweep_list, 512, 0));
  p->sweep_blocks = std::max(1, occ2) * p->sms;
  CGC_CUDA(cudaStreamSynchronize(p->stream));
  *out = p.release();
  return ok();
}

// Inputs of the set_* calls go into linear device planes (one copy per
// plane, no kernel); the fused upload kernel of the next solve reads them.
// Host uploads run on a copy stream of their own, after the upload kernel of
// the last enqueued solve has read the planes (event inputs_read), and the
// setter returns once the host array has been read: the reference's setters
// copy at call time too (graph_cut.hpp:284-285, 298-299).  Device-pointer
// setters copy device to device on the solve stream.
static int ensure_lin(Pool& p, bool bwd) {
  if (!p.lin) {
    CGC_CUDA(cudaMalloc(&p.lin, 5 * (size_t)p.sumN * 4));
    CGC_CUDA(cudaStreamCreateWithFlags(&p.copy_stream, cudaStreamNonBlocking));
  }
  if (bwd && !p.lin_bwd) CGC_CUDA(cudaMalloc(&p.lin_bwd, 3 * (size_t)p.sumN * 4));
  return CGC_OK;
}

static int copy_plane(Pool& p, int32_t* dst, const int32_t* src, int64_t N, bool host) {
  if (host) {
    CGC_CUDA(cudaStreamWaitEvent(p.copy_stream, p.inputs_read, 0));  // no-op before the first record
    CGC_CUDA(cudaMemcpyAsync(dst, src, N * 4, cudaMemcpyHostToDevice, p.copy_stream));
  } else {
    CGC_CUDA(cudaMemcpyAsync(dst, src, N * 4, cudaMemcpyDeviceToDevice, p.stream));
  }
  return CGC_OK;
}

int pool_put_tlinks(Pool& p, int inst, const int32_t* capS, const int32_t* capT, bool host) {
  if (inst < 0 || inst >= p.ninst || !capS || !capT) return fail(CGC_ERR_ARG, "set_tlinks: bad arguments");
  const InstGeo& G = p.geo[inst];
  const int64_t N = (int64_t)G.X * G.Y * G.Z;
  if (int rc = ensure_lin(p, false)) return rc;
  int32_t* s = p.lin + p.voff[inst];
  int32_t* c = p.lin + p.sumN + p.voff[inst];
  if (int rc = copy_plane(p, s, capS, N, host)) return rc;
  if (int rc = copy_plane(p, c, capT, N, host)) return rc;
  if (host) CGC_CUDA(cudaStreamSynchronize(p.copy_stream));
  p.host_in[8 * (size_t)inst] = s;
  p.host_in[8 * (size_t)inst + 1] = c;
  p.uploaded[inst] |= 1u;
  p.solved = false;
  p.seg_valid = false;
  return ok();
}

int pool_put_nlinks(Pool& p, int inst, int axis, const int32_t* fwd, const int32_t* bwd, bool host) {
  if (inst < 0 || inst >= p.ninst || axis < 0 || axis > 2 || !fwd || !bwd)
    return fail(CGC_ERR_ARG, "set_nlinks: bad arguments");
  const InstGeo& G = p.geo[inst];
  const int64_t N = (int64_t)G.X * G.Y * G.Z;
  const bool same = bwd == fwd;  // symmetric weights: one plane
  if (int rc = ensure_lin(p, !same)) return rc;
  int32_t* f = p.lin + (2 + axis) * p.sumN + p.voff[inst];
  int32_t* b = same ? f : p.lin_bwd + axis * p.sumN + p.voff[inst];
  if (int rc = copy_plane(p, f, fwd, N, host)) return rc;
  if (!same)
    if (int rc = copy_plane(p, b, bwd, N, host)) return rc;
  if (host) CGC_CUDA(cudaStreamSynchronize(p.copy_stream));
  p.host_in[8 * (size_t)inst + 2 + axis] = f;
  p.host_in[8 * (size_t)inst + 5 + axis] = b;
  p.uploaded[inst] |= 2u << axis;
  p.solved = false;
  p.seg_valid = false;
  return ok();
}

cgc_options resolve_options(const cgc_options* o) {
  cgc_options r{};
  r.struct_size = sizeof(cgc_options);
  r.local_pulses = 4;
  r.sweeps_per_relabel = 8;
  r.wait_limit_us = 20 * 1000 * 1000;
  r.max_sweeps = 1 << 17;
  r.persistent = 1;
  r.region_relabels = 2;
  r.stall_sweeps = 0;
  r.ctas_per_sm = 2;
  r.relabel = 2;
  if (o) {
    if (o->local_pulses > 0) r.local_pulses = std::min(o->local_pulses, 64);
    if (o->sweeps_per_relabel > 0) r.sweeps_per_relabel = o->sweeps_per_relabel;
    if (o->wait_limit_us > 0) r.wait_limit_us = o->wait_limit_us;
    if (o->max_sweeps > 0) r.max_sweeps = o->max_sweeps;
    if (o->persistent) r.persistent = o->persistent;
    if (o->region_relabels) r.region_relabels = o->region_relabels < 0 ? 0 : std::min(o->region_relabels, 16);
    if (o->stall_sweeps) r.stall_sweeps = o->stall_sweeps < 0 ? 0 : o->stall_sweeps;
    if (o->ctas_per_sm >= 2 && o->ctas_per_sm <= 4) r.ctas_per_sm = o->ctas_per_sm;
    r.bfs_warp_min = o->bfs_warp_min > 0 ? o->bfs_warp_min : 0;
    r.exclusive = o->exclusive > 0 ? 1 : 0;
    if (o->relabel == 1 || o->relabel == 2) r.relabel = o->relabel;
    r.learned = (o->learned == 2 || o->learned == 3) ? o->learned : (o->learned > 0 ? 1 : 0);
    r.trace_cycles = o->trace_cycles > 0 ? std::min(o->trace_cycles, 64) : 0;
  }
  return r;
}

uint64_t wait_limit_ns(const cgc_options& o) {
  return (uint64_t)(o.wait_limit_us > 0 ? o.wait_limit_us : 20 * 1000 * 1000) * 1000ull;
}

// Parameters of the persistent solve kernel from resolved options.
SolveParams solve_params(const cgc_options& o) {
  SolveParams prm;
  prm.L = o.local_pulses;
  prm.R = o.region_relabels;
  prm.K = o.sweeps_per_relabel;
  prm.stall = o.stall_sweeps;
  prm.learned = o.learned;
  prm.trace_cycles = o.trace_cycles > 0 ? o.trace_cycles : 0;
  prm.max_sweeps = (int64_t)o.max_sweeps;
  prm.limit_ns = wait_limit_ns(o);
  prm.bfs_warp_min = o.ctas_per_sm >= 3 ? o.bfs_warp_min : 0;  // kernels k_solve3w / k_solve4w
  prm.exclusive = o.exclusive ? 1 : 0;
  prm.incremental = o.relabel == 2 ? 1 : 0;
  return prm;
}

// host-driven BFS (or reachability) pass; returns rounds executed
template <bool REACH>
static int host_bfs(Pool& p, uint32_t& id, int64_t& rounds) {
  DevPool& d = p.dp;
  int32_t* bl[3] = {d.lists, d.lists + d.T, d.lists + 2 * d.T};
  CGC_CUDA(cudaMemsetAsync(d.cnt + C_BFS0, 0, 3 * 4, p.stream));
  const int gi = std::min<int>(d.T, p.sms * 8);
  if (REACH) { k_reach_init<<<gi, 512, 0, p.stream>>>(d, id, bl[0], d.cnt + C_BFS0); note_launch(); }
  else {
    k_bfs_init<<<gi, 512, 0, p.stream>>>(d); note_launch();
    k_bfs_queue<<<(d.T + 255) / 256, 256, 0, p.stream>>>(d, id, bl[0], d.cnt + C_BFS0); note_launch();
  }
  CGC_CUDA(cudaGetLastError());
  for (int k = 0;; ++k) {
    CGC_CUDA(cudaMemcpyAsync(p.pinned_cnt, d.cnt + C_BFS0 + k % 3, 4, cudaMemcpyDeviceToHost, p.stream));
    CGC_CUDA(cudaStreamSynchronize(p.stream));
    const int n = p.pinned_cnt[0];
    if (n == 0) { id += k + 1; break; }
    CGC_CUDA(cudaMemsetAsync(d.cnt + C_BFS0 + (k + 1) % 3, 0, 4, p.stream));
    const int gb = std::min(n, p.sweep_blocks);
    if (REACH) { k_reach_round<<<gb, 512, 0, p.stream>>>(d, bl[k % 3], d.cnt + C_BFS0 + k % 3, id + k + 1, bl[(k + 1) % 3], d.cnt + C_BFS0 + (k + 1) % 3); note_launch(); }
    else { k_bfs_round<<<gb, 512, 0, p.stream>>>(d, bl[k % 3], d.cnt + C_BFS0 + k % 3, id + k + 1, bl[(k + 1) % 3], d.cnt + C_BFS0 + (k + 1) % 3); note_launch(); }
    CGC_CUDA(cudaGetLastError());
    ++rounds;
  }
  return CGC_OK;
}

// Buffers of the host-path outputs: both cut sets of every instance (1/0
// bytes, linear order) and the device table of their addresses.
static int ensure_segbuf(Pool& p) {
  if (p.segbuf) return CGC_OK;
  CGC_CUDA(cudaMalloc(&p.segbuf, 2 * (size_t)p.sumN));
  CGC_CUDA(cudaMalloc(&p.d_segtab, 2 * (size_t)p.ninst * sizeof(uint8_t*)));
  std::vector<uint8_t*> tab(2 * (size_t)p.ninst);
  for (int i = 0; i < p.ninst; ++i) {
    tab[2 * i] = p.segbuf + p.voff[i];               // source side
    tab[2 * i + 1] = p.segbuf + p.sumN + p.voff[i];  // sink side
  }
  CGC_CUDA(cudaMemcpy(p.d_segtab, tab.data(), tab.size() * sizeof(uint8_t*), cudaMemcpyHostToDevice));
  return CGC_OK;
}

// Enqueues one solve of the set_* inputs on p.stream: fused upload and
// preflow, the solve, and both cut sets of every instance into segbuf.  With
// the persistent solve (the default) nothing synchronises the host, so the
// next grid's host uploads can run while this one solves; the host-driven
// schedule (persistent = -1) runs its loop here.
int pool_solve_async(Pool& p, const cgc_options* opts) {
  if (p.pending) return fail(CGC_ERR_STATE, "maxflow: the previous solve of this handle was not waited for");
  const cgc_options o = resolve_options(opts);
  DevPool& d = p.dp;
  for (int i = 0; i < p.ninst; ++i)
    if (!(p.uploaded[i] & 1u)) return fail(CGC_ERR_STATE, "maxflow: set_tlinks was not called since the last solve");
  // axes not set since the last solve have zero capacity
  std::vector<const int32_t*> in = p.host_in;
  for (int i = 0; i < p.ninst; ++i)
    for (int a = 0; a < 3; ++a)
      if (!(p.uploaded[i] & (2u << a))) in[8 * (size_t)i + 2 + a] = in[8 * (size_t)i + 5 + a] = nullptr;
  const SolveParams prm = solve_params(o);
  if (o.persistent > 0 && (prm.learned || prm.trace_cycles))  // buffers and weights before anything is queued
    if (int rc = ensure_sched(p, prm.learned != 0, prm.trace_cycles)) return rc;
  if (int rc = ensure_segbuf(p)) return rc;
  if (p.ninst > 1) {
    if (!p.d_host_in) CGC_CUDA(cudaMalloc(&p.d_host_in, 8 * (size_t)p.ninst * sizeof(int32_t*)));
    // pageable source: the table is staged before the call returns
    CGC_CUDA(cudaMemcpyAsync(p.d_host_in, in.data(), in.size() * sizeof(int32_t*), cudaMemcpyHostToDevice, p.stream));
  }
  p.launches0 = g_launches.load();
  CGC_CUDA(cudaEventRecord(p.ev[0], p.stream));
  CGC_CUDA(cudaMemsetAsync(d.flow, 0, (size_t)p.ninst * 8, p.stream));
  CGC_CUDA(cudaMemsetAsync(d.stats, 0, S_NSTATS * 8, p.stream));
  CGC_CUDA(cudaMemsetAsync(d.err, 0, 4, p.stream));
  CGC_CUDA(cudaMemsetAsync(d.bar, 0, 8, p.stream));
  CGC_CUDA(cudaMemsetAsync(d.stamp_bfs, 0, (size_t)d.T * 4, p.stream));
  CGC_CUDA(cudaMemsetAsync(d.stamp_sw, 0, 2 * (size_t)d.T * 4, p.stream));
  CGC_CUDA(cudaMemsetAsync(d.stamp_inc, 0, (size_t)d.T * 4, p.stream));
  if (p.ninst == 1) {
    InputPlanes ip;
    for (int k = 0; k < 8; ++k) ip.p[k] = in[k];
    k_put_one<<<d.T, 128, 0, p.stream>>>(d, ip);
  } else {
    k_put_all<<<d.T, 128, 0, p.stream>>>(d, p.d_host_in);
  }
  note_launch();
  CGC_CUDA(cudaGetLastError());
  CGC_CUDA(cudaEventRecord(p.inputs_read, p.stream));  // the setters may overwrite the planes from here on
  // the inputs are consumed: another solve needs new set_* calls
  for (auto& u : p.uploaded) u = 0;
  p.solved = false;
  p.seg_valid = false;
  p.pending = true;
  p.pending_persistent = o.persistent;

  int rc = CGC_OK;
  if (o.persistent > 0) {
    CGC_CUDA(cudaEventRecord(p.ev[2], p.stream));
    rc = launch_solve(p, o, d, prm, p.stream);
    CGC_CUDA(cudaEventRecord(p.ev[3], p.stream));
  } else {
    // the host loop reads counters back every round; a preparation error
    // (overflowing capacities) stops it before it starts
    rc = check_device_error(p, "maxflow");
    CGC_CUDA(cudaEventRecord(p.ev[2], p.stream));
    int64_t sweeps = 0, relabels = 0, rounds = 0;
    uint32_t id = 1;
    int32_t* sl = d.lists + 3 * d.T;
    while (!rc) {
      rc = host_bfs<false>(p, id, rounds);
      if (rc) break;
      ++relabels;
      CGC_CUDA(cudaMemsetAsync(d.cnt + C_SW0, 0, 8, p.stream));
      k_compact<<<(d.T + 255) / 256, 256, 0, p.stream>>>(d, 0, sl, d.cnt + C_SW0); note_launch();
      k_compact<<<(d.T + 255) / 256, 256, 0, p.stream>>>(d, 1, sl + d.T, d.cnt + C_SW0 + 1); note_launch();
      CGC_CUDA(cudaMemcpyAsync(p.pinned_cnt, d.cnt + C_SW0, 8, cudaMemcpyDeviceToHost, p.stream));
      CGC_CUDA(cudaStreamSynchronize(p.stream));
      if (p.pinned_cnt[0] + p.pinned_cnt[1] == 0) break;
      if (sweeps >= o.max_sweeps) { rc = fail(CGC_ERR_NOT_CONVERGED, "maxflow: max_sweeps reached"); break; }
      for (int j = 0; j < 2 * o.sweeps_per_relabel; ++j) {
        const int par = j & 1;
        if (j > 0) {
          CGC_CUDA(cudaMemsetAsync(d.cnt + C_SW0 + par, 0, 4, p.stream));
          k_compact<<<(d.T + 255) / 256, 256, 0, p.stream>>>(d, par, sl + par * d.T, d.cnt + C_SW0 + par); note_launch();
        }
        k_sweep_list<<<p.sweep_blocks, 512, 0, p.stream>>>(d, sl + par * d.T, d.cnt + C_SW0 + par, o.local_pulses, o.region_relabels); note_launch();
        CGC_CUDA(cudaGetLastError());
        ++sweeps;
      }
    }
    if (!rc) rc = host_bfs<true>(p, id, rounds);
    CGC_CUDA(cudaEventRecord(p.ev[3], p.stream));
    p.host_counts[0] = sweeps;
    p.host_counts[1] = relabels;
    p.host_counts[2] = rounds;
  }
  if (!rc) {
    const unsigned gx = (unsigned)std::min<int64_t>(std::max<int64_t>((p.maxN + 32767) / 32768, 1), 4096);
    k_seg_all<<<dim3(gx, (unsigned)std::min(p.ninst, 65535)), 256, 0, p.stream>>>(d, p.d_segtab);
    note_launch();
    CGC_CUDA(cudaGetLastError());
  }
  CGC_CUDA(cudaEventRecord(p.ev[1], p.stream));
  if (rc) {
    // nothing to wait for: leave the stream idle and report now
    cudaStreamSynchronize(p.stream);
    p.pending = false;
    return rc;
  }
  return ok();
}

// Waits for the solve enqueued by pool_solve_async; reports device errors and
// reads the flows and statistics.
int pool_solve_wait(Pool& p) {
  if (!p.pending) return fail(CGC_ERR_STATE, "wait: no solve was enqueued");
  p.pending = false;
  CGC_CUDA(cudaEventSynchronize(p.ev[1]));
  if (int rc = check_device_error(p, "maxflow")) return rc;
  float ms = 0.f, kms = 0.f;
  cudaEventElapsedTime(&ms, p.ev[0], p.ev[1]);
  cudaEventElapsedTime(&kms, p.ev[2], p.ev[3]);
  unsigned long long stats[S_NSTATS];
  CGC_CUDA(cudaMemcpyAsync(stats, p.dp.stats, sizeof(stats), cudaMemcpyDeviceToHost, p.stream));
  CGC_CUDA(cudaMemcpyAsync(p.flows.data(), p.dp.flow, (size_t)p.ninst * 8, cudaMemcpyDeviceToHost, p.stream));
  CGC_CUDA(cudaStreamSynchronize(p.stream));
  std::memset(&p.st, 0, sizeof(p.st));
  for (int64_t f : p.flows) p.st.flow += f;
  if (p.pending_persistent > 0) {
    p.st.sweeps = (int64_t)stats[S_SWEEPS];
    p.st.global_relabels = (int64_t)stats[S_RELABELS];
    p.st.bfs_rounds = (int64_t)stats[S_ROUNDS];
  } else {
    p.st.sweeps = p.host_counts[0];
    p.st.global_relabels = p.host_counts[1];
    p.st.bfs_rounds = p.host_counts[2];
  }
  p.st.tiles_swept = (int64_t)stats[S_TILES_SWEPT];
  p.st.tiles_relabelled = (int64_t)stats[S_TILES_BFS];
  p.st.tiles_checked = (int64_t)stats[S_TILES_CHECK];
  p.st.pulses = (int64_t)stats[S_PULSES];
  p.st.solve_ms = ms;
  p.st.kernel_ms = kms;
  p.st.launches = g_launches.load() - p.launches0;
  p.st.bfs_ms = 1e-6 * (double)stats[S_NS_BFS];
  p.st.sweep_ms = 1e-6 * (double)stats[S_NS_SWEEP];
  p.st.reach_ms = 1e-6 * (double)stats[S_NS_REACH];
  p.st.sched_ms = 1e-6 * (double)stats[S_NS_SCHED];
  p.solved = true;
  p.seg_valid = true;
  return ok();
}

int pool_solve(Pool& p, const cgc_options* opts) {
  if (int rc = pool_solve_async(p, opts)) return rc;
  return pool_solve_wait(p);
}

int pool_segments(Pool& p, int inst, int which, uint8_t* out, uint8_t mask, uint8_t bg, bool host) {
  if (inst < 0 || inst >= p.ninst || !out || (which != CGC_SEG_SINK_REACH && which != CGC_SEG_SOURCE_MIN))
    return fail(CGC_ERR_ARG, "get_segments: bad arguments");
  if (p.pending) return fail(CGC_ERR_STATE, "get_segments: wait for the solve first");
  if (!p.solved) return fail(CGC_ERR_STATE, "get_segments: call maxflow first");
  const InstGeo& G = p.geo[inst];
  const int64_t N = (int64_t)G.X * G.Y * G.Z;
  if ((host || !p.seg_valid || mask != 1 || bg != 0) && !p.segtmp) CGC_CUDA(cudaMalloc(&p.segtmp, p.maxN));
  const unsigned blocks = (unsigned)std::min<int64_t>(std::max<int64_t>((N + 4095) / 4096, 1), 8 * (int64_t)p.sms);
  const uint8_t* src = nullptr;  // device bytes to copy to `out` as they are
  if (p.seg_valid) {
    // the host-path solve wrote both sets as 1/0 bytes
    const uint8_t* set = p.segbuf + (which == CGC_SEG_SOURCE_MIN ? 0 : p.sumN) + p.voff[inst];
    if (mask == 1 && bg == 0) {
      src = set;
    } else {
      uint8_t* dst = host ? p.segtmp : out;
      k_mask_remap<<<blocks, 256, 0, p.stream>>>(set, dst, N, mask, bg); note_launch();
      src = host ? p.segtmp : nullptr;
    }
  } else {
    // after a device-resident solve: from the solver state
    uint8_t* dst = host ? p.segtmp : out;
    k_segments_lin<<<blocks, 256, 0, p.stream>>>(p.dp, inst, which, dst, mask, bg); note_launch();
    src = host ? p.segtmp : nullptr;
  }
  CGC_CUDA(cudaGetLastError());
  if (src) CGC_CUDA(cudaMemcpyAsync(out, src, N, host ? cudaMemcpyDeviceToHost : cudaMemcpyDeviceToDevice, p.stream));
  CGC_CUDA(cudaStreamSynchronize(p.stream));
  return ok();
}

int pool_residuals(Pool& p, int inst, int32_t* const res[6], int32_t* resT, int32_t* excess) {
  if (inst < 0 || inst >= p.ninst) return fail(CGC_ERR_ARG, "get_residuals: bad instance");
  if (p.pending) return fail(CGC_ERR_STATE, "get_residuals: wait for the solve first");
  if (!p.solved) return fail(CGC_ERR_STATE, "get_residuals: call maxflow first");
  const InstGeo& G = p.geo[inst];
  const int64_t N = (int64_t)G.X * G.Y * G.Z;
  if (!p.resid) CGC_CUDA(cudaMalloc(&p.resid, (size_t)p.maxN * 4));
  const int blocks = (int)std::min<int64_t>((N + 255) / 256, 65535);
  auto one = [&](const int32_t* plane, int32_t* out) -> int {
    if (!out) return CGC_OK;
    k_unpermute<<<blocks, 256, 0, p.stream>>>(p.dp, inst, plane, p.resid); note_launch();
    CGC_CUDA(cudaGetLastError());
    CGC_CUDA(cudaMemcpyAsync(out, p.resid, N * 4, cudaMemcpyDeviceToHost, p.stream));
    CGC_CUDA(cudaStreamSynchronize(p.stream));
    return CGC_OK;
  };
  int rc;
  if (res)
    for (int d = 0; d < 6; ++d)
      if ((rc = one(p.dp.r + d * p.Np, res[d]))) return rc;
  if ((rc = one(p.dp.rT, resT))) return rc;
  if ((rc = one(p.dp.e, excess))) return rc;
  return ok();
}

// Distance labels of the last solve in linear order (INT32_MIN where the
// sink cannot be reached).
int pool_labels(Pool& p, int inst, int32_t* labels) {
  if (inst < 0 || inst >= p.ninst || !labels) return fail(CGC_ERR_ARG, "get_labels: bad arguments");
  if (p.pending) return fail(CGC_ERR_STATE, "get_labels: wait for the solve first");
  if (!p.solved) return fail(CGC_ERR_STATE, "get_labels: call maxflow first");
  const InstGeo& G = p.geo[inst];
  const int64_t N = (int64_t)G.X * G.Y * G.Z;
  if (!p.resid) CGC_CUDA(cudaMalloc(&p.resid, (size_t)p.maxN * 4));
  k_unpermute<<<(int)std::min<int64_t>((N + 255) / 256, 65535), 256, 0, p.stream>>>(p.dp, inst, p.dp.h, p.resid);
  note_launch();
  CGC_CUDA(cudaGetLastError());
  CGC_CUDA(cudaMemcpyAsync(labels, p.resid, N * 4, cudaMemcpyDeviceToHost, p.stream));
  CGC_CUDA(cudaStreamSynchronize(p.stream));
  for (int64_t v = 0; v < N; ++v)
    if (labels[v] >= INF) labels[v] = INT32_MIN;
  return ok();
}

int pool_trace(Pool& p, int64_t* out, int32_t cap, int32_t* count) {
  if (!p.solved) return fail(CGC_ERR_STATE, "trace: call maxflow first");
  unsigned long long n = 0;
  CGC_CUDA(cudaMemcpy(&n, p.dp.stats + S_TRACE_N, 8, cudaMemcpyDeviceToHost));
  *count = (int32_t)n;
  if (out && cap > 0) {
    const int64_t m = std::min<int64_t>((int64_t)n, cap);
    CGC_CUDA(cudaMemcpy(out, p.dp.trace, (size_t)m * 16, cudaMemcpyDeviceToHost));
  }
  return ok();
}

}  // namespace cgc

// ===========================================================================
// C ABI
// ===========================================================================
using cgc::Pool;

struct cgc_grid { Pool* p; };
struct cgc_batch { Pool* p; };

extern "C" {

const char* cgc_last_error(void) { return cgc::g_last_error.c_str(); }
const char* cgc_version(void) { return "cgc 0.1 (sm_100a)"; }
int64_t cgc_launch_count(void) { return (int64_t)cgc::g_launches.load(); }

int cgc_init(int device) {
  int n = 0;
  cudaError_t e = cudaGetDeviceCount(&n);
  if (e != cudaSuccess || n == 0) return cgc::fail(CGC_ERR_NO_DEVICE, "cgc_init: no CUDA device");
  if (device < 0 || device >= n) return cgc::fail(CGC_ERR_ARG, "cgc_init: bad device index");
  CGC_CUDA(cudaSetDevice(device));
  CGC_CUDA(cudaFree(nullptr));
  return cgc::ok();
}

int cgc_grid_create(int32_t X, int32_t Y, int32_t Z, void* stream, cgc_grid** out) {
  if (!out) return cgc::fail(CGC_ERR_ARG, "cgc_grid_create: null output");
  int32_t ext[3] = {X, Y, Z};
  Pool* p = nullptr;
  int rc = cgc::pool_create(1, ext, stream, &p);
  if (rc) return rc;
  *out = new cgc_grid{p};
  return cgc::ok();
}
int cgc_grid_destroy(cgc_grid* g) {
  if (!g) return cgc::ok();
  delete g->p;
  delete g;
  return cgc::ok();
}
int cgc_grid_set_tlinks(cgc_grid* g, const int32_t* capS, const int32_t* capT) {
  if (!g) return cgc::fail(CGC_ERR_ARG, "null grid");
  return cgc::pool_put_tlinks(*g->p, 0, capS, capT, true);
}
int cgc_grid_set_nlinks(cgc_grid* g, int axis, const int32_t* fwd, const int32_t* bwd) {
  if (!g) return cgc::fail(CGC_ERR_ARG, "null grid");
  return cgc::pool_put_nlinks(*g->p, 0, axis, fwd, bwd, true);
}
int cgc_grid_set_tlinks_device(cgc_grid* g, const int32_t* capS, const int32_t* capT) {
  if (!g) return cgc::fail(CGC_ERR_ARG, "null grid");
  return cgc::pool_put_tlinks(*g->p, 0, capS, capT, false);
}
int cgc_grid_set_nlinks_device(cgc_grid* g, int axis, const int32_t* fwd, const int32_t* bwd) {
  if (!g) return cgc::fail(CGC_ERR_ARG, "null grid");
  return cgc::pool_put_nlinks(*g->p, 0, axis, fwd, bwd, false);
}
int cgc_grid_maxflow(cgc_grid* g, const cgc_options* opts, int64_t* flow) {
  if (!g) return cgc::fail(CGC_ERR_ARG, "null grid");
  int rc = cgc::pool_solve(*g->p, opts);
  if (rc) return rc;
  if (flow) *flow = g->p->flows[0];
  return cgc::ok();
}
int cgc_grid_maxflow_async(cgc_grid* g, const cgc_options* opts) {
  if (!g) return cgc::fail(CGC_ERR_ARG, "null grid");
  return cgc::pool_solve_async(*g->p, opts);
}
int cgc_grid_wait(cgc_grid* g, int64_t* flow) {
  if (!g) return cgc::fail(CGC_ERR_ARG, "null grid");
  int rc = cgc::pool_solve_wait(*g->p);
  if (rc) return rc;
  if (flow) *flow = g->p->flows[0];
  return cgc::ok();
}
int cgc_grid_get_segments(cgc_grid* g, int which, uint8_t* out, uint8_t mask, uint8_t background) {
  if (!g) return cgc::fail(CGC_ERR_ARG, "null grid");
  return cgc::pool_segments(*g->p, 0, which, out, mask, background, true);
}
int cgc_grid_get_segments_device(cgc_grid* g, int which, uint8_t* out, uint8_t mask, uint8_t background) {
  if (!g) return cgc::fail(CGC_ERR_ARG, "null grid");
  return cgc::pool_segments(*g->p, 0, which, out, mask, background, false);
}
int cgc_grid_get_labels(cgc_grid* g, int32_t* labels) {
  if (!g) return cgc::fail(CGC_ERR_ARG, "null grid");
  return cgc::pool_labels(*g->p, 0, labels);
}
int cgc_grid_get_residuals(cgc_grid* g, int32_t* const res[6], int32_t* resT, int32_t* excess) {
  if (!g) return cgc::fail(CGC_ERR_ARG, "null grid");
  return cgc::pool_residuals(*g->p, 0, res, resT, excess);
}
int cgc_grid_trace(cgc_grid* g, int64_t* out, int32_t cap, int32_t* count) {
  if (!g || !count) return cgc::fail(CGC_ERR_ARG, "null argument");
  return cgc::pool_trace(*g->p, out, cap, count);
}
int cgc_batch_trace(cgc_batch* b, int64_t* out, int32_t cap, int32_t* count) {
  if (!b || !count) return cgc::fail(CGC_ERR_ARG, "null argument");
  return cgc::pool_trace(*b->p, out, cap, count);
}
int cgc_grid_sched_trace(cgc_grid* g, uint16_t* feat, uint8_t* pulses, uint8_t* sink, int32_t max_cycles,
                         int32_t* cycles) {
  if (!g || !cycles) return cgc::fail(CGC_ERR_ARG, "null argument");
  return cgc::pool_sched_trace(*g->p, feat, pulses, sink, max_cycles, cycles);
}
int cgc_grid_stats(cgc_grid* g, cgc_stats* out) {
  if (!g || !out) return cgc::fail(CGC_ERR_ARG, "null argument");
  *out = g->p->st;
  return cgc::ok();
}

int cgc_batch_create(int32_t count, const int32_t* extents, void* stream, cgc_batch** out) {
  if (!out) return cgc::fail(CGC_ERR_ARG, "cgc_batch_create: null output");
  Pool* p = nullptr;
  int rc = cgc::pool_create(count, extents, stream, &p);
  if (rc) return rc;
  *out = new cgc_batch{p};
  return cgc::ok();
}
int cgc_batch_destroy(cgc_batch* b) {
  if (!b) return cgc::ok();
  delete b->p;
  delete b;
  return cgc::ok();
}
int cgc_batch_set_tlinks(cgc_batch* b, int32_t i, const int32_t* capS, const int32_t* capT) {
  if (!b) return cgc::fail(CGC_ERR_ARG, "null batch");
  return cgc::pool_put_tlinks(*b->p, i, capS, capT, true);
}
int cgc_batch_set_nlinks(cgc_batch* b, int32_t i, int axis, const int32_t* fwd, const int32_t* bwd) {
  if (!b) return cgc::fail(CGC_ERR_ARG, "null batch");
  return cgc::pool_put_nlinks(*b->p, i, axis, fwd, bwd, true);
}
int cgc_batch_maxflow(cgc_batch* b, const cgc_options* opts, int64_t* flows) {
  if (!b) return cgc::fail(CGC_ERR_ARG, "null batch");
  int rc = cgc::pool_solve(*b->p, opts);
  if (rc) return rc;
  if (flows) std::memcpy(flows, b->p->flows.data(), b->p->flows.size() * 8);
  return cgc::ok();
}
int cgc_batch_get_segments(cgc_batch* b, int32_t i, int which, uint8_t* out, uint8_t mask, uint8_t background) {
  if (!b) return cgc::fail(CGC_ERR_ARG, "null batch");
  return cgc::pool_segments(*b->p, i, which, out, mask, background, true);
}
int cgc_batch_stats(cgc_batch* b, cgc_stats* out) {
  if (!b || !out) return cgc::fail(CGC_ERR_ARG, "null argument");
  *out = b->p->st;
  return cgc::ok();
}

}  // extern "C"
