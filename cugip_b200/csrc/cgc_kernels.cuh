// Tile routines and kernels of the grid push-relabel engine (sm_100a).
//
// One CTA of 512 threads owns one 8x8x8 tile at a time; thread l owns voxel
// (l&7, (l>>3)&7, l>>6).  The voxel's own state (excess, height, sink
// residual, six out-residuals) lives in registers; heights of the tile plus a
// one-voxel halo live in shared memory so that neighbours can be read.
//
// Push sweep (replaces the per-level push of
// include/cugip/advanced_operations/detail/graph_cut_push.hpp:160-186,236-318,
// 461-482).  A visit runs up to L synchronous pulses of the Goldberg-Tarjan
// parallel push-relabel inside the tile: every active voxel (e>0, h<INF)
// pushes to the sink if h==1 and along every admissible residual edge
// (h(u)==h(v)-1), then every voxel that is still active and has no
// admissible edge relabels to 1+min over its residual neighbours.  Labels are
// fixed during a push step and relabels read the old labels, so the labelling
// stays valid.  Under the parity schedule only tiles with (tx+ty+tz) of one
// parity run at a time; face neighbours always have the other parity, so the
// halo heights are exact and the tile's pushes across a face (int32 atomics on
// the neighbour's excess, plain adds on the neighbour's reverse residual,
// which has a single writer) are ordinary valid pushes.
//
// Global relabel (replaces the level-synchronous BFS of
// detail/graph_cut_relabeling.hpp:47-112,651-751,1004-1029).  Exact BFS
// distance to the sink over reverse residual edges, computed by tile-local
// Bellman-Ford relaxation to a fixed point in shared memory; a tile whose face
// heights dropped re-queues its face neighbours.  Vertices the BFS does not
// reach keep INF, which is the gap heuristic.
//
// Exact sink flow.  Pushes to the sink are capped by the sink residual (the
// reference moves all excess of any sink-adjacent vertex,
// detail/graph_cut_push.hpp:26-41); the flow is accumulated in int64.
#pragma once
#include <cuda_runtime.h>
#include "cgc.h"
#include "cgc_device.cuh"

namespace cgc {

__device__ __forceinline__ int halo_index(int x, int y, int z) { return (z + 1) * 100 + (y + 1) * 10 + (x + 1); }

// offsets of the 6 neighbours in the halo array and inside a tile
__device__ __forceinline__ int hoff(int d) {
  return d == PX ? 1 : d == MX ? -1 : d == PY ? 10 : d == MY ? -10 : d == PZ ? 100 : -100;
}
__device__ __forceinline__ int loff(int d) {
  return d == PX ? 1 : d == MX ? -1 : d == PY ? 8 : d == MY ? -8 : d == PZ ? 64 : -64;
}
// local index in the neighbouring tile when stepping out of the tile along d
__device__ __forceinline__ int xoff(int d) {
  return d == PX ? -7 : d == MX ? 7 : d == PY ? -56 : d == MY ? 56 : d == PZ ? -448 : 448;
}
__device__ __forceinline__ bool inside(int d, int x, int y, int z) {
  return d == PX ? x < 7 : d == MX ? x > 0 : d == PY ? y < 7 : d == MY ? y > 0 : d == PZ ? z < 7 : z > 0;
}
// entry of voxel (x,y,z) on face d in the order of for_halo_entry (a + 8b)
__device__ __forceinline__ int face_entry(int d, int x, int y, int z) {
  return (d == PX || d == MX) ? y + 8 * z : (d == PY || d == MY) ? x + 8 * z : x + 8 * y;
}
// bit mask of the faces of the tile the voxel lies on
__device__ __forceinline__ int face_bits(int x, int y, int z) {
  return ((x == 7) << PX) | ((x == 0) << MX) | ((y == 7) << PY) | ((y == 0) << MY) | ((z == 7) << PZ) | ((z == 0) << MZ);
}

__device__ __forceinline__ uint64_t globaltimer_ns() {
  uint64_t t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}

__device__ __forceinline__ void raise_error(const DevPool& P, int code) { atomicCAS(P.err, 0, code); }

// Bounds-checked build (-DCGC_BOUNDS_CHECK; cugip_b200/build.py --bounds-check
// builds libcgc_bounds.so): every tile, neighbour-tile and worklist index the
// tile routines compute is checked against its array.  An index out of range
// records CGC_ERR_ARG in the error word (the first one also its value in
// stats[S_BOUND_AT]) and the access is skipped; nothing traps.  The product
// build compiles the checks out.
#ifdef CGC_BOUNDS_CHECK
static __device__ __noinline__ bool bound_fail(const DevPool& P, long long i) {
  if (atomicCAS(P.err, 0, CGC_ERR_ARG) == 0) P.stats[S_BOUND_AT] = (unsigned long long)i;
  return false;
}
#define CGC_IN_BOUNDS(P, i, lim) \
  ((long long)(i) >= 0 && (long long)(i) < (long long)(lim) ? true : ::cgc::bound_fail((P), (long long)(i)))
#else
#define CGC_IN_BOUNDS(P, i, lim) true
#endif

// Face f of the halo: thread k in [0,64) of face f writes halo entry (a,b) of
// that face from the neighbouring tile (INF outside the grid).
template <typename F>
__device__ __forceinline__ void for_halo_entry(int l, F&& fn) {
  if (l < 384) {
    const int f = l >> 6, k = l & 63, a = k & 7, b = k >> 3;
    int hi, src;
    switch (f) {
      case PX: hi = (b + 1) * 100 + (a + 1) * 10 + 9; src = 8 * a + 64 * b; break;
      case MX: hi = (b + 1) * 100 + (a + 1) * 10;     src = 7 + 8 * a + 64 * b; break;
      case PY: hi = (b + 1) * 100 + 90 + (a + 1);     src = a + 64 * b; break;
      case MY: hi = (b + 1) * 100 + (a + 1);          src = a + 56 + 64 * b; break;
      case PZ: hi = 900 + (b + 1) * 10 + (a + 1);     src = a + 8 * b; break;
      default: hi = (b + 1) * 10 + (a + 1);           src = a + 8 * b + 448; break;
    }
    fn(f, hi, src);
  }
}

__device__ __forceinline__ void load_halo_heights(const DevPool& P, int t, int (*sh)[HALO]) {
  for_halo_entry(threadIdx.x, [&](int f, int hi, int src) {
    const int nt = __ldcg(P.nbr + f * P.T + t);
    const int v = (nt >= 0 && CGC_IN_BOUNDS(P, nt, P.T)) ? __ldcg(P.h + (int64_t)nt * TV + src) : INF;
    sh[0][hi] = v;
    sh[1][hi] = v;
  });
}

// warp-aggregated append of `pred` items to list/cnt
// (worklists hold at most T entries: stamps let a tile in once per list)
__device__ __forceinline__ void warp_append(const DevPool& P, bool pred, int32_t item, int32_t* list, int32_t* cnt) {
  const unsigned mask = __ballot_sync(0xffffffffu, pred);
  if (!mask) return;
  const int lane = threadIdx.x & 31;
  const int leader = __ffs(mask) - 1;
  int base = 0;
  if (lane == leader) base = atomicAdd(cnt, __popc(mask));
  base = __shfl_sync(0xffffffffu, base, leader);
  const int k = base + __popc(mask & ((1u << lane) - 1));
  if (pred && CGC_IN_BOUNDS(P, k, P.T)) list[k] = item;
}

__device__ __forceinline__ void queue_tile(const DevPool& P, uint32_t* stamp, int t, uint32_t id, int32_t* list,
                                           int32_t* cnt) {
  if (!CGC_IN_BOUNDS(P, t, P.T)) return;
  if (atomicExch(stamp + t, id) != id) {
    const int k = atomicAdd(cnt, 1);
    if (CGC_IN_BOUNDS(P, k, P.T)) list[k] = t;
  }
}


// block-wide int64 sum (512 threads); result valid in thread 0
__device__ __forceinline__ long long block_sum64(long long v, long long* red) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
  const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
  if (lane == 0) red[w] = v;
  __syncthreads();
  long long s = 0;
  if (threadIdx.x < 32) {
    s = (lane < (int)(blockDim.x >> 5)) ? red[lane] : 0;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) s += __shfl_down_sync(0xffffffffu, s, o);
  }
  return s;
}

// Shared state is double buffered (pulse / iteration parity), so one
// pulse needs two barriers and one BFS iteration needs one.
struct SweepShared {
  int h[2][HALO];
  int out[2][6][TV];
  int facc[6][64];          // flow pushed out of the tile per face entry (for_halo_entry order)
  unsigned long long sink;  // flow delivered to the sink by this visit
  int nb[6];                // face neighbours of the tile (-1 outside)
  int flags;
  int lastout;  // last pulse (1-based) that moved flow out of the tile or into the sink
};

struct BfsShared {
  int h[2][HALO];
  int flags;
};

struct ReachShared {
  unsigned char rc[2][HALO];
  unsigned char m[HALO];
  int flags;
};

// ---------------------------------------------------------------------------
// One visit of the push sweep to tile t (L pulses at most).
//   APPEND: queue the tile itself (if still active) for sweep id_self and the
//   tiles it pushed into for sweep id_next (persistent schedule); otherwise
//   only the act[] flags are maintained (host-driven schedule).
// optional per-visit bookkeeping of the persistent schedule
struct SweepExtra {
  int32_t* sink_tiles = nullptr;  // counter of tiles that delivered sink flow in this sweep
  uint8_t* tr_pulses = nullptr;   // trace: pulses of the first visit in this cycle
  uint8_t* tr_sink = nullptr;     // trace: delivered sink flow in this cycle
};

//   stamp_q: the stamps the queued tiles get (null: P.stamp_sw).
template <bool APPEND>
__device__ inline void sweep_tile(const DevPool& P, const int t, const int L, const int R, SweepShared& S,
                           const uint32_t id_next, int32_t* list_next, int32_t* cnt_next,
                           const uint32_t id_self, int32_t* list_self, int32_t* cnt_self,
                           const SweepExtra ex = SweepExtra(), uint32_t* stamp_q = nullptr) {
  if (!stamp_q) stamp_q = P.stamp_sw;
  if (!CGC_IN_BOUNDS(P, t, P.T)) return;  // uniform over the block
  const int l = threadIdx.x;
  const int x = l & 7, y = (l >> 3) & 7, z = l >> 6;
  const int64_t g = (int64_t)t * TV + l;
  const int64_t Np = P.Np;
  int e = __ldcg(P.e + g), h = __ldcg(P.h + g), rT = __ldcg(P.rT + g);
  int r[6];
#pragma unroll
  for (int d = 0; d < 6; ++d) r[d] = __ldcg(P.r + d * Np + g);
  const int hi = halo_index(x, y, z);
  S.h[0][hi] = h;
  load_halo_heights(P, t, S.h);
  const int inst = __ldcg(P.tinst + t);
  const int hdead = P.geo[inst].hdead;
  if (l < 6) S.nb[l] = __ldcg(P.nbr + l * P.T + t);  // read by the write-back
  if (l < 384) (&S.facc[0][0])[l] = 0;
  if (l == 0) { S.flags = 0; S.lastout = 0; S.sink = 0ull; }
  __syncthreads();

  int sink = 0;
  int pulses = 0;
  int cur = 0;
  for (int round = 0;; ++round) {
    if (R > 0) {
      // Region relabel: exact distance d(v) to the sink or to the (frozen)
      // halo inside the tile, then h = max(h, d).  d is a lower bound of the
      // true distance and max(h, d) keeps every residual edge valid, so this
      // is an ordinary (multi-step) relabel; d = INF means v cannot reach the
      // sink at all.
      int dd = (rT > 0) ? 1 : INF;
      S.h[cur][hi] = dd;
      __syncthreads();
      for (int it = 0; it < 600; ++it) {  // Bellman-Ford: < 512 steps in a tile
        int mn = dd;
#pragma unroll
        for (int d = 0; d < 6; ++d)
          if (r[d] > 0) mn = min(mn, S.h[cur][hi + hoff(d)] + 1);
        S.h[cur ^ 1][hi] = mn;
        const int any = __syncthreads_or(mn < dd);
        dd = mn;
        cur ^= 1;
        if (!any) break;
      }
      int hn = max(h, dd);
      if (hn >= hdead) hn = INF;
      h = hn;
      S.h[cur][hi] = h;
      __syncthreads();
    }
    int any = 1;
    for (int p = 0; p < L; ++p) {
      int hn[6];
#pragma unroll
      for (int d = 0; d < 6; ++d) hn[d] = S.h[cur][hi + hoff(d)];
      bool moved_out = false;
      const bool act = e > 0 && h < INF;
      if (act && rT > 0 && h == 1) {
        const int dl = min(e, rT);
        e -= dl; rT -= dl; sink += dl;
        moved_out = dl > 0;
      }
      // pushes; in-tile amounts (0 included) go to S.out for the receiver,
      // amounts across a face to the face accumulator (this voxel is its
      // only writer)
#pragma unroll
      for (int d = 0; d < 6; ++d) {
        int dl = 0;
        if (act && e > 0 && r[d] > 0 && hn[d] == h - 1) {
          dl = min(e, r[d]);
          e -= dl; r[d] -= dl;
        }
        if (inside(d, x, y, z)) {
          S.out[cur][d][l] = dl;
        } else if (dl > 0) {
          S.facc[d][face_entry(d, x, y, z)] += dl;
          moved_out = true;
        }
      }
      if (moved_out) S.lastout = pulses + 1;  // same value from every writer of this pulse
      __syncthreads();
#pragma unroll
      for (int d = 0; d < 6; ++d) {
        if (inside(d, x, y, z)) {
          const int din = S.out[cur][d ^ 1][l + loff(d)];
          e += din; r[d] += din;
        }
      }
      int hnew = h;
      if (e > 0 && h < INF) {
        // the labels of the pulse start, read again from S.h[cur] (the new
        // ones go to the other buffer) rather than kept in registers
        bool adm = (rT > 0 && h == 1);
        int mn = (rT > 0) ? 0 : INF;
#pragma unroll
        for (int d = 0; d < 6; ++d) {
          if (r[d] > 0) {
            const int hd = S.h[cur][hi + hoff(d)];
            adm = adm || (hd == h - 1);
            mn = min(mn, hd);
          }
        }
        if (!adm) {
          hnew = (mn >= INF) ? INF : mn + 1;
          if (hnew >= hdead) hnew = INF;
        }
      }
      ++pulses;
      S.h[cur ^ 1][hi] = hnew;
      any = __syncthreads_or(e > 0 && hnew < INF);
      h = hnew;
      cur ^= 1;
      if (!any) break;
    }
    if (!any || round + 1 >= max(R, 1)) break;
  }

  // write back the tile
  P.e[g] = e; P.h[g] = h; P.rT[g] = rT;
  unsigned m = ((rT > 0) ? 64u : 0u) | ((e > 0) ? 128u : 0u);
#pragma unroll
  for (int d = 0; d < 6; ++d) { P.r[d * Np + g] = r[d]; m |= (r[d] > 0 ? 1u : 0u) << d; }
  P.rmask[g] = (uint8_t)m;
  // flow that left the tile: excess and reverse residual of the neighbour,
  // one face entry per thread (the pulses ended with a barrier)
  for_halo_entry(l, [&](int f, int, int src) {
    const int a = (&S.facc[0][0])[l];
    if (a > 0) {
      const int nt = S.nb[f];
      if (nt < 0) { raise_error(P, CGC_ERR_OVERFLOW); return; }  // capacity leaving the grid
      if (!CGC_IN_BOUNDS(P, nt, P.T)) return;
      const int64_t ng = (int64_t)nt * TV + src;
      atomicAdd(P.e + ng, a);
      atomicAdd(P.r + (f ^ 1) * Np + ng, a);
      atomicOr((unsigned*)(P.rmask + (ng & ~(int64_t)3)), (128u | (1u << (f ^ 1))) << (8 * (int)(ng & 3)));
      atomicOr(&S.flags, 1 << f);
    }
  });
  // sink flow of the visit: warp sums into one shared total before the barrier
  unsigned long long ws = (unsigned long long)sink;
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) ws += __shfl_down_sync(0xffffffffu, ws, o);
  if ((l & 31) == 0 && ws) atomicAdd(&S.sink, ws);
  const int still = __syncthreads_or(e > 0 && h < INF);
  const unsigned long long total = S.sink;
  if (l == 0) {
    P.act[t] = (uint8_t)(still ? 1 : 0);
    if (total) {
      atomicAdd(P.flow + inst, total);
      if (ex.sink_tiles) atomicAdd(ex.sink_tiles, 1);
      if (ex.tr_sink) ex.tr_sink[t] = 1;
    }
    // trace label: productive pulses of the tile's first visit in the cycle
    // (255 marks a visited tile that moved nothing out)
    if (ex.tr_pulses && ex.tr_pulses[t] == 0) ex.tr_pulses[t] = (uint8_t)(S.lastout > 0 ? min(S.lastout, 254) : 255);
    atomicAdd(P.stats + S_TILES_SWEPT, 1ull);
    atomicAdd(P.stats + S_PULSES, (unsigned long long)pulses);
  }
  // the tile re-queues itself from another warp than thread 0's face chain,
  // so the two dependent atomic chains overlap
  if (APPEND && l == 32 && still) queue_tile(P, stamp_q, t, id_self, list_self, cnt_self);
  if (l < 6 && ((S.flags >> l) & 1) && CGC_IN_BOUNDS(P, S.nb[l], P.T)) {
    const int nt = S.nb[l];
    P.act[nt] = 1;
    if (APPEND) queue_tile(P, stamp_q, nt, id_next, list_next, cnt_next);
  }
  __syncthreads();
}

// Upload of tile t of an instance from its linear (x-fastest) device inputs
// ip[0..7] = capS, capT, fwd x/y/z, bwd x/y/z (a null n-link pointer is
// zero), fused with the preflow initialisation: the t-links cancel
// (m = min(capS, capT) goes straight to the sink, the rest of capS becomes
// excess), the residual planes and the residual bit mask are written, and
// capacities that could overflow int32 excess or residuals raise
// CGC_ERR_OVERFLOW.  Every value that needs (the capacity into the voxel from
// each neighbour: bwd[v] from +a, fwd[v - stride] from -a) is an input this
// thread reads anyway, so the solve starts after one pass over the planes.
// Replaces initResidualsKernel and pushThroughTLinksFromSourceKernel
// (detail/graph_cut_implementation.hpp:28-40, detail/graph_cut_push.hpp:11-24).
//
// One CTA of 128 threads per tile; thread q owns the four voxels 4q..4q+3 of
// the tile (four consecutive x of one row).  The kernel is bound by load
// latency, so every load of a thread is issued unconditionally and at once:
// indices outside the instance are clamped to a valid voxel and missing
// planes read capS, and the values are masked afterwards.  The outputs are
// 16-byte stores into the tile-blocked planes.
__device__ __forceinline__ void put_tile4(const DevPool& P, const int t, const int32_t* const* ip) {
  __shared__ long long red[4];
  if (!CGC_IN_BOUNDS(P, t, P.T)) return;  // uniform over the block
  const int inst = P.tinst[t];
  const InstGeo G = P.geo[inst];
  const int lt = t - G.tile_base;
  const int tx = lt % G.TX, ty = (lt / G.TX) % G.TY, tz = lt / (G.TX * G.TY);
  const int q = threadIdx.x, l0 = 4 * q;
  const int x0 = tx * 8 + (l0 & 7), y = ty * 8 + ((l0 >> 3) & 7), z = tz * 8 + (l0 >> 6);
  const int64_t g0 = (int64_t)t * TV + l0;
  const int32_t* cs = ip[0];
  const int32_t* ct = ip[1];
  const int32_t* fp[3];
  const int32_t* bp[3];
  bool hasf[3], hasb[3];
#pragma unroll
  for (int a = 0; a < 3; ++a) {
    fp[a] = ip[2 + a]; bp[a] = ip[5 + a];
    hasf[a] = fp[a] != nullptr; hasb[a] = bp[a] != nullptr;
    if (!hasf[a]) fp[a] = cs;  // read something valid, then mask
    if (!hasb[a]) bp[a] = cs;
  }
  // vrow: the thread's first voxel, or voxel 0 when that lies outside the instance
  const bool row = y < G.Y && z < G.Z && x0 < G.X;
  const int64_t vrow = row ? x0 + (int64_t)G.X * (y + (int64_t)G.Y * z) : 0;
  const int ex[3] = {G.X, G.Y, G.Z};
  const int64_t st[3] = {1, (int64_t)G.X, (int64_t)G.X * G.Y};
  const int co[3] = {0, y, z};  // x is per voxel
  // loads (all independent).  With 16-byte aligned planes (the choice is
  // uniform over the block: one instance per tile), each plane row of the
  // thread's four voxels v..v+3 is read as the one or two aligned int4 that
  // cover it (load_row4); a row that would reach past the plane's end falls
  // back to scalar loads.  Otherwise one scalar load per voxel and plane.
  int s[4], c[4], fv[3][4], bv[3][4], fm[3][4], bm[3][4];
  bool ok[4];
#pragma unroll
  for (int k = 0; k < 4; ++k) ok[k] = row && x0 + k < G.X;
  uintptr_t align = reinterpret_cast<uintptr_t>(cs) | reinterpret_cast<uintptr_t>(ct);
#pragma unroll
  for (int a = 0; a < 3; ++a) align |= reinterpret_cast<uintptr_t>(fp[a]) | reinterpret_cast<uintptr_t>(bp[a]);
  const int64_t N = (int64_t)G.X * G.Y * G.Z;
  if ((align & 15) == 0) {
    // p[v .. v+3] from aligned int4 loads (p 16-byte aligned, 0 <= v < N)
    auto load_row4 = [N](int (&o)[4], const int32_t* p, int64_t v) {
      const int m = (int)(v & 3);
      const int64_t a = v - m;
      if (a + (m ? 8 : 4) <= N) {
        const int4 A = __ldg(reinterpret_cast<const int4*>(p + a));
        const int4 B = m ? __ldg(reinterpret_cast<const int4*>(p + a + 4)) : A;
        const int w[8] = {A.x, A.y, A.z, A.w, B.x, B.y, B.z, B.w};
#pragma unroll
        for (int k = 0; k < 4; ++k) o[k] = m == 0 ? w[k] : m == 1 ? w[k + 1] : m == 2 ? w[k + 2] : w[k + 3];
      } else {
#pragma unroll
        for (int k = 0; k < 4; ++k) o[k] = p[v + k < N ? v + k : v];
      }
    };
    load_row4(s, cs, vrow);
    load_row4(c, ct, vrow);
#pragma unroll
    for (int a = 0; a < 3; ++a) {
      load_row4(fv[a], fp[a], vrow);
      load_row4(bv[a], bp[a], vrow);
    }
    const int64_t vx = row && x0 > 0 ? vrow - 1 : vrow;  // -x neighbour of the first voxel
    fm[0][0] = __ldg(fp[0] + vx);
    bm[0][0] = __ldg(bp[0] + vx);
#pragma unroll
    for (int k = 1; k < 4; ++k) { fm[0][k] = fv[0][k - 1]; bm[0][k] = bv[0][k - 1]; }
#pragma unroll
    for (int a = 1; a < 3; ++a) {
      const int64_t vm = row && co[a] > 0 ? vrow - st[a] : vrow;
      load_row4(fm[a], fp[a], vm);
      load_row4(bm[a], bp[a], vm);
    }
  } else {
#pragma unroll
    for (int k = 0; k < 4; ++k) {
      const int64_t v = ok[k] ? vrow + k : vrow;
      s[k] = cs[v];
      c[k] = ct[v];
#pragma unroll
      for (int a = 0; a < 3; ++a) {
        const int cc = a == 0 ? x0 + k : co[a];
        const int64_t vm = cc > 0 && ok[k] ? v - st[a] : v;
        fv[a][k] = fp[a][v];
        bv[a][k] = bp[a][v];
        fm[a][k] = fp[a][vm];
        bm[a][k] = bp[a][vm];
      }
    }
  }
  int r[6][4];
  long long inflow[4];
  bool neg = false, bad = false;
#pragma unroll
  for (int k = 0; k < 4; ++k) {
    inflow[k] = 0;
    if (!ok[k]) { s[k] = 0; c[k] = 0; }
#pragma unroll
    for (int a = 0; a < 3; ++a) {
      const int cc = a == 0 ? x0 + k : co[a];
      const bool up = ok[k] && cc + 1 < ex[a], dn = ok[k] && cc > 0;
      r[2 * a][k] = up && hasf[a] ? fv[a][k] : 0;        // v -> v + e_a
      const int back_p = up && hasb[a] ? bv[a][k] : 0;   // v + e_a -> v
      r[2 * a + 1][k] = dn && hasb[a] ? bm[a][k] : 0;    // v -> v - e_a
      const int back_m = dn && hasf[a] ? fm[a][k] : 0;   // v - e_a -> v
      inflow[k] += (long long)back_p + back_m;
      bad = bad || (long long)r[2 * a][k] + back_p > 2147483647ll || (long long)r[2 * a + 1][k] + back_m > 2147483647ll;
    }
    neg = neg || s[k] < 0 || c[k] < 0;
#pragma unroll
    for (int d = 0; d < 6; ++d) neg = neg || r[d][k] < 0;
  }
  if (neg) raise_error(P, CGC_ERR_ARG);
  // t-link cancellation: min(capS, capT) flows straight through
  int e[4], rT[4];
  unsigned m4 = 0;
  long long tot = 0;
#pragma unroll
  for (int k = 0; k < 4; ++k) {
    const int mcap = min(s[k], c[k]);
    e[k] = s[k] - mcap;
    rT[k] = c[k] - mcap;
    tot += mcap;
    unsigned m = (rT[k] > 0 ? 64u : 0u) | (e[k] > 0 ? 128u : 0u);
#pragma unroll
    for (int d = 0; d < 6; ++d) m |= (r[d][k] > 0 ? 1u : 0u) << d;
    m4 |= m << (8 * k);
    bad = bad || inflow[k] + e[k] > 2147483647ll;
  }
  if (bad) raise_error(P, CGC_ERR_OVERFLOW);
  *reinterpret_cast<int4*>(P.e + g0) = make_int4(e[0], e[1], e[2], e[3]);
  *reinterpret_cast<int4*>(P.rT + g0) = make_int4(rT[0], rT[1], rT[2], rT[3]);
#pragma unroll
  for (int d = 0; d < 6; ++d)
    *reinterpret_cast<int4*>(P.r + d * P.Np + g0) = make_int4(r[d][0], r[d][1], r[d][2], r[d][3]);
  // no label yet (INF would read as "dead" to the first global relabel)
  *reinterpret_cast<int4*>(P.h + g0) = make_int4(0, 0, 0, 0);
  *reinterpret_cast<uint32_t*>(P.rmask + g0) = m4;
  *reinterpret_cast<uint32_t*>(P.reach + g0) = 0u;
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) tot += __shfl_down_sync(0xffffffffu, tot, o);
  if ((q & 31) == 0) red[q >> 5] = tot;
  __syncthreads();
  if (q == 0) {
    const long long sum = red[0] + red[1] + red[2] + red[3];
    P.act[t] = 0;
    if (sum) atomicAdd(P.flow + inst, (unsigned long long)sum);
  }
}

// ---------------------------------------------------------------------------
// Cut sets in linear voxel order, four voxels per thread: voxels v0..v0+3 of
// an instance (v0 a multiple of 4) are gathered from the tile layout (one
// 64-bit division per four voxels, all loads issued at once from clamped
// indices), and the four output bytes go out as one 32-bit store when the
// destination is aligned, so a warp writes whole 128-byte lines.
// Bit 0 of each byte of *sink: height < INF; of *source: in the minimal
// source set.
__device__ __forceinline__ void seg_gather4(const DevPool& P, const InstGeo& G, int64_t v0, int64_t N,
                                            unsigned* sink, unsigned* source) {
  int64_t rest = v0 / G.X;
  int x = (int)(v0 - rest * G.X);
  int y = (int)(rest % G.Y), z = (int)(rest / G.Y);
  int64_t gk[4];
#pragma unroll
  for (int k = 0; k < 4; ++k) {
    const int64_t t = G.tile_base + (x >> 3) + (int64_t)G.TX * ((y >> 3) + (int64_t)G.TY * (z >> 3));
    gk[k] = t * TV + (x & 7) + 8 * (y & 7) + 64 * (z & 7);
    if (v0 + k >= N) gk[k] = gk[0];
    if (++x == G.X) { x = 0; if (++y == G.Y) { y = 0; ++z; } }
  }
  unsigned a = 0, b = 0;
  int hv[4];
  unsigned char rv[4];
#pragma unroll
  for (int k = 0; k < 4; ++k) {
    hv[k] = sink ? __ldcg(P.h + gk[k]) : INF;
    rv[k] = source ? __ldcg(P.reach + gk[k]) : (unsigned char)0;
  }
#pragma unroll
  for (int k = 0; k < 4; ++k) {
    a |= (hv[k] < INF ? 1u : 0u) << (8 * k);
    b |= (rv[k] ? 1u : 0u) << (8 * k);
  }
  if (sink) *sink = a;
  if (source) *source = b;
}

// the bytes of `bits` (0 or 1 each) as mask / bg at out[v0 .. min(v0 + 4, N))
__device__ __forceinline__ void seg_store4(uint8_t* out, int64_t v0, int64_t N, unsigned bits, uint8_t mask,
                                           uint8_t bg) {
  unsigned w = 0;
#pragma unroll
  for (int k = 0; k < 4; ++k) w |= (unsigned)(((bits >> (8 * k)) & 1u) ? mask : bg) << (8 * k);
  uint8_t* p = out + v0;
  if (v0 + 4 <= N && ((reinterpret_cast<uintptr_t>(p) & 3u) == 0)) {
    *reinterpret_cast<unsigned*>(p) = w;
  } else {
    for (int k = 0; k < 4 && v0 + k < N; ++k) p[k] = (uint8_t)(w >> (8 * k));
  }
}

// ---------------------------------------------------------------------------
// BFS seeding, first step: bfs_init_tile_w (a warp per tile).
// Second BFS seeding step, one thread per tile: queue every tile that is not
// all seeds and holds a seed or touches a seed on a neighbour's face.
__device__ __forceinline__ bool bfs_seed_tile(const DevPool& P, const int t) {
  bool q = false;
  if (t < P.T) {
    const int f = __ldcg(P.tflag + t);
    if (!(f & (TF_ALL_SEED | TF_DEAD))) {
      q = (f & TF_HAS_SEED) != 0;
#pragma unroll
      for (int d = 0; d < 6; ++d) {
        const int nt = __ldcg(P.nbr + d * P.T + t);
        if (nt >= 0 && CGC_IN_BOUNDS(P, nt, P.T) && ((__ldcg(P.tflag + nt) >> (1 + (d ^ 1))) & 1))
          q = true;  // dead tiles have no seed bits
      }
    }
  }
  return q;
}

__device__ __forceinline__ void bfs_queue_tile(const DevPool& P, const int t, const uint32_t id0, int32_t* list0,
                                               int32_t* cnt0) {
  const bool q = bfs_seed_tile(P, t);
  if (q) P.stamp_bfs[t] = id0;
  warp_append(P, q, t, list0, cnt0);
}

// One BFS visit: relax h(v) = min(h(v), 1 + h(u)) over residual edges v->u
// until the tile is stable; re-queue face neighbours whose halo changed.
__device__ inline void bfs_tile(const DevPool& P, const int t, BfsShared& S, const uint32_t id_next,
                         int32_t* list_next, int32_t* cnt_next) {
  if (!CGC_IN_BOUNDS(P, t, P.T)) return;  // uniform over the block
  if (__ldcg(P.tflag + t) & TF_DEAD) return;  // uniform over the block; nothing can change
  const int l = threadIdx.x;
  const int nb = l < 6 ? __ldcg(P.nbr + l * P.T + t) : -1;  // face neighbour, for the re-queue
  const int x = l & 7, y = (l >> 3) & 7, z = l >> 6;
  const int64_t g = (int64_t)t * TV + l;
  int h = __ldcg(P.h + g);
  const int h0 = h;
  const unsigned m = __ldcg(P.rmask + g);
  const bool has_excess = (m & 128u) != 0;
  const int hi = halo_index(x, y, z);
  S.h[0][hi] = h;
  load_halo_heights(P, t, S.h);
  if (l == 0) S.flags = 0;
  __syncthreads();
  int cur = 0;
  for (int it = 0; it < 1024; ++it) {  // converges in < 512 steps (path length in a tile)
    int mn = h;
#pragma unroll
    for (int d = 0; d < 6; ++d)
      if ((m >> d) & 1u) mn = min(mn, S.h[cur][hi + hoff(d)] + 1);
    S.h[cur ^ 1][hi] = mn;
    const int any = __syncthreads_or(mn < h);
    h = mn;
    cur ^= 1;
    if (!any) break;
  }
  if (h < h0) {
    P.h[g] = h;
    const int fb = face_bits(x, y, z);
    if (fb) atomicOr(&S.flags, fb);
  }
  const int act = __syncthreads_or(has_excess && h < INF);
  if (l == 0) {
    P.act[t] = (uint8_t)(act ? 1 : 0);  // heights only drop in later visits: the last visit's value is final
    atomicAdd(P.stats + S_TILES_BFS, 1ull);
  }
  if (l < 6 && ((S.flags >> l) & 1) && nb >= 0) queue_tile(P, P.stamp_bfs, nb, id_next, list_next, cnt_next);
  __syncthreads();
}

// ---------------------------------------------------------------------------
// Incremental global relabel.  Heights are a valid labelling at all times
// (h <= d, the exact distance to the sink), and h(v) == d(v) exactly when v is
// supported: a sink-adjacent voxel at height 1 (rT > 0), or a voxel with a
// residual edge to a supported neighbour exactly one lower.  (Along a shortest
// path every step of a valid labelling drops by at most one, so h == d forces
// each step to drop by exactly one down to a seed at 1.)  Right after an exact
// relabel every finite voxel is supported; a sweep cycle can break support
// only inside the tiles it queued (their heights and out-residuals changed)
// and, through their face voxels, in the face neighbours of those tiles.  So
// the invalidation pass below visits those tiles, sets every unsupported
// voxel to INF and re-checks the neighbours of every voxel it drops; the
// voxels it leaves finite are exact, and the tile Bellman-Ford (bfs_tile)
// started from the tiles with dropped voxels recomputes the rest exactly.
// The heights that come out equal the full BFS's bit for bit.

// a tile's sweep stamps (both halves under exclusive sweeps) were written
// after id c0, i.e. the tile was queued during the current sweep cycle
__device__ __forceinline__ bool queued_since(const DevPool& P, int t, uint32_t c0, bool exclusive) {
  const uint32_t a = __ldcg(P.stamp_sw + t);
  const uint32_t b = exclusive ? __ldcg(P.stamp_sw + P.T + t) : 0u;
  return (int32_t)(a - c0) > 0 || (exclusive && (int32_t)(b - c0) > 0);
}

// Seed of the invalidation pass, one thread per tile: tiles queued during the
// cycle and their face neighbours.
__device__ __forceinline__ void inval_queue_tile(const DevPool& P, const int t, const uint32_t c0, const bool exclusive,
                                                 const uint32_t id0, int32_t* list0, int32_t* cnt0) {
  bool q = false;
  if (t < P.T) {
    q = queued_since(P, t, c0, exclusive);
#pragma unroll
    for (int d = 0; d < 6; ++d) {
      const int nt = __ldcg(P.nbr + d * P.T + t);
      if (!q && nt >= 0 && CGC_IN_BOUNDS(P, nt, P.T)) q = queued_since(P, nt, c0, exclusive);
    }
    if (q && (__ldcg(P.tflag + t) & TF_DEAD)) q = false;  // all INF, nothing to check
  }
  if (q) P.stamp_bfs[t] = id0;
  warp_append(P, q, t, list0, cnt0);
}

// One invalidation visit: drop unsupported voxels of tile t to INF until the
// tile is stable (drops are monotone, so in-place updates are safe and the
// result is the largest supported set); re-queue the face neighbours of
// dropped face voxels, and list the tile once (stamp_inc) for the BFS rounds.
__device__ inline void inval_tile(const DevPool& P, const int t, BfsShared& S, const uint32_t id_next,
                                  int32_t* list_next, int32_t* cnt_next, const uint32_t id_bfs, int32_t* list_bfs,
                                  int32_t* cnt_bfs) {
  if (!CGC_IN_BOUNDS(P, t, P.T)) return;  // uniform over the block
  const int l = threadIdx.x;
  const int nb = l < 6 ? __ldcg(P.nbr + l * P.T + t) : -1;  // face neighbour, for the re-queue
  const int x = l & 7, y = (l >> 3) & 7, z = l >> 6;
  const int64_t g = (int64_t)t * TV + l;
  int h = __ldcg(P.h + g);
  const unsigned m = __ldcg(P.rmask + g);
  const int hi = halo_index(x, y, z);
  S.h[0][hi] = h;
  load_halo_heights(P, t, S.h);
  if (l == 0) S.flags = 0;
  __syncthreads();
  bool dropped = false;
  for (int it = 0; it < 1024; ++it) {  // a drop per step climbs one height: < 512 steps in a tile
    bool drop = false;
    if (h < INF && !((m & 64u) && h == 1)) {
      bool sup = false;
#pragma unroll
      for (int d = 0; d < 6; ++d)
        if ((m >> d) & 1u) sup = sup || S.h[0][hi + hoff(d)] == h - 1;
      drop = !sup;
    }
    if (drop) {
      h = INF;
      S.h[0][hi] = INF;
      dropped = true;
    }
    if (!__syncthreads_or(drop)) break;
  }
  if (dropped) {
    P.h[g] = INF;
    const int fb = face_bits(x, y, z);
    if (fb) atomicOr(&S.flags, fb);
  }
  const int any = __syncthreads_or(dropped);
  if (l == 0) atomicAdd(P.stats + S_TILES_CHECK, 1ull);
  if (l == 32 && any) queue_tile(P, P.stamp_inc, t, id_bfs, list_bfs, cnt_bfs);
  if (l < 6 && ((S.flags >> l) & 1) && nb >= 0) queue_tile(P, P.stamp_bfs, nb, id_next, list_next, cnt_next);
  __syncthreads();
}

// ---------------------------------------------------------------------------
// Source-side reachability (canonical cut) after the maximum preflow:
// closure of {v : e(v) > 0} over residual edges, seeded by reach_init_tile_w
// (a warp per tile).
__device__ inline void reach_tile(const DevPool& P, const int t, ReachShared& S, const uint32_t id_next,
                           int32_t* list_next, int32_t* cnt_next) {
  if (!CGC_IN_BOUNDS(P, t, P.T)) return;  // uniform over the block
  const int l = threadIdx.x;
  const int nb = l < 6 ? __ldcg(P.nbr + l * P.T + t) : -1;  // face neighbour, for the re-queue
  const int x = l & 7, y = (l >> 3) & 7, z = l >> 6;
  const int64_t g = (int64_t)t * TV + l;
  int rc = __ldcg(P.reach + g);
  const int rc0 = rc;
  const int hi = halo_index(x, y, z);
  S.rc[0][hi] = (unsigned char)rc;
  S.m[hi] = __ldcg(P.rmask + g);
  for_halo_entry(l, [&](int f, int hh, int src) {
    const int nt = __ldcg(P.nbr + f * P.T + t);
    unsigned char rv = 0, mv = 0;
    if (nt >= 0 && CGC_IN_BOUNDS(P, nt, P.T)) {
      rv = __ldcg(P.reach + (int64_t)nt * TV + src);
      mv = __ldcg(P.rmask + (int64_t)nt * TV + src);
    }
    S.rc[0][hh] = rv; S.rc[1][hh] = rv; S.m[hh] = mv;
  });
  if (l == 0) S.flags = 0;
  __syncthreads();
  int cur = 0;
  for (int it = 0; it < 1024; ++it) {
    bool ch = false;
    if (!rc) {
#pragma unroll
      for (int d = 0; d < 6; ++d) {
        const int u = hi + hoff(d);
        if (S.rc[cur][u] && ((S.m[u] >> (d ^ 1)) & 1u)) ch = true;
      }
    }
    if (ch) rc = 1;
    S.rc[cur ^ 1][hi] = (unsigned char)rc;
    const int any = __syncthreads_or(ch);
    cur ^= 1;
    if (!any) break;
  }
  if (rc && !rc0) {
    P.reach[g] = 1;
    const int fb = face_bits(x, y, z);
    if (fb) atomicOr(&S.flags, fb);
  }
  __syncthreads();
  if (l < 6 && ((S.flags >> l) & 1) && nb >= 0) queue_tile(P, P.stamp_bfs, nb, id_next, list_next, cnt_next);
  __syncthreads();
}

}  // namespace cgc
