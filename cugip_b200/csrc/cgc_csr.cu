// Generic (non-grid) graphs: exact push-relabel over a CSR residual graph.
//
// The reference solves every graph through one CSR layout
// (include/cugip/advanced_operations/graph_cut.hpp:239-290: neighbour lists,
// one residual pair per undirected edge) with a level-synchronous BFS
// relabel and per-level pushes (detail/graph_cut_relabeling.hpp:1004-1029,
// detail/graph_cut_push.hpp:461-482).  Grids go to the tile engine; this file
// handles every other edge list with the same options, statuses and cut
// semantics:
//   * CSR built on the device: per-vertex degree count, exclusive scan,
//     atomic scatter of the two arcs of every edge with reverse-arc links.
//     The original arc capacities are kept, so a graph can be solved again.
//   * one cooperative launch per solve: exact global relabel (BFS from the
//     vertices with a sink residual over reverse residual arcs, heights set by
//     CAS), then up to K synchronous pulses over a deduplicated active-vertex
//     list: a push step with fixed labels (a vertex pushes along arcs to
//     neighbours one level lower; excess and reverse residuals of the
//     neighbour by atomics) and a relabel step (1 + the lowest residual
//     neighbour; labels only grow, so concurrent relabels keep them valid).
//     The solve ends when an exact relabel leaves no active vertex.
//   * int32 capacities, int64 flow, t-links cancelled up front (min(capS,
//     capT) flows straight through), pushes to the sink capped by its residual.
//   * cuts: sink side = vertices with a finite height after the last exact
//     relabel (the reference's fill_segments, graph_cut.hpp:304-333); source
//     side = residual closure of the vertices that hold excess.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstring>
#include <string>
#include <vector>

#include "cgc.h"
#include "cgc_internal.h"
#include "cgc_pool.h"
#include "cgc_sync.cuh"

namespace cgc {
namespace {

constexpr int CSR_THREADS = 256;
constexpr int SCAN_BLOCK = 1024;

enum CsrStat { CS_PULSES = 0, CS_RELABELS, CS_LEVELS, CS_PUSHES, CS_BFS_VISITS, CS_NS_BFS, CS_NS_PUSH, CS_NS_REACH, CS_N = 16 };
enum CsrCounter { CC_BFS0 = 0, CC_PULSE0 = 3, CC_N = 8 };

struct CsrDev {
  int32_t n;
  int64_t arcs;
  int32_t hdead;             // heights >= hdead cannot reach the sink (n + 1)
  const int32_t* row;        // n + 1: first arc of each vertex
  const int32_t* to;         // arcs: head vertex
  const int32_t* rev;        // arcs: index of the reverse arc
  int32_t* res;              // arcs: residual capacity
  const int32_t* res0;       // arcs: capacity
  const int32_t* capS;       // n
  const int32_t* capT;       // n
  int32_t* e;                // n: excess
  int32_t* h;                // n: height
  int32_t* rT;               // n: sink residual
  int32_t* reach;            // n: source side
  uint32_t* stamp;           // n: last list the vertex was queued for
  int32_t* list;             // 2n: two vertex lists
  int32_t* cnt;              // CC_N counters
  unsigned long long* flow;  // 1
  unsigned long long* stats; // CS_N
  int32_t* err;
  uint32_t* bar;             // 2
};

struct CsrParams {
  int K;                 // pulses between exact relabels
  int64_t max_pulses;    // safety cap
  uint64_t limit_ns;     // bounded barrier waits
};

__device__ __forceinline__ int ldv(const int32_t* p) { return *(volatile const int32_t*)p; }

// warp-aggregated append (all lanes of the warp call it)
__device__ __forceinline__ void csr_append(bool pred, int32_t item, int32_t* list, int32_t* cnt) {
  const unsigned mask = __ballot_sync(0xffffffffu, pred);
  if (!mask) return;
  const int lane = threadIdx.x & 31;
  const int leader = __ffs(mask) - 1;
  int base = 0;
  if (lane == leader) base = atomicAdd(cnt, __popc(mask));
  base = __shfl_sync(0xffffffffu, base, leader);
  if (pred) list[base + __popc(mask & ((1u << lane) - 1))] = item;
}

// ---------------------------------------------------------------- CSR build
__global__ void k_csr_degree(int64_t m, const int32_t* __restrict__ a, const int32_t* __restrict__ b, int32_t* deg) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < m; i += (int64_t)gridDim.x * blockDim.x) {
    const int u = a[i], v = b[i];
    if (u == v) continue;  // a self loop carries no flow
    atomicAdd(deg + u, 1);
    atomicAdd(deg + v, 1);
  }
}

// exclusive scan, pass 1: each block scans SCAN_BLOCK entries
__global__ void __launch_bounds__(SCAN_BLOCK) k_scan_block(const int32_t* in, int32_t* out, int32_t* bsum, int n) {
  __shared__ int32_t ws[SCAN_BLOCK / 32];
  const int i = blockIdx.x * SCAN_BLOCK + threadIdx.x, lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  const int v = i < n ? in[i] : 0;
  int x = v;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const int y = __shfl_up_sync(0xffffffffu, x, o);
    if (lane >= o) x += y;
  }
  if (lane == 31) ws[w] = x;
  __syncthreads();
  if (w == 0) {
    int s = ws[lane];
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const int y = __shfl_up_sync(0xffffffffu, s, o);
      if (lane >= o) s += y;
    }
    ws[lane] = s;
  }
  __syncthreads();
  const int incl = x + (w > 0 ? ws[w - 1] : 0);
  if (i < n) out[i] = incl - v;
  if (threadIdx.x == SCAN_BLOCK - 1) bsum[blockIdx.x] = incl;
}

// pass 2: exclusive scan of the block sums by one block; total into *total
__global__ void __launch_bounds__(SCAN_BLOCK) k_scan_sums(int32_t* bsum, int nb, int32_t* total) {
  __shared__ int32_t ws[SCAN_BLOCK / 32];
  __shared__ int32_t carry;
  if (threadIdx.x == 0) carry = 0;
  __syncthreads();
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  for (int base = 0; base < nb; base += SCAN_BLOCK) {
    const int i = base + threadIdx.x;
    const int v = i < nb ? bsum[i] : 0;
    int x = v;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const int y = __shfl_up_sync(0xffffffffu, x, o);
      if (lane >= o) x += y;
    }
    if (lane == 31) ws[w] = x;
    __syncthreads();
    if (w == 0) {
      int s = ws[lane];
#pragma unroll
      for (int o = 1; o < 32; o <<= 1) {
        const int y = __shfl_up_sync(0xffffffffu, s, o);
        if (lane >= o) s += y;
      }
      ws[lane] = s;
    }
    __syncthreads();
    const int incl = x + (w > 0 ? ws[w - 1] : 0);
    const int c = carry;
    if (i < nb) bsum[i] = c + incl - v;
    __syncthreads();
    if (threadIdx.x == SCAN_BLOCK - 1) carry = c + incl;
    __syncthreads();
  }
  if (threadIdx.x == 0) *total = carry;
}

// pass 3: add the block offsets
__global__ void k_scan_add(int32_t* out, const int32_t* bsum, int n) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) out[i] += bsum[i / SCAN_BLOCK];
}

__global__ void k_csr_scatter(int64_t m, const int32_t* __restrict__ a, const int32_t* __restrict__ b,
                              const int32_t* __restrict__ fwd, const int32_t* __restrict__ bwd, const int32_t* row,
                              int32_t* cur, int32_t* to, int32_t* rev, int32_t* res0) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < m; i += (int64_t)gridDim.x * blockDim.x) {
    const int u = a[i], v = b[i];
    if (u == v) continue;
    const int pu = row[u] + atomicAdd(cur + u, 1);
    const int pv = row[v] + atomicAdd(cur + v, 1);
    to[pu] = v; rev[pu] = pv; res0[pu] = fwd[i];
    to[pv] = u; rev[pv] = pu; res0[pv] = bwd[i];
  }
}

// ---------------------------------------------------------------- solve
__global__ void k_csr_prepare(CsrDev D) {
  const int64_t nt = (int64_t)gridDim.x * blockDim.x, gt = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  for (int64_t a = gt; a < D.arcs; a += nt) D.res[a] = D.res0[a];
  long long through = 0;
  for (int64_t v = gt; v < D.n; v += nt) {
    const int s = D.capS[v], t = D.capT[v], mn = min(s, t);
    D.e[v] = s - mn;
    D.rT[v] = t - mn;
    D.h[v] = 0;
    D.stamp[v] = 0;
    through += mn;
    // Excess and residuals stay int32: the excess is at most the source
    // excess plus every capacity into v, a residual at most the two
    // capacities of its edge.
    long long inflow = s - mn;
    bool bad = false;
    const int a1 = D.row[v + 1];
    for (int a = D.row[v]; a < a1; ++a) {
      const long long back = D.res0[D.rev[a]];
      inflow += back;
      if (back + D.res0[a] > 2147483647ll) bad = true;
    }
    if (bad || inflow > 2147483647ll) atomicCAS(D.err, 0, CGC_ERR_OVERFLOW);
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) through += __shfl_down_sync(0xffffffffu, through, o);
  if ((threadIdx.x & 31) == 0 && through) atomicAdd(D.flow, (unsigned long long)through);
}

__global__ void __launch_bounds__(CSR_THREADS) k_csr_solve(CsrDev D, CsrParams prm) {
  const int n = D.n;
  const int lane = threadIdx.x & 31;
  const int gt = blockIdx.x * blockDim.x + threadIdx.x, nt = gridDim.x * blockDim.x;
  int32_t* const L[2] = {D.list, D.list + n};
  int32_t* const cb = D.cnt + CC_BFS0;    // 3 rotating counters of the BFS frontiers
  int32_t* const cp = D.cnt + CC_PULSE0;  // 3 rotating counters of the pulse lists
  const bool lead = gt == 0;
  uint32_t sid = 0;
  long long pulses = 0, relabels = 0, levels = 0;
  unsigned long long ns_bfs = 0, ns_push = 0, ns_reach = 0;
  uint64_t tmark = sync_globaltimer_ns();
  auto lap = [&](unsigned long long& acc) {
    const uint64_t now = sync_globaltimer_ns();
    acc += now - tmark;
    tmark = now;
  };
  auto sync = [&]() { return grid_barrier(D.bar, D.err, prm.limit_ns); };
  // frontier BFS over lists L[k&1] with counters cb[k%3]; `visit` appends
  // to the next frontier; returns the number of rounds, -1 on a failed barrier
  auto bfs = [&](auto&& visit) -> int {
    int k = 0;
    for (;;) {
      const int nf = ldv(cb + k % 3);
      if (nf == 0) return k;
      if (lead) cb[(k + 2) % 3] = 0;
      for (int i = gt; i < nf; i += nt) visit(L[k & 1][i], k, L[(k + 1) & 1], cb + (k + 1) % 3);
      ++k;
      if (!sync()) return -1;
    }
  };

  for (;;) {
    // ------------------------------------------------ exact global relabel
    if (lead) { cb[0] = cb[1] = cb[2] = 0; cp[0] = cp[1] = cp[2] = 0; }
    if (!sync()) return;
    for (int v = gt; v - lane < n; v += nt) {
      const bool seed = v < n && __ldcg(D.rT + v) > 0;
      if (v < n) D.h[v] = seed ? 1 : INF;
      csr_append(seed, v, L[0], cb + 0);
    }
    if (!sync()) return;
    const int rounds = bfs([&](int u, int k, int32_t* next, int32_t* cnext) {
      const int lev = k + 2;  // the frontier of round k has height k + 1
      const int a1 = D.row[u + 1];
      for (int a = D.row[u]; a < a1; ++a) {
        const int v = D.to[a];
        if (__ldcg(D.res + D.rev[a]) > 0 && ldv(D.h + v) == INF && atomicCAS(D.h + v, INF, lev) == INF)
          next[atomicAdd(cnext, 1)] = v;
      }
    });
    if (rounds < 0) return;
    levels += rounds;
    ++relabels;
    lap(ns_bfs);
    // ------------------------------------------------ active vertices
    ++sid;
    for (int v = gt; v - lane < n; v += nt) {
      const bool act = v < n && __ldcg(D.e + v) > 0 && __ldcg(D.h + v) < INF;
      if (act) D.stamp[v] = sid;
      csr_append(act, v, L[0], cp + 0);
    }
    if (!sync()) return;
    if (ldv(cp + 0) == 0) break;
    if (pulses >= prm.max_pulses) {
      if (lead) atomicCAS(D.err, 0, CGC_ERR_NOT_CONVERGED);
      break;
    }
    // ------------------------------------------------ pulses
    for (int p = 0; p < prm.K; ++p) {
      const int ncur = ldv(cp + p % 3);
      if (ncur == 0) break;
      if (lead) cp[(p + 2) % 3] = 0;
      ++sid;
      const int32_t* lc = L[p & 1];
      int32_t* ln = L[(p + 1) & 1];
      int32_t* cn = cp + (p + 1) % 3;
      // push step: labels fixed
      for (int i = gt; i < ncur; i += nt) {
        const int v = lc[i];
        int ev = __ldcg(D.e + v);
        const int hv = __ldcg(D.h + v);
        if (ev <= 0 || hv >= INF) continue;
        const int e0 = ev;
        const int rt = __ldcg(D.rT + v);
        if (rt > 0 && hv == 1) {
          const int dl = min(ev, rt);
          D.rT[v] = rt - dl;
          ev -= dl;
          atomicAdd(D.flow, (unsigned long long)dl);
        }
        const int a1 = D.row[v + 1];
        for (int a = D.row[v]; a < a1 && ev > 0; ++a) {
          const int r = __ldcg(D.res + a);
          if (r <= 0) continue;
          const int u = D.to[a];
          if (__ldcg(D.h + u) != hv - 1) continue;
          const int dl = min(ev, r);
          D.res[a] = r - dl;  // only v writes this arc in this step
          atomicAdd(D.res + D.rev[a], dl);
          atomicAdd(D.e + u, dl);
          ev -= dl;
          if (atomicExch(D.stamp + u, sid) != sid) ln[atomicAdd(cn, 1)] = u;
        }
        if (ev != e0) atomicSub(D.e + v, e0 - ev);
        if (ev > 0 && atomicExch(D.stamp + v, sid) != sid) ln[atomicAdd(cn, 1)] = v;
      }
      if (!sync()) return;
      // relabel step: an active vertex without an admissible arc moves to one
      // above its lowest residual neighbour
      const int nn = ldv(cn);
      for (int i = gt; i < nn; i += nt) {
        const int v = ln[i];
        const int hv = __ldcg(D.h + v);
        if (__ldcg(D.e + v) <= 0 || hv >= INF) continue;
        const int rt = __ldcg(D.rT + v);
        if (rt > 0 && hv == 1) continue;
        int mn = rt > 0 ? 0 : INF;
        bool adm = false;
        const int a1 = D.row[v + 1];
        for (int a = D.row[v]; a < a1; ++a) {
          if (__ldcg(D.res + a) <= 0) continue;
          const int hu = ldv(D.h + D.to[a]);
          if (hu == hv - 1) { adm = true; break; }
          mn = min(mn, hu);
        }
        if (!adm) {
          int hn = mn >= INF ? INF : mn + 1;
          if (hn >= D.hdead) hn = INF;
          D.h[v] = hn;
        }
      }
      ++pulses;
      if (!sync()) return;
    }
    lap(ns_push);
  }
  lap(ns_bfs);
  // ------------------------------------------------ source side: residual
  // closure of the vertices that hold excess
  if (lead) { cb[0] = cb[1] = cb[2] = 0; }
  if (!sync()) return;
  for (int v = gt; v - lane < n; v += nt) {
    const bool seed = v < n && __ldcg(D.e + v) > 0;
    if (v < n) D.reach[v] = seed ? 1 : 0;
    csr_append(seed, v, L[0], cb + 0);
  }
  if (!sync()) return;
  const int rrounds = bfs([&](int u, int, int32_t* next, int32_t* cnext) {
    const int a1 = D.row[u + 1];
    for (int a = D.row[u]; a < a1; ++a) {
      const int v = D.to[a];
      if (__ldcg(D.res + a) > 0 && ldv(D.reach + v) == 0 && atomicCAS(D.reach + v, 0, 1) == 0)
        next[atomicAdd(cnext, 1)] = v;
    }
  });
  if (rrounds < 0) return;
  lap(ns_reach);
  if (lead) {
    D.stats[CS_PULSES] = (unsigned long long)pulses;
    D.stats[CS_RELABELS] = (unsigned long long)relabels;
    D.stats[CS_LEVELS] = (unsigned long long)levels;
    D.stats[CS_NS_BFS] = ns_bfs;
    D.stats[CS_NS_PUSH] = ns_push;
    D.stats[CS_NS_REACH] = ns_reach;
  }
}

__global__ void k_csr_segments(CsrDev D, int which, uint8_t* out, uint8_t mask, uint8_t bg) {
  for (int64_t v = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; v < D.n; v += (int64_t)gridDim.x * blockDim.x) {
    const bool in = which == CGC_SEG_SOURCE_MIN ? D.reach[v] != 0 : D.h[v] < INF;
    out[v] = in ? mask : bg;
  }
}

int grid_blocks(int64_t work, int threads) { return (int)std::max<int64_t>(1, std::min<int64_t>((work + threads - 1) / threads, 1 << 16)); }

}  // namespace
}  // namespace cgc

struct cgc_graph {
  int device = 0;
  cudaStream_t stream = nullptr;
  int32_t n = 0;
  int64_t m = 0;
  void* dbuf = nullptr;
  uint8_t* seg = nullptr;
  cgc::CsrDev d{};
  int coop_blocks = 0;
  bool tlinks = false, solved = false;
  cgc_stats st{};
};

namespace {

using cgc::fail;
using cgc::ok;

void graph_free(cgc_graph* g) {
  if (!g) return;
  if (g->dbuf) cudaFree(g->dbuf);
  delete g;
}

int graph_create(int32_t n, int64_t m, const int32_t* a, const int32_t* b, const int32_t* cab, const int32_t* cba,
                 void* stream, cgc_graph** out) {
  using namespace cgc;
  if (!out) return fail(CGC_ERR_ARG, "cgc_graph_create: null output");
  *out = nullptr;
  if (n <= 0 || m < 0 || (m > 0 && (!a || !b || !cab || !cba)))
    return fail(CGC_ERR_ARG, "cgc_graph_create: bad arguments");
  int64_t loops = 0;
  for (int64_t i = 0; i < m; ++i) {
    if (a[i] < 0 || a[i] >= n || b[i] < 0 || b[i] >= n)
      return fail(CGC_ERR_ARG, "cgc_graph_create: edge " + std::to_string(i) + " has a vertex outside [0, n)");
    if (cab[i] < 0 || cba[i] < 0)
      return fail(CGC_ERR_ARG, "cgc_graph_create: negative capacity on edge " + std::to_string(i));
    loops += a[i] == b[i];
  }
  const int64_t arcs = 2 * (m - loops);
  if (arcs > 2147483647ll || n > 2147483646) return fail(CGC_ERR_ARG, "cgc_graph_create: graph too large for int32 arc ids");
  cgc_graph* g = new (std::nothrow) cgc_graph();
  if (!g) return fail(CGC_ERR_OOM, "cgc_graph_create: host allocation");
  g->n = n;
  g->m = m;
  g->stream = (cudaStream_t)stream;
  int rc = [&]() -> int {
    CGC_CUDA(cudaGetDevice(&g->device));
    auto al = [](int64_t bytes) { return (bytes + 255) & ~(int64_t)255; };
    const int nb = (int)((n + SCAN_BLOCK - 1) / SCAN_BLOCK);
    int64_t off = 0;
    const int64_t o_row = off; off += al(((int64_t)n + 1) * 4);
    const int64_t o_to = off; off += al(arcs * 4);
    const int64_t o_rev = off; off += al(arcs * 4);
    const int64_t o_res = off; off += al(arcs * 4);
    const int64_t o_res0 = off; off += al(arcs * 4);
    const int64_t o_cs = off; off += al((int64_t)n * 4);
    const int64_t o_ct = off; off += al((int64_t)n * 4);
    const int64_t o_e = off; off += al((int64_t)n * 4);
    const int64_t o_h = off; off += al((int64_t)n * 4);
    const int64_t o_rt = off; off += al((int64_t)n * 4);
    const int64_t o_rc = off; off += al((int64_t)n * 4);
    const int64_t o_st = off; off += al((int64_t)n * 4);
    const int64_t o_li = off; off += al(2 * (int64_t)n * 4);
    const int64_t o_cnt = off; off += al(CC_N * 4);
    const int64_t o_fl = off; off += al(8);
    const int64_t o_sta = off; off += al(CS_N * 8);
    const int64_t o_err = off; off += al(4);
    const int64_t o_bar = off; off += al(8);
    const int64_t o_seg = off; off += al(n);
    const int64_t o_bs = off; off += al((int64_t)nb * 4);
    CGC_CUDA(cudaMalloc(&g->dbuf, off));
    CGC_CUDA(cudaMemsetAsync(g->dbuf, 0, off, g->stream));
    char* base = (char*)g->dbuf;
    CsrDev& d = g->d;
    d.n = n;
    d.arcs = arcs;
    d.hdead = (int32_t)std::min<int64_t>((int64_t)n + 1, INF);
    d.row = (int32_t*)(base + o_row);
    d.to = (int32_t*)(base + o_to);
    d.rev = (int32_t*)(base + o_rev);
    d.res = (int32_t*)(base + o_res);
    d.res0 = (int32_t*)(base + o_res0);
    d.capS = (int32_t*)(base + o_cs);
    d.capT = (int32_t*)(base + o_ct);
    d.e = (int32_t*)(base + o_e);
    d.h = (int32_t*)(base + o_h);
    d.rT = (int32_t*)(base + o_rt);
    d.reach = (int32_t*)(base + o_rc);
    d.stamp = (uint32_t*)(base + o_st);
    d.list = (int32_t*)(base + o_li);
    d.cnt = (int32_t*)(base + o_cnt);
    d.flow = (unsigned long long*)(base + o_fl);
    d.stats = (unsigned long long*)(base + o_sta);
    d.err = (int32_t*)(base + o_err);
    d.bar = (uint32_t*)(base + o_bar);
    g->seg = (uint8_t*)(base + o_seg);
    int32_t* bsum = (int32_t*)(base + o_bs);
    if (m > 0) {
      // edges to the device, then degrees -> row offsets -> arcs
      int32_t* stage = nullptr;
      CGC_CUDA(cudaMalloc(&stage, 4 * m * 4));
      int rc2 = [&]() -> int {
        CGC_CUDA(cudaMemcpyAsync(stage, a, m * 4, cudaMemcpyHostToDevice, g->stream));
        CGC_CUDA(cudaMemcpyAsync(stage + m, b, m * 4, cudaMemcpyHostToDevice, g->stream));
        CGC_CUDA(cudaMemcpyAsync(stage + 2 * m, cab, m * 4, cudaMemcpyHostToDevice, g->stream));
        CGC_CUDA(cudaMemcpyAsync(stage + 3 * m, cba, m * 4, cudaMemcpyHostToDevice, g->stream));
        int32_t* deg = d.reach;   // scratch until the first solve
        int32_t* cur = (int32_t*)d.stamp;
        const int eb = grid_blocks(m, 256);
        k_csr_degree<<<eb, 256, 0, g->stream>>>(m, stage, stage + m, deg); note_launch();
        k_scan_block<<<nb, SCAN_BLOCK, 0, g->stream>>>(deg, (int32_t*)d.row, bsum, n); note_launch();
        k_scan_sums<<<1, SCAN_BLOCK, 0, g->stream>>>(bsum, nb, (int32_t*)d.row + n); note_launch();
        k_scan_add<<<grid_blocks(n, 256), 256, 0, g->stream>>>((int32_t*)d.row, bsum, n); note_launch();
        k_csr_scatter<<<eb, 256, 0, g->stream>>>(m, stage, stage + m, stage + 2 * m, stage + 3 * m, d.row, cur,
                                                 (int32_t*)d.to, (int32_t*)d.rev, (int32_t*)d.res0); note_launch();
        CGC_CUDA(cudaGetLastError());
        CGC_CUDA(cudaMemsetAsync(deg, 0, (size_t)n * 4, g->stream));
        CGC_CUDA(cudaMemsetAsync(cur, 0, (size_t)n * 4, g->stream));
        CGC_CUDA(cudaStreamSynchronize(g->stream));
        return CGC_OK;
      }();
      cudaFree(stage);
      if (rc2) return rc2;
    }
    cudaDeviceProp prop;
    CGC_CUDA(cudaGetDeviceProperties(&prop, g->device));
    int occ = 0;
    CGC_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, k_csr_solve, CSR_THREADS, 0));
    // enough CTAs to cover the vertices, at most the co-resident count
    const int want = grid_blocks(n, CSR_THREADS);
    g->coop_blocks = std::max(1, std::min(std::max(1, occ) * prop.multiProcessorCount, want));
    CGC_CUDA(cudaStreamSynchronize(g->stream));
    return CGC_OK;
  }();
  if (rc) {
    graph_free(g);
    return rc;
  }
  *out = g;
  return ok();
}

int graph_maxflow(cgc_graph* g, const cgc_options* opts, int64_t* flow) {
  using namespace cgc;
  if (!g) return fail(CGC_ERR_ARG, "cgc_graph_maxflow: null graph");
  if (!g->tlinks) return fail(CGC_ERR_STATE, "cgc_graph_maxflow: set the terminal capacities first");
  const cgc_options o = resolve_options(opts);
  CsrParams prm;
  prm.K = std::max(1, 2 * o.sweeps_per_relabel);
  prm.max_pulses = (int64_t)o.max_sweeps;
  prm.limit_ns = wait_limit_ns(o);
  const long long launches0 = g_launches.load();
  CsrDev& d = g->d;
  cudaEvent_t ev[4] = {};
  for (auto& e : ev) CGC_CUDA(cudaEventCreate(&e));
  auto destroy = [&]() {
    for (auto& e : ev)
      if (e) cudaEventDestroy(e);
  };
  int rc = [&]() -> int {
    CGC_CUDA(cudaEventRecord(ev[0], g->stream));
    CGC_CUDA(cudaMemsetAsync(d.flow, 0, 8, g->stream));
    CGC_CUDA(cudaMemsetAsync(d.stats, 0, CS_N * 8, g->stream));
    CGC_CUDA(cudaMemsetAsync(d.err, 0, 4, g->stream));
    CGC_CUDA(cudaMemsetAsync(d.bar, 0, 8, g->stream));
    CGC_CUDA(cudaMemsetAsync(d.cnt, 0, CC_N * 4, g->stream));
    k_csr_prepare<<<grid_blocks(std::max<int64_t>(d.arcs, d.n), 256), 256, 0, g->stream>>>(d); note_launch();
    CGC_CUDA(cudaGetLastError());
    CGC_CUDA(cudaEventRecord(ev[1], g->stream));
    cudaLaunchConfig_t cfg = {};
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeCooperative;
    attr[0].val.cooperative = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    cfg.stream = g->stream;
    cfg.gridDim = dim3(g->coop_blocks);
    cfg.blockDim = dim3(CSR_THREADS);
    if (int rc2 = coop_launch_ordered(g->device, g->stream, [&]() -> int {
          CGC_CUDA(cudaLaunchKernelEx(&cfg, k_csr_solve, d, prm));
          return CGC_OK;
        }))
      return rc2;
    note_launch();
    CGC_CUDA(cudaEventRecord(ev[2], g->stream));
    CGC_CUDA(cudaEventRecord(ev[3], g->stream));
    CGC_CUDA(cudaEventSynchronize(ev[3]));
    int32_t err = 0;
    CGC_CUDA(cudaMemcpy(&err, d.err, 4, cudaMemcpyDeviceToHost));
    if (err == CGC_ERR_TIMEOUT) return fail(CGC_ERR_TIMEOUT, "cgc_graph_maxflow: a grid barrier timed out");
    if (err == CGC_ERR_NOT_CONVERGED) return fail(CGC_ERR_NOT_CONVERGED, "cgc_graph_maxflow: pulse cap reached");
    if (err == CGC_ERR_OVERFLOW)
      return fail(CGC_ERR_OVERFLOW, "cgc_graph_maxflow: capacities may overflow int32 excess or residuals");
    if (err) return fail(err, "cgc_graph_maxflow: device error");
    unsigned long long f = 0, stats[CS_N];
    CGC_CUDA(cudaMemcpy(&f, d.flow, 8, cudaMemcpyDeviceToHost));
    CGC_CUDA(cudaMemcpy(stats, d.stats, sizeof(stats), cudaMemcpyDeviceToHost));
    float ms = 0.f, kms = 0.f;
    cudaEventElapsedTime(&ms, ev[0], ev[3]);
    cudaEventElapsedTime(&kms, ev[1], ev[2]);
    std::memset(&g->st, 0, sizeof(g->st));
    g->st.flow = (int64_t)f;
    g->st.sweeps = (int64_t)stats[CS_PULSES];
    g->st.global_relabels = (int64_t)stats[CS_RELABELS];
    g->st.bfs_rounds = (int64_t)stats[CS_LEVELS];
    g->st.pulses = (int64_t)stats[CS_PULSES];
    g->st.solve_ms = ms;
    g->st.kernel_ms = kms;
    g->st.launches = g_launches.load() - launches0;
    g->st.bfs_ms = 1e-6 * (double)stats[CS_NS_BFS];
    g->st.sweep_ms = 1e-6 * (double)stats[CS_NS_PUSH];
    g->st.reach_ms = 1e-6 * (double)stats[CS_NS_REACH];
    if (flow) *flow = (int64_t)f;
    g->solved = true;
    return CGC_OK;
  }();
  destroy();
  return rc ? rc : ok();
}

}  // namespace

extern "C" {

int cgc_graph_create(int32_t n, int64_t m, const int32_t* a, const int32_t* b, const int32_t* cap_ab,
                     const int32_t* cap_ba, void* stream, cgc_graph** out) {
  return graph_create(n, m, a, b, cap_ab, cap_ba, stream, out);
}

int cgc_graph_destroy(cgc_graph* g) {
  if (!g) return cgc::fail(CGC_ERR_ARG, "cgc_graph_destroy: null graph");
  graph_free(g);
  return cgc::ok();
}

int cgc_graph_set_tlinks(cgc_graph* g, const int32_t* capS, const int32_t* capT) {
  if (!g || !capS || !capT) return cgc::fail(CGC_ERR_ARG, "cgc_graph_set_tlinks: bad arguments");
  for (int32_t v = 0; v < g->n; ++v)
    if (capS[v] < 0 || capT[v] < 0)
      return cgc::fail(CGC_ERR_ARG, "cgc_graph_set_tlinks: negative capacity at vertex " + std::to_string(v));
  CGC_CUDA(cudaMemcpyAsync((void*)g->d.capS, capS, (size_t)g->n * 4, cudaMemcpyHostToDevice, g->stream));
  CGC_CUDA(cudaMemcpyAsync((void*)g->d.capT, capT, (size_t)g->n * 4, cudaMemcpyHostToDevice, g->stream));
  CGC_CUDA(cudaStreamSynchronize(g->stream));
  g->tlinks = true;
  return cgc::ok();
}

int cgc_graph_maxflow(cgc_graph* g, const cgc_options* opts, int64_t* flow) { return graph_maxflow(g, opts, flow); }

int cgc_graph_get_segments(cgc_graph* g, int which, uint8_t* out, uint8_t mask, uint8_t background) {
  if (!g || !out || (which != CGC_SEG_SINK_REACH && which != CGC_SEG_SOURCE_MIN))
    return cgc::fail(CGC_ERR_ARG, "cgc_graph_get_segments: bad arguments");
  if (!g->solved) return cgc::fail(CGC_ERR_STATE, "cgc_graph_get_segments: call maxflow first");
  cgc::k_csr_segments<<<cgc::grid_blocks(g->n, 256), 256, 0, g->stream>>>(g->d, which, g->seg, mask, background);
  cgc::note_launch();
  CGC_CUDA(cudaGetLastError());
  CGC_CUDA(cudaMemcpyAsync(out, g->seg, (size_t)g->n, cudaMemcpyDeviceToHost, g->stream));
  CGC_CUDA(cudaStreamSynchronize(g->stream));
  return cgc::ok();
}

int cgc_graph_get_state(cgc_graph* g, int32_t* labels, int32_t* excess) {
  if (!g) return cgc::fail(CGC_ERR_ARG, "cgc_graph_get_state: null graph");
  if (!g->solved) return cgc::fail(CGC_ERR_STATE, "cgc_graph_get_state: call maxflow first");
  if (labels) CGC_CUDA(cudaMemcpyAsync(labels, g->d.h, (size_t)g->n * 4, cudaMemcpyDeviceToHost, g->stream));
  if (excess) CGC_CUDA(cudaMemcpyAsync(excess, g->d.e, (size_t)g->n * 4, cudaMemcpyDeviceToHost, g->stream));
  CGC_CUDA(cudaStreamSynchronize(g->stream));
  if (labels)
    for (int32_t v = 0; v < g->n; ++v)
      if (labels[v] >= cgc::INF) labels[v] = INT32_MIN;
  return cgc::ok();
}

int cgc_graph_stats(cgc_graph* g, cgc_stats* st) {
  if (!g || !st) return cgc::fail(CGC_ERR_ARG, "cgc_graph_stats: bad arguments");
  *st = g->st;
  return cgc::ok();
}

}  // extern "C"
