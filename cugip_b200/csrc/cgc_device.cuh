// Device-side data structures and tile routines of the grid push-relabel engine.
//
// HBM layout.  Every instance is padded to whole 8x8x8 tiles; all instances of
// a pool share one tile index space.  Each per-voxel quantity is a plane of
// T*512 entries in tile-major ("blocked") order: voxel (x,y,z) of tile t sits
// at t*512 + (x&7) + 8*(y&7) + 64*(z&7), so one tile of one plane is a
// contiguous 2 KB run (fully coalesced, one 128-byte line per warp-row).
//   e      int32  excess
//   h      int32  height (distance label); INF = unreachable from the sink side
//   rT     int32  residual of the sink t-link
//   r[d]   int32  residual of the n-link to the neighbour in direction d
//                 (d = +x,-x,+y,-y,+z,-z; 0 where the neighbour is outside)
//   rmask  uint8  bit d: r[d] > 0, bit 6: rT > 0 (the BFS reads 1 byte, not 28)
//   reach  uint8  source-side reachability (canonical cut)
// Padding voxels have zero capacities everywhere and never become active.
//
// The residual graph of the reference is a CSR edge list with one residual
// pair per undirected edge (include/cugip/advanced_operations/detail/edge_record.hpp:36-57,
// graph_cut.hpp:239-290); on a grid the neighbours are implicit, so the
// engine keeps one out-residual plane per direction instead.
#pragma once
#include <cstdint>
#include <cuda_bf16.h>

namespace cgc {

constexpr int TILE = 8;
constexpr int TV = 512;            // voxels per tile
constexpr int INF = 0x3fffffff;    // height of vertices that cannot reach the sink
constexpr int HALO = 1000;         // 10x10x10 heights with a one-voxel halo

enum Dir { PX = 0, MX = 1, PY = 2, MY = 3, PZ = 4, MZ = 5 };

// counters in DevPool::cnt
enum Counter {
  C_BFS0 = 0,      // 3 BFS worklists
  C_SW0 = 3,       // 4 sweep worklists
  C_ACT = 7,       // active tiles after the last global relabel
  C_ROUNDS = 8,    // BFS rounds executed
  C_SINKT0 = 9,    // 3 slots: tiles that delivered flow to the sink in a sweep
  C_TAKE0 = 12,    // 3 slots: next list entry to hand out in a round (persistent solve)
  C_INC = 15,      // incremental relabel: tiles with dropped voxels (the BFS rounds' first list)
  C_NCOUNTERS = 16
};

// statistics in DevPool::stats (unsigned long long)
enum Stat {
  S_TILES_SWEPT = 0, S_PULSES = 1, S_TILES_BFS = 2, S_SWEEPS = 3, S_RELABELS = 4, S_ROUNDS = 5,
  S_NS_BFS = 6, S_NS_SWEEP = 7, S_NS_REACH = 8, S_TRACE_N = 9, S_TRACE_CYC = 10, S_NS_SCHED = 11,
  S_BOUND_AT = 12 /* bounds-checked build: the first index found out of range */,
  S_TILES_CHECK = 13 /* tile visits of the incremental relabels' invalidation passes */, S_NSTATS = 14
};

// phase trace records written by the persistent solve (two words each):
//   word 0 = kind << 56 | index << 24 | tiles, word 1 = ns since the launch
//   (TR_FLOW: word 1 = the flow delivered so far, all instances together)
enum TraceKind { TR_BFS_ROUND = 1, TR_RELABEL_DONE = 2, TR_SWEEP = 3, TR_REACH_ROUND = 4, TR_FLOW = 5 };
constexpr int TRACE_CAP = 16384;

// BFS seed summary of a tile (DevPool::tflag)
enum TileFlag {
  TF_ALL_SEED = 1, TF_FACE0 = 2 /* bits 1..6: a seed on face d */, TF_HAS_SEED = 128,
  TF_DEAD = 256 /* every voxel cannot reach the sink: stays so for the rest of the solve */
};

struct InstGeo {
  int32_t X, Y, Z;      // voxel extents
  int32_t TX, TY, TZ;   // tile extents
  int32_t tile_base;    // first tile of the instance
  int32_t hdead;        // heights >= hdead cannot reach the sink (voxel count + 1)
};

struct DevPool {
  int32_t T;            // tiles
  int32_t ninst;
  int64_t Np;           // T*512
  int32_t* e;
  int32_t* h;
  int32_t* rT;
  int32_t* r;           // 6 planes: r + d*Np
  uint8_t* rmask;
  uint8_t* reach;
  const int32_t* nbr;   // 6*T: neighbour tile in direction d, -1 outside
  const int32_t* tinst; // T: instance of the tile
  const uint8_t* tpar;  // T: (tx+ty+tz)&1
  uint8_t* act;         // T: tile holds an active voxel (e>0, h<INF)
  uint16_t* tflag;      // T: BFS seed summary (TF_* bits)
  uint32_t* stamp_bfs;  // T: last BFS round the tile was queued for
  uint32_t* stamp_sw;   // 2*T: last sweep the tile was queued for (exclusive sweeps: half s&1 for sweep s)
  uint32_t* stamp_inc;  // T: last incremental relabel that listed the tile for its BFS rounds (may be null:
                        //    then every relabel is a full BFS)
  int32_t* lists;       // 7*T worklists: 3 for the BFS, 4 for the sweeps
  int32_t* cnt;         // C_NCOUNTERS
  unsigned long long* flow;   // ninst: flow value (int64 as two's complement)
  const InstGeo* geo;   // ninst
  unsigned long long* stats;  // S_NSTATS
  int32_t* err;         // first error code raised on the device
  uint32_t* bar;        // grid barrier: [0] arrivals, [1] generation
  unsigned long long* trace;  // 2*TRACE_CAP words of phase records (may be null)
  // learned scheduler (null unless used)
  __nv_bfloat16* sfeat;       // T*16 tile features
  __nv_bfloat16* sact0;       // T*16 activations of conv 1
  __nv_bfloat16* sact1;       // T*16 activations of conv 2
  const uint2* swfrag;        // 3 layers of convolution weights in mma fragment order (cgc_sched.cuh)
  const float* swhead;        // 2*16 weights + 2 biases
  uint8_t* sbudget;           // T: pulses per visit until the next relabel
  uint8_t* sprio;             // T: 1 = high priority
  // scheduling traces for training (null unless recorded)
  __nv_bfloat16* tfeat;       // cycles*T*16 features at the start of each relabel cycle
  uint8_t* tpulses;           // cycles*T: pulses of the tile's first visit in the cycle (0 = not visited)
  uint8_t* tsink;             // cycles*T: 1 if the tile delivered flow to the sink during the cycle
};

// parameters of the persistent solve kernel
struct SolveParams {
  int L;                 // pulses per tile visit (per region-relabel round)
  int R;                 // region-relabel rounds per tile visit (0: pulses only)
  int K;                 // sweep pairs between global relabels
  int stall;             // relabel after this many sweeps without sink flow (0: never)
  int learned;           // 1: budgets and priorities from the learned scheduler
  int trace_cycles;      // record scheduling traces for the first trace_cycles relabel cycles
  int64_t max_sweeps;    // cap on sweeps (parity steps)
  uint64_t limit_ns;     // bounded barrier wait
  int bfs_warp_min = 0;  // BFS rounds with at least this many tiles per CTA run a warp per tile (0: never)
  int exclusive = 0;     // 1: exclusive sweeps (cgc_options.exclusive), 0: parity sweeps
  int incremental = 0;   // 1: global relabels after the first of a solve are incremental (cgc_options.relabel)
};

// kernels of cgc_engine.cu launched from other translation units
__global__ void k_put_tlinks(DevPool P, int inst, const int32_t* __restrict__ capS, const int32_t* __restrict__ capT);
__global__ void k_put_nlinks(DevPool P, int inst, int axis, const int32_t* __restrict__ fwd,
                             const int32_t* __restrict__ bwd);
__global__ void k_prepare(DevPool P);
__global__ void k_solve(DevPool P, SolveParams prm);
__global__ void k_solve3(DevPool P, SolveParams prm);
__global__ void k_solve4(DevPool P, SolveParams prm);
__global__ void k_solve3w(DevPool P, SolveParams prm);
__global__ void k_solve4w(DevPool P, SolveParams prm);
__global__ void k_segments(DevPool P, int inst, int which, uint8_t* out, uint8_t mask, uint8_t bg);
// kernels of cgc_batch.cu
__global__ void k_put_all(DevPool P, const int32_t* const* __restrict__ in);
__global__ void k_seg_all(DevPool P, uint8_t* const* __restrict__ out);

}  // namespace cgc
