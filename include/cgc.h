/*
 * cgc.h — C ABI of the B200 grid graph-cut (max-flow / min-cut) engine.
 *
 * Plain pointers and sizes only; every entry point returns an int status
 * (CGC_OK == 0).  The message of the last failure on the calling thread is
 * returned by cgc_last_error().
 *
 * Each entry point names the interface of cugip's graph-cut path that it
 * replaces (paths relative to the cugip source tree).
 *
 * Graph model (identical to cugip::Graph<TFlow>):
 *   - one vertex per voxel, vertex id = x + X*(y + Y*z) (x fastest);
 *   - a t-link from the source with capacity capS[v] and one to the sink
 *     with capacity capT[v]  (include/cugip/advanced_operations/graph_cut.hpp:64-67);
 *   - an n-link between each pair of 6-neighbours with a forward capacity
 *     (lower id -> higher id) and a backward capacity (higher -> lower),
 *     the EdgeRecord(min,max) + fwd/bwd convention of
 *     include/cugip/advanced_operations/graph_cut.hpp:57-62 and
 *     include/cugip/advanced_operations/detail/edge_record.hpp:12-17.
 * Capacities are int32 >= 0; the flow value is returned as int64 and is exact.
 */
#ifndef CGC_H
#define CGC_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- status codes ------------------------------------------------------ */
enum {
  CGC_OK = 0,
  CGC_ERR_ARG = 1,           /* bad argument (null pointer, bad extent, bad axis) */
  CGC_ERR_OOM = 2,           /* device or host allocation failed                  */
  CGC_ERR_CUDA = 3,          /* a CUDA runtime call failed                         */
  CGC_ERR_TIMEOUT = 4,       /* a bounded device-side wait gave up                 */
  CGC_ERR_NOT_CONVERGED = 5, /* max_sweeps reached before the max flow was proven  */
  CGC_ERR_OVERFLOW = 6,      /* capacities could overflow the int32 residual/excess range */
  CGC_ERR_STATE = 7,         /* call out of order (e.g. segments before max_flow)  */
  CGC_ERR_NOT_GRID = 8,      /* edge list is not a 6-connected grid                */
  CGC_ERR_NO_DEVICE = 9      /* no CUDA device                                     */
};

/* axes for cgc_grid_set_nlinks */
enum { CGC_AXIS_X = 0, CGC_AXIS_Y = 1, CGC_AXIS_Z = 2 };

/* which labelling cgc_grid_get_segments returns */
enum {
  /* vertices that can reach the sink in the final residual graph: the set
     cugip marks with label in [0, n] (graph_cut.hpp:304-333) and the set
     Boykov-Kolmogorov's what_segment()==SINK returns
     (benchmarks/graph_cut/boykov_kolmogorov.cpp:81) */
  CGC_SEG_SINK_REACH = 0,
  /* vertices reachable from the source in the final residual graph: the
     minimal source side of the minimum cut (the canonical cut) */
  CGC_SEG_SOURCE_MIN = 1
};

/* Solver options; zero-initialise and set struct_size = sizeof(cgc_options).
   A zero field means "use the default".  Replaces the compile-time policies
   GraphCutPolicy / RelabelPolicy / PushPolicy
   (include/cugip/advanced_operations/detail/graph_cut_policies.hpp:23-89). */
typedef struct cgc_options {
  int32_t struct_size;
  int32_t local_pulses;       /* push/relabel pulses per region-relabel round (1..64), default 4 */
  int32_t sweeps_per_relabel; /* sweep pairs between global relabels, default 8 */
  int32_t wait_limit_us;      /* bound of every device-side wait (grid barriers of the persistent
                                 solve), in microseconds; default 20 s.  A wait that runs out ends
                                 the solve with CGC_ERR_TIMEOUT; the handle stays usable */
  int32_t max_sweeps;         /* safety cap on sweeps, default 1<<17; CGC_ERR_NOT_CONVERGED when reached */
  int32_t persistent;         /* 1 = one cooperative launch per solve (default), -1 = host loop */
  int32_t region_relabels;    /* region-relabel rounds per tile visit (default 2, -1 = none) */
  int32_t stall_sweeps;       /* persistent: relabel early after this many sweep pairs without sink flow (0 = never) */
  int32_t ctas_per_sm;        /* persistent: 2 (default, 64 registers), 3 (40) or 4 (32 registers) */
  int32_t learned;            /* persistent: learned scheduler, 1 = budgets + priorities, 2 = budgets only
                                 (both only in cycles with more active tiles than twice the CTAs), 3 = budgets
                                 capped at local_pulses in every cycle + priorities where 1 uses them */
  int32_t trace_cycles;       /* persistent: record scheduling traces of the first trace_cycles relabel cycles */
  int32_t bfs_warp_min;       /* persistent, 3 or 4 CTAs/SM: BFS rounds with at least this many tiles per CTA
                                 visit a tile with one warp (0 = never, the default) */
  int32_t exclusive;          /* persistent: 1 = every sweep visits each queued tile, except a tile that has a
                                 face neighbour of the sweep's parity queued for the same sweep (which waits one
                                 sweep); 0 = checkerboard sweeps, one parity at a time (the default) */
  int32_t relabel;            /* persistent: global relabels after the first of a solve, 1 = full BFS from the
                                 sink, 2 = incremental (re-checks the tiles the last sweep cycle queued and
                                 recomputes only the labels it invalidated; the labels equal the full BFS's);
                                 0 = the default (2) */
  int32_t reserved[2];
} cgc_options;

/* Per-solve statistics (filled by cgc_grid_stats). */
typedef struct cgc_stats {
  int64_t flow;
  int64_t sweeps;            /* parity sweeps executed */
  int64_t global_relabels;   /* exact BFS relabels executed */
  int64_t bfs_rounds;        /* tile rounds over all BFS passes */
  int64_t tiles_swept;       /* tile visits by the push sweep */
  int64_t tiles_relabelled;  /* tile visits by the BFS */
  int64_t pulses;            /* total local pulses executed over all tile visits */
  double  solve_ms;          /* device time of the last maxflow (upload, preflow, solve and both cut sets) */
  double  kernel_ms;         /* device time of the solve kernel(s) alone */
  int64_t launches;          /* kernels launched by the last maxflow */
  double  bfs_ms;            /* persistent solve: time in exact global relabels */
  double  sweep_ms;          /* persistent solve: time in push sweeps */
  double  reach_ms;          /* persistent solve: time in the source-side reachability */
  double  sched_ms;          /* persistent solve: time in the learned scheduler (features + CNN) */
  int64_t tiles_checked;     /* tile visits of the incremental relabels' invalidation passes */
  int64_t reserved[1];
} cgc_stats;

/* Kernels launched by this library on the calling process since load
 * (uploads, solve, outputs): for launch accounting in benchmarks. */
int64_t cgc_launch_count(void);

typedef struct cgc_grid cgc_grid;

/* ---- library ------------------------------------------------------------ */
const char* cgc_last_error(void);
const char* cgc_version(void);
/* Initialises the CUDA device and returns CGC_ERR_NO_DEVICE without one. */
int cgc_init(int device);

/* ---- single grid ---------------------------------------------------------
 * Replaces cugip::Graph<TFlow>::set_vertex_count
 * (include/cugip/advanced_operations/graph_cut.hpp:213-237): allocates all
 * device state for an X*Y*Z grid (about 40 bytes per voxel, padded to 8^3
 * tiles).  stream may be NULL (legacy default stream). */
int cgc_grid_create(int32_t X, int32_t Y, int32_t Z, void* stream, cgc_grid** out);
int cgc_grid_destroy(cgc_grid* g);

/* Replaces Graph::set_tweights (graph_cut.hpp:292-302).  Host arrays of X*Y*Z
 * int32 >= 0, copied to the device before the call returns. */
int cgc_grid_set_tlinks(cgc_grid* g, const int32_t* capS, const int32_t* capT);

/* Replaces Graph::set_nweights (graph_cut.hpp:239-290) for a grid: the n-links
 * along one axis.  fwd[v] is the capacity v -> v+e_axis, bwd[v] the capacity
 * v+e_axis -> v; entries on the last slice of the axis are ignored.  When
 * fwd == bwd (symmetric weights) the plane is copied once. Host arrays. */
int cgc_grid_set_nlinks(cgc_grid* g, int axis, const int32_t* fwd, const int32_t* bwd);

/* Edge-list front door, replacing Graph::set_vertex_count + set_nweights
 * (graph_cut.hpp:213-290) for callers that build EdgeRecord lists: edge i
 * joins vertices a[i] and b[i] with capacity fwd[i] from a[i] to b[i] and
 * bwd[i] from b[i] to a[i] (for EdgeRecord(first,second), pass first/second).
 * The edges must form a 6-connected X*Y*Z grid with linear ids (x fastest);
 * the extents are recovered from the id strides, written to dims_out (may be
 * NULL) and the n-links are uploaded.  Parallel edges add up.  Returns
 * CGC_ERR_NOT_GRID for any other graph. */
int cgc_detect_grid(int32_t n, int64_t m, const uint32_t* a, const uint32_t* b, int32_t* dims);
int cgc_grid_create_from_edges(int32_t n, int64_t m, const uint32_t* a, const uint32_t* b,
                               const int32_t* fwd, const int32_t* bwd, void* stream, cgc_grid** out,
                               int32_t* dims_out);

/* ---- generic graphs ----------------------------------------------------------
 * Any edge list (the non-grid path of Graph::set_vertex_count / set_nweights /
 * set_tweights / max_flow / fill_segments, graph_cut.hpp:213-333): n vertices,
 * edge i joins a[i] and b[i] with capacity cap_ab[i] from a[i] to b[i] and
 * cap_ba[i] back (EdgeRecord(first, second) with the forward and backward
 * weights).  Self loops are ignored, parallel edges are separate arcs.  The
 * residual graph is built on the device (CSR); arrays are host memory and are
 * copied.  The options' sweeps_per_relabel sets the pulses between exact
 * relabels (2x) and max_sweeps caps the pulses.  Cut semantics as for grids. */
typedef struct cgc_graph cgc_graph;
int cgc_graph_create(int32_t n, int64_t m, const int32_t* a, const int32_t* b, const int32_t* cap_ab,
                     const int32_t* cap_ba, void* stream, cgc_graph** out);
int cgc_graph_destroy(cgc_graph* g);
int cgc_graph_set_tlinks(cgc_graph* g, const int32_t* capS, const int32_t* capT);
int cgc_graph_maxflow(cgc_graph* g, const cgc_options* opts, int64_t* flow);
int cgc_graph_get_segments(cgc_graph* g, int which, uint8_t* out, uint8_t mask, uint8_t background);
int cgc_graph_stats(cgc_graph* g, cgc_stats* stats);
/* Final distance labels (INT32_MIN where the sink cannot be reached) and
 * excess per vertex of the last solve (host arrays of n, either may be NULL). */
int cgc_graph_get_state(cgc_graph* g, int32_t* labels, int32_t* excess);

/* Same as the two setters above with device pointers (no host copies). */
int cgc_grid_set_tlinks_device(cgc_grid* g, const int32_t* capS, const int32_t* capT);
int cgc_grid_set_nlinks_device(cgc_grid* g, int axis, const int32_t* fwd, const int32_t* bwd);

/* Replaces Graph::max_flow / max_flow(policy)
 * (graph_cut.hpp:69-100 -> MinimalGraphCutComputation::run,
 * detail/graph_cut_implementation.hpp:286-308).  Runs push-relabel to the
 * exact maximum flow; *flow receives the int64 flow value.  opts may be NULL.
 * Blocks until done.  Unlike the reference, the graph may be solved again
 * after new set_* calls. */
int cgc_grid_maxflow(cgc_grid* g, const cgc_options* opts, int64_t* flow);

/* The same solve in two halves, for callers that overlap the host uploads of
 * one grid with the solve of another (no counterpart in the reference, whose
 * max_flow blocks, graph_cut.hpp:69-100).  cgc_grid_maxflow_async queues the
 * solve of the capacities set so far (fused upload and preflow, the solve and
 * both cut sets) on the grid's stream and returns without waiting; errors
 * found on the device are reported by cgc_grid_wait, which blocks until the
 * solve is done and writes the flow (may be NULL).  Between the two calls the
 * grid's set_* calls may already copy the next inputs (they wait until the
 * queued solve has read the previous ones), while the calls that read results
 * or solve (maxflow, get_segments, get_residuals, autotune) return
 * CGC_ERR_STATE.  To overlap two grids, give each its own stream. */
int cgc_grid_maxflow_async(cgc_grid* g, const cgc_options* opts);
int cgc_grid_wait(cgc_grid* g, int64_t* flow);

/* Replaces Graph::fill_segments (graph_cut.hpp:318-333): out[v] = mask if v is
 * in the chosen set (CGC_SEG_*), else background.  Host array of X*Y*Z. */
int cgc_grid_get_segments(cgc_grid* g, int which, uint8_t* out, uint8_t mask, uint8_t background);
/* Same into device memory. */
int cgc_grid_get_segments_device(cgc_grid* g, int which, uint8_t* out, uint8_t mask, uint8_t background);

/* Final residual capacities (host arrays of X*Y*Z each, linear layout):
 * res[d] for d = +x,-x,+y,-y,+z,-z (entries that leave the grid are 0), the
 * sink t-link residual resT and the excess left at each voxel.  For
 * certificates and tests; any pointer may be NULL. */
int cgc_grid_get_residuals(cgc_grid* g, int32_t* const res[6], int32_t* resT, int32_t* excess);

/* Distance labels of the last solve (host array of X*Y*Z, linear layout): the
 * exact distance to the sink found by the final global relabel, INT32_MIN
 * (the reference's INVALID_LABEL, detail/graph_cut_policies.hpp:34) where the
 * sink cannot be reached.  For trace objects and tests. */
int cgc_grid_get_labels(cgc_grid* g, int32_t* labels);

int cgc_grid_stats(cgc_grid* g, cgc_stats* out);

/* Phase trace of the last persistent solve (extends the reference's trace
 * hooks, graph_cut.hpp:26-45, with per-step detail): *count receives the
 * number of records; up to `cap` records of two int64 each are copied to out:
 * word 0 = kind << 56 | index << 24 | tiles (kind 1 = BFS round, 2 = global
 * relabel done (tiles = active tiles), 3 = sweep, 4 = reachability round,
 * 5 = flow at global relabel `index`), word 1 = nanoseconds since the launch
 * (kind 5: the exact flow delivered so far). */
int cgc_grid_trace(cgc_grid* g, int64_t* out, int32_t cap, int32_t* count);

/* ---- allocation-free solve of a small grid ---------------------------------
 * No counterpart in the reference.  For callers that may not allocate device
 * memory: processes whose device memory belongs to another allocator (a
 * framework's caching pool or a fixed budget) and real-time loops that cannot
 * take the device-wide synchronisation of cudaMalloc / cudaFree.  The caller
 * passes device inputs (capS, capT and the fwd/bwd n-link planes of each axis
 * as in cgc_grid_set_nlinks; a NULL axis means zero capacity) and device
 * outputs (source_side / sink_side: X*Y*Z bytes of 1/0, each may be NULL); the
 * flow is written to the host int64 *flow and the call blocks until done.
 * All working state lives in one static device array that every GPU loading
 * this library holds until exit, so the grid may hold at most
 * CGC_NOALLOC_MAX_VOXELS voxels after rounding each extent up to a multiple of
 * 8 (64^3 fits); larger grids return CGC_ERR_ARG.  The first call on a device
 * sets that device up and should come before any stream capture: it looks up
 * the array's device address, which is then kept for the life of the process,
 * so resetting the device (cudaDeviceReset) after that first call is not
 * supported.  Every call blocks the calling thread: it waits for `stream` and
 * reads the flow and the device status back into host memory before it
 * returns.  Calls share the array: calls that overlap on the GPU race and must
 * not be issued, and a call should not overlap another solve of this library
 * on another stream (both are grid-wide cooperative launches). */
#define CGC_NOALLOC_MAX_VOXELS 262144
int cgc_grid_maxflow_noalloc(int32_t X, int32_t Y, int32_t Z, const int32_t* capS, const int32_t* capT,
                             const int32_t* const fwd[3], const int32_t* const bwd[3],
                             const cgc_options* opts, void* stream, int64_t* flow,
                             uint8_t* source_side, uint8_t* sink_side);

/* ---- batch of grids (uneven sizes, one solve) ----------------------------
 * Replaces nothing in the reference (it solves one graph per Graph object);
 * all instances share one tile pool and are solved by the same launches. */
typedef struct cgc_batch cgc_batch;
int cgc_batch_create(int32_t count, const int32_t* extents /* 3*count: X,Y,Z */, void* stream, cgc_batch** out);
int cgc_batch_destroy(cgc_batch* b);
int cgc_batch_set_tlinks(cgc_batch* b, int32_t i, const int32_t* capS, const int32_t* capT);
int cgc_batch_set_nlinks(cgc_batch* b, int32_t i, int axis, const int32_t* fwd, const int32_t* bwd);
int cgc_batch_maxflow(cgc_batch* b, const cgc_options* opts, int64_t* flows /* count */);
int cgc_batch_get_segments(cgc_batch* b, int32_t i, int which, uint8_t* out, uint8_t mask, uint8_t background);
int cgc_batch_stats(cgc_batch* b, cgc_stats* out);

/* Device-resident batches (no counterpart in the reference).  Bind each
 * instance's device inputs once (capS, capT and the per-axis fwd/bwd n-link
 * planes as in cgc_grid_set_nlinks; bwd may be NULL for symmetric n-links, a
 * NULL axis is zero) and optional device outputs (X*Y*Z bytes of 1/0 for the
 * minimal source side and the sink-reachable side).  The pointers are read
 * again by every later solve, so new capacities are picked up by writing into
 * the same buffers.  cgc_batch_enqueue queues one solve of every instance on
 * the batch's stream without synchronising the host (flows_dev: device int64
 * per instance, may be NULL); cgc_batch_graph_create captures that sequence
 * once into a CUDA graph and cgc_batch_graph_launch replays it.
 * cgc_batch_wait synchronises, returns the device status and copies the flows
 * to the host (flows may be NULL). */
int cgc_batch_bind_inputs(cgc_batch* b, int32_t i, const int32_t* capS, const int32_t* capT,
                          const int32_t* const fwd[3], const int32_t* const bwd[3]);
int cgc_batch_bind_outputs(cgc_batch* b, int32_t i, uint8_t* source_side, uint8_t* sink_side);
int cgc_batch_enqueue(cgc_batch* b, const cgc_options* opts, int64_t* flows_dev);
int cgc_batch_graph_create(cgc_batch* b, const cgc_options* opts, int64_t* flows_dev);
int cgc_batch_graph_launch(cgc_batch* b);
int cgc_batch_wait(cgc_batch* b, int64_t* flows);

/* Autotuner (replaces the compile-time policies of
 * detail/graph_cut_policies.hpp:23-89 with measured choices).  Times each
 * candidate option set (n == 0: a built-in grid over local_pulses,
 * region_relabels, sweeps_per_relabel and ctas_per_sm) `repeats` times on the
 * grid's or batch's current capacities (set with the set_* calls, or bound
 * device inputs), writes the fastest to *best (and its time in ms to
 * *best_ms, either may be NULL) and caches it for the size class; the
 * capacities are restored, so maxflow can follow directly.  With the
 * environment variable CGC_AUTOTUNE_CACHE naming a file, results are appended
 * to it and read back by cgc_autotune_lookup in later processes. */
int cgc_grid_autotune(cgc_grid* g, const cgc_options* candidates, int32_t n, int32_t repeats,
                      cgc_options* best, double* best_ms);
int cgc_batch_autotune(cgc_batch* b, const cgc_options* candidates, int32_t n, int32_t repeats,
                       cgc_options* best, double* best_ms);
/* Cached options for a size class (total voxels, instance count); CGC_ERR_STATE if none. */
int cgc_autotune_lookup(int64_t voxels, int32_t instances, cgc_options* out);

/* ---- learned tile scheduler (no counterpart in the reference) -------------
 * After every exact global relabel a small CNN over the tile grid (BF16
 * weights and activations, FP32 accumulation; three 3x3x3 convolutions with
 * 16 channels, then a linear head) reads per-tile features (log2 excess sum,
 * active voxel count, 8-bin height histogram) and sets each tile's pulse
 * budget (1..32) and priority; cgc_options.learned = 1 turns it on.  It only
 * reorders pushes and relabels, so flows and cuts equal the plain solver's.
 * Weights: 3*27*16*16 BF16 convolution weights ([layer][tap][cin][cout]) and
 * 34 FP32 head values ([2][16] weights, then 2 biases); the file format is the
 * 8-byte tag "CGCSCHD1" followed by both arrays. */
int cgc_scheduler_load(const uint16_t* conv_bf16, const float* head);
int cgc_scheduler_load_file(const char* path);
/* The CNN of the loaded weights on stacks of D^3 tile grids (device arrays:
 * feat grids*D^3*16 BF16 features, x fastest; budget and prio one byte per
 * tile; logits, may be NULL, the head's two logits per tile), with the same
 * tensor-core kernels the solve runs.  For tests and tools. */
int cgc_scheduler_infer(int32_t grids, int32_t D, const uint16_t* feat, uint8_t* budget, uint8_t* prio, float* logits,
                        void* stream);
/* Scheduling traces of the last solve run with cgc_options.trace_cycles > 0:
 * for each recorded relabel cycle c and tile t (tile order of the grid,
 * x fastest), feat[(c*T + t)*16 + k] (BF16 features), pulses[c*T + t] (pulses
 * of the tile's first visit in the cycle, 0 = not visited) and sink[c*T + t]
 * (1 if the tile delivered flow to the sink).  *cycles receives the number of
 * recorded cycles; at most max_cycles are copied (host pointers, may be NULL). */
int cgc_grid_sched_trace(cgc_grid* g, uint16_t* feat, uint8_t* pulses, uint8_t* sink, int32_t max_cycles,
                         int32_t* cycles);
/* Training kernels of the scheduler: Adam steps on device batches of feature
 * grids (grids * D^3 * 16 BF16) with device float targets per tile (prio in
 * {0,1}, budget in [0,1], mask 1 for tiles that count); count = sum of mask. */
typedef struct cgc_trainer cgc_trainer;
int cgc_trainer_create(int32_t max_grids, int32_t D, uint64_t seed, cgc_trainer** out);
int cgc_trainer_destroy(cgc_trainer* t);
int cgc_trainer_step(cgc_trainer* t, int32_t grids, const uint16_t* feat, const float* prio, const float* budget,
                     const float* mask, float count, float lr, float* loss);
int cgc_trainer_eval(cgc_trainer* t, int32_t grids, const uint16_t* feat, const float* prio, const float* budget,
                     const float* mask, float count, float* loss, float* accuracy);
int cgc_trainer_weights(cgc_trainer* t, uint16_t* conv_bf16, float* head);
int cgc_batch_trace(cgc_batch* b, int64_t* out, int32_t cap, int32_t* count);

/* ---- segmentation graph from an image and markers -------------------------
 * Replaces the reference's host-side graph construction of its segmentation
 * front-end (benchmarks/graph_cut/graph_cut.cpp:33-98): on the device, from a
 * float image and a uint8 marker volume (x fastest, device pointers; markers
 * may be NULL), writes int32 capacity volumes ready for the *_device setters:
 * capS/capT = hard_tlink where the marker is 128 / 255, every voxel within 2
 * voxels of the border is forced to the source (capS = hard_tlink, capT = 0),
 * and the symmetric n-link to the +x/+y/+z neighbour (0 on the last slice) is
 * round(nlink_scale * exp(-(Ii-Ij)^2 / 2 * sigma^2)) -- the reference's
 * formula as written (graph_cut.cpp:73) -- or, with CGC_BUILD_GAUSSIAN,
 * round(nlink_scale * exp(-(Ii-Ij)^2 / (2 sigma^2))).  Asynchronous on stream. */
#define CGC_BUILD_GAUSSIAN 1
int cgc_build_segmentation_graph(int32_t X, int32_t Y, int32_t Z, const float* image, const uint8_t* markers,
                                 float sigma, int32_t nlink_scale, int32_t hard_tlink, int32_t flags,
                                 int32_t* capS, int32_t* capT, int32_t* nx, int32_t* ny, int32_t* nz, void* stream);

#ifdef __cplusplus
}
#endif
#endif /* CGC_H */
