// Host-side pool of grid instances shared by the translation units of libcgc.
#pragma once
#include <cuda_runtime.h>

#include <atomic>
#include <cstdint>
#include <functional>
#include <string>
#include <vector>

#include "cgc.h"
#include "cgc_device.cuh"
#include "cgc_internal.h"

namespace cgc {

#define CGC_CUDA(call)                                                                      \
  do {                                                                                      \
    cudaError_t e_ = (call);                                                                \
    if (e_ != cudaSuccess)                                                                  \
      return ::cgc::fail(e_ == cudaErrorMemoryAllocation ? CGC_ERR_OOM : CGC_ERR_CUDA,      \
                  std::string(#call) + ": " + cudaGetErrorString(e_));                      \
  } while (0)

extern std::atomic<long long> g_launches;
void note_launch();

struct Pool {
  int device = 0;
  cudaStream_t stream = nullptr;
  int ninst = 0;
  std::vector<InstGeo> geo;
  std::vector<uint32_t> uploaded;  // bit 0 tlinks, bits 1..3 axes
  int64_t maxN = 0;
  int32_t T = 0;
  int64_t Np = 0;
  DevPool dp{};
  void* dbuf = nullptr;          // all device state
  // Inputs of the set_* calls: linear (x-fastest) planes, the instances back
  // to back at voff[i]; read by the fused upload kernel of the next solve.
  int64_t sumN = 0;
  std::vector<int64_t> voff;
  int32_t* lin = nullptr;        // 5 planes of sumN: capS, capT, fwd x/y/z (first set_* call)
  int32_t* lin_bwd = nullptr;    // 3 planes of sumN: bwd x/y/z (first asymmetric n-link upload)
  std::vector<const int32_t*> host_in;  // 8 per instance: planes the next solve reads (null = zero)
  const int32_t** d_host_in = nullptr;  // device copy of host_in (batches of more than one instance)
  cudaStream_t copy_stream = nullptr;   // host -> device copies of the setters
  cudaEvent_t inputs_read = nullptr;    // recorded after the upload kernel of the last solve
  // cut sets of the last host-path solve (1/0 bytes, linear order): source
  // side at [0, sumN), sink side at [sumN, 2 sumN)
  uint8_t* segbuf = nullptr;
  uint8_t** d_segtab = nullptr;  // 2 per instance: pointers into segbuf
  bool seg_valid = false;        // segbuf holds the last solve's cut sets
  uint8_t* segtmp = nullptr;     // maxN bytes for remapped masks (mask / background values)
  int32_t* resid = nullptr;      // maxN int32 for cgc_grid_get_residuals
  cudaEvent_t ev[4] = {nullptr, nullptr, nullptr, nullptr};  // solve and kernel timing
  bool pending = false;          // a host-path solve was enqueued and not yet waited for
  int pending_persistent = 1;    // its options' persistent field
  long long launches0 = 0;       // launch counter when it was enqueued
  int64_t host_counts[3] = {0, 0, 0};  // host-driven schedule: sweeps, relabels, BFS rounds
  int32_t* pinned_cnt = nullptr; // host-pinned counters
  bool solved = false;
  int sms = 148;
  int coop_blocks = 0;           // co-resident CTAs of k_solve
  int coop_blocks3 = 0;          // co-resident CTAs of k_solve3
  int coop_blocks4 = 0;          // co-resident CTAs of k_solve4
  int sweep_blocks = 0;
  cgc_stats st{};
  std::vector<int64_t> flows;
  // device-resident batch path (cgc_batch_bind_* / cgc_batch_enqueue)
  std::vector<const int32_t*> in_ptrs;   // 8 per instance: capS, capT, fwd[3], bwd[3]
  std::vector<uint8_t*> out_ptrs;        // 2 per instance: source side, sink side
  const int32_t** d_in = nullptr;        // device copy of in_ptrs
  uint8_t** d_out = nullptr;             // device copy of out_ptrs
  bool tables_dirty = true;
  cudaStream_t cap_stream = nullptr;     // capture stream (the legacy stream cannot be captured)
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t graph_exec = nullptr;
  int graph_kernels = 0;                 // kernel nodes in the captured graph
  // learned scheduler buffers (cgc_sched_train.cu)
  void* sbuf = nullptr;
  void* tbuf = nullptr;
  int trace_cap = 0;
  uint64_t sched_wver = 0;
  ~Pool() {
    if (sbuf) cudaFree(sbuf);
    if (tbuf) cudaFree(tbuf);
    if (graph_exec) cudaGraphExecDestroy(graph_exec);
    if (graph) cudaGraphDestroy(graph);
    if (cap_stream) cudaStreamDestroy(cap_stream);
    if (d_in) cudaFree(d_in);
    if (d_out) cudaFree(d_out);
    if (dbuf) cudaFree(dbuf);
    if (lin) cudaFree(lin);
    if (lin_bwd) cudaFree(lin_bwd);
    if (d_host_in) cudaFree(d_host_in);
    if (segbuf) cudaFree(segbuf);
    if (d_segtab) cudaFree(d_segtab);
    if (segtmp) cudaFree(segtmp);
    if (resid) cudaFree(resid);
    if (inputs_read) cudaEventDestroy(inputs_read);
    for (auto e : ev)
      if (e) cudaEventDestroy(e);
    if (copy_stream) cudaStreamDestroy(copy_stream);
    if (pinned_cnt) cudaFreeHost(pinned_cnt);
  }
};


int check_device_error(Pool& p, const char* where);
int pool_create(int32_t count, const int32_t* ext, void* stream, Pool** out);
int pool_put_tlinks(Pool& p, int inst, const int32_t* capS, const int32_t* capT, bool host);
int pool_put_nlinks(Pool& p, int inst, int axis, const int32_t* fwd, const int32_t* bwd, bool host);
cgc_options resolve_options(const cgc_options* o);
uint64_t wait_limit_ns(const cgc_options& o);
SolveParams solve_params(const cgc_options& o);
int pool_solve(Pool& p, const cgc_options* opts);
// host path in two halves: enqueue a solve of the set_* inputs on p.stream
// (no host synchronisation), then wait for it and read flows and statistics
int pool_solve_async(Pool& p, const cgc_options* opts);
int pool_solve_wait(Pool& p);
// runs `launch` (a cooperative launch into `stream`) after every earlier
// cooperative launch of this library on the device has ended
int coop_launch_ordered(int device, cudaStream_t stream, const std::function<int()>& launch);
// cooperative launch of the persistent solve kernel selected by the options
int launch_solve(Pool& p, const cgc_options& o, const DevPool& d, const SolveParams& prm, cudaStream_t stream);
int pool_segments(Pool& p, int inst, int which, uint8_t* out, uint8_t mask, uint8_t bg, bool host);
int pool_residuals(Pool& p, int inst, int32_t* const res[6], int32_t* resT, int32_t* excess);
int pool_trace(Pool& p, int64_t* out, int32_t cap, int32_t* count);
int pool_labels(Pool& p, int inst, int32_t* labels);
// device-resident batch path (cgc_batch.cu)
int pool_bind_inputs(Pool& p, int inst, const int32_t* capS, const int32_t* capT, const int32_t* const fwd[3],
                     const int32_t* const bwd[3]);
int pool_bind_outputs(Pool& p, int inst, uint8_t* source_side, uint8_t* sink_side);
int pool_enqueue(Pool& p, const cgc_options* opts, int64_t* flows_dev, cudaStream_t stream);
int pool_wait(Pool& p, cudaStream_t stream);
int pool_graph_create(Pool& p, const cgc_options* opts, int64_t* flows_dev);
int pool_graph_launch(Pool& p);
// learned scheduler (cgc_sched_train.cu)
int ensure_sched(Pool& p, bool learned, int trace_cycles);
int pool_sched_trace(Pool& p, uint16_t* feat, uint8_t* pulses, uint8_t* sink, int32_t max_cycles, int32_t* cycles);

}  // namespace cgc
