// Device-resident batch path: many grid instances whose capacities already
// sit in device memory are uploaded, solved and written back by a fixed
// sequence of 4 kernels and 6 memory operations with no host synchronisation
// -- one pointer-table upload kernel for all instances, the preflow kernel,
// one persistent cooperative solve, one pointer-table output kernel -- which
// is captured once into a CUDA graph and replayed per batch.
//
// The reference solves one graph per Graph object with a host round trip per
// BFS level and per push level (detail/graph_cut_relabeling.hpp:962-984,
// detail/graph_cut_push.hpp:395-459); it has no batch path.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstring>
#include <string>

#include "cgc.h"
#include "cgc_kernels.cuh"
#include "cgc_pool.h"

namespace cgc {

// Upload of every instance from its bound device inputs (8 pointers per
// instance: capS, capT, fwd x/y/z, bwd x/y/z; a null n-link pointer is zero),
// fused with the preflow initialisation (put_tile4, cgc_kernels.cuh).
__global__ void __launch_bounds__(128) k_put_all(DevPool P, const int32_t* const* __restrict__ in) {
  put_tile4(P, blockIdx.x, in + 8 * P.tinst[blockIdx.x]);
}

// Both cut sets of every instance into its bound device outputs (1/0 bytes),
// in linear voxel order: grid row blockIdx.y takes instances blockIdx.y,
// blockIdx.y + gridDim.y, ... (one each unless there are more than 65535),
// and its CTAs stride over an instance four voxels per thread
// (seg_gather4 / seg_store4).
__global__ void __launch_bounds__(256) k_seg_all(DevPool P, uint8_t* const* __restrict__ out) {
  for (int inst = blockIdx.y; inst < P.ninst; inst += gridDim.y) {
    const InstGeo G = P.geo[inst];
    uint8_t* src = out[2 * inst];
    uint8_t* snk = out[2 * inst + 1];
    if (!src && !snk) continue;
    const int64_t N = (int64_t)G.X * G.Y * G.Z;
    for (int64_t v0 = 4 * ((int64_t)blockIdx.x * blockDim.x + threadIdx.x); v0 < N;
         v0 += 4 * (int64_t)gridDim.x * blockDim.x) {
      unsigned a = 0, b = 0;
      seg_gather4(P, G, v0, N, snk ? &a : nullptr, src ? &b : nullptr);
      if (src) seg_store4(src, v0, N, b, 1, 0);
      if (snk) seg_store4(snk, v0, N, a, 1, 0);
    }
  }
}

static int ensure_tables(Pool& p) {
  if (!p.d_in) {
    CGC_CUDA(cudaMalloc(&p.d_in, sizeof(int32_t*) * 8 * p.ninst));
    CGC_CUDA(cudaMalloc(&p.d_out, sizeof(uint8_t*) * 2 * p.ninst));
    p.in_ptrs.assign(8 * (size_t)p.ninst, nullptr);
    p.out_ptrs.assign(2 * (size_t)p.ninst, nullptr);
  }
  return CGC_OK;
}

int pool_bind_inputs(Pool& p, int inst, const int32_t* capS, const int32_t* capT, const int32_t* const fwd[3],
                     const int32_t* const bwd[3]) {
  if (inst < 0 || inst >= p.ninst || !capS || !capT) return fail(CGC_ERR_ARG, "bind_inputs: bad arguments");
  int rc = ensure_tables(p);
  if (rc) return rc;
  const int32_t** ip = p.in_ptrs.data() + 8 * (size_t)inst;
  ip[0] = capS;
  ip[1] = capT;
  for (int a = 0; a < 3; ++a) {
    ip[2 + a] = fwd ? fwd[a] : nullptr;
    ip[5 + a] = bwd ? bwd[a] : (fwd ? fwd[a] : nullptr);
  }
  CGC_CUDA(cudaMemcpy(p.d_in + 8 * (size_t)inst, ip, 8 * sizeof(int32_t*), cudaMemcpyHostToDevice));
  return ok();
}

int pool_bind_outputs(Pool& p, int inst, uint8_t* source_side, uint8_t* sink_side) {
  if (inst < 0 || inst >= p.ninst) return fail(CGC_ERR_ARG, "bind_outputs: bad instance");
  int rc = ensure_tables(p);
  if (rc) return rc;
  p.out_ptrs[2 * (size_t)inst] = source_side;
  p.out_ptrs[2 * (size_t)inst + 1] = sink_side;
  CGC_CUDA(cudaMemcpy(p.d_out + 2 * (size_t)inst, p.out_ptrs.data() + 2 * (size_t)inst, 2 * sizeof(uint8_t*),
                      cudaMemcpyHostToDevice));
  return ok();
}

// Enqueues one batched solve on `stream` without synchronising the host.
int pool_enqueue(Pool& p, const cgc_options* opts, int64_t* flows_dev, cudaStream_t stream) {
  if (!p.d_in) return fail(CGC_ERR_STATE, "enqueue: no device inputs bound");
  if (p.pending) return fail(CGC_ERR_STATE, "enqueue: a host-path solve of this handle was not waited for");
  for (int i = 0; i < p.ninst; ++i)
    if (!p.in_ptrs[8 * (size_t)i]) return fail(CGC_ERR_STATE, "enqueue: instance without bound inputs");
  const cgc_options o = resolve_options(opts);
  if (o.learned > 0 || o.trace_cycles > 0) {  // buffers and weights before anything is queued
    int rc = ensure_sched(p, o.learned > 0, o.trace_cycles);
    if (rc) return rc;
  }
  DevPool& d = p.dp;
  CGC_CUDA(cudaMemsetAsync(d.flow, 0, (size_t)p.ninst * 8, stream));
  CGC_CUDA(cudaMemsetAsync(d.stats, 0, S_NSTATS * 8, stream));
  CGC_CUDA(cudaMemsetAsync(d.err, 0, 4, stream));
  CGC_CUDA(cudaMemsetAsync(d.bar, 0, 8, stream));
  CGC_CUDA(cudaMemsetAsync(d.stamp_bfs, 0, (size_t)d.T * 4, stream));
  CGC_CUDA(cudaMemsetAsync(d.stamp_sw, 0, 2 * (size_t)d.T * 4, stream));
  CGC_CUDA(cudaMemsetAsync(d.stamp_inc, 0, (size_t)d.T * 4, stream));
  k_put_all<<<d.T, 128, 0, stream>>>(d, p.d_in);
  note_launch();
  const SolveParams prm = solve_params(o);
  if (int rc = launch_solve(p, o, d, prm, stream)) return rc;
  bool any_out = false;
  for (uint8_t* q : p.out_ptrs) any_out = any_out || q;
  if (any_out) {
    const unsigned gx = (unsigned)std::min<int64_t>(std::max<int64_t>((p.maxN + 32767) / 32768, 1), 4096);
    k_seg_all<<<dim3(gx, (unsigned)std::min(p.ninst, 65535)), 256, 0, stream>>>(d, p.d_out);
    note_launch();
  }
  if (flows_dev) CGC_CUDA(cudaMemcpyAsync(flows_dev, d.flow, (size_t)p.ninst * 8, cudaMemcpyDeviceToDevice, stream));
  CGC_CUDA(cudaGetLastError());
  for (auto& u : p.uploaded) u = 0;
  p.solved = true;
  p.seg_valid = false;
  return ok();
}

// Waits for the last enqueued or replayed batch; reports device errors and
// refreshes flows and statistics.
int pool_wait(Pool& p, cudaStream_t stream) {
  CGC_CUDA(cudaStreamSynchronize(stream));
  int rc = check_device_error(p, "batch");
  if (rc) return rc;
  unsigned long long stats[S_NSTATS];
  CGC_CUDA(cudaMemcpyAsync(stats, p.dp.stats, sizeof(stats), cudaMemcpyDeviceToHost, stream));
  CGC_CUDA(cudaMemcpyAsync(p.flows.data(), p.dp.flow, (size_t)p.ninst * 8, cudaMemcpyDeviceToHost, stream));
  CGC_CUDA(cudaStreamSynchronize(stream));
  std::memset(&p.st, 0, sizeof(p.st));
  for (int64_t f : p.flows) p.st.flow += f;
  p.st.sweeps = (int64_t)stats[S_SWEEPS];
  p.st.global_relabels = (int64_t)stats[S_RELABELS];
  p.st.bfs_rounds = (int64_t)stats[S_ROUNDS];
  p.st.tiles_swept = (int64_t)stats[S_TILES_SWEPT];
  p.st.tiles_relabelled = (int64_t)stats[S_TILES_BFS];
  p.st.tiles_checked = (int64_t)stats[S_TILES_CHECK];
  p.st.pulses = (int64_t)stats[S_PULSES];
  p.st.bfs_ms = 1e-6 * (double)stats[S_NS_BFS];
  p.st.sweep_ms = 1e-6 * (double)stats[S_NS_SWEEP];
  p.st.reach_ms = 1e-6 * (double)stats[S_NS_REACH];
  p.st.sched_ms = 1e-6 * (double)stats[S_NS_SCHED];
  return ok();
}

int pool_graph_create(Pool& p, const cgc_options* opts, int64_t* flows_dev) {
  if (p.graph_exec) { cudaGraphExecDestroy(p.graph_exec); p.graph_exec = nullptr; }
  if (p.graph) { cudaGraphDestroy(p.graph); p.graph = nullptr; }
  if (!p.cap_stream) CGC_CUDA(cudaStreamCreateWithFlags(&p.cap_stream, cudaStreamNonBlocking));
  {
    const cgc_options o = resolve_options(opts);
    if (o.learned > 0 || o.trace_cycles > 0) {  // allocations and weight uploads stay outside the capture
      int rc = ensure_sched(p, o.learned > 0, o.trace_cycles);
      if (rc) return rc;
    }
  }
  CGC_CUDA(cudaStreamBeginCapture(p.cap_stream, cudaStreamCaptureModeThreadLocal));
  const long long before = g_launches.load();
  int rc = pool_enqueue(p, opts, flows_dev, p.cap_stream);
  cudaGraph_t g = nullptr;
  cudaError_t e = cudaStreamEndCapture(p.cap_stream, &g);
  g_launches.store(before);  // capture does not launch anything
  if (rc) { if (g) cudaGraphDestroy(g); return rc; }
  if (e != cudaSuccess) return fail(CGC_ERR_CUDA, std::string("cudaStreamEndCapture: ") + cudaGetErrorString(e));
  p.graph = g;
  CGC_CUDA(cudaGraphInstantiate(&p.graph_exec, p.graph, 0));
  size_t nodes = 0;
  CGC_CUDA(cudaGraphGetNodes(p.graph, nullptr, &nodes));
  p.graph_kernels = 0;
  std::vector<cudaGraphNode_t> all(nodes);
  CGC_CUDA(cudaGraphGetNodes(p.graph, all.data(), &nodes));
  for (auto nd : all) {
    cudaGraphNodeType ty;
    CGC_CUDA(cudaGraphNodeGetType(nd, &ty));
    if (ty == cudaGraphNodeTypeKernel) ++p.graph_kernels;
  }
  return ok();
}

int pool_graph_launch(Pool& p) {
  if (!p.graph_exec) return fail(CGC_ERR_STATE, "graph_launch: no graph (call cgc_batch_graph_create)");
  if (p.pending) return fail(CGC_ERR_STATE, "graph_launch: a host-path solve of this handle was not waited for");
  CGC_CUDA(cudaGraphLaunch(p.graph_exec, p.stream));
  for (int i = 0; i < p.graph_kernels; ++i) note_launch();
  for (auto& u : p.uploaded) u = 0;
  p.solved = true;
  p.seg_valid = false;
  return ok();
}

}  // namespace cgc

struct cgc_batch { cgc::Pool* p; };

extern "C" {

int cgc_batch_bind_inputs(cgc_batch* b, int32_t i, const int32_t* capS, const int32_t* capT,
                          const int32_t* const fwd[3], const int32_t* const bwd[3]) {
  if (!b) return cgc::fail(CGC_ERR_ARG, "null batch");
  return cgc::pool_bind_inputs(*b->p, i, capS, capT, fwd, bwd);
}
int cgc_batch_bind_outputs(cgc_batch* b, int32_t i, uint8_t* source_side, uint8_t* sink_side) {
  if (!b) return cgc::fail(CGC_ERR_ARG, "null batch");
  return cgc::pool_bind_outputs(*b->p, i, source_side, sink_side);
}
int cgc_batch_enqueue(cgc_batch* b, const cgc_options* opts, int64_t* flows_dev) {
  if (!b) return cgc::fail(CGC_ERR_ARG, "null batch");
  return cgc::pool_enqueue(*b->p, opts, flows_dev, b->p->stream);
}
int cgc_batch_graph_create(cgc_batch* b, const cgc_options* opts, int64_t* flows_dev) {
  if (!b) return cgc::fail(CGC_ERR_ARG, "null batch");
  return cgc::pool_graph_create(*b->p, opts, flows_dev);
}
int cgc_batch_graph_launch(cgc_batch* b) {
  if (!b) return cgc::fail(CGC_ERR_ARG, "null batch");
  return cgc::pool_graph_launch(*b->p);
}
int cgc_batch_wait(cgc_batch* b, int64_t* flows) {
  if (!b) return cgc::fail(CGC_ERR_ARG, "null batch");
  int rc = cgc::pool_wait(*b->p, b->p->stream);
  if (rc) return rc;
  if (flows) std::memcpy(flows, b->p->flows.data(), b->p->flows.size() * 8);
  return cgc::ok();
}

}  // extern "C"
