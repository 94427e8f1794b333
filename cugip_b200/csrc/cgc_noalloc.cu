// Allocation-free solve of one small grid.
//
// Some callers may not allocate device memory: a process whose device memory
// is owned by another allocator (a framework's caching pool, or a fixed
// memory budget handed out up front) must not see a library call cudaMalloc,
// and a real-time loop cannot afford the device-wide synchronisation that
// cudaMalloc / cudaFree imply.  cgc_grid_maxflow_noalloc serves them: the
// caller passes its inputs and outputs in device memory, and all working
// state of the solve (residual planes, heights, tile tables, worklists,
// counters) lives in one file-scope __device__ array of fixed size, which
// every GPU that loads this library holds until the process exits.
//
// Limits and rules:
//   * at most CGC_NOALLOC_MAX_VOXELS voxels after padding each extent to a
//     multiple of 8 (64^3 fits exactly); larger grids are rejected with
//     CGC_ERR_ARG before anything is launched;
//   * the first call on a device sets that device up (looks up the array's
//     device address with cudaGetSymbolAddress and sizes the cooperative
//     launch); make that first call before any stream capture.  The address
//     is kept for the life of the process, so a cudaDeviceReset after the
//     first call on a device is not supported;
//   * every call blocks the calling thread: it reads the flow and the device
//     status back into host memory and waits for the stream;
//   * every call shares the one array, which keeps the previous call's
//     contents; the call clears everything that must start at zero.  Calls
//     that overlap on the GPU (from several host threads or streams) race on
//     the array and give wrong results: issue them one after another;
//   * no cudaMalloc, cudaFree or allocating library routine is called.
#include <cuda_runtime.h>

#include <cstring>
#include <mutex>
#include <string>

#include "cgc.h"
#include "cgc_internal.h"
#include "cgc_device.cuh"
#include "cgc_pool.h"

namespace cgc {
namespace {

constexpr int64_t kMaxVoxels = CGC_NOALLOC_MAX_VOXELS;
constexpr int64_t kMaxTiles = kMaxVoxels / TV;
constexpr int kMaxDevices = 64;

constexpr int64_t al256(int64_t b) { return (b + 255) & ~(int64_t)255; }

// byte offsets of the pieces of the scratch array
constexpr int64_t kOffE = 0;
constexpr int64_t kOffH = kOffE + al256(kMaxVoxels * 4);
constexpr int64_t kOffRT = kOffH + al256(kMaxVoxels * 4);
constexpr int64_t kOffR = kOffRT + al256(kMaxVoxels * 4);
constexpr int64_t kOffRmask = kOffR + al256(6 * kMaxVoxels * 4);
constexpr int64_t kOffReach = kOffRmask + al256(kMaxVoxels);
constexpr int64_t kOffNbr = kOffReach + al256(kMaxVoxels);
constexpr int64_t kOffTinst = kOffNbr + al256(6 * kMaxTiles * 4);
constexpr int64_t kOffTpar = kOffTinst + al256(kMaxTiles * 4);
constexpr int64_t kOffAct = kOffTpar + al256(kMaxTiles);
constexpr int64_t kOffTflag = kOffAct + al256(kMaxTiles);
constexpr int64_t kOffStampB = kOffTflag + al256(kMaxTiles * 2);
constexpr int64_t kOffStampS = kOffStampB + al256(kMaxTiles * 4);
constexpr int64_t kOffStampI = kOffStampS + al256(kMaxTiles * 4);
constexpr int64_t kOffLists = kOffStampI + al256(kMaxTiles * 4);
constexpr int64_t kOffCnt = kOffLists + al256(7 * kMaxTiles * 4);
constexpr int64_t kOffFlow = kOffCnt + al256(C_NCOUNTERS * 4);
constexpr int64_t kOffGeo = kOffFlow + al256(8);
constexpr int64_t kOffStats = kOffGeo + al256(sizeof(InstGeo));
constexpr int64_t kOffErr = kOffStats + al256(S_NSTATS * 8);
constexpr int64_t kOffBar = kOffErr + al256(4);
constexpr int64_t kScratchBytes = kOffBar + al256(8);

}  // namespace

// The working state of cgc_grid_maxflow_noalloc (about 9.6 MB).  Host code
// must not pass this name to a kernel: on the host it is only a stand-in
// symbol, and its device address comes from cudaGetSymbolAddress.
static __device__ __align__(256) unsigned char g_noalloc_scratch[kScratchBytes];

namespace {

struct DeviceSetup {
  bool ready = false;
  unsigned char* scratch = nullptr;  // device address of g_noalloc_scratch
  int coop_blocks = 0;
};
std::mutex g_setup_mutex;
DeviceSetup g_setup[kMaxDevices];

// Once per device, with that device current.
int setup_device(int dev, DeviceSetup** out) {
  if (dev < 0 || dev >= kMaxDevices) return fail(CGC_ERR_ARG, "cgc_grid_maxflow_noalloc: device index out of range");
  std::lock_guard<std::mutex> lock(g_setup_mutex);
  DeviceSetup& s = g_setup[dev];
  if (!s.ready) {
    void* ptr = nullptr;
    cudaError_t e = cudaGetSymbolAddress(&ptr, g_noalloc_scratch);
    if (e != cudaSuccess)
      return fail(CGC_ERR_CUDA, std::string("cudaGetSymbolAddress(g_noalloc_scratch): ") + cudaGetErrorString(e));
    int occ = 0, sms = 0;
    e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, k_solve, 512, 0);
    if (e == cudaSuccess) e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    if (e != cudaSuccess) return fail(CGC_ERR_CUDA, std::string("noalloc set-up: ") + cudaGetErrorString(e));
    s.scratch = static_cast<unsigned char*>(ptr);
    s.coop_blocks = (occ > 0 ? occ : 1) * sms;
    s.ready = true;
  }
  *out = &s;
  return CGC_OK;
}

// Tile tables of a single instance, built on the device.
__global__ void k_noalloc_tables(DevPool P, InstGeo G) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t == 0) *const_cast<InstGeo*>(P.geo) = G;
  if (t >= P.T) return;
  const int tx = t % G.TX, ty = (t / G.TX) % G.TY, tz = t / (G.TX * G.TY);
  int32_t* nbr = const_cast<int32_t*>(P.nbr);
  nbr[PX * P.T + t] = tx + 1 < G.TX ? t + 1 : -1;
  nbr[MX * P.T + t] = tx > 0 ? t - 1 : -1;
  nbr[PY * P.T + t] = ty + 1 < G.TY ? t + G.TX : -1;
  nbr[MY * P.T + t] = ty > 0 ? t - G.TX : -1;
  nbr[PZ * P.T + t] = tz + 1 < G.TZ ? t + G.TX * G.TY : -1;
  nbr[MZ * P.T + t] = tz > 0 ? t - G.TX * G.TY : -1;
  const_cast<int32_t*>(P.tinst)[t] = 0;
  const_cast<uint8_t*>(P.tpar)[t] = (uint8_t)((tx + ty + tz) & 1);
}

}  // namespace
}  // namespace cgc

#define NA_CUDA(call)                                                                       \
  do {                                                                                      \
    cudaError_t e_ = (call);                                                                \
    if (e_ != cudaSuccess) return ::cgc::fail(CGC_ERR_CUDA, std::string(#call) + ": " + cudaGetErrorString(e_)); \
  } while (0)

extern "C" int cgc_grid_maxflow_noalloc(int32_t X, int32_t Y, int32_t Z, const int32_t* capS, const int32_t* capT,
                                        const int32_t* const fwd[3], const int32_t* const bwd[3],
                                        const cgc_options* opts, void* stream, int64_t* flow,
                                        uint8_t* source_side, uint8_t* sink_side) {
  using namespace cgc;
  if (X <= 0 || Y <= 0 || Z <= 0 || !capS || !capT || !flow)
    return fail(CGC_ERR_ARG, "cgc_grid_maxflow_noalloc: bad arguments");
  const int64_t TX = (X + 7) / 8, TY = (Y + 7) / 8, TZ = (Z + 7) / 8;
  const int64_t T = TX * TY * TZ;
  if (T * TV > kMaxVoxels)
    return fail(CGC_ERR_ARG, "cgc_grid_maxflow_noalloc: grid needs " + std::to_string(T * TV) +
                                 " padded voxels; the static scratch holds at most " + std::to_string(kMaxVoxels) +
                                 " (extents rounded up to multiples of 8)");
  int dev = 0;
  NA_CUDA(cudaGetDevice(&dev));
  DeviceSetup* su = nullptr;
  int rc = setup_device(dev, &su);
  if (rc) return rc;
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  unsigned char* base = su->scratch;

  DevPool P{};
  P.T = (int32_t)T; P.ninst = 1; P.Np = T * TV;
  P.e = (int32_t*)(base + kOffE); P.h = (int32_t*)(base + kOffH); P.rT = (int32_t*)(base + kOffRT);
  P.r = (int32_t*)(base + kOffR);  // planes are kMaxVoxels apart below
  P.rmask = base + kOffRmask; P.reach = base + kOffReach;
  P.nbr = (const int32_t*)(base + kOffNbr); P.tinst = (const int32_t*)(base + kOffTinst);
  P.tpar = base + kOffTpar; P.act = base + kOffAct; P.tflag = (uint16_t*)(base + kOffTflag);
  P.stamp_bfs = (uint32_t*)(base + kOffStampB); P.stamp_sw = (uint32_t*)(base + kOffStampS);
  P.stamp_inc = (uint32_t*)(base + kOffStampI);
  P.lists = (int32_t*)(base + kOffLists); P.cnt = (int32_t*)(base + kOffCnt);
  P.flow = (unsigned long long*)(base + kOffFlow); P.geo = (const InstGeo*)(base + kOffGeo);
  P.stats = (unsigned long long*)(base + kOffStats); P.err = (int32_t*)(base + kOffErr);
  P.bar = (uint32_t*)(base + kOffBar);
  // the residual planes are addressed as r + d*Np: use the actual Np (the
  // 6 planes of this grid fit in the 6*kMaxVoxels bytes reserved for them)

  InstGeo G{};
  G.X = X; G.Y = Y; G.Z = Z;
  G.TX = (int32_t)TX; G.TY = (int32_t)TY; G.TZ = (int32_t)TZ;
  G.tile_base = 0;
  G.hdead = (int32_t)((int64_t)X * Y * Z + 1);  // distances to the sink are at most X*Y*Z

  // everything that must start at zero: counters, flow, statistics, error
  // word, barrier, queue stamps
  NA_CUDA(cudaMemsetAsync(base + kOffCnt, 0, kOffBar + 8 - kOffCnt, st));
  NA_CUDA(cudaMemsetAsync(base + kOffStampB, 0, kOffLists - kOffStampB, st));
  k_noalloc_tables<<<(unsigned)((T + 255) / 256), 256, 0, st>>>(P, G);
  NA_CUDA(cudaGetLastError());
  k_put_tlinks<<<(unsigned)T, 512, 0, st>>>(P, 0, capS, capT);
  NA_CUDA(cudaGetLastError());
  for (int a = 0; a < 3; ++a) {
    k_put_nlinks<<<(unsigned)T, 512, 0, st>>>(P, 0, a, fwd ? fwd[a] : nullptr, bwd ? bwd[a] : nullptr);
    NA_CUDA(cudaGetLastError());
  }
  k_prepare<<<(unsigned)T, 512, 0, st>>>(P);
  NA_CUDA(cudaGetLastError());

  cgc_options o = resolve_options(opts);
  o.learned = 0;  // the learned scheduler and its traces need allocated buffers
  o.trace_cycles = 0;
  o.exclusive = 0;  // the scratch holds one half of stamps
  const SolveParams prm = solve_params(o);
  void* args[] = {(void*)&P, (void*)&prm};
  // a preparation error (overflowing capacities) makes every CTA leave at its
  // first barrier
  NA_CUDA(cudaLaunchCooperativeKernel((const void*)k_solve, dim3(su->coop_blocks), dim3(512), args, 0, st));
  if (source_side) {
    k_segments<<<(unsigned)((G.hdead + 254) / 256 < 65535 ? (G.hdead + 254) / 256 : 65535), 256, 0, st>>>(
        P, 0, CGC_SEG_SOURCE_MIN, source_side, 1, 0);
    NA_CUDA(cudaGetLastError());
  }
  if (sink_side) {
    k_segments<<<(unsigned)((G.hdead + 254) / 256 < 65535 ? (G.hdead + 254) / 256 : 65535), 256, 0, st>>>(
        P, 0, CGC_SEG_SINK_REACH, sink_side, 1, 0);
    NA_CUDA(cudaGetLastError());
  }
  struct { unsigned long long flow; int32_t err; } res;
  NA_CUDA(cudaMemcpyAsync(&res.flow, base + kOffFlow, 8, cudaMemcpyDeviceToHost, st));
  NA_CUDA(cudaMemcpyAsync(&res.err, base + kOffErr, 4, cudaMemcpyDeviceToHost, st));
  NA_CUDA(cudaStreamSynchronize(st));
  if (res.err) {
    const char* what = res.err == CGC_ERR_OVERFLOW ? "capacities may overflow int32 excess/residuals"
                     : res.err == CGC_ERR_ARG ? "negative capacity"
                     : res.err == CGC_ERR_TIMEOUT ? "a device-side wait timed out"
                     : res.err == CGC_ERR_NOT_CONVERGED ? "max_sweeps reached before convergence"
                     : "device error";
    return fail(res.err, std::string("cgc_grid_maxflow_noalloc: ") + what);
  }
  *flow = (int64_t)res.flow;
  return ok();
}
