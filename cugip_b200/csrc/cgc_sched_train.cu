// Learned scheduler: weights, trace buffers and hand-written training kernels.
//
// The network (see cgc_sched.cuh): features[16] -> conv3x3x3(16) -> ReLU ->
// conv3x3x3(16) -> ReLU -> conv3x3x3(16) -> ReLU -> linear head(2): a priority
// logit (trained with binary cross-entropy against "the tile delivered flow
// to the sink during the relabel cycle") and a budget logit (sigmoid trained
// with squared error against the last productive pulse of the tile's first
// visit -- the last pulse that moved flow out of the tile or into the sink).
// The forward pass runs on the tensor cores with the routine of the solve's
// scheduler stage (BF16 weights and activations, FP32 accumulation), so the
// network is trained on exactly the numbers inference computes; the backward
// passes run in FP32 on the CUDA cores (the gradients are not BF16 values),
// and Adam updates FP32 master weights.
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <mutex>
#include <random>
#include <string>
#include <vector>

#include "cgc.h"
#include "cgc_pool.h"
#include "cgc_sched.cuh"

namespace cgc {
namespace {

std::mutex g_wmu;
std::vector<uint16_t> g_wconv;  // 3 * SCHED_WCONV bf16 bits
std::vector<float> g_whead;     // SCHED_NHEAD
uint64_t g_wver = 0;            // 0: nothing loaded

}  // namespace

// The convolution weights ([layer][tap][cin][cout] BF16 bits) as the B
// fragments of mma.sync.m16n8k16 ([layer][tap][half][lane] -> 2 registers):
// register 0 holds cin 2q, 2q+1 and register 1 cin 2q+8, 2q+9 of output
// channel 8*half + g (g = lane / 4, q = lane % 4), lower cin in the low half.
std::vector<uint32_t> fragment_order(const std::vector<uint16_t>& w) {
  std::vector<uint32_t> f((size_t)3 * SCHED_FRAG * 2);
  for (int l = 0; l < 3; ++l)
    for (int k = 0; k < SCHED_TAPS; ++k)
      for (int h = 0; h < 2; ++h)
        for (int lane = 0; lane < 32; ++lane) {
          const int g = lane >> 2, q = lane & 3, co = 8 * h + g;
          auto wv = [&](int ci) -> uint32_t { return w[(size_t)l * SCHED_WCONV + (k * SCHED_C + ci) * SCHED_C + co]; };
          const size_t at = (((size_t)l * SCHED_TAPS + k) * 2 + h) * 32 + lane;
          f[2 * at] = wv(2 * q) | (wv(2 * q + 1) << 16);
          f[2 * at + 1] = wv(2 * q + 8) | (wv(2 * q + 9) << 16);
        }
  return f;
}

// Device buffers of the scheduler for one pool (allocated on first use).
int ensure_sched(Pool& p, bool learned, int trace_cycles) {
  DevPool& d = p.dp;
  const int64_t T = d.T;
  if (!p.sbuf) {
    const size_t bytes = (size_t)3 * T * SCHED_C * 2 + (size_t)3 * SCHED_FRAG * 8 + SCHED_NHEAD * 4 + 2 * (size_t)T;
    CGC_CUDA(cudaMalloc(&p.sbuf, bytes));
    CGC_CUDA(cudaMemset(p.sbuf, 0, bytes));
    char* q = (char*)p.sbuf;
    d.sfeat = (__nv_bfloat16*)q; q += (size_t)T * SCHED_C * 2;
    d.sact0 = (__nv_bfloat16*)q; q += (size_t)T * SCHED_C * 2;
    d.sact1 = (__nv_bfloat16*)q; q += (size_t)T * SCHED_C * 2;
    d.swfrag = (const uint2*)q; q += (size_t)3 * SCHED_FRAG * 8;
    d.swhead = (const float*)q; q += SCHED_NHEAD * 4;
    d.sbudget = (uint8_t*)q; q += T;
    d.sprio = (uint8_t*)q;
  }
  if (learned) {
    std::lock_guard<std::mutex> lock(g_wmu);
    if (!g_wver) return fail(CGC_ERR_STATE, "learned scheduler requested but no weights are loaded (cgc_scheduler_load)");
    if (p.sched_wver != g_wver) {
      const std::vector<uint32_t> frag = fragment_order(g_wconv);
      CGC_CUDA(cudaMemcpy((void*)d.swfrag, frag.data(), frag.size() * 4, cudaMemcpyHostToDevice));
      CGC_CUDA(cudaMemcpy((void*)d.swhead, g_whead.data(), g_whead.size() * 4, cudaMemcpyHostToDevice));
      p.sched_wver = g_wver;
    }
  }
  if (trace_cycles > p.trace_cap) {
    if (p.tbuf) { cudaFree(p.tbuf); p.tbuf = nullptr; }
    const size_t bytes = (size_t)trace_cycles * T * (SCHED_C * 2 + 2);
    CGC_CUDA(cudaMalloc(&p.tbuf, bytes));
    char* q = (char*)p.tbuf;
    d.tfeat = (__nv_bfloat16*)q; q += (size_t)trace_cycles * T * SCHED_C * 2;
    d.tpulses = (uint8_t*)q; q += (size_t)trace_cycles * T;
    d.tsink = (uint8_t*)q;
    p.trace_cap = trace_cycles;
  }
  return CGC_OK;
}

int pool_sched_trace(Pool& p, uint16_t* feat, uint8_t* pulses, uint8_t* sink, int32_t max_cycles, int32_t* cycles) {
  if (!p.solved) return fail(CGC_ERR_STATE, "sched_trace: call maxflow first");
  unsigned long long n = 0;
  CGC_CUDA(cudaMemcpy(&n, p.dp.stats + S_TRACE_CYC, 8, cudaMemcpyDeviceToHost));
  *cycles = (int32_t)n;
  const int64_t m = std::min<int64_t>((int64_t)n, max_cycles);
  const int64_t T = p.dp.T;
  if (m > 0) {
    if (feat) CGC_CUDA(cudaMemcpy(feat, p.dp.tfeat, (size_t)m * T * SCHED_C * 2, cudaMemcpyDeviceToHost));
    if (pulses) CGC_CUDA(cudaMemcpy(pulses, p.dp.tpulses, (size_t)m * T, cudaMemcpyDeviceToHost));
    if (sink) CGC_CUDA(cudaMemcpy(sink, p.dp.tsink, (size_t)m * T, cudaMemcpyDeviceToHost));
  }
  return ok();
}

// ===========================================================================
// training kernels: positions p index (grid g, tile x, y, z) of D^3 grids,
// channels-last [p][16]
// ===========================================================================
namespace {

__device__ __forceinline__ float bf16_round(float v) { return __bfloat162float(__float2bfloat16(v)); }

__device__ __forceinline__ int nb_index(int p, int D, int k, bool neg) {
  const int D3 = D * D * D;
  const int g = p / D3, r = p % D3;
  const int x = r % D, y = (r / D) % D, z = r / (D * D);
  int dx = k % 3 - 1, dy = (k / 3) % 3 - 1, dz = k / 9 - 1;
  if (neg) { dx = -dx; dy = -dy; dz = -dz; }
  const int nx = x + dx, ny = y + dy, nz = z + dz;
  if (nx < 0 || ny < 0 || nz < 0 || nx >= D || ny >= D || nz >= D) return -1;
  return g * D3 + nx + D * (ny + D * nz);
}

// Training forward of one convolution layer on the tensor cores: conv_rows16,
// the routine of the solve's scheduler stage, on stacks of D^3 grids, so the
// trained network sees exactly the inference numerics.  Writes the ReLU'd BF16
// output (the next layer's input, may be null) and its float copy (kept for
// the backward pass).
__global__ void __launch_bounds__(256) k_train_conv_fwd(GridSpace sp, const uint32_t* __restrict__ in,
                                                        const uint2* __restrict__ wf, uint32_t* out16, float* out32) {
  const int lane = threadIdx.x & 31, g = lane >> 2, q = lane & 3;
  const int T = sp.count(), nchunks = (T + 15) >> 4;
  for (int c = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5); c < nchunks; c += gridDim.x * (blockDim.x >> 5)) {
    const int ta = (c << 4) + g, tb = ta + 8;
    const bool va = ta < T, vb = tb < T;
    const GridCoord ca = sp.coord(va ? ta : 0), cb = sp.coord(vb ? tb : 0);
    float acc[2][4];
    conv_rows16(in, wf, [&](int row, int k) {
      return row < 8 ? (va ? sp.tap(ca, k) : -1) : (vb ? sp.tap(cb, k) : -1);
    }, acc);
#pragma unroll
    for (int h = 0; h < 2; ++h) {
      float o[4];
#pragma unroll
      for (int i = 0; i < 4; ++i) o[i] = __bfloat162float(__float2bfloat16(fmaxf(acc[h][i], 0.f)));
      const int ch = 8 * h + 2 * q;
      if (va) {
        if (out16) out16[(int64_t)ta * 8 + 4 * h + q] = pack_bf16x2(o[0], o[1]);
        out32[(int64_t)ta * SCHED_C + ch] = o[0];
        out32[(int64_t)ta * SCHED_C + ch + 1] = o[1];
      }
      if (vb) {
        if (out16) out16[(int64_t)tb * 8 + 4 * h + q] = pack_bf16x2(o[2], o[3]);
        out32[(int64_t)tb * SCHED_C + ch] = o[2];
        out32[(int64_t)tb * SCHED_C + ch + 1] = o[3];
      }
    }
  }
}

// B fragments (fragment_order's layout) of the BF16-rounded master weights.
__global__ void k_frag_from_f32(const float* __restrict__ wr, uint2* __restrict__ wf) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;  // (layer, tap, half, lane)
  if (i >= 3 * SCHED_FRAG) return;
  const int lane = i & 31, h = (i >> 5) & 1, k = (i >> 6) % SCHED_TAPS, l = (i >> 6) / SCHED_TAPS;
  const int g = lane >> 2, q = lane & 3, co = 8 * h + g;
  const float* w = wr + (size_t)l * SCHED_WCONV + co;
  wf[i] = make_uint2(pack_bf16x2(w[(k * SCHED_C + 2 * q) * SCHED_C], w[(k * SCHED_C + 2 * q + 1) * SCHED_C]),
                     pack_bf16x2(w[(k * SCHED_C + 2 * q + 8) * SCHED_C], w[(k * SCHED_C + 2 * q + 9) * SCHED_C]));
}

__global__ void k_feat_to_f32(const __nv_bfloat16* in, float* out, int64_t n) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
    out[i] = __bfloat162float(in[i]);
}

// head, loss and the gradient entering the last activation
__global__ void k_head_loss(const float* A3, const float* Wh, const float* yprio, const float* ybud, const float* mask,
                            float inv_n, float* dA3, float* gWh, float* loss, float* correct, int NP) {
  const int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= NP) return;
  const float* a = A3 + (int64_t)p * SCHED_C;
  float o0 = Wh[2 * SCHED_C], o1 = Wh[2 * SCHED_C + 1];
#pragma unroll
  for (int c = 0; c < SCHED_C; ++c) { o0 = fmaf(Wh[c], a[c], o0); o1 = fmaf(Wh[SCHED_C + c], a[c], o1); }
  float g0 = 0.f, g1 = 0.f;
  if (mask[p] > 0.f) {
    const float y = yprio[p], yb = ybud[p];
    const float s0 = 1.f / (1.f + expf(-o0)), s1 = 1.f / (1.f + expf(-o1));
    const float l0 = fmaxf(o0, 0.f) - o0 * y + log1pf(expf(-fabsf(o0)));
    const float l1 = (s1 - yb) * (s1 - yb);
    atomicAdd(loss, (l0 + l1) * inv_n);
    if (correct) atomicAdd(correct, ((o0 >= 0.f) == (y > 0.5f)) ? inv_n : 0.f);
    g0 = (s0 - y) * inv_n;
    g1 = 2.f * (s1 - yb) * s1 * (1.f - s1) * inv_n;
  }
  float* d = dA3 + (int64_t)p * SCHED_C;
#pragma unroll
  for (int c = 0; c < SCHED_C; ++c) d[c] = (a[c] > 0.f) ? (g0 * Wh[c] + g1 * Wh[SCHED_C + c]) : 0.f;
  if (gWh && (g0 != 0.f || g1 != 0.f)) {
#pragma unroll
    for (int c = 0; c < SCHED_C; ++c) {
      if (a[c] != 0.f) {
        atomicAdd(gWh + c, g0 * a[c]);
        atomicAdd(gWh + SCHED_C + c, g1 * a[c]);
      }
    }
    atomicAdd(gWh + 2 * SCHED_C, g0);
    atomicAdd(gWh + 2 * SCHED_C + 1, g1);
  }
}

// dIn[q][ci] = (sum_k sum_co W[k][ci][co] * dPre[q - off_k][co]) * relu'(In[q][ci])
__global__ void k_conv_bwd_data(const float* dPre, const float* W, const float* In, float* dIn, int NP, int D) {
  const int q = blockIdx.x * 16 + (threadIdx.x >> 4), ci = threadIdx.x & 15;
  if (q >= NP) return;
  float acc = 0.f;
  for (int k = 0; k < SCHED_TAPS; ++k) {
    const int p = nb_index(q, D, k, true);
    if (p < 0) continue;
    const float* g = dPre + (int64_t)p * SCHED_C;
    const float* w = W + (k * SCHED_C + ci) * SCHED_C;
#pragma unroll
    for (int co = 0; co < SCHED_C; ++co) acc = fmaf(w[co], g[co], acc);
  }
  dIn[(int64_t)q * SCHED_C + ci] = (In[(int64_t)q * SCHED_C + ci] > 0.f) ? acc : 0.f;
}

// gW[k][ci][co] += sum_p X[nb(p,k)][ci] * dPre[p][co]; block = (tap k, chunk)
__global__ void k_conv_bwd_weight(const float* X, const float* dPre, float* gW, int NP, int D, int chunk) {
  __shared__ float xs[64][SCHED_C];
  __shared__ float gs[64][SCHED_C];
  const int k = blockIdx.y;
  const int ci = threadIdx.x >> 4, co = threadIdx.x & 15;
  const int p0 = blockIdx.x * chunk, p1 = min(NP, p0 + chunk);
  float acc = 0.f;
  for (int pb = p0; pb < p1; pb += 64) {
    for (int i = threadIdx.x; i < 64 * SCHED_C; i += blockDim.x) {
      const int pp = pb + i / SCHED_C, c = i % SCHED_C;
      float xv = 0.f, gv = 0.f;
      if (pp < p1) {
        const int q = nb_index(pp, D, k, false);
        xv = q >= 0 ? X[(int64_t)q * SCHED_C + c] : 0.f;
        gv = dPre[(int64_t)pp * SCHED_C + c];
      }
      xs[i / SCHED_C][c] = xv;
      gs[i / SCHED_C][c] = gv;
    }
    __syncthreads();
#pragma unroll 8
    for (int j = 0; j < 64; ++j) acc = fmaf(xs[j][ci], gs[j][co], acc);
    __syncthreads();
  }
  atomicAdd(gW + (k * SCHED_C + ci) * SCHED_C + co, acc);
}

__global__ void k_adam(float* w, const float* g, float* m, float* v, int n, float lr, float b1, float b2, float eps,
                       float c1, float c2) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const float gi = g[i];
  const float mi = b1 * m[i] + (1.f - b1) * gi;
  const float vi = b2 * v[i] + (1.f - b2) * gi * gi;
  m[i] = mi;
  v[i] = vi;
  w[i] -= lr * (mi / c1) / (sqrtf(vi / c2) + eps);
}

__global__ void k_round_bf16(const float* w, float* wr, int n) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) wr[i] = bf16_round(w[i]);
}

}  // namespace

// Trainer state: parameters [conv 3*SCHED_WCONV | head SCHED_NHEAD] in one
// FP32 array with Adam moments, plus activations for `max_grids` grids.
struct Trainer {
  int max_grids = 0, D = 0, NP = 0;
  int nparam = 3 * SCHED_WCONV + SCHED_NHEAD;
  int64_t steps = 0;
  float *w = nullptr, *wr = nullptr, *g = nullptr, *m = nullptr, *v = nullptr;
  float *X = nullptr, *A[3] = {nullptr, nullptr, nullptr}, *dA = nullptr, *dB = nullptr, *stat = nullptr;
  uint32_t* A16[2] = {nullptr, nullptr};  // BF16 copies of layers 0 and 1 (the tensor-core inputs)
  uint2* wf = nullptr;                    // weights in mma fragment order
  ~Trainer() {
    for (float* q : {w, wr, g, m, v, X, A[0], A[1], A[2], dA, dB, stat})
      if (q) cudaFree(q);
    for (void* q : {(void*)A16[0], (void*)A16[1], (void*)wf})
      if (q) cudaFree(q);
  }
};

static int trainer_forward_backward(Trainer& tr, int grids, const uint16_t* feat, const float* yp, const float* yb,
                                    const float* mask, float count, bool backward, float* loss, float* acc) {
  const int NP = grids * tr.D * tr.D * tr.D;
  if (grids <= 0 || grids > tr.max_grids) return fail(CGC_ERR_ARG, "trainer: bad grid count");
  const float inv_n = count > 0 ? 1.f / count : 0.f;
  CGC_CUDA(cudaMemset(tr.stat, 0, 2 * sizeof(float)));
  if (backward) CGC_CUDA(cudaMemset(tr.g, 0, tr.nparam * sizeof(float)));
  k_feat_to_f32<<<1024, 256>>>((const __nv_bfloat16*)feat, tr.X, (int64_t)NP * SCHED_C);
  const int blocks = (NP + 15) / 16;
  k_frag_from_f32<<<(3 * SCHED_FRAG + 255) / 256, 256>>>(tr.wr, tr.wf);
  const GridSpace sp{grids, tr.D};
  const unsigned cblocks = (unsigned)std::min((NP + 127) / 128, 8192);
  const uint32_t* in16 = reinterpret_cast<const uint32_t*>(feat);
  for (int l = 0; l < 3; ++l) {
    k_train_conv_fwd<<<cblocks, 256>>>(sp, in16, tr.wf + (size_t)l * SCHED_FRAG, l < 2 ? tr.A16[l] : nullptr, tr.A[l]);
    if (l < 2) in16 = tr.A16[l];
  }
  const float* wh = tr.wr + 3 * SCHED_WCONV;
  k_head_loss<<<(NP + 255) / 256, 256>>>(tr.A[2], wh, yp, yb, mask, inv_n, tr.dA,
                                         backward ? tr.g + 3 * SCHED_WCONV : nullptr, tr.stat, tr.stat + 1, NP);
  if (backward) {
    // dA holds dPre of layer 2 (relu' applied); walk back
    float* dcur = tr.dA;
    float* dnext = tr.dB;
    for (int l = 2; l >= 0; --l) {
      const float* X = l == 0 ? tr.X : tr.A[l - 1];
      const int chunk = 2048;
      dim3 gw((NP + chunk - 1) / chunk, SCHED_TAPS);
      k_conv_bwd_weight<<<gw, 256>>>(X, dcur, tr.g + l * SCHED_WCONV, NP, tr.D, chunk);
      if (l > 0) {
        k_conv_bwd_data<<<blocks, 256>>>(dcur, tr.wr + l * SCHED_WCONV, tr.A[l - 1], dnext, NP, tr.D);
        std::swap(dcur, dnext);
      }
    }
  }
  CGC_CUDA(cudaGetLastError());
  float st[2];
  CGC_CUDA(cudaMemcpy(st, tr.stat, sizeof(st), cudaMemcpyDeviceToHost));
  if (loss) *loss = st[0];
  if (acc) *acc = st[1];
  return CGC_OK;
}

}  // namespace cgc

namespace cgc {
namespace {
__global__ void __launch_bounds__(256) k_infer_layer(GridSpace sp, int layer, SchedIO io) {
  sched_layer(sp, layer, io, blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5), gridDim.x * (blockDim.x >> 5),
              nullptr);
}
}  // namespace
}  // namespace cgc

struct cgc_trainer { cgc::Trainer t; };

extern "C" {

int cgc_scheduler_load(const uint16_t* conv_bf16, const float* head) {
  if (!conv_bf16 || !head) return cgc::fail(CGC_ERR_ARG, "cgc_scheduler_load: null weights");
  std::lock_guard<std::mutex> lock(cgc::g_wmu);
  cgc::g_wconv.assign(conv_bf16, conv_bf16 + 3 * cgc::SCHED_WCONV);
  cgc::g_whead.assign(head, head + cgc::SCHED_NHEAD);
  ++cgc::g_wver;
  return cgc::ok();
}

int cgc_scheduler_load_file(const char* path) {
  if (!path) return cgc::fail(CGC_ERR_ARG, "cgc_scheduler_load_file: null path");
  FILE* f = std::fopen(path, "rb");
  if (!f) return cgc::fail(CGC_ERR_ARG, std::string("cannot open ") + path);
  char magic[8] = {0};
  std::vector<uint16_t> conv(3 * cgc::SCHED_WCONV);
  std::vector<float> head(cgc::SCHED_NHEAD);
  const bool okr = std::fread(magic, 1, 8, f) == 8 && std::memcmp(magic, "CGCSCHD1", 8) == 0 &&
                   std::fread(conv.data(), 2, conv.size(), f) == conv.size() &&
                   std::fread(head.data(), 4, head.size(), f) == head.size();
  std::fclose(f);
  if (!okr) return cgc::fail(CGC_ERR_ARG, std::string("not a scheduler weight file: ") + path);
  return cgc_scheduler_load(conv.data(), head.data());
}

int cgc_scheduler_infer(int32_t grids, int32_t D, const uint16_t* feat, uint8_t* budget, uint8_t* prio, float* logits,
                        void* stream) {
  using namespace cgc;
  if (grids <= 0 || D <= 0 || !feat || !budget || !prio) return fail(CGC_ERR_ARG, "cgc_scheduler_infer: bad arguments");
  std::vector<uint32_t> frag;
  std::vector<float> head;
  {
    std::lock_guard<std::mutex> lock(g_wmu);
    if (!g_wver) return fail(CGC_ERR_STATE, "cgc_scheduler_infer: no weights are loaded (cgc_scheduler_load)");
    frag = fragment_order(g_wconv);
    head = g_whead;
  }
  const int64_t T = (int64_t)grids * D * D * D;
  if (T > (int64_t)1 << 30) return fail(CGC_ERR_ARG, "cgc_scheduler_infer: too many tiles");
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  char* buf = nullptr;
  const size_t act_bytes = (size_t)T * SCHED_C * 2;
  CGC_CUDA(cudaMalloc(&buf, 2 * act_bytes + frag.size() * 4 + head.size() * 4));
  auto release = [&]() { cudaFree(buf); };
  uint32_t* a0 = reinterpret_cast<uint32_t*>(buf);
  uint32_t* a1 = reinterpret_cast<uint32_t*>(buf + act_bytes);
  uint2* wf = reinterpret_cast<uint2*>(buf + 2 * act_bytes);
  float* wh = reinterpret_cast<float*>(buf + 2 * act_bytes + frag.size() * 4);
  cudaError_t e = cudaMemcpyAsync(wf, frag.data(), frag.size() * 4, cudaMemcpyHostToDevice, st);
  if (e == cudaSuccess) e = cudaMemcpyAsync(wh, head.data(), head.size() * 4, cudaMemcpyHostToDevice, st);
  const GridSpace sp{grids, D};
  const unsigned blocks = (unsigned)std::min<int64_t>((T + 127) / 128, 8192);
  for (int layer = 0; layer < 3 && e == cudaSuccess; ++layer) {
    SchedIO io{};
    io.in = layer == 0 ? reinterpret_cast<const uint32_t*>(feat) : (layer == 1 ? a0 : a1);
    io.out = layer == 0 ? a0 : a1;
    io.wf = wf + (size_t)layer * SCHED_FRAG;
    io.wh = wh;
    io.budget = budget;
    io.prio = prio;
    io.logits = logits;
    k_infer_layer<<<blocks, 256, 0, st>>>(sp, layer, io);
    note_launch();
    e = cudaGetLastError();
  }
  if (e == cudaSuccess) e = cudaStreamSynchronize(st);
  release();
  if (e != cudaSuccess) return fail(CGC_ERR_CUDA, std::string("cgc_scheduler_infer: ") + cudaGetErrorString(e));
  return ok();
}

int cgc_trainer_create(int32_t max_grids, int32_t D, uint64_t seed, cgc_trainer** out) {
  if (!out || max_grids <= 0 || D <= 0) return cgc::fail(CGC_ERR_ARG, "cgc_trainer_create: bad arguments");
  cgc_trainer* T = new cgc_trainer();
  cgc::Trainer& tr = T->t;
  tr.max_grids = max_grids;
  tr.D = D;
  tr.NP = max_grids * D * D * D;
  const size_t np = tr.nparam;
  const size_t act = (size_t)tr.NP * cgc::SCHED_C;
  cudaError_t e = cudaSuccess;
  for (float** q : {&tr.w, &tr.wr, &tr.g, &tr.m, &tr.v})
    if (e == cudaSuccess) e = cudaMalloc(q, np * sizeof(float));
  for (float** q : {&tr.X, &tr.A[0], &tr.A[1], &tr.A[2], &tr.dA, &tr.dB})
    if (e == cudaSuccess) e = cudaMalloc(q, act * sizeof(float));
  if (e == cudaSuccess) e = cudaMalloc(&tr.stat, 4 * sizeof(float));
  for (uint32_t** q : {&tr.A16[0], &tr.A16[1]})
    if (e == cudaSuccess) e = cudaMalloc(q, act * 2);
  if (e == cudaSuccess) e = cudaMalloc(&tr.wf, (size_t)3 * cgc::SCHED_FRAG * sizeof(uint2));
  if (e != cudaSuccess) { delete T; return cgc::fail(CGC_ERR_OOM, "cgc_trainer_create: device allocation"); }
  // He-uniform initialisation of the convolutions, small head
  std::mt19937_64 rng(seed);
  std::uniform_real_distribution<float> u(-1.f, 1.f);
  std::vector<float> w(np, 0.f);
  const float bc = std::sqrt(6.f / (cgc::SCHED_TAPS * cgc::SCHED_C));
  for (int i = 0; i < 3 * cgc::SCHED_WCONV; ++i) w[i] = bc * u(rng);
  for (int i = 0; i < 2 * cgc::SCHED_C; ++i) w[3 * cgc::SCHED_WCONV + i] = 0.25f * u(rng);
  cudaMemcpy(tr.w, w.data(), np * 4, cudaMemcpyHostToDevice);
  cudaMemset(tr.m, 0, np * 4);
  cudaMemset(tr.v, 0, np * 4);
  cgc::k_round_bf16<<<(int)((np + 255) / 256), 256>>>(tr.w, tr.wr, (int)np);
  if (cudaGetLastError() != cudaSuccess) { delete T; return cgc::fail(CGC_ERR_CUDA, "cgc_trainer_create: init"); }
  *out = T;
  return cgc::ok();
}

int cgc_trainer_destroy(cgc_trainer* t) {
  delete t;
  return cgc::ok();
}

int cgc_trainer_step(cgc_trainer* T, int32_t grids, const uint16_t* feat, const float* prio, const float* budget,
                     const float* mask, float count, float lr, float* loss) {
  if (!T) return cgc::fail(CGC_ERR_ARG, "null trainer");
  cgc::Trainer& tr = T->t;
  int rc = cgc::trainer_forward_backward(tr, grids, feat, prio, budget, mask, count, true, loss, nullptr);
  if (rc) return rc;
  ++tr.steps;
  const float b1 = 0.9f, b2 = 0.999f;
  const float c1 = 1.f - std::pow(b1, (float)tr.steps), c2 = 1.f - std::pow(b2, (float)tr.steps);
  cgc::k_adam<<<(tr.nparam + 255) / 256, 256>>>(tr.w, tr.g, tr.m, tr.v, tr.nparam, lr, b1, b2, 1e-8f, c1, c2);
  cgc::k_round_bf16<<<(tr.nparam + 255) / 256, 256>>>(tr.w, tr.wr, tr.nparam);
  CGC_CUDA(cudaGetLastError());
  return cgc::ok();
}

int cgc_trainer_eval(cgc_trainer* T, int32_t grids, const uint16_t* feat, const float* prio, const float* budget,
                     const float* mask, float count, float* loss, float* accuracy) {
  if (!T) return cgc::fail(CGC_ERR_ARG, "null trainer");
  int rc = cgc::trainer_forward_backward(T->t, grids, feat, prio, budget, mask, count, false, loss, accuracy);
  return rc ? rc : cgc::ok();
}

int cgc_trainer_weights(cgc_trainer* T, uint16_t* conv_bf16, float* head) {
  if (!T || !conv_bf16 || !head) return cgc::fail(CGC_ERR_ARG, "null argument");
  cgc::Trainer& tr = T->t;
  std::vector<float> w(tr.nparam);
  CGC_CUDA(cudaMemcpy(w.data(), tr.w, w.size() * 4, cudaMemcpyDeviceToHost));
  for (int i = 0; i < 3 * cgc::SCHED_WCONV; ++i) {
    __nv_bfloat16 b = __float2bfloat16(w[i]);
    std::memcpy(conv_bf16 + i, &b, 2);
  }
  for (int i = 0; i < cgc::SCHED_NHEAD; ++i) head[i] = w[3 * cgc::SCHED_WCONV + i];
  return cgc::ok();
}

}  // extern "C"
