// Device-side construction of the segmentation grid graph from an image and a
// marker volume.
//
// The reference builds this graph on the host, voxel by voxel
// (benchmarks/graph_cut/graph_cut.cpp:33-98, the same in
// benchmarks/graph_cut/boykov_kolmogorov.cpp:44-68):
//   * source t-link = hard weight where marker == 128, sink t-link = hard
//     weight where marker == 255, and every voxel within 2 voxels of the
//     volume border (min(c) <= 1 or min(size - c) <= 2) is forced to the
//     source with no sink link;
//   * one n-link per 6-neighbour pair with the same weight both ways,
//     w = exp(-(I_i - I_j)^2 / 2 * sigma^2) in float -- as written, with the
//     operator precedence of graph_cut.cpp:73 (the sigma^2 multiplies);
//     flag CGC_BUILD_GAUSSIAN selects the Gaussian exp(-(I_i-I_j)^2 / (2 sigma^2)).
// The engine is exact over integers, so the weights are scaled by
// nlink_scale and rounded (half away from zero); the hard t-link is an int.
#include <cuda_runtime.h>

#include <cmath>
#include <string>

#include "cgc.h"
#include "cgc_internal.h"
#include "cgc_pool.h"

namespace cgc {
namespace {

__device__ __forceinline__ int32_t round_half_away(float v) { return (int32_t)floorf(v + 0.5f); }

__device__ __forceinline__ int32_t nlink(float a, float b, float sigma2, int gaussian, float scale) {
  const float d = a - b;
  const float q = gaussian ? (d * d) / (2.0f * sigma2) : (d * d) / 2.0f * sigma2;
  return round_half_away(scale * expf(-q));
}

__global__ void k_build(int X, int Y, int Z, const float* __restrict__ img, const uint8_t* __restrict__ mk, float sigma2,
                        int gaussian, float scale, int32_t hard, int32_t* capS, int32_t* capT, int32_t* nx, int32_t* ny,
                        int32_t* nz) {
  const int64_t N = (int64_t)X * Y * Z;
  for (int64_t v = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; v < N; v += (int64_t)gridDim.x * blockDim.x) {
    const int x = (int)(v % X), y = (int)((v / X) % Y), z = (int)(v / ((int64_t)X * Y));
    const uint8_t m = mk ? mk[v] : 0;
    int32_t s = m == 128 ? hard : 0, t = m == 255 ? hard : 0;
    const int lo = min(x, min(y, z)), hi = min(X - x, min(Y - y, Z - z));
    if (lo <= 1 || hi <= 2) { s = hard; t = 0; }
    capS[v] = s;
    capT[v] = t;
    const float iv = img[v];
    nx[v] = x + 1 < X ? nlink(iv, img[v + 1], sigma2, gaussian, scale) : 0;
    ny[v] = y + 1 < Y ? nlink(iv, img[v + X], sigma2, gaussian, scale) : 0;
    nz[v] = z + 1 < Z ? nlink(iv, img[v + (int64_t)X * Y], sigma2, gaussian, scale) : 0;
  }
}

}  // namespace
}  // namespace cgc

extern "C" int cgc_build_segmentation_graph(int32_t X, int32_t Y, int32_t Z, const float* image, const uint8_t* markers,
                                            float sigma, int32_t nlink_scale, int32_t hard_tlink, int32_t flags,
                                            int32_t* capS, int32_t* capT, int32_t* nx, int32_t* ny, int32_t* nz,
                                            void* stream) {
  if (X <= 0 || Y <= 0 || Z <= 0 || !image || !capS || !capT || !nx || !ny || !nz)
    return cgc::fail(CGC_ERR_ARG, "cgc_build_segmentation_graph: bad arguments");
  if (nlink_scale < 0 || hard_tlink < 0 || !(sigma > 0.0f))
    return cgc::fail(CGC_ERR_ARG, "cgc_build_segmentation_graph: scales must be >= 0 and sigma > 0");
  if ((int64_t)hard_tlink + 6ll * nlink_scale > 2147483647ll)
    return cgc::fail(CGC_ERR_OVERFLOW, "cgc_build_segmentation_graph: hard_tlink + 6*nlink_scale exceeds int32");
  const int64_t N = (int64_t)X * Y * Z;
  const int blocks = (int)std::min<int64_t>((N + 255) / 256, 1 << 16);
  cgc::k_build<<<blocks, 256, 0, (cudaStream_t)stream>>>(X, Y, Z, image, markers, sigma * sigma,
                                                          (flags & CGC_BUILD_GAUSSIAN) ? 1 : 0, (float)nlink_scale,
                                                          hard_tlink, capS, capT, nx, ny, nz);
  cgc::note_launch();
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return cgc::fail(CGC_ERR_CUDA, std::string("cgc_build_segmentation_graph: ") + cudaGetErrorString(e));
  return cgc::ok();
}
