// Edge-list front door: cugip::Graph<TFlow>::set_nweights takes an arbitrary
// list of EdgeRecord(first,second) with forward/backward capacities
// (include/cugip/advanced_operations/graph_cut.hpp:239-290) and builds a CSR
// graph on the host.  The engine here is grid-native, so this entry point
// recognises an edge list that is a 6-connected X*Y*Z grid with linear vertex
// ids (x fastest) -- the shape every grid front-end of the reference produces
// (benchmarks/graph_cut/boykov_kolmogorov.cpp:47-64 numbers voxels this way)
// -- and scatters its capacities into the per-axis n-link planes.  Anything
// else returns CGC_ERR_NOT_GRID.
#include <algorithm>
#include <cstdint>
#include <cstring>
#include <string>
#include <vector>

#include "cgc.h"
#include "cgc_internal.h"

namespace {

// axis of the grid edge (lo, lo+d) in an X*Y*Z grid, or -1 if it is not one
int axis_of(int64_t lo, int64_t d, int64_t X, int64_t Y, int64_t Z) {
  const int64_t XY = X * Y;
  if (d == 1 && X > 1 && lo % X != X - 1) return 0;
  if (d == X && Y > 1 && (lo / X) % Y != Y - 1) return 1;
  if (d == XY && Z > 1) return 2;
  return -1;
}

bool try_dims(int64_t n, int64_t X, int64_t XY, int64_t m, const uint32_t* a, const uint32_t* b) {
  if (X <= 0 || XY <= 0 || XY % X != 0 || n % XY != 0) return false;
  const int64_t Y = XY / X, Z = n / XY;
  for (int64_t i = 0; i < m; ++i) {
    const int64_t lo = std::min<int64_t>(a[i], b[i]), hi = std::max<int64_t>(a[i], b[i]);
    if (axis_of(lo, hi - lo, X, Y, Z) < 0) return false;
  }
  return true;
}

}  // namespace

extern "C" int cgc_detect_grid(int32_t n, int64_t m, const uint32_t* a, const uint32_t* b, int32_t* dims) {
  if (n <= 0 || m < 0 || (m > 0 && (!a || !b)) || !dims) return cgc::fail(CGC_ERR_ARG, "cgc_detect_grid: bad arguments");
  std::vector<int64_t> ds;
  for (int64_t i = 0; i < m; ++i) {
    if (a[i] >= (uint32_t)n || b[i] >= (uint32_t)n || a[i] == b[i])
      return cgc::fail(CGC_ERR_NOT_GRID, "cgc_detect_grid: vertex id out of range or self loop");
    const int64_t d = (int64_t)std::max(a[i], b[i]) - (int64_t)std::min(a[i], b[i]);
    if (std::find(ds.begin(), ds.end(), d) == ds.end()) {
      ds.push_back(d);
      if (ds.size() > 3) return cgc::fail(CGC_ERR_NOT_GRID, "edge list has more than 3 distinct id strides");
    }
  }
  std::sort(ds.begin(), ds.end());
  std::vector<std::pair<int64_t, int64_t>> cand;  // (X, X*Y)
  if (ds.empty()) cand.push_back({n, n});
  else if (ds.size() == 1) {
    cand.push_back({ds[0] == 1 ? n : ds[0], n});
    if (ds[0] != 1) cand.push_back({1, ds[0]});
  } else if (ds.size() == 2) {
    if (ds[0] == 1) { cand.push_back({ds[1], n}); cand.push_back({n, ds[1]}); cand.push_back({1, ds[1]}); }
    else cand.push_back({ds[0], ds[1]});
  } else {
    if (ds[0] == 1) cand.push_back({ds[1], ds[2]});
  }
  for (auto& c : cand) {
    int64_t X = c.first, XY = c.second;
    if (XY > n || X > XY) continue;
    if (try_dims(n, X, XY, m, a, b)) {
      dims[0] = (int32_t)X; dims[1] = (int32_t)(XY / X); dims[2] = (int32_t)(n / XY);
      return cgc::ok();
    }
  }
  return cgc::fail(CGC_ERR_NOT_GRID, "edge list is not a 6-connected grid with linear vertex ids");
}

extern "C" int cgc_grid_create_from_edges(int32_t n, int64_t m, const uint32_t* a, const uint32_t* b,
                                          const int32_t* fwd, const int32_t* bwd, void* stream, cgc_grid** out,
                                          int32_t* dims_out) {
  if (!out || (m > 0 && (!fwd || !bwd))) return cgc::fail(CGC_ERR_ARG, "cgc_grid_create_from_edges: bad arguments");
  int32_t dims[3];
  int rc = cgc_detect_grid(n, m, a, b, dims);
  if (rc) return rc;
  std::vector<int32_t> planes;
  try { planes.assign((size_t)6 * n, 0); } catch (...) { return cgc::fail(CGC_ERR_OOM, "host allocation"); }
  for (int64_t i = 0; i < m; ++i) {
    const bool ab = a[i] < b[i];
    const int64_t lo = ab ? a[i] : b[i], hi = ab ? b[i] : a[i];
    const int axis = axis_of(lo, hi - lo, dims[0], dims[1], dims[2]);
    const int64_t up = ab ? fwd[i] : bwd[i];    // lo -> hi
    const int64_t down = ab ? bwd[i] : fwd[i];  // hi -> lo
    int32_t& f = planes[(size_t)(2 * axis) * n + lo];
    int32_t& g = planes[(size_t)(2 * axis + 1) * n + lo];
    if (up < 0 || down < 0) return cgc::fail(CGC_ERR_ARG, "negative n-link capacity");
    if ((int64_t)f + up > 2147483647 || (int64_t)g + down > 2147483647)
      return cgc::fail(CGC_ERR_OVERFLOW, "parallel edges overflow int32");
    f += (int32_t)up;  // parallel edges add up
    g += (int32_t)down;
  }
  cgc_grid* g = nullptr;
  rc = cgc_grid_create(dims[0], dims[1], dims[2], stream, &g);
  if (rc) return rc;
  for (int ax = 0; ax < 3; ++ax) {
    rc = cgc_grid_set_nlinks(g, ax, planes.data() + (size_t)(2 * ax) * n, planes.data() + (size_t)(2 * ax + 1) * n);
    if (rc) { cgc_grid_destroy(g); return rc; }
  }
  *out = g;
  if (dims_out) std::memcpy(dims_out, dims, sizeof(dims));
  return cgc::ok();
}
