// Autotuner for the solve schedule.
//
// The reference fixes its schedule at compile time (GraphCutPolicy /
// RelabelPolicy / PushPolicy, include/cugip/advanced_operations/detail/
// graph_cut_policies.hpp:23-89).  Here the knobs are runtime options:
// pulses per region-relabel round (L), region-relabel rounds per tile visit
// (R), sweep pairs between exact global relabels (K) and the shape of the
// persistent kernel (a 512-thread CTA per tile visit at 2, 3 or 4 CTAs per SM,
// or a warp per tile visit).  The autotuner times candidate
// settings on the caller's own uploaded instance(s), keeps the fastest per size
// class (instance count, voxel count) in a process-wide cache and, when the
// environment variable CGC_AUTOTUNE_CACHE names a file, appends each result to
// it and reads it back on the first lookup.  The flow and cut sets do not
// depend on the schedule; only the time does.
#include <cuda_runtime.h>

#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <map>
#include <mutex>
#include <string>
#include <vector>

#include "cgc.h"
#include "cgc_pool.h"

namespace cgc {
namespace {

std::mutex g_mu;
std::map<std::pair<int, int>, std::pair<cgc_options, double>> g_cache;
bool g_loaded = false;

std::pair<int, int> size_class(int64_t voxels, int32_t instances) {
  const int ib = instances <= 1 ? 0 : (int)std::ceil(std::log2((double)instances));
  const int vb = voxels <= 1 ? 0 : (int)std::floor(2.0 * std::log2((double)voxels));
  return {ib, vb};
}

void load_cache_locked() {
  if (g_loaded) return;
  g_loaded = true;
  const char* path = std::getenv("CGC_AUTOTUNE_CACHE");
  if (!path) return;
  FILE* f = std::fopen(path, "r");
  if (!f) return;
  // line: size class (2), L R K ctas stall learned bfs_warp_min exclusive
  // relabel, milliseconds (lines without exclusive and relabel are read too)
  char line[256];
  while (std::fgets(line, sizeof line, f)) {
    int ib, vb, L, R, K, cta, st, lr, bw, ex = 0, rl = 0;
    double ms;
    if (std::sscanf(line, "%d %d %d %d %d %d %d %d %d %d %d %lf", &ib, &vb, &L, &R, &K, &cta, &st, &lr, &bw, &ex, &rl,
                    &ms) != 12 &&
        std::sscanf(line, "%d %d %d %d %d %d %d %d %d %lf", &ib, &vb, &L, &R, &K, &cta, &st, &lr, &bw, &ms) != 10)
      continue;
    cgc_options o{};
    o.struct_size = sizeof(cgc_options);
    o.local_pulses = L; o.region_relabels = R; o.sweeps_per_relabel = K; o.ctas_per_sm = cta; o.stall_sweeps = st;
    o.learned = lr;
    o.bfs_warp_min = bw;
    o.exclusive = ex;
    o.relabel = rl;
    g_cache[{ib, vb}] = {o, ms};
  }
  std::fclose(f);
}

void store(std::pair<int, int> key, const cgc_options& o, double ms) {
  std::lock_guard<std::mutex> lock(g_mu);
  load_cache_locked();
  g_cache[key] = {o, ms};
  if (const char* path = std::getenv("CGC_AUTOTUNE_CACHE")) {
    if (FILE* f = std::fopen(path, "a")) {
      std::fprintf(f, "%d %d %d %d %d %d %d %d %d %d %d %.6f\n", key.first, key.second, o.local_pulses,
                   o.region_relabels, o.sweeps_per_relabel, o.ctas_per_sm, o.stall_sweeps, o.learned, o.bfs_warp_min,
                   o.exclusive, o.relabel, ms);
      std::fclose(f);
    }
  }
}

std::vector<cgc_options> default_candidates() {
  std::vector<cgc_options> c;
  for (int cta : {2, 3, 4})
    for (int R : {1, 2, 4})
      for (int L : {2, 4, 8})
        for (int K : {4, 8, 16})
          for (int bw : {0, 8}) {
            if (bw && cta == 2) continue;  // warp-per-tile BFS rounds exist at 3 and 4 CTAs/SM
            cgc_options o{};
            o.struct_size = sizeof(cgc_options);
            o.local_pulses = L; o.region_relabels = R; o.sweeps_per_relabel = K; o.ctas_per_sm = cta;
            o.bfs_warp_min = bw;
            c.push_back(o);
          }
  return c;
}

bool inputs_bound(const Pool& p) {
  if (!p.d_in) return false;
  for (int i = 0; i < p.ninst; ++i)
    if (!p.in_ptrs[8 * (size_t)i]) return false;
  return true;
}

int64_t total_voxels(const Pool& p) {
  int64_t n = 0;
  for (const InstGeo& G : p.geo) n += (int64_t)G.X * G.Y * G.Z;
  return n;
}

}  // namespace

int pool_autotune(Pool& p, const cgc_options* cands, int32_t n, int32_t repeats, cgc_options* best, double* best_ms) {
  std::vector<cgc_options> cand = (cands && n > 0) ? std::vector<cgc_options>(cands, cands + n) : default_candidates();
  if (repeats <= 0) repeats = 1;
  const bool bound = inputs_bound(p);
  if (p.pending) return fail(CGC_ERR_STATE, "autotune: a solve of this handle was not waited for");
  if (!bound)
    for (int i = 0; i < p.ninst; ++i)
      if (!(p.uploaded[i] & 1u)) return fail(CGC_ERR_STATE, "autotune: set the capacities (or bind device inputs) first");
  // the set_* inputs stay in their linear planes through a solve: marking
  // them as set again restores them
  const std::vector<uint32_t> uploaded = p.uploaded;
  auto restore = [&]() -> int {
    if (!bound) p.uploaded = uploaded;
    return CGC_OK;
  };
  cudaEvent_t e0, e1;
  CGC_CUDA(cudaEventCreate(&e0));
  CGC_CUDA(cudaEventCreate(&e1));
  double best_t = 1e30;
  int best_i = -1;
  int rc = CGC_OK;
  for (size_t i = 0; i < cand.size() && rc == CGC_OK; ++i) {
    double t_min = 1e30;
    bool ok_all = true;
    for (int r = 0; r < repeats; ++r) {
      if ((rc = restore())) break;
      float ms = 0.f;
      if (bound) {
        CGC_CUDA(cudaEventRecord(e0, p.stream));
        if ((rc = pool_enqueue(p, &cand[i], nullptr, p.stream))) break;
        CGC_CUDA(cudaEventRecord(e1, p.stream));
        if (pool_wait(p, p.stream)) { ok_all = false; break; }
        CGC_CUDA(cudaEventElapsedTime(&ms, e0, e1));
      } else {
        if (pool_solve(p, &cand[i])) { ok_all = false; break; }
        ms = (float)p.st.solve_ms;
      }
      t_min = std::min(t_min, (double)ms);
    }
    if (ok_all && t_min < best_t) { best_t = t_min; best_i = (int)i; }
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  int rc2 = restore();
  if (rc) return rc;
  if (rc2) return rc2;
  if (best_i < 0) return fail(CGC_ERR_STATE, "autotune: every candidate failed");
  cgc_options b = resolve_options(&cand[best_i]);
  store(size_class(total_voxels(p), p.ninst), b, best_t);
  if (best) *best = b;
  if (best_ms) *best_ms = best_t;
  p.solved = false;
  return ok();
}

}  // namespace cgc

struct cgc_grid { cgc::Pool* p; };
struct cgc_batch { cgc::Pool* p; };

extern "C" {

int cgc_grid_autotune(cgc_grid* g, const cgc_options* candidates, int32_t n, int32_t repeats, cgc_options* best,
                      double* best_ms) {
  if (!g) return cgc::fail(CGC_ERR_ARG, "null grid");
  return cgc::pool_autotune(*g->p, candidates, n, repeats, best, best_ms);
}

int cgc_batch_autotune(cgc_batch* b, const cgc_options* candidates, int32_t n, int32_t repeats, cgc_options* best,
                       double* best_ms) {
  if (!b) return cgc::fail(CGC_ERR_ARG, "null batch");
  return cgc::pool_autotune(*b->p, candidates, n, repeats, best, best_ms);
}

int cgc_autotune_lookup(int64_t voxels, int32_t instances, cgc_options* out) {
  if (!out) return cgc::fail(CGC_ERR_ARG, "null output");
  std::lock_guard<std::mutex> lock(cgc::g_mu);
  cgc::load_cache_locked();
  auto it = cgc::g_cache.find(cgc::size_class(voxels, instances));
  if (it == cgc::g_cache.end()) return cgc::fail(CGC_ERR_STATE, "autotune: no entry for this size class");
  *out = it->second.first;
  return cgc::ok();
}

}  // extern "C"
