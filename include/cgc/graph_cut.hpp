// cgc/graph_cut.hpp — header-only C++ facade over the C ABI of libcgc.so that
// mirrors cugip's graph-cut API, so reference callers switch by changing the
// include and the namespace:
//
//   cugip::Graph<TFlow>            include/cugip/advanced_operations/graph_cut.hpp:47-146
//   cugip::EdgeRecord              include/cugip/advanced_operations/detail/edge_record.hpp:10-29
//   cugip::DummyTraceObject        include/cugip/advanced_operations/graph_cut.hpp:26-45
//   cugip::GraphCutPolicy          include/cugip/advanced_operations/detail/graph_cut_policies.hpp:80-89
//   CUGIP_CHECK_RESULT -> throw    include/cugip/exception.hpp:33-47
//
// Capacities are exact integers: TFlow may be an integer type or a floating
// type holding integral values in [0, 2^31); anything else throws.  The flow is
// returned as TFlow (computed in int64).
#pragma once

#include <cstdint>
#include <cmath>
#include <stdexcept>
#include <string>
#include <type_traits>
#include <vector>

#include "../cgc.h"

namespace cgc {

class Exception : public std::runtime_error {
 public:
  Exception(int code, const std::string& what) : std::runtime_error(what), code_(code) {}
  int code() const { return code_; }

 private:
  int code_;
};

inline void check(int rc, const char* where) {
  if (rc != CGC_OK) throw Exception(rc, std::string(where) + ": " + cgc_last_error());
}

// Same layout as cugip::EdgeRecord: a union of a 64-bit id with
// {second, first}; the constructor stores (min, max).
typedef unsigned NodeId;
struct EdgeRecord {
  EdgeRecord(NodeId a, NodeId b) : second(a < b ? b : a), first(a < b ? a : b) {}
  EdgeRecord() : second(0), first(0) {}
  NodeId second;
  NodeId first;
};
static_assert(sizeof(EdgeRecord) == 8, "EdgeRecord layout");

// Runtime policy (the reference's compile-time GraphCutPolicy knobs).
struct GraphCutPolicy {
  int local_pulses = 0;        // pulses per region-relabel round of a tile visit
  int region_relabels = 0;     // region relabels per tile visit (-1: none)
  int sweeps_per_relabel = 0;  // sweep pairs between exact global relabels
  int persistent = 0;          // 1: one cooperative launch, -1: host loop
  int wait_limit_us = 0;       // bound of every device-side wait in microseconds (0: 20 s)
  int max_sweeps = 0;          // safety cap (0: default)
  int stall_sweeps = 0;        // relabel early after this many idle sweep pairs (0: never)
  int ctas_per_sm = 0;         // 2 (default), 3 or 4 CTAs per SM
  int learned = 0;             // learned scheduler: 1 budgets + priorities, 2 budgets only
  int bfs_warp_min = 0;        // 3/4 CTAs per SM: BFS rounds with this many tiles per CTA use a warp per tile
  int exclusive = 0;           // 1: sweeps visit every queued tile without a queued face neighbour of the sweep's parity
  int relabel = 0;             // global relabels after a solve's first: 1 full BFS, 2 incremental (0: default, 2)
  cgc_options options() const {
    cgc_options o{};
    o.struct_size = sizeof(cgc_options);
    o.local_pulses = local_pulses;
    o.region_relabels = region_relabels;
    o.sweeps_per_relabel = sweeps_per_relabel;
    o.persistent = persistent;
    o.wait_limit_us = wait_limit_us;
    o.max_sweeps = max_sweeps;
    o.stall_sweeps = stall_sweeps;
    o.ctas_per_sm = ctas_per_sm;
    o.learned = learned;
    o.bfs_warp_min = bfs_warp_min;
    o.exclusive = exclusive;
    o.relabel = relabel;
    return o;
  }
  // The autotuner's choice for a size class (cgc_autotune_lookup), if any
  // solve of that class was tuned in this process or is in the cache file.
  static bool autotuned(int64_t voxels, int32_t instances, GraphCutPolicy* out) {
    cgc_options o{};
    o.struct_size = sizeof(cgc_options);
    if (cgc_autotune_lookup(voxels, instances, &o) != CGC_OK) return false;
    out->local_pulses = o.local_pulses;
    out->region_relabels = o.region_relabels;
    out->sweeps_per_relabel = o.sweeps_per_relabel;
    out->persistent = o.persistent;
    out->wait_limit_us = o.wait_limit_us;
    out->max_sweeps = o.max_sweeps;
    out->stall_sweeps = o.stall_sweeps;
    out->ctas_per_sm = o.ctas_per_sm;
    out->learned = o.learned;
    out->bfs_warp_min = o.bfs_warp_min;
    out->exclusive = o.exclusive;
    out->relabel = o.relabel;
    return true;
  }
};

class GridGraph;
class GenericGraph;
template <typename TFlow>
class Graph;

// Read-only view of a solve handed to the trace hooks, in place of the
// reference's device-side GraphCutData (detail/graph_cut_data.hpp:20-140,
// passed by MinCut::compute, detail/graph_cut_implementation.hpp:134-196):
//  * vertexCount() and mEdgeCount as there;
//  * iteration() (-1 before the first) and flow(): the exact flow delivered
//    when the reported iteration's push phase ended (0 in computationStarted;
//    -1 where the engine keeps no per-iteration record: generic graphs);
//  * for the final state (finalState(): the last afterPush and
//    computationFinished), host copies in vertex-id order, read from the device
//    on first use: vertexExcess() and labels() (the distance to the sink after
//    the last exact relabel, INVALID_LABEL where the sink cannot be reached --
//    the reference's label convention, graph_cut_policies.hpp:34).  Earlier
//    states are not kept: the whole solve is one device launch.
// Without the reference's CSR layout there are no device arrays to hand out.
template <typename TFlow>
class GraphCutData {
 public:
  static const int INVALID_LABEL = INT32_MIN;
  int mEdgeCount = 0;

  int vertexCount() const { return n_; }
  int iteration() const { return iteration_; }
  int64_t flow() const { return flow_; }
  bool finalState() const { return final_; }
  const cgc_stats& stats() const { return stats_; }
  const std::vector<TFlow>& vertexExcess() const {
    load();
    return excess_;
  }
  const std::vector<int>& labels() const {
    load();
    return labels_;
  }

 private:
  template <typename T>
  friend class Graph;
  void load() const;

  int n_ = 0;
  int iteration_ = -1;
  int64_t flow_ = 0;
  bool final_ = false;
  cgc_stats stats_{};
  const GridGraph* grid_ = nullptr;
  const GenericGraph* generic_ = nullptr;
  mutable bool loaded_ = false;
  mutable std::vector<TFlow> excess_;
  mutable std::vector<int> labels_;
};

// Trace protocol of the reference (graph_cut.hpp:26-45).  The solve runs as
// one device launch, so the per-iteration hooks are replayed after it: one
// iteration per exact global relabel, with the level starts of that relabel's
// BFS rounds and the flow at the end of its push phase from the solve's phase
// trace.  afterRelabel's level starts also bind to a parameter of type
// const thrust::host_vector<int>& (thrust converts from std::vector).
struct DummyTraceObject {
  template <typename TFlow>
  void computationStarted(const GraphCutData<TFlow>&) {}
  void beginIteration(int) {}
  void afterRelabel(int, const std::vector<int>&) {}
  template <typename TFlow>
  void afterPush(int, bool, const GraphCutData<TFlow>&) {}
  template <typename TFlow>
  void computationFinished(TFlow, const GraphCutData<TFlow>&) {}
};

namespace detail {
template <typename T>
std::vector<int32_t> to_i32(const T* a, size_t n, const char* what) {
  std::vector<int32_t> out(n);
  for (size_t i = 0; i < n; ++i) {
    const double v = static_cast<double>(a[i]);
    if (!(v >= 0.0) || v > 2147483647.0 || (std::is_floating_point<T>::value && std::floor(v) != v))
      throw Exception(CGC_ERR_ARG, std::string(what) + ": capacities must be integers in [0, 2^31)");
    out[i] = static_cast<int32_t>(v);
  }
  return out;
}
}  // namespace detail

// X*Y*Z grid graph with per-axis n-link volumes (vertex id = x + X*(y + Y*z)).
class GridGraph {
 public:
  GridGraph(int X, int Y, int Z, void* stream = nullptr) : X_(X), Y_(Y), Z_(Z) {
    check(cgc_grid_create(X, Y, Z, stream, &g_), "cgc_grid_create");
  }
  explicit GridGraph(cgc_grid* adopt, int X, int Y, int Z) : g_(adopt), X_(X), Y_(Y), Z_(Z) {}
  GridGraph(const GridGraph&) = delete;
  GridGraph& operator=(const GridGraph&) = delete;
  ~GridGraph() { cgc_grid_destroy(g_); }

  size_t size() const { return (size_t)X_ * Y_ * Z_; }
  void set_tweights(const int32_t* capS, const int32_t* capT) { check(cgc_grid_set_tlinks(g_, capS, capT), "set_tweights"); }
  void set_nweights(int axis, const int32_t* fwd, const int32_t* bwd) {
    check(cgc_grid_set_nlinks(g_, axis, fwd, bwd), "set_nweights");
  }
  int64_t max_flow(const GraphCutPolicy* policy = nullptr) {
    int64_t f = 0;
    cgc_options o;
    if (policy) o = policy->options();
    check(cgc_grid_maxflow(g_, policy ? &o : nullptr, &f), "max_flow");
    return f;
  }
  void segments(int which, uint8_t* out, uint8_t mask = 255, uint8_t bg = 0) const {
    check(cgc_grid_get_segments(g_, which, out, mask, bg), "fill_segments");
  }
  // distance labels (INT32_MIN: cannot reach the sink) and excess of the last solve
  void labels(int32_t* out) const { check(cgc_grid_get_labels(g_, out), "labels"); }
  void excess(int32_t* out) const { check(cgc_grid_get_residuals(g_, nullptr, nullptr, out), "excess"); }
  cgc_stats stats() const {
    cgc_stats s;
    check(cgc_grid_stats(g_, &s), "stats");
    return s;
  }
  // Phase records of the last persistent solve (cgc_grid_trace): kind 1 = BFS
  // round, 2 = global relabel done (tiles = active tiles), 3 = sweep, 4 =
  // reachability round, 5 = flow at a global relabel; `tiles` = tiles in the
  // round; `value` = ns since the launch (kind 5: the exact flow so far).
  struct PhaseRecord {
    int kind;
    int64_t index;
    int tiles;
    int64_t value;
  };
  std::vector<PhaseRecord> trace() const {
    int32_t n = 0;
    check(cgc_grid_trace(g_, nullptr, 0, &n), "trace");
    std::vector<int64_t> buf(2 * (size_t)n);
    if (n > 0) check(cgc_grid_trace(g_, buf.data(), n, &n), "trace");
    std::vector<PhaseRecord> out((size_t)n);
    for (int32_t i = 0; i < n; ++i) {
      const uint64_t w = (uint64_t)buf[2 * (size_t)i];
      out[(size_t)i] = PhaseRecord{(int)(w >> 56), (int64_t)((w >> 24) & 0xffffffffu), (int)(w & 0xffffffu),
                                   buf[2 * (size_t)i + 1]};
    }
    return out;
  }
  cgc_grid* handle() const { return g_; }

 private:
  cgc_grid* g_ = nullptr;
  int X_, Y_, Z_;
};

// Any edge list on the GPU (cgc_graph_*): the non-grid path of Graph.
class GenericGraph {
 public:
  GenericGraph(int32_t n, int64_t m, const int32_t* a, const int32_t* b, const int32_t* cap_ab, const int32_t* cap_ba)
      : n_(n) {
    check(cgc_graph_create(n, m, a, b, cap_ab, cap_ba, nullptr, &g_), "set_nweights");
  }
  GenericGraph(const GenericGraph&) = delete;
  GenericGraph& operator=(const GenericGraph&) = delete;
  ~GenericGraph() { if (g_) cgc_graph_destroy(g_); }

  size_t size() const { return (size_t)n_; }
  void set_tweights(const int32_t* capS, const int32_t* capT) { check(cgc_graph_set_tlinks(g_, capS, capT), "set_tweights"); }
  int64_t max_flow(const GraphCutPolicy* policy = nullptr) {
    int64_t f = 0;
    cgc_options o;
    if (policy) o = policy->options();
    check(cgc_graph_maxflow(g_, policy ? &o : nullptr, &f), "max_flow");
    return f;
  }
  void segments(int which, uint8_t* out, uint8_t mask = 255, uint8_t bg = 0) const {
    check(cgc_graph_get_segments(g_, which, out, mask, bg), "fill_segments");
  }
  // distance labels (INT32_MIN: cannot reach the sink) and excess of the last solve
  void state(int32_t* labels, int32_t* excess) const { check(cgc_graph_get_state(g_, labels, excess), "state"); }
  cgc_stats stats() const {
    cgc_stats s;
    check(cgc_graph_stats(g_, &s), "stats");
    return s;
  }

 private:
  cgc_graph* g_ = nullptr;
  int32_t n_;
};

template <typename TFlow>
void GraphCutData<TFlow>::load() const {
  if (loaded_ || !final_) return;  // earlier states are not kept
  loaded_ = true;
  std::vector<int32_t> ex((size_t)n_), lb((size_t)n_);
  if (grid_) {
    grid_->excess(ex.data());
    grid_->labels(lb.data());
  } else if (generic_) {
    generic_->state(lb.data(), ex.data());
  }
  excess_.assign(ex.begin(), ex.end());
  labels_.assign(lb.begin(), lb.end());
}

// Drop-in for cugip::Graph<TFlow> (graph_cut.hpp:47-146).  An edge list that
// forms a 6-connected grid with linear vertex ids goes to the tile engine,
// any other graph to the generic engine.  Unlike the reference, the graph can
// be solved again after setting new weights.
template <typename TFlow>
class Graph {
 public:
  typedef int VertexId;
  typedef TFlow EdgeWeight;

  void set_vertex_count(int count) {
    n_ = count;
    grid_.reset();
    generic_.reset();
    tlink_s_.clear();
    tlink_t_.clear();
  }

  void set_nweights(int edge_count, const EdgeRecord* edges, const EdgeWeight* fwd, const EdgeWeight* bwd) {
    std::vector<uint32_t> a(edge_count), b(edge_count);
    for (int i = 0; i < edge_count; ++i) { a[i] = edges[i].first; b[i] = edges[i].second; }
    std::vector<int32_t> f = detail::to_i32(fwd, edge_count, "set_nweights");
    std::vector<int32_t> w = detail::to_i32(bwd, edge_count, "set_nweights");
    cgc_grid* g = nullptr;
    int32_t dims[3];
    grid_.reset();
    generic_.reset();
    edges_ = edge_count;
    const int rc = cgc_grid_create_from_edges(n_, edge_count, a.data(), b.data(), f.data(), w.data(), nullptr, &g, dims);
    if (rc == CGC_ERR_NOT_GRID) {
      std::vector<int32_t> ai(a.begin(), a.end()), bi(b.begin(), b.end());
      generic_.reset(new GenericGraph(n_, edge_count, ai.data(), bi.data(), f.data(), w.data()));
    } else {
      check(rc, "set_nweights");
      grid_.reset(new GridGraph(g, dims[0], dims[1], dims[2]));
    }
    // t-links set earlier (the reference accepts them in either order) apply
    // to the new graph as well
    if (!tlink_s_.empty()) apply_tlinks();
  }

  void set_tweights(const EdgeWeight* capSource, const EdgeWeight* capSink) {
    tlink_s_ = detail::to_i32(capSource, (size_t)n_, "set_tweights");
    tlink_t_ = detail::to_i32(capSink, (size_t)n_, "set_tweights");
    if (grid_ || generic_) apply_tlinks();
  }

  TFlow max_flow() {
    DummyTraceObject trace;
    return max_flow_with_tracing(trace);
  }
  // The flow as an exact int64.  max_flow() returns it converted to TFlow,
  // which for Graph<float> rounds flows above 2^24 (float's 24-bit mantissa).
  int64_t max_flow_exact() {
    max_flow();
    return last_flow_;
  }
  template <typename TPolicy>
  int64_t max_flow_exact(TPolicy& policy) {
    max_flow(policy);
    return last_flow_;
  }
  int64_t last_flow() const { return last_flow_; }
  template <typename TPolicy>
  TFlow max_flow(TPolicy& policy) {
    DummyTraceObject trace;
    return max_flow_with_tracing(policy, trace);
  }
  template <typename TTraceObject>
  TFlow max_flow_with_tracing(TTraceObject& trace) {
    GraphCutPolicy policy;
    return max_flow_with_tracing(policy, trace);
  }
  template <typename TPolicy, typename TTraceObject>
  TFlow max_flow_with_tracing(TPolicy& policy, TTraceObject& trace) {
    if (!grid_ && !generic_) throw Exception(CGC_ERR_STATE, "max_flow: set_nweights was not called");
    GraphCutData<TFlow> data;
    data.n_ = n_;
    data.mEdgeCount = edges_;
    data.grid_ = grid_.get();
    data.generic_ = generic_.get();
    trace.computationStarted(data);
    const GraphCutPolicy& p = policy;
    const int64_t f = grid_ ? grid_->max_flow(&p) : generic_->max_flow(&p);
    last_flow_ = f;
    data.stats_ = grid_ ? grid_->stats() : generic_->stats();
    // One iteration per exact global relabel, as in the reference's MinCut
    // loop (detail/graph_cut_implementation.hpp:150-175).  afterRelabel gets
    // the level starts of that relabel's BFS: the running count of tiles
    // visited per BFS round (the reference counts vertices per level); the
    // push phase that follows is reported by afterPush, with the flow at the
    // next relabel (the final flow after the last iteration).
    std::vector<std::vector<int>> levels;
    std::vector<int64_t> flow_at;  // flow_at[r]: flow at global relabel r + 1
    if (grid_) {
      std::vector<int> cur{0};
      for (const auto& r : grid_->trace()) {
        if (r.kind == 1) {
          cur.push_back(cur.back() + r.tiles);
        } else if (r.kind == 2) {
          levels.push_back(cur);
          cur.assign(1, 0);
        } else if (r.kind == 5) {
          flow_at.push_back(r.value);
        }
      }
    }
    const int64_t iters = data.stats_.global_relabels;
    for (int64_t i = 0; i < iters; ++i) {
      const bool last = i + 1 == iters;
      data.iteration_ = (int)i;
      data.final_ = last;
      data.flow_ = last ? f : (i + 1 < (int64_t)flow_at.size() ? flow_at[(size_t)i + 1] : -1);
      trace.beginIteration((int)i);
      trace.afterRelabel((int)i, i < (int64_t)levels.size() ? levels[(size_t)i] : std::vector<int>{0});
      trace.afterPush((int)i, last, data);
    }
    data.final_ = true;
    data.flow_ = f;
    const GraphCutData<TFlow>& done = data;
    trace.computationFinished(static_cast<TFlow>(f), done);
    return static_cast<TFlow>(f);
  }

  // out[i] = mask for vertices that can reach the sink (cugip's fill_segments,
  // graph_cut.hpp:304-333), background elsewhere.  out must be indexable by
  // vertex id.
  template <typename THostArrayView>
  void fill_segments(THostArrayView out, uint8_t mask = 255, uint8_t background = 0) const {
    fill(CGC_SEG_SINK_REACH, out, mask, background);
  }
  // The minimal source side of the minimum cut (the canonical cut).
  template <typename THostArrayView>
  void fill_source_segments(THostArrayView out, uint8_t mask = 255, uint8_t background = 0) const {
    fill(CGC_SEG_SOURCE_MIN, out, mask, background);
  }

  GridGraph* grid() const { return grid_.get(); }
  GenericGraph* generic() const { return generic_.get(); }

 private:
  void apply_tlinks() {
    if (grid_) grid_->set_tweights(tlink_s_.data(), tlink_t_.data());
    else generic_->set_tweights(tlink_s_.data(), tlink_t_.data());
  }

  template <typename THostArrayView>
  void fill(int which, THostArrayView& out, uint8_t mask, uint8_t background) const {
    if (!grid_ && !generic_) throw Exception(CGC_ERR_STATE, "fill_segments: no graph");
    std::vector<uint8_t> tmp(grid_ ? grid_->size() : generic_->size());
    if (grid_) grid_->segments(which, tmp.data(), mask, background);
    else generic_->segments(which, tmp.data(), mask, background);
    for (size_t i = 0; i < tmp.size(); ++i) out[i] = tmp[i];
  }

  template <typename T>
  struct Owned {
    T* p = nullptr;
    ~Owned() { delete p; }
    void reset(T* q = nullptr) { delete p; p = q; }
    T* get() const { return p; }
    T* operator->() const { return p; }
    explicit operator bool() const { return p != nullptr; }
  };

  int n_ = 0;
  int edges_ = 0;
  int64_t last_flow_ = 0;
  Owned<GridGraph> grid_;
  Owned<GenericGraph> generic_;
  std::vector<int32_t> tlink_s_, tlink_t_;  // host copy of the last t-links
};

}  // namespace cgc
