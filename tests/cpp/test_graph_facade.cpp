// Reference-style C++ use of the cgc facade: the 4x4 graph of the reference's
// test/graph_cut.cu:13-67 through cgc::Graph<float> (the reference's float
// API), the same through Graph<int>, the layered graphs of the reference's
// unit_tests/graph_cut_test.cu:22-65,172-198 (known flows 1024*8 and
// 2*1024*8; not a grid, so the generic engine solves them) and a grid through
// cgc::GridGraph.
#include <cstdio>
#include <cstdlib>
#include <string>
#include <vector>

#include <cgc/cugip.hpp>
#include <cgc/graph_cut.hpp>
#include <cgc_volume.h>

#define EXPECT(c)                                                       \
  do {                                                                  \
    if (!(c)) { std::printf("FAILED %s:%d %s\n", __FILE__, __LINE__, #c); std::exit(1); } \
  } while (0)

struct CountingTrace : cgc::DummyTraceObject {
  int iterations = 0, relabels = 0, pushes = 0, last_levels = 0;
  bool done_seen = false, levels_ok = true;
  long long finished = -1;
  void beginIteration(int) { ++iterations; }
  void afterRelabel(int, const std::vector<int>& starts) {
    ++relabels;
    for (size_t i = 1; i < starts.size(); ++i) levels_ok = levels_ok && starts[i] >= starts[i - 1];
    last_levels = (int)starts.size();
  }
  template <typename T>
  void afterPush(int, bool done, const cgc::GraphCutData<T>&) { ++pushes; done_seen = done_seen || done; }
  template <typename T>
  void computationFinished(T flow, const cgc::GraphCutData<T>&) { finished = (long long)flow; }
};

// A trace object with the hook signatures of the reference benchmark's
// TraceObject (benchmarks/graph_cut/graph_cut.cu:82-177): non-const
// GraphCutData<float>& in computationStarted / afterPush, a const one in
// computationFinished, which checks the reference's invariant (excess only at
// vertices whose label is invalid, graph_cut.cu:171).
struct ReferenceShapedTrace {
  int vertices = 0, edges = 0, iterations = 0;
  size_t level_entries = 0;
  std::vector<long long> flows;
  bool done = false, invariant = false;
  float final_flow = -1.f;
  void computationStarted(cugip::GraphCutData<float>& aData) {
    vertices = aData.vertexCount();
    edges = aData.mEdgeCount;
  }
  void beginIteration(int) { ++iterations; }
  void afterRelabel(int, const std::vector<int>& aLevelStarts) { level_entries += aLevelStarts.size(); }
  void afterPush(int, bool aDone, cugip::GraphCutData<float>& aGraph) {
    flows.push_back((long long)aGraph.flow());
    done = aDone;
  }
  void computationFinished(float aFlow, const cugip::GraphCutData<float>& aData) {
    final_flow = aFlow;
    const std::vector<float>& excess = aData.vertexExcess();
    const std::vector<int>& labels = aData.labels();
    invariant = (int)excess.size() == aData.vertexCount() && labels.size() == excess.size();
    for (size_t i = 0; i < excess.size() && invariant; ++i)
      invariant = excess[i] <= 0.0f || labels[i] == cugip::GraphCutData<float>::INVALID_LABEL;
  }
};

// The 512x512x128 tube workload (flow 22 895 482, above float's 2^24) given
// to cugip::Graph<float> as an edge list, as the reference's front-end builds
// it: the exact flow through max_flow_exact and the trace protocol.
void full_size_tubes() {
  cgc_volume_spec spec;
  EXPECT(cgc_volume_preset(3, 0, &spec) == CGC_OK);
  const int64_t X = spec.X, Y = spec.Y, Z = spec.Z, N = X * Y * Z;
  std::vector<int32_t> cs(N), ct(N), nx(N), ny(N), nz(N);
  EXPECT(cgc_volume_generate(&spec, cs.data(), ct.data(), nx.data(), ny.data(), nz.data(), nullptr) == CGC_OK);
  std::vector<cugip::EdgeRecord> edges;
  std::vector<float> w;
  edges.reserve(3 * N);
  w.reserve(3 * N);
  for (int64_t z = 0; z < Z; ++z)
    for (int64_t y = 0; y < Y; ++y)
      for (int64_t x = 0; x < X; ++x) {
        const int64_t v = x + X * (y + Y * z);
        if (x + 1 < X) { edges.emplace_back((unsigned)v, (unsigned)(v + 1)); w.push_back((float)nx[v]); }
        if (y + 1 < Y) { edges.emplace_back((unsigned)v, (unsigned)(v + X)); w.push_back((float)ny[v]); }
        if (z + 1 < Z) { edges.emplace_back((unsigned)v, (unsigned)(v + X * Y)); w.push_back((float)nz[v]); }
      }
  std::vector<float> s(cs.begin(), cs.end()), t(ct.begin(), ct.end());
  cugip::Graph<float> graph;
  graph.set_vertex_count((int)N);
  graph.set_nweights((int)edges.size(), edges.data(), w.data(), w.data());
  graph.set_tweights(s.data(), t.data());
  EXPECT(graph.grid() != nullptr);
  ReferenceShapedTrace trace;
  const float f = graph.max_flow_with_tracing(trace);
  EXPECT(graph.last_flow() == 22895482LL);
  EXPECT((double)f == (double)(float)22895482LL);
  EXPECT(trace.vertices == (int)N && trace.edges == (int)edges.size());
  EXPECT(trace.iterations >= 1 && (int)trace.flows.size() == trace.iterations && trace.done);
  for (size_t i = 1; i < trace.flows.size(); ++i) EXPECT(trace.flows[i] >= trace.flows[i - 1]);
  EXPECT(trace.flows.back() == 22895482LL);
  EXPECT(trace.invariant && trace.level_entries >= (size_t)trace.iterations);
  // a second solve with new weights through the exact accessor
  graph.set_tweights(s.data(), t.data());
  graph.set_nweights((int)edges.size(), edges.data(), w.data(), w.data());
  EXPECT(graph.max_flow_exact() == 22895482LL);
  std::printf("full size ok\n");
}

template <typename W>
void four_by_four() {
  cgc::Graph<W> graph;
  graph.set_vertex_count(16);
  int v1[24] = {0, 1, 2, 4, 5, 6, 8, 9, 10, 12, 13, 14, 0, 1, 2, 3, 4, 5, 6, 7, 8, 9, 10, 11};
  int v2[24] = {1, 2, 3, 5, 6, 7, 9, 10, 11, 13, 14, 15, 4, 5, 6, 7, 8, 9, 10, 11, 12, 13, 14, 15};
  cgc::EdgeRecord edges[24];
  for (int i = 0; i < 24; ++i) edges[i] = cgc::EdgeRecord(v1[i], v2[i]);
  W w[24] = {5, 5, 5, 5, 5, 5, 5, 5, 5, 5, 5, 5, 5, 5, 5, 5, 1, 1, 1, 1, 5, 5, 5, 5};
  W src[16] = {100, 100, 100, 100, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0};
  W snk[16] = {0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 100, 100, 100, 100};
  graph.set_nweights(24, edges, w, w);
  graph.set_tweights(src, snk);
  CountingTrace trace;
  W flow = graph.max_flow_with_tracing(trace);
  EXPECT(flow == (W)4);
  EXPECT(trace.finished == 4 && trace.iterations >= 1);
  EXPECT(trace.relabels == trace.iterations && trace.pushes == trace.iterations && trace.done_seen);
  EXPECT(trace.levels_ok && trace.last_levels >= 1);
  std::vector<unsigned char> seg(16);
  graph.fill_segments(seg.data());
  for (int i = 0; i < 16; ++i) EXPECT(seg[i] == (i < 8 ? 0 : 255));
  graph.fill_source_segments(seg.data(), 1, 0);
  for (int i = 0; i < 16; ++i) EXPECT(seg[i] == (i < 8 ? 1 : 0));
  // solving again after re-setting the weights gives the same answer
  graph.set_tweights(src, snk);
  graph.set_nweights(24, edges, w, w);
  EXPECT(graph.max_flow() == (W)4);
}

// layers of `size` vertices; vertex i of a layer joins vertices i..i+nbrs-1
// (mod size) of the next layer with weight 20 forward, 40 backward, except a
// 1 / 2 bottleneck at the middle layer; terminals on the first and last layer
template <typename W>
void layered(bool flip, long long expected) {
  const int layers = 100, size = 1024, nbrs = 8;
  cgc::Graph<W> graph;
  graph.set_vertex_count(layers * size);
  std::vector<cgc::EdgeRecord> edges;
  std::vector<W> fw, bw;
  for (int layer = 1; layer < layers; ++layer) {
    const W weight = layer == layers / 2 ? (W)1 : (W)20;
    for (int i = 0; i < size; ++i)
      for (int j = 0; j < nbrs; ++j) {
        edges.emplace_back((layer - 1) * size + i, layer * size + (i + j) % size);
        fw.push_back(weight);
        bw.push_back(2 * weight);
      }
  }
  std::vector<W> first(layers * size, (W)0), last(layers * size, (W)0);
  for (int i = 0; i < size; ++i) {
    first[i] = (W)100000;
    last[(layers - 1) * size + i] = (W)100000;
  }
  graph.set_nweights((int)edges.size(), edges.data(), fw.data(), bw.data());
  if (flip) graph.set_tweights(last.data(), first.data());
  else graph.set_tweights(first.data(), last.data());
  EXPECT(graph.generic() != nullptr && graph.grid() == nullptr);
  EXPECT((long long)graph.max_flow() == expected);
  std::vector<unsigned char> seg(layers * size);
  graph.fill_segments(seg.data());
  // the bottleneck layer separates the sides
  const int sink_first = flip ? 0 : (layers / 2) * size;
  EXPECT(seg[sink_first] == 255 && seg[flip ? (layers - 1) * size : 0] == 0);
}

int main(int argc, char** argv) {
  if (argc > 1 && std::string(argv[1]) == "--full-size") {
    full_size_tubes();
    return 0;
  }
  four_by_four<float>();
  four_by_four<int>();
  layered<float>(false, 1024 * 8);
  layered<float>(true, 2 * 1024 * 8);
  layered<int>(false, 1024 * 8);
  // non-integral weights are rejected
  bool threw = false;
  try {
    cgc::Graph<float> g;
    g.set_vertex_count(2);
    float s[2] = {0.5f, 0.f}, t[2] = {0.f, 1.f};
    g.set_tweights(s, t);
  } catch (const cgc::Exception& e) {
    threw = e.code() == CGC_ERR_ARG;
  }
  EXPECT(threw);
  // grid facade: a chain along x with a bottleneck
  cgc::GridGraph g(16, 1, 1);
  std::vector<int32_t> cs(16, 0), ct(16, 0), nx(16, 9), z(16, 0);
  cs[0] = 50; ct[15] = 50; nx[7] = 3; nx[15] = 0;
  g.set_tweights(cs.data(), ct.data());
  g.set_nweights(CGC_AXIS_X, nx.data(), nx.data());
  EXPECT(g.max_flow() == 3);
  // every kernel shape a policy selects gives the same flow on a 48^3 grid
  // with pseudo-random weights
  {
    const int X = 48, Y = 48, Z = 48, N = X * Y * Z;
    std::vector<int32_t> s(N), t(N), ax[3];
    unsigned v = 12345u;
    auto rnd = [&v](int m) { v = v * 1664525u + 1013904223u; return (int32_t)((v >> 8) % (unsigned)m); };
    for (int i = 0; i < N; ++i) { s[i] = rnd(100) < 30 ? rnd(40) : 0; t[i] = rnd(100) < 30 ? rnd(40) : 0; }
    for (auto& a : ax) { a.resize(N); for (auto& c : a) c = rnd(25); }
    cgc::GridGraph grid(X, Y, Z);
    auto solve = [&](const cgc::GraphCutPolicy* p) {
      grid.set_tweights(s.data(), t.data());
      for (int k = 0; k < 3; ++k) grid.set_nweights(k, ax[k].data(), ax[k].data());
      return grid.max_flow(p);
    };
    const int64_t f0 = solve(nullptr);
    EXPECT(f0 > 0);
    cgc::GraphCutPolicy pols[6];
    pols[0].ctas_per_sm = 3; pols[0].bfs_warp_min = 1;
    pols[1].ctas_per_sm = 4; pols[1].region_relabels = 4; pols[1].local_pulses = 2;
    pols[2].ctas_per_sm = 4; pols[2].bfs_warp_min = 8;
    pols[3].region_relabels = -1; pols[3].local_pulses = 8;
    pols[4].persistent = -1; pols[4].sweeps_per_relabel = 4;
    pols[5].stall_sweeps = 2; pols[5].ctas_per_sm = 3;
    for (const auto& p : pols) EXPECT(solve(&p) == f0);
    cgc::GraphCutPolicy tuned;
    EXPECT(!cgc::GraphCutPolicy::autotuned((int64_t)N * 7 + 1, 1, &tuned));
  }
  std::printf("cpp facade ok\n");
  return 0;
}
