// The reference's spelling of the graph-cut API.  Code written against
// cugip::Graph<TFlow> (include/cugip/advanced_operations/graph_cut.hpp:47-146)
// and trace objects whose hooks take cugip::GraphCutData<TFlow>
// (the protocol of graph_cut.hpp:26-45, e.g. the benchmark's TraceObject in
// benchmarks/graph_cut/graph_cut.cu:82-177) compile against this library by
// including this header in place of the reference's.
#pragma once

#include <cgc/graph_cut.hpp>

namespace cugip {

using cgc::DummyTraceObject;
using cgc::EdgeRecord;
using cgc::GraphCutPolicy;
template <typename TFlow>
using Graph = cgc::Graph<TFlow>;
template <typename TFlow>
using GraphCutData = cgc::GraphCutData<TFlow>;

}  // namespace cugip
