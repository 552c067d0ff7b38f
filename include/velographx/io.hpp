// velographx::load_edge_list over the B200 device graph: same name, signature
// and errors as the reference's include/velographx/io.hpp:6 (src/io.cpp:23-53);
// the text is parsed on the device (vx_graph_load_edge_list in vx_b200.h).
#pragma once

#include <filesystem>

#include "csr_graph.hpp"

namespace velographx {

inline CsrGraph load_edge_list(const std::filesystem::path& path, bool directed = false) {
  vx_graph* g = nullptr;
  detail::check(vx_graph_load_edge_list(path.string().c_str(), directed ? 1 : 0, &g));
  return CsrGraph(DynamicGraph::adopt(g));
}

}  // namespace velographx
