// velographx::io::save_binary / load_binary over the B200 device graph.
//
// Same names, signatures and file format as the reference's
// include/velographx/io/binary_graph.hpp:9-20; the rows are merged and the
// pairs filtered and bulk-loaded on the device (vx_graph_save_binary,
// vx_graph_load_binary in vx_b200.h).  Errors throw std::runtime_error with the
// reference's messages.
#pragma once

#include <string>

#include "../storage/dynamic_graph.hpp"

namespace velographx::io {

inline void save_binary(const DynamicGraph& g, const std::string& path) {
  detail::check(vx_graph_save_binary(g.handle(), path.c_str()));
}

inline DynamicGraph load_binary(const std::string& path, bool directed = false) {
  vx_graph* g = nullptr;
  detail::check(vx_graph_load_binary(path.c_str(), directed ? 1 : 0, &g));
  return DynamicGraph::adopt(g);
}

}  // namespace velographx::io
