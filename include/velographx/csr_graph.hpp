// velographx::CsrGraph -- the static graph the reference's load_edge_list
// returns (include/velographx/csr_graph.hpp:9-40), here backed by a compact
// device graph (vx_graph).  Same member names and semantics: self-loops and
// duplicate edges dropped, vertex_count() = max id + 1 (0 without edges),
// neighbors()/in_neighbors() ascending and std::out_of_range beyond the vertex
// count, has_edge() false for ids outside the graph.  A span returned by
// neighbors() or in_neighbors() points into a host copy owned by this object
// and stays valid until the next call of the same member.
#pragma once

#include <cstddef>
#include <span>
#include <stdexcept>
#include <utility>
#include <vector>

#include "storage/dynamic_graph.hpp"
#include "types.hpp"

namespace velographx {

class CsrGraph {
 public:
  using Edge = std::pair<VertexId, VertexId>;

  explicit CsrGraph(DynamicGraph&& g) : g_(std::move(g)) {}

  [[nodiscard]] std::size_t vertex_count() const { return g_.vertex_count(); }
  [[nodiscard]] std::size_t edge_entry_count() const { return g_.edge_count_directed(); }
  [[nodiscard]] bool directed() const { return g_.directed(); }
  [[nodiscard]] std::span<const VertexId> neighbors(VertexId v) const {
    check_vertex(v);
    out_ = g_.neighbors(v);
    return out_;
  }
  [[nodiscard]] std::span<const VertexId> in_neighbors(VertexId v) const {
    check_vertex(v);
    in_ = g_.in_neighbors(v);
    return in_;
  }
  [[nodiscard]] std::size_t degree(VertexId v) const { return neighbors(v).size(); }
  [[nodiscard]] bool has_edge(VertexId u, VertexId v) const {
    const std::size_t n = vertex_count();
    if (u >= n || v >= n) return false;
    return g_.has_edge(u, v);
  }
  template <class Fn>
  void for_each_neighbor(VertexId v, Fn&& fn) const {
    for (const auto dst : neighbors(v)) fn(dst);
  }
  template <class Fn>
  void for_each_in_neighbor(VertexId v, Fn&& fn) const {
    for (const auto src : in_neighbors(v)) fn(src);
  }
  // The device graph behind it (no reference counterpart).
  [[nodiscard]] const DynamicGraph& graph() const noexcept { return g_; }

 private:
  void check_vertex(VertexId v) const {
    if (v >= vertex_count()) throw std::out_of_range("vertex id outside graph");
  }
  DynamicGraph g_;
  mutable std::vector<VertexId> out_, in_;
};

}  // namespace velographx
