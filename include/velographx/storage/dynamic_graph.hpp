// velographx::DynamicGraph backed by the B200 device graph (vx_b200.h).
//
// Same names and signatures as the reference's
// include/velographx/storage/dynamic_graph.hpp (EdgeUpdate / UpdateBatch
// :17-29, DynamicGraph :479-639) so callers recompile unchanged.  The logical
// graph lives in device memory; row queries copy one row back to the host.
#pragma once

#include <cstddef>
#include <cstdint>
#include <span>
#include <stdexcept>
#include <string>
#include <utility>
#include <vector>

#include "../../vx_b200.h"
#include "../types.hpp"

namespace velographx {

struct EdgeUpdate {
  VertexId src{};
  VertexId dst{};
  bool add{true};
  std::uint64_t timestamp{0};
};

struct UpdateBatch {
  std::vector<EdgeUpdate> updates;
  void add(VertexId u, VertexId v, std::uint64_t ts = 0) { updates.push_back({u, v, true, ts}); }
  void remove(VertexId u, VertexId v, std::uint64_t ts = 0) { updates.push_back({u, v, false, ts}); }
  [[nodiscard]] bool empty() const noexcept { return updates.empty(); }
};

namespace detail {

[[noreturn]] inline void throw_status(int rc) {
  char msg[1024];
  vx_last_error(msg, sizeof msg);
  if (rc == VX_ERR_INVALID) throw std::invalid_argument(msg);
  if (rc == VX_ERR_RANGE) throw std::out_of_range(msg);
  if (rc == VX_ERR_OVERFLOW) throw std::overflow_error(msg);
  if (rc == VX_ERR_FORMAT || rc == VX_ERR_IO) throw std::runtime_error(msg);
  throw std::runtime_error(std::string("vx_b200: ") + msg);
}

inline void check(int rc) {
  if (rc != VX_OK) throw_status(rc);
}

// Structure-of-arrays copy of a batch (the device upload layout).
struct BatchArrays {
  std::vector<std::uint32_t> src, dst;
  std::vector<std::uint8_t> add;
  explicit BatchArrays(const UpdateBatch& b) {
    const auto n = b.updates.size();
    src.resize(n);
    dst.resize(n);
    add.resize(n);
    for (std::size_t i = 0; i < n; ++i) {
      src[i] = b.updates[i].src;
      dst[i] = b.updates[i].dst;
      add[i] = b.updates[i].add ? 1 : 0;
    }
  }
};

}  // namespace detail

class DynamicGraph {
 public:
  explicit DynamicGraph(std::size_t vertices = 0, bool directed = false) {
    detail::check(vx_graph_create(vertices, directed ? 1 : 0, &g_));
  }
  // Takes ownership of a graph the C ABI created (the file loaders).  No
  // reference counterpart.
  static DynamicGraph adopt(vx_graph* g) { return DynamicGraph(g, 0); }
  ~DynamicGraph() { vx_graph_destroy(g_); }
  DynamicGraph(const DynamicGraph&) = delete;
  DynamicGraph& operator=(const DynamicGraph&) = delete;
  DynamicGraph(DynamicGraph&& o) noexcept : g_(o.g_) { o.g_ = nullptr; }
  DynamicGraph& operator=(DynamicGraph&& o) noexcept {
    if (this != &o) {
      vx_graph_destroy(g_);
      g_ = o.g_;
      o.g_ = nullptr;
    }
    return *this;
  }

  [[nodiscard]] std::size_t vertex_count() const {
    std::size_t n = 0;
    detail::check(vx_graph_vertex_count(g_, &n));
    return n;
  }
  [[nodiscard]] std::uint64_t version() const {
    std::uint64_t v = 0;
    detail::check(vx_graph_version(g_, &v));
    return v;
  }
  [[nodiscard]] bool directed() const {
    int d = 0;
    detail::check(vx_graph_directed(g_, &d));
    return d != 0;
  }

  // :493-500 -- grows the vertex count; the version is unchanged
  void ensure_vertex(VertexId v) { detail::check(vx_graph_ensure_vertex(g_, v)); }

  void bulk_load_edges(const std::vector<std::pair<VertexId, VertexId>>& edges) {
    std::vector<std::uint32_t> uv(edges.size() * 2);
    for (std::size_t i = 0; i < edges.size(); ++i) {
      uv[2 * i] = edges[i].first;
      uv[2 * i + 1] = edges[i].second;
    }
    detail::check(vx_graph_bulk_load(g_, uv.data(), edges.size()));
  }

  void add_edge(VertexId u, VertexId v) {
    UpdateBatch b;
    b.add(u, v);
    apply(b);
  }
  void remove_edge(VertexId u, VertexId v) {
    UpdateBatch b;
    b.remove(u, v);
    apply(b);
  }

  void apply(const UpdateBatch& batch) {
    if (batch.empty()) return;
    detail::BatchArrays a(batch);
    detail::check(vx_graph_apply(g_, a.src.data(), a.dst.data(), a.add.data(), a.src.size()));
  }

  [[nodiscard]] std::vector<VertexId> neighbors(VertexId u) const { return row(u, false); }
  [[nodiscard]] std::vector<VertexId> in_neighbors(VertexId v) const { return row(v, true); }

  template <class Fn>
  void for_each_neighbor(VertexId u, Fn&& fn) const {
    for (auto v : neighbors(u)) fn(v);
  }
  template <class Fn>
  void for_each_in_neighbor(VertexId v, Fn&& fn) const {
    for (auto u : in_neighbors(v)) fn(u);
  }

  // :573-581 -- the row as of the last consolidation.  The span points into a
  // host copy owned by this object, valid until the next compact_*neighbors
  // call in the same direction (the reference's points into its own storage,
  // valid until the next mutation).
  [[nodiscard]] std::span<const VertexId> compact_neighbors(VertexId u) const {
    compact_row(u, false, compact_out_buf_);
    return compact_out_buf_;
  }
  [[nodiscard]] std::span<const VertexId> compact_in_neighbors(VertexId v) const {
    compact_row(v, true, compact_in_buf_);
    return compact_in_buf_;
  }

  [[nodiscard]] bool has_edge(VertexId u, VertexId v) const {
    int r = 0;
    detail::check(vx_graph_has_edge(g_, u, v, &r));
    return r != 0;
  }
  [[nodiscard]] std::size_t edge_count_directed() const {
    std::size_t n = 0;
    detail::check(vx_graph_edge_count_directed(g_, &n));
    return n;
  }
  // :593-595
  [[nodiscard]] std::size_t base_edge_count_directed() const {
    std::size_t n = 0;
    detail::check(vx_graph_base_edge_count_directed(g_, &n));
    return n;
  }
  // :599-605 -- device bytes of the graph's storage
  [[nodiscard]] std::size_t storage_bytes() const {
    std::size_t n = 0;
    detail::check(vx_graph_storage_bytes(g_, &n));
    return n;
  }
  // :607-610
  [[nodiscard]] double delta_ratio() const {
    const std::size_t base = base_edge_count_directed();
    return static_cast<double>(delta_edge_count()) / static_cast<double>(base > 1 ? base : 1);
  }
  [[nodiscard]] std::size_t delta_edge_count() const {
    std::size_t n = 0;
    detail::check(vx_graph_delta_edge_count(g_, &n));
    return n;
  }
  [[nodiscard]] bool is_compact() const {
    int c = 0;
    detail::check(vx_graph_is_compact(g_, &c));
    return c != 0;
  }
  [[nodiscard]] std::size_t dirty_out_segment_count() const { return dirty().first; }
  [[nodiscard]] std::size_t dirty_in_segment_count() const { return dirty().second; }

  bool maybe_compact(double threshold = 0.25) {
    int c = 0;
    detail::check(vx_graph_maybe_compact(g_, threshold, &c));
    return c != 0;
  }
  void compact() { detail::check(vx_graph_compact(g_)); }

  [[nodiscard]] vx_graph* handle() const noexcept { return g_; }

 private:
  std::vector<VertexId> row(VertexId u, bool in) const {
    std::size_t n = 0;
    auto fn = in ? vx_graph_in_neighbors : vx_graph_neighbors;
    detail::check(fn(g_, u, nullptr, 0, &n));
    std::vector<VertexId> out(n);
    if (n) detail::check(fn(g_, u, out.data(), n, &n));
    return out;
  }
  void compact_row(VertexId u, bool in, std::vector<VertexId>& out) const {
    std::size_t n = 0;
    auto fn = in ? vx_graph_compact_in_neighbors : vx_graph_compact_neighbors;
    detail::check(fn(g_, u, nullptr, 0, &n));
    out.resize(n);
    if (n) detail::check(fn(g_, u, out.data(), n, &n));
  }
  std::pair<std::size_t, std::size_t> dirty() const {
    std::size_t o = 0, i = 0;
    detail::check(vx_graph_dirty_rows(g_, &o, &i));
    return {o, i};
  }

  DynamicGraph(vx_graph* g, int) : g_(g) {}

  vx_graph* g_ = nullptr;
  mutable std::vector<VertexId> compact_out_buf_, compact_in_buf_;
};

}  // namespace velographx
