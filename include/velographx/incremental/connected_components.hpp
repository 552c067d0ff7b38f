// velographx::BasicIncrementalComponents<DynamicGraph> / IncrementalComponents
// backed by the B200 kernels (vx_cc_* in vx_b200.h).
//
// Same names and signatures as the reference's
// include/velographx/incremental/connected_components.hpp:16-170.  The
// partition after every batch equals the reference's; component(v) returns
// the smallest vertex id of v's component (the reference returns a
// union-find root that depends on its union order, and compares labels only
// for equality).  Labels stay in device memory; component() reads a host copy
// refreshed after every apply.
#pragma once

#include <cstddef>
#include <cstdint>
#include <stdexcept>
#include <vector>

#include "../storage/dynamic_graph.hpp"

namespace velographx {

template <class Graph>
class BasicIncrementalComponents;

template <>
class BasicIncrementalComponents<DynamicGraph> {
 public:
  // :19-25 -- std::invalid_argument for a directed graph
  explicit BasicIncrementalComponents(DynamicGraph& g) : g_(g) {
    detail::check(vx_cc_create(g.handle(), &c_));
  }
  ~BasicIncrementalComponents() { vx_cc_destroy(c_); }
  BasicIncrementalComponents(const BasicIncrementalComponents&) = delete;
  BasicIncrementalComponents& operator=(const BasicIncrementalComponents&) = delete;

  // :27-30 -- std::out_of_range beyond the vertices the labels cover
  [[nodiscard]] std::uint32_t component(VertexId v) {
    const auto& l = labels();
    if (v >= l.size()) throw std::out_of_range("vertex id outside graph");
    return l[v];
  }
  // :31-33
  [[nodiscard]] std::size_t last_repaired_vertices() const {
    std::uint64_t n = 0;
    detail::check(vx_cc_last_repaired_vertices(c_, &n));
    return static_cast<std::size_t>(n);
  }
  // :35-91
  void apply(const UpdateBatch& batch) {
    detail::BatchArrays a(batch);
    stale_ = true;
    detail::check(vx_cc_apply(c_, a.src.data(), a.dst.data(), a.add.data(), a.src.size()));
  }

  // Every vertex's label (no reference counterpart).
  [[nodiscard]] const std::vector<std::uint32_t>& labels() const {
    if (stale_) {
      std::size_t n = 0;
      detail::check(vx_cc_labels(c_, nullptr, 0, &n));
      host_.resize(n);
      if (n) detail::check(vx_cc_labels(c_, host_.data(), n, &n));
      stale_ = false;
    }
    return host_;
  }
  [[nodiscard]] vx_cc* handle() const noexcept { return c_; }
  // Marks the host copy of the labels stale after a call made directly
  // through the C ABI on handle().
  void mark_stale() const noexcept { stale_ = true; }

 private:
  DynamicGraph& g_;
  vx_cc* c_ = nullptr;
  mutable std::vector<std::uint32_t> host_;
  mutable bool stale_ = true;
};

using IncrementalComponents = BasicIncrementalComponents<DynamicGraph>;

}  // namespace velographx
