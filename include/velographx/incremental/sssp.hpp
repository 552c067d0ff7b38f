// velographx::BasicIncrementalSSSP<DynamicGraph> / IncrementalSSSP (unit
// weights) backed by the B200 BFS kernels (vx_bfs_* in vx_b200.h).
//
// Same names and signatures as the reference's
// include/velographx/incremental/sssp.hpp:14-69: 64-bit distances with the
// unreachable value UINT64_MAX / 4 (incremental/dijkstra.hpp:14).  The
// reference relaxes from the added edges of an insert-only batch and
// recomputes after any batch holding a removal; here an insert-only batch is
// the same relaxation on the device, and a batch with removals is the
// device's exact incremental repair (the distances a recompute gives), with a
// recompute when the source entered the graph after construction (the case in
// which the reference's recompute and the repair differ).
#pragma once

#include <cstddef>
#include <cstdint>
#include <limits>
#include <vector>

#include "../storage/dynamic_graph.hpp"

namespace velographx {

template <class Graph>
class BasicIncrementalSSSP;

template <>
class BasicIncrementalSSSP<DynamicGraph> {
 public:
  static constexpr std::uint64_t unreachable = std::numeric_limits<std::uint64_t>::max() / 4;

  // :17 -- a fraction above 1 keeps the repair from falling back: the result
  // is the same either way
  BasicIncrementalSSSP(DynamicGraph& g, VertexId source) : g_(g), source_(source) {
    detail::check(vx_bfs_create(g.handle(), source, 2.0, &b_));
  }
  ~BasicIncrementalSSSP() { vx_bfs_destroy(b_); }
  BasicIncrementalSSSP(const BasicIncrementalSSSP&) = delete;
  BasicIncrementalSSSP& operator=(const BasicIncrementalSSSP&) = delete;

  // :19
  [[nodiscard]] const std::vector<std::uint64_t>& distances() const {
    if (stale_) {
      std::size_t n = 0;
      detail::check(vx_bfs_distances(b_, nullptr, 0, &n));
      std::vector<std::uint32_t> d(n);
      if (n) detail::check(vx_bfs_distances(b_, d.data(), n, &n));
      host_.resize(n);
      for (std::size_t i = 0; i < n; ++i) host_[i] = d[i] == 0xFFFFFFFFu ? unreachable : d[i];
      stale_ = false;
    }
    return host_;
  }
  // :21-27
  void apply(const UpdateBatch& batch) {
    bool removal = false;
    for (const auto& e : batch.updates) removal |= !e.add;
    detail::BatchArrays a(batch);
    stale_ = true;
    detail::check(vx_bfs_apply(b_, a.src.data(), a.dst.data(), a.add.data(), a.src.size()));
    if (removal && source_ < g_.vertex_count()) {
      const auto& d = distances();
      if (source_ < d.size() && d[source_] != 0) recompute();
    }
  }
  // :29-35
  void recompute() {
    stale_ = true;
    detail::check(vx_bfs_recompute(b_));
  }
  [[nodiscard]] vx_bfs* handle() const noexcept { return b_; }

 private:
  DynamicGraph& g_;
  VertexId source_;
  vx_bfs* b_ = nullptr;
  mutable std::vector<std::uint64_t> host_;
  mutable bool stale_ = true;
};

using IncrementalSSSP = BasicIncrementalSSSP<DynamicGraph>;

}  // namespace velographx
