// velographx::BasicIncrementalBFS<DynamicGraph> / IncrementalBFS backed by the
// B200 kernels (vx_b200.h).
//
// Same names and signatures as the reference's
// include/velographx/incremental/bfs.hpp:13-27, 383.  Distances stay in device
// memory; distances() copies them into a host vector when they changed since
// the last read.  Only the DynamicGraph instantiation exists: the device path
// is the product, there is no host traversal.
#pragma once

#include <cstddef>
#include <cstdint>
#include <limits>
#include <vector>

#include "../storage/dynamic_graph.hpp"

namespace velographx {

template <class Graph>
class BasicIncrementalBFS;

template <>
class BasicIncrementalBFS<DynamicGraph> {
 public:
  static constexpr std::uint32_t unreachable = std::numeric_limits<std::uint32_t>::max();

  BasicIncrementalBFS(DynamicGraph& g, VertexId source, double deletion_fallback_fraction = 0.35) : g_(g) {
    detail::check(vx_bfs_create(g.handle(), source, deletion_fallback_fraction, &b_));
  }
  ~BasicIncrementalBFS() { vx_bfs_destroy(b_); }
  BasicIncrementalBFS(const BasicIncrementalBFS&) = delete;
  BasicIncrementalBFS& operator=(const BasicIncrementalBFS&) = delete;

  [[nodiscard]] const std::vector<std::uint32_t>& distances() const {
    if (stale_) {
      std::size_t n = 0;
      detail::check(vx_bfs_distances(b_, nullptr, 0, &n));
      host_.resize(n);
      if (n) detail::check(vx_bfs_distances(b_, host_.data(), n, &n));
      stale_ = false;
    }
    return host_;
  }
  [[nodiscard]] std::size_t reachable_count() const { return stats().reachable_count; }
  [[nodiscard]] std::size_t last_deletion_candidates() const { return stats().last_deletion_candidates; }
  [[nodiscard]] std::size_t last_affected_vertices() const { return stats().last_affected_vertices; }
  [[nodiscard]] bool last_used_full_recompute() const { return stats().last_used_full_recompute != 0; }

  void apply(const UpdateBatch& batch) {
    detail::BatchArrays a(batch);
    stale_ = true;
    detail::check(vx_bfs_apply(b_, a.src.data(), a.dst.data(), a.add.data(), a.src.size()));
  }
  void recompute() {
    stale_ = true;
    detail::check(vx_bfs_recompute(b_));
  }

  [[nodiscard]] vx_bfs* handle() const noexcept { return b_; }
  // Marks the host copy of the distances stale after a call made directly
  // through the C ABI on handle().
  void mark_stale() const noexcept { stale_ = true; }
  [[nodiscard]] DynamicGraph& graph() const noexcept { return g_; }

 private:
  vx_bfs_stats_t stats() const {
    vx_bfs_stats_t s{};
    detail::check(vx_bfs_stats(b_, &s));
    return s;
  }

  DynamicGraph& g_;
  vx_bfs* b_ = nullptr;
  mutable std::vector<std::uint32_t> host_;
  mutable bool stale_ = true;
};

using IncrementalBFS = BasicIncrementalBFS<DynamicGraph>;

}  // namespace velographx
