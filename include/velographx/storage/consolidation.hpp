// velographx consolidation policy and snapshot over the B200 device graph.
//
// Same names, signatures and decisions as the reference's
// include/velographx/storage/consolidation.hpp:11-163.  The policy, the
// signal and the hysteresis controller are host arithmetic on figures the
// caller supplies, restated from the reference; consolidate_to_csr_snapshot
// rebuilds the logical graph into a fresh device CSR (vx_graph_snapshot), and
// neighbor_scan_ns() measures on the device the neighbour-iteration cost the
// signal compares (no reference counterpart: the reference's callers time it
// themselves).
#pragma once

#include <cstddef>
#include <cstdint>
#include <utility>

#include "dynamic_graph.hpp"

namespace velographx {

struct ConsolidationSnapshot {
  DynamicGraph graph;
  std::size_t source_storage_bytes{0};
  std::size_t consolidated_storage_bytes{0};
  std::size_t directed_edges{0};
};

struct ConsolidationPolicy {
  double max_storage_growth_ratio{1.25};
  double max_neighbor_latency_ratio{1.25};
};

// :27-33 -- a wider storage envelope for graphs of 100M+ directed arcs
inline ConsolidationPolicy scale_aware_consolidation_policy(std::size_t directed_edges,
                                                            double latency_ratio = 1.25) noexcept {
  constexpr std::size_t kLargeGraphDirectedArcs = 100'000'000;
  return {directed_edges >= kLargeGraphDirectedArcs ? 1.50 : 1.25, latency_ratio};
}

struct ConsolidationSignal {
  double storage_growth_ratio{1.0};
  double neighbor_latency_ratio{1.0};
  bool storage_limit_exceeded{false};
  bool latency_limit_exceeded{false};
  bool should_consolidate{false};
};

// :43-63 -- ratios of the current layout to the canonical one; a ratio with a
// zero (or negative) canonical figure counts as 1
inline ConsolidationSignal evaluate_consolidation(std::size_t current_storage_bytes,
                                                  std::size_t canonical_storage_bytes,
                                                  double current_neighbor_latency,
                                                  double canonical_neighbor_latency,
                                                  ConsolidationPolicy policy = {}) noexcept {
  ConsolidationSignal s;
  s.storage_growth_ratio = canonical_storage_bytes == 0 ? 1.0
                                                        : static_cast<double>(current_storage_bytes) /
                                                              static_cast<double>(canonical_storage_bytes);
  s.neighbor_latency_ratio =
      canonical_neighbor_latency <= 0.0 ? 1.0 : current_neighbor_latency / canonical_neighbor_latency;
  s.storage_limit_exceeded = s.storage_growth_ratio >= policy.max_storage_growth_ratio;
  s.latency_limit_exceeded = s.neighbor_latency_ratio >= policy.max_neighbor_latency_ratio;
  s.should_consolidate = s.storage_limit_exceeded || s.latency_limit_exceeded;
  return s;
}

struct ConsolidationControllerConfig {
  std::size_t min_epochs_between_consolidations{10};
  std::size_t latency_breach_samples{5};
  double min_storage_growth_for_latency_trigger{1.10};
};

// :69-121 -- storage growth triggers at once; a latency trigger needs patch
// growth, a run of breaching samples, and the cooldown after the last
// consolidation (samples inside the cooldown do not count towards the run)
class ConsolidationController {
 public:
  explicit ConsolidationController(ConsolidationControllerConfig config = {}) : config_(config) {}

  bool observe(const ConsolidationSignal& signal, std::size_t epoch) noexcept {
    if (signal.storage_limit_exceeded) {
      streak_ = 0;
      return true;
    }
    const bool cooled = last_ == 0 || epoch >= last_ + config_.min_epochs_between_consolidations;
    if (!cooled) {
      streak_ = 0;
      return false;
    }
    const bool grown = signal.storage_growth_ratio >= config_.min_storage_growth_for_latency_trigger;
    const bool breach = signal.latency_limit_exceeded && grown;
    streak_ = breach ? streak_ + 1 : 0;
    return breach && streak_ >= config_.latency_breach_samples;
  }

  void mark_consolidated(std::size_t epoch) noexcept {
    last_ = epoch;
    streak_ = 0;
  }

  std::size_t latency_breach_streak() const noexcept { return streak_; }
  std::size_t last_consolidation_epoch() const noexcept { return last_; }

 private:
  ConsolidationControllerConfig config_{};
  std::size_t streak_{0};
  std::size_t last_{0};
};

// :132-163 -- the source is not modified
inline ConsolidationSnapshot consolidate_to_csr_snapshot(const DynamicGraph& source) {
  vx_graph* g = nullptr;
  detail::check(vx_graph_snapshot(source.handle(), &g));
  DynamicGraph consolidated = DynamicGraph::adopt(g);
  const std::size_t source_bytes = source.storage_bytes();
  const std::size_t consolidated_bytes = consolidated.storage_bytes();
  const std::size_t directed_edges = source.edge_count_directed();
  return {std::move(consolidated), source_bytes, consolidated_bytes, directed_edges};
}

// Device time of one pass over every live arc, per arc (ns): the neighbour
// latency evaluate_consolidation compares between a graph and its snapshot.
inline double neighbor_scan_ns(const DynamicGraph& g) {
  std::uint64_t arcs = 0;
  double ns = 0.0;
  detail::check(vx_graph_scan_rows(g.handle(), &arcs, &ns));
  return arcs ? ns / static_cast<double>(arcs) : 0.0;
}

}  // namespace velographx
