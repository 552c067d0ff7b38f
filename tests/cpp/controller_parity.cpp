// Drives the consolidation policy, signal and controller
// (velographx/storage/consolidation.hpp) through a seeded sequence of
// storage/latency figures and epochs and prints every decision.  The test
// compiles it once against this repository's headers and once against the
// reference's, and compares the two outputs line by line.
#include <cstdint>
#include <cstdio>

#include "velographx/storage/consolidation.hpp"

namespace {
uint64_t state = 0x2545F4914F6CDD1Dull;
uint64_t next() {
  state ^= state << 13;
  state ^= state >> 7;
  state ^= state << 17;
  return state;
}
double unit() { return (double)(next() >> 11) / 9007199254740992.0; }
}  // namespace

int main() {
  using namespace velographx;
  for (int run = 0; run < 20; ++run) {
    ConsolidationControllerConfig cfg;
    cfg.min_epochs_between_consolidations = 1 + next() % 12;
    cfg.latency_breach_samples = 1 + next() % 6;
    cfg.min_storage_growth_for_latency_trigger = 1.0 + 0.3 * unit();
    ConsolidationController ctl(cfg);
    const auto pol = scale_aware_consolidation_policy((size_t)(next() % 200'000'000), 1.0 + 0.5 * unit());
    std::printf("run %d policy %.6f %.6f\n", run, pol.max_storage_growth_ratio, pol.max_neighbor_latency_ratio);
    size_t epoch = 0;
    for (int t = 0; t < 400; ++t) {
      epoch += 1 + next() % 3;
      const size_t canon = (size_t)(next() % 4 == 0 ? 0 : 1000 + next() % 100000);
      const size_t cur = canon + (size_t)(next() % 60000);
      const double cl = next() % 7 == 0 ? 0.0 : 1.0 + 5.0 * unit();
      const double ll = cl * (0.8 + 0.9 * unit());
      const auto sig = evaluate_consolidation(cur, canon, ll, cl, pol);
      const bool go = ctl.observe(sig, epoch);
      std::printf("%zu %.9f %.9f %d %d %d -> %d streak %zu last %zu\n", epoch, sig.storage_growth_ratio,
                  sig.neighbor_latency_ratio, (int)sig.storage_limit_exceeded, (int)sig.latency_limit_exceeded,
                  (int)sig.should_consolidate, (int)go, ctl.latency_breach_streak(), ctl.last_consolidation_epoch());
      if (go && next() % 4 != 0) ctl.mark_consolidated(epoch);
    }
  }
  return 0;
}
