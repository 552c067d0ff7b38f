// Multi-root BFS state (bit-parallel traversal of up to kMaxRoots roots).
#pragma once

#include <cstddef>
#include <cstdint>

#include "graph.cuh"

namespace vxh {

constexpr uint32_t kMaxRoots = 256;
constexpr uint32_t kMrTraceLevels = 64;  // levels with a trace entry (later ones share the last)

struct MrCounters {
  // Per-level counters rotate over three slots (level % 3); a level's slots
  // are cleared two levels ahead, so no block can clear a count that another
  // block has already started for the current level.
  uint32_t qn[3];    // frontier queue lengths
  uint32_t tn[3];    // touched heads of a push level
  uint32_t nbig[3];  // rows of a level long enough for the whole grid
  uint32_t gnext[3]; // next 32-vertex group of a pull level
  unsigned long long mf[3];  // out-arcs of the frontier's rows (the push cost of the level)
  uint32_t levels;
  uint32_t err;
  unsigned long long arcs;  // reached-arc total (mrbfs_reached_arcs)
  // per level: globaltimer at its start, then its frontier size with bit 63
  // set for a pull level; after the last level, the closing stamp
  unsigned long long trace[2 * kMrTraceLevels + 1];
};

struct MrBfs {
  Graph* g = nullptr;
  size_t K = 0, W = 0, V = 0;
  uint32_t* roots = nullptr;
  uint32_t* vis = nullptr;
  uint32_t* frn[3] = {nullptr, nullptr, nullptr};
  uint32_t* nxt = nullptr;
  uint32_t* touched = nullptr;
  uint32_t* q[3] = {nullptr, nullptr, nullptr};
  uint32_t* tl = nullptr;
  uint32_t* big = nullptr;     // rows of a level that the whole grid reads
  uint32_t* biglen = nullptr;  // their lengths
  uint32_t* dist = nullptr;  // [K][V]
  MrCounters* ctr = nullptr;
  MrCounters* hctr = nullptr;
  uint32_t* barrier = nullptr;
  float pull_frac = 0.02f;
  int grid = 0;
};

int mrbfs_create(MrBfs** out, Graph* g, const uint32_t* host_roots, size_t k);
void mrbfs_destroy(MrBfs* m);
int mrbfs_run(MrBfs* m);   // enqueues the traversal on the graph's stream
int mrbfs_sync(MrBfs* m);  // waits and checks the device error word
int mrbfs_reached_arcs(MrBfs* m, unsigned long long* out);
// The last run's level trace: {start ns, n_f | pull << 63} per level, then
// the closing stamp; writes up to cap values, *n = the full count.
int mrbfs_level_trace(MrBfs* m, unsigned long long* out, size_t cap, size_t* n);

}  // namespace vxh
