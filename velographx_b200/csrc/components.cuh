// Connected components of an undirected device graph maintained across
// update batches (include/velographx/incremental/connected_components.hpp of
// the reference).
#pragma once

#include <cstddef>
#include <cstdint>

#include "graph.cuh"

namespace vxh {

struct Components {
  Graph* g = nullptr;
  size_t n = 0;    // vertices covered by the labels (the reference's parent_.size())
  size_t cap = 0;
  uint32_t* label = nullptr;  // label[v] = smallest id of v's component
  uint32_t* aroot = nullptr;  // bitmap of affected roots (clear between batches)
  uint32_t* aff = nullptr;    // bitmap of affected vertices (clear between batches)
  uint32_t* ctr = nullptr;    // {effective deletion seen, -, affected count (u64)}
  size_t last_repaired = 0;
};

int cc_create(Components** out, Graph* g);
void cc_destroy(Components* c);
int cc_rebuild(Components* c);
// The batch already in g->batch (ops on the device): stage, mark, commit, repair.
int cc_apply_staged(Components* c, size_t n, size_t vertex_bound);
int cc_labels(Components* c, uint32_t* host_out, size_t cap, size_t* n);

}  // namespace vxh
