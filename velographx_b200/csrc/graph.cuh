// Device-resident dynamic graph (the B200 counterpart of
// velographx::DynamicGraph, include/velographx/storage/dynamic_graph.hpp:479-816).
#pragma once

#include <cstddef>
#include <cstdint>
#include <cuda_runtime.h>

#include "prims.cuh"
#include "vx_common.cuh"

namespace vxh {

// Device counters of one graph; lives in device memory, mirrored to pinned
// host memory on demand.
struct GraphCounters {
  unsigned long long arena_top[2];   // per direction (0 = out, 1 = in)
  unsigned long long delta_live[2];  // delta entries (overlay "present")
  unsigned long long tombs[2];       // tombstoned base arcs (overlay "absent")
  unsigned long long dirty_rows[2];  // rows touched since last compaction
  uint32_t final_arcs;               // F: canonical arcs of the current batch
  uint32_t rm_arcs, ins_arcs;        // delta removals / insertions of the batch
  uint32_t rm_runs, ins_runs;        // row runs among them
  uint32_t err;                      // vxb::kErr* bits
  uint32_t max_vertex_plus1;         // max(src,dst)+1 over non-self-loop ops
  uint32_t rev_arcs;                 // reversed changed arcs (directed graphs)
  uint32_t scratch32;                // single-value readbacks (has_edge, maybe_compact)
};

struct Adjacency {
  uint64_t* off = nullptr;
  uint32_t* col = nullptr;
  size_t off_cap = 0, col_cap = 0;
  uint32_t Vb = 0;
  uint64_t A = 0;  // arcs stored in the base CSR, tombstones included
  uint2* drow = nullptr;
  uint32_t* dcap = nullptr;
  uint32_t* tcnt = nullptr;    // tombstones per row
  uint32_t* dirty = nullptr;   // dirty-row bitmap
  uint32_t* darena = nullptr;
  size_t arena_cap = 0;
  uint64_t arena_bound = 0;    // host-side upper bound of arena_top
  void free_all();
};

// Canonical arcs of one batch, sorted by (u, v), last op per arc kept.
// flags: bit0 desired state (add), bit1 arc is in the base CSR, bit2 arc was
// present before the batch, bit3 state changes.
enum : uint8_t { kFAdd = 1, kFInBase = 2, kFCur = 4, kFChanged = 8 };

struct BatchBuffers {
  size_t cap = 0;       // op capacity
  uint32_t* src = nullptr;
  uint32_t* dst = nullptr;
  uint8_t* add = nullptr;
  // the op arrays the next staging reads: src/dst/add after a host upload, or
  // the caller's own device arrays (read in place)
  const uint32_t* in_src = nullptr;
  const uint32_t* in_dst = nullptr;
  const uint8_t* in_add = nullptr;
  uint64_t* keys = nullptr;
  uint64_t* keys_alt = nullptr;
  uint32_t* vals = nullptr;
  uint32_t* vals_alt = nullptr;
  uint32_t* flag = nullptr;   // generic flag / position scratch
  uint32_t* pos = nullptr;
  // canonical arcs (out direction)
  uint32_t* fu = nullptr;
  uint32_t* fv = nullptr;
  uint8_t* ff = nullptr;
  uint64_t* fpos = nullptr;
  // delta work lists
  uint32_t* lu = nullptr;
  uint32_t* lv = nullptr;
  uint32_t* runs = nullptr;
  // reversed canonical arcs (in direction, directed graphs)
  uint32_t* ru = nullptr;
  uint32_t* rv = nullptr;
  uint8_t* rf = nullptr;
  uint64_t* rpos = nullptr;
  int ensure(size_t ops);
  void free_all();
};

struct Graph {
  bool directed = false;
  size_t V = 0, Vcap = 0;
  uint64_t version = 0;
  Adjacency adj[2];  // [0] out, [1] in (unused when undirected)
  GraphCounters* ctr = nullptr;    // device
  GraphCounters* hctr = nullptr;   // pinned host mirror
  cudaStream_t stream = nullptr;
  Scratch scratch;
  BatchBuffers batch;
  uint64_t* pinned_scalar = nullptr;  // small pinned buffer for readbacks
  size_t batch_ops = 0;               // ops of the batch currently staged
  size_t arena_limit_entries = 0;     // consolidate instead of growing past this

  Adjacency& in() { return directed ? adj[1] : adj[0]; }
  vxb::DevGraph view();
};

int graph_create(Graph** out, size_t vertices, bool directed);
void graph_destroy(Graph* g);
int graph_grow(Graph* g, size_t vertices);
int graph_bulk_load(Graph* g, const uint32_t* d_uv, size_t n_edges);
// Stage a batch already in g->batch.{src,dst,add}: canonicalise + classify on
// the pre-batch graph.  vertex_bound bounds every non-self-loop id + 1.
// classify = false leaves the arcs unclassified (a fused repair classifies them itself).
int graph_stage_batch(Graph* g, size_t n, size_t vertex_bound, bool classify = true);
// The part of staging that precedes canonicalisation: arena room for a batch
// of n ops (consolidating first when the arena would pass its limit) and the
// vertex growth.  A caller that canonicalises and classifies the batch
// itself fills batch.{fu,fv,ff,fpos} and ctr->final_arcs, then commits.
int graph_prepare_batch(Graph* g, size_t n, size_t vertex_bound);
// Apply the staged batch to the device structure (after any pre-batch reads):
// removals first (tombstones, delta removals), then insertions.
int graph_commit_batch(Graph* g);
int graph_commit_removals(Graph* g);
int graph_commit_insertions(Graph* g);
int graph_consolidate(Graph* g);
int graph_reserve_stream(Graph* g, uint64_t entries, int* fits);
// One-launch canonicalisation of the staged batch in a thread-block cluster
// (sort, last-op-wins dedupe, compaction, classification); *done = false when
// the batch exceeds one cluster's capacity.
int canon_cluster(Graph* g, size_t n, int b, uint32_t bound, bool* done);
size_t canon_cluster_capacity();
// maybe_compact(threshold) (dynamic_graph.hpp:620-631, 764-789): consolidates when
// any dirty row's overlay density reaches the threshold; *compacted = 1 then.
int graph_maybe_compact(Graph* g, double threshold, int* compacted);
int graph_sync_counters(Graph* g);  // copies counters to g->hctr (synchronises)
int graph_row(Graph* g, int dir, uint32_t u, uint32_t* host_out, size_t cap, size_t* n);
int graph_has_edge(Graph* g, uint32_t u, uint32_t v, int* out);
// The compact row of u (compact_neighbors / compact_in_neighbors,
// dynamic_graph.hpp:573-581): the base CSR row as of the last consolidation,
// arcs deleted since then included; *n = its length.
int graph_compact_row(Graph* g, int dir, uint32_t u, uint32_t* host_out, size_t cap, size_t* n);
// Device bytes held by the graph's storage (storage_bytes, dynamic_graph.hpp:599-605).
size_t graph_storage_bytes(const Graph* g);
uint64_t graph_edge_count_directed(const Graph* g);  // needs synced counters

}  // namespace vxh
