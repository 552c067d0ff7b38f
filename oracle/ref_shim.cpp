// C-ABI shim over the UNMODIFIED VeloGraphX reference, compiled by
// oracle/Makefile against the reference's own headers and sources
// (include/velographx/storage/dynamic_graph.hpp,
//  include/velographx/incremental/bfs.hpp, src/csr_graph.cpp,
//  src/algorithms.cpp) into oracle/_ref/libvxref.so.
//
// TEST INFRASTRUCTURE ONLY: it pins the C restatement in vx_oracle.c, generates
// the golden fixtures under tests/golden/, and is the "reference" CPU baseline
// timed by bench.py.  Nothing in the product loads it.
//
// The function set mirrors vx_oracle.h with a vxr_ prefix, plus the binary
// graph format (include/velographx/io/binary_graph.hpp) and the maintained
// connected components and unit-weight SSSP on the same graph
// (include/velographx/incremental/connected_components.hpp, sssp.hpp).
#include <atomic>
#include <cstdint>
#include <cstring>
#include <stdexcept>
#include <string>
#include <thread>
#include <utility>
#include <vector>

#include "velographx/algorithms.hpp"
#include "velographx/csr_graph.hpp"
#include "velographx/incremental/bfs.hpp"
#include "velographx/incremental/connected_components.hpp"
#include "velographx/incremental/sssp.hpp"
#include "velographx/io/binary_graph.hpp"
#include "velographx/storage/dynamic_graph.hpp"

using velographx::DynamicGraph;
using velographx::IncrementalBFS;
using velographx::UpdateBatch;
using velographx::VertexId;

namespace {
UpdateBatch make_batch(const uint32_t* src, const uint32_t* dst, const uint8_t* add, size_t n) {
  UpdateBatch b;
  b.updates.reserve(n);
  for (size_t i = 0; i < n; ++i) {
    if (add[i]) b.add(src[i], dst[i]);
    else b.remove(src[i], dst[i]);
  }
  return b;
}
}  // namespace

extern "C" {

void* vxr_graph_create(size_t vertices, int directed) {
  return new DynamicGraph(vertices, directed != 0);
}
void vxr_graph_destroy(void* g) { delete static_cast<DynamicGraph*>(g); }
size_t vxr_graph_vertex_count(void* g) { return static_cast<DynamicGraph*>(g)->vertex_count(); }
uint64_t vxr_graph_version(void* g) { return static_cast<DynamicGraph*>(g)->version(); }

int vxr_graph_bulk_load(void* g, const uint32_t* uv, size_t n) {
  std::vector<std::pair<VertexId, VertexId>> edges(n);
  for (size_t i = 0; i < n; ++i) edges[i] = {uv[2 * i], uv[2 * i + 1]};
  static_cast<DynamicGraph*>(g)->bulk_load_edges(edges);
  return 0;
}

int vxr_graph_apply(void* g, const uint32_t* src, const uint32_t* dst, const uint8_t* add, size_t n) {
  static_cast<DynamicGraph*>(g)->apply(make_batch(src, dst, add, n));
  return 0;
}

size_t vxr_graph_neighbors(void* g, uint32_t u, uint32_t* out, size_t cap) {
  auto row = static_cast<DynamicGraph*>(g)->neighbors(u);
  std::memcpy(out, row.data(), std::min(cap, row.size()) * sizeof(uint32_t));
  return row.size();
}

size_t vxr_graph_in_neighbors(void* g, uint32_t v, uint32_t* out, size_t cap) {
  auto row = static_cast<DynamicGraph*>(g)->in_neighbors(v);
  std::memcpy(out, row.data(), std::min(cap, row.size()) * sizeof(uint32_t));
  return row.size();
}

int vxr_graph_has_edge(void* g, uint32_t u, uint32_t v) {
  return static_cast<DynamicGraph*>(g)->has_edge(u, v) ? 1 : 0;
}
size_t vxr_graph_edge_count_directed(void* g) {
  return static_cast<DynamicGraph*>(g)->edge_count_directed();
}
size_t vxr_graph_delta_edge_count(void* g) { return static_cast<DynamicGraph*>(g)->delta_edge_count(); }
int vxr_graph_is_compact(void* g) { return static_cast<DynamicGraph*>(g)->is_compact() ? 1 : 0; }
size_t vxr_graph_dirty_out_count(void* g) { return static_cast<DynamicGraph*>(g)->dirty_out_segment_count(); }
size_t vxr_graph_dirty_in_count(void* g) { return static_cast<DynamicGraph*>(g)->dirty_in_segment_count(); }
void vxr_graph_compact(void* g) { static_cast<DynamicGraph*>(g)->compact(); }
void vxr_graph_ensure_vertex(void* g, uint32_t v) { static_cast<DynamicGraph*>(g)->ensure_vertex(v); }
size_t vxr_graph_base_edge_count_directed(void* g) {
  return static_cast<DynamicGraph*>(g)->base_edge_count_directed();
}
size_t vxr_graph_compact_neighbors(void* g, uint32_t u, uint32_t* out, size_t cap) {
  auto* dg = static_cast<DynamicGraph*>(g);
  if (u >= dg->vertex_count()) return 0;
  auto row = dg->compact_neighbors(u);
  if (out) std::memcpy(out, row.data(), std::min(cap, row.size()) * sizeof(uint32_t));
  return row.size();
}
size_t vxr_graph_compact_in_neighbors(void* g, uint32_t v, uint32_t* out, size_t cap) {
  auto* dg = static_cast<DynamicGraph*>(g);
  if (v >= dg->vertex_count()) return 0;
  auto row = dg->compact_in_neighbors(v);
  if (out) std::memcpy(out, row.data(), std::min(cap, row.size()) * sizeof(uint32_t));
  return row.size();
}
int vxr_graph_maybe_compact(void* g, double t) {
  return static_cast<DynamicGraph*>(g)->maybe_compact(t) ? 1 : 0;
}

void* vxr_bfs_create(void* g, uint32_t source, double frac) {
  return new IncrementalBFS(*static_cast<DynamicGraph*>(g), source, frac);
}
void vxr_bfs_destroy(void* b) { delete static_cast<IncrementalBFS*>(b); }
void vxr_bfs_recompute(void* b) { static_cast<IncrementalBFS*>(b)->recompute(); }
int vxr_bfs_apply(void* b, const uint32_t* src, const uint32_t* dst, const uint8_t* add, size_t n) {
  static_cast<IncrementalBFS*>(b)->apply(make_batch(src, dst, add, n));
  return 0;
}
size_t vxr_bfs_distances(void* b, uint32_t* out, size_t cap) {
  const auto& d = static_cast<IncrementalBFS*>(b)->distances();
  if (out) std::memcpy(out, d.data(), std::min(cap, d.size()) * sizeof(uint32_t));
  return d.size();
}
size_t vxr_bfs_reachable_count(void* b) { return static_cast<IncrementalBFS*>(b)->reachable_count(); }
size_t vxr_bfs_last_deletion_candidates(void* b) {
  return static_cast<IncrementalBFS*>(b)->last_deletion_candidates();
}
size_t vxr_bfs_last_affected_vertices(void* b) {
  return static_cast<IncrementalBFS*>(b)->last_affected_vertices();
}
int vxr_bfs_last_used_full_recompute(void* b) {
  return static_cast<IncrementalBFS*>(b)->last_used_full_recompute() ? 1 : 0;
}

// Static CSR (src/csr_graph.cpp) for the multicore thread-per-root BFS that
// benchmarks/thread_scaling_bfs.cpp:78-108 times: T threads pull roots from an
// atomic counter and run bfs_distances (src/algorithms.cpp:11-27) per root.
void* vxr_csr_create(const uint32_t* uv, size_t n, int directed) {
  std::vector<velographx::CsrGraph::Edge> edges(n);
  for (size_t i = 0; i < n; ++i) edges[i] = {uv[2 * i], uv[2 * i + 1]};
  return new velographx::CsrGraph(std::move(edges), directed != 0);
}
void vxr_csr_destroy(void* c) { delete static_cast<velographx::CsrGraph*>(c); }
size_t vxr_csr_vertex_count(void* c) { return static_cast<velographx::CsrGraph*>(c)->vertex_count(); }

// Runs bfs_distances for every root on `threads` threads; writes per-root
// reached-arc sums (sum of out-degrees of reached vertices) into arcs_out and,
// if dist_out is non-null, root r's distances into dist_out + r*V.
int vxr_csr_multi_bfs(void* c, const uint32_t* roots, size_t k, int threads,
                      uint64_t* arcs_out, uint32_t* dist_out) {
  auto* g = static_cast<velographx::CsrGraph*>(c);
  const size_t V = g->vertex_count();
  std::atomic<size_t> next{0};
  std::atomic<int> failed{0};
  auto worker = [&]() {
    for (;;) {
      const size_t r = next.fetch_add(1);
      if (r >= k) break;
      try {
        auto d = velographx::bfs_distances(*g, roots[r]);
        uint64_t arcs = 0;
        for (size_t v = 0; v < V; ++v)
          if (d[v] != velographx::kUnreachable) arcs += g->degree(static_cast<VertexId>(v));
        if (arcs_out) arcs_out[r] = arcs;
        if (dist_out) std::memcpy(dist_out + r * V, d.data(), V * sizeof(uint32_t));
      } catch (...) {
        failed.store(1);
      }
    }
  };
  std::vector<std::thread> pool;
  for (int t = 0; t < (threads > 0 ? threads : 1); ++t) pool.emplace_back(worker);
  for (auto& t : pool) t.join();
  return failed.load() ? -1 : 0;
}


// ---- binary graph format ----------------------------------------------------
// Errors: the exception's message in err (cap bytes), return -1 / null.
static void put_error(const std::exception& e, char* err, size_t cap) {
  if (err && cap) {
    std::strncpy(err, e.what(), cap - 1);
    err[cap - 1] = 0;
  }
}

int vxr_save_binary(void* g, const char* path, char* err, size_t cap) {
  try {
    velographx::io::save_binary(*static_cast<DynamicGraph*>(g), path);
    return 0;
  } catch (const std::exception& e) {
    put_error(e, err, cap);
  }
  return -1;
}

void* vxr_load_binary(const char* path, int directed, char* err, size_t cap) {
  try {
    return new DynamicGraph(velographx::io::load_binary(path, directed != 0));
  } catch (const std::exception& e) {
    put_error(e, err, cap);
  }
  return nullptr;
}


// ---- IncrementalComponents / IncrementalSSSP ---------------------------------
void* vxr_cc_create(void* g) {
  try {
    return new velographx::IncrementalComponents(*static_cast<DynamicGraph*>(g));
  } catch (const std::exception&) {
    return nullptr;
  }
}
void vxr_cc_destroy(void* c) { delete static_cast<velographx::IncrementalComponents*>(c); }
int vxr_cc_apply(void* c, const uint32_t* src, const uint32_t* dst, const uint8_t* add, size_t n) {
  static_cast<velographx::IncrementalComponents*>(c)->apply(make_batch(src, dst, add, n));
  return 0;
}
// labels of v in [0, n): writes component(v), or UINT32_MAX where component()
// throws out_of_range; returns the first v that throws (the labels' size)
size_t vxr_cc_labels(void* c, uint32_t* out, size_t n) {
  auto* cc = static_cast<velographx::IncrementalComponents*>(c);
  size_t covered = n;
  for (size_t v = 0; v < n; ++v) {
    try {
      out[v] = cc->component(static_cast<VertexId>(v));
    } catch (const std::out_of_range&) {
      out[v] = 0xFFFFFFFFu;
      if (covered == n) covered = v;
    }
  }
  return covered;
}
size_t vxr_cc_last_repaired(void* c) {
  return static_cast<velographx::IncrementalComponents*>(c)->last_repaired_vertices();
}

void* vxr_sssp_create(void* g, uint32_t source) {
  return new velographx::IncrementalSSSP(*static_cast<DynamicGraph*>(g), source);
}
void vxr_sssp_destroy(void* s) { delete static_cast<velographx::IncrementalSSSP*>(s); }
int vxr_sssp_apply(void* s, const uint32_t* src, const uint32_t* dst, const uint8_t* add, size_t n) {
  static_cast<velographx::IncrementalSSSP*>(s)->apply(make_batch(src, dst, add, n));
  return 0;
}
void vxr_sssp_recompute(void* s) { static_cast<velographx::IncrementalSSSP*>(s)->recompute(); }
size_t vxr_sssp_distances(void* s, uint64_t* out, size_t cap) {
  const auto& d = static_cast<velographx::IncrementalSSSP*>(s)->distances();
  if (out) std::memcpy(out, d.data(), std::min(cap, d.size()) * sizeof(uint64_t));
  return d.size();
}

}  // extern "C"
