// C ABI (include/vx_b200.h) over the device graph and BFS.
#include <algorithm>
#include <atomic>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <string>

#include "../../include/vx_b200.h"
#include "bfs.cuh"
#include "vstream.cuh"
#include "components.cuh"
#include "graph.cuh"
#include "io.cuh"
#include "mrbfs.cuh"
#include "selector.cuh"

namespace vxh {

static thread_local char g_err[1024] = "";
static std::atomic<uint64_t> g_launches{0};

void count_launch() { g_launches.fetch_add(1, std::memory_order_relaxed); }

void set_error(const char* fmt, ...) {
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(g_err, sizeof(g_err), fmt, ap);
  va_end(ap);
}

}  // namespace vxh

struct vx_graph {
  vxh::Graph* g;
};
struct vx_bfs {
  vxh::Bfs* b;
  vx_graph* owner;
};
struct vx_cc {
  vxh::Components* c;
};
struct vx_mrbfs {
  vxh::MrBfs* m;
};
struct vx_selector {
  vxh::Selector* s;
};
struct vx_heuristic {
  vxh::HeuristicState h;
};

namespace {

int fail(int code, const char* msg) {
  vxh::set_error("%s", msg);
  return code;
}

// Host batch -> device batch buffers; returns the vertex count after the batch.
int upload_batch(vxh::Graph* g, const uint32_t* src, const uint32_t* dst, const uint8_t* add, size_t n,
                 size_t* v_after) {
  size_t vmax = g->V;
  for (size_t i = 0; i < n; ++i) {
    if (src[i] == dst[i]) continue;  // self-loops never grow the graph
    const size_t m = (size_t)std::max(src[i], dst[i]) + 1;
    if (m > vmax) vmax = m;
  }
  if (vmax > vxb::kMaxVertices) return fail(VX_ERR_RANGE, "vertex id beyond the supported maximum (2^31 - 1)");
  if (int rc = g->batch.ensure(n)) return rc;
  cudaStream_t s = g->stream;
  VX_CUDA_TRY(cudaMemcpyAsync(g->batch.src, src, n * 4, cudaMemcpyHostToDevice, s));
  VX_CUDA_TRY(cudaMemcpyAsync(g->batch.dst, dst, n * 4, cudaMemcpyHostToDevice, s));
  VX_CUDA_TRY(cudaMemcpyAsync(g->batch.add, add, n, cudaMemcpyHostToDevice, s));
  g->batch.in_src = g->batch.src;
  g->batch.in_dst = g->batch.dst;
  g->batch.in_add = g->batch.add;
  *v_after = vmax;
  return 0;
}

// A device batch is read in place by the staging kernels (stream-ordered).
int stage_device_batch(vxh::Graph* g, const uint32_t* d_src, const uint32_t* d_dst, const uint8_t* d_add, size_t n) {
  if (int rc = g->batch.ensure(n)) return rc;
  g->batch.in_src = d_src;
  g->batch.in_dst = d_dst;
  g->batch.in_add = d_add;
  return 0;
}

}  // namespace

extern "C" {

int vx_last_error(char* buf, size_t cap) {
  const size_t n = strlen(vxh::g_err);
  if (buf && cap) {
    const size_t m = std::min(n, cap - 1);
    memcpy(buf, vxh::g_err, m);
    buf[m] = 0;
  }
  return (int)n;
}

uint64_t vx_launch_count(void) { return vxh::g_launches.load(std::memory_order_relaxed); }

int vx_graph_create(size_t vertices, int directed, vx_graph** out) {
  if (!out) return fail(VX_ERR_INVALID, "null output pointer");
  vxh::Graph* g = nullptr;
  if (int rc = vxh::graph_create(&g, vertices, directed != 0)) return rc;
  *out = new vx_graph{g};
  return VX_OK;
}

int vx_graph_destroy(vx_graph* g) {
  if (!g) return VX_OK;
  vxh::graph_destroy(g->g);
  delete g;
  return VX_OK;
}

int vx_graph_vertex_count(vx_graph* g, size_t* out) {
  if (!g || !out) return fail(VX_ERR_INVALID, "null argument");
  *out = g->g->V;
  return VX_OK;
}

int vx_graph_version(vx_graph* g, uint64_t* out) {
  if (!g || !out) return fail(VX_ERR_INVALID, "null argument");
  *out = g->g->version;
  return VX_OK;
}

int vx_graph_directed(vx_graph* g, int* out) {
  if (!g || !out) return fail(VX_ERR_INVALID, "null argument");
  *out = g->g->directed ? 1 : 0;
  return VX_OK;
}

int vx_graph_bulk_load(vx_graph* g, const uint32_t* uv, size_t n) {
  if (!g || (!uv && n)) return fail(VX_ERR_INVALID, "null argument");
  uint32_t* d = nullptr;
  if (cudaMalloc(&d, std::max<size_t>(n, 1) * 8) != cudaSuccess) return fail(VX_ERR_NOMEM, "bulk load upload");
  int rc = VX_OK;
  // on the graph's own (non-blocking) stream: a plain cudaMemcpy from pageable
  // memory may return before its DMA lands and is not ordered before the load
  // kernels on that stream
  if (n && cudaMemcpyAsync(d, uv, n * 8, cudaMemcpyHostToDevice, g->g->stream) != cudaSuccess)
    rc = fail(VX_ERR_CUDA, "bulk copy");
  if (!rc) rc = vxh::graph_bulk_load(g->g, d, n);
  cudaFree(d);
  return rc;
}

int vx_graph_bulk_load_device(vx_graph* g, const uint32_t* d_uv, size_t n) {
  if (!g || (!d_uv && n)) return fail(VX_ERR_INVALID, "null argument");
  return vxh::graph_bulk_load(g->g, d_uv, n);
}

int vx_graph_apply(vx_graph* g, const uint32_t* src, const uint32_t* dst, const uint8_t* add, size_t n) {
  if (!g || (n && (!src || !dst || !add))) return fail(VX_ERR_INVALID, "null argument");
  if (n == 0) return VX_OK;  // empty batch: no version bump (dynamic_graph.hpp:545)
  size_t v_after = 0;
  if (int rc = upload_batch(g->g, src, dst, add, n, &v_after)) return rc;
  if (int rc = vxh::graph_stage_batch(g->g, n, v_after)) return rc;
  return vxh::graph_commit_batch(g->g);
}

int vx_graph_apply_device(vx_graph* g, const uint32_t* d_src, const uint32_t* d_dst, const uint8_t* d_add, size_t n,
                          size_t vertex_count_after) {
  if (!g || (n && (!d_src || !d_dst || !d_add))) return fail(VX_ERR_INVALID, "null argument");
  if (n == 0) return VX_OK;
  if (vertex_count_after < g->g->V) return fail(VX_ERR_INVALID, "vertex_count_after below vertex_count");
  if (int rc = stage_device_batch(g->g, d_src, d_dst, d_add, n)) return rc;
  if (int rc = vxh::graph_stage_batch(g->g, n, vertex_count_after)) return rc;
  return vxh::graph_commit_batch(g->g);
}

int vx_graph_neighbors(vx_graph* g, uint32_t u, uint32_t* out, size_t cap, size_t* n) {
  if (!g || !n) return fail(VX_ERR_INVALID, "null argument");
  return vxh::graph_row(g->g, 0, u, out, cap, n);
}

int vx_graph_in_neighbors(vx_graph* g, uint32_t v, uint32_t* out, size_t cap, size_t* n) {
  if (!g || !n) return fail(VX_ERR_INVALID, "null argument");
  return vxh::graph_row(g->g, 1, v, out, cap, n);
}

int vx_graph_load_edge_list(const char* path, int directed, vx_graph** out) {
  if (!path || !out) return fail(VX_ERR_INVALID, "null argument");
  vxh::Graph* g = nullptr;
  if (int rc = vxh::graph_load_edge_list(path, directed != 0, &g)) return rc;
  *out = new vx_graph{g};
  return VX_OK;
}

int vx_graph_save_binary(vx_graph* g, const char* path) {
  if (!g || !path) return fail(VX_ERR_INVALID, "null argument");
  return vxh::graph_save_binary(g->g, path);
}

int vx_graph_load_binary(const char* path, int directed, vx_graph** out) {
  if (!path || !out) return fail(VX_ERR_INVALID, "null argument");
  vxh::Graph* g = nullptr;
  if (int rc = vxh::graph_load_binary(path, directed != 0, &g)) return rc;
  *out = new vx_graph{g};
  return VX_OK;
}

int vx_graph_snapshot(vx_graph* g, vx_graph** out) {
  if (!g || !out) return fail(VX_ERR_INVALID, "null argument");
  vxh::Graph* s = nullptr;
  if (int rc = vxh::graph_snapshot(g->g, &s)) return rc;
  *out = new vx_graph{s};
  return VX_OK;
}

int vx_graph_scan_rows(vx_graph* g, uint64_t* arcs, double* ns) {
  if (!g || !arcs || !ns) return fail(VX_ERR_INVALID, "null argument");
  return vxh::graph_scan_rows(g->g, arcs, ns);
}

int vx_graph_ensure_vertex(vx_graph* g, uint32_t v) {
  if (!g) return fail(VX_ERR_INVALID, "null argument");
  if ((size_t)v + 1 > vxb::kMaxVertices) return fail(VX_ERR_RANGE, "vertex id beyond the supported maximum (2^31 - 1)");
  // grows the vertex count only; the version is unchanged (dynamic_graph.hpp:493-500)
  return vxh::graph_grow(g->g, (size_t)v + 1);
}

int vx_graph_compact_neighbors(vx_graph* g, uint32_t u, uint32_t* out, size_t cap, size_t* n) {
  if (!g || !n) return fail(VX_ERR_INVALID, "null argument");
  return vxh::graph_compact_row(g->g, 0, u, out, cap, n);
}

int vx_graph_compact_in_neighbors(vx_graph* g, uint32_t v, uint32_t* out, size_t cap, size_t* n) {
  if (!g || !n) return fail(VX_ERR_INVALID, "null argument");
  return vxh::graph_compact_row(g->g, 1, v, out, cap, n);
}

int vx_graph_base_edge_count_directed(vx_graph* g, size_t* out) {
  if (!g || !out) return fail(VX_ERR_INVALID, "null argument");
  *out = (size_t)g->g->adj[0].A;
  return VX_OK;
}

int vx_graph_storage_bytes(vx_graph* g, size_t* out) {
  if (!g || !out) return fail(VX_ERR_INVALID, "null argument");
  *out = vxh::graph_storage_bytes(g->g);
  return VX_OK;
}

int vx_graph_has_edge(vx_graph* g, uint32_t u, uint32_t v, int* out) {
  if (!g || !out) return fail(VX_ERR_INVALID, "null argument");
  return vxh::graph_has_edge(g->g, u, v, out);
}

int vx_graph_edge_count_directed(vx_graph* g, size_t* out) {
  if (!g || !out) return fail(VX_ERR_INVALID, "null argument");
  if (int rc = vxh::graph_sync_counters(g->g)) return rc;
  *out = (size_t)vxh::graph_edge_count_directed(g->g);
  return VX_OK;
}

int vx_graph_delta_edge_count(vx_graph* g, size_t* out) {
  if (!g || !out) return fail(VX_ERR_INVALID, "null argument");
  if (int rc = vxh::graph_sync_counters(g->g)) return rc;
  *out = (size_t)(g->g->hctr->delta_live[0] + g->g->hctr->tombs[0]);
  return VX_OK;
}

int vx_graph_is_compact(vx_graph* g, int* out) {
  if (!g || !out) return fail(VX_ERR_INVALID, "null argument");
  if (int rc = vxh::graph_sync_counters(g->g)) return rc;
  const vxh::GraphCounters* c = g->g->hctr;
  *out = (c->delta_live[0] + c->tombs[0] + c->delta_live[1] + c->tombs[1]) == 0;
  return VX_OK;
}

int vx_graph_dirty_rows(vx_graph* g, size_t* out_rows, size_t* in_rows) {
  if (!g || !out_rows || !in_rows) return fail(VX_ERR_INVALID, "null argument");
  if (int rc = vxh::graph_sync_counters(g->g)) return rc;
  *out_rows = (size_t)g->g->hctr->dirty_rows[0];
  *in_rows = (size_t)g->g->hctr->dirty_rows[g->g->directed ? 1 : 0];
  return VX_OK;
}

int vx_graph_compact(vx_graph* g) {
  if (!g) return fail(VX_ERR_INVALID, "null argument");
  int compact = 0;
  if (int rc = vx_graph_is_compact(g, &compact)) return rc;
  if (compact) return VX_OK;
  return vxh::graph_consolidate(g->g);
}

int vx_graph_maybe_compact(vx_graph* g, double threshold, int* compacted) {
  if (!g || !compacted) return fail(VX_ERR_INVALID, "null argument");
  return vxh::graph_maybe_compact(g->g, threshold, compacted);
}

int vx_graph_stream(vx_graph* g, void** stream) {
  if (!g || !stream) return fail(VX_ERR_INVALID, "null argument");
  *stream = (void*)g->g->stream;
  return VX_OK;
}

int vx_graph_synchronize(vx_graph* g) {
  if (!g) return fail(VX_ERR_INVALID, "null argument");
  return vxh::graph_sync_counters(g->g);
}

int vx_bfs_create(vx_graph* g, uint32_t source, double frac, vx_bfs** out) {
  if (!g || !out) return fail(VX_ERR_INVALID, "null argument");
  vxh::Bfs* b = nullptr;
  if (int rc = vxh::bfs_create(&b, g->g, source, frac)) return rc;
  *out = new vx_bfs{b, g};
  return VX_OK;
}

int vx_bfs_destroy(vx_bfs* b) {
  if (!b) return VX_OK;
  vxh::bfs_destroy(b->b);
  delete b;
  return VX_OK;
}

int vx_bfs_recompute(vx_bfs* b) {
  if (!b) return fail(VX_ERR_INVALID, "null argument");
  return vxh::bfs_recompute(b->b);
}

int vx_bfs_apply(vx_bfs* b, const uint32_t* src, const uint32_t* dst, const uint8_t* add, size_t n) {
  if (!b || (n && (!src || !dst || !add))) return fail(VX_ERR_INVALID, "null argument");
  vxh::Graph* g = b->b->g;
  size_t v_after = g->V;
  if (n)
    if (int rc = upload_batch(g, src, dst, add, n, &v_after)) return rc;
  return vxh::bfs_apply_staged(b->b, n, v_after);
}

int vx_bfs_apply_device(vx_bfs* b, const uint32_t* d_src, const uint32_t* d_dst, const uint8_t* d_add, size_t n,
                        size_t vertex_count_after) {
  if (!b || (n && (!d_src || !d_dst || !d_add))) return fail(VX_ERR_INVALID, "null argument");
  vxh::Graph* g = b->b->g;
  if (n) {
    if (vertex_count_after < g->V) return fail(VX_ERR_INVALID, "vertex_count_after below vertex_count");
    if (int rc = stage_device_batch(g, d_src, d_dst, d_add, n)) return rc;
  }
  return vxh::bfs_apply_staged(b->b, n, std::max<size_t>(vertex_count_after, g->V));
}

int vx_bfs_distances(vx_bfs* b, uint32_t* host_out, size_t cap, size_t* n) {
  if (!b || !n) return fail(VX_ERR_INVALID, "null argument");
  vxh::Bfs* x = b->b;
  *n = x->dist_len;
  const size_t m = std::min(cap, x->dist_len);
  if (host_out && m) {
    VX_CUDA_TRY(cudaMemcpyAsync(host_out, x->dist, m * 4, cudaMemcpyDeviceToHost, x->g->stream));
  }
  return vxh::bfs_sync(x);
}

int vx_bfs_distances_device(vx_bfs* b, const uint32_t** d_dist, size_t* n) {
  if (!b || !d_dist || !n) return fail(VX_ERR_INVALID, "null argument");
  *d_dist = b->b->dist;
  *n = b->b->dist_len;
  return VX_OK;
}

int vx_bfs_stats(vx_bfs* b, vx_bfs_stats_t* out) {
  if (!b || !out) return fail(VX_ERR_INVALID, "null argument");
  if (int rc = vxh::bfs_sync(b->b)) return rc;
  const vxh::BfsCounters* c = b->b->hctr;
  out->reachable_count = c->reachable;
  out->last_deletion_candidates = c->candidates;
  out->last_affected_vertices = c->affected;
  out->last_used_full_recompute = c->full ? 1 : 0;
  out->levels = c->levels;
  out->readback_bytes = (uint32_t)sizeof(vxh::BfsCounters);
  out->reserved = 0;
  return VX_OK;
}

int vx_bfs_reached_arcs(vx_bfs* b, uint64_t* out) {
  if (!b || !out) return fail(VX_ERR_INVALID, "null argument");
  unsigned long long a = 0;
  if (int rc = vxh::bfs_reached_arcs(b->b, &a)) return rc;
  *out = a;
  return VX_OK;
}

int vx_bfs_apply_stream(vx_bfs* b, const uint32_t* src, const uint32_t* dst, const uint8_t* add,
                        const uint64_t* offsets, size_t nbatches, uint64_t* digests, uint32_t* stats) {
  if (!b || !offsets || (nbatches && offsets[nbatches] && (!src || !dst || !add)))
    return fail(VX_ERR_INVALID, "null argument");
  size_t applied = 0;
  if (int rc = vxh::bfs_apply_stream(b->b, src, dst, add, offsets, nbatches, digests, stats, &applied)) return rc;
  for (size_t t = applied; t < nbatches; ++t) {
    const uint64_t lo = offsets[t];
    if (int rc = vx_bfs_apply(b, src + lo, dst + lo, add + lo, offsets[t + 1] - lo)) return rc;
    if (digests)
      if (int rc = vxh::bfs_digest(b->b, reinterpret_cast<uint64_t*>(digests + t))) return rc;
    if (stats) {
      if (int rc = vxh::bfs_sync(b->b)) return rc;
      const vxh::BfsCounters& c = *b->b->hctr;
      stats[4 * t + 0] = c.candidates;
      stats[4 * t + 1] = c.affected;
      stats[4 * t + 2] = c.full;
      stats[4 * t + 3] = (uint32_t)c.reachable;
    }
  }
  return VX_OK;
}

int vx_bfs_set_fused(vx_bfs* b, int fused) {
  if (!b) return fail(VX_ERR_INVALID, "null argument");
  b->b->tune.fused = fused != 0;
  return VX_OK;
}

int vx_graph_reserve(vx_graph* g, size_t max_batch_ops, size_t total_ops) {
  if (!g) return fail(VX_ERR_INVALID, "null argument");
  if (int rc = g->g->batch.ensure(max_batch_ops)) return rc;
  int fits = 0;
  const int arcs_per_op = g->g->directed ? 1 : 2;  // in the out adjacency
  if (int rc = vxh::graph_reserve_stream(g->g, 8ull * arcs_per_op * total_ops + 8, &fits)) return rc;
  return VX_OK;  // past the arena limit the stream consolidates as it goes
}

int vx_bfs_reserve_stream(vx_bfs* b, size_t ops, size_t batches, size_t max_batch_ops) {
  if (!b) return fail(VX_ERR_INVALID, "null argument");
  if (int rc = b->b->sb.ensure(ops, batches, 2 * std::max<size_t>(max_batch_ops, 1))) return rc;
  const size_t window = std::min<size_t>(b->b->tune.stream_window, batches);
  if (window == 0 || b->b->g->directed) return VX_OK;
  const size_t wops = std::min<size_t>(ops, window * std::max<size_t>(max_batch_ops, 1));
  return vxh::stream_versions_reserve(b->b, wops, b->b->g->V, window);
}

int vx_bfs_digest(vx_bfs* b, uint64_t* out) {
  if (!b || !out) return fail(VX_ERR_INVALID, "null argument");
  return vxh::bfs_digest(b->b, out);
}

int vx_bfs_phase_trace(vx_bfs* b, uint64_t* out, size_t cap, size_t* n) {
  if (!b || !n || (cap && !out)) return fail(VX_ERR_INVALID, "null argument");
  return vxh::bfs_phase_trace(b->b, reinterpret_cast<unsigned long long*>(out), cap, n);
}

int vx_bfs_level_trace(vx_bfs* b, uint64_t* out, size_t cap, size_t* n) {
  if (!b || !n) return fail(VX_ERR_INVALID, "null argument");
  return vxh::bfs_level_trace(b->b, reinterpret_cast<unsigned long long*>(out), cap, n);
}

int vx_bfs_autotune(vx_bfs* b, const uint32_t* roots, size_t k, float* chosen) {
  if (!b || (k && !roots)) return fail(VX_ERR_INVALID, "null argument");
  if (k == 0) return fail(VX_ERR_INVALID, "autotune needs at least one root");
  for (size_t i = 0; i < k; ++i)
    if (roots[i] >= b->b->g->V) return fail(VX_ERR_RANGE, "autotune root beyond the vertex count");
  return vxh::bfs_autotune(b->b, roots, k, chosen);
}

int vx_bfs_get_tuning(vx_bfs* b, float* alpha, float* beta, uint32_t* large_row) {
  if (!b || !alpha || !beta || !large_row) return fail(VX_ERR_INVALID, "null argument");
  *alpha = b->b->tune.alpha;
  *beta = b->b->tune.beta;
  *large_row = b->b->tune.large_row;
  return VX_OK;
}

int vx_bfs_set_accounting(vx_bfs* b, int on) {
  if (!b) return fail(VX_ERR_INVALID, "null argument");
  return vxh::bfs_set_accounting(b->b, on);
}

int vx_bfs_accounting(vx_bfs* b, uint64_t* out5) {
  if (!b || !out5) return fail(VX_ERR_INVALID, "null argument");
  return vxh::bfs_accounting(b->b, reinterpret_cast<unsigned long long*>(out5));
}

int vx_bfs_set_update_blocks(vx_bfs* b, uint32_t blocks) {
  if (!b) return fail(VX_ERR_INVALID, "null argument");
  b->b->tune.update_blocks = blocks;
  return VX_OK;
}

int vx_bfs_set_stream_window(vx_bfs* b, uint32_t batches) {
  if (!b) return fail(VX_ERR_INVALID, "null argument");
  b->b->tune.stream_window = batches;
  return VX_OK;
}

int vx_bfs_set_window_pull_fraction(vx_bfs* b, float frac) {
  if (!b || !(frac > 0.f)) return fail(VX_ERR_INVALID, "invalid pull fraction");
  b->b->tune.window_pull_frac = frac;
  return VX_OK;
}

int vx_bfs_set_handover(vx_bfs* b, float multiple) {
  if (!b || multiple != multiple) return fail(VX_ERR_INVALID, "invalid handover multiple");
  b->b->tune.handover = multiple;
  return VX_OK;
}

int vx_bfs_window_trace(vx_bfs* b, uint64_t* out, size_t cap, size_t* n) {
  if (!b || !n || (cap && !out)) return fail(VX_ERR_INVALID, "null argument");
  return vxh::stream_versions_trace(b->b, reinterpret_cast<unsigned long long*>(out), cap, n);
}

int vx_bfs_set_tuning(vx_bfs* b, float alpha, float beta, uint32_t large_row) {
  if (!b || !(alpha > 0.f) || !(beta > 0.f) || large_row < 32) return fail(VX_ERR_INVALID, "invalid tuning");
  b->b->tune.alpha = alpha;
  b->b->tune.beta = beta;
  b->b->tune.large_row = large_row;
  return VX_OK;
}

int vx_cc_create(vx_graph* g, vx_cc** out) {
  if (!g || !out) return fail(VX_ERR_INVALID, "null argument");
  vxh::Components* c = nullptr;
  if (int rc = vxh::cc_create(&c, g->g)) return rc;
  *out = new vx_cc{c};
  return VX_OK;
}

int vx_cc_destroy(vx_cc* c) {
  if (!c) return VX_OK;
  vxh::cc_destroy(c->c);
  delete c;
  return VX_OK;
}

int vx_cc_apply(vx_cc* c, const uint32_t* src, const uint32_t* dst, const uint8_t* add, size_t n) {
  if (!c || (n && (!src || !dst || !add))) return fail(VX_ERR_INVALID, "null argument");
  if (n == 0) {
    c->c->last_repaired = 0;
    return VX_OK;
  }
  size_t v_after = 0;
  if (int rc = upload_batch(c->c->g, src, dst, add, n, &v_after)) return rc;
  return vxh::cc_apply_staged(c->c, n, v_after);
}

int vx_cc_labels(vx_cc* c, uint32_t* out, size_t cap, size_t* n) {
  if (!c || !n || (cap && !out)) return fail(VX_ERR_INVALID, "null argument");
  return vxh::cc_labels(c->c, out, cap, n);
}

int vx_cc_last_repaired_vertices(vx_cc* c, uint64_t* out) {
  if (!c || !out) return fail(VX_ERR_INVALID, "null argument");
  *out = c->c->last_repaired;
  return VX_OK;
}

int vx_mrbfs_create(vx_graph* g, const uint32_t* roots, size_t k, vx_mrbfs** out) {
  if (!g || !roots || !out) return fail(VX_ERR_INVALID, "null argument");
  vxh::MrBfs* m = nullptr;
  if (int rc = vxh::mrbfs_create(&m, g->g, roots, k)) return rc;
  *out = new vx_mrbfs{m};
  return VX_OK;
}

int vx_mrbfs_destroy(vx_mrbfs* m) {
  if (!m) return VX_OK;
  vxh::mrbfs_destroy(m->m);
  delete m;
  return VX_OK;
}

int vx_mrbfs_run(vx_mrbfs* m) {
  if (!m) return fail(VX_ERR_INVALID, "null argument");
  return vxh::mrbfs_run(m->m);
}

int vx_mrbfs_distances(vx_mrbfs* m, uint32_t* host_out, size_t cap, size_t* n) {
  if (!m || !n) return fail(VX_ERR_INVALID, "null argument");
  vxh::MrBfs* x = m->m;
  *n = x->K * x->V;
  if (int rc = vxh::mrbfs_sync(x)) return rc;
  const size_t c = std::min(cap, *n);
  if (host_out && c) VX_CUDA_TRY(cudaMemcpy(host_out, x->dist, c * 4, cudaMemcpyDeviceToHost));
  return VX_OK;
}

int vx_mrbfs_distances_device(vx_mrbfs* m, const uint32_t** d_dist, size_t* n) {
  if (!m || !d_dist || !n) return fail(VX_ERR_INVALID, "null argument");
  *d_dist = m->m->dist;
  *n = m->m->K * m->m->V;
  return VX_OK;
}

int vx_mrbfs_reached_arcs(vx_mrbfs* m, uint64_t* out) {
  if (!m || !out) return fail(VX_ERR_INVALID, "null argument");
  unsigned long long a = 0;
  if (int rc = vxh::mrbfs_reached_arcs(m->m, &a)) return rc;
  *out = a;
  return VX_OK;
}

int vx_mrbfs_levels(vx_mrbfs* m, uint32_t* out) {
  if (!m || !out) return fail(VX_ERR_INVALID, "null argument");
  if (int rc = vxh::mrbfs_sync(m->m)) return rc;
  *out = m->m->hctr->levels;
  return VX_OK;
}

int vx_mrbfs_level_trace(vx_mrbfs* m, uint64_t* out, size_t cap, size_t* n) {
  if (!m || !n || (cap && !out)) return fail(VX_ERR_INVALID, "null argument");
  return vxh::mrbfs_level_trace(m->m, reinterpret_cast<unsigned long long*>(out), cap, n);
}

int vx_mrbfs_set_pull_fraction(vx_mrbfs* m, float frac) {
  if (!m || !(frac > 0.f)) return fail(VX_ERR_INVALID, "invalid pull fraction");
  m->m->pull_frac = frac;
  return VX_OK;
}

int vx_multiroot_bfs(vx_graph* g, const uint32_t* roots, size_t k, uint32_t* out, size_t cap) {
  vx_mrbfs* m = nullptr;
  if (int rc = vx_mrbfs_create(g, roots, k, &m)) return rc;
  size_t n = 0;
  int rc = vx_mrbfs_run(m);
  if (!rc) rc = vx_mrbfs_distances(m, out, cap, &n);
  vx_mrbfs_destroy(m);
  return rc;
}

int vx_bfs_stage(vx_bfs* b, const uint32_t* src, const uint32_t* dst, const uint8_t* add, size_t n) {
  if (!b || (n && (!src || !dst || !add))) return fail(VX_ERR_INVALID, "null argument");
  vxh::Graph* g = b->b->g;
  size_t v_after = g->V;
  if (n)
    if (int rc = upload_batch(g, src, dst, add, n, &v_after)) return rc;
  return vxh::bfs_stage(b->b, n, v_after);
}

int vx_bfs_staged_features(vx_bfs* b, float prev_affected_fraction, float* out16) {
  if (!b || !out16) return fail(VX_ERR_INVALID, "null argument");
  vxh::Bfs* x = b->b;
  vxh::Graph* g = x->g;
  if (int rc = vxh::bfs_sync(x)) return rc;
  if (int rc = vxh::graph_sync_counters(g)) return rc;
  vxh::SelInputs in;
  in.ops = x->staged_ops;
  in.edges = vxh::graph_edge_count_directed(g);
  in.vertices = (uint32_t)g->V;
  in.levels = x->hctr->levels;
  in.reachable_fraction = (float)((double)x->hctr->reachable / (double)std::max<size_t>(1, g->V));
  in.prev_affected_fraction = prev_affected_fraction;
  if (x->staged_ops == 0) {
    for (int i = 0; i < vxh::kSelFeatures; ++i) out16[i] = 0.f;
    return VX_OK;
  }
  return vxh::batch_features(x, x->staged_ops, in, out16);
}

int vx_bfs_run_repair(vx_bfs* b) {
  if (!b) return fail(VX_ERR_INVALID, "null argument");
  return vxh::bfs_repair_staged(b->b);
}

int vx_bfs_run_full(vx_bfs* b) {
  if (!b) return fail(VX_ERR_INVALID, "null argument");
  return vxh::bfs_full_staged(b->b);
}

int vx_selector_create(uint64_t seed, vx_selector** out) {
  if (!out) return fail(VX_ERR_INVALID, "null argument");
  vxh::Selector* s = nullptr;
  if (int rc = vxh::selector_create(&s, seed)) return rc;
  *out = new vx_selector{s};
  return VX_OK;
}

int vx_selector_destroy(vx_selector* s) {
  if (!s) return VX_OK;
  vxh::selector_destroy(s->s);
  delete s;
  return VX_OK;
}

int vx_selector_train(vx_selector* s, const float* X, const float* Y, size_t n, uint32_t epochs, uint32_t batch,
                      float lr, uint32_t seed, float* final_loss) {
  if (!s || !X || !Y) return fail(VX_ERR_INVALID, "null argument");
  return vxh::selector_train(s->s, X, Y, n, epochs, batch, lr, seed, final_loss);
}

int vx_selector_gradients(vx_selector* s, const float* X, const float* Y, size_t n, float* grad, float* loss) {
  if (!s || !X || !Y || !grad) return fail(VX_ERR_INVALID, "null argument");
  return vxh::selector_gradients(s->s, X, Y, n, grad, loss);
}

int vx_selector_predict(vx_selector* s, const float* X, size_t n, float* Y) {
  if (!s || (n && (!X || !Y))) return fail(VX_ERR_INVALID, "null argument");
  return vxh::selector_predict(s->s, X, n, Y);
}

int vx_selector_set_params(vx_selector* s, const float* params) {
  if (!s || !params) return fail(VX_ERR_INVALID, "null argument");
  return vxh::selector_set_params(s->s, params);
}

int vx_selector_get_params(vx_selector* s, float* params) {
  if (!s || !params) return fail(VX_ERR_INVALID, "null argument");
  return vxh::selector_get_params(s->s, params);
}

int vx_heuristic_create(size_t vertices, double initial_reachable_fraction, double initial_full_us,
                        vx_heuristic** out) {
  if (!out) return fail(VX_ERR_INVALID, "null argument");
  vx_heuristic* h = new vx_heuristic();
  h->h.large_scale = vertices >= 200000;  // publication_policy_bfs.cpp:94
  h->h.initial_reachable_fraction = initial_reachable_fraction;
  h->h.ema_full_us = initial_full_us;
  h->h.have_full = true;
  *out = h;
  return VX_OK;
}

int vx_heuristic_destroy(vx_heuristic* h) {
  delete h;
  return VX_OK;
}

int vx_heuristic_decide(vx_heuristic* h, double update_fraction, double shallow_fraction, int* choose_full) {
  if (!h || !choose_full) return fail(VX_ERR_INVALID, "null argument");
  *choose_full = vxh::heuristic_decide(h->h, update_fraction, shallow_fraction) ? 1 : 0;
  return VX_OK;
}

int vx_heuristic_observe(vx_heuristic* h, int observed_full, double execution_us, double affected_fraction) {
  if (!h) return fail(VX_ERR_INVALID, "null argument");
  vxh::heuristic_observe(h->h, observed_full != 0, execution_us, affected_fraction);
  return VX_OK;
}

}  // extern "C"
