/*
 * vx_b200.h -- C ABI of the B200 dynamic-BFS library (libvx_b200.so).
 *
 * This is the boundary a VeloGraphX host binds to replace its CPU dynamic-BFS
 * path.  Every entry point names the reference interface it replaces
 * (paths relative to the VeloGraphX project root).  Plain pointers and sizes
 * only; no C++ or torch types.
 *
 * Conventions
 *   - Every function returns an int status: VX_OK (0) or a negative VX_ERR_*.
 *     vx_last_error() returns the message of the calling thread's last error.
 *   - Host-pointer variants copy their inputs; *_device variants take device
 *     pointers on the current CUDA device and enqueue on the graph's stream.
 *   - Objects are single-threaded, like the reference classes
 *     (include/velographx/storage/dynamic_graph.hpp, incremental/bfs.hpp).
 *   - Vertex ids are uint32 and must be below 2^31 (bit 31 marks deleted base
 *     arcs on the device).  The unreachable distance is 0xFFFFFFFF
 *     (include/velographx/types.hpp:7).
 */
#ifndef VX_B200_H
#define VX_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define VX_OK 0
#define VX_ERR_INVALID (-1) /* malformed argument  (std::invalid_argument)   */
#define VX_ERR_RANGE (-2)   /* id or size out of the supported range        */
#define VX_ERR_CUDA (-3)    /* CUDA runtime error   (std::runtime_error)     */
#define VX_ERR_NOMEM (-4)   /* device allocation failed                     */
#define VX_ERR_DEVICE (-5)  /* a kernel reported an error word (bounded wait
                               expired, loop bound, bad id, arena overflow)  */

#define VX_UNREACHABLE 0xFFFFFFFFu

typedef struct vx_graph vx_graph;
typedef struct vx_bfs vx_bfs;

typedef struct vx_bfs_stats_t {
  uint64_t reachable_count;          /* bfs.hpp:24 */
  uint64_t last_deletion_candidates; /* bfs.hpp:25 */
  uint64_t last_affected_vertices;   /* bfs.hpp:26 */
  int32_t last_used_full_recompute;  /* bfs.hpp:27 */
  uint32_t levels;                   /* BFS levels of the last full recompute */
  uint32_t readback_bytes;           /* bytes this call copied device -> host */
  uint32_t reserved;
} vx_bfs_stats_t;

/* Copies the calling thread's last error message; returns its length. */
int vx_last_error(char* buf, size_t cap);
/* Kernels launched by this library since it was loaded (all threads). */
uint64_t vx_launch_count(void);

/* ---- DynamicGraph (include/velographx/storage/dynamic_graph.hpp) -------- */

/* DynamicGraph(size_t vertices = 0, bool directed = false)   :481-487 */
int vx_graph_create(size_t vertices, int directed, vx_graph** out);
int vx_graph_destroy(vx_graph* g);
/* vertex_count() :489, version() :490, directed() :491 */
int vx_graph_vertex_count(vx_graph* g, size_t* out);
int vx_graph_version(vx_graph* g, uint64_t* out);
int vx_graph_directed(vx_graph* g, int* out);
/* bulk_load_edges(const vector<pair<VertexId,VertexId>>&)   :502-529
 * uv holds n (u, v) pairs, row-major. */
int vx_graph_bulk_load(vx_graph* g, const uint32_t* uv, size_t n);
int vx_graph_bulk_load_device(vx_graph* g, const uint32_t* d_uv, size_t n);
/* apply(const UpdateBatch&)   :543-549 (add_edge / remove_edge :531-541 are
 * one-op batches).  Op i is (src[i], dst[i]); add[i] != 0 inserts. */
int vx_graph_apply(vx_graph* g, const uint32_t* src, const uint32_t* dst, const uint8_t* add, size_t n);
/* Device-resident batch.  vertex_count_after must equal
 * max(vertex_count, 1 + max over non-self-loop ops of max(src, dst)); ids at or
 * beyond it are rejected (VX_ERR_DEVICE at the next synchronising call). */
int vx_graph_apply_device(vx_graph* g, const uint32_t* d_src, const uint32_t* d_dst, const uint8_t* d_add,
                          size_t n, size_t vertex_count_after);
/* neighbors(u) :551-553 / in_neighbors(v) :555-557: writes up to cap ids in
 * ascending order, *n = full row length. */
int vx_graph_neighbors(vx_graph* g, uint32_t u, uint32_t* out, size_t cap, size_t* n);
int vx_graph_in_neighbors(vx_graph* g, uint32_t v, uint32_t* out, size_t cap, size_t* n);
/* has_edge(u, v) :583-587 */
int vx_graph_has_edge(vx_graph* g, uint32_t u, uint32_t v, int* out);
/* edge_count_directed() :589-591, delta_edge_count() :597, is_compact() :569-571,
 * dirty_out/in_segment_count() :612-618 */
int vx_graph_edge_count_directed(vx_graph* g, size_t* out);
int vx_graph_delta_edge_count(vx_graph* g, size_t* out);
int vx_graph_is_compact(vx_graph* g, int* out);
int vx_graph_dirty_rows(vx_graph* g, size_t* out_rows, size_t* in_rows);
/* compact() :633-639 and maybe_compact(threshold) :620-631.  The device merges
 * the whole overlay into a fresh CSR; maybe_compact does so when any dirty row
 * reaches the reference's density rule and returns 1 in *compacted. */
int vx_graph_compact(vx_graph* g);
int vx_graph_maybe_compact(vx_graph* g, double threshold, int* compacted);
/* The graph's CUDA stream (cudaStream_t) and a host-side wait for it. */
int vx_graph_stream(vx_graph* g, void** stream);
int vx_graph_synchronize(vx_graph* g);

/* ---- BasicIncrementalBFS<DynamicGraph> (include/velographx/incremental/bfs.hpp) */

/* BasicIncrementalBFS(Graph&, VertexId source, double deletion_fallback_fraction = 0.35)
 * :18-21.  Holds g (non-owning); runs recompute(). */
int vx_bfs_create(vx_graph* g, uint32_t source, double deletion_fallback_fraction, vx_bfs** out);
int vx_bfs_destroy(vx_bfs* b);
/* recompute() :100-120 */
int vx_bfs_recompute(vx_bfs* b);
/* apply(const UpdateBatch&) :29-98 -- also applies the batch to the graph. */
int vx_bfs_apply(vx_bfs* b, const uint32_t* src, const uint32_t* dst, const uint8_t* add, size_t n);
int vx_bfs_apply_device(vx_bfs* b, const uint32_t* d_src, const uint32_t* d_dst, const uint8_t* d_add, size_t n,
                        size_t vertex_count_after);
/* distances() :23 -- copies min(cap, len) entries, *n = len. */
int vx_bfs_distances(vx_bfs* b, uint32_t* host_out, size_t cap, size_t* n);
/* Device pointer to the distance vector (valid until the next call on b). */
int vx_bfs_distances_device(vx_bfs* b, const uint32_t** d_dist, size_t* n);
/* reachable_count / last_* getters :24-27 */
int vx_bfs_stats(vx_bfs* b, vx_bfs_stats_t* out);
/* Sum of out-degrees of reached vertices (arcs traversed by a full top-down
 * BFS), for TEPS reporting. */
int vx_bfs_reached_arcs(vx_bfs* b, uint64_t* out);
/* Per-level trace of the last full BFS: for each level {globaltimer ns,
 * frontier size | bottom_up << 63}, then a closing timestamp; *n = entries.
 * No reference counterpart (diagnostics). */
int vx_bfs_level_trace(vx_bfs* b, uint64_t* out, size_t cap, size_t* n);
/* Direction switch (alpha, beta) and grid-expanded row length of the full BFS.
 * No reference counterpart: the reference BFS is top-down only. */
int vx_bfs_set_tuning(vx_bfs* b, float alpha, float beta, uint32_t large_row);

/* ---- Multi-root BFS (up to 256 roots, one launch) ----------------------
 * For every root r, row r of the result equals BasicIncrementalBFS(g,
 * roots[r]).distances() (bfs.hpp:100-120); the reference's multicore harness
 * benchmarks/thread_scaling_bfs.cpp:78-108 computes the same with one thread
 * per root.  Distances are laid out root-major: dist[r * V + v]. */
typedef struct vx_mrbfs vx_mrbfs;
int vx_mrbfs_create(vx_graph* g, const uint32_t* roots, size_t k, vx_mrbfs** out);
int vx_mrbfs_destroy(vx_mrbfs* m);
/* Enqueues the traversal on the graph's stream (asynchronous). */
int vx_mrbfs_run(vx_mrbfs* m);
/* Waits, then copies min(cap, k*V) distances; *n = k*V. */
int vx_mrbfs_distances(vx_mrbfs* m, uint32_t* host_out, size_t cap, size_t* n);
int vx_mrbfs_distances_device(vx_mrbfs* m, const uint32_t** d_dist, size_t* n);
/* Sum over roots of the out-degrees of reached vertices (for TEPS), and the
 * level count of the last run. */
int vx_mrbfs_reached_arcs(vx_mrbfs* m, uint64_t* out);
int vx_mrbfs_levels(vx_mrbfs* m, uint32_t* out);
/* Pull (bottom-up) when the frontier holds more than frac * V vertices. */
int vx_mrbfs_set_pull_fraction(vx_mrbfs* m, float frac);
/* One-shot form: create, run, copy k*V distances into out (cap entries). */
int vx_multiroot_bfs(vx_graph* g, const uint32_t* roots, size_t k, uint32_t* out, size_t cap);

#ifdef __cplusplus
}
#endif
#endif
