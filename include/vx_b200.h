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
 *     pointers on the current CUDA device and enqueue on the graph's stream,
 *     which reads the arrays in place: they must stay unchanged until that
 *     stream has run the call's work.
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
#define VX_ERR_FORMAT (-6)  /* malformed input file   (std::runtime_error)   */
#define VX_ERR_OVERFLOW (-7) /* id beyond uint32 in a file (std::overflow_error) */
#define VX_ERR_IO (-8)      /* cannot open, read or write a file (std::runtime_error) */

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
/* ensure_vertex(v) :493-500: grows the vertex count to v + 1 (never shrinks;
 * the version is unchanged). */
int vx_graph_ensure_vertex(vx_graph* g, uint32_t v);
/* compact_neighbors(u) :573-576 / compact_in_neighbors(v) :578-581: the row as
 * of the last consolidation (the base CSR row; arcs deleted since are still
 * in it), ascending; writes up to cap ids, *n = full length. */
int vx_graph_compact_neighbors(vx_graph* g, uint32_t u, uint32_t* out, size_t cap, size_t* n);
int vx_graph_compact_in_neighbors(vx_graph* g, uint32_t v, uint32_t* out, size_t cap, size_t* n);
/* base_edge_count_directed() :593-595: arcs of the compact representation. */
int vx_graph_base_edge_count_directed(vx_graph* g, size_t* out);
/* storage_bytes() :599-605: here the device bytes the graph's storage holds
 * (its layout differs from the reference's host layout). */
int vx_graph_storage_bytes(vx_graph* g, size_t* out);
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
/* ---- On-disk formats --------------------------------------------------
 * load_edge_list(path, directed) (include/velographx/io.hpp:6, src/io.cpp:23-53):
 * a text edge list, one "u v" per line, blank lines and lines starting with '#'
 * or '%' (after leading whitespace) skipped; parsed on the device.  The result
 * is a new graph with the file's edges bulk-loaded (self-loops and duplicates
 * dropped, vertex count max id + 1), the logical graph of the reference's
 * CsrGraph.  Errors name the first bad line as the reference does:
 * "malformed edge list at line N" and "unexpected trailing data at line N"
 * (VX_ERR_FORMAT), "vertex id exceeds uint32 range at line N"
 * (VX_ERR_OVERFLOW), "unable to open edge-list file" (VX_ERR_IO). */
int vx_graph_load_edge_list(const char* path, int directed, vx_graph** out);
/* io::save_binary(g, path) (include/velographx/io/binary_graph.hpp:9-14): the
 * reference's format -- u64 magic 0x564758303031, u64 vertex count, u64
 * edge_count_directed, then (u32 u, u32 v) for every arc, rows in vertex
 * order, each ascending.  The graph is not modified. */
int vx_graph_save_binary(vx_graph* g, const char* path);
/* io::load_binary(path, directed) (binary_graph.hpp:15-20): a new graph with
 * the file's vertex count and, for an undirected graph, the pairs with u <= v;
 * version 1 when any pair was kept, else 0.  Errors: "cannot open input"
 * (VX_ERR_IO), "invalid VeloGraphX binary graph", "truncated graph file"
 * (VX_ERR_FORMAT). */
int vx_graph_load_binary(const char* path, int directed, vx_graph** out);

/* ---- Consolidation (include/velographx/storage/consolidation.hpp) -------
 * consolidate_to_csr_snapshot(source) :132-163: a new graph holding the
 * source's logical edges as a fresh CSR (compact, version 1, the source's
 * vertex count and direction); the source is not modified.  The rows are
 * merged and re-sorted on the device. */
int vx_graph_snapshot(vx_graph* g, vx_graph** out);
/* Device time (ns) of one pass over every live arc of the graph and the arcs
 * visited: the neighbour-iteration cost the consolidation signal compares
 * between a graph and its snapshot (evaluate_consolidation, :49-63, takes it
 * from the caller).  No reference counterpart. */
int vx_graph_scan_rows(vx_graph* g, uint64_t* arcs, double* ns);

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
/* Phase trace of the last incremental apply (29 entries): globaltimer ns at
 * the pre-batch kernel's entry, after its seeds, after its cascade; at the
 * post-batch kernel's entry, after the boundary distances, after its seeds,
 * after the relaxation (0 = phase not run); the work items pushed by the
 * cascade and by the relaxation; then, for the cascade and the relaxation,
 * the work-ring processing rounds, tickets, idle rounds, termination checks,
 * SM cycles spent processing (summed over blocks) and the longest round;
 * then the ns the last vx_bfs_apply_stream launch spent in each per-batch
 * phase (classify, removals, cascade, insertions, post-batch repair,
 * end-of-batch barrier), summed over its batches; then the batches of the
 * last apply or stream launch whose cascade, and whose relaxation, passed its
 * time budget (vx_bfs_set_handover) and handed over to a BFS.  No reference
 * counterpart (diagnostics). */
int vx_bfs_phase_trace(vx_bfs* b, uint64_t* out, size_t cap, size_t* n);
/* A stream of update batches applied in order, with the same result after
 * every batch as vx_bfs_apply on each: batch t is ops [offsets[t],
 * offsets[t+1]) of the host arrays (offsets[0] == 0, nbatches + 1 entries).
 * Undirected graphs: without stats, every batch but the last goes through
 * version-parallel windows (vx_bfs_set_stream_window): each window's batches
 * are answered together by one bit-parallel BFS over the window's graph
 * versions, then committed to the graph as one merged batch; the last batch
 * goes through the update launch, so that the repair counters after the call
 * are its own.  With stats, the whole stream runs in one persistent update
 * launch after one upload and one stream-wide canonicalisation.  Directed
 * graphs are applied batch by batch.  The distances after every batch, the
 * graph and its version count are the same on every route.  Optional host
 * outputs: digests[t] = vx_bfs_digest after batch t; stats[4t..4t+3] =
 * {last_deletion_candidates, last_affected_vertices,
 * last_used_full_recompute, reachable_count mod 2^32} after batch t.  The
 * reference applies batches one call at a time (bfs.hpp:29-98); this entry
 * has no counterpart there. */
int vx_bfs_apply_stream(vx_bfs* b, const uint32_t* src, const uint32_t* dst, const uint8_t* add,
                        const uint64_t* offsets, size_t nbatches, uint64_t* digests, uint32_t* stats);
/* Order-independent 64-bit digest of the current distances: the sum over v of
 * splitmix64((v << 32) | dist[v]) modulo 2^64 (splitmix64: add
 * 0x9E3779B97F4A7C15, then the two xor-shift-multiply rounds and the final
 * xor-shift of Steele et al.).  No reference counterpart (verification). */
int vx_bfs_digest(vx_bfs* b, uint64_t* out);
/* Device memory reserved ahead of an update stream, so that no batch
 * allocates (an allocation synchronises the device): batch buffers for
 * batches of up to max_batch_ops ops and delta-arena room for total_ops more
 * ops.  No reference counterpart. */
int vx_graph_reserve(vx_graph* g, size_t max_batch_ops, size_t total_ops);
/* The batched stream path's buffers for streams of up to `ops` ops in
 * `batches` batches, the largest max_batch_ops ops.  No reference counterpart. */
int vx_bfs_reserve_stream(vx_bfs* b, size_t ops, size_t batches, size_t max_batch_ops);
/* Direction switch (alpha, beta) and grid-expanded row length of the full BFS.
 * No reference counterpart: the reference BFS is top-down only. */
int vx_bfs_set_tuning(vx_bfs* b, float alpha, float beta, uint32_t large_row);
/* Autotuner of the full BFS: times a grid of 36 (alpha, beta, large_row)
 * candidates (alpha 4/14/40/120, beta 8/24/96, large_row 512/1024/4096) on a
 * full BFS from each of the k roots (all below the vertex count; each root
 * timed twice, the faster run kept), keeps the one with the smallest mean
 * time over the roots on b (every later recompute and fallback uses it) and
 * writes {alpha, beta, large_row, mean ms} to chosen (4 floats, may be
 * null).  b's own distances are recomputed afterwards.  No reference
 * counterpart: the reference BFS is top-down only. */
int vx_bfs_autotune(vx_bfs* b, const uint32_t* roots, size_t k, float* chosen);
int vx_bfs_get_tuning(vx_bfs* b, float* alpha, float* beta, uint32_t* large_row);
/* Algorithmic-byte accounting of the update launches (measurement only; off
 * by default, and every counted event costs an atomic when on).  on != 0
 * zeroes the counters and starts counting; vx_bfs_accounting copies the five
 * sums since then: {row arcs the repair scanned (cascade checks, expansions,
 * boundary rows, relaxations), vertices it visited (checks, ring items,
 * invalidations, heads of canonical arcs), delta-row entries the commit read
 * and wrote, canonical arcs, batches}.  No reference counterpart. */
int vx_bfs_set_accounting(vx_bfs* b, int on);
int vx_bfs_accounting(vx_bfs* b, uint64_t* out5);
/* Thread blocks of the persistent update launch (fused single batch and
 * batched stream): 0 (default) = one per SM; any count up to the co-resident
 * maximum (larger counts are clamped to it).  Fewer blocks shorten the grid
 * barriers and the work ring's polling.  Results are the same for every
 * value.  No reference counterpart. */
int vx_bfs_set_update_blocks(vx_bfs* b, uint32_t blocks);
/* Batches per version-parallel window of vx_bfs_apply_stream (1..256,
 * default 256; larger values are clamped to 256); 0 sends every batch through
 * the persistent update launch.  Same results for every value.  No reference
 * counterpart. */
int vx_bfs_set_stream_window(vx_bfs* b, uint32_t batches);
/* Level trace of the last version-parallel window's traversal: for each
 * level (up to 64) its start time in ns and its frontier size with bit 63
 * set for a pull level, then a closing timestamp; copies min(cap, *n)
 * values, *n = 2 * levels + 1 (0 before any window).  No reference
 * counterpart (diagnostics). */
int vx_bfs_window_trace(vx_bfs* b, uint64_t* out, size_t cap, size_t* n);
/* A version-parallel window's level pulls (bottom-up) when its frontier
 * holds more than frac * V vertices (default 0.02), or when its frontier's
 * rows hold more than a twelfth of the graph's arcs.  Same results for every
 * value.  No reference counterpart. */
int vx_bfs_set_window_pull_fraction(vx_bfs* b, float frac);
/* Time budget of the repair phases, in multiples of the last full BFS's time
 * (default 1): a deletion cascade that runs longer hands over to a BFS of the
 * graph without the batch's deletions (the affected set is the vertices
 * whose distance it raises), a relaxation that runs longer to a full BFS of
 * the post-batch graph; 0 hands over at a phase's first work-ring round, a
 * negative value never.  Same distances and counters for every value.  No
 * reference counterpart. */
int vx_bfs_set_handover(vx_bfs* b, float multiple);
/* fused != 0 (default): an undirected batch's commit and repair run in one
 * persistent launch after staging; 0: the per-phase path (a launch per commit
 * step and for each half of the repair) -- the plain baseline the batched
 * stream path is measured against.  Same results either way.  No reference
 * counterpart. */
int vx_bfs_set_fused(vx_bfs* b, int fused);

/* ---- BasicIncrementalComponents<DynamicGraph>
 *      (include/velographx/incremental/connected_components.hpp) ----------
 * Connected components of an undirected graph, maintained on the device.  The
 * partition after every batch equals the reference's; each component is
 * labelled by its smallest vertex id (the reference's labels are union-find
 * roots, which depend on its union order; its API compares them only for
 * equality). */
typedef struct vx_cc vx_cc;
/* BasicIncrementalComponents(Graph&) :19-25 -- VX_ERR_INVALID for a directed
 * graph; labels every vertex (last_repaired_vertices = vertex count). */
int vx_cc_create(vx_graph* g, vx_cc** out);
int vx_cc_destroy(vx_cc* c);
/* apply(const UpdateBatch&) :35-91 -- also applies the batch to the graph. */
int vx_cc_apply(vx_cc* c, const uint32_t* src, const uint32_t* dst, const uint8_t* add, size_t n);
/* component(v) :27-30 for every v: copies min(cap, len) labels, *n = len (the
 * vertex count when the labels were last updated). */
int vx_cc_labels(vx_cc* c, uint32_t* out, size_t cap, size_t* n);
/* last_repaired_vertices() :31-33 */
int vx_cc_last_repaired_vertices(vx_cc* c, uint64_t* out);

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
/* Level trace of the last run: for each level (up to 64) its start time in
 * ns and its frontier size with bit 63 set for a pull level, then a closing
 * timestamp; copies min(cap, *n) values, *n = 2 * levels + 1.  No reference
 * counterpart (diagnostics). */
int vx_mrbfs_level_trace(vx_mrbfs* m, uint64_t* out, size_t cap, size_t* n);
/* A level pulls (bottom-up) when its frontier holds more than frac * V
 * vertices (default 0.02), or when its frontier's rows hold more than a
 * twelfth of the graph's arcs (pushing an arc costs about twelve pulled
 * ones). */
int vx_mrbfs_set_pull_fraction(vx_mrbfs* m, float frac);
/* One-shot form: create, run, copy k*V distances into out (cap entries). */
int vx_multiroot_bfs(vx_graph* g, const uint32_t* roots, size_t k, uint32_t* out, size_t cap);

/* ---- Allocation-free full BFS ---------------------------------------------
 * No counterpart in the reference.  For callers that cannot call cudaMalloc
 * (their device memory is owned by another allocator, or they must not block
 * on the driver's allocator once running): the same direction-optimising BFS
 * as vx_bfs_recompute, on a CSR the caller holds in device memory (out- and
 * in-rows; pass the same arrays twice for an undirected graph), writing
 * `vertices` distances to d_dist.  Every column id must be below `vertices`
 * (the kernel indexes d_dist and the scratch bitmaps by column id and does not
 * check it) and rows must be free of duplicates; a source at or beyond
 * `vertices` gives all-unreachable and *reachable = 0, as in the reference.  All other working
 * memory is one file-scope device array (~8.5 MB per GPU that loads the
 * library, held until exit), so at most 262,144 vertices (larger counts
 * return VX_ERR_RANGE).  Calls share that array: calls that overlap on the
 * GPU race, so issue them one at a time per device.  The first call on a
 * device looks up the array's address on that device; make it before any
 * stream capture.  Runs on `stream` (a cudaStream_t, 0 for the legacy
 * stream), waits for completion, and returns the reachable count. */
int vx_bfs_csr_static(const uint64_t* d_out_offsets, const uint32_t* d_out_cols, const uint64_t* d_in_offsets,
                      const uint32_t* d_in_cols, uint32_t vertices, uint64_t arcs, uint32_t source, uint32_t* d_dist,
                      void* stream, uint64_t* reachable);

/* ---- Repair-vs-recompute selector -----------------------------------------
 * The reference chooses between IncrementalBFS::apply and graph.apply +
 * recompute in its benchmark harnesses (benchmarks/publication_policy_bfs.cpp:
 * 163-235).  Here: 16 batch features computed on the device, a 16-64-64-2 fp32
 * MLP (5,378 parameters) trained and evaluated by the library's own kernels,
 * and the reference's adaptive heuristic as the fallback. */
#define VX_SEL_FEATURES 16
#define VX_SEL_PARAMS 5378
typedef struct vx_selector vx_selector;
typedef struct vx_heuristic vx_heuristic;

/* Stage a host batch (canonicalise + classify, no mutation) and compute its
 * features; then run exactly one of vx_bfs_run_repair (IncrementalBFS::apply,
 * bfs.hpp:29-98) or vx_bfs_run_full (graph apply + recompute). */
int vx_bfs_stage(vx_bfs* b, const uint32_t* src, const uint32_t* dst, const uint8_t* add, size_t n);
int vx_bfs_staged_features(vx_bfs* b, float prev_affected_fraction, float* out16);
int vx_bfs_run_repair(vx_bfs* b);
int vx_bfs_run_full(vx_bfs* b);

int vx_selector_create(uint64_t seed, vx_selector** out);
int vx_selector_destroy(vx_selector* s);
/* Adam on standardised log-time targets: X n x 16, Y n x 2 (repair, full). */
int vx_selector_train(vx_selector* s, const float* X, const float* Y, size_t n, uint32_t epochs, uint32_t batch,
                      float lr, uint32_t seed, float* final_loss);
/* Mean-squared-error gradient of one minibatch (n <= 64) -> grad[5378]. */
int vx_selector_gradients(vx_selector* s, const float* X, const float* Y, size_t n, float* grad, float* loss);
int vx_selector_predict(vx_selector* s, const float* X, size_t n, float* Y);
int vx_selector_set_params(vx_selector* s, const float* params);
int vx_selector_get_params(vx_selector* s, float* params);

/* The reference's adaptive selector (publication_policy_bfs.cpp:163-235, EMA
 * updates :285-320), used as the fallback and as the baseline of regret. */
int vx_heuristic_create(size_t vertices, double initial_reachable_fraction, double initial_full_us,
                        vx_heuristic** out);
int vx_heuristic_destroy(vx_heuristic* h);
int vx_heuristic_decide(vx_heuristic* h, double update_fraction, double shallow_fraction, int* choose_full);
int vx_heuristic_observe(vx_heuristic* h, int observed_full, double execution_us, double affected_fraction);

#ifdef __cplusplus
}
#endif
#endif
