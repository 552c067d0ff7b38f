/*
 * CPU oracle for the dynamic-BFS path: a plain-C restatement of VeloGraphX's
 * DynamicGraph (include/velographx/storage/dynamic_graph.hpp) and
 * BasicIncrementalBFS (include/velographx/incremental/bfs.hpp).
 *
 * TEST INFRASTRUCTURE ONLY.  This library is the checker that the CUDA path is
 * compared against; the product never links, loads or calls it.  It is pinned
 * against the reference's own code (oracle/_ref, built from the reference
 * headers by oracle/Makefile) and against the golden vectors under
 * tests/golden/.
 *
 * All functions return 0 on success and a negative value on bad input, unless
 * they return a count.
 */
#ifndef VX_ORACLE_H
#define VX_ORACLE_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define VXO_UNREACHABLE 0xFFFFFFFFu

typedef struct vxo_graph vxo_graph;
typedef struct vxo_bfs vxo_bfs;

/* DynamicGraph(size_t vertices, bool directed)  dynamic_graph.hpp:481-487 */
vxo_graph* vxo_graph_create(size_t vertices, int directed);
void vxo_graph_destroy(vxo_graph* g);
size_t vxo_graph_vertex_count(const vxo_graph* g);
uint64_t vxo_graph_version(const vxo_graph* g);
int vxo_graph_directed(const vxo_graph* g);
/* bulk_load_edges  dynamic_graph.hpp:502-529; uv holds n (u,v) pairs */
int vxo_graph_bulk_load(vxo_graph* g, const uint32_t* uv, size_t n);
/* apply(UpdateBatch)  dynamic_graph.hpp:543-549 */
int vxo_graph_apply(vxo_graph* g, const uint32_t* src, const uint32_t* dst,
                    const uint8_t* add, size_t n);
/* neighbors / in_neighbors  dynamic_graph.hpp:551-557: writes up to cap ids,
 * returns the full row length. */
size_t vxo_graph_neighbors(const vxo_graph* g, uint32_t u, uint32_t* out, size_t cap);
size_t vxo_graph_in_neighbors(const vxo_graph* g, uint32_t v, uint32_t* out, size_t cap);
int vxo_graph_has_edge(const vxo_graph* g, uint32_t u, uint32_t v);
size_t vxo_graph_edge_count_directed(const vxo_graph* g);
size_t vxo_graph_delta_edge_count(const vxo_graph* g);
int vxo_graph_is_compact(const vxo_graph* g);
size_t vxo_graph_dirty_out_count(const vxo_graph* g);
size_t vxo_graph_dirty_in_count(const vxo_graph* g);
void vxo_graph_compact(vxo_graph* g);
/* ensure_vertex  dynamic_graph.hpp:493-500 */
void vxo_graph_ensure_vertex(vxo_graph* g, uint32_t v);
/* base_edge_count_directed  dynamic_graph.hpp:593-595 */
size_t vxo_graph_base_edge_count_directed(const vxo_graph* g);
/* compact_neighbors / compact_in_neighbors  dynamic_graph.hpp:573-581 */
size_t vxo_graph_compact_neighbors(const vxo_graph* g, uint32_t u, uint32_t* out, size_t cap);
size_t vxo_graph_compact_in_neighbors(const vxo_graph* g, uint32_t v, uint32_t* out, size_t cap);
int vxo_graph_maybe_compact(vxo_graph* g, double threshold);

/* BasicIncrementalBFS(Graph&, VertexId, double)  bfs.hpp:18-21 */
vxo_bfs* vxo_bfs_create(vxo_graph* g, uint32_t source, double deletion_fallback_fraction);
void vxo_bfs_destroy(vxo_bfs* b);
void vxo_bfs_recompute(vxo_bfs* b);
int vxo_bfs_apply(vxo_bfs* b, const uint32_t* src, const uint32_t* dst,
                  const uint8_t* add, size_t n);
/* copies min(len, cap) distances; returns len (== vertex count at last update) */
size_t vxo_bfs_distances(const vxo_bfs* b, uint32_t* out, size_t cap);
size_t vxo_bfs_reachable_count(const vxo_bfs* b);
size_t vxo_bfs_last_deletion_candidates(const vxo_bfs* b);
size_t vxo_bfs_last_affected_vertices(const vxo_bfs* b);
int vxo_bfs_last_used_full_recompute(const vxo_bfs* b);

/* Plain queue BFS on a caller-built CSR (src/algorithms.cpp:11-27 over
 * src/csr_graph.cpp:7-42).  Returns -1 if source >= V. */
int vxo_csr_bfs(const uint64_t* offsets, const uint32_t* cols, size_t V,
                uint32_t source, uint32_t* dist);

#ifdef __cplusplus
}
#endif
#endif
