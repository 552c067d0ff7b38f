// Whole-graph exports: the on-disk formats (the reference's
// include/velographx/io.hpp, include/velographx/io/binary_graph.hpp,
// src/io.cpp) and the consolidation snapshot (storage/consolidation.hpp).
#pragma once

#include "graph.cuh"

namespace vxh {

// Status codes of the file entry points (the C ABI's VX_ERR_FORMAT,
// VX_ERR_OVERFLOW and VX_ERR_IO).
constexpr int kErrFormat = -6;    // malformed file (std::runtime_error)
constexpr int kErrOverflow = -7;  // an id beyond uint32 (std::overflow_error)
constexpr int kErrIo = -8;        // cannot open, read or write (std::runtime_error)

// load_edge_list(path, directed) (src/io.cpp:23-53): a new graph holding the
// file's edges (bulk-loaded: self-loops and duplicates dropped, vertex count
// max id + 1).
int graph_load_edge_list(const char* path, bool directed, Graph** out);
// save_binary(g, path) (binary_graph.hpp:9-14).
int graph_save_binary(Graph* g, const char* path);
// load_binary(path, directed) (binary_graph.hpp:15-20): a new graph.
int graph_load_binary(const char* path, bool directed, Graph** out);
// consolidate_to_csr_snapshot(source) (consolidation.hpp:132-163): a new
// compact graph with the source's logical edges and vertex count.
int graph_snapshot(Graph* src, Graph** out);
// Device time of one pass over every live arc (the neighbour-iteration cost
// of the current layout) and the arcs it visited.
int graph_scan_rows(Graph* g, uint64_t* arcs, double* ns);

}  // namespace vxh
