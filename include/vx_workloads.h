/*
 * vx_workloads.h -- seeded synthetic inputs for benchmarks and tests
 * (exported by libvx_b200.so).  Not part of the reference-replacing boundary:
 * the reference generates its publication graphs in Python
 * (scripts/prepare_publication_datasets.py:80-111); these produce the same
 * distributions deterministically per (seed, edge index), multi-threaded.
 * Outputs are (u, v) pairs, row-major; self-loops and duplicates are kept (the
 * graph loader drops them, as bulk_load_edges does).
 */
#ifndef VX_WORKLOADS_H
#define VX_WORKLOADS_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* R-MAT: edge_factor << scale pairs over 2^scale vertices, initiator
 * (a, b, c, 1 - a - b - c). */
int vx_gen_rmat(uint32_t scale, uint32_t edge_factor, double a, double b, double c, uint64_t seed,
                uint32_t* uv_out);
/* n uniform random pairs over [0, vertices) (Erdos-Renyi G(n, m) with
 * replacement). */
int vx_gen_uniform(uint32_t vertices, uint64_t n, uint64_t seed, uint32_t* uv_out);
/* rows x cols 4-neighbour lattice (vertex r*cols+c) followed by `extra`
 * uniform random long-range pairs; writes vx_gen_grid_edge_count() pairs. */
int vx_gen_grid(uint32_t rows, uint32_t cols, uint64_t extra, uint64_t seed, uint32_t* uv_out);
uint64_t vx_gen_grid_edge_count(uint32_t rows, uint32_t cols, uint64_t extra);

#ifdef __cplusplus
}
#endif
#endif
