// Connected components of an undirected device graph, maintained across
// update batches (the reference's BasicIncrementalComponents,
// include/velographx/incremental/connected_components.hpp:16-165).
//
// Labels live in device memory as a compressed union-find forest: label[v] is
// the root of v's set, and every union hooks the larger root under the smaller
// one (atomicCAS), so a root is always the smallest vertex id of its
// component.  A batch is applied as the reference applies it:
//   1. the batch is canonicalised and classified against the pre-batch graph
//      (the graph's own staging: last op per edge, present-before bit);
//   2. the components of the endpoints of every effective deletion are marked
//      affected, and their vertices counted (last_repaired_vertices);
//   3. the batch is committed to the graph;
//   4. affected vertices restart as singletons and are united along their
//      arcs to other affected vertices in the post-batch graph;
//   5. the final additions are united;
//   6. every label is compressed to its root.
// The partition equals the reference's after every batch.  The labels are the
// components' smallest ids, where the reference's are whichever union-find
// roots its union order left (the reference's tests compare labels only for
// equality).
#include <algorithm>
#include <cstring>

#include "components.cuh"
#include "frontier.cuh"
#include "graph_dev.cuh"

namespace vxh {

namespace {

constexpr int kCcThreads = 256;

unsigned cc_grid(uint64_t n) {
  return (unsigned)std::max<uint64_t>(1, std::min<uint64_t>((n + kCcThreads - 1) / kCcThreads, 148ull * 64));
}

__device__ __forceinline__ uint32_t cc_find(uint32_t* label, uint32_t x) {
  // path halving; parents only ever move to smaller ids of the same set
  uint32_t p = __ldcg(&label[x]);
  while (p != x) {
    const uint32_t gp = __ldcg(&label[p]);
    if (gp != p) __stcg(&label[x], gp);
    x = p;
    p = gp;
  }
  return x;
}

__device__ __forceinline__ void cc_union(uint32_t* label, uint32_t a, uint32_t b) {
  for (int guard = 0; guard < (1 << 20); ++guard) {
    a = cc_find(label, a);
    b = cc_find(label, b);
    if (a == b) return;
    if (a > b) {
      const uint32_t t = a;
      a = b;
      b = t;
    }
    if (atomicCAS(&label[b], b, a) == b) return;  // hook the larger root under the smaller
  }
}

__global__ void cc_identity_kernel(uint32_t* label, uint32_t lo, uint32_t hi) {
  for (uint32_t v = lo + blockIdx.x * blockDim.x + threadIdx.x; v < hi; v += gridDim.x * blockDim.x) label[v] = v;
}

// Unites u with every live neighbour v of u (v > u: each undirected edge once)
// that passes the filter: all of them (only_affected == 0), or those where
// both ends are affected.  One warp per row.
__global__ void cc_rows_kernel(vxb::DevAdj a, uint32_t V, uint32_t* label, const uint32_t* aff, int only_affected) {
  const uint32_t nw = (gridDim.x * blockDim.x) >> 5;
  for (uint32_t u = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; u < V; u += nw) {
    if (only_affected && !((aff[u >> 5] >> (u & 31)) & 1u)) continue;
    auto visit = [&](bool valid, uint32_t v, uint32_t) {
      if (!valid || v <= u || v >= V) return;
      if (only_affected && !((aff[v >> 5] >> (v & 31)) & 1u)) return;
      cc_union(label, u, v);
    };
    frontier::warp_row(a, u, visit);
  }
}

// Every label becomes its root.  The walk only reads: with path halving, a
// thread that read a vertex's old parent could store it back after the
// vertex's own thread had stored the root, leaving a label that is not a
// root.  Here each thread stores only its own label, and a concurrent reader
// sees either the old parent or the root, both ancestors.
__global__ void cc_compress_kernel(uint32_t* label, uint32_t V) {
  for (uint32_t v = blockIdx.x * blockDim.x + threadIdx.x; v < V; v += gridDim.x * blockDim.x) {
    uint32_t x = v, p = __ldcg(&label[v]);
    while (p != x) {
      x = p;
      p = __ldcg(&label[x]);
    }
    __stcg(&label[v], x);
  }
}

// Step 2: roots of the endpoints of effective deletions (present before the
// batch, final op a removal), among the pre-batch vertices.
__global__ void cc_mark_roots_kernel(const uint32_t* fu, const uint32_t* fv, const uint8_t* ff, const uint32_t* F,
                                     const uint32_t* label, uint32_t n_old, uint32_t* aroot, uint32_t* any) {
  const uint32_t nf = *F;
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < nf; i += gridDim.x * blockDim.x) {
    const uint8_t f = ff[i];
    if ((f & kFAdd) || !(f & kFCur)) continue;
    const uint32_t u = fu[i], v = fv[i];
    if (u >= n_old || v >= n_old) continue;
    const uint32_t ru = label[u], rv = label[v];
    atomicOr(&aroot[ru >> 5], 1u << (ru & 31));
    atomicOr(&aroot[rv >> 5], 1u << (rv & 31));
    *any = 1u;
  }
}

// Affected vertices (their root is marked) as a bitmap, counted.
__global__ void cc_mark_vertices_kernel(const uint32_t* label, uint32_t n_old, const uint32_t* aroot, uint32_t* aff,
                                        unsigned long long* count) {
  unsigned long long c = 0;
  for (uint32_t w = blockIdx.x * blockDim.x + threadIdx.x; w < (n_old + 31) / 32; w += gridDim.x * blockDim.x) {
    uint32_t bits = 0;
    for (uint32_t k = 0; k < 32; ++k) {
      const uint32_t v = w * 32 + k;
      if (v >= n_old) break;
      const uint32_t r = label[v];
      if ((aroot[r >> 5] >> (r & 31)) & 1u) bits |= 1u << k;
    }
    aff[w] = bits;
    c += __popc(bits);
  }
  c = vxb::warp_sum(c);
  if ((threadIdx.x & 31) == 0 && c) atomicAdd(count, c);
}

__global__ void cc_reset_affected_kernel(uint32_t* label, uint32_t n_old, const uint32_t* aff) {
  for (uint32_t v = blockIdx.x * blockDim.x + threadIdx.x; v < n_old; v += gridDim.x * blockDim.x)
    if ((aff[v >> 5] >> (v & 31)) & 1u) label[v] = v;
}

// Step 5: the final additions of the batch (their edges exist now).
__global__ void cc_union_adds_kernel(const uint32_t* fu, const uint32_t* fv, const uint8_t* ff, const uint32_t* F,
                                     uint32_t* label) {
  const uint32_t nf = *F;
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < nf; i += gridDim.x * blockDim.x)
    if ((ff[i] & kFAdd) && fu[i] < fv[i]) cc_union(label, fu[i], fv[i]);
}

int ensure_labels(Components* c, size_t V) {
  if (V <= c->cap && c->label) return 0;
  size_t cap = std::max<size_t>(c->cap ? c->cap : 1024, 1024);
  while (cap < V) cap *= 2;
  cudaStream_t s = c->g->stream;
  uint32_t *label = nullptr, *aroot = nullptr, *aff = nullptr;
  const size_t words = cap / 32 + 1;
  if (cudaMalloc(&label, cap * 4) != cudaSuccess || cudaMalloc(&aroot, words * 4) != cudaSuccess ||
      cudaMalloc(&aff, words * 4) != cudaSuccess) {
    cudaFree(label);
    cudaFree(aroot);
    set_error("components: allocation for %zu vertices failed", cap);
    return -4;
  }
  VX_CUDA_TRY(cudaMemsetAsync(aroot, 0, words * 4, s));
  VX_CUDA_TRY(cudaMemsetAsync(aff, 0, words * 4, s));
  if (c->label && c->n) VX_CUDA_TRY(cudaMemcpyAsync(label, c->label, c->n * 4, cudaMemcpyDeviceToDevice, s));
  VX_CUDA_TRY(cudaStreamSynchronize(s));
  cudaFree(c->label);
  cudaFree(c->aroot);
  cudaFree(c->aff);
  c->label = label;
  c->aroot = aroot;
  c->aff = aff;
  c->cap = cap;
  return 0;
}

}  // namespace

int cc_rebuild(Components* c) {
  Graph* g = c->g;
  const size_t V = g->V;
  if (int rc = ensure_labels(c, std::max<size_t>(V, 1))) return rc;
  cudaStream_t s = g->stream;
  if (V) {
    count_launch();
    cc_identity_kernel<<<cc_grid(V), kCcThreads, 0, s>>>(c->label, 0, (uint32_t)V);
    count_launch();
    cc_rows_kernel<<<cc_grid(32ull * V), kCcThreads, 0, s>>>(g->view().out, (uint32_t)V, c->label, nullptr, 0);
    count_launch();
    cc_compress_kernel<<<cc_grid(V), kCcThreads, 0, s>>>(c->label, (uint32_t)V);
    VX_CUDA_TRY(cudaGetLastError());
  }
  c->n = V;
  c->last_repaired = V;
  return 0;
}

int cc_create(Components** out, Graph* g) {
  if (g->directed) {
    set_error("IncrementalComponents requires an undirected graph; use an explicitly defined weak/strong "
              "connectivity algorithm for directed graphs");
    return -1;
  }
  Components* c = new Components();
  c->g = g;
  if (cudaMalloc(&c->ctr, 16) != cudaSuccess) {
    set_error("components: counter allocation failed");
    delete c;
    return -4;
  }
  if (int rc = cc_rebuild(c)) {
    cc_destroy(c);
    return rc;
  }
  *out = c;
  return 0;
}

void cc_destroy(Components* c) {
  if (!c) return;
  if (c->g && c->g->stream) cudaStreamSynchronize(c->g->stream);
  cudaFree(c->label);
  cudaFree(c->aroot);
  cudaFree(c->aff);
  cudaFree(c->ctr);
  delete c;
}

int cc_apply_staged(Components* c, size_t n, size_t vertex_bound) {
  Graph* g = c->g;
  cudaStream_t s = g->stream;
  c->last_repaired = 0;
  if (n == 0) return 0;  // an empty batch changes nothing (connected_components.hpp:32-35)
  const uint32_t n_old = (uint32_t)c->n;
  if (int rc = graph_stage_batch(g, n, vertex_bound)) return rc;
  BatchBuffers& B = g->batch;
  const uint32_t* F = &g->ctr->final_arcs;
  const uint32_t words_old = (n_old + 31) / 32;
  uint32_t* any = c->ctr;                                                   // effective deletion seen
  unsigned long long* count = reinterpret_cast<unsigned long long*>(c->ctr + 2);  // affected vertices
  VX_CUDA_TRY(cudaMemsetAsync(c->ctr, 0, 16, s));
  const uint64_t m = 2 * n;  // canonical arcs of an undirected batch, at most
  if (n_old) {
    count_launch();
    cc_mark_roots_kernel<<<cc_grid(m), kCcThreads, 0, s>>>(B.fu, B.fv, B.ff, F, c->label, n_old, c->aroot, any);
    count_launch();
    cc_mark_vertices_kernel<<<cc_grid(words_old), kCcThreads, 0, s>>>(c->label, n_old, c->aroot, c->aff, count);
  }
  uint32_t hc[4] = {0, 0, 0, 0};
  VX_CUDA_TRY(cudaMemcpyAsync(hc, c->ctr, 16, cudaMemcpyDeviceToHost, s));
  VX_CUDA_TRY(cudaStreamSynchronize(s));
  c->last_repaired = (size_t)hc[2] | ((size_t)hc[3] << 32);
  const bool affected = hc[0] != 0;
  if (int rc = graph_commit_batch(g)) return rc;
  const size_t V = g->V;
  if (int rc = ensure_labels(c, std::max<size_t>(V, 1))) return rc;
  if (V > n_old) {
    count_launch();
    cc_identity_kernel<<<cc_grid(V - n_old), kCcThreads, 0, s>>>(c->label, n_old, (uint32_t)V);
    VX_CUDA_TRY(cudaMemsetAsync(c->aff + words_old, 0, ((V + 31) / 32 + 1 - words_old) * 4, s));
  }
  if (affected) {
    count_launch();
    cc_reset_affected_kernel<<<cc_grid(n_old), kCcThreads, 0, s>>>(c->label, n_old, c->aff);
    count_launch();
    cc_rows_kernel<<<cc_grid(32ull * V), kCcThreads, 0, s>>>(g->view().out, (uint32_t)V, c->label, c->aff, 1);
  }
  count_launch();
  cc_union_adds_kernel<<<cc_grid(m), kCcThreads, 0, s>>>(B.fu, B.fv, B.ff, F, c->label);
  count_launch();
  cc_compress_kernel<<<cc_grid(V), kCcThreads, 0, s>>>(c->label, (uint32_t)V);
  // the marks start clear for the next batch
  VX_CUDA_TRY(cudaMemsetAsync(c->aroot, 0, ((c->cap / 32) + 1) * 4, s));
  VX_CUDA_TRY(cudaMemsetAsync(c->aff, 0, ((c->cap / 32) + 1) * 4, s));
  VX_CUDA_TRY(cudaGetLastError());
  c->n = V;
  return 0;
}

int cc_labels(Components* c, uint32_t* host_out, size_t cap, size_t* n) {
  *n = c->n;
  const size_t k = std::min(cap, c->n);
  if (host_out && k) VX_CUDA_TRY(cudaMemcpyAsync(host_out, c->label, k * 4, cudaMemcpyDeviceToHost, c->g->stream));
  VX_CUDA_TRY(cudaStreamSynchronize(c->g->stream));
  return 0;
}

}  // namespace vxh
