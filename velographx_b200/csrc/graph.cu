// Device-resident dynamic graph: bulk load, batch apply, consolidation and
// row queries.  Semantics follow velographx::DynamicGraph
// (include/velographx/storage/dynamic_graph.hpp):
//   * bulk_load_edges (:502-529): self-loops dropped, undirected edges stored
//     as two arcs, duplicates removed, vertex count grown to max id + 1;
//   * apply (:543-549, :717-733): per arc the LAST op of the batch wins
//     (sequential per-op application has exactly that final state), self-loops
//     ignored, the vertex count grows to max(src,dst)+1 over every other op,
//     removals included; overlay cancellation = a tombstone cleared again or a
//     delta entry removed again;
//   * compact (:633-639): the overlay is merged into a fresh base CSR.
#include <algorithm>
#include <cstring>

#include "graph.cuh"
#include "graph_dev.cuh"

namespace vxh {

using vxb::DevAdj;
using vxb::DevGraph;
using vxb::kIdMask;
using vxb::kTomb;

namespace {

constexpr int kBlock = 256;

inline unsigned grid_for(size_t n, int block = kBlock) {
  size_t g = (n + block - 1) / block;
  if (g < 1) g = 1;
  const size_t cap = (size_t)sm_count() * 32;
  return (unsigned)std::min(g, cap);
}

inline int bits_for(size_t v) {  // bits to represent v - 1 (v >= 1)
  int b = 1;
  while (b < 32 && ((size_t)1 << b) < v) ++b;
  return b;
}

using gdev::bsearch_u32;
using gdev::mark_dirty;
using gdev::mark_dirty_count;
using gdev::warp_merge_inplace;
using gdev::warp_merge_to;

// ----------------------------------------------------------- bulk build --

__global__ void bulk_expand_kernel(const uint32_t* uv, size_t n, int directed, int b, uint64_t* keys) {
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
    const uint32_t u = uv[2 * i], v = uv[2 * i + 1];
    const bool ok = u != v;
    if (directed) {
      keys[i] = ok ? (((uint64_t)u << b) | v) : ~0ull;
    } else {
      keys[2 * i] = ok ? (((uint64_t)u << b) | v) : ~0ull;
      keys[2 * i + 1] = ok ? (((uint64_t)v << b) | u) : ~0ull;
    }
  }
}

__global__ void max_id_kernel(const uint32_t* uv, size_t n, uint32_t* out) {
  uint32_t m = 0;
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
    const uint32_t u = uv[2 * i], v = uv[2 * i + 1];
    if (u != v) m = max(m, max(u, v) + 1);
  }
  m = vxb::warp_max(m);
  if ((threadIdx.x & 31) == 0 && m) atomicMax(out, m);
}

__global__ void unique_flag_kernel(const uint64_t* keys, size_t n, uint32_t* flag) {
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
    const uint64_t k = keys[i];
    flag[i] = (k != ~0ull) && (i == 0 || keys[i - 1] != k);
  }
}

// Writes col[] of the unique arcs and the CSR offsets: off[w] for every w in
// (previous arc's row, u] is the index of the first arc of row u.  Invalid
// keys (~0) sort last, so the key before a first-of-run key is the previous
// unique arc.
__global__ void build_csr_kernel(const uint64_t* keys, const uint32_t* flag, const uint32_t* pos, size_t n,
                                 int b, uint64_t* off, uint32_t* col, const uint32_t* total,
                                 uint32_t* last_row) {
  const uint64_t mask = ((uint64_t)1 << b) - 1;
  const uint32_t A = *total;
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
    if (!flag[i]) continue;
    const uint64_t k = keys[i];
    const uint32_t u = (uint32_t)(k >> b), v = (uint32_t)(k & mask);
    const uint32_t p = pos[i];
    col[p] = v;
    const int64_t prev = i > 0 ? (int64_t)(keys[i - 1] >> b) : -1;
    for (int64_t w = prev + 1; w <= (int64_t)u; ++w) off[w] = p;
    if (p + 1 == A) *last_row = u + 1;
  }
}

// off[w] = A for every row after the last arc's row (last_row holds row+1, or
// 0 when there are no arcs).
__global__ void csr_tail_kernel(const uint32_t* total, const uint32_t* last_row, uint32_t V, uint64_t* off) {
  const uint32_t A = *total, first = *last_row;
  for (size_t w = first + blockIdx.x * (size_t)blockDim.x + threadIdx.x; w <= V; w += (size_t)gridDim.x * blockDim.x)
    off[w] = A;
}

// ---------------------------------------------------------- batch stage --

__global__ void expand_ops_kernel(const uint32_t* src, const uint32_t* dst, const uint8_t* add, size_t n,
                                  int directed, int b, uint32_t bound, uint64_t* keys, uint32_t* vals,
                                  vxh::GraphCounters* ctr) {
  uint32_t m = 0;
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
    const uint32_t u = src[i], v = dst[i];
    const uint32_t val = ((uint32_t)i << 1) | (add[i] ? 1u : 0u);
    bool ok = u != v;
    if (ok && (u >= bound || v >= bound)) {
      atomicOr(&ctr->err, vxb::kErrBadVertex);
      ok = false;
    }
    if (ok) m = max(m, max(u, v) + 1);
    if (directed) {
      keys[i] = ok ? (((uint64_t)u << b) | v) : ~0ull;
      vals[i] = val;
    } else {
      keys[2 * i] = ok ? (((uint64_t)u << b) | v) : ~0ull;
      keys[2 * i + 1] = ok ? (((uint64_t)v << b) | u) : ~0ull;
      vals[2 * i] = val;
      vals[2 * i + 1] = val;
    }
  }
  m = vxb::warp_max(m);
  if ((threadIdx.x & 31) == 0 && m) atomicMax(&ctr->max_vertex_plus1, m);
}

// Last element of every run of equal keys (stable sort keeps op order, so it
// carries the batch's final op for that arc).
__global__ void last_of_run_kernel(const uint64_t* keys, size_t m, uint32_t* flag) {
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < m; i += (size_t)gridDim.x * blockDim.x) {
    const uint64_t k = keys[i];
    flag[i] = (k != ~0ull) && (i + 1 == m || keys[i + 1] != k);
  }
}

__global__ void compact_final_kernel(const uint64_t* keys, const uint32_t* vals, const uint32_t* flag,
                                     const uint32_t* pos, size_t m, int b, uint32_t* fu, uint32_t* fv,
                                     uint8_t* ff) {
  const uint64_t mask = ((uint64_t)1 << b) - 1;
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < m; i += (size_t)gridDim.x * blockDim.x) {
    if (!flag[i]) continue;
    const uint32_t p = pos[i];
    fu[p] = (uint32_t)(keys[i] >> b);
    fv[p] = (uint32_t)(keys[i] & mask);
    ff[p] = (uint8_t)(vals[i] & 1u);
  }
}

// Pre-batch state of each canonical arc: base position / tombstone / delta.
__global__ void classify_kernel(DevAdj a, const uint32_t* fu, const uint32_t* fv, uint8_t* ff, uint64_t* fpos,
                                const uint32_t* count) {
  const uint32_t F = *count;
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < F; i += gridDim.x * blockDim.x)
    ff[i] = gdev::classify_arc(a, fu[i], fv[i], ff[i], fpos[i]);
}

// Reversed changed arcs (v, u) for the in-adjacency of directed graphs.
__global__ void reverse_keys_kernel(const uint32_t* fu, const uint32_t* fv, const uint8_t* ff,
                                    const uint32_t* count, size_t m, int b, uint64_t* keys, uint32_t* vals) {
  const uint32_t F = *count;
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < m; i += (size_t)gridDim.x * blockDim.x) {
    if (i < F && (ff[i] & vxh::kFChanged)) {
      keys[i] = ((uint64_t)fv[i] << b) | fu[i];
      vals[i] = ff[i] & vxh::kFAdd;
    } else {
      keys[i] = ~0ull;
      vals[i] = 0;
    }
  }
}

__global__ void count_valid_kernel(const uint64_t* keys, size_t m, uint32_t* flag) {
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < m; i += (size_t)gridDim.x * blockDim.x)
    flag[i] = keys[i] != ~0ull;
}

// --------------------------------------------------------- batch commit --

// mode 0: tombstone base arcs the batch deletes; mode 1: revive base arcs it re-adds.
__global__ void tomb_kernel(DevAdj a, const uint32_t* fu, const uint8_t* ff, const uint64_t* fpos,
                            const uint32_t* count, int mode, unsigned long long* tombs,
                            unsigned long long* dirty_rows) {
  const uint32_t F = *count;
  long long delta = 0;
  uint32_t dirtied = 0;
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < F; i += gridDim.x * blockDim.x)
    delta += gdev::tomb_arc(a, fu[i], ff[i], fpos[i], mode, dirtied);
  delta = vxb::warp_sum(delta);
  dirtied = vxb::warp_sum(dirtied);
  if ((threadIdx.x & 31) == 0 && delta) atomicAdd(tombs, (unsigned long long)delta);
  if ((threadIdx.x & 31) == 0 && dirtied) atomicAdd(dirty_rows, (unsigned long long)dirtied);
}

// mode 0: delta removals (state present -> absent, arc not in base)
// mode 1: delta insertions (state absent -> present, arc not in base)
__global__ void delta_flag_kernel(const uint8_t* ff, const uint32_t* count, size_t m, int mode, uint32_t* flag) {
  const uint32_t F = *count;
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < m; i += (size_t)gridDim.x * blockDim.x) {
    uint32_t x = 0;
    if (i < F) {
      const uint8_t f = ff[i];
      x = !(f & vxh::kFInBase) && (f & vxh::kFChanged) && (((f & vxh::kFAdd) != 0) == (mode == 1));
    }
    flag[i] = x;
  }
}

__global__ void compact_pairs_kernel(const uint32_t* fu, const uint32_t* fv, const uint32_t* flag,
                                     const uint32_t* pos, size_t m, uint32_t* lu, uint32_t* lv) {
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < m; i += (size_t)gridDim.x * blockDim.x) {
    if (flag[i]) {
      lu[pos[i]] = fu[i];
      lv[pos[i]] = fv[i];
    }
  }
}

__global__ void run_flag_kernel(const uint32_t* lu, const uint32_t* count, size_t m, uint32_t* flag) {
  const uint32_t n = *count;
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < m; i += (size_t)gridDim.x * blockDim.x)
    flag[i] = i < n && (i == 0 || lu[i] != lu[i - 1]);
}

__global__ void compact_index_kernel(const uint32_t* flag, const uint32_t* pos, size_t m, uint32_t* out) {
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < m; i += (size_t)gridDim.x * blockDim.x)
    if (flag[i]) out[pos[i]] = (uint32_t)i;
}

// One CTA builds a delta work list and its row runs (batches of at most
// kListMax canonical arcs): selected arcs are compacted in order with a block
// scan, then every entry whose row differs from its predecessor starts a run.
// Replaces the flag / scan / compact / run-flag / scan / compact launches.
constexpr int kListThreads = 1024;
constexpr int kListItems = 32;
constexpr size_t kListMax = (size_t)kListThreads * kListItems;

// Exclusive scan of the 32 per-warp counts of a 1024-thread block; every
// thread gets its warp's base, *total the block sum.
__device__ uint32_t warp_bases_1024(uint32_t warp_count, uint32_t* wsum, uint32_t* total) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  __syncthreads();
  if (lane == 0) wsum[warp] = warp_count;
  __syncthreads();
  if (warp == 0) {
    const uint32_t w = wsum[lane];
    uint32_t wi = w;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const uint32_t y = __shfl_up_sync(0xFFFFFFFFu, wi, o);
      if (lane >= o) wi += y;
    }
    wsum[lane] = wi - w;
    if (lane == 31) *total = wi;
  }
  __syncthreads();
  return wsum[warp];
}

// Round r takes items [r * 1024, (r + 1) * 1024), one per thread, so a list
// of F canonical arcs costs ceil(F / 1024) rounds of coalesced loads; ballots
// and a block scan of the warp counts give each selected item its position.
__global__ void __launch_bounds__(kListThreads) build_list_kernel(const uint32_t* fu, const uint32_t* fv,
                                                                   const uint8_t* ff, const uint32_t* count,
                                                                   int mode, uint32_t* lu, uint32_t* lv,
                                                                   uint32_t* runs, uint32_t* nlist,
                                                                   uint32_t* nruns) {
  __shared__ uint32_t wsum[32];
  __shared__ uint32_t total;
  const uint32_t F = *count;
  auto selected = [&](uint32_t i) {
    if (i >= F) return false;
    const uint8_t f = ff[i];
    return !(f & kFInBase) && (f & kFChanged) && (((f & kFAdd) != 0) == (mode == 1));
  };
  uint32_t n = 0;
  for (uint32_t r0 = 0; r0 < F; r0 += kListThreads) {
    const uint32_t i = r0 + threadIdx.x;
    const bool sel = selected(i);
    const uint32_t m = __ballot_sync(0xFFFFFFFFu, sel);
    const uint32_t wb = warp_bases_1024(__popc(m), wsum, &total);
    if (sel) {
      const uint32_t o = n + wb + __popc(m & vxb::lanemask_lt());
      lu[o] = fu[i];
      lv[o] = fv[i];
    }
    n += total;
  }
  if (threadIdx.x == 0) *nlist = n;
  __syncthreads();  // the compacted list is visible to the whole block
  uint32_t nr = 0;
  for (uint32_t r0 = 0; r0 < n; r0 += kListThreads) {
    const uint32_t k = r0 + threadIdx.x;
    const bool st = k < n && (k == 0 || lu[k] != lu[k - 1]);
    const uint32_t m = __ballot_sync(0xFFFFFFFFu, st);
    const uint32_t wb = warp_bases_1024(__popc(m), wsum, &total);
    if (st) runs[nr + wb + __popc(m & vxb::lanemask_lt())] = k;
    nr += total;
  }
  if (threadIdx.x == 0) *nruns = nr;
}

// One warp per row run: drop the run's arcs from the row's sorted delta list
// (forward in-place compaction: every kept entry moves to a lower index).
__global__ void delta_remove_kernel(DevAdj a, const uint32_t* lu, const uint32_t* lv, const uint32_t* runs,
                                    const uint32_t* nruns_p, const uint32_t* nlist_p,
                                    unsigned long long* live, unsigned long long* dirty_rows) {
  const uint32_t nruns = *nruns_p, nlist = *nlist_p;
  const int lane = threadIdx.x & 31;
  const uint32_t warps = gridDim.x * (blockDim.x >> 5);
  unsigned long long dropped = 0, dirtied = 0;
  for (uint32_t r = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5); r < nruns; r += warps) {
    const uint32_t s = runs[r], e = (r + 1 < nruns) ? runs[r + 1] : nlist;
    const uint32_t u = lu[s];
    const uint2 row = a.drow[u];
    uint32_t* A = a.darena + row.x;
    uint32_t written = 0;
    for (uint32_t base = 0; base < row.y; base += 32) {
      const uint32_t j = base + lane;
      const bool in = j < row.y;
      const uint32_t x = in ? A[j] : 0u;
      const bool keep = in && !bsearch_u32(lv, s, e, x);
      const uint32_t mask = __ballot_sync(0xFFFFFFFFu, keep);
      const uint32_t p = written + __popc(mask & vxb::lanemask_lt());
      __syncwarp();
      if (keep) A[p] = x;
      written += __popc(mask);
      __syncwarp();
    }
    if (lane == 0) {
      a.drow[u].y = written;
      dropped += row.y - written;
      dirtied += mark_dirty_count(a.dirty, u);
    }
  }
  // one update of each shared counter per warp (per row they serialised)
  if (lane == 0 && dropped) atomicAdd(live, (unsigned long long)(-(long long)dropped));
  if (lane == 0 && dirtied) atomicAdd(dirty_rows, dirtied);
}

// One warp per row run: merge the run's arcs into the row's delta list, in
// place when capacity allows, else into a fresh power-of-two block from the
// arena (capacity doubling, >= 8 entries).
__global__ void delta_insert_kernel(DevAdj a, size_t arena_cap, const uint32_t* lu, const uint32_t* lv,
                                    const uint32_t* runs, const uint32_t* nruns_p, const uint32_t* nlist_p,
                                    unsigned long long* arena_top, unsigned long long* live,
                                    unsigned long long* dirty_rows, uint32_t* err) {
  const uint32_t nruns = *nruns_p, nlist = *nlist_p;
  const int lane = threadIdx.x & 31;
  const uint32_t warps = gridDim.x * (blockDim.x >> 5);
  unsigned long long added = 0, dirtied = 0;
  for (uint32_t r = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5); r < nruns; r += warps) {
    const uint32_t s = runs[r], e = (r + 1 < nruns) ? runs[r + 1] : nlist;
    const uint32_t u = lu[s], nB = e - s;
    const uint2 row = a.drow[u];
    const uint32_t cap = a.dcap[u];
    const uint32_t cnew = row.y + nB;
    if (cnew <= cap) {
      warp_merge_inplace(a.darena + row.x, row.y, lv + s, nB);
      if (lane == 0) a.drow[u].y = cnew;
    } else {
      uint32_t ncap = 8;
      while (ncap < cnew) ncap <<= 1;
      unsigned long long off = 0;
      if (lane == 0) off = atomicAdd(arena_top, (unsigned long long)ncap);
      off = __shfl_sync(0xFFFFFFFFu, off, 0);
      if (off + ncap > arena_cap) {
        if (lane == 0) atomicOr(err, vxb::kErrArenaOverflow);
        continue;
      }
      warp_merge_to(a.darena + off, a.darena + row.x, row.y, lv + s, nB);
      if (lane == 0) {
        a.drow[u] = make_uint2((uint32_t)off, cnew);
        a.dcap[u] = ncap;
      }
    }
    if (lane == 0) {
      added += nB;
      dirtied += mark_dirty_count(a.dirty, u);
    }
  }
  // one update of each shared counter per warp (per row they serialised)
  if (lane == 0 && added) atomicAdd(live, added);
  if (lane == 0 && dirtied) atomicAdd(dirty_rows, dirtied);
}

// ---------------------------------------------------------- consolidate --

__global__ void live_degree_kernel(DevAdj a, uint32_t V, uint32_t* deg) {
  for (uint32_t u = blockIdx.x * blockDim.x + threadIdx.x; u < V; u += gridDim.x * blockDim.x) {
    uint64_t b, e;
    vxb::base_range(a, u, b, e);
    deg[u] = (uint32_t)(e - b) - a.tcnt[u] + a.drow[u].y;
  }
}

// One warp per row: copy the live base arcs, then merge the delta row in.
__global__ void consolidate_rows_kernel(DevAdj a, uint32_t V, const uint64_t* noff, uint32_t* ncol) {
  const int lane = threadIdx.x & 31;
  const uint32_t warps = gridDim.x * (blockDim.x >> 5);
  for (uint32_t u = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5); u < V; u += warps) {
    uint64_t b, e;
    vxb::base_range(a, u, b, e);
    uint32_t* out = ncol + noff[u];
    uint32_t written = 0;
    const bool tomb = a.tcnt[u] != 0;
    for (uint64_t base = b; base < e; base += 32) {
      const uint64_t j = base + lane;
      const uint32_t x = j < e ? a.col[j] : kTomb;
      const bool keep = !tomb ? (j < e) : (j < e && !(x & kTomb));
      const uint32_t mask = __ballot_sync(0xFFFFFFFFu, keep);
      if (keep) out[written + __popc(mask & vxb::lanemask_lt())] = x & kIdMask;
      written += __popc(mask);
    }
    const uint2 r = a.drow[u];
    if (r.y) {
      __syncwarp();
      warp_merge_inplace(out, written, a.darena + r.x, r.y);
    }
  }
}

__global__ void row_copy_kernel(DevAdj a, uint32_t u, uint32_t* out, uint32_t* n_out) {
  // single warp: live base arcs, then merge the delta row
  const int lane = threadIdx.x & 31;
  uint64_t b, e;
  vxb::base_range(a, u, b, e);
  uint32_t written = 0;
  for (uint64_t base = b; base < e; base += 32) {
    const uint64_t j = base + lane;
    const uint32_t x = j < e ? a.col[j] : kTomb;
    const bool keep = j < e && !(x & kTomb);
    const uint32_t mask = __ballot_sync(0xFFFFFFFFu, keep);
    if (keep) out[written + __popc(mask & vxb::lanemask_lt())] = x;
    written += __popc(mask);
  }
  const uint2 r = a.drow[u];
  __syncwarp();
  if (r.y) warp_merge_inplace(out, written, a.darena + r.x, r.y);
  if (lane == 0) *n_out = written + r.y;
}

__global__ void has_edge_kernel(DevAdj a, uint32_t u, uint32_t v, uint32_t* out) {
  uint64_t b, e;
  vxb::base_range(a, u, b, e);
  const uint64_t p = vxb::lower_bound_masked(a.col, b, e, v);
  uint32_t r;
  if (p < e && (a.col[p] & kIdMask) == v) {
    r = !(a.col[p] & kTomb);
  } else {
    const uint2 d = a.drow[u];
    r = bsearch_u32(a.darena, d.x, d.x + d.y, v);
  }
  *out = r;
}

__global__ void vx_transpose_keys_kernel(uint64_t* keys, size_t m, int b) {
  const uint64_t mask = ((uint64_t)1 << b) - 1;
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < m; i += (size_t)gridDim.x * blockDim.x) {
    const uint64_t k = keys[i];
    if (k != ~0ull) keys[i] = ((k & mask) << b) | (k >> b);
  }
}

template <typename T>
int grow_array(T** p, size_t old_n, size_t new_n, cudaStream_t s) {
  T* q = nullptr;
  if (cudaMalloc(&q, new_n * sizeof(T)) != cudaSuccess) {
    set_error("device allocation of %zu bytes failed", new_n * sizeof(T));
    return -4;
  }
  VX_CUDA_TRY(cudaMemsetAsync(q, 0, new_n * sizeof(T), s));
  if (*p && old_n) VX_CUDA_TRY(cudaMemcpyAsync(q, *p, old_n * sizeof(T), cudaMemcpyDeviceToDevice, s));
  if (*p) {
    VX_CUDA_TRY(cudaStreamSynchronize(s));
    cudaFree(*p);
  }
  *p = q;
  return 0;
}

template <typename T>
int alloc_array(T** p, size_t n) {
  if (*p) cudaFree(*p);
  *p = nullptr;
  if (cudaMalloc(p, std::max<size_t>(n, 1) * sizeof(T)) != cudaSuccess) {
    *p = nullptr;
    set_error("device allocation of %zu bytes failed", n * sizeof(T));
    return -4;
  }
  return 0;
}

int grow_arena(Adjacency& a, size_t need_entries, cudaStream_t s) {
  // grows 4x at a time: a growth copies the arena and synchronises the stream
  size_t ncap = std::max<size_t>(a.arena_cap * 4, std::max<size_t>(need_entries, 1u << 22));
  if (ncap >= 0xFFFFFFFFull) ncap = 0xFFFFFFFFull - 1;
  if (ncap < need_entries) {
    set_error("delta arena would exceed 2^32 entries");
    return -4;
  }
  return grow_array(&a.darena, a.arena_cap, ncap, s) ? -4 : (a.arena_cap = ncap, 0);
}

}  // namespace

// Any dirty row whose overlay (delta entries + tombstones) over
// max(8, base row length) reaches the threshold (dynamic_graph.hpp:774-783)?
__global__ void dense_dirty_kernel(DevAdj a, uint32_t V, double threshold, uint32_t* flag) {
  for (uint32_t u = blockIdx.x * blockDim.x + threadIdx.x; u < V; u += gridDim.x * blockDim.x) {
    if (!((a.dirty[u >> 5] >> (u & 31)) & 1u)) continue;
    const uint32_t overlay = a.drow[u].y + a.tcnt[u];
    if (overlay == 0) continue;
    uint64_t b, e;
    vxb::base_range(a, u, b, e);
    const double budget = (double)((e - b) > 8 ? (e - b) : 8);
    if ((double)overlay / budget >= threshold) *flag = 1u;
  }
}

// ------------------------------------------------------------ host side --

void Adjacency::free_all() {
  cudaFree(off);
  cudaFree(col);
  cudaFree(drow);
  cudaFree(dcap);
  cudaFree(tcnt);
  cudaFree(dirty);
  cudaFree(darena);
  *this = Adjacency();
}

int BatchBuffers::ensure(size_t ops) {
  if (ops <= cap) return 0;
  free_all();
  size_t c = std::max<size_t>(ops, 1024);
  const size_t arcs = 2 * c;
  int rc = 0;
  rc |= alloc_array(&src, c);
  rc |= alloc_array(&dst, c);
  rc |= alloc_array(&add, c);
  rc |= alloc_array(&keys, arcs);
  rc |= alloc_array(&keys_alt, arcs);
  rc |= alloc_array(&vals, arcs);
  rc |= alloc_array(&vals_alt, arcs);
  rc |= alloc_array(&flag, arcs);
  rc |= alloc_array(&pos, arcs);
  rc |= alloc_array(&fu, arcs);
  rc |= alloc_array(&fv, arcs);
  rc |= alloc_array(&ff, arcs);
  rc |= alloc_array(&fpos, arcs);
  rc |= alloc_array(&lu, arcs);
  rc |= alloc_array(&lv, arcs);
  rc |= alloc_array(&runs, arcs);
  rc |= alloc_array(&ru, arcs);
  rc |= alloc_array(&rv, arcs);
  rc |= alloc_array(&rf, arcs);
  rc |= alloc_array(&rpos, arcs);
  if (rc) {
    free_all();
    return -4;
  }
  cap = c;
  return 0;
}

void BatchBuffers::free_all() {
  void* ptrs[] = {src, dst, add, keys, keys_alt, vals, vals_alt, flag, pos, fu,
                  fv, ff, fpos, lu, lv, runs, ru, rv, rf, rpos};
  for (void* p : ptrs) cudaFree(p);
  *this = BatchBuffers();
}

DevGraph Graph::view() {
  DevGraph d;
  auto mk = [](Adjacency& a) {
    DevAdj x;
    x.off = a.off;
    x.col = a.col;
    x.Vb = a.Vb;
    x.drow = a.drow;
    x.dcap = a.dcap;
    x.darena = a.darena;
    x.tcnt = a.tcnt;
    x.dirty = a.dirty;
    return x;
  };
  d.out = mk(adj[0]);
  d.in = mk(in());
  d.V = (uint32_t)V;
  d.directed = directed;
  return d;
}

static DevAdj devadj(Adjacency& a) {
  DevAdj x;
  x.off = a.off;
  x.col = a.col;
  x.Vb = a.Vb;
  x.drow = a.drow;
  x.dcap = a.dcap;
  x.darena = a.darena;
  x.tcnt = a.tcnt;
  x.dirty = a.dirty;
  return x;
}

int graph_grow(Graph* g, size_t vertices) {
  if (vertices > vxb::kMaxVertices) {
    set_error("vertex count %zu exceeds the supported maximum %u", vertices, vxb::kMaxVertices);
    return -2;
  }
  if (vertices <= g->V) return 0;
  if (vertices > g->Vcap) {
    size_t c = std::max<size_t>(g->Vcap ? g->Vcap : 1024, 1024);
    while (c < vertices) c *= 2;
    c = std::min<size_t>(c, (size_t)vxb::kMaxVertices + 32);
    const int ndir = g->directed ? 2 : 1;
    for (int d = 0; d < ndir; ++d) {
      Adjacency& a = g->adj[d];
      if (grow_array(&a.drow, g->Vcap, c, g->stream) || grow_array(&a.dcap, g->Vcap, c, g->stream) ||
          grow_array(&a.tcnt, g->Vcap, c, g->stream) ||
          grow_array(&a.dirty, (g->Vcap + 31) / 32, (c + 31) / 32, g->stream))
        return -4;
    }
    g->Vcap = c;
  }
  g->V = vertices;
  return 0;
}

int graph_create(Graph** out, size_t vertices, bool directed) {
  Graph* g = new Graph();
  g->directed = directed;
  if (cudaStreamCreateWithFlags(&g->stream, cudaStreamNonBlocking) != cudaSuccess ||
      cudaMalloc(&g->ctr, sizeof(GraphCounters)) != cudaSuccess ||
      cudaMallocHost(&g->hctr, sizeof(GraphCounters)) != cudaSuccess ||
      cudaMallocHost(&g->pinned_scalar, 4096) != cudaSuccess) {
    set_error("CUDA initialisation failed: %s", cudaGetErrorString(cudaGetLastError()));
    graph_destroy(g);
    return -3;
  }
  cudaMemsetAsync(g->ctr, 0, sizeof(GraphCounters), g->stream);
  memset(g->hctr, 0, sizeof(GraphCounters));
  g->arena_limit_entries = (size_t)1 << 28;
  const int ndir = directed ? 2 : 1;
  for (int d = 0; d < ndir; ++d) {
    Adjacency& a = g->adj[d];
    if (alloc_array(&a.off, 1) || grow_arena(a, 1u << 20, g->stream)) {
      graph_destroy(g);
      return -4;
    }
    cudaMemsetAsync(a.off, 0, sizeof(uint64_t), g->stream);
    a.off_cap = 1;
  }
  if (int rc = graph_grow(g, vertices)) {
    graph_destroy(g);
    return rc;
  }
  *out = g;
  return 0;
}

void graph_destroy(Graph* g) {
  if (!g) return;
  if (g->stream) cudaStreamSynchronize(g->stream);
  g->adj[0].free_all();
  g->adj[1].free_all();
  g->batch.free_all();
  g->scratch.release();
  cudaFree(g->ctr);
  cudaFreeHost(g->hctr);
  cudaFreeHost(g->pinned_scalar);
  if (g->stream) cudaStreamDestroy(g->stream);
  delete g;
}

int graph_sync_counters(Graph* g) {
  VX_CUDA_TRY(cudaMemcpyAsync(g->hctr, g->ctr, sizeof(GraphCounters), cudaMemcpyDeviceToHost, g->stream));
  VX_CUDA_TRY(cudaStreamSynchronize(g->stream));
  for (int d = 0; d < 2; ++d) g->adj[d].arena_bound = std::max<uint64_t>(g->hctr->arena_top[d], 0);
  if (g->hctr->err) {
    const uint32_t e = g->hctr->err;
    set_error("device error word 0x%x (%s%s%s%s)", e, (e & vxb::kErrBadVertex) ? "vertex id out of bound " : "",
              (e & vxb::kErrArenaOverflow) ? "delta arena overflow " : "",
              (e & vxb::kErrBarrierTimeout) ? "grid barrier timeout " : "",
              (e & vxb::kErrLoopBound) ? "loop bound exceeded" : "");
    return -5;
  }
  return 0;
}

uint64_t graph_edge_count_directed(const Graph* g) {
  return g->adj[0].A + g->hctr->delta_live[0] - g->hctr->tombs[0];
}

// Builds adjacency a from sorted keys holding (u << b | v) arcs (duplicates
// and ~0 padding allowed).  flag/pos are scratch arrays of m entries.
static int build_adjacency(Graph* g, Adjacency& a, uint64_t* keys, size_t m, int b, uint32_t* flag,
                           uint32_t* pos) {
  cudaStream_t s = g->stream;
  uint32_t* total = reinterpret_cast<uint32_t*>(&g->ctr->final_arcs);
  uint32_t* last_row = reinterpret_cast<uint32_t*>(&g->ctr->rm_arcs);
  VX_CUDA_TRY(cudaMemsetAsync(last_row, 0, 4, s));
  vxh::count_launch();
  unique_flag_kernel<<<grid_for(m), kBlock, 0, s>>>(keys, m, flag);
  if (int rc = scan_exclusive_u32(flag, pos, m, total, g->scratch, s)) return rc;
  VX_CUDA_TRY(cudaMemcpyAsync(g->pinned_scalar, total, 4, cudaMemcpyDeviceToHost, s));
  VX_CUDA_TRY(cudaStreamSynchronize(s));
  const uint32_t A = *reinterpret_cast<uint32_t*>(g->pinned_scalar);
  if (alloc_array(&a.col, A) || alloc_array(&a.off, g->V + 1)) return -4;
  a.col_cap = A;
  a.off_cap = g->V + 1;
  vxh::count_launch();
  build_csr_kernel<<<grid_for(m), kBlock, 0, s>>>(keys, flag, pos, m, b, a.off, a.col, total, last_row);
  vxh::count_launch();
  csr_tail_kernel<<<grid_for(g->V + 1), kBlock, 0, s>>>(total, last_row, (uint32_t)g->V, a.off);
  VX_CUDA_TRY(cudaGetLastError());
  a.Vb = (uint32_t)g->V;
  a.A = A;
  VX_CUDA_TRY(cudaMemsetAsync(a.drow, 0, g->Vcap * sizeof(uint2), s));
  VX_CUDA_TRY(cudaMemsetAsync(a.dcap, 0, g->Vcap * sizeof(uint32_t), s));
  VX_CUDA_TRY(cudaMemsetAsync(a.tcnt, 0, g->Vcap * sizeof(uint32_t), s));
  VX_CUDA_TRY(cudaMemsetAsync(a.dirty, 0, ((g->Vcap + 31) / 32) * sizeof(uint32_t), s));
  a.arena_bound = 0;
  return 0;
}

int graph_bulk_load(Graph* g, const uint32_t* d_uv, size_t n) {
  cudaStream_t s = g->stream;
  // vertex growth: max id + 1 over non-self-loop edges
  uint32_t* mx = reinterpret_cast<uint32_t*>(&g->ctr->max_vertex_plus1);
  VX_CUDA_TRY(cudaMemsetAsync(mx, 0, 4, s));
  if (n) {
    vxh::count_launch();
    max_id_kernel<<<grid_for(n), kBlock, 0, s>>>(d_uv, n, mx);
  }
  VX_CUDA_TRY(cudaMemcpyAsync(g->pinned_scalar, mx, 4, cudaMemcpyDeviceToHost, s));
  VX_CUDA_TRY(cudaStreamSynchronize(s));
  const uint32_t need = *reinterpret_cast<uint32_t*>(g->pinned_scalar);
  if (int rc = graph_grow(g, std::max<size_t>(g->V, need))) return rc;
  const size_t m = g->directed ? n : 2 * n;
  const size_t mm = std::max<size_t>(m, 1);
  uint64_t *keys = nullptr, *alt = nullptr;
  uint32_t *flag = nullptr, *pos = nullptr;
  if (cudaMalloc(&keys, mm * 8) != cudaSuccess || cudaMalloc(&alt, mm * 8) != cudaSuccess ||
      cudaMalloc(&flag, mm * 4) != cudaSuccess || cudaMalloc(&pos, mm * 4) != cudaSuccess) {
    cudaFree(keys);
    cudaFree(alt);
    cudaFree(flag);
    set_error("bulk load: allocation for %zu arcs failed", m);
    return -4;
  }
  const int b = bits_for(std::max<size_t>(g->V, 2));
  int rc = 0;
  const int ndir = g->directed ? 2 : 1;
  for (int d = 0; d < ndir && !rc; ++d) {
    if (n) {
      vxh::count_launch();
      bulk_expand_kernel<<<grid_for(n), kBlock, 0, s>>>(d_uv, n, g->directed, b, keys);
      if (d == 1) {
        vxh::count_launch();
        vx_transpose_keys_kernel<<<grid_for(m), kBlock, 0, s>>>(keys, m, b);
      }
    }
    bool in_alt = false;
    rc = radix_sort_u64(keys, alt, nullptr, nullptr, m, 2 * b, &in_alt, g->scratch, s);
    if (!rc) rc = build_adjacency(g, g->adj[d], in_alt ? alt : keys, m, b, flag, pos);
  }
  cudaStreamSynchronize(s);
  cudaFree(keys);
  cudaFree(alt);
  cudaFree(flag);
  cudaFree(pos);
  if (rc) return rc;
  GraphCounters z;
  memset(&z, 0, sizeof(z));
  VX_CUDA_TRY(cudaMemcpyAsync(g->ctr, &z, sizeof(z), cudaMemcpyHostToDevice, s));
  VX_CUDA_TRY(cudaStreamSynchronize(s));
  memset(g->hctr, 0, sizeof(GraphCounters));
  ++g->version;
  return 0;
}

// Reserve arena room for `arcs` insertions in adjacency a (host-side bound:
// a row's blocks sum to < 8 entries per insertion ever made into it).
static int reserve_arena(Graph* g, Adjacency& a, size_t arcs, int* need_consolidate) {
  const uint64_t need = a.arena_bound + 8ull * arcs + 8;
  if (need <= a.arena_cap) return 0;
  if (need > g->arena_limit_entries || need >= 0xFFFFFFF0ull) {
    *need_consolidate = 1;
    return 0;
  }
  return grow_arena(a, need, g->stream);
}

// Arena room for a whole update stream whose batches insert at most
// `entries` delta entries in total (the sum of the per-batch bounds):
// consolidates first when the bound passes the limit; *fits = 0 when even
// the consolidated graph cannot take it in one go.
int graph_reserve_stream(Graph* g, uint64_t entries, int* fits) {
  *fits = 1;
  Adjacency& a = g->adj[0];
  if (a.arena_bound + entries + 8 > g->arena_limit_entries || a.arena_bound + entries + 8 >= 0xFFFFFFF0ull) {
    if (int rc = graph_consolidate(g)) return rc;
    if (a.arena_bound + entries + 8 > g->arena_limit_entries || a.arena_bound + entries + 8 >= 0xFFFFFFF0ull) {
      *fits = 0;
      return 0;
    }
  }
  if (a.arena_bound + entries + 8 > a.arena_cap) return grow_arena(a, a.arena_bound + entries + 8, g->stream);
  return 0;
}

static int scan_count(Graph* g, const uint32_t* flag, uint32_t* pos, size_t m, uint32_t* total) {
  return scan_exclusive_u32(flag, pos, m, total, g->scratch, g->stream);
}

int graph_prepare_batch(Graph* g, size_t n, size_t vertex_bound) {
  g->batch_ops = n;
  if (vertex_bound > vxb::kMaxVertices) {
    set_error("vertex id beyond the supported maximum");
    return -2;
  }
  const size_t m = g->directed ? n : 2 * n;
  // arena room (consolidate first if the bound passed the limit)
  int consolidate = 0;
  for (int d = 0; d < (g->directed ? 2 : 1); ++d)
    if (int rc = reserve_arena(g, g->adj[d], m, &consolidate)) return rc;
  if (consolidate) {
    if (int rc = graph_consolidate(g)) return rc;
    for (int d = 0; d < (g->directed ? 2 : 1); ++d)
      if (int rc = reserve_arena(g, g->adj[d], m, &consolidate)) return rc;
  }
  return graph_grow(g, std::max<size_t>(g->V, vertex_bound));
}

int graph_stage_batch(Graph* g, size_t n, size_t vertex_bound, bool classify) {
  cudaStream_t s = g->stream;
  BatchBuffers& B = g->batch;
  const size_t m = g->directed ? n : 2 * n;
  if (int rc = graph_prepare_batch(g, n, vertex_bound)) return rc;
  const int b = bits_for(std::max<size_t>(g->V, 2));
  if (n == 0) {  // a non-empty batch's staging sets these counts itself
    VX_CUDA_TRY(cudaMemsetAsync(&g->ctr->final_arcs, 0, 5 * sizeof(uint32_t), s));
    return 0;
  }
  bool done = false;
  if (int rc = canon_cluster(g, n, b, (uint32_t)g->V, &done)) return rc;
  if (done) {
    if (!classify) return 0;
    vxh::count_launch();
    classify_kernel<<<grid_for(m), kBlock, 0, s>>>(devadj(g->adj[0]), B.fu, B.fv, B.ff, B.fpos,
                                                    &g->ctr->final_arcs);
    VX_CUDA_TRY(cudaGetLastError());
    return 0;
  }
  vxh::count_launch();
  expand_ops_kernel<<<grid_for(n), kBlock, 0, s>>>(B.in_src, B.in_dst, B.in_add, n, g->directed, b, (uint32_t)g->V,
                                                    B.keys, B.vals, g->ctr);
  VX_CUDA_TRY(cudaGetLastError());
  bool in_alt = false;
  if (int rc = radix_sort_u64(B.keys, B.keys_alt, B.vals, B.vals_alt, m, 2 * b, &in_alt, g->scratch, s)) return rc;
  uint64_t* keys = in_alt ? B.keys_alt : B.keys;
  uint32_t* vals = in_alt ? B.vals_alt : B.vals;
  vxh::count_launch();
  last_of_run_kernel<<<grid_for(m), kBlock, 0, s>>>(keys, m, B.flag);
  if (int rc = scan_count(g, B.flag, B.pos, m, &g->ctr->final_arcs)) return rc;
  vxh::count_launch();
  compact_final_kernel<<<grid_for(m), kBlock, 0, s>>>(keys, vals, B.flag, B.pos, m, b, B.fu, B.fv, B.ff);
  VX_CUDA_TRY(cudaGetLastError());
  if (!classify) return 0;
  vxh::count_launch();
  classify_kernel<<<grid_for(m), kBlock, 0, s>>>(devadj(g->adj[0]), B.fu, B.fv, B.ff, B.fpos,
                                                  &g->ctr->final_arcs);
  VX_CUDA_TRY(cudaGetLastError());
  return 0;
}

// Applies one canonical arc list (u, v, flags, base positions) to adjacency a.
// Applies one half of a canonical arc list (u, v, flags, base positions) to
// adjacency a: mode 0 the deletions (tombstones, delta removals), mode 1 the
// insertions (revived tombstones, delta insertions).
static int commit_list(Graph* g, Adjacency& a, int dir, uint32_t* fu, uint32_t* fv, uint8_t* ff, uint64_t* fpos,
                       const uint32_t* count, size_t m, int mode) {
  cudaStream_t s = g->stream;
  BatchBuffers& B = g->batch;
  GraphCounters* c = g->ctr;
  DevAdj da = devadj(a);
  vxh::count_launch();
  tomb_kernel<<<grid_for(m), kBlock, 0, s>>>(da, fu, ff, fpos, count, mode, &c->tombs[dir], &c->dirty_rows[dir]);
  uint32_t* nlist = mode == 0 ? &c->rm_arcs : &c->ins_arcs;
  uint32_t* nruns = mode == 0 ? &c->rm_runs : &c->ins_runs;
  if (m <= kListMax) {
    vxh::count_launch();
    build_list_kernel<<<1, kListThreads, 0, s>>>(fu, fv, ff, count, mode, B.lu, B.lv, B.runs, nlist, nruns);
  } else {
    vxh::count_launch();
    delta_flag_kernel<<<grid_for(m), kBlock, 0, s>>>(ff, count, m, mode, B.flag);
    if (int rc = scan_count(g, B.flag, B.pos, m, nlist)) return rc;
    vxh::count_launch();
    compact_pairs_kernel<<<grid_for(m), kBlock, 0, s>>>(fu, fv, B.flag, B.pos, m, B.lu, B.lv);
    vxh::count_launch();
    run_flag_kernel<<<grid_for(m), kBlock, 0, s>>>(B.lu, nlist, m, B.flag);
    if (int rc = scan_count(g, B.flag, B.pos, m, nruns)) return rc;
    vxh::count_launch();
    compact_index_kernel<<<grid_for(m), kBlock, 0, s>>>(B.flag, B.pos, m, B.runs);
  }
  const unsigned wg = grid_for(m * 32, kBlock);
  vxh::count_launch();
  if (mode == 0)
    delta_remove_kernel<<<wg, kBlock, 0, s>>>(da, B.lu, B.lv, B.runs, nruns, nlist, &c->delta_live[dir],
                                              &c->dirty_rows[dir]);
  else
    delta_insert_kernel<<<wg, kBlock, 0, s>>>(da, a.arena_cap, B.lu, B.lv, B.runs, nruns, nlist,
                                              &c->arena_top[dir], &c->delta_live[dir], &c->dirty_rows[dir],
                                              &c->err);
  VX_CUDA_TRY(cudaGetLastError());
  if (mode == 1) a.arena_bound += 8ull * m + 8;
  return 0;
}

// Reversed changed arcs (v, u) of a directed batch, sorted by (v, u) and
// classified against the in-CSR (before either adjacency changes).
static int prepare_reverse(Graph* g, size_t m) {
  cudaStream_t s = g->stream;
  BatchBuffers& B = g->batch;
  const int b = bits_for(std::max<size_t>(g->V, 2));
  vxh::count_launch();
  reverse_keys_kernel<<<grid_for(m), kBlock, 0, s>>>(B.fu, B.fv, B.ff, &g->ctr->final_arcs, m, b, B.keys, B.vals);
  bool in_alt = false;
  if (int rc = radix_sort_u64(B.keys, B.keys_alt, B.vals, B.vals_alt, m, 2 * b, &in_alt, g->scratch, s)) return rc;
  uint64_t* keys = in_alt ? B.keys_alt : B.keys;
  uint32_t* vals = in_alt ? B.vals_alt : B.vals;
  vxh::count_launch();
  count_valid_kernel<<<grid_for(m), kBlock, 0, s>>>(keys, m, B.flag);
  if (int rc = scan_count(g, B.flag, B.pos, m, &g->ctr->rev_arcs)) return rc;
  vxh::count_launch();
  compact_final_kernel<<<grid_for(m), kBlock, 0, s>>>(keys, vals, B.flag, B.pos, m, b, B.ru, B.rv, B.rf);
  vxh::count_launch();
  classify_kernel<<<grid_for(m), kBlock, 0, s>>>(devadj(g->adj[1]), B.ru, B.rv, B.rf, B.rpos, &g->ctr->rev_arcs);
  VX_CUDA_TRY(cudaGetLastError());
  return 0;
}

static int commit_half(Graph* g, int mode) {
  const size_t n = g->batch_ops;
  if (n == 0) return 0;
  BatchBuffers& B = g->batch;
  const size_t m = g->directed ? n : 2 * n;
  if (mode == 0 && g->directed)
    if (int rc = prepare_reverse(g, m)) return rc;
  if (int rc = commit_list(g, g->adj[0], 0, B.fu, B.fv, B.ff, B.fpos, &g->ctr->final_arcs, m, mode)) return rc;
  if (g->directed)
    if (int rc = commit_list(g, g->adj[1], 1, B.ru, B.rv, B.rf, B.rpos, &g->ctr->rev_arcs, m, mode)) return rc;
  return 0;
}

int graph_commit_removals(Graph* g) { return commit_half(g, 0); }

int graph_commit_insertions(Graph* g) {
  if (int rc = commit_half(g, 1)) return rc;
  if (g->batch_ops) ++g->version;
  return 0;
}

int graph_commit_batch(Graph* g) {
  if (int rc = graph_commit_removals(g)) return rc;
  return graph_commit_insertions(g);
}

int graph_consolidate(Graph* g) {
  cudaStream_t s = g->stream;
  const int ndir = g->directed ? 2 : 1;
  const uint32_t V = (uint32_t)g->V;
  for (int d = 0; d < ndir; ++d) {
    Adjacency& a = g->adj[d];
    uint32_t* deg = nullptr;
    uint64_t *noff = nullptr, *total = nullptr;
    uint32_t* ncol = nullptr;
    if (alloc_array(&deg, V + 1) || alloc_array(&noff, V + 1) || alloc_array(&total, 1)) return -4;
    vxh::count_launch();
    live_degree_kernel<<<grid_for(V), kBlock, 0, s>>>(devadj(a), V, deg);
    if (int rc = scan_exclusive_u32_to_u64(deg, noff, V, total, g->scratch, s)) return rc;
    VX_CUDA_TRY(cudaMemcpyAsync(noff + V, total, 8, cudaMemcpyDeviceToDevice, s));
    VX_CUDA_TRY(cudaMemcpyAsync(g->pinned_scalar, total, 8, cudaMemcpyDeviceToHost, s));
    VX_CUDA_TRY(cudaStreamSynchronize(s));
    const uint64_t A = g->pinned_scalar[0];
    if (alloc_array(&ncol, A)) return -4;
    vxh::count_launch();
    consolidate_rows_kernel<<<grid_for((size_t)V * 32), kBlock, 0, s>>>(devadj(a), V, noff, ncol);
    VX_CUDA_TRY(cudaGetLastError());
    VX_CUDA_TRY(cudaStreamSynchronize(s));
    cudaFree(a.off);
    cudaFree(a.col);
    cudaFree(deg);
    cudaFree(total);
    a.off = noff;
    a.col = ncol;
    a.off_cap = V + 1;
    a.col_cap = A;
    a.Vb = V;
    a.A = A;
    VX_CUDA_TRY(cudaMemsetAsync(a.drow, 0, g->Vcap * sizeof(uint2), s));
    VX_CUDA_TRY(cudaMemsetAsync(a.dcap, 0, g->Vcap * sizeof(uint32_t), s));
    VX_CUDA_TRY(cudaMemsetAsync(a.tcnt, 0, g->Vcap * sizeof(uint32_t), s));
    VX_CUDA_TRY(cudaMemsetAsync(a.dirty, 0, ((g->Vcap + 31) / 32) * sizeof(uint32_t), s));
    VX_CUDA_TRY(cudaMemsetAsync(&g->ctr->arena_top[d], 0, 8, s));
    VX_CUDA_TRY(cudaMemsetAsync(&g->ctr->delta_live[d], 0, 8, s));
    VX_CUDA_TRY(cudaMemsetAsync(&g->ctr->tombs[d], 0, 8, s));
    VX_CUDA_TRY(cudaMemsetAsync(&g->ctr->dirty_rows[d], 0, 8, s));
    a.arena_bound = 0;
  }
  return 0;
}

int graph_maybe_compact(Graph* g, double threshold, int* compacted) {
  *compacted = 0;
  cudaStream_t s = g->stream;
  uint32_t* flag = &g->ctr->scratch32;
  VX_CUDA_TRY(cudaMemsetAsync(flag, 0, 4, s));
  for (int d = 0; d < (g->directed ? 2 : 1); ++d) {
    vxh::count_launch();
    dense_dirty_kernel<<<grid_for(g->V), kBlock, 0, s>>>(devadj(g->adj[d]), (uint32_t)g->V, threshold, flag);
  }
  VX_CUDA_TRY(cudaGetLastError());
  VX_CUDA_TRY(cudaMemcpyAsync(g->pinned_scalar, flag, 4, cudaMemcpyDeviceToHost, s));
  VX_CUDA_TRY(cudaStreamSynchronize(s));
  if (*reinterpret_cast<uint32_t*>(g->pinned_scalar) == 0) return 0;
  *compacted = 1;
  return graph_consolidate(g);
}

int graph_row(Graph* g, int dir, uint32_t u, uint32_t* host_out, size_t cap, size_t* n) {
  *n = 0;
  if (u >= g->V) return 0;
  Adjacency& a = dir == 0 ? g->adj[0] : g->in();
  // row length bound: base row + delta row
  cudaStream_t s = g->stream;
  uint64_t be[2] = {0, 0};
  if (u < a.Vb) VX_CUDA_TRY(cudaMemcpyAsync(be, a.off + u, 16, cudaMemcpyDeviceToHost, s));
  uint2 dr = make_uint2(0, 0);
  VX_CUDA_TRY(cudaMemcpyAsync(&dr, a.drow + u, sizeof(uint2), cudaMemcpyDeviceToHost, s));
  VX_CUDA_TRY(cudaStreamSynchronize(s));
  const size_t bound = (be[1] - be[0]) + dr.y + 1;
  uint32_t* buf = nullptr;
  if (cudaMalloc(&buf, (bound + 1) * 4) != cudaSuccess) {
    set_error("row buffer allocation failed");
    return -4;
  }
  vxh::count_launch();
  row_copy_kernel<<<1, 32, 0, s>>>(devadj(a), u, buf, buf + bound);
  uint32_t cnt = 0;
  cudaError_t e = cudaMemcpyAsync(&cnt, buf + bound, 4, cudaMemcpyDeviceToHost, s);
  if (e == cudaSuccess) e = cudaStreamSynchronize(s);
  if (e == cudaSuccess && host_out && cap)
    e = cudaMemcpy(host_out, buf, std::min<size_t>(cap, cnt) * 4, cudaMemcpyDeviceToHost);
  cudaFree(buf);
  if (e != cudaSuccess) {
    set_error("row copy failed: %s", cudaGetErrorString(e));
    return -3;
  }
  *n = cnt;
  return 0;
}

int graph_compact_row(Graph* g, int dir, uint32_t u, uint32_t* host_out, size_t cap, size_t* n) {
  *n = 0;
  Adjacency& a = dir == 0 ? g->adj[0] : g->in();
  if (u >= g->V || u >= a.Vb) return 0;  // vertices added after the base build have empty base rows
  cudaStream_t s = g->stream;
  uint64_t* be = g->pinned_scalar;
  VX_CUDA_TRY(cudaMemcpyAsync(be, a.off + u, 16, cudaMemcpyDeviceToHost, s));
  VX_CUDA_TRY(cudaStreamSynchronize(s));
  const size_t len = (size_t)(be[1] - be[0]);
  if (host_out && cap && len) {
    const size_t m = std::min(cap, len);
    VX_CUDA_TRY(cudaMemcpyAsync(host_out, a.col + be[0], m * 4, cudaMemcpyDeviceToHost, s));
    VX_CUDA_TRY(cudaStreamSynchronize(s));
    // a tombstoned base arc is still part of the compact row (the overlay,
    // not the base, records its deletion)
    for (size_t i = 0; i < m; ++i) host_out[i] &= vxb::kIdMask;
  }
  *n = len;
  return 0;
}

size_t graph_storage_bytes(const Graph* g) {
  size_t bytes = sizeof(GraphCounters);
  const int ndir = g->directed ? 2 : 1;
  for (int d = 0; d < ndir; ++d) {
    const Adjacency& a = g->adj[d];
    bytes += a.off_cap * sizeof(uint64_t) + a.col_cap * sizeof(uint32_t) + a.arena_cap * sizeof(uint32_t);
    bytes += g->Vcap * (sizeof(uint2) + 2 * sizeof(uint32_t)) + (g->Vcap + 31) / 32 * sizeof(uint32_t);
  }
  return bytes;
}

int graph_has_edge(Graph* g, uint32_t u, uint32_t v, int* out) {
  *out = 0;
  if (u >= g->V) return 0;
  uint32_t* r = &g->ctr->scratch32;
  vxh::count_launch();
  has_edge_kernel<<<1, 1, 0, g->stream>>>(devadj(g->adj[0]), u, v, r);
  VX_CUDA_TRY(cudaMemcpyAsync(g->pinned_scalar, r, 4, cudaMemcpyDeviceToHost, g->stream));
  VX_CUDA_TRY(cudaStreamSynchronize(g->stream));
  *out = *reinterpret_cast<uint32_t*>(g->pinned_scalar) != 0;
  return 0;
}

}  // namespace vxh

