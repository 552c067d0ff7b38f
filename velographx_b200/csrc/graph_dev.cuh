// Device building blocks of the graph commit, shared by the per-batch
// kernels (graph.cu) and the persistent stream kernel (bfs.cu): sorted-array
// search, warp merges of sorted lists into delta rows, dirty-row marking, the
// classification of one canonical arc and the tombstone update of one arc.
#pragma once

#include <cstdint>

#include "graph.cuh"

namespace vxh {
namespace gdev {

using vxb::DevAdj;
using vxb::kIdMask;
using vxb::kTomb;

__device__ __forceinline__ bool bsearch_u32(const uint32_t* a, uint32_t lo, uint32_t hi, uint32_t x) {
  const uint32_t p = vxb::lower_bound_u32(a, lo, hi, x);
  return p < hi && a[p] == x;
}

// Merge-path co-rank: number of A elements among the k smallest of A U B
// (both sorted, disjoint values).
__device__ __forceinline__ uint32_t corank(uint32_t k, const uint32_t* A, uint32_t nA, const uint32_t* B,
                                           uint32_t nB) {
  uint32_t lo = k > nB ? k - nB : 0u, hi = k < nA ? k : nA;
  while (lo < hi) {
    const uint32_t mid = (lo + hi) >> 1;
    if (A[mid] < B[k - mid - 1]) lo = mid + 1;
    else hi = mid;
  }
  return lo;
}

__device__ __forceinline__ uint32_t merged_at(uint32_t k, const uint32_t* A, uint32_t nA, const uint32_t* B,
                                              uint32_t nB) {
  const uint32_t i = corank(k, A, nA, B, nB), j = k - i;
  return (j >= nB || (i < nA && A[i] < B[j])) ? A[i] : B[j];
}

// Merges of a short list (nB <= 32, the usual run of one row in a batch):
// lane j holds B[j] and its final index slot_j = lower_bound(A, B[j]) + j,
// found once by parallel row searches.  Output k is then B[j] where
// k == slot_j, else A[k - t] with t the number of slots below k (a register
// scan over the lanes), so each 32 outputs cost one load instead of a
// co-rank search each.
__device__ __forceinline__ uint32_t short_merge_slot(const uint32_t* A, uint32_t nA, uint32_t nB, uint32_t bv) {
  const uint32_t lane = threadIdx.x & 31;
  return lane < nB ? vxb::lower_bound_u32(A, 0, nA, bv) + lane : 0xFFFFFFFFu;
}

// Whole warp: whether output k is one of B (then *bval) and, if not, the
// number of B slots below k.
__device__ __forceinline__ bool short_merge_pick(uint32_t k, uint32_t slot, uint32_t bv, uint32_t nB, uint32_t& t,
                                                 uint32_t& bval) {
  bool hit = false;
  t = 0;
  for (uint32_t j = 0; j < nB; ++j) {
    const uint32_t sj = __shfl_sync(0xFFFFFFFFu, slot, j);
    const uint32_t bj = __shfl_sync(0xFFFFFFFFu, bv, j);
    t += sj < k;
    if (sj == k) {
      hit = true;
      bval = bj;
    }
  }
  return hit;
}

// Warp-cooperative merge of sorted B[0..nB) into sorted A[0..nA) where A has
// room for nA + nB entries.  Output chunks are produced from the back; every
// output k only reads A at positions <= k, so no unread input is overwritten.
__device__ inline void warp_merge_inplace(uint32_t* A, uint32_t nA, const uint32_t* B, uint32_t nB) {
  const int lane = threadIdx.x & 31;
  const uint32_t total = nA + nB;
  if (nB <= 32) {
    const uint32_t bv = (uint32_t)lane < nB ? B[lane] : 0u;
    const uint32_t slot = short_merge_slot(A, nA, nB, bv);
    for (int64_t top = total; top > 0; top -= 32) {
      const int64_t k = top - 32 + lane;
      uint32_t t = 0, val = 0;
      const bool hit = short_merge_pick(k < 0 ? 0xFFFFFFFFu : (uint32_t)k, slot, bv, nB, t, val);
      if (k >= 0 && !hit) val = A[k - t];
      __syncwarp();
      if (k >= 0) A[k] = val;
      __syncwarp();
    }
    return;
  }
  for (int64_t top = total; top > 0; top -= 32) {
    const int64_t k = top - 32 + lane;
    uint32_t val = 0;
    if (k >= 0) val = merged_at((uint32_t)k, A, nA, B, nB);
    __syncwarp();
    if (k >= 0) A[k] = val;
    __syncwarp();
  }
}

__device__ inline void warp_merge_to(uint32_t* out, const uint32_t* A, uint32_t nA, const uint32_t* B, uint32_t nB) {
  const int lane = threadIdx.x & 31;
  if (nB <= 32) {
    const uint32_t bv = (uint32_t)lane < nB ? B[lane] : 0u;
    const uint32_t slot = short_merge_slot(A, nA, nB, bv);
    for (uint32_t k0 = 0; k0 < nA + nB; k0 += 32) {
      const uint32_t k = k0 + lane;
      uint32_t t = 0, val = 0;
      const bool hit = short_merge_pick(k, slot, bv, nB, t, val);
      if (k < nA + nB) out[k] = hit ? val : A[k - t];
    }
    return;
  }
  for (uint32_t k = lane; k < nA + nB; k += 32) out[k] = merged_at(k, A, nA, B, nB);
}

__device__ __forceinline__ void mark_dirty(uint32_t* dirty, uint32_t u, unsigned long long* counter) {
  const uint32_t bit = 1u << (u & 31);
  const uint32_t old = atomicOr(&dirty[u >> 5], bit);
  if (!(old & bit)) atomicAdd(counter, 1ull);
}

// Marks row u dirty; 1 when this call dirtied it (for a caller that counts
// newly dirtied rows itself, once per warp).
__device__ __forceinline__ uint32_t mark_dirty_count(uint32_t* dirty, uint32_t u) {
  const uint32_t bit = 1u << (u & 31);
  return (atomicOr(&dirty[u >> 5], bit) & bit) ? 0u : 1u;
}

// Pre-batch state of canonical arc (u, v) whose desired state is bit 0 of
// `add`: in the base CSR (position in fpos, live unless tombstoned) or in the
// row's sorted delta list; flags kFInBase / kFCur / kFChanged.
__device__ __forceinline__ uint8_t classify_arc(const DevAdj& a, uint32_t u, uint32_t v, uint8_t add,
                                                uint64_t& fpos) {
  uint8_t f = add & kFAdd;
  uint64_t b, e;
  vxb::base_range(a, u, b, e);
  const uint64_t p = vxb::lower_bound_masked(a.col, b, e, v);
  bool cur = false;
  if (p < e && (a.col[p] & kIdMask) == v) {
    f |= kFInBase;
    cur = !(a.col[p] & kTomb);
    fpos = p;
  } else {
    const uint2 r = a.drow[u];
    cur = bsearch_u32(a.darena, r.x, r.x + r.y, v);
    fpos = ~0ull;
  }
  if (cur) f |= kFCur;
  if (cur != ((f & kFAdd) != 0)) f |= kFChanged;
  return f;
}

// mode 0 tombstones a base arc the batch deletes, mode 1 revives one it
// re-adds; returns the change of the tombstone count and adds the row to
// `dirtied` when this call dirtied it (callers sum both per warp).
__device__ __forceinline__ long long tomb_arc(const DevAdj& a, uint32_t u, uint8_t f, uint64_t p, int mode,
                                              uint32_t& dirtied) {
  if (!(f & kFInBase) || !(f & kFChanged)) return 0;
  if (((f & kFAdd) != 0) != (mode == 1)) return 0;
  long long delta;
  if (f & kFAdd) {
    a.col[p] &= kIdMask;
    atomicSub(&a.tcnt[u], 1u);
    delta = -1;
  } else {
    a.col[p] |= kTomb;
    atomicAdd(&a.tcnt[u], 1u);
    delta = 1;
  }
  dirtied += mark_dirty_count(a.dirty, u);
  return delta;
}

}  // namespace gdev
}  // namespace vxh
