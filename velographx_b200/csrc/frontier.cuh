// Device building blocks shared by the single-root and multi-root BFS
// kernels: grid-stride indices, row expansion (flattened small rows,
// warp-walked medium rows), a block-aggregated frontier queue, timers.
#pragma once

#include <cstdint>

#include "vx_common.cuh"

namespace vxh {
namespace frontier {

using vxb::DevAdj;
using vxb::kIdMask;
using vxb::kTomb;
using vxb::kUnreachable;

__device__ __forceinline__ uint32_t ld_cg(const uint32_t* p) { return __ldcg(p); }

__device__ __forceinline__ uint32_t gtid() { return blockIdx.x * blockDim.x + threadIdx.x; }
__device__ __forceinline__ uint32_t nthreads() { return gridDim.x * blockDim.x; }
__device__ __forceinline__ uint32_t gwarp() { return gtid() >> 5; }
__device__ __forceinline__ uint32_t nwarps() { return nthreads() >> 5; }

__device__ __forceinline__ bool test_bit(const uint32_t* bm, uint32_t v) { return (bm[v >> 5] >> (v & 31)) & 1u; }

__device__ __forceinline__ uint32_t degree_of(const DevAdj& a, uint32_t u) {
  uint64_t b, e;
  vxb::base_range(a, u, b, e);
  return (uint32_t)(e - b) + a.drow[u].y;
}

// The W per-vertex words at base (W = 1, 2, 4 or 8 consecutive words, base
// aligned to 4 * W bytes), one vector load per 16 bytes.
template <uint32_t W>
__device__ __forceinline__ void load_words(const uint32_t* base, uint32_t* out) {
  if constexpr (W == 1) {
    out[0] = base[0];
  } else if constexpr (W == 2) {
    const uint2 t = *reinterpret_cast<const uint2*>(base);
    out[0] = t.x;
    out[1] = t.y;
  } else {
#pragma unroll
    for (uint32_t h = 0; h < W / 4; ++h) {
      const uint4 t = reinterpret_cast<const uint4*>(base)[h];
      out[4 * h] = t.x;
      out[4 * h + 1] = t.y;
      out[4 * h + 2] = t.z;
      out[4 * h + 3] = t.w;
    }
  }
}

// The listed rows (lengths len[0, n)) of which this warp holds a slice, when
// row r is cut into slices of `slice` arcs and its slices are dealt to the
// warps starting at warp r (mod the warp count): f(r, len_r, first slice)
// for each, warp-uniformly.  The lengths are read 32 at a time, so a warp
// passes the rows it has no slice of without a round trip per row.
template <class F>
__device__ __forceinline__ void for_my_rows(const uint32_t* len, uint32_t n, uint32_t slice, F&& f) {
  const uint32_t lane = threadIdx.x & 31, nw = nwarps(), gw = gwarp();
  for (uint32_t r0 = 0; r0 < n; r0 += 32) {
    const uint32_t r = r0 + lane;
    const uint32_t l = r < n ? __ldcg(&len[r]) : 0u;
    const uint32_t s0 = (gw + nw - r % nw) % nw;
    uint32_t mine = __ballot_sync(0xFFFFFFFFu, r < n && s0 < (l + slice - 1) / slice);
    while (mine) {
      const uint32_t k = __ffs(mine) - 1;
      mine &= mine - 1;
      f(r0 + k, __shfl_sync(0xFFFFFFFFu, l, k), __shfl_sync(0xFFFFFFFFu, s0, k));
    }
  }
}

// --------------------------------------------------- row expansion core --

constexpr uint32_t FULL = 0xFFFFFFFFu;

// Flattened expansion of per-lane segments arr[start, start+len) across the
// warp (Merrill-style gather: warp scan of the lengths, then each lane finds
// the owner of element k by a 5-step shuffle search).  f(valid, x, owner) is
// called warp-uniformly.
template <class F>
__device__ __forceinline__ void gather_segments(const uint32_t* arr, uint64_t start, uint32_t len, uint32_t u,
                                                bool tombs, F& f) {
  const int lane = threadIdx.x & 31;
  uint32_t incl = len;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const uint32_t y = __shfl_up_sync(FULL, incl, o);
    if (lane >= o) incl += y;
  }
  const uint32_t excl = incl - len;
  const uint32_t total = __shfl_sync(FULL, incl, 31);
  for (uint32_t k0 = 0; k0 < total; k0 += 32) {
    const uint32_t k = k0 + lane;
    const bool ok = k < total;
    int owner = 0;
#pragma unroll
    for (int step = 16; step >= 1; step >>= 1) {
      const int cand = owner + step;
      const uint32_t ex = __shfl_sync(FULL, excl, cand & 31);
      if (cand < 32 && ex <= k) owner = cand;
    }
    const uint64_t st = __shfl_sync(FULL, start, owner);
    const uint32_t ex = __shfl_sync(FULL, excl, owner);
    const uint32_t ou = __shfl_sync(FULL, u, owner);
    const uint32_t x = ok ? arr[st + (k - ex)] : kTomb;
    f(ok && !(tombs && (x & kTomb)), x & kIdMask, ou);
  }
}

// Expands the rows of the (up to) 32 lane vertices: rows of >= 32 arcs are
// walked by the whole warp, shorter ones flattened across lanes.  Lanes pass
// an empty range (b == e, dr.y == 0) when they have no row.
template <class F>
__device__ __forceinline__ void expand_lanes(const DevAdj& a, uint32_t u, uint64_t b, uint64_t e, uint2 dr, F& f) {
  const int lane = threadIdx.x & 31;
  uint32_t blen = (uint32_t)(e - b), dlen = dr.y;
  uint32_t med = __ballot_sync(FULL, blen >= 32);
  while (med) {
    const int l = __ffs(med) - 1;
    med &= med - 1;
    const uint64_t bb = __shfl_sync(FULL, b, l), ee = __shfl_sync(FULL, e, l);
    const uint32_t uu = __shfl_sync(FULL, u, l);
    for (uint64_t j0 = bb; j0 < ee; j0 += 32) {
      const uint64_t j = j0 + lane;
      const uint32_t x = j < ee ? a.col[j] : kTomb;
      f(!(x & kTomb), x & kIdMask, uu);
    }
  }
  if (blen >= 32) blen = 0;
  gather_segments(a.col, b, blen, u, true, f);
  med = __ballot_sync(FULL, dlen >= 32);
  while (med) {
    const int l = __ffs(med) - 1;
    med &= med - 1;
    const uint32_t bb = __shfl_sync(FULL, dr.x, l), ee = bb + __shfl_sync(FULL, dr.y, l);
    const uint32_t uu = __shfl_sync(FULL, u, l);
    for (uint32_t j0 = bb; j0 < ee; j0 += 32) {
      const uint32_t j = j0 + lane;
      const bool ok = j < ee;
      f(ok, ok ? a.darena[j] : 0u, uu);
    }
  }
  if (dlen >= 32) dlen = 0;
  gather_segments(a.darena, (uint64_t)dr.x, dlen, u, false, f);
}

// The whole warp walks one row (all lanes pass the same u); f as above.
template <class F>
__device__ __forceinline__ void warp_row(const DevAdj& a, uint32_t u, F& f) {
  const int lane = threadIdx.x & 31;
  uint64_t b, e;
  vxb::base_range(a, u, b, e);
  for (uint64_t j0 = b; j0 < e; j0 += 32) {
    const uint64_t j = j0 + lane;
    const uint32_t x = j < e ? a.col[j] : kTomb;
    f(!(x & kTomb), x & kIdMask, u);
  }
  const uint2 dr = a.drow[u];
  for (uint32_t j0 = dr.x; j0 < dr.x + dr.y; j0 += 32) {
    const uint32_t j = j0 + lane;
    const bool ok = j < dr.x + dr.y;
    f(ok, ok ? a.darena[j] : 0u, u);
  }
}

__device__ __forceinline__ uint64_t globaltimer() {
  uint64_t t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}

// Block-aggregated frontier queue: warps reserve slots in shared memory
// (shared atomics); the block flushes with one global atomic per phase.  Warps
// that find the buffer full append straight to the global queue.
constexpr uint32_t kBlockQueueCap = 2048;
struct BlockQueue {
  uint32_t cnt;
  uint32_t gbase;
  uint32_t items[kBlockQueueCap];
};

// gbase0: the global counter's value that corresponds to gq[0] (a counter
// that is not reset between uses, as the bottom-up candidate lists use).
__device__ __forceinline__ void bq_push(BlockQueue& bq, bool pred, uint32_t v, uint32_t* gcnt, uint32_t* gq,
                                        uint32_t gbase0 = 0u) {
  const uint32_t mask = __ballot_sync(FULL, pred);
  if (!mask) return;
  const int lane = threadIdx.x & 31;
  const int leader = __ffs(mask) - 1;
  const uint32_t n = __popc(mask);
  uint32_t base = 0;
  if (lane == leader) base = atomicAdd(&bq.cnt, n);
  base = __shfl_sync(FULL, base, leader);
  const uint32_t r = __popc(mask & vxb::lanemask_lt());
  const uint32_t spill = base + n > kBlockQueueCap ? base + n - max(base, kBlockQueueCap) : 0u;
  uint32_t gb = 0;
  if (spill && lane == leader) gb = atomicAdd(gcnt, spill);
  gb = __shfl_sync(FULL, gb, leader);
  if (pred) {
    const uint32_t slot = base + r;
    if (slot < kBlockQueueCap) bq.items[slot] = v;
    else gq[(gb - gbase0) + (slot - max(base, kBlockQueueCap))] = v;
  }
}

// Block-uniform: moves the buffered entries to the global queue.
__device__ __forceinline__ void bq_flush(BlockQueue& bq, uint32_t* gcnt, uint32_t* gq, uint32_t gbase0 = 0u) {
  __syncthreads();
  const uint32_t n = min(bq.cnt, kBlockQueueCap);
  if (threadIdx.x == 0) bq.gbase = n ? atomicAdd(gcnt, n) : 0u;
  __syncthreads();
  for (uint32_t i = threadIdx.x; i < n; i += blockDim.x) gq[(bq.gbase - gbase0) + i] = bq.items[i];
  __syncthreads();
  if (threadIdx.x == 0) bq.cnt = 0;
  __syncthreads();
}

}  // namespace frontier
}  // namespace vxh
