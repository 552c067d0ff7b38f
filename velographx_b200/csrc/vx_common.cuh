// Shared definitions for the B200 dynamic-BFS library (sm_100a).
//
// Device graph layout (one "adjacency" per direction; an undirected graph uses
// the same adjacency for out- and in-rows):
//
//   base CSR     off[Vb+1] (u64) + col[A] (u32).  Bit 31 of a column is the
//                tombstone: a base arc deleted since the last consolidation.
//                Rows are sorted by the low 31 bits.
//   delta rows   drow[v] = {offset, count} into darena, dcap[v] = capacity.
//                Each delta row is a sorted list of arcs present in the logical
//                graph but absent from the base CSR.
//
// The logical row of u is (base row minus tombstones) U (delta row), which is
// exactly the reference's base/patch row merged with its PackedDeltaStore
// overlay (dynamic_graph.hpp:659-681): an overlay "absent" entry is our
// tombstone, an overlay "present" entry is our delta entry.
#pragma once

#include <cstdint>
#include <cstdio>
#include <cuda_runtime.h>

namespace vxb {

constexpr uint32_t kUnreachable = 0xFFFFFFFFu;
constexpr uint32_t kTomb = 0x80000000u;
constexpr uint32_t kIdMask = 0x7FFFFFFFu;
constexpr uint32_t kMaxVertices = 0x7FFFFFFFu;  // ids must leave bit 31 free

// Device error word bits (reported as VX_ERR_DEVICE, with the word in the
// message, by the next synchronising call).
constexpr uint32_t kErrBarrierTimeout = 1u << 0;
constexpr uint32_t kErrLoopBound = 1u << 1;
constexpr uint32_t kErrArenaOverflow = 1u << 2;
constexpr uint32_t kErrBadVertex = 1u << 3;
constexpr uint32_t kErrDrainTimeout = 1u << 4;  // a repair work ring stopped draining

struct DevAdj {
  const uint64_t* off;  // [Vb + 1]
  uint32_t* col;        // [off[Vb]]
  uint32_t Vb;          // vertices covered by the base CSR
  uint2* drow;          // [Vcap] {offset, count}
  uint32_t* dcap;       // [Vcap]
  uint32_t* darena;     // delta arena
  uint32_t* tcnt;       // [Vcap] tombstones per row
  uint32_t* dirty;      // [Vcap/32] rows changed since the last consolidation
};

struct DevGraph {
  DevAdj out;
  DevAdj in;  // == out for undirected graphs
  uint32_t V;
  int directed;
};

__device__ __forceinline__ void base_range(const DevAdj& a, uint32_t u, uint64_t& b, uint64_t& e) {
  if (u < a.Vb) {
    b = a.off[u];
    e = a.off[u + 1];
  } else {
    b = e = 0;
  }
}

__device__ __forceinline__ uint32_t lane_id() { return threadIdx.x & 31u; }
__device__ __forceinline__ uint32_t lanemask_lt() {
  uint32_t m;
  asm volatile("mov.u32 %0, %%lanemask_lt;" : "=r"(m));
  return m;
}

template <typename T>
__device__ __forceinline__ T warp_sum(T v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xFFFFFFFFu, v, o);
  return v;
}

template <typename T>
__device__ __forceinline__ T warp_max(T v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    T w = __shfl_xor_sync(0xFFFFFFFFu, v, o);
    v = w > v ? w : v;
  }
  return v;
}

// splitmix64's finaliser (Steele, Lea and Flood, "Fast splittable
// pseudorandom number generators", OOPSLA 2014): the per-entry hash of the
// distance digests, sum over v of mix64(v << 32 | dist[v]) modulo 2^64.
__host__ __device__ __forceinline__ unsigned long long mix64(unsigned long long z) {
  z += 0x9E3779B97F4A7C15ull;
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
  return z ^ (z >> 31);
}

// Warp-aggregated append: every lane with `pred` gets a unique slot in
// list[0..*count).  Returns the lane's slot (or UINT32_MAX when !pred).
__device__ __forceinline__ uint32_t warp_append(bool pred, uint32_t* count) {
  const uint32_t mask = __ballot_sync(0xFFFFFFFFu, pred);
  if (mask == 0) return 0xFFFFFFFFu;
  const uint32_t leader = __ffs(mask) - 1;
  uint32_t base = 0;
  if (lane_id() == leader) base = atomicAdd(count, __popc(mask));
  base = __shfl_sync(0xFFFFFFFFu, base, leader);
  return pred ? base + __popc(mask & lanemask_lt()) : 0xFFFFFFFFu;
}

// Lower bounds in sorted rows, 8-ary: while more than 8 candidates remain, a
// step reads 7 evenly spaced pivots at once (one dependent round trip) and
// keeps the eighth of the range that holds the answer; the last <= 8 entries
// are read together and counted.  A hub row of 2^17 arcs takes 6 dependent
// round trips where a binary search takes 17.  key(v) is the compared value
// of an entry (the low 31 bits for base rows, whose bit 31 is the tombstone).
template <class I, class K>
__device__ __forceinline__ I lower_bound_8ary(const uint32_t* a, I lo, I hi, uint32_t x, K key) {
  while (hi - lo > 8) {
    const I step = (hi - lo) / 8;
    uint32_t pv[7];
#pragma unroll
    for (int k = 0; k < 7; ++k) pv[k] = key(a[lo + step * (I)(k + 1)]);
    uint32_t below = 0;  // pivots below x; they are sorted, so these are the first ones
#pragma unroll
    for (int k = 0; k < 7; ++k) below += pv[k] < x ? 1u : 0u;
    const I nhi = below < 7 ? lo + step * (I)(below + 1) : hi;
    lo = below ? lo + step * (I)below + 1 : lo;
    hi = nhi;
  }
  uint32_t tail[8];
#pragma unroll
  for (int k = 0; k < 8; ++k) tail[k] = lo + (I)k < hi ? key(a[lo + (I)k]) : 0xFFFFFFFFu;
  I n = 0;
#pragma unroll
  for (int k = 0; k < 8; ++k) n += (lo + (I)k < hi && tail[k] < x) ? (I)1 : (I)0;
  return lo + n;
}

__device__ __forceinline__ uint64_t lower_bound_masked(const uint32_t* a, uint64_t lo, uint64_t hi, uint32_t x) {
  return lower_bound_8ary<uint64_t>(a, lo, hi, x, [](uint32_t v) { return v & kIdMask; });
}

__device__ __forceinline__ uint32_t lower_bound_u32(const uint32_t* a, uint32_t lo, uint32_t hi, uint32_t x) {
  return lower_bound_8ary<uint32_t>(a, lo, hi, x, [](uint32_t v) { return v; });
}

// Grid-wide barrier for cooperative (co-resident) launches on one arrival
// word.  Block 0 adds 2^31 - (nblocks - 1) and every other block adds 1, so
// the word's low 31 bits return to zero and its top bit flips exactly when
// the last block of a barrier arrives; each block waits until the top bit
// differs from the one its own arrival returned.  The critical path after the
// last arrival is that one atomic and the pollers' next load, with no separate
// release step.  bar[0] is the word (kBarrierWords words, zeroed at setup:
// the low bits must be zero when a barrier starts).  The wait is bounded:
// after kBarrierSpinLimit polls a block records kErrBarrierTimeout in *err and
// proceeds, so a broken launch ends instead of hanging the device.
constexpr uint32_t kBarrierWords = 32;
constexpr uint32_t kBarrierSpinLimit = 1u << 22;

__device__ __forceinline__ void grid_barrier(uint32_t* bar, uint32_t nblocks, uint32_t* err) {
  __syncthreads();
  if (threadIdx.x == 0) {
    const uint32_t inc = blockIdx.x == 0 ? 0x80000000u - (nblocks - 1u) : 1u;
    __threadfence();
    const uint32_t old = atomicAdd(bar, inc);
    volatile uint32_t* v = bar;
    uint32_t spins = 0;
    while (((*v ^ old) & 0x80000000u) == 0u) {
      if (++spins > kBarrierSpinLimit) {
        atomicOr(err, kErrBarrierTimeout);
        break;
      }
      if (spins > 64) __nanosleep(spins < 1024 ? 32 : 256);
    }
    __threadfence();
  }
  __syncthreads();
}

}  // namespace vxb

// Host-side error plumbing (defined in capi.cu).
namespace vxh {
void set_error(const char* fmt, ...);
// Counts every kernel launch the library issues (read by vx_launch_count).
void count_launch();
}

#define VX_CUDA_TRY(expr)                                                          \
  do {                                                                             \
    cudaError_t _e = (expr);                                                       \
    if (_e != cudaSuccess) {                                                       \
      ::vxh::set_error("%s:%d: %s: %s", __FILE__, __LINE__, #expr, cudaGetErrorString(_e)); \
      return -3;                                                                   \
    }                                                                              \
  } while (0)
