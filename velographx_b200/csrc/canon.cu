// Batch canonicalisation in one thread-block-cluster launch (sm_100a).
//
// A batch of n ops becomes m arcs (n directed, 2n undirected: (u,v) and
// (v,u) carry the same op).  Each arc is packed as
//     key = u << (b + sh) | v << sh | op_index << 1 | add        (sh = S + 1)
// and the cluster sorts the keys by their (u, v) bits with a stable LSD radix
// sort: arcs stay in op order inside equal (u, v) runs, so the last key of a
// run carries the batch's final op for that arc -- the state sequential
// application (dynamic_graph.hpp:543-549, 717-733) leaves.  Up to 8 CTAs of
// the cluster each hold kTile keys in shared memory; per 8-bit pass every CTA
// ranks its keys with warp-private histograms, reads the other CTAs' digit
// totals through distributed shared memory, and scatters every key straight
// into the shared memory of the CTA that owns its destination.  The epilogue
// keeps the last key of every run, compacts them across the cluster and
// hands the canonical arcs to the (wide) classification kernel -- the work of
// six separate launches.
#include <cooperative_groups.h>

#include "graph.cuh"

namespace cg = cooperative_groups;

namespace vxh {

namespace {

constexpr int kThreads = 1024;
constexpr int kDigits = 256;
constexpr int kMaxCluster = 8;     // portable cluster size (capacity of the largest tile)
constexpr int kMaxClusterNP = 16;  // non-portable size for the small tiles
// Tile shapes: 1 or 2 keys per thread spread small batches over up to 16
// CTAs (each pass is bound by its synchronisation, not by the keys), 4 keys
// per thread mid-size ones over 8, and 11 keys per thread hold the largest
// batch one cluster can take.
template <int ITEMS>
struct Tile {
  static constexpr int kItems = ITEMS;
  static constexpr int kTile = kThreads * ITEMS;
  static constexpr size_t kSmem = 2ull * kTile * 8 + (kThreads / 32) * kDigits * 4 + 3 * kDigits * 4 + 64 * 4;
  static_assert(kSmem <= 227 * 1024, "cluster tile exceeds shared memory");
};

__device__ __forceinline__ uint32_t lanemask_lt() { return vxb::lanemask_lt(); }

// Stable rank of the CTA's keys by one digit (warp w owns positions
// [w*kItems*32, (w+1)*kItems*32); see prims.cu for the same scheme).
template <int kItems>
__device__ void rank_keys(const uint32_t (&d)[kItems], uint32_t (&rank)[kItems], uint32_t* warp_hist,
                          uint32_t* total) {
  constexpr int W = kThreads / 32;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  uint32_t* h = warp_hist + warp * kDigits;
  for (int i = lane; i < kDigits; i += 32) h[i] = 0;
  __syncwarp();
#pragma unroll
  for (int r = 0; r < kItems; ++r) {
    const uint32_t peers = __match_any_sync(0xFFFFFFFFu, d[r]);
    const uint32_t base = h[d[r]];
    __syncwarp();
    if (lane == __ffs(peers) - 1) h[d[r]] = base + __popc(peers);
    __syncwarp();
    rank[r] = base + __popc(peers & lanemask_lt());
  }
  __syncthreads();
  for (int dd = threadIdx.x; dd < kDigits; dd += kThreads) {
    uint32_t s = 0;
    for (int w = 0; w < W; ++w) {
      const uint32_t c = warp_hist[w * kDigits + dd];
      warp_hist[w * kDigits + dd] = s;
      s += c;
    }
    total[dd] = s;
  }
  __syncthreads();
#pragma unroll
  for (int r = 0; r < kItems; ++r) rank[r] += h[d[r]];
}

// Exclusive scan of 256 values by warp 0 (8 per lane); in-place.
__device__ void scan256(uint32_t* v) {
  if (threadIdx.x < 32) {
    uint32_t loc[8], run = 0;
#pragma unroll
    for (int j = 0; j < 8; ++j) {
      loc[j] = v[threadIdx.x * 8 + j];
      run += loc[j];
    }
    uint32_t incl = run;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const uint32_t y = __shfl_up_sync(0xFFFFFFFFu, incl, o);
      if ((int)threadIdx.x >= o) incl += y;
    }
    uint32_t ex = incl - run;
#pragma unroll
    for (int j = 0; j < 8; ++j) {
      v[threadIdx.x * 8 + j] = ex;
      ex += loc[j];
    }
  }
}

template <int ITEMS>
__global__ void __launch_bounds__(kThreads, 1)
    canon_cluster_kernel(const uint32_t* src, const uint32_t* dst, const uint8_t* add, uint32_t n, int directed,
                         int b, int sh, uint32_t bound, int passes, uint32_t* fu, uint32_t* fv, uint8_t* ff,
                         GraphCounters* ctr) {
  constexpr int kItems = Tile<ITEMS>::kItems;
  constexpr int kTile = Tile<ITEMS>::kTile;
  cg::cluster_group cluster = cg::this_cluster();
  const uint32_t C = cluster.num_blocks();
  const uint32_t r = cluster.block_rank();
  extern __shared__ __align__(16) unsigned char smem[];
  uint64_t* A = reinterpret_cast<uint64_t*>(smem);
  uint64_t* B = A + kTile;
  uint32_t* warp_hist = reinterpret_cast<uint32_t*>(B + kTile);
  uint32_t* total = warp_hist + (kThreads / 32) * kDigits;
  uint32_t* offs = total + kDigits;
  uint32_t* alld = offs + kDigits;
  uint32_t* misc = alld + kDigits;  // [0..31] warp sums, [32] CTA run count, [33] CTA base
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const uint32_t m = directed ? n : 2 * n;

  // ---- expand ops into packed arc keys (global slot s = r * kTile + j)
  uint32_t mx = 0;
  for (uint32_t j = threadIdx.x; j < (uint32_t)kTile; j += kThreads) {
    const uint32_t s = r * kTile + j;
    uint64_t key = ~0ull;
    if (s < m) {
      const uint32_t i = directed ? s : (s >> 1);
      uint32_t u = src[i], v = dst[i];
      if (!directed && (s & 1)) {
        const uint32_t t = u;
        u = v;
        v = t;
      }
      bool ok = u != v;
      if (ok && (u >= bound || v >= bound)) {
        if ((s & 1) == 0 || directed) atomicOr(&ctr->err, vxb::kErrBadVertex);
        ok = false;
      }
      if (ok) {
        mx = max(mx, max(u, v) + 1);
        key = ((uint64_t)u << (b + sh)) | ((uint64_t)v << sh) | ((uint64_t)i << 1) | (add[i] ? 1ull : 0ull);
      }
    }
    A[j] = key;
  }
  mx = vxb::warp_max(mx);
  if (lane == 0 && mx) atomicMax(&ctr->max_vertex_plus1, mx);
  __syncthreads();

  // ---- stable LSD passes over the (u, v) bits
  const int pos0 = warp * kItems * 32 + lane;
  for (int p = 0; p < passes; ++p) {
    const int shift = sh + 8 * p;
    uint64_t k[kItems];
    uint32_t d[kItems], rank[kItems];
#pragma unroll
    for (int j = 0; j < kItems; ++j) {
      k[j] = A[pos0 + 32 * j];
      d[j] = (uint32_t)(k[j] >> shift) & 0xFFu;
    }
    rank_keys<kItems>(d, rank, warp_hist, total);
    cluster.sync();  // every CTA's digit totals are final
    if (threadIdx.x < kDigits) {
      const uint32_t dd = threadIdx.x;
      uint32_t before = 0, all = 0;
      for (uint32_t rr = 0; rr < C; ++rr) {
        const uint32_t t = rr == r ? total[dd] : cluster.map_shared_rank(total, rr)[dd];
        if (rr < r) before += t;
        all += t;
      }
      offs[dd] = before;
      alld[dd] = all;
    }
    __syncthreads();
    scan256(alld);
    __syncthreads();
#pragma unroll
    for (int j = 0; j < kItems; ++j) {
      const uint32_t g = alld[d[j]] + offs[d[j]] + rank[j];
      const uint32_t dest = g / kTile, loc = g % kTile;
      uint64_t* out = dest == r ? B : cluster.map_shared_rank(B, dest);
      out[loc] = k[j];
    }
    cluster.sync();  // all keys landed; totals of this pass no longer read
    uint64_t* t = A;
    A = B;
    B = t;
  }

  // ---- last key of every (u, v) run, compacted across the cluster
  const uint64_t vmask = ((uint64_t)1 << b) - 1;
  const uint32_t j0 = threadIdx.x * kItems;
  uint32_t cnt = 0;
  bool keep[kItems];
#pragma unroll
  for (int j = 0; j < kItems; ++j) {
    const uint32_t jj = j0 + j;
    const uint64_t key = A[jj];
    uint64_t next;
    if (jj + 1 < (uint32_t)kTile) next = A[jj + 1];
    else next = (r + 1 < C) ? cluster.map_shared_rank(A, r + 1)[0] : ~0ull;
    keep[j] = key != ~0ull && (next >> sh) != (key >> sh);
    cnt += keep[j];
  }
  uint32_t incl = cnt;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const uint32_t y = __shfl_up_sync(0xFFFFFFFFu, incl, o);
    if (lane >= o) incl += y;
  }
  if (lane == 31) misc[warp] = incl;
  __syncthreads();
  if (threadIdx.x < 32) {
    const uint32_t w = misc[threadIdx.x];
    uint32_t wi = w;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const uint32_t y = __shfl_up_sync(0xFFFFFFFFu, wi, o);
      if ((int)threadIdx.x >= o) wi += y;
    }
    misc[threadIdx.x] = wi - w;
    if (threadIdx.x == 31) misc[32] = wi;
  }
  cluster.sync();  // CTA totals visible cluster-wide
  if (threadIdx.x == 0) {
    uint32_t base = 0;
    for (uint32_t rr = 0; rr < r; ++rr) base += cluster.map_shared_rank(misc, rr)[32];
    misc[33] = base;
    if (r == C - 1) ctr->final_arcs = base + misc[32];
  }
  __syncthreads();
  uint32_t out = misc[33] + misc[warp] + incl - cnt;
#pragma unroll
  for (int j = 0; j < kItems; ++j) {
    if (!keep[j]) continue;
    const uint64_t key = A[j0 + j];
    const uint32_t u = (uint32_t)(key >> (b + sh)), v = (uint32_t)((key >> sh) & vmask);
    const uint8_t f = (uint8_t)(key & 1ull);
    fu[out] = u;
    fv[out] = v;
    ff[out] = f;
    ++out;
  }
  cluster.sync();  // keep shared memory alive until every remote read is done
}

}  // namespace

size_t canon_cluster_capacity() { return (size_t)kMaxCluster * Tile<11>::kTile; }

template <int ITEMS>
static int launch_canon(Graph* g, size_t n, size_t m, int b, int sh, uint32_t bound, bool* launched) {
  using T = Tile<ITEMS>;
  *launched = false;
  static bool attr = false;
  if (!attr) {
    VX_CUDA_TRY(cudaFuncSetAttribute(canon_cluster_kernel<ITEMS>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                     (int)T::kSmem));
    VX_CUDA_TRY(cudaFuncSetAttribute(canon_cluster_kernel<ITEMS>, cudaFuncAttributeNonPortableClusterSizeAllowed, 1));
    attr = true;
  }
  const unsigned C = (unsigned)((m + T::kTile - 1) / T::kTile);
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3(C);
  cfg.blockDim = dim3(kThreads);
  cfg.dynamicSmemBytes = T::kSmem;
  cfg.stream = g->stream;
  cudaLaunchAttribute at[1];
  at[0].id = cudaLaunchAttributeClusterDimension;
  at[0].val.clusterDim.x = C;
  at[0].val.clusterDim.y = 1;
  at[0].val.clusterDim.z = 1;
  cfg.attrs = at;
  cfg.numAttrs = 1;
  if (C > (unsigned)kMaxCluster) {  // a non-portable size: only where the device can place it
    static int fits[kMaxClusterNP + 1] = {};
    if (!fits[C]) {
      int clusters = 0;
      fits[C] = cudaOccupancyMaxActiveClusters(&clusters, canon_cluster_kernel<ITEMS>, &cfg) == cudaSuccess &&
                        clusters > 0
                    ? 1
                    : -1;
      cudaGetLastError();
    }
    if (fits[C] < 0) return 0;
  }
  const int passes = (2 * b + 7) / 8;
  BatchBuffers& B = g->batch;
  count_launch();
  VX_CUDA_TRY(cudaLaunchKernelEx(&cfg, canon_cluster_kernel<ITEMS>, B.in_src, B.in_dst, B.in_add, (uint32_t)n,
                                 (int)g->directed, b, sh, bound, passes, B.fu, B.fv, B.ff, g->ctr));
  *launched = true;
  return 0;
}

// Canonicalises the staged batch when it fits one cluster (*done = true);
// returns a negative status on a launch error.
int canon_cluster(Graph* g, size_t n, int b, uint32_t bound, bool* done) {
  *done = false;
  const size_t m = g->directed ? n : 2 * n;
  int sbits = 1;
  while (sbits < 32 && ((size_t)1 << sbits) < n) ++sbits;
  const int sh = sbits + 1;
  if (m == 0 || m > canon_cluster_capacity() || 2 * b + sh > 64) return 0;
  bool launched = false;
  int rc = 0;
  if (m <= (size_t)kMaxClusterNP * Tile<1>::kTile) rc = launch_canon<1>(g, n, m, b, sh, bound, &launched);
  if (!rc && !launched && m <= (size_t)kMaxClusterNP * Tile<2>::kTile)
    rc = launch_canon<2>(g, n, m, b, sh, bound, &launched);
  if (!rc && !launched && m <= (size_t)kMaxCluster * Tile<4>::kTile)
    rc = launch_canon<4>(g, n, m, b, sh, bound, &launched);
  if (!rc && !launched) rc = launch_canon<11>(g, n, m, b, sh, bound, &launched);
  *done = launched;
  return rc;
}

}  // namespace vxh
