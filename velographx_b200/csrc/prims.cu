// Stable LSD radix sort and exclusive scans (see prims.cuh).
//
// Radix sort: 8-bit digits.  n <= kSmallN runs as one CTA that keeps the whole
// array in shared memory for every pass (one launch per sort -- the common case
// for update batches).  Larger inputs run three kernels per pass: per-tile
// digit histograms (digit-major so one exclusive scan yields every tile's
// global digit offset), the scan, and a stable scatter.  Stability inside a
// tile comes from ranking items in position order: round r covers positions
// [r*BLOCK, (r+1)*BLOCK); within a round, warps are ordered and lanes inside a
// warp are ranked with __match_any_sync.
#include "prims.cuh"
#include "vx_common.cuh"

namespace vxh {

namespace {

constexpr int kDigits = 256;

// ------------------------------------------------------------------ scan --

constexpr int kScanBlock = 256;
constexpr int kScanItems = 8;
constexpr int kScanTile = kScanBlock * kScanItems;

template <typename T>
__device__ T block_exclusive_scan(T v, T* warp_tot, T* block_total) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  T incl = v;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    T y = __shfl_up_sync(0xFFFFFFFFu, incl, o);
    if (lane >= o) incl += y;
  }
  if (lane == 31) warp_tot[warp] = incl;
  __syncthreads();
  if (warp == 0) {
    T w = lane < (kScanBlock / 32) ? warp_tot[lane] : T(0);
    T wi = w;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      T y = __shfl_up_sync(0xFFFFFFFFu, wi, o);
      if (lane >= o) wi += y;
    }
    if (lane < (kScanBlock / 32)) warp_tot[lane] = wi - w;
    if (lane == (kScanBlock / 32) - 1) *block_total = wi;
  }
  __syncthreads();
  return incl - v + warp_tot[warp];
}

template <typename In, typename Out>
__global__ void __launch_bounds__(kScanBlock) scan_reduce_kernel(const In* in, size_t n, Out* partial) {
  __shared__ Out red[kScanBlock / 32];
  const size_t base = (size_t)blockIdx.x * kScanTile;
  Out s = 0;
#pragma unroll
  for (int i = 0; i < kScanItems; ++i) {
    const size_t idx = base + (size_t)i * kScanBlock + threadIdx.x;
    if (idx < n) s += (Out)in[idx];
  }
  s = vxb::warp_sum(s);
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = s;
  __syncthreads();
  if (threadIdx.x == 0) {
    Out t = 0;
    for (int w = 0; w < kScanBlock / 32; ++w) t += red[w];
    partial[blockIdx.x] = t;
  }
}

// Exclusive scan of one tile plus an optional per-tile offset.
template <typename In, typename Out>
__global__ void __launch_bounds__(kScanBlock) scan_tile_kernel(const In* in, Out* out, size_t n,
                                                               const Out* tile_offset, Out* total) {
  __shared__ Out buf[kScanTile];
  __shared__ Out warp_tot[32];
  __shared__ Out btot;
  const size_t base = (size_t)blockIdx.x * kScanTile;
#pragma unroll
  for (int i = 0; i < kScanItems; ++i) {
    const int j = i * kScanBlock + threadIdx.x;
    const size_t idx = base + j;
    buf[j] = idx < n ? (Out)in[idx] : Out(0);
  }
  __syncthreads();
  Out local[kScanItems];
  Out s = 0;
#pragma unroll
  for (int i = 0; i < kScanItems; ++i) {
    local[i] = buf[threadIdx.x * kScanItems + i];
    s += local[i];
  }
  const Out off = tile_offset ? tile_offset[blockIdx.x] : Out(0);
  Out run = block_exclusive_scan<Out>(s, warp_tot, &btot) + off;
#pragma unroll
  for (int i = 0; i < kScanItems; ++i) {
    buf[threadIdx.x * kScanItems + i] = run;
    run += local[i];
  }
  __syncthreads();
#pragma unroll
  for (int i = 0; i < kScanItems; ++i) {
    const int j = i * kScanBlock + threadIdx.x;
    const size_t idx = base + j;
    if (idx < n) out[idx] = buf[j];
  }
  if (total && blockIdx.x == gridDim.x - 1 && threadIdx.x == 0) *total = off + btot;
}

size_t scan_levels_bytes(size_t n, size_t elem) {
  size_t bytes = 0;
  while (n > (size_t)kScanTile) {
    n = (n + kScanTile - 1) / kScanTile;
    bytes += ((n * elem + 255) / 256) * 256;
  }
  return bytes + 256;
}

template <typename In, typename Out>
int scan_impl(const In* in, Out* out, size_t n, Out* total, char* scratch, cudaStream_t s) {
  if (n == 0) {
    if (total) VX_CUDA_TRY(cudaMemsetAsync(total, 0, sizeof(Out), s));
    return 0;
  }
  const size_t nblk = (n + kScanTile - 1) / kScanTile;
  if (nblk == 1) {
    vxh::count_launch();
    scan_tile_kernel<In, Out><<<1, kScanBlock, 0, s>>>(in, out, n, nullptr, total);
    VX_CUDA_TRY(cudaGetLastError());
    return 0;
  }
  Out* partial = reinterpret_cast<Out*>(scratch);
  char* rest = scratch + ((nblk * sizeof(Out) + 255) / 256) * 256;
  vxh::count_launch();
  scan_reduce_kernel<In, Out><<<(unsigned)nblk, kScanBlock, 0, s>>>(in, n, partial);
  VX_CUDA_TRY(cudaGetLastError());
  int rc = scan_impl<Out, Out>(partial, partial, nblk, nullptr, rest, s);
  if (rc) return rc;
  vxh::count_launch();
  scan_tile_kernel<In, Out><<<(unsigned)nblk, kScanBlock, 0, s>>>(in, out, n, partial, total);
  VX_CUDA_TRY(cudaGetLastError());
  return 0;
}

// ------------------------------------------------------------ radix sort --

constexpr int kSmallBlock = 1024;
constexpr int kSmallItems = 8;
constexpr size_t kSmallN = (size_t)kSmallBlock * kSmallItems;
constexpr int kBigBlock = 256;
constexpr int kBigItems = 16;
constexpr int kBigTile = kBigBlock * kBigItems;

__device__ __forceinline__ uint32_t digit_of(uint64_t k, int shift) {
  return (uint32_t)(k >> shift) & 0xFFu;
}

// Stable block-wide digit ranking with warp-private histograms.
//
// Warp w owns the ITEMS*32 consecutive tile positions starting at
// w*ITEMS*32; round r of the warp holds positions w*ITEMS*32 + r*32 + lane.
// Each warp ranks its own items in position order (match_any peers + a
// private 256-bin histogram, no block barrier), then one pass over the
// histograms gives every warp its per-digit offset.  The returned rank of an
// item is its position among equal digits of the tile (earlier warps, earlier
// rounds, lower lanes first), and digit_total[d] the tile's count of digit d.
template <int BLOCK, int ITEMS>
__device__ void rank_tile(const uint32_t (&d)[ITEMS], uint32_t (&rank)[ITEMS], uint32_t* warp_hist /*[W][256]*/,
                          uint32_t* digit_total /*[256]*/) {
  constexpr int W = BLOCK / 32;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  uint32_t* h = warp_hist + warp * kDigits;
  for (int i = lane; i < kDigits; i += 32) h[i] = 0;
  __syncwarp();
#pragma unroll
  for (int r = 0; r < ITEMS; ++r) {
    const uint32_t peers = __match_any_sync(0xFFFFFFFFu, d[r]);
    const uint32_t base = h[d[r]];
    __syncwarp();
    if (lane == __ffs(peers) - 1) h[d[r]] = base + __popc(peers);
    __syncwarp();
    rank[r] = base + __popc(peers & vxb::lanemask_lt());
  }
  __syncthreads();
  for (int dd = threadIdx.x; dd < kDigits; dd += BLOCK) {
    uint32_t s = 0;
#pragma unroll 4
    for (int w = 0; w < W; ++w) {
      const uint32_t c = warp_hist[w * kDigits + dd];
      warp_hist[w * kDigits + dd] = s;
      s += c;
    }
    digit_total[dd] = s;
  }
  __syncthreads();
#pragma unroll
  for (int r = 0; r < ITEMS; ++r) rank[r] += h[d[r]];
}

// Whole sort inside one CTA.  Shared layout: keys[kSmallN] u64, vals[kSmallN]
// u32, warp_hist[32*256], digit_total[256], digit_base[256].
__global__ void __launch_bounds__(kSmallBlock) small_sort_kernel(uint64_t* keys, uint32_t* vals, size_t n,
                                                                  int passes) {
  extern __shared__ __align__(16) unsigned char smem[];
  uint64_t* sk = reinterpret_cast<uint64_t*>(smem);
  uint32_t* sv = reinterpret_cast<uint32_t*>(sk + kSmallN);
  uint32_t* warp_hist = sv + kSmallN;
  uint32_t* total = warp_hist + (kSmallBlock / 32) * kDigits;
  uint32_t* dbase = total + kDigits;
  for (size_t i = threadIdx.x; i < kSmallN; i += kSmallBlock) {
    sk[i] = i < n ? keys[i] : ~0ull;
    if (vals) sv[i] = i < n ? vals[i] : 0u;
  }
  __syncthreads();
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int pos0 = warp * kSmallItems * 32 + lane;
  for (int p = 0; p < passes; ++p) {
    const int shift = p * 8;
    uint64_t k[kSmallItems];
    uint32_t v[kSmallItems], d[kSmallItems], rank[kSmallItems];
#pragma unroll
    for (int r = 0; r < kSmallItems; ++r) {
      k[r] = sk[pos0 + r * 32];
      v[r] = vals ? sv[pos0 + r * 32] : 0u;
      d[r] = digit_of(k[r], shift);
    }
    rank_tile<kSmallBlock, kSmallItems>(d, rank, warp_hist, total);
    if (threadIdx.x < 32) {
      // exclusive scan of the 256 digit totals by one warp (8 per lane)
      uint32_t loc[8], run = 0;
#pragma unroll
      for (int j = 0; j < 8; ++j) {
        loc[j] = total[threadIdx.x * 8 + j];
        run += loc[j];
      }
      uint32_t incl = run;
#pragma unroll
      for (int o = 1; o < 32; o <<= 1) {
        const uint32_t y = __shfl_up_sync(0xFFFFFFFFu, incl, o);
        if (threadIdx.x >= o) incl += y;
      }
      uint32_t ex = incl - run;
#pragma unroll
      for (int j = 0; j < 8; ++j) {
        dbase[threadIdx.x * 8 + j] = ex;
        ex += loc[j];
      }
    }
    __syncthreads();
#pragma unroll
    for (int r = 0; r < kSmallItems; ++r) {
      const uint32_t dst = dbase[d[r]] + rank[r];
      sk[dst] = k[r];
      if (vals) sv[dst] = v[r];
    }
    __syncthreads();
  }
  for (size_t i = threadIdx.x; i < n; i += kSmallBlock) {
    keys[i] = sk[i];
    if (vals) vals[i] = sv[i];
  }
}

constexpr size_t kSmallSmem =
    kSmallN * 8 + kSmallN * 4 + (kSmallBlock / 32) * kDigits * 4 + kDigits * 4 * 2;
static_assert(kSmallSmem <= 227 * 1024, "small sort exceeds shared memory");

__global__ void __launch_bounds__(kBigBlock) radix_hist_kernel(const uint64_t* keys, size_t n, int shift,
                                                               uint32_t* hist, uint32_t nblk) {
  __shared__ uint32_t h[kDigits];
  for (int i = threadIdx.x; i < kDigits; i += kBigBlock) h[i] = 0;
  __syncthreads();
  const size_t base = (size_t)blockIdx.x * kBigTile;
#pragma unroll 4
  for (int r = 0; r < kBigItems; ++r) {
    const size_t idx = base + (size_t)r * kBigBlock + threadIdx.x;
    if (idx < n) atomicAdd(&h[digit_of(keys[idx], shift)], 1u);
  }
  __syncthreads();
  for (int i = threadIdx.x; i < kDigits; i += kBigBlock) hist[(size_t)i * nblk + blockIdx.x] = h[i];
}

__global__ void __launch_bounds__(kBigBlock) radix_scatter_kernel(const uint64_t* keys, const uint32_t* vals,
                                                                  uint64_t* keys_out, uint32_t* vals_out,
                                                                  size_t n, int shift,
                                                                  const uint32_t* offsets, uint32_t nblk) {
  __shared__ uint32_t warp_hist[(kBigBlock / 32) * kDigits];
  __shared__ uint32_t total[kDigits];
  __shared__ uint32_t gbase[kDigits];
  for (int i = threadIdx.x; i < kDigits; i += kBigBlock) gbase[i] = offsets[(size_t)i * nblk + blockIdx.x];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const size_t pos0 = (size_t)blockIdx.x * kBigTile + warp * kBigItems * 32 + lane;
  uint64_t k[kBigItems];
  uint32_t v[kBigItems], d[kBigItems], rank[kBigItems];
#pragma unroll
  for (int r = 0; r < kBigItems; ++r) {
    const size_t idx = pos0 + r * 32;
    const bool valid = idx < n;
    k[r] = valid ? keys[idx] : ~0ull;
    v[r] = (valid && vals) ? vals[idx] : 0u;
    d[r] = valid ? digit_of(k[r], shift) : 255u;
  }
  rank_tile<kBigBlock, kBigItems>(d, rank, warp_hist, total);
#pragma unroll
  for (int r = 0; r < kBigItems; ++r) {
    if (pos0 + r * 32 < n) {
      const uint32_t dst = gbase[d[r]] + rank[r];
      keys_out[dst] = k[r];
      if (vals) vals_out[dst] = v[r];
    }
  }
}

}  // namespace

int Scratch::ensure(size_t bytes) {
  if (bytes <= cap) return 0;
  release();
  size_t c = bytes < (1u << 20) ? (1u << 20) : bytes + bytes / 4;
  if (cudaMalloc(&ptr, c) != cudaSuccess) {
    ptr = nullptr;
    cap = 0;
    set_error("scratch allocation of %zu bytes failed", c);
    return -4;
  }
  cap = c;
  return 0;
}

void Scratch::release() {
  if (ptr) cudaFree(ptr);
  ptr = nullptr;
  cap = 0;
}

int sm_count() {
  static int cached = 0;
  if (!cached) {
    int dev = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&cached, cudaDevAttrMultiProcessorCount, dev);
    if (cached <= 0) cached = 148;
  }
  return cached;
}

size_t scan_scratch_bytes(size_t n) { return scan_levels_bytes(n, 8) + 512; }

int scan_exclusive_u32_to_u64(const uint32_t* in, uint64_t* out, size_t n, uint64_t* total_dev,
                              Scratch& scratch, cudaStream_t s) {
  if (int rc = scratch.ensure(scan_scratch_bytes(n))) return rc;
  return scan_impl<uint32_t, uint64_t>(in, out, n, total_dev, static_cast<char*>(scratch.ptr), s);
}

int scan_exclusive_u32(const uint32_t* in, uint32_t* out, size_t n, uint32_t* total_dev, Scratch& scratch,
                       cudaStream_t s) {
  if (int rc = scratch.ensure(scan_scratch_bytes(n))) return rc;
  return scan_impl<uint32_t, uint32_t>(in, out, n, total_dev, static_cast<char*>(scratch.ptr), s);
}

size_t radix_sort_scratch_bytes(size_t n) {
  const size_t nblk = (n + kBigTile - 1) / kBigTile;
  const size_t hist = ((nblk * kDigits * 4 + 255) / 256) * 256;
  return hist + scan_levels_bytes(nblk * kDigits, 4) + 512;
}

int radix_sort_u64(uint64_t* keys, uint64_t* keys_alt, uint32_t* vals, uint32_t* vals_alt, size_t n,
                   int key_bits, bool* in_alt, Scratch& scratch, cudaStream_t s) {
  *in_alt = false;
  if (n <= 1) return 0;
  if (key_bits < 1) key_bits = 1;
  if (key_bits > 64) key_bits = 64;
  const int passes = (key_bits + 7) / 8;
  if (n <= kSmallN) {
    static bool attr_set = false;
    if (!attr_set) {
      VX_CUDA_TRY(cudaFuncSetAttribute(small_sort_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       (int)kSmallSmem));
      attr_set = true;
    }
    vxh::count_launch();
    small_sort_kernel<<<1, kSmallBlock, kSmallSmem, s>>>(keys, vals, n, passes);
    VX_CUDA_TRY(cudaGetLastError());
    return 0;
  }
  if (int rc = scratch.ensure(radix_sort_scratch_bytes(n))) return rc;
  const uint32_t nblk = (uint32_t)((n + kBigTile - 1) / kBigTile);
  uint32_t* hist = static_cast<uint32_t*>(scratch.ptr);
  char* scan_scratch = static_cast<char*>(scratch.ptr) + ((size_t(nblk) * kDigits * 4 + 255) / 256) * 256;
  uint64_t *ki = keys, *ko = keys_alt;
  uint32_t *vi = vals, *vo = vals_alt;
  for (int p = 0; p < passes; ++p) {
    const int shift = p * 8;
    vxh::count_launch();
    radix_hist_kernel<<<nblk, kBigBlock, 0, s>>>(ki, n, shift, hist, nblk);
    VX_CUDA_TRY(cudaGetLastError());
    if (int rc = scan_impl<uint32_t, uint32_t>(hist, hist, size_t(nblk) * kDigits, nullptr, scan_scratch, s))
      return rc;
    vxh::count_launch();
    radix_scatter_kernel<<<nblk, kBigBlock, 0, s>>>(ki, vi, ko, vo, n, shift, hist, nblk);
    VX_CUDA_TRY(cudaGetLastError());
    uint64_t* tk = ki;
    ki = ko;
    ko = tk;
    uint32_t* tv = vi;
    vi = vo;
    vo = tv;
  }
  *in_alt = (passes & 1) != 0;
  return 0;
}

}  // namespace vxh
