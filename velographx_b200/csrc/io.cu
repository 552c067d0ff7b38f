// Whole-graph exports -- the on-disk formats and the consolidation snapshot --
// with the device doing the bulk work:
//
//   load_edge_list  (src/io.cpp:23-53)                 a text edge list parsed on
//                   the device -- newline positions by a chunked count and scan,
//                   one thread per line, first bad line reported as the
//                   reference reports it -- then a device bulk load;
//   save_binary     (include/velographx/io/binary_graph.hpp:9-14)  every row of
//                   the logical graph merged on the device (base arcs without
//                   tombstones + delta arcs, ascending) into (u, v) pairs;
//   load_binary     (binary_graph.hpp:15-20)             pairs uploaded, the
//                   undirected filter u <= v applied on the device, then a
//                   device bulk load (the same logical graph, version and vertex
//                   count as the reference's apply + compact);
//   consolidate_to_csr_snapshot  (include/velographx/storage/consolidation.hpp:
//                   132-163)  the same export bulk-loaded into a fresh graph,
//                   the source untouched.
#include <algorithm>
#include <cstdio>
#include <cstring>
#include <memory>
#include <vector>

#include "graph.cuh"
#include "frontier.cuh"
#include "graph_dev.cuh"
#include "io.cuh"
#include "prims.cuh"

namespace vxh {

namespace {

constexpr uint64_t kBinaryMagic = 0x564758303031ull;  // binary_graph.hpp:11
constexpr uint32_t kChunk = 16384;                      // bytes per block of the newline passes
constexpr int kIoThreads = 256;

enum : uint32_t { kLineEdge = 0, kLineSkip = 1, kLineMalformed = 2, kLineOverflow = 3, kLineTrailing = 4 };

// C-locale isspace (the characters std::isspace and std::ws skip).
__device__ __forceinline__ bool is_space(uint8_t c) { return c == ' ' || (c >= '\t' && c <= '\r'); }

// Newlines in each kChunk-byte chunk (one block per chunk).
__global__ void nl_count_kernel(const uint8_t* buf, size_t n, uint32_t* cnt) {
  const size_t lo = (size_t)blockIdx.x * kChunk, hi = min(n, lo + kChunk);
  uint32_t c = 0;
  for (size_t i = lo + threadIdx.x; i < hi; i += blockDim.x) c += buf[i] == '\n';
  c = __reduce_add_sync(0xFFFFFFFFu, c);
  __shared__ uint32_t ws[kIoThreads / 32];
  if ((threadIdx.x & 31) == 0) ws[threadIdx.x >> 5] = c;
  __syncthreads();
  if (threadIdx.x == 0) {
    uint32_t t = 0;
    for (int w = 0; w < kIoThreads / 32; ++w) t += ws[w];
    cnt[blockIdx.x] = t;
  }
}

// starts[k + 1] = position after the k-th newline (starts[0] = 0): one warp
// per chunk walks it in order, a ballot per 32 bytes.
__global__ void nl_write_kernel(const uint8_t* buf, size_t n, const uint64_t* base, uint64_t* starts) {
  const size_t lo = (size_t)blockIdx.x * kChunk, hi = min(n, lo + kChunk);
  uint64_t at = base[blockIdx.x];
  const int lane = threadIdx.x & 31;
  for (size_t i0 = lo; i0 < hi; i0 += 32) {
    const size_t i = i0 + lane;
    const bool nl = i < hi && buf[i] == '\n';
    const uint32_t m = __ballot_sync(0xFFFFFFFFu, nl);
    if (nl) starts[at + 1 + __popc(m & ((1u << lane) - 1u))] = i + 1;
    at += __popc(m);
  }
}

// Reads an unsigned 64-bit value the way std::istream >> uint64_t does in the
// C locale: leading whitespace, an optional sign, decimal digits; a magnitude
// past 2^64 - 1 fails, a minus sign negates modulo 2^64.
__device__ bool read_u64(const uint8_t* s, size_t& i, size_t e, unsigned long long& out) {
  while (i < e && is_space(s[i])) ++i;
  bool neg = false;
  if (i < e && (s[i] == '+' || s[i] == '-')) {
    neg = s[i] == '-';
    ++i;
  }
  if (i >= e || s[i] < '0' || s[i] > '9') return false;
  unsigned long long v = 0;
  bool over = false;
  while (i < e && s[i] >= '0' && s[i] <= '9') {
    const unsigned d = s[i] - '0';
    if (v > (~0ull - d) / 10ull) over = true;
    v = v * 10ull + d;
    ++i;
  }
  if (over) return false;
  out = neg ? 0ull - v : v;
  return true;
}

// One line [lo, hi) of the edge list: kLineEdge with (u, v), kLineSkip for a
// blank line or a comment ('#' or '%' after leading whitespace), else the
// error the reference raises for it (io.cpp:37-49, in its order: two values,
// then the uint32 range, then nothing but whitespace after them).
__global__ void parse_lines_kernel(const uint8_t* buf, size_t n, const uint64_t* starts, uint64_t nlines,
                                   uint2* uv, uint32_t* keep, unsigned long long* first_error) {
  for (uint64_t j = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; j < nlines;
       j += (uint64_t)gridDim.x * blockDim.x) {
    const size_t lo = starts[j];
    const size_t hi = j + 1 < nlines ? starts[j + 1] - 1 : n;  // the newline is not part of the line
    size_t i = lo;
    while (i < hi && is_space(buf[i])) ++i;
    uint32_t st = kLineEdge;
    unsigned long long u = 0, v = 0;
    if (i >= hi || buf[i] == '#' || buf[i] == '%') {
      st = kLineSkip;
    } else if (!read_u64(buf, i, hi, u) || !read_u64(buf, i, hi, v)) {
      st = kLineMalformed;
    } else if (u > 0xFFFFFFFFull || v > 0xFFFFFFFFull) {
      st = kLineOverflow;
    } else {
      while (i < hi && is_space(buf[i])) ++i;
      if (i < hi) st = kLineTrailing;
    }
    keep[j] = st == kLineEdge;
    uv[j] = make_uint2((uint32_t)u, (uint32_t)v);
    if (st >= kLineMalformed) atomicMin(first_error, (j << 3) | st);
  }
}

__global__ void compact_pairs_kernel(const uint2* uv, const uint32_t* keep, const uint32_t* pos, uint64_t nlines,
                                     uint2* out) {
  for (uint64_t j = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; j < nlines;
       j += (uint64_t)gridDim.x * blockDim.x)
    if (keep[j]) out[pos[j]] = uv[j];
}

// Live degree of every row (base arcs without tombstones + delta arcs).
__global__ void live_degree_kernel(vxb::DevAdj a, uint32_t V, uint32_t* deg) {
  for (uint32_t u = blockIdx.x * blockDim.x + threadIdx.x; u < V; u += gridDim.x * blockDim.x) {
    uint64_t b, e;
    vxb::base_range(a, u, b, e);
    deg[u] = (uint32_t)(e - b) - (u < a.Vb ? a.tcnt[u] : 0u) + a.drow[u].y;
  }
}

// Row u of the logical graph as (u, v) pairs at out[off[u]...], ascending,
// one warp per row: the live base arcs are compacted into vals (in order),
// the row's sorted delta arcs (disjoint from them) merged in place, and the
// pairs written.
__global__ void export_rows_kernel(vxb::DevAdj a, uint32_t V, const uint64_t* off, uint32_t* vals, uint2* out) {
  const int lane = threadIdx.x & 31;
  const uint32_t warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const uint32_t nw = (gridDim.x * blockDim.x) >> 5;
  for (uint32_t u = warp; u < V; u += nw) {
    uint64_t b, e;
    vxb::base_range(a, u, b, e);
    const uint2 dr = a.drow[u];
    uint32_t* row = vals + off[u];
    uint32_t live = 0;
    for (uint64_t j0 = b; j0 < e; j0 += 32) {
      const uint64_t j = j0 + lane;
      const uint32_t x = j < e ? a.col[j] : vxb::kTomb;
      const bool ok = !(x & vxb::kTomb);
      const uint32_t m = __ballot_sync(0xFFFFFFFFu, ok);
      if (ok) row[live + __popc(m & ((1u << lane) - 1u))] = x;
      live += __popc(m);
    }
    __syncwarp();
    if (dr.y) gdev::warp_merge_inplace(row, live, a.darena + dr.x, dr.y);
    __syncwarp();
    const uint32_t total = live + dr.y;
    for (uint32_t k = lane; k < total; k += 32) out[off[u] + k] = make_uint2(u, row[k]);
    __syncwarp();
  }
}

// Undirected load_binary keeps a pair only when u <= v (binary_graph.hpp:19);
// a dropped pair becomes a self-loop, which the bulk load ignores.
__global__ void keep_upper_kernel(uint2* uv, uint64_t m, unsigned long long* kept) {
  unsigned long long c = 0;
  for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < m; i += (uint64_t)gridDim.x * blockDim.x) {
    const uint2 p = uv[i];
    if (p.x > p.y) uv[i] = make_uint2(p.x, p.x);
    else ++c;
  }
  c = vxb::warp_sum(c);
  if ((threadIdx.x & 31) == 0 && c) atomicAdd(kept, c);
}

unsigned grid_of(uint64_t n, int per = kIoThreads) {
  const uint64_t b = (n + per - 1) / per;
  return (unsigned)std::max<uint64_t>(1, std::min<uint64_t>(b, 65535ull * 16));
}

struct FileCloser {
  void operator()(FILE* f) const {
    if (f) fclose(f);
  }
};
using File = std::unique_ptr<FILE, FileCloser>;

// Device buffers freed on every exit path.
struct DevBufs {
  std::vector<void*> p;
  template <class T>
  int alloc(T** out, size_t count) {
    void* q = nullptr;
    if (cudaMalloc(&q, std::max<size_t>(count, 1) * sizeof(T)) != cudaSuccess) {
      set_error("I/O: device allocation of %zu bytes failed", count * sizeof(T));
      return -4;
    }
    p.push_back(q);
    *out = static_cast<T*>(q);
    return 0;
  }
  ~DevBufs() {
    for (void* q : p) cudaFree(q);
  }
};

int read_file(const char* path, std::vector<uint8_t>& data, const char* open_msg) {
  File f(fopen(path, "rb"));
  if (!f || fseek(f.get(), 0, SEEK_END) != 0) {
    set_error("%s", open_msg);
    return kErrIo;
  }
  const long sz = ftell(f.get());
  if (sz < 0 || fseek(f.get(), 0, SEEK_SET) != 0) {
    set_error("%s", open_msg);
    return kErrIo;
  }
  data.resize((size_t)sz);
  if (sz && fread(data.data(), 1, (size_t)sz, f.get()) != (size_t)sz) {
    set_error("%s", open_msg);
    return kErrIo;
  }
  return 0;
}

}  // namespace

int graph_load_edge_list(const char* path, bool directed, Graph** out) {
  std::vector<uint8_t> text;
  if (int rc = read_file(path, text, "unable to open edge-list file")) return rc;
  Graph* g = nullptr;
  if (int rc = graph_create(&g, 0, directed)) return rc;
  std::unique_ptr<Graph, void (*)(Graph*)> guard(g, graph_destroy);
  cudaStream_t s = g->stream;
  const size_t n = text.size();
  const size_t nchunks = std::max<size_t>(1, (n + kChunk - 1) / kChunk);
  DevBufs d;
  uint8_t* buf = nullptr;
  uint32_t* cnt = nullptr;
  uint64_t *base = nullptr, *tot = nullptr;
  if (int rc = d.alloc(&buf, n) | d.alloc(&cnt, nchunks) | d.alloc(&base, nchunks) | d.alloc(&tot, 1)) return rc;
  if (n) VX_CUDA_TRY(cudaMemcpyAsync(buf, text.data(), n, cudaMemcpyHostToDevice, s));
  uint64_t newlines = 0;
  if (n) {
    count_launch();
    nl_count_kernel<<<(unsigned)nchunks, kIoThreads, 0, s>>>(buf, n, cnt);
    if (int rc = scan_exclusive_u32_to_u64(cnt, base, nchunks, tot, g->scratch, s)) return rc;
    VX_CUDA_TRY(cudaMemcpyAsync(&newlines, tot, 8, cudaMemcpyDeviceToHost, s));
    VX_CUDA_TRY(cudaStreamSynchronize(s));
  }
  const uint64_t nlines = newlines + 1;  // the text after the last newline is a line too (maybe empty)
  if (nlines >= 0xFFFFFFFFull) {
    set_error("edge list of %llu lines exceeds the supported 2^32 - 1", (unsigned long long)nlines);
    return -2;
  }
  uint64_t* starts = nullptr;
  uint2 *uv = nullptr, *edges = nullptr;
  uint32_t *keep = nullptr, *pos = nullptr, *kept = nullptr;
  unsigned long long* err = nullptr;
  if (int rc = d.alloc(&starts, nlines) | d.alloc(&uv, nlines) | d.alloc(&keep, nlines) | d.alloc(&pos, nlines) |
               d.alloc(&kept, 1) | d.alloc(&err, 1))
    return rc;
  VX_CUDA_TRY(cudaMemsetAsync(starts, 0, 8, s));
  VX_CUDA_TRY(cudaMemsetAsync(err, 0xFF, 8, s));
  if (n) {
    count_launch();
    nl_write_kernel<<<(unsigned)nchunks, 32, 0, s>>>(buf, n, base, starts);
  }
  count_launch();
  parse_lines_kernel<<<grid_of(nlines), kIoThreads, 0, s>>>(buf, n, starts, nlines, uv, keep, err);
  unsigned long long first_err = 0;
  VX_CUDA_TRY(cudaMemcpyAsync(&first_err, err, 8, cudaMemcpyDeviceToHost, s));
  VX_CUDA_TRY(cudaStreamSynchronize(s));
  if (first_err != ~0ull) {
    const unsigned long long line = (first_err >> 3) + 1;
    switch ((uint32_t)(first_err & 7u)) {
      case kLineOverflow:
        set_error("vertex id exceeds uint32 range at line %llu", line);
        return kErrOverflow;
      case kLineTrailing:
        set_error("unexpected trailing data at line %llu", line);
        return kErrFormat;
      default:
        set_error("malformed edge list at line %llu", line);
        return kErrFormat;
    }
  }
  if (int rc = scan_exclusive_u32(keep, pos, nlines, kept, g->scratch, s)) return rc;
  uint32_t nedges = 0;
  VX_CUDA_TRY(cudaMemcpyAsync(&nedges, kept, 4, cudaMemcpyDeviceToHost, s));
  VX_CUDA_TRY(cudaStreamSynchronize(s));
  if (int rc = d.alloc(&edges, nedges)) return rc;
  count_launch();
  compact_pairs_kernel<<<grid_of(nlines), kIoThreads, 0, s>>>(uv, keep, pos, nlines, edges);
  if (int rc = graph_bulk_load(g, reinterpret_cast<const uint32_t*>(edges), nedges)) return rc;
  *out = guard.release();
  return 0;
}

namespace {

// Every arc of the logical graph as (u, v) pairs in `pairs` (m entries, rows
// in vertex order, each ascending), on the graph's stream.
int export_arcs(Graph* g, DevBufs& d, uint2** pairs_out, uint64_t* m_out) {
  cudaStream_t s = g->stream;
  if (int rc = graph_sync_counters(g)) return rc;
  const uint64_t n = g->V, m = graph_edge_count_directed(g);
  const vxb::DevAdj a = g->view().out;
  uint32_t *deg = nullptr, *vals = nullptr;
  uint64_t *off = nullptr, *tot = nullptr;
  uint2* pairs = nullptr;
  if (int rc = d.alloc(&deg, n) | d.alloc(&off, n) | d.alloc(&tot, 1) | d.alloc(&vals, m) | d.alloc(&pairs, m))
    return rc;
  if (n) {
    count_launch();
    live_degree_kernel<<<grid_of(n), kIoThreads, 0, s>>>(a, (uint32_t)n, deg);
    if (int rc = scan_exclusive_u32_to_u64(deg, off, n, tot, g->scratch, s)) return rc;
    uint64_t total = 0;
    VX_CUDA_TRY(cudaMemcpyAsync(&total, tot, 8, cudaMemcpyDeviceToHost, s));
    VX_CUDA_TRY(cudaStreamSynchronize(s));
    if (total != m) {
      set_error("graph export: %llu live arcs against an edge count of %llu", (unsigned long long)total,
                (unsigned long long)m);
      return -5;
    }
    count_launch();
    export_rows_kernel<<<grid_of(32 * n), kIoThreads, 0, s>>>(a, (uint32_t)n, off, vals, pairs);
  }
  *pairs_out = pairs;
  *m_out = m;
  return 0;
}

// Sum over every live arc of the logical graph (base arcs without tombstones,
// then delta arcs), one warp per row: the neighbour-iteration cost of the
// current layout.
__global__ void scan_rows_kernel(vxb::DevAdj a, uint32_t V, unsigned long long* out) {
  const int lane = threadIdx.x & 31;
  const uint32_t nw = (gridDim.x * blockDim.x) >> 5;
  unsigned long long acc = 0, arcs = 0;
  for (uint32_t u = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; u < V; u += nw) {
    auto visit = [&](bool valid, uint32_t v, uint32_t) {
      if (valid) {
        acc += v;
        ++arcs;
      }
    };
    frontier::warp_row(a, u, visit);
  }
  acc = vxb::warp_sum(acc);
  arcs = vxb::warp_sum(arcs);
  if (lane == 0 && arcs) {
    atomicAdd(&out[0], acc);
    atomicAdd(&out[1], arcs);
  }
}

}  // namespace

int graph_snapshot(Graph* src, Graph** out) {
  DevBufs d;
  uint2* pairs = nullptr;
  uint64_t m = 0;
  if (int rc = export_arcs(src, d, &pairs, &m)) return rc;
  Graph* g = nullptr;
  if (int rc = graph_create(&g, src->V, src->directed)) return rc;
  std::unique_ptr<Graph, void (*)(Graph*)> guard(g, graph_destroy);
  // the pairs are read on the new graph's stream: the export must be done
  VX_CUDA_TRY(cudaStreamSynchronize(src->stream));
  if (!src->directed && m) {  // each undirected edge once (u < v); the load adds both arcs
    unsigned long long* kept = nullptr;
    if (int rc = d.alloc(&kept, 1)) return rc;
    VX_CUDA_TRY(cudaMemsetAsync(kept, 0, 8, g->stream));
    count_launch();
    keep_upper_kernel<<<grid_of(m), kIoThreads, 0, g->stream>>>(pairs, m, kept);
  }
  if (int rc = graph_bulk_load(g, reinterpret_cast<const uint32_t*>(pairs), m)) return rc;
  *out = guard.release();
  return 0;
}

int graph_scan_rows(Graph* g, uint64_t* arcs, double* ns) {
  cudaStream_t s = g->stream;
  DevBufs d;
  unsigned long long* acc = nullptr;
  if (int rc = d.alloc(&acc, 2)) return rc;
  cudaEvent_t e0, e1;
  VX_CUDA_TRY(cudaEventCreate(&e0));
  VX_CUDA_TRY(cudaEventCreate(&e1));
  VX_CUDA_TRY(cudaMemsetAsync(acc, 0, 16, s));
  VX_CUDA_TRY(cudaEventRecord(e0, s));
  if (g->V) {
    count_launch();
    scan_rows_kernel<<<grid_of(32ull * g->V), kIoThreads, 0, s>>>(g->view().out, (uint32_t)g->V, acc);
  }
  VX_CUDA_TRY(cudaEventRecord(e1, s));
  unsigned long long h[2] = {0, 0};
  VX_CUDA_TRY(cudaMemcpyAsync(h, acc, 16, cudaMemcpyDeviceToHost, s));
  VX_CUDA_TRY(cudaStreamSynchronize(s));
  float ms = 0.f;
  VX_CUDA_TRY(cudaEventElapsedTime(&ms, e0, e1));
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  *arcs = h[1];
  *ns = (double)ms * 1e6;
  return 0;
}

int graph_save_binary(Graph* g, const char* path) {
  cudaStream_t s = g->stream;
  DevBufs d;
  uint2* pairs = nullptr;
  uint64_t m = 0;
  if (int rc = export_arcs(g, d, &pairs, &m)) return rc;
  const uint64_t n = g->V;
  std::vector<uint2> host(m);
  if (m) VX_CUDA_TRY(cudaMemcpyAsync(host.data(), pairs, m * sizeof(uint2), cudaMemcpyDeviceToHost, s));
  VX_CUDA_TRY(cudaStreamSynchronize(s));
  File f(fopen(path, "wb"));
  if (!f) {
    set_error("cannot open output");
    return kErrIo;
  }
  const uint64_t hdr[3] = {kBinaryMagic, n, m};
  if (fwrite(hdr, sizeof(hdr), 1, f.get()) != 1 || (m && fwrite(host.data(), sizeof(uint2), m, f.get()) != m)) {
    set_error("cannot write output");
    return kErrIo;
  }
  return 0;
}

int graph_load_binary(const char* path, bool directed, Graph** out) {
  File f(fopen(path, "rb"));
  if (!f) {
    set_error("cannot open input");
    return kErrIo;
  }
  uint64_t hdr[3] = {0, 0, 0};
  const size_t got = fread(hdr, sizeof(uint64_t), 3, f.get());
  if (got < 3) memset(hdr + got, 0, (3 - got) * sizeof(uint64_t));  // unread fields read as zero
  if (hdr[0] != kBinaryMagic) {
    set_error("invalid VeloGraphX binary graph");
    return kErrFormat;
  }
  const uint64_t n = hdr[1], m = hdr[2];
  if (n > vxb::kMaxVertices) {
    set_error("vertex count %llu exceeds the supported maximum %u", (unsigned long long)n, vxb::kMaxVertices);
    return -2;
  }
  // all m pairs must be there (the reference stops at the first short read)
  if (fseek(f.get(), 0, SEEK_END) != 0) {
    set_error("cannot open input");
    return kErrIo;
  }
  const long sz = ftell(f.get());
  if (sz < 24 || (uint64_t)(sz - 24) / 8 < m) {
    set_error("truncated graph file");
    return kErrFormat;
  }
  std::vector<uint2> host(m);
  if (fseek(f.get(), 24, SEEK_SET) != 0 || (m && fread(host.data(), sizeof(uint2), m, f.get()) != m)) {
    set_error("truncated graph file");
    return kErrFormat;
  }
  Graph* g = nullptr;
  if (int rc = graph_create(&g, n, directed)) return rc;
  std::unique_ptr<Graph, void (*)(Graph*)> guard(g, graph_destroy);
  cudaStream_t s = g->stream;
  DevBufs d;
  uint2* uv = nullptr;
  unsigned long long* kept = nullptr;
  if (int rc = d.alloc(&uv, m) | d.alloc(&kept, 1)) return rc;
  if (m) VX_CUDA_TRY(cudaMemcpyAsync(uv, host.data(), m * sizeof(uint2), cudaMemcpyHostToDevice, s));
  unsigned long long nkept = m;
  if (!directed && m) {
    VX_CUDA_TRY(cudaMemsetAsync(kept, 0, 8, s));
    count_launch();
    keep_upper_kernel<<<grid_of(m), kIoThreads, 0, s>>>(uv, m, kept);
    VX_CUDA_TRY(cudaMemcpyAsync(&nkept, kept, 8, cudaMemcpyDeviceToHost, s));
    VX_CUDA_TRY(cudaStreamSynchronize(s));
  }
  // the reference applies one batch of the kept pairs (version 1 when it is
  // not empty) and compacts; a bulk load gives that graph and version
  if (nkept) {
    if (int rc = graph_bulk_load(g, reinterpret_cast<const uint32_t*>(uv), m)) return rc;
  }
  *out = guard.release();
  return 0;
}

}  // namespace vxh
