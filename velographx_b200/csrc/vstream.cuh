// Version-parallel batched stream (internal): a window of consecutive update
// batches of an undirected graph answered by one bit-parallel BFS over the
// window's graph versions.
#pragma once

#include <cstddef>
#include <cstdint>

#include "bfs.cuh"

namespace vxh {

constexpr uint32_t kMaxVersions = 256;  // versions per window (8 words of bits per vertex)

struct VsCounters {
  // per-level counters, rotated over three slots like the multi-root BFS's
  uint32_t qn[3];     // frontier queue lengths
  uint32_t tn[3];     // touched heads of a push level
  uint32_t nbig[3];   // rows of a level long enough for the whole grid
  uint32_t gnext[3];  // next 32-vertex group of a pull level
  unsigned long long mf[3];  // arcs of the frontier's rows (the push cost of the level)
  uint32_t levels;
  uint32_t err;
  uint32_t seed;      // the source is reached at the window's start
  uint32_t runs;      // distinct touched arcs
  unsigned long long reach;   // finite distances of the last version
  unsigned long long common;  // digest deltas of discoveries made in every version at once
  // per level: globaltimer at its start, then its frontier size with bit 63
  // set for a pull level; after the last level, the closing stamp
  unsigned long long trace[2 * 64 + 1];
};

struct VersionBufs {
  size_t ops_cap = 0, v_cap = 0, w = 0, k_cap = 0;
  // touched arcs of the window
  uint64_t* keys = nullptr;
  uint64_t* keys_alt = nullptr;
  uint32_t* vals = nullptr;
  uint32_t* vals_alt = nullptr;
  uint32_t* flag = nullptr;
  uint32_t* pos = nullptr;
  uint32_t* tu = nullptr;
  uint32_t* tx = nullptr;
  uint32_t* tmask = nullptr;  // [runs][w]
  uint32_t* tpre = nullptr;   // bitmap over tails: a touched arc present at the window's start
  uint2* trow = nullptr;      // per tail: [first, end) of its touched arcs
  uint32_t* boff = nullptr;   // window-relative op offsets of the batches [k + 1]
  uint32_t* vlen = nullptr;   // distance-vector length after each version [k]
  // traversal state, [V][w] words per vertex
  uint32_t* vis = nullptr;
  uint32_t* frn[3] = {nullptr, nullptr, nullptr};
  uint32_t* nxt = nullptr;
  uint32_t* touched = nullptr;
  uint32_t* q[3] = {nullptr, nullptr, nullptr};
  uint32_t* tl = nullptr;
  uint32_t* big = nullptr;
  uint32_t* biglen = nullptr;
  unsigned long long* dig = nullptr;     // [k] digest deltas, a difference array over the versions
  unsigned long long* bucket = nullptr;  // [k] unreachable terms by first version
  VsCounters* ctr = nullptr;
  VsCounters* hctr = nullptr;
  unsigned long long* hdig = nullptr;    // pinned copies [2k]
  uint32_t* barrier = nullptr;
  int grid[4] = {0, 0, 0, 0};  // cooperative grid per word count (1, 2, 4, 8)

  int ensure(size_t ops, size_t V, size_t w, size_t k);
  void free_all();
  VersionBufs() = default;
  VersionBufs(const VersionBufs&) = delete;
  VersionBufs& operator=(const VersionBufs&) = delete;
  ~VersionBufs() { free_all(); }
};

// Applies batches [t0, t1) of an uploaded stream (ops d_src/d_dst/d_add,
// host offsets hoff and per-batch vertex counts vpost, both indexed by
// absolute batch) to b's graph and distances: the versions' distances by one
// bit-parallel BFS over the graph at the window's start plus the window's
// touched arcs with per-version presence, then the window's ops committed as
// one merged batch (the last op per edge wins, as batch by batch).  Writes
// the digest of every version to digests[t0..t1) when digests is not null.
// Requires an undirected graph and t1 - t0 <= kMaxVersions.
int stream_versions(Bfs* b, const uint32_t* d_src, const uint32_t* d_dst, const uint8_t* d_add, const uint64_t* hoff,
                    const uint32_t* vpost, size_t t0, size_t t1, uint64_t* digests);

// Buffers for windows of up to k batches and `ops` ops over V vertices (and
// the graph's batch buffers for the merged commit), so that no window
// allocates.
int stream_versions_reserve(Bfs* b, size_t ops, size_t V, size_t k);

// Level trace of the last window's traversal: {start ns, n_f | pull << 63}
// per level (up to 64), then the closing stamp; *n = 2 * levels + 1 (0 when
// no window ran).
int stream_versions_trace(Bfs* b, unsigned long long* out, size_t cap, size_t* n);

}  // namespace vxh
