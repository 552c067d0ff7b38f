// Version-parallel batched stream.
//
// A window of k <= 256 consecutive batches of an undirected graph has k graph
// versions: version b is the graph after the window's batch b.  Every arc
// that no op of the window touches is present in all of them; every touched
// arc (u, v) gets a k-bit presence mask: its state at the window's start,
// then, batch by batch, the last op of that batch on (u, v) if any (the
// reference's last-op-wins rule, bfs.hpp:38-50, and its per-arc application,
// dynamic_graph.hpp:717-733).  One bit-parallel BFS from the source over the
// graph at the window's start, with every touched arc filtered by its mask,
// then gives each vertex the level at which it is reached in each version:
// exactly the distances IncrementalBFS::apply leaves after each batch, which
// equal a fresh BFS of that version (bfs.hpp:100-120) -- except for the
// reference's quirk of a source out of range at construction, which never
// becomes reached: the traversal starts only when the source is reached at
// the window's start.
//
// The traversal is the multi-root BFS's (push levels over queued frontier
// rows, pull levels over flattened in-rows with early exit, rows of 2,048+
// arcs over the whole grid), with version bits in place of root bits.  A row
// is read in three parts: its base CSR arcs, its delta arcs, and its touched
// arcs with their masks; base and delta arcs that are also touched (present at
// the window's start) are skipped there, found by a binary search in the
// row's sorted touched list, so they count only through their masks.
//
// Outputs: the distances of the last version (the object's new state), its
// reachable count, and optionally each version's digest (sum over v <
// len_b of splitmix64(v << 32 | dist_b[v])), accumulated as the unreachable
// term of every vertex plus, per discovery, the difference to its level.
// The window's ops are then committed to the graph as one merged batch.
#include <algorithm>
#include <cstring>
#include <vector>

#include "frontier.cuh"
#include "graph.cuh"
#include "graph_dev.cuh"
#include "prims.cuh"
#include "vstream.cuh"

namespace vxh {

namespace {

using namespace frontier;

constexpr int kVsThreads = 512;

// The block's staging of frontier and touched-list appends: one global
// atomic per block per phase instead of one per warp step.
__shared__ BlockQueue vs_bq;
// The block's sum of the degrees of the vertices it adds to the next frontier
// (the push cost of the next level).
__shared__ unsigned long long vs_mf;

// A level pulls when pushing its frontier's rows would cost more than this
// many times fewer arcs than the graph holds (a pushed arc costs about this
// many pulled ones).
constexpr unsigned long long kPushArcCost = 12;

// Block-uniform: the block's frontier-degree sum added to *dst.
__device__ __forceinline__ void mf_flush(unsigned long long* dst) {
  __syncthreads();
  if (threadIdx.x == 0 && vs_mf) {
    atomicAdd(dst, vs_mf);
    vs_mf = 0;
  }
  __syncthreads();
}
constexpr uint32_t kVsWarps = kVsThreads / 32;
// 32-vertex groups a warp claims per atomic of a pull level (one counter
// per level: a claim per group serialised on it)
constexpr uint32_t kClaimGroups = 4;
constexpr uint32_t kVsHead = 8;        // in-arcs a lane reads itself before the flattened rounds
constexpr uint32_t kVsHeadStep = 4;    // of which it loads this many at a time
constexpr uint32_t kVsBigPull = 2048;  // pull rows this long are read by the whole grid
constexpr uint32_t kVsBigPush = 1024;  // push rows this long are expanded by the whole grid
constexpr uint32_t kVsPushSlice = 128; // arcs of a hub row a warp takes at a time
constexpr int kVsTBits = 8;            // version field of the sort keys
constexpr uint32_t kNoEntry = 0xFFFFFFFFu;

struct VsParams {
  vxb::DevAdj a;          // adjacency at the window's start (out == in)
  uint32_t V;             // vertices covered (the last version's distance length)
  uint32_t K;             // versions
  uint32_t source;
  uint32_t len0;          // distance length at the window's start
  const uint32_t* tx;     // touched arcs' heads, sorted by (tail, head)
  const uint32_t* tmask;  // [runs][W] presence masks
  const uint2* trow;      // per tail: [first, end) of its touched arcs
  const uint32_t* tpre;   // bitmap of tails with a touched arc present at the start
  const uint32_t* vlen;   // distance length after each version
  uint32_t* dist;         // distances of the last version
  uint32_t* vis;          // [V][W]
  uint32_t* frn[3];
  uint32_t* nxt;
  uint32_t* touched;
  uint32_t* q[3];
  uint32_t* tl;
  uint32_t* big;
  uint32_t* biglen;
  unsigned long long* dig;     // [K] digest deltas as a difference array over the versions (null: no digests)
  unsigned long long* bucket;  // [K]
  VsCounters* c;
  uint32_t* bar;
  uint32_t nblocks;
  float pull_frac;
  unsigned long long arcs;  // arcs of the graph (a pull level reads up to all of them)
};

__device__ __forceinline__ bool vs_sync(const VsParams& p) {
  vxb::grid_barrier(p.bar, p.nblocks, &p.c->err);
  return __ldcg(&p.c->err) == 0u;
}

__device__ __forceinline__ uint32_t vmask(uint32_t K, uint32_t w) {
  const uint32_t rem = K - 32 * w;
  return rem >= 32 ? 0xFFFFFFFFu : ((1u << rem) - 1u);
}

// ------------------------------------------------------ window set-up --

// Keys (tail, head, version) of both arcs of every op of the window, the op
// index as value; self-loops get the all-ones key, which sorts last.
__global__ void vs_keys_kernel(const uint32_t* src, const uint32_t* dst, size_t n, const uint32_t* boff, uint32_t k,
                               int bbits, uint64_t* keys, uint32_t* vals) {
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
    // batch of op i: the last t with boff[t] <= i
    uint32_t lo = 0, hi = k;  // boff[lo] <= i < boff[hi]
    while (hi - lo > 1) {
      const uint32_t mid = (lo + hi) >> 1;
      if (boff[mid] <= (uint32_t)i) lo = mid;
      else hi = mid;
    }
    const uint64_t u = src[i], v = dst[i];
    uint64_t k1 = ~0ull, k2 = ~0ull;
    if (u != v) {
      k1 = (u << (bbits + kVsTBits)) | (v << kVsTBits) | lo;
      k2 = (v << (bbits + kVsTBits)) | (u << kVsTBits) | lo;
    }
    keys[2 * i] = k1;
    keys[2 * i + 1] = k2;
    vals[2 * i] = (uint32_t)i;
    vals[2 * i + 1] = (uint32_t)i;
  }
}

// flag[j] = key j starts the run of a distinct arc
__global__ void vs_runs_kernel(const uint64_t* keys, size_t m, uint32_t* flag) {
  for (size_t j = blockIdx.x * (size_t)blockDim.x + threadIdx.x; j < m; j += (size_t)gridDim.x * blockDim.x) {
    const uint64_t x = keys[j];
    flag[j] = x != ~0ull && (j == 0 || (keys[j - 1] >> kVsTBits) != (x >> kVsTBits)) ? 1u : 0u;
  }
}

// One thread per distinct arc: its presence at the window's start (the
// pre-window graph), then its state after each version, as a mask.
//
// The same walk gives the arc's final state (its last op), so the arc is
// also written, classified against the pre-window graph, as the merged
// batch's canonical arc r for the commit (arcs in (tail, head) order).
template <uint32_t W>
__global__ void vs_mask_kernel(vxb::DevAdj a, const uint64_t* keys, const uint32_t* vals, const uint32_t* flag,
                               const uint32_t* pos, size_t m, const uint8_t* add, uint32_t K, int bbits,
                               uint32_t* tu, uint32_t* tx, uint32_t* tmask, uint32_t* tpre, uint32_t* bfu,
                               uint32_t* bfv, uint8_t* bff, uint64_t* bfpos) {
  const uint64_t vmask_bits = (1ull << bbits) - 1;
  for (size_t j = blockIdx.x * (size_t)blockDim.x + threadIdx.x; j < m; j += (size_t)gridDim.x * blockDim.x) {
    if (!flag[j]) continue;
    const uint64_t arc = keys[j] >> kVsTBits;
    const uint32_t u = (uint32_t)(arc >> bbits), x = (uint32_t)(arc & vmask_bits);
    uint64_t fpos;
    const uint8_t f0 = gdev::classify_arc(a, u, x, 0, fpos);
    const bool pre = (f0 & kFCur) != 0;
    uint32_t mk[W];
#pragma unroll
    for (uint32_t w = 0; w < W; ++w) mk[w] = 0;
    bool on = pre;
    uint32_t from = 0;  // versions [from, t) keep the state `on`
    auto fill = [&](uint32_t lo, uint32_t hi) {
#pragma unroll
      for (uint32_t w = 0; w < W; ++w) {
        const uint32_t a0 = max(lo, 32 * w), a1 = min(hi, 32 * w + 32);
        if (a0 < a1) {
          const uint32_t span = a1 - a0;
          const uint32_t bits = span >= 32 ? 0xFFFFFFFFu : ((1u << span) - 1u);
          mk[w] |= bits << (a0 - 32 * w);
        }
      }
    };
    for (size_t i = j; i < m && (keys[i] >> kVsTBits) == arc; ++i) {
      const uint32_t t = (uint32_t)(keys[i] & ((1u << kVsTBits) - 1));
      if (on) fill(from, t);
      on = (add[vals[i]] & 1u) != 0;
      from = t;
    }
    if (on) fill(from, K);
    const uint32_t r = pos[j];
    tu[r] = u;
    tx[r] = x;
#pragma unroll
    for (uint32_t w = 0; w < W; ++w) tmask[(size_t)r * W + w] = mk[w];
    if (pre) atomicOr(&tpre[u >> 5], 1u << (u & 31));
    // `on` is now the last op's state: the arc's desired final state
    bfu[r] = u;
    bfv[r] = x;
    bff[r] = (uint8_t)((on ? kFAdd : 0) | (f0 & (kFInBase | kFCur)) | (on != pre ? kFChanged : 0));
    bfpos[r] = fpos;
  }
}

// trow[u] = [first, end) of u's touched arcs (the rest of trow stays zero)
__global__ void vs_rows_kernel(const uint32_t* tu, const uint32_t* runs, uint2* trow) {
  const uint32_t R = *runs;
  for (uint32_t r = blockIdx.x * blockDim.x + threadIdx.x; r < R; r += gridDim.x * blockDim.x) {
    const uint32_t u = tu[r];
    if (r == 0 || tu[r - 1] != u) trow[u].x = r;
    if (r + 1 == R || tu[r + 1] != u) trow[u].y = r + 1;
  }
}

// ---------------------------------------------------------- traversal --

// The three parts of a row: base arcs [b, b + nb), delta arcs [dx, dx + dy),
// touched arcs [tb, tb + tn); pre: base or delta arcs may also be touched.
struct VsRow {
  uint64_t b;
  uint32_t nb, dx, dy, tb, tn;
  bool pre;
};

__device__ __forceinline__ VsRow vs_row(const VsParams& p, uint32_t v) {
  VsRow r;
  uint64_t e;
  vxb::base_range(p.a, v, r.b, e);
  r.nb = (uint32_t)(e - r.b);
  const uint2 dr = p.a.drow[v];
  r.dx = dr.x;
  r.dy = dr.y;
  const uint2 tr = p.trow[v];
  r.tb = tr.x;
  r.tn = tr.y - tr.x;
  r.pre = (p.tpre[v >> 5] >> (v & 31)) & 1u;
  return r;
}

// Head of arc k of a row, with its touched entry in e (kNoEntry: present in
// every version); kTomb when the arc is skipped (tombstoned, or touched and
// counted through its entry).
__device__ __forceinline__ uint32_t vs_arc(const VsParams& p, uint64_t b, uint32_t nb, uint32_t dx, uint32_t dy,
                                           uint32_t tb, uint32_t tn, bool pre, uint32_t k, uint32_t& e) {
  e = kNoEntry;
  uint32_t x;
  if (k < nb) {
    x = p.a.col[b + k];
    if (x & kTomb) return kTomb;
  } else if (k < nb + dy) {
    x = p.a.darena[dx + (k - nb)];
  } else {
    e = tb + (k - nb - dy);
    return p.tx[e];
  }
  if (pre && gdev::bsearch_u32(p.tx, tb, tb + tn, x)) return kTomb;
  return x;
}

// Per-thread sums flushed once at the end of the launch.
struct VsSums {
  unsigned long long common = 0;  // digest deltas of vertices reached in every version at once
  unsigned long long reach = 0;   // discoveries in the last version
};

// Records v's newly reached versions `nw` at distance lvl: visited and
// frontier words, the last version's distance.  Returns whether any version
// is new.
template <uint32_t W>
__device__ __forceinline__ bool vs_discover(const VsParams& p, uint32_t v, const uint32_t* vis, const uint32_t* nw,
                                            uint32_t* fn, uint32_t lvl, VsSums& s) {
  bool any = false;
#pragma unroll
  for (uint32_t w = 0; w < W; ++w) {
    if (nw[w]) {
      any = true;
      p.vis[(size_t)v * W + w] = vis[w] | nw[w];
      fn[(size_t)v * W + w] = nw[w];
    }
  }
  if (!any) return false;
  const uint32_t lw = (p.K - 1) >> 5, lb = (p.K - 1) & 31;
  if ((nw[lw] >> lb) & 1u) {
    p.dist[v] = lvl;
    ++s.reach;
  }
  return true;
}

// Digest deltas of a discovery (v reached at distance lvl in the versions
// `nw`): one reached in every version goes to the thread's register sum;
// otherwise the delta is added, as a difference array over the versions, at
// every run boundary of the mask (+d where a run of versions starts, -d
// where it ends), so a vertex reached from some version on costs one
// shared-memory atomic however many versions it covers.
template <uint32_t W>
__device__ __forceinline__ void vs_digest(const VsParams& p, uint32_t v, const uint32_t* nw, uint32_t lvl, VsSums& s,
                                          unsigned long long* sdig) {
  bool any = false, all = true;
#pragma unroll
  for (uint32_t w = 0; w < W; ++w) {
    any = any || nw[w] != 0u;
    all = all && nw[w] == vmask(p.K, w);
  }
  if (!any) return;
  const unsigned long long d = vxb::mix64(((unsigned long long)v << 32) | lvl) -
                               vxb::mix64(((unsigned long long)v << 32) | kUnreachable);
  if (all) {
    s.common += d;
    return;
  }
  uint32_t carry = 0;  // the mask's bit just below the word
#pragma unroll
  for (uint32_t w = 0; w < W; ++w) {
    const uint32_t m = nw[w];
    uint32_t t = m ^ ((m << 1) | carry);  // bits that differ from the bit below
    carry = m >> 31;
    while (t) {
      const uint32_t b = __ffs(t) - 1;
      t &= t - 1;
      const uint32_t ver = 32 * w + b;
      if (ver < p.K) atomicAdd(&sdig[ver], ((m >> b) & 1u) ? d : (unsigned long long)0 - d);
    }
  }
}

// The listed vertices' versions accumulated in nxt become their new ones
// (nxt cleared, and the touched bits when `touched`), in warp-uniform rounds.
template <uint32_t W>
__device__ void vs_finalize(const VsParams& p, const uint32_t* list, uint32_t n, uint32_t* fn, uint32_t level,
                            uint32_t* qn, uint32_t* qout, unsigned long long* mf, VsSums& s, unsigned long long* sdig,
                            bool touched) {
  const uint32_t lane = threadIdx.x & 31;
  for (uint32_t base = gwarp() * 32; base < n; base += nwarps() * 32) {
    const uint32_t i = base + lane;
    const bool valid = i < n;
    const uint32_t x = valid ? list[i] : 0u;
    uint32_t vis[W], nw[W];
#pragma unroll
    for (uint32_t w = 0; w < W; ++w) {
      vis[w] = 0u;
      nw[w] = 0u;
      if (!valid) continue;
      const size_t o = (size_t)x * W + w;
      vis[w] = p.vis[o];
      nw[w] = __ldcg(&p.nxt[o]) & ~vis[w];
      p.nxt[o] = 0u;
    }
    if (valid && touched) p.touched[x >> 5] = 0u;
    const bool any = valid && vs_discover<W>(p, x, vis, nw, fn, level + 1, s);
    if (p.dig && valid) vs_digest<W>(p, x, nw, level + 1, s, sdig);
    bq_push(vs_bq, any, x, qn, qout);
    unsigned long long deg = 0;
    if (any) {
      const VsRow r = vs_row(p, x);
      deg = r.nb + r.dy + r.tn;
    }
    deg = vxb::warp_sum(deg);
    if (lane == 0 && deg) atomicAdd(&vs_mf, deg);
  }
  bq_flush(vs_bq, qn, qout);
  mf_flush(mf);
}

template <uint32_t W>
struct VsSlots {
  static constexpr uint32_t value = W <= 2 ? 8 : 4;
};

// Per-warp staging of a pull group: its 32 rows and OR accumulators.
struct VsStage {
  uint64_t rb[32];
  uint32_t nb[32];
  uint32_t dx[32];
  uint32_t dy[32];
  uint32_t tb[32];
  uint32_t tn[32];  // bit 31: pre
  uint32_t acc[32 * 8];
};

// Pull level: groups of 32 consecutive vertices from a counter; the rows of
// the group's vertices that some version has not reached are read as one
// flattened arc list, kSlots arcs per lane per round, each arc's frontier
// words (masked by its presence for touched arcs) OR-ed into its owner's
// accumulator; owners reached in every version stop.  Long rows are read by
// the whole grid after a barrier, through nxt.  Ends with a grid barrier.
template <uint32_t W>
__device__ bool vs_pull(const VsParams& p, const uint32_t* fc, uint32_t* fn, uint32_t level, uint32_t* gnext,
                        uint32_t* nbig, uint32_t* qn, uint32_t* qout, unsigned long long* mf, VsStage& ws,
                        VsSums& s, unsigned long long* sdig) {
  constexpr uint32_t kSlots = VsSlots<W>::value;
  const uint32_t lane = threadIdx.x & 31;
  uint32_t cur = 0, end = 0;  // the warp's claimed groups [cur, end), warp-uniform
  for (;;) {
    if (cur == end) {
      uint32_t c0 = 0;
      if (lane == 0) c0 = atomicAdd(gnext, kClaimGroups);
      cur = __shfl_sync(FULL, c0, 0);
      end = cur + kClaimGroups;
    }
    const uint32_t base = cur++ * 32;
    if (base >= p.V) break;
    const uint32_t v = base + lane;
    uint32_t vis[W];
    bool done = true;
#pragma unroll
    for (uint32_t w = 0; w < W; ++w) {
      vis[w] = v < p.V ? p.vis[(size_t)v * W + w] : vmask(p.K, w);
      done = done && vis[w] == vmask(p.K, w);
      ws.acc[lane * W + w] = 0u;
    }
    uint32_t len = 0, rowlen = 0;
    if (!done) {
      const VsRow r = vs_row(p, v);
      len = r.nb + r.dy + r.tn;
      rowlen = len;
      if (len >= kVsBigPull) {  // the whole grid reads it after the barrier
        const uint32_t slot = atomicAdd(nbig, 1u);
        p.big[slot] = v;
        p.biglen[slot] = len;
        len = 0;
      }
      ws.rb[lane] = r.b;
      ws.nb[lane] = r.nb;
      ws.dx[lane] = r.dx;
      ws.dy[lane] = r.dy;
      ws.tb[lane] = r.tb;
      ws.tn[lane] = r.tn | (r.pre ? 0x80000000u : 0u);
      // head: the lane first reads the first kVsHead arcs of its own row,
      // kVsHeadStep loads in flight, and stops as soon as every version has
      // reached its vertex (most vertices find a parent reached in every
      // version among their first arcs); the flattened rounds read the rest
      const uint32_t hn = min(len, kVsHead);
      uint32_t hacc[W];
#pragma unroll
      for (uint32_t w = 0; w < W; ++w) hacc[w] = 0u;
      for (uint32_t h0 = 0; h0 < hn; h0 += kVsHeadStep) {
        uint32_t hx[kVsHeadStep], he[kVsHeadStep];
#pragma unroll
        for (uint32_t k = 0; k < kVsHeadStep; ++k) {
          he[k] = kNoEntry;
          hx[k] = h0 + k < hn ? vs_arc(p, r.b, r.nb, r.dx, r.dy, r.tb, r.tn, r.pre, h0 + k, he[k]) : kTomb;
        }
#pragma unroll
        for (uint32_t k = 0; k < kVsHeadStep; ++k) {
          if (hx[k] & kTomb) continue;
          uint32_t f[W];
          load_words<W>(fc + (size_t)hx[k] * W, f);
          if (he[k] != kNoEntry) {
            uint32_t mk[W];
            load_words<W>(p.tmask + (size_t)he[k] * W, mk);
#pragma unroll
            for (uint32_t w = 0; w < W; ++w) f[w] &= mk[w];
          }
#pragma unroll
          for (uint32_t w = 0; w < W; ++w) hacc[w] |= f[w];
        }
        bool fin = true;
#pragma unroll
        for (uint32_t w = 0; w < W; ++w) fin = fin && (vis[w] | hacc[w]) == vmask(p.K, w);
        if (fin) {
          len = hn;  // nothing left for the rounds
          break;
        }
      }
      len -= hn;
#pragma unroll
      for (uint32_t w = 0; w < W; ++w) ws.acc[lane * W + w] = hacc[w];
    }
    uint32_t incl = len;
#pragma unroll
    for (uint32_t d = 1; d < 32; d <<= 1) {
      const uint32_t t = __shfl_up_sync(FULL, incl, d);
      if (lane >= d) incl += t;
    }
    const uint32_t T = __shfl_sync(FULL, incl, 31);
    uint32_t active = __ballot_sync(FULL, len > 0);
    __syncwarp();
    for (uint32_t j0 = 0; j0 < T && active; j0 += 32 * kSlots) {
      uint32_t x[kSlots], e[kSlots], own[kSlots];
#pragma unroll
      for (uint32_t u = 0; u < kSlots; ++u) {
        const uint32_t j = j0 + u * 32 + lane;
        uint32_t o = 0, lo = 0;
#pragma unroll
        for (uint32_t step = 16; step >= 1; step >>= 1) {
          const uint32_t t = __shfl_sync(FULL, incl, o + step - 1);
          if (t <= j) {
            o += step;
            lo = t;
          }
        }
        own[u] = o;
        x[u] = kTomb;
        e[u] = kNoEntry;
        if (j < T && ((active >> o) & 1u)) {
          const uint32_t tn = ws.tn[o];
          x[u] = vs_arc(p, ws.rb[o], ws.nb[o], ws.dx[o], ws.dy[o], ws.tb[o], tn & 0x7FFFFFFFu, (tn >> 31) != 0,
                        kVsHead + (j - lo), e[u]);  // past the owner's head
        }
      }
      uint32_t m[kSlots][W];
#pragma unroll
      for (uint32_t u = 0; u < kSlots; ++u) {
        if (x[u] & kTomb) {
#pragma unroll
          for (uint32_t w = 0; w < W; ++w) m[u][w] = 0u;
          continue;
        }
        load_words<W>(fc + (size_t)x[u] * W, m[u]);
        if (e[u] != kNoEntry) {
          uint32_t mk[W];
          load_words<W>(p.tmask + (size_t)e[u] * W, mk);
#pragma unroll
          for (uint32_t w = 0; w < W; ++w) m[u][w] &= mk[w];
        }
      }
#pragma unroll
      for (uint32_t u = 0; u < kSlots; ++u)
#pragma unroll
        for (uint32_t w = 0; w < W; ++w)
          if (m[u][w]) atomicOr(&ws.acc[own[u] * W + w], m[u][w]);
      __syncwarp();
      bool fin = false;
      if ((active >> lane) & 1u) {
        fin = true;
#pragma unroll
        for (uint32_t w = 0; w < W; ++w) fin = fin && (vis[w] | ws.acc[lane * W + w]) == vmask(p.K, w);
      }
      active &= ~__ballot_sync(FULL, fin);
    }
    __syncwarp();
    uint32_t nw[W];
#pragma unroll
    for (uint32_t w = 0; w < W; ++w) nw[w] = ws.acc[lane * W + w] & ~vis[w];
    const bool any = v < p.V && vs_discover<W>(p, v, vis, nw, fn, level + 1, s);
    if (p.dig && v < p.V) vs_digest<W>(p, v, nw, level + 1, s, sdig);
    bq_push(vs_bq, any, v, qn, qout);
    const unsigned long long dsum = vxb::warp_sum(any ? (unsigned long long)rowlen : 0ull);
    if (lane == 0 && dsum) atomicAdd(&vs_mf, dsum);
    __syncwarp();  // the next group overwrites the stage
  }
  bq_flush(vs_bq, qn, qout);
  mf_flush(mf);
  if (!vs_sync(p)) return false;
  const uint32_t nb = __ldcg(nbig);
  if (nb == 0) return true;
  // long rows: every warp takes 32 * kSlots-arc slices, the slices of row r
  // starting at warp r (mod the warp count); a warp skips, from the listed
  // length alone, the rows it has no slice of
  const uint32_t nw_ = nwarps(), gw = gwarp();
  for_my_rows(p.biglen, nb, 32 * kSlots, [&](uint32_t r, uint32_t, uint32_t) {
    const uint32_t v = p.big[r];
    uint32_t vis[W];
#pragma unroll
    for (uint32_t w = 0; w < W; ++w) vis[w] = __ldcg(&p.vis[(size_t)v * W + w]);
    const VsRow rw = vs_row(p, v);
    const uint32_t total = rw.nb + rw.dy + rw.tn;
    const uint32_t nslices = (total + 32 * kSlots - 1) / (32 * kSlots);
    for (uint32_t sl = (gw + nw_ - r % nw_) % nw_; sl < nslices; sl += nw_) {
      bool full = true;
#pragma unroll
      for (uint32_t w = 0; w < W; ++w) full = full && (vis[w] | __ldcg(&p.nxt[(size_t)v * W + w])) == vmask(p.K, w);
      if (full) break;
      uint32_t x[kSlots], e[kSlots];
#pragma unroll
      for (uint32_t u = 0; u < kSlots; ++u) {
        const uint32_t k = sl * 32 * kSlots + u * 32 + lane;
        x[u] = kTomb;
        e[u] = kNoEntry;
        if (k < total) x[u] = vs_arc(p, rw.b, rw.nb, rw.dx, rw.dy, rw.tb, rw.tn, rw.pre, k, e[u]);
      }
      uint32_t add[W];
#pragma unroll
      for (uint32_t w = 0; w < W; ++w) add[w] = 0u;
#pragma unroll
      for (uint32_t u = 0; u < kSlots; ++u) {
        if (x[u] & kTomb) continue;
        uint32_t f[W];
        load_words<W>(fc + (size_t)x[u] * W, f);
        if (e[u] != kNoEntry) {
          uint32_t mk[W];
          load_words<W>(p.tmask + (size_t)e[u] * W, mk);
#pragma unroll
          for (uint32_t w = 0; w < W; ++w) f[w] &= mk[w];
        }
#pragma unroll
        for (uint32_t w = 0; w < W; ++w) add[w] |= f[w];
      }
#pragma unroll
      for (uint32_t w = 0; w < W; ++w) {
        const uint32_t red = __reduce_or_sync(FULL, add[w]) & ~vis[w];
        if (lane == 0 && red) atomicOr(&p.nxt[(size_t)v * W + w], red);
      }
    }
  });
  if (!vs_sync(p)) return false;
  vs_finalize<W>(p, p.big, nb, fn, level, qn, qout, mf, s, sdig, false);
  return vs_sync(p);
}

// Push: one warp per queued frontier vertex u walks u's three row parts with
// u's frontier words; every head gets the words (masked for touched arcs)
// that it has not been reached in, OR-ed into nxt, and is listed once.
template <uint32_t W>
__device__ __forceinline__ void vs_push_arcs(const VsParams& p, const VsRow& r, const uint32_t* fw, uint32_t k0,
                                             uint32_t kend, uint32_t kstep, uint32_t* tcount) {
  const uint32_t lane = threadIdx.x & 31;
  for (uint32_t k = k0 + lane; k - lane < kend; k += kstep) {
    bool fresh = false;
    uint32_t x = kTomb;
    if (k < kend) {
      uint32_t e;
      x = vs_arc(p, r.b, r.nb, r.dx, r.dy, r.tb, r.tn, r.pre, k, e);
      if (!(x & kTomb)) {
        // bits already OR-ed into a head are not OR-ed again (one atomic per
        // new bit at a hub, not one per arc; the thread that added bits
        // lists the head)
        bool any = false;
        uint32_t vx[W];
        load_words<W>(p.vis + (size_t)x * W, vx);
#pragma unroll
        for (uint32_t w = 0; w < W; ++w) {
          uint32_t m = fw[w] & ~vx[w];
          if (m && e != kNoEntry) m &= p.tmask[(size_t)e * W + w];
          if (m) m &= ~__ldcg(&p.nxt[(size_t)x * W + w]);
          if (m) {
            atomicOr(&p.nxt[(size_t)x * W + w], m);
            any = true;
          }
        }
        if (any) {
          const uint32_t bit = 1u << (x & 31);
          fresh = !(__ldcg(&p.touched[x >> 5]) & bit) && !(atomicOr(&p.touched[x >> 5], bit) & bit);
        }
      }
    }
    bq_push(vs_bq, fresh, x, tcount, p.tl);
  }
}

template <uint32_t W>
__device__ bool vs_push(const VsParams& p, const uint32_t* fc, uint32_t* fn, uint32_t level, uint32_t n_f,
                        const uint32_t* qin, uint32_t* tn, uint32_t* nbig, uint32_t* qn, uint32_t* qout,
                        unsigned long long* mf, VsSums& s, unsigned long long* sdig) {
  const uint32_t lane = threadIdx.x & 31;
  for (uint32_t i = gwarp(); i < n_f; i += nwarps()) {
    const uint32_t u = qin[i];
    const VsRow r = vs_row(p, u);
    const uint32_t total = r.nb + r.dy + r.tn;
    if (total >= kVsBigPush) {  // a hub: the whole grid, after the barrier
      if (lane == 0) {
        const uint32_t slot = atomicAdd(nbig, 1u);
        p.big[slot] = u;
        p.biglen[slot] = total;
      }
      continue;
    }
    uint32_t fw[W];
#pragma unroll
    for (uint32_t w = 0; w < W; ++w) fw[w] = fc[(size_t)u * W + w];
    vs_push_arcs<W>(p, r, fw, 0, total, 32, tn);
  }
  bq_flush(vs_bq, tn, p.tl);
  if (!vs_sync(p)) return false;
  const uint32_t nb = __ldcg(nbig);
  // hub rows: kVsPushSlice-arc slices, the slices of row j starting at warp j
  // (mod the warp count); a warp skips the rows it has no slice of
  const uint32_t nw = nwarps();
  for_my_rows(p.biglen, nb, kVsPushSlice, [&](uint32_t j, uint32_t total, uint32_t sl) {
    const uint32_t nsl = (total + kVsPushSlice - 1) / kVsPushSlice;
    const uint32_t u = p.big[j];
    const VsRow r = vs_row(p, u);
    uint32_t fw[W];
    load_words<W>(fc + (size_t)u * W, fw);
    for (; sl < nsl; sl += nw)
      vs_push_arcs<W>(p, r, fw, sl * kVsPushSlice, min(total, (sl + 1) * kVsPushSlice), 32, tn);
  });
  bq_flush(vs_bq, tn, p.tl);
  if (nb && !vs_sync(p)) return false;
  vs_finalize<W>(p, p.tl, __ldcg(tn), fn, level, qn, qout, mf, s, sdig, true);
  return vs_sync(p);
}

template <uint32_t W>
__global__ void __launch_bounds__(kVsThreads, 2) vs_bfs_kernel(VsParams p) {
  __shared__ VsStage stage[kVsWarps];
  __shared__ unsigned long long sdig[kMaxVersions];
  VsCounters* c = p.c;
  VsSums s;
  if (threadIdx.x == 0) {
    vs_bq.cnt = 0;
    vs_mf = 0;
  }
  for (uint32_t i = threadIdx.x; i < p.K; i += blockDim.x) sdig[i] = 0ull;
  // the source is reached at the window's start (the object's distances are
  // still the pre-window ones here)
  if (gtid() == 0) c->seed = p.source < p.len0 && p.dist[p.source] == 0u ? 1u : 0u;
  if (!vs_sync(p)) return;
  const bool seed = __ldcg(&c->seed) != 0u;
  // the distance vector starts unreachable; every vertex's unreachable digest
  // term goes to the first version whose distance vector covers it
  unsigned long long base0 = 0;
  for (uint32_t v = gtid(); v < p.V; v += nthreads()) {
    p.dist[v] = kUnreachable;
    if (!p.dig) continue;
    const unsigned long long h = vxb::mix64(((unsigned long long)v << 32) | kUnreachable);
    if (v < p.vlen[0]) {
      base0 += h;
    } else {
      uint32_t lo = 0, hi = p.K;  // first version b with vlen[b] > v: vlen[lo] <= v < vlen[hi]
      while (hi - lo > 1) {
        const uint32_t mid = (lo + hi) >> 1;
        if (p.vlen[mid] <= v) lo = mid;
        else hi = mid;
      }
      if (hi < p.K) atomicAdd(&p.bucket[hi], h);
    }
  }
  if (!vs_sync(p)) return;
  if (seed && gtid() == 0) {
    uint32_t zero[W], all[W];
#pragma unroll
    for (uint32_t w = 0; w < W; ++w) {
      zero[w] = 0u;
      all[w] = vmask(p.K, w);
    }
    vs_discover<W>(p, p.source, zero, all, p.frn[0], 0, s);
    if (p.dig)
      s.common += vxb::mix64((unsigned long long)p.source << 32) -
                  vxb::mix64(((unsigned long long)p.source << 32) | kUnreachable);
    p.q[0][0] = p.source;
    c->qn[0] = 1;
    const VsRow r = vs_row(p, p.source);
    c->mf[0] = r.nb + r.dy + r.tn;
  }
  if (!vs_sync(p)) return;
  uint32_t prev_n = 0, level = 0;
  for (;; ++level) {
    if (level > p.V + 1) {
      if (gtid() == 0) atomicOr(&c->err, vxb::kErrLoopBound);
      break;
    }
    const int cur = level % 3, nx = (level + 1) % 3, clr = (level + 2) % 3;
    const uint32_t n_f = __ldcg(&c->qn[cur]);
    if (n_f == 0) break;
    if (gtid() == 0) {  // counters of level + 2: no block uses them before the next barrier
      c->qn[clr] = 0;
      c->tn[clr] = 0;
      c->nbig[clr] = 0;
      c->gnext[clr] = 0;
      c->mf[clr] = 0;
    }
    // frontier words of level - 1 are no longer read: cleared through its
    // queue when it was small, else all of them
    if ((unsigned long long)prev_n * 8 < p.V) {
      for (uint32_t i = gtid(); i < prev_n * W; i += nthreads()) p.frn[clr][(size_t)p.q[clr][i / W] * W + i % W] = 0u;
    } else {
      for (size_t i = gtid(); i < (size_t)p.V * W; i += nthreads()) p.frn[clr][i] = 0u;
    }
    const uint32_t* fc = p.frn[cur];
    uint32_t* fn = p.frn[nx];
    // pull for a large frontier, or for one whose rows would cost more to
    // push than reading up to every arc costs to pull
    const bool pull = (float)n_f > p.pull_frac * (float)p.V || __ldcg(&c->mf[cur]) * kPushArcCost > p.arcs;
    if (gtid() == 0) {
      const uint32_t t = min(level, 63u);
      c->trace[2 * t] = globaltimer();
      c->trace[2 * t + 1] = (unsigned long long)n_f | ((unsigned long long)pull << 63);
    }
    bool ok;
    if (pull)
      ok = vs_pull<W>(p, fc, fn, level, &c->gnext[cur], &c->nbig[cur], &c->qn[nx], p.q[nx], &c->mf[nx],
                      stage[threadIdx.x >> 5], s, sdig);
    else
      ok = vs_push<W>(p, fc, fn, level, n_f, p.q[cur], &c->tn[cur], &c->nbig[cur], &c->qn[nx], p.q[nx], &c->mf[nx],
                      s, sdig);
    if (!ok) return;
    prev_n = n_f;
  }
  if (gtid() == 0) {
    c->levels = level;
    c->trace[2 * min(level, 64u)] = globaltimer();
  }
  // per-thread sums, then the block's per-version digest deltas
  const unsigned long long common = vxb::warp_sum(s.common), reach = vxb::warp_sum(s.reach),
                           b0 = vxb::warp_sum(base0);
  if ((threadIdx.x & 31) == 0) {
    if (common) atomicAdd(&c->common, common);
    if (reach) atomicAdd(&c->reach, reach);
    if (b0) atomicAdd(&p.bucket[0], b0);
  }
  __syncthreads();
  if (p.dig)
    for (uint32_t i = threadIdx.x; i < p.K; i += blockDim.x)
      if (sdig[i]) atomicAdd(&p.dig[i], sdig[i]);
}

}  // namespace

// ----------------------------------------------------------------- host --

void VersionBufs::free_all() {
  // every pointer is freed and cleared in place (the destructor calls this,
  // so no temporary VersionBufs may be made here)
  void** ptrs[] = {(void**)&keys, (void**)&keys_alt, (void**)&vals,   (void**)&vals_alt, (void**)&flag,
                   (void**)&pos,  (void**)&tu,       (void**)&tx,     (void**)&tmask,    (void**)&tpre,
                   (void**)&trow, (void**)&boff,     (void**)&vlen,   (void**)&vis,      (void**)&frn[0],
                   (void**)&frn[1], (void**)&frn[2], (void**)&nxt,    (void**)&touched,  (void**)&q[0],
                   (void**)&q[1], (void**)&q[2],     (void**)&tl,     (void**)&big,      (void**)&biglen,
                   (void**)&dig,
                   (void**)&bucket, (void**)&ctr,    (void**)&barrier};
  for (void** x : ptrs) {
    cudaFree(*x);
    *x = nullptr;
  }
  cudaFreeHost(hctr);
  cudaFreeHost(hdig);
  hctr = nullptr;
  hdig = nullptr;
  ops_cap = v_cap = w = k_cap = 0;
}

int VersionBufs::ensure(size_t ops, size_t V, size_t words, size_t k) {
  if (ops <= ops_cap && V <= v_cap && words <= w && k <= k_cap) return 0;
  const size_t N = std::max(ops, ops_cap), NV = std::max(V, v_cap), NW = std::max(words, w),
               NK = std::max(k, k_cap);
  free_all();
  const size_t m = 2 * std::max<size_t>(N, 1), vw = std::max<size_t>(NV, 1) * NW, bw = NV / 32 + 1;
  bool ok = true;
  auto al = [&](auto** q_, size_t count, size_t size) {
    if (ok && cudaMalloc((void**)q_, std::max<size_t>(count, 1) * size) != cudaSuccess) ok = false;
  };
  al(&keys, m, 8);
  al(&keys_alt, m, 8);
  al(&vals, m, 4);
  al(&vals_alt, m, 4);
  al(&flag, m, 4);
  al(&pos, m, 4);
  al(&tu, m, 4);
  al(&tx, m, 4);
  al(&tmask, m * NW, 4);
  al(&tpre, bw, 4);
  al(&trow, NV, 8);
  al(&boff, NK + 1, 4);
  al(&vlen, NK, 4);
  al(&vis, vw, 4);
  for (int i = 0; i < 3; ++i) {
    al(&frn[i], vw, 4);
    al(&q[i], NV, 4);
  }
  al(&nxt, vw, 4);
  al(&touched, bw, 4);
  al(&tl, NV, 4);
  al(&big, NV, 4);
  al(&biglen, NV, 4);
  al(&dig, NK, 8);
  al(&bucket, NK, 8);
  al(&ctr, 1, sizeof(VsCounters));
  al(&barrier, vxb::kBarrierWords, 4);
  if (ok && (cudaMallocHost(&hctr, sizeof(VsCounters)) != cudaSuccess ||
             cudaMallocHost(&hdig, 2 * NK * 8) != cudaSuccess))
    ok = false;
  if (!ok) {
    free_all();
    set_error("version-parallel stream: allocation failed (%zu ops, %zu vertices)", N, NV);
    return -4;
  }
  ops_cap = N;
  v_cap = NV;
  w = NW;
  k_cap = NK;
  return 0;
}

namespace {

template <uint32_t W>
int launch_versions(VersionBufs& S, VsParams& p, int slot, cudaStream_t st) {
  const void* kern = (const void*)vs_bfs_kernel<W>;
  if (!S.grid[slot]) {
    int per_sm = 0;
    VX_CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, kVsThreads, 0));
    if (per_sm < 1) {
      set_error("version-parallel BFS kernel cannot be resident on an SM");
      return -3;
    }
    S.grid[slot] = per_sm * sm_count();
  }
  p.nblocks = (uint32_t)S.grid[slot];
  void* args[] = {&p};
  count_launch();
  VX_CUDA_TRY(cudaLaunchCooperativeKernel(kern, dim3(p.nblocks), dim3(kVsThreads), args, 0, st));
  return 0;
}

template <uint32_t W>
void launch_masks(VersionBufs& S, BatchBuffers& B, const vxb::DevAdj& a, const uint64_t* keys, const uint32_t* vals,
                  size_t m, const uint8_t* add, uint32_t K, int bbits, unsigned grid, cudaStream_t st) {
  count_launch();
  vs_mask_kernel<W><<<grid, 256, 0, st>>>(a, keys, vals, S.flag, S.pos, m, add, K, bbits, S.tu, S.tx, S.tmask,
                                          S.tpre, B.fu, B.fv, B.ff, B.fpos);
}

}  // namespace

static uint32_t version_words(size_t k) { return k <= 32 ? 1 : k <= 64 ? 2 : k <= 128 ? 4 : 8; }

int stream_versions_reserve(Bfs* b, size_t ops, size_t V, size_t k) {
  k = std::min<size_t>(std::max<size_t>(k, 1), kMaxVersions);
  if (!b->vb) b->vb = new VersionBufs();
  if (int rc = b->vb->ensure(ops, std::max<size_t>(V, 1), version_words(k), k)) return rc;
  return b->g->batch.ensure(ops);
}

int stream_versions_trace(Bfs* b, unsigned long long* out, size_t cap, size_t* n) {
  *n = 0;
  if (!b->vb || !b->vb->hctr) return 0;
  const VsCounters& c = *b->vb->hctr;
  const uint32_t levels = std::min<uint32_t>(c.levels, 64);
  if (!levels) return 0;
  *n = 2 * (size_t)levels + 1;
  for (size_t i = 0; i < std::min(cap, *n); ++i) out[i] = i + 1 == *n ? c.trace[2 * levels] : c.trace[i];
  return 0;
}

int stream_versions(Bfs* b, const uint32_t* d_src, const uint32_t* d_dst, const uint8_t* d_add, const uint64_t* hoff,
                    const uint32_t* vpost, size_t t0, size_t t1, uint64_t* digests) {
  Graph* g = b->g;
  cudaStream_t st = g->stream;
  const size_t k = t1 - t0;
  if (g->directed || k == 0 || k > kMaxVersions) {
    set_error("version-parallel stream: undirected graphs, 1..%u batches per window", kMaxVersions);
    return -1;
  }
  const size_t o0 = hoff[t0], n = hoff[t1] - hoff[t0];
  const size_t len0 = b->dist_len;
  const size_t V = std::max<size_t>(len0, vpost[t1 - 1]);
  const uint32_t words = version_words(k);
  const int slot = words == 1 ? 0 : words == 2 ? 1 : words == 4 ? 2 : 3;
  int bbits = 1;
  while (bbits < 32 && ((size_t)1 << bbits) < std::max<size_t>(V, 2)) ++bbits;
  if (2 * bbits + kVsTBits > 64) {
    set_error("version-parallel stream: vertex ids too wide for the sort keys");
    return -2;
  }
  size_t nonempty = 0;
  std::vector<uint32_t> hb(k + 1), hl(k);
  for (size_t t = 0; t < k; ++t) {
    hb[t] = (uint32_t)(hoff[t0 + t] - o0);
    hl[t] = (uint32_t)std::max<size_t>(len0, vpost[t0 + t]);
    if (hoff[t0 + t + 1] > hoff[t0 + t]) ++nonempty;
  }
  hb[k] = (uint32_t)n;
  // arena room for the merged commit (a consolidation, if one is due, comes
  // here, before anything reads the pre-window layout) and the window's new
  // vertices (empty rows at its start)
  if (int rc = g->batch.ensure(std::max<size_t>(n, 1))) return rc;
  if (int rc = graph_prepare_batch(g, n, vpost[t1 - 1])) return rc;
  if (int rc = bfs_ensure_capacity(b, std::max<size_t>(V, 1))) return rc;
  if (!b->vb) b->vb = new VersionBufs();
  VersionBufs& S = *b->vb;
  if (int rc = S.ensure(n, V, words, k)) return rc;
  VX_CUDA_TRY(cudaMemcpyAsync(S.boff, hb.data(), (k + 1) * 4, cudaMemcpyHostToDevice, st));
  VX_CUDA_TRY(cudaMemcpyAsync(S.vlen, hl.data(), k * 4, cudaMemcpyHostToDevice, st));
  VX_CUDA_TRY(cudaMemsetAsync(S.ctr, 0, sizeof(VsCounters), st));
  VX_CUDA_TRY(cudaMemsetAsync(S.trow, 0, V * 8, st));
  VX_CUDA_TRY(cudaMemsetAsync(S.tpre, 0, (V / 32 + 1) * 4, st));
  const size_t vw = V * words;
  VX_CUDA_TRY(cudaMemsetAsync(S.vis, 0, vw * 4, st));
  VX_CUDA_TRY(cudaMemsetAsync(S.nxt, 0, vw * 4, st));
  for (int i = 0; i < 3; ++i) VX_CUDA_TRY(cudaMemsetAsync(S.frn[i], 0, vw * 4, st));
  VX_CUDA_TRY(cudaMemsetAsync(S.touched, 0, (V / 32 + 1) * 4, st));
  VX_CUDA_TRY(cudaMemsetAsync(S.barrier, 0, vxb::kBarrierWords * 4, st));
  if (digests) {
    VX_CUDA_TRY(cudaMemsetAsync(S.dig, 0, k * 8, st));
    VX_CUDA_TRY(cudaMemsetAsync(S.bucket, 0, k * 8, st));
  }
  const vxb::DevAdj a = g->view().out;
  uint64_t* keys = S.keys;
  uint32_t* vals = S.vals;
  const size_t m = 2 * n;
  if (n) {
    const unsigned gn = (unsigned)std::max<size_t>(1, std::min<size_t>((n + 255) / 256, (size_t)sm_count() * 32));
    const unsigned gm = (unsigned)std::max<size_t>(1, std::min<size_t>((m + 255) / 256, (size_t)sm_count() * 32));
    count_launch();
    vs_keys_kernel<<<gn, 256, 0, st>>>(d_src + o0, d_dst + o0, n, S.boff, (uint32_t)k, bbits, S.keys, S.vals);
    VX_CUDA_TRY(cudaGetLastError());
    bool in_alt = false;
    if (int rc = radix_sort_u64(S.keys, S.keys_alt, S.vals, S.vals_alt, m, 2 * bbits + kVsTBits, &in_alt,
                                g->scratch, st))
      return rc;
    keys = in_alt ? S.keys_alt : S.keys;
    vals = in_alt ? S.vals_alt : S.vals;
    count_launch();
    vs_runs_kernel<<<gm, 256, 0, st>>>(keys, m, S.flag);
    if (int rc = scan_exclusive_u32(S.flag, S.pos, m, &S.ctr->runs, g->scratch, st)) return rc;
    VX_CUDA_TRY(cudaMemcpyAsync(&g->ctr->final_arcs, &S.ctr->runs, 4, cudaMemcpyDeviceToDevice, st));
    switch (words) {
      case 1: launch_masks<1>(S, g->batch, a, keys, vals, m, d_add + o0, (uint32_t)k, bbits, gm, st); break;
      case 2: launch_masks<2>(S, g->batch, a, keys, vals, m, d_add + o0, (uint32_t)k, bbits, gm, st); break;
      case 4: launch_masks<4>(S, g->batch, a, keys, vals, m, d_add + o0, (uint32_t)k, bbits, gm, st); break;
      default: launch_masks<8>(S, g->batch, a, keys, vals, m, d_add + o0, (uint32_t)k, bbits, gm, st); break;
    }
    count_launch();
    vs_rows_kernel<<<gm, 256, 0, st>>>(S.tu, &S.ctr->runs, S.trow);
    VX_CUDA_TRY(cudaGetLastError());
  }
  VsParams p;
  memset(&p, 0, sizeof(p));
  p.a = a;
  p.V = (uint32_t)V;
  p.K = (uint32_t)k;
  p.source = b->source;
  p.len0 = (uint32_t)len0;
  p.tx = S.tx;
  p.tmask = S.tmask;
  p.trow = S.trow;
  p.tpre = S.tpre;
  p.vlen = S.vlen;
  p.dist = b->dist;
  p.vis = S.vis;
  for (int i = 0; i < 3; ++i) {
    p.frn[i] = S.frn[i];
    p.q[i] = S.q[i];
  }
  p.nxt = S.nxt;
  p.touched = S.touched;
  p.tl = S.tl;
  p.big = S.big;
  p.biglen = S.biglen;
  p.dig = digests ? S.dig : nullptr;
  p.bucket = S.bucket;
  p.c = S.ctr;
  p.bar = S.barrier;
  p.pull_frac = b->tune.window_pull_frac;
  p.arcs = g->adj[0].A;
  int rc = 0;
  switch (words) {
    case 1: rc = launch_versions<1>(S, p, slot, st); break;
    case 2: rc = launch_versions<2>(S, p, slot, st); break;
    case 4: rc = launch_versions<4>(S, p, slot, st); break;
    default: rc = launch_versions<8>(S, p, slot, st); break;
  }
  if (rc) return rc;
  // the object's state: the last version's distances (written by the
  // launch), its reachable count, and no repair counters of its own
  VX_CUDA_TRY(cudaMemcpyAsync(&b->ctr->reachable, &S.ctr->reach, 8, cudaMemcpyDeviceToDevice, st));
  VX_CUDA_TRY(cudaMemsetAsync(&b->ctr->candidates, 0, 4 * sizeof(uint32_t), st));
  b->dist_len = V;
  // the window's ops as one batch, staged by the mask kernel: the last op per
  // edge decides its final state, as applying the batches in order does; the
  // version counter advances once per non-empty batch
  if (n) {
    if (int rc2 = graph_commit_batch(g)) return rc2;
    g->version += nonempty - 1;
  }
  VX_CUDA_TRY(cudaMemcpyAsync(S.hctr, S.ctr, sizeof(VsCounters), cudaMemcpyDeviceToHost, st));
  if (digests) {
    VX_CUDA_TRY(cudaMemcpyAsync(S.hdig, S.dig, k * 8, cudaMemcpyDeviceToHost, st));
    VX_CUDA_TRY(cudaMemcpyAsync(S.hdig + k, S.bucket, k * 8, cudaMemcpyDeviceToHost, st));
  }
  VX_CUDA_TRY(cudaStreamSynchronize(st));
  if (S.hctr->err) {
    set_error("version-parallel stream: device error word 0x%x", S.hctr->err);
    return -5;
  }
  if (digests) {
    // both per-version arrays are difference arrays: prefix sums
    unsigned long long base = 0, delta = 0;
    for (size_t t = 0; t < k; ++t) {
      base += S.hdig[k + t];
      delta += S.hdig[t];
      digests[t0 + t] = base + delta + S.hctr->common;
    }
  }
  return 0;
}

}  // namespace vxh
