// Multi-root BFS: up to 256 independent BFS traversals in one persistent
// cooperative launch, bit-parallel over the roots.
//
// Every vertex carries W = ceil(K/32) words of "reached by root r" bits and
// rotating frontier words; a level expands all roots at once, so each row is
// read once per level instead of once per root.  Sparse levels push the
// frontier words of the queued vertices along their rows (atomicOr into the
// next-level words of the heads, heads queued once through a touched bitmap);
// dense levels pull: every vertex not yet reached by all roots ORs the
// frontier words of its in-neighbours and stops as soon as every root has
// reached it.  Distances are written as dist[r * V + v]; for every root they
// equal BasicIncrementalBFS::recompute (include/velographx/incremental/bfs.hpp:100-120)
// from that root, and the reference's multicore harness
// (benchmarks/thread_scaling_bfs.cpp:78-108) runs the same roots one thread each.
#include <algorithm>
#include <cstring>

#include "frontier.cuh"
#include "graph.cuh"
#include "mrbfs.cuh"

namespace vxh {

namespace {

using namespace frontier;

constexpr int kThreads = 512;

// The block's staging of frontier and touched-list appends: one global
// atomic per block per phase instead of one per warp step (the appends of a
// level that reaches millions of vertices serialised on one counter).
__shared__ BlockQueue mr_bq;
// The block's sum of the out-degrees of the vertices it adds to the next
// frontier (the push cost of the next level).
__shared__ unsigned long long mr_mf;

// A level pulls when pushing its frontier's rows would cost more than this
// many times fewer arcs than the graph holds: a pushed arc (a visited check,
// a next-word check, an atomic) costs about this many pulled arcs.
constexpr unsigned long long kPushArcCost = 12;

// Block-uniform: the block's frontier-degree sum added to *dst.
__device__ __forceinline__ void mf_flush(unsigned long long* dst) {
  __syncthreads();
  if (threadIdx.x == 0 && mr_mf) {
    atomicAdd(dst, mr_mf);
    mr_mf = 0;
  }
  __syncthreads();
}

struct MrParams {
  vxb::DevGraph g;
  uint32_t V, K, W;
  const uint32_t* roots;
  uint32_t* vis;     // [V][W]
  uint32_t* frn[3];  // [V][W] rotating frontier words
  uint32_t* nxt;     // [V][W] pushed words of the level being built
  uint32_t* touched; // bitmap
  uint32_t* q[3];    // rotating frontier queues
  uint32_t* tl;      // touched list of a push level
  uint32_t* big;     // rows of a level that the whole grid reads
  uint32_t* biglen;  // their lengths
  uint32_t* dist;    // [K][V]
  MrCounters* c;
  uint32_t* bar;
  uint32_t nblocks;
  float pull_frac;   // pull when the frontier holds more than V * pull_frac vertices
  unsigned long long arcs;  // arcs of the graph (a pull level reads up to all of them)
};

__device__ __forceinline__ bool mr_sync(const MrParams& p) {
  vxb::grid_barrier(p.bar, p.nblocks, &p.c->err);
  return __ldcg(&p.c->err) == 0u;
}

__device__ __forceinline__ uint32_t word_mask(const MrParams& p, uint32_t w) {
  const uint32_t rem = p.K - 32 * w;
  return rem >= 32 ? 0xFFFFFFFFu : ((1u << rem) - 1u);
}

// Record newly reached roots of v at distance lvl; returns whether any.
__device__ __forceinline__ void write_dists(const MrParams& p, uint32_t v, uint32_t w, uint32_t bits, uint32_t lvl) {
  while (bits) {
    const uint32_t b = __ffs(bits) - 1;
    bits &= bits - 1;
    p.dist[(size_t)(32 * w + b) * p.V + v] = lvl;
  }
}

// Push: the warp walks the row of frontier vertex u with u's frontier words
// in registers.  W (words per vertex) is a compile-time constant so the
// per-vertex word arrays stay in registers.
template <uint32_t W>
struct PushVisit {
  const MrParams* p;
  uint32_t fw[W];
  uint32_t* tcount;
  __device__ __forceinline__ void operator()(bool valid, uint32_t x, uint32_t) {
    bool fresh = false;
    if (valid) {
      // a head's bits are read before they are OR-ed in: a hub that many
      // frontier rows reach takes one atomic per new bit, not one per arc
      // (the thread whose atomic added bits lists the head)
      bool any = false;
      uint32_t vx[W];
      load_words<W>(p->vis + (size_t)x * W, vx);
#pragma unroll
      for (uint32_t w = 0; w < W; ++w) {
        uint32_t m = fw[w] & ~vx[w];
        if (m) m &= ~__ldcg(&p->nxt[(size_t)x * W + w]);
        if (m) {
          atomicOr(&p->nxt[(size_t)x * W + w], m);
          any = true;
        }
      }
      if (any) {
        const uint32_t bit = 1u << (x & 31);
        fresh = !(__ldcg(&p->touched[x >> 5]) & bit) && !(atomicOr(&p->touched[x >> 5], bit) & bit);
      }
    }
    bq_push(mr_bq, fresh, x, tcount, p->tl);
  }
};

// arc slots a lane loads per round of a pull group (fewer when every arc
// brings more frontier words into registers)
template <uint32_t W>
struct MrSlots {
  static constexpr uint32_t value = W <= 2 ? 8 : 4;
};
constexpr uint32_t kMrHead = 8;          // in-arcs a lane reads itself before the flattened rounds
constexpr uint32_t kMrHeadStep = 4;      // of which it loads this many at a time
constexpr uint32_t kMrBigRow = 1024;     // push rows this long are expanded by the whole grid
constexpr uint32_t kMrPushSlice = 128;   // arcs of a hub row a warp takes at a time
constexpr uint32_t kMrBigPull = 2048;    // pull rows this long are read by the whole grid
constexpr uint32_t kMrWarps = kThreads / 32;
// 32-vertex groups a warp claims per atomic of a pull level (one counter
// per level: a claim per group serialised on it)
constexpr uint32_t kClaimGroups = 4;

// Per-warp staging of one pull group: the rows of its 32 vertices and their
// OR accumulators ([lane][word]).
struct MrWarpStage {
  uint64_t rb[32];
  uint32_t nb[32];
  uint32_t dx[32];
  uint32_t acc[32 * 8];
};

// Newly reached roots of the warp's 32 consecutive vertices (v = base + lane)
// at distance lvl, one root at a time, so every store of a root's row covers
// the warp's vertices together.
template <uint32_t W>
__device__ __forceinline__ void write_dists_warp(const MrParams& p, uint32_t v, const uint32_t* acc, uint32_t lvl) {
#pragma unroll
  for (uint32_t w = 0; w < W; ++w) {
    uint32_t roots = __reduce_or_sync(FULL, acc[w]);
    while (roots) {
      const uint32_t b = __ffs(roots) - 1;
      roots &= roots - 1;
      if ((acc[w] >> b) & 1u) p.dist[(size_t)(32 * w + b) * p.V + v] = lvl;
    }
  }
}

// Pull level.  Warps take groups of 32 consecutive vertices from a counter.
// The in-rows of a group's vertices that some root has not reached yet are
// read as one flattened arc list: each round, every lane loads MrSlots<W> arcs (a
// lane finds the owner of its arc by a binary search over the group's
// inclusive row ends), then their frontier words, and ORs them into the
// owner's accumulator in shared memory; an owner that every root has reached
// stops being read.  Rows of kMrBigPull arcs or more are listed and read by
// the whole grid afterwards, with the words OR-ed into nxt (zero outside push
// levels).  Ends with a grid barrier; returns false when one failed.
template <uint32_t W>
__device__ bool pull_level(const MrParams& p, const uint32_t* fc, uint32_t* fn, uint32_t level, uint32_t* gnext,
                           uint32_t* nbig, uint32_t* qn, uint32_t* qout, unsigned long long* mf, MrWarpStage& ws) {
  constexpr uint32_t kMrU = MrSlots<W>::value;
  const DevAdj& a = p.g.in;
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
      vis[w] = v < p.V ? p.vis[(size_t)v * W + w] : word_mask(p, w);
      done = done && vis[w] == word_mask(p, w);
      ws.acc[lane * W + w] = 0u;
    }
    uint32_t len = 0, rowlen = 0;
    if (!done) {
      uint64_t b, e;
      vxb::base_range(a, v, b, e);
      const uint2 dr = a.drow[v];
      const uint32_t nb = (uint32_t)(e - b);
      len = nb + dr.y;
      rowlen = len;
      if (len >= kMrBigPull) {  // the whole grid reads it after the barrier
        const uint32_t slot = atomicAdd(nbig, 1u);
        p.big[slot] = v;
        p.biglen[slot] = len;
        len = 0;
      }
      ws.rb[lane] = b;
      ws.nb[lane] = nb;
      ws.dx[lane] = dr.x;
      // head: the lane first reads the first kMrHead arcs of its own row,
      // kMrHeadStep loads in flight, and stops as soon as every root has
      // reached its vertex; the flattened rounds below read the rest
      const uint32_t hn = min(len, kMrHead);
      uint32_t hacc[W];
#pragma unroll
      for (uint32_t w = 0; w < W; ++w) hacc[w] = 0u;
      for (uint32_t h0 = 0; h0 < hn; h0 += kMrHeadStep) {
        uint32_t hx[kMrHeadStep];
#pragma unroll
        for (uint32_t k = 0; k < kMrHeadStep; ++k) {
          const uint32_t j = h0 + k;
          hx[k] = j >= hn ? kTomb : (j < nb ? a.col[b + j] : a.darena[dr.x + (j - nb)]);
        }
#pragma unroll
        for (uint32_t k = 0; k < kMrHeadStep; ++k) {
          if (hx[k] & kTomb) continue;
          uint32_t f[W];
          load_words<W>(fc + (size_t)hx[k] * W, f);
#pragma unroll
          for (uint32_t w = 0; w < W; ++w) hacc[w] |= f[w];
        }
        bool fin = true;
#pragma unroll
        for (uint32_t w = 0; w < W; ++w) fin = fin && (vis[w] | hacc[w]) == word_mask(p, w);
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
    for (uint32_t j0 = 0; j0 < T && active; j0 += 32 * kMrU) {
      uint32_t x[kMrU], own[kMrU];
#pragma unroll
      for (uint32_t u = 0; u < kMrU; ++u) {
        const uint32_t j = j0 + u * 32 + lane;
        // owner = lanes whose row ends at or before j; the last end found is
        // where the owner's row starts in the flattened list
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
        if (j < T && ((active >> o) & 1u)) {
          const uint32_t k = kMrHead + (j - lo), nbo = ws.nb[o];  // past the owner's head
          x[u] = k < nbo ? a.col[ws.rb[o] + k] : a.darena[ws.dx[o] + (k - nbo)];
        }
      }
      uint32_t m[kMrU][W];
#pragma unroll
      for (uint32_t u = 0; u < kMrU; ++u) {
        if (x[u] & kTomb) {
#pragma unroll
          for (uint32_t w = 0; w < W; ++w) m[u][w] = 0u;
        } else {
          load_words<W>(fc + (size_t)x[u] * W, m[u]);
        }
      }
#pragma unroll
      for (uint32_t u = 0; u < kMrU; ++u)
#pragma unroll
        for (uint32_t w = 0; w < W; ++w)
          if (m[u][w]) atomicOr(&ws.acc[own[u] * W + w], m[u][w]);
      __syncwarp();
      bool fin = false;
      if ((active >> lane) & 1u) {
        fin = true;
#pragma unroll
        for (uint32_t w = 0; w < W; ++w) fin = fin && (vis[w] | ws.acc[lane * W + w]) == word_mask(p, w);
      }
      active &= ~__ballot_sync(FULL, fin);
    }
    __syncwarp();
    uint32_t acc[W];
    bool any = false;
#pragma unroll
    for (uint32_t w = 0; w < W; ++w) {
      acc[w] = ws.acc[lane * W + w] & ~vis[w];
      if (acc[w]) {
        any = true;
        p.vis[(size_t)v * W + w] = vis[w] | acc[w];
        fn[(size_t)v * W + w] = acc[w];
      }
    }
    write_dists_warp<W>(p, v, acc, level + 1);
    bq_push(mr_bq, any, v, qn, qout);
    const unsigned long long dsum = vxb::warp_sum(any ? (unsigned long long)rowlen : 0ull);
    if (lane == 0 && dsum) atomicAdd(&mr_mf, dsum);
    __syncwarp();  // the next group overwrites the stage
  }
  bq_flush(mr_bq, qn, qout);
  mf_flush(mf);
  if (!mr_sync(p)) return false;
  const uint32_t nb = __ldcg(nbig);
  if (nb == 0) return true;
  // long rows: every warp takes 32 * MrSlots<W>-arc slices; the slices of row r
  // start at warp r (mod the warp count) so the rows spread over the grid.  A
  // warp skips, from the listed length alone, the rows it has no slice of.
  const uint32_t nw = nwarps(), gw = gwarp();
  for_my_rows(p.biglen, nb, 32 * kMrU, [&](uint32_t r, uint32_t, uint32_t) {
    const uint32_t v = p.big[r];
    uint32_t vis[W];
#pragma unroll
    for (uint32_t w = 0; w < W; ++w) vis[w] = __ldcg(&p.vis[(size_t)v * W + w]);
    uint64_t b, e;
    vxb::base_range(a, v, b, e);
    const uint2 dr = a.drow[v];
    const uint32_t nbv = (uint32_t)(e - b), total = nbv + dr.y;
    const uint32_t nslices = (total + 32 * kMrU - 1) / (32 * kMrU);
    for (uint32_t s = (gw + nw - r % nw) % nw; s < nslices; s += nw) {
      bool full = true;
#pragma unroll
      for (uint32_t w = 0; w < W; ++w) full = full && (vis[w] | __ldcg(&p.nxt[(size_t)v * W + w])) == word_mask(p, w);
      if (full) break;
      uint32_t x[kMrU];
#pragma unroll
      for (uint32_t u = 0; u < kMrU; ++u) {
        const uint32_t k = s * 32 * kMrU + u * 32 + lane;
        x[u] = k >= total ? kTomb : (k < nbv ? a.col[b + k] : a.darena[dr.x + (k - nbv)]);
      }
      uint32_t add[W];
#pragma unroll
      for (uint32_t w = 0; w < W; ++w) add[w] = 0u;
#pragma unroll
      for (uint32_t u = 0; u < kMrU; ++u) {
        if (x[u] & kTomb) continue;
        uint32_t f[W];
        load_words<W>(fc + (size_t)x[u] * W, f);
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
  if (!mr_sync(p)) return false;
  for (uint32_t r = gtid(); r < nb; r += nthreads()) {
    const uint32_t v = p.big[r];
    bool any = false;
#pragma unroll
    for (uint32_t w = 0; w < W; ++w) {
      const size_t o = (size_t)v * W + w;
      const uint32_t m = __ldcg(&p.nxt[o]) & ~p.vis[o];
      p.nxt[o] = 0u;
      if (!m) continue;
      any = true;
      p.vis[o] |= m;
      fn[o] = m;
      write_dists(p, v, w, m, level + 1);
    }
    if (any) {
      qout[atomicAdd(qn, 1u)] = v;
      atomicAdd(&mr_mf, (unsigned long long)p.biglen[r]);
    }
  }
  mf_flush(mf);
  return mr_sync(p);
}

template <uint32_t W>
__global__ void __launch_bounds__(kThreads, 2) mrbfs_kernel(MrParams p) {
  __shared__ MrWarpStage stage[kMrWarps];
  MrCounters* c = p.c;
  if (threadIdx.x == 0) {
    mr_bq.cnt = 0;
    mr_mf = 0;
  }
  __syncthreads();
  // roots (queued once per distinct vertex)
  for (uint32_t r = gtid(); r < p.K; r += nthreads()) {
    const uint32_t v = p.roots[r];
    if (v >= p.V) continue;
    atomicOr(&p.vis[(size_t)v * W + r / 32], 1u << (r & 31));
    atomicOr(&p.frn[0][(size_t)v * W + r / 32], 1u << (r & 31));
    p.dist[(size_t)r * p.V + v] = 0;
    const uint32_t bit = 1u << (v & 31);
    if (!(atomicOr(&p.touched[v >> 5], bit) & bit)) {
      p.q[0][atomicAdd(&c->qn[0], 1u)] = v;
      atomicAdd(&c->mf[0], (unsigned long long)degree_of(p.g.out, v));
    }
  }
  if (!mr_sync(p)) return;
  for (uint32_t i = gtid(); i < __ldcg(&c->qn[0]); i += nthreads()) p.touched[p.q[0][i] >> 5] = 0u;
  if (!mr_sync(p)) return;
  uint32_t prev_n = 0;
  uint32_t level = 0;
  for (;; ++level) {
    if (level > p.V + 1) {
      if (gtid() == 0) atomicOr(&c->err, vxb::kErrLoopBound);
      break;
    }
    const int cur = level % 3, nx = (level + 1) % 3, clr = (level + 2) % 3;
    const uint32_t n_f = __ldcg(&c->qn[cur]);
    if (n_f == 0) break;
    if (gtid() == 0) {  // counters of level+2: no block uses them before the next barrier
      c->qn[clr] = 0;
      c->tn[clr] = 0;
      c->nbig[clr] = 0;
      c->gnext[clr] = 0;
      c->mf[clr] = 0;
    }
    // frontier words of level-1 are no longer read: clear them for reuse,
    // through its queue when it was small, else all of them with plain stores
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
      const uint32_t t = min(level, kMrTraceLevels - 1);
      c->trace[2 * t] = globaltimer();
      c->trace[2 * t + 1] = (unsigned long long)n_f | ((unsigned long long)pull << 63);
    }
    if (pull) {
      // pull: every vertex not reached by all roots ORs its in-neighbours'
      // frontier words, stopping once all roots reached it
      if (!pull_level<W>(p, fc, fn, level, &c->gnext[cur], &c->nbig[cur], &c->qn[nx], p.q[nx], &c->mf[nx],
                         stage[threadIdx.x >> 5]))
        return;
    } else {
      // push along the rows of the queued frontier vertices, one warp each
      const DevAdj& a = p.g.out;
      PushVisit<W> pv{&p, {}, &c->tn[cur]};
      for (uint32_t i = gwarp(); i < n_f; i += nwarps()) {
        const uint32_t u = p.q[cur][i];
        const uint32_t deg = degree_of(a, u);
        if (deg >= kMrBigRow) {  // a hub: the whole grid, after the barrier
          if ((threadIdx.x & 31) == 0) {
            const uint32_t slot = atomicAdd(&c->nbig[cur], 1u);
            p.big[slot] = u;
            p.biglen[slot] = deg;
          }
          continue;
        }
#pragma unroll
        for (uint32_t w = 0; w < W; ++w) pv.fw[w] = fc[(size_t)u * W + w];
        warp_row(a, u, pv);
      }
      bq_flush(mr_bq, &c->tn[cur], p.tl);
      if (!mr_sync(p)) return;
      const uint32_t nbig = __ldcg(&c->nbig[cur]);
      // hub rows: kMrPushSlice-arc slices, the slices of row r starting at
      // warp r (mod the warp count); a warp skips the rows it has no slice of
      const uint32_t nw = nwarps();
      for_my_rows(p.biglen, nbig, kMrPushSlice, [&](uint32_t r, uint32_t deg, uint32_t sl) {
        const uint32_t nsl = (deg + kMrPushSlice - 1) / kMrPushSlice;
        const uint32_t u = p.big[r];
#pragma unroll
        for (uint32_t w = 0; w < W; ++w) pv.fw[w] = fc[(size_t)u * W + w];
        uint64_t b, e;
        vxb::base_range(a, u, b, e);
        const uint2 dr = a.drow[u];
        const uint32_t nbv = (uint32_t)(e - b);
        for (; sl < nsl; sl += nw) {
          for (uint32_t k0 = sl * kMrPushSlice; k0 < min(deg, (sl + 1) * kMrPushSlice); k0 += 32) {
            const uint32_t k = k0 + (threadIdx.x & 31);
            uint32_t x = kTomb;
            if (k < nbv) x = a.col[b + k];
            else if (k < deg) x = a.darena[dr.x + (k - nbv)];
            pv(!(x & kTomb), x & kIdMask, u);
          }
        }
      });
      bq_flush(mr_bq, &c->tn[cur], p.tl);
      if (nbig && !mr_sync(p)) return;
      // the touched heads' new roots, in warp-uniform rounds so the next
      // frontier is appended one atomic per warp (per head, the appends of
      // a push level that reaches millions of heads serialised on qn)
      const uint32_t nt = __ldcg(&c->tn[cur]);
      for (uint32_t base = gwarp() * 32; base < nt; base += nwarps() * 32) {
        const uint32_t i = base + (threadIdx.x & 31);
        bool any = false;
        uint32_t x = 0;
        if (i < nt) {
          x = p.tl[i];
          for (uint32_t w = 0; w < W; ++w) {
            const size_t o = (size_t)x * W + w;
            const uint32_t m = p.nxt[o] & ~p.vis[o];
            p.nxt[o] = 0u;
            if (!m) continue;
            any = true;
            p.vis[o] |= m;
            fn[o] = m;
            write_dists(p, x, w, m, level + 1);
          }
          p.touched[x >> 5] = 0u;
        }
        bq_push(mr_bq, any, x, &c->qn[nx], p.q[nx]);
        const unsigned long long dsum = vxb::warp_sum(any ? (unsigned long long)degree_of(p.g.out, x) : 0ull);
        if ((threadIdx.x & 31) == 0 && dsum) atomicAdd(&mr_mf, dsum);
      }
      bq_flush(mr_bq, &c->qn[nx], p.q[nx]);
      mf_flush(&c->mf[nx]);
      if (!mr_sync(p)) return;
    }
    prev_n = n_f;
  }
  if (gtid() == 0) {
    c->levels = level;
    c->trace[2 * min(level, kMrTraceLevels)] = globaltimer();
  }
}

__global__ void mr_arcs_kernel(vxb::DevAdj a, const uint32_t* dist, uint32_t V, uint32_t K,
                               unsigned long long* out) {
  unsigned long long s = 0;
  const size_t total = (size_t)V * K;
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < total; i += (size_t)gridDim.x * blockDim.x) {
    if (dist[i] == kUnreachable) continue;
    const uint32_t v = (uint32_t)(i % V);
    uint64_t b, e;
    vxb::base_range(a, v, b, e);
    s += (e - b) - a.tcnt[v] + a.drow[v].y;
  }
  s = vxb::warp_sum(s);
  if ((threadIdx.x & 31) == 0 && s) atomicAdd(out, s);
}

}  // namespace

int mrbfs_create(MrBfs** out, Graph* g, const uint32_t* host_roots, size_t k) {
  if (k == 0 || k > kMaxRoots) {
    set_error("multi-root BFS takes 1..%u roots", kMaxRoots);
    return -1;
  }
  MrBfs* m = new MrBfs();
  m->g = g;
  m->K = k;
  const size_t words = (k + 31) / 32;
  m->W = words <= 1 ? 1 : words <= 2 ? 2 : words <= 4 ? 4 : 8;  // kernel instantiations
  const size_t V = std::max<size_t>(g->V, 1);
  m->V = V;
  const size_t vw = V * m->W;
  bool ok = cudaMalloc(&m->roots, k * 4) == cudaSuccess && cudaMalloc(&m->vis, vw * 4) == cudaSuccess &&
            cudaMalloc(&m->nxt, vw * 4) == cudaSuccess && cudaMalloc(&m->touched, ((V + 31) / 32) * 4) == cudaSuccess &&
            cudaMalloc(&m->tl, V * 4) == cudaSuccess && cudaMalloc(&m->big, V * 4) == cudaSuccess && cudaMalloc(&m->biglen, V * 4) == cudaSuccess &&
            cudaMalloc(&m->dist, V * k * 4) == cudaSuccess &&
            cudaMalloc(&m->ctr, sizeof(MrCounters)) == cudaSuccess &&
            cudaMalloc(&m->barrier, vxb::kBarrierWords * 4) == cudaSuccess &&
            cudaMallocHost(&m->hctr, sizeof(MrCounters)) == cudaSuccess;
  for (int i = 0; i < 3 && ok; ++i)
    ok = cudaMalloc(&m->frn[i], vw * 4) == cudaSuccess && cudaMalloc(&m->q[i], V * 4) == cudaSuccess;
  if (!ok) {
    set_error("multi-root BFS allocation failed (%zu roots, %zu vertices)", k, V);
    mrbfs_destroy(m);
    return -4;
  }
  cudaMemcpyAsync(m->roots, host_roots, k * 4, cudaMemcpyHostToDevice, g->stream);
  cudaMemsetAsync(m->barrier, 0, vxb::kBarrierWords * 4, g->stream);
  cudaMemsetAsync(m->touched, 0, ((V + 31) / 32) * 4, g->stream);
  *out = m;
  return 0;
}

void mrbfs_destroy(MrBfs* m) {
  if (!m) return;
  if (m->g && m->g->stream) cudaStreamSynchronize(m->g->stream);
  void* ptrs[] = {m->roots, m->vis, m->nxt, m->touched, m->tl, m->big, m->biglen, m->dist, m->ctr, m->barrier,
                  m->frn[0], m->frn[1], m->frn[2], m->q[0], m->q[1], m->q[2]};
  for (void* p : ptrs) cudaFree(p);
  cudaFreeHost(m->hctr);
  delete m;
}

int mrbfs_run(MrBfs* m) {
  Graph* g = m->g;
  cudaStream_t s = g->stream;
  if (g->V != m->V) {
    set_error("graph vertex count changed since the multi-root BFS was created");
    return -1;
  }
  const size_t vw = m->V * m->W;
  VX_CUDA_TRY(cudaMemsetAsync(m->vis, 0, vw * 4, s));
  VX_CUDA_TRY(cudaMemsetAsync(m->nxt, 0, vw * 4, s));
  for (int i = 0; i < 3; ++i) VX_CUDA_TRY(cudaMemsetAsync(m->frn[i], 0, vw * 4, s));
  VX_CUDA_TRY(cudaMemsetAsync(m->dist, 0xFF, m->V * m->K * 4, s));
  VX_CUDA_TRY(cudaMemsetAsync(m->ctr, 0, sizeof(MrCounters), s));
  const void* kern = m->W <= 1 ? (const void*)mrbfs_kernel<1>
                     : m->W <= 2 ? (const void*)mrbfs_kernel<2>
                     : m->W <= 4 ? (const void*)mrbfs_kernel<4>
                                 : (const void*)mrbfs_kernel<8>;
  if (!m->grid) {
    int per_sm = 0;
    VX_CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, kThreads, 0));
    if (per_sm < 1) {
      set_error("multi-root BFS kernel cannot be resident on an SM");
      return -3;
    }
    m->grid = per_sm * sm_count();
  }
  MrParams p;
  memset(&p, 0, sizeof(p));
  p.g = g->view();
  p.V = (uint32_t)m->V;
  p.K = (uint32_t)m->K;
  p.W = (uint32_t)m->W;
  p.roots = m->roots;
  p.vis = m->vis;
  for (int i = 0; i < 3; ++i) {
    p.frn[i] = m->frn[i];
    p.q[i] = m->q[i];
  }
  p.nxt = m->nxt;
  p.touched = m->touched;
  p.tl = m->tl;
  p.big = m->big;
  p.biglen = m->biglen;
  p.dist = m->dist;
  p.c = m->ctr;
  p.bar = m->barrier;
  p.nblocks = (uint32_t)m->grid;
  p.pull_frac = m->pull_frac;
  p.arcs = g->adj[0].A;
  void* args[] = {&p};
  count_launch();
  VX_CUDA_TRY(cudaLaunchCooperativeKernel(kern, dim3(m->grid), dim3(kThreads), args, 0, s));
  return 0;
}

int mrbfs_sync(MrBfs* m) {
  cudaStream_t s = m->g->stream;
  VX_CUDA_TRY(cudaMemcpyAsync(m->hctr, m->ctr, sizeof(MrCounters), cudaMemcpyDeviceToHost, s));
  VX_CUDA_TRY(cudaStreamSynchronize(s));
  if (m->hctr->err) {
    set_error("multi-root BFS device error word 0x%x", m->hctr->err);
    return -5;
  }
  return 0;
}

int mrbfs_level_trace(MrBfs* m, unsigned long long* out, size_t cap, size_t* n) {
  if (int rc = mrbfs_sync(m)) return rc;
  const uint32_t levels = std::min<uint32_t>(m->hctr->levels, kMrTraceLevels);
  *n = 2 * (size_t)levels + 1;
  for (size_t i = 0; i < std::min(cap, *n); ++i)
    out[i] = i + 1 == *n ? m->hctr->trace[2 * levels] : m->hctr->trace[i];
  return 0;
}

int mrbfs_reached_arcs(MrBfs* m, unsigned long long* out) {
  cudaStream_t s = m->g->stream;
  unsigned long long* d = &m->ctr->arcs;
  VX_CUDA_TRY(cudaMemsetAsync(d, 0, 8, s));
  count_launch();
  mr_arcs_kernel<<<sm_count() * 8, 256, 0, s>>>(m->g->view().out, m->dist, (uint32_t)m->V, (uint32_t)m->K, d);
  VX_CUDA_TRY(cudaGetLastError());
  if (int rc = mrbfs_sync(m)) return rc;
  *out = m->hctr->arcs;
  return 0;
}

}  // namespace vxh
