// Full BFS and incremental repair as persistent cooperative kernels.
//
// One kernel (bfs_kernel) runs in three modes, all inside a single
// co-resident grid that synchronises with the bounded grid_barrier:
//
//   kModeFull  recompute (bfs.hpp:100-120) as a direction-optimising BFS:
//              top-down levels expand a frontier queue with warp-cooperative
//              gathers (rows < 32 arcs flattened across the warp, medium rows
//              expanded by the whole warp, rows >= tune.large_row expanded by
//              the whole grid), bottom-up levels sweep the visited bitmap a
//              warp per 32 vertices and stop each scan at the first parent in
//              the frontier bitmap.  Claims are atomicOr on the visited bitmap,
//              frontier queues are appended with warp-aggregated atomics.
//   kModePre   the pre-batch part of apply (bfs.hpp:38-70, 222-259): deletion
//              candidates and the support-count fixpoint, level by level in
//              ascending distance order.
//   kModePost  the post-batch part (bfs.hpp:72-97, 261-354): either the
//              fallback full BFS, or invalidate / boundary seed / bucketed
//              settle of the affected vertices followed by insertion relax and
//              decrease propagation.
#include <algorithm>
#include <cstring>

#include "bfs.cuh"
#include "frontier.cuh"

namespace vxh {

using vxb::DevAdj;
using vxb::kIdMask;
using vxb::kTomb;
using vxb::kUnreachable;

namespace {

using namespace frontier;

constexpr int kThreads = 512;
enum { kModeFull = 0, kModePre = 1, kModePost = 2 };

struct Params {
  vxb::DevGraph g;
  uint32_t V;         // vertices of the graph in this phase
  uint32_t dist_len;  // logical length of the distance vector in this phase
  uint32_t source;
  uint32_t* dist;
  uint32_t* vis;
  uint32_t* fb[3];
  uint32_t* q[3];
  uint32_t* big;
  uint32_t* lst_a;
  uint32_t* lst_t;
  uint32_t* old;
  uint32_t* tent;
  uint32_t* lost;
  uint32_t* aff;
  uint32_t* inq[2];
  const uint32_t* fu;
  const uint32_t* fv;
  const uint8_t* ff;
  const uint32_t* F;
  BfsCounters* c;
  unsigned long long total_arcs;
  unsigned long long fallback_limit;
  float alpha, beta;
  uint32_t large_row;
  uint32_t nblocks;
  unsigned long long* trace;  // optional per-level {time, n_f | bottom-up << 63}
  uint32_t* bar;              // grid barrier words
};

constexpr uint32_t kTraceLevels = 256;

// Grid barrier; returns false once any block recorded a device error (a
// barrier that gave up waiting, a loop bound), so every persistent loop ends.
__device__ __forceinline__ bool sync_grid(const Params& p) {
  vxb::grid_barrier(p.bar, p.nblocks, &p.c->err);
  return __ldcg(&p.c->err) == 0u;
}


// ------------------------------------------------------------ top-down --

struct TdVisit {
  const Params* p;
  uint32_t level;
  uint32_t* qout;
  uint32_t* fbn;
  uint32_t* cnt_n;
  bool want_deg;
  unsigned long long mloc;
  BlockQueue* bq;
  // Claim x for the next level (warp-uniform).
  __device__ __forceinline__ void operator()(bool valid, uint32_t x, uint32_t) {
    bool claim = false;
    const uint32_t bit = 1u << (x & 31);
    if (valid) {
      const uint32_t w = p->vis[x >> 5];
      if (!(w & bit)) claim = !(atomicOr(&p->vis[x >> 5], bit) & bit);
    }
    if (claim) {
      p->dist[x] = level + 1;
      atomicOr(&fbn[x >> 5], bit);
      if (want_deg) mloc += degree_of(p->g.out, x);
    }
    bq_push(*bq, claim, x, cnt_n, qout);
  }
  __device__ __forceinline__ void flush(unsigned long long* dst) {
    if (!want_deg) return;
    const unsigned long long sum = vxb::warp_sum(mloc);
    if ((threadIdx.x & 31) == 0 && sum) atomicAdd(dst, sum);
    mloc = 0;
  }
};

__device__ void td_level(const Params& p, TdVisit& t, const uint32_t* qin, uint32_t n_f, uint32_t* cnt_big) {
  const DevAdj& a = p.g.out;
  const int lane = threadIdx.x & 31;
  if (n_f <= nwarps()) {
    // small frontier: one warp per vertex, so no warp walks several rows
    for (uint32_t i = gwarp(); i < n_f; i += nwarps()) {
      const uint32_t u = qin[i];
      const bool big = degree_of(a, u) >= p.large_row;
      if (big) {
        if (lane == 0) p.big[atomicAdd(cnt_big, 1u)] = u;
        continue;
      }
      warp_row(a, u, t);
    }
    return;
  }
  for (uint32_t base = gwarp() * 32; base < n_f; base += nwarps() * 32) {
    const uint32_t i = base + lane;
    const bool act = i < n_f;
    const uint32_t u = act ? qin[i] : 0u;
    uint64_t b = 0, e = 0;
    uint2 dr = make_uint2(0, 0);
    if (act) {
      vxb::base_range(a, u, b, e);
      dr = a.drow[u];
    }
    const bool big = act && (e - b) + dr.y >= p.large_row;
    const uint32_t slot = vxb::warp_append(big, cnt_big);
    if (big) {
      p.big[slot] = u;
      b = e = 0;
      dr = make_uint2(0, 0);
    }
    expand_lanes(a, u, b, e, dr, t);
  }
}

// Top-down expansion of a small frontier (n_f <= kLbMax) as one flat edge
// space: every block stages the frontier's row ranges and their degree prefix
// in shared memory, then each warp takes 32 consecutive edges per step and
// finds their owners by binary search -- the same number of edges per warp
// however skewed the rows are (a 30-vertex frontier of hubs included).
constexpr uint32_t kLbMax = 1024;
struct LbStage {
  uint32_t pref[kLbMax + 1];
  uint64_t base[kLbMax];
  uint32_t blen[kLbMax];
  uint32_t dx[kLbMax];
};

__device__ void td_level_lb(const Params& p, TdVisit& t, const uint32_t* qin, uint32_t n_f, LbStage& st) {
  const DevAdj& a = p.g.out;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  // stage: two frontier entries per thread (blockDim 512 covers kLbMax)
  uint32_t len[2], sum = 0;
#pragma unroll
  for (int h = 0; h < 2; ++h) {
    const uint32_t i = threadIdx.x * 2 + h;
    len[h] = 0;
    if (i < n_f) {
      const uint32_t u = qin[i];
      uint64_t b, e;
      vxb::base_range(a, u, b, e);
      const uint2 dr = a.drow[u];
      st.base[i] = b;
      st.blen[i] = (uint32_t)(e - b);
      st.dx[i] = dr.x;
      len[h] = (uint32_t)(e - b) + dr.y;
    }
    sum += len[h];
  }
  uint32_t incl = sum;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const uint32_t y = __shfl_up_sync(FULL, incl, o);
    if (lane >= o) incl += y;
  }
  __shared__ uint32_t wsum[kThreads / 32];
  if (lane == 31) wsum[warp] = incl;
  __syncthreads();
  if (warp == 0) {
    const uint32_t w = lane < kThreads / 32 ? wsum[lane] : 0u;
    uint32_t wi = w;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const uint32_t y = __shfl_up_sync(FULL, wi, o);
      if (lane >= o) wi += y;
    }
    if (lane < kThreads / 32) wsum[lane] = wi - w;
  }
  __syncthreads();
  uint32_t ex = wsum[warp] + incl - sum;
#pragma unroll
  for (int h = 0; h < 2; ++h) {
    const uint32_t i = threadIdx.x * 2 + h;
    if (i < n_f) st.pref[i] = ex;
    ex += len[h];
  }
  if (threadIdx.x * 2 + 1 == n_f - 1 || (threadIdx.x * 2 == n_f - 1)) st.pref[n_f] = ex;
  __syncthreads();
  const uint32_t M = st.pref[n_f];
  for (uint32_t e0 = gwarp() * 32; e0 < M; e0 += nwarps() * 32) {
    const uint32_t e = e0 + lane;
    bool valid = false;
    uint32_t x = 0;
    if (e < M) {
      uint32_t lo = 0, hi = n_f;  // last i with pref[i] <= e
      while (hi - lo > 1) {
        const uint32_t mid = (lo + hi) >> 1;
        if (st.pref[mid] <= e) lo = mid;
        else hi = mid;
      }
      const uint32_t j = e - st.pref[lo];
      if (j < st.blen[lo]) {
        x = a.col[st.base[lo] + j];
        valid = !(x & kTomb);
        x &= kIdMask;
      } else {
        x = a.darena[st.dx[lo] + (j - st.blen[lo])];
        valid = true;
      }
    }
    t(valid, x, 0u);
  }
  __syncthreads();  // st is reused by the next level
}

// Rows of at least large_row arcs: every warp of the grid takes a slice.
template <class F>
__device__ void grid_rows(const DevAdj& a, const uint32_t* rows, uint32_t n, F& f) {
  const int lane = threadIdx.x & 31;
  for (uint32_t r = 0; r < n; ++r) {
    const uint32_t u = rows[r];
    uint64_t b, e;
    vxb::base_range(a, u, b, e);
    for (uint64_t j0 = b + (uint64_t)gwarp() * 32; j0 < e; j0 += (uint64_t)nwarps() * 32) {
      const uint64_t j = j0 + lane;
      const uint32_t x = j < e ? a.col[j] : kTomb;
      f(!(x & kTomb), x & kIdMask, u);
    }
    const uint2 dr = a.drow[u];
    for (uint32_t j0 = dr.x + gwarp() * 32; j0 < dr.x + dr.y; j0 += nwarps() * 32) {
      const uint32_t j = j0 + lane;
      const bool ok = j < dr.x + dr.y;
      f(ok, ok ? a.darena[j] : 0u, u);
    }
  }
}

// ----------------------------------------------------------- bottom-up --

constexpr uint32_t kBuHead = 8;  // arcs a lane scans itself before the warp helps

// One warp per 32 unvisited-candidate vertices (a visited-bitmap word).  Each
// lane scans the first kBuHead in-arcs of its row; the remainder of longer
// rows is scanned by the whole warp 32 arcs at a time; every scan stops at the
// first parent found in the frontier bitmap.
__device__ void bu_level(const Params& p, uint32_t level, const uint32_t* fbc, uint32_t* fbn, uint32_t* qout,
                         uint32_t* cnt_n, BlockQueue& bq) {
  const DevAdj& a = p.g.in;
  const int lane = threadIdx.x & 31;
  const uint32_t words = (p.V + 31) >> 5;
  for (uint32_t w = gwarp(); w < words; w += nwarps()) {
    const uint32_t visw = p.vis[w];
    if (visw == FULL) continue;
    const uint32_t v = w * 32 + lane;
    const bool todo = !((visw >> lane) & 1u);
    uint64_t b = 0, e = 0;
    uint2 dr = make_uint2(0, 0);
    if (todo) {
      vxb::base_range(a, v, b, e);
      dr = a.drow[v];
    }
    const uint32_t nb = (uint32_t)(e - b), total = nb + dr.y;
    bool found = false;
    // every lane first scans the head of its own row (rows are sorted, and in
    // skewed graphs the hubs that fill the frontier sit at small ids), four
    // independent loads in flight per step
    const uint32_t head = todo ? min(total, kBuHead) : 0u;
    for (uint32_t k = 0; k < head && !found; k += 4) {
      uint32_t x[4];
#pragma unroll
      for (int j = 0; j < 4; ++j) {
        const uint32_t kk = k + j;
        x[j] = kk >= head ? kTomb : (kk < nb ? a.col[b + kk] : a.darena[dr.x + (kk - nb)]);
      }
#pragma unroll
      for (int j = 0; j < 4; ++j) found = found || (!(x[j] & kTomb) && test_bit(fbc, x[j]));
    }
    // the rest of the longer rows: whole warp, 32 arcs per step, early exit
    uint32_t longm = __ballot_sync(FULL, todo && !found && total > head);
    while (longm) {
      const int l = __ffs(longm) - 1;
      longm &= longm - 1;
      const uint64_t bb = __shfl_sync(FULL, b, l);
      const uint32_t nbl = __shfl_sync(FULL, nb, l), tot = __shfl_sync(FULL, total, l);
      const uint32_t dx = __shfl_sync(FULL, dr.x, l);
      bool hit_l = false;
      for (uint32_t k0 = kBuHead; k0 < tot; k0 += 32) {
        const uint32_t k = k0 + lane;
        bool hit = false;
        if (k < tot) {
          const uint32_t x = k < nbl ? a.col[bb + k] : a.darena[dx + (k - nbl)];
          hit = !(x & kTomb) && test_bit(fbc, x);
        }
        if (__any_sync(FULL, hit)) {
          hit_l = true;
          break;
        }
      }
      if (lane == l) found = hit_l;
    }
    const uint32_t newly = __ballot_sync(FULL, found);
    if (found) p.dist[v] = level + 1;
    if (lane == 0 && newly) {
      p.vis[w] = visw | newly;
      fbn[w] = newly;
    }
    bq_push(bq, found, v, cnt_n, qout);
  }
  bq_flush(bq, cnt_n, qout);
}

// ------------------------------------------------------------ full BFS --

__device__ void full_bfs(const Params& p) {
  __shared__ BlockQueue bq;
  __shared__ LbStage lbst;
  BfsCounters* c = p.c;
  if (threadIdx.x == 0) bq.cnt = 0;
  const uint32_t V = p.V;
  const uint32_t words = (V + 31) >> 5;
  for (uint32_t i = gtid(); i < V; i += nthreads()) p.dist[i] = kUnreachable;
  for (uint32_t i = gtid(); i < words; i += nthreads()) {
    // bits past V count as visited so bottom-up never scans them
    const uint32_t lo = i * 32;
    p.vis[i] = (lo + 32 <= V) ? 0u : (FULL << (V - lo));
    p.fb[0][i] = p.fb[1][i] = p.fb[2][i] = 0u;
  }
  if (gtid() == 0) {
    for (int k = 0; k < 3; ++k) {
      c->lvl_n[k] = 0;
      c->lvl_big[k] = 0;
      c->lvl_m[k] = 0;
    }
  }
  if (!sync_grid(p)) return;
  if (p.source >= V) {
    if (gtid() == 0) {
      c->reachable = 0;
      c->levels = 0;
      c->arcs = 0;
    }
    return;
  }
  if (gtid() == 0) {
    const uint32_t s = p.source;
    p.dist[s] = 0;
    p.vis[s >> 5] |= 1u << (s & 31);
    p.fb[0][s >> 5] |= 1u << (s & 31);
    p.q[0][0] = s;
    c->lvl_n[0] = 1;
    c->lvl_m[0] = degree_of(p.g.out, s);
  }
  if (!sync_grid(p)) return;
  unsigned long long m_visited = 0, reached = 0;
  bool bottom_up = false, left_bu = false;
  uint32_t prev_n = 0;
  uint32_t level = 0;
  for (;; ++level) {
    if (level > V + 1) {
      if (gtid() == 0) atomicOr(&c->err, vxb::kErrLoopBound);
      break;
    }
    const int cur = level % 3, nxt = (level + 1) % 3, clr = (level + 2) % 3;
    const uint32_t n_f = ld_cg(&c->lvl_n[cur]);
    const unsigned long long m_f = __ldcg(&c->lvl_m[cur]);
    if (n_f == 0) break;
    reached += n_f;
    m_visited += m_f;
    if (!bottom_up && !left_bu) {
      const unsigned long long m_u = p.total_arcs > m_visited ? p.total_arcs - m_visited : 0ull;
      if ((double)m_f * p.alpha > (double)m_u && level > 0) bottom_up = true;
    } else if (bottom_up && (double)n_f * p.beta < (double)V && n_f < prev_n) {
      bottom_up = false;
      left_bu = true;
    }
    if (gtid() == 0) {
      c->lvl_n[clr] = 0;
      c->lvl_m[clr] = 0;
      c->lvl_big[clr] = 0;
      if (p.trace && level < kTraceLevels) {
        p.trace[2 * level] = globaltimer();
        p.trace[2 * level + 1] = (unsigned long long)n_f | ((unsigned long long)bottom_up << 63);
      }
    }
    // clear the frontier bitmap of level-1 through its queue
    for (uint32_t i = gtid(); i < prev_n; i += nthreads()) p.fb[clr][p.q[clr][i] >> 5] = 0u;
    if (bottom_up) {
      bu_level(p, level, p.fb[cur], p.fb[nxt], p.q[nxt], &c->lvl_n[nxt], bq);
      if (!sync_grid(p)) return;
    } else {
      TdVisit t{&p, level, p.q[nxt], p.fb[nxt], &c->lvl_n[nxt], !left_bu, 0ull, &bq};
      if (n_f <= kLbMax) td_level_lb(p, t, p.q[cur], n_f, lbst);
      else td_level(p, t, p.q[cur], n_f, &c->lvl_big[cur]);
      t.flush(&c->lvl_m[nxt]);
      bq_flush(bq, &c->lvl_n[nxt], p.q[nxt]);
      if (!sync_grid(p)) return;
      const uint32_t nbig = ld_cg(&c->lvl_big[cur]);
      if (nbig) {
        grid_rows(p.g.out, p.big, nbig, t);
        t.flush(&c->lvl_m[nxt]);
        bq_flush(bq, &c->lvl_n[nxt], p.q[nxt]);
        if (!sync_grid(p)) return;
      }
    }
    prev_n = n_f;
  }
  if (gtid() == 0) {
    c->reachable = reached;
    c->levels = level;
    c->arcs = m_visited;
    if (p.trace && level < kTraceLevels) {
      p.trace[2 * level] = globaltimer();
      p.trace[2 * level + 1] = 0;
    }
  }
}

// ------------------------------------------------------------- helpers --

__device__ __forceinline__ bool is_sp(const Params& p, uint32_t u, uint32_t v) {
  if (u >= p.dist_len || v >= p.dist_len) return false;
  const uint32_t du = p.dist[u], dv = p.dist[v];
  return du != kUnreachable && dv != kUnreachable && du + 1 == dv;
}

// Does v (at distance d >= 1) keep a shortest parent: an in-neighbour x at
// distance d-1 that is not affected, in the pre-batch graph minus the batch's
// deletions (already committed)?  Whole warp, stops at the first such parent.
// "v has none" is exactly the reference's lost >= support test
// (bfs.hpp:229-240): lost counts every shortest parent that is deleted or
// affected, each once, and support counts all of them.
__device__ bool warp_has_surviving_parent(const Params& p, uint32_t v, uint32_t d) {
  const DevAdj& a = p.g.in;
  const int lane = threadIdx.x & 31;
  uint64_t b, e;
  vxb::base_range(a, v, b, e);
  const uint2 dr = a.drow[v];
  const uint64_t nb = e - b, total = nb + dr.y;
  for (uint64_t k0 = 0; k0 < total; k0 += 32) {
    const uint64_t k = k0 + lane;
    bool ok = false;
    if (k < total) {
      uint32_t x;
      bool valid = true;
      if (k < nb) {
        x = a.col[b + k];
        valid = !(x & kTomb);
      } else {
        x = a.darena[dr.x + (uint32_t)(k - nb)];
      }
      ok = valid && x < p.dist_len && p.dist[x] + 1 == d && !test_bit(p.aff, x);
    }
    if (__any_sync(FULL, ok)) return true;
  }
  return false;
}

__device__ __forceinline__ void mark_affected(const Params& p, uint32_t v) {
  atomicOr(&p.aff[v >> 5], 1u << (v & 31));
  const uint32_t slot = atomicAdd(&p.c->a_n, 1u);
  p.lst_a[slot] = v;
}

// Children one level deeper of a newly affected vertex become touched.
struct TouchChildren {
  const Params* p;
  uint32_t d;
  uint32_t* plist;
  uint32_t* pcount;
  __device__ __forceinline__ void operator()(bool valid, uint32_t x, uint32_t) {
    bool fresh = false;
    if (valid && x < p->dist_len && p->dist[x] == d + 1) fresh = atomicOr(&p->lost[x], 1u) == 0u;
    const uint32_t s1 = vxb::warp_append(fresh, pcount);
    if (fresh) plist[s1] = x;
    const uint32_t s2 = vxb::warp_append(fresh, &p->c->touched_n);
    if (fresh) p->lst_t[s2] = x;
  }
};

// ------------------------------------------------ long rows of the repair --
// A repair frontier is small, so a hub in it would leave one warp walking
// tens of thousands of arcs while the rest of the grid waits at the next
// barrier.  The warp passes therefore defer rows of at least large_row arcs
// to a list, and the whole grid walks those rows after the barrier.

__device__ __forceinline__ bool defer_row(const Params& p, const DevAdj& a, uint32_t v) {
  return degree_of(a, v) >= p.large_row;
}

// Lane form for expand_lanes callers: a lane whose row is long appends its
// vertex to p.big and hands expand_lanes an empty range instead.
__device__ __forceinline__ void defer_lanes(const Params& p, uint32_t* cnt, bool act, uint32_t u, uint64_t& b,
                                            uint64_t& e, uint2& dr) {
  const bool big = act && (e - b) + dr.y >= p.large_row;
  const uint32_t slot = vxb::warp_append(big, cnt);
  if (big) {
    p.big[slot] = u;
    b = e = 0;
    dr = make_uint2(0, 0);
  }
}

// Surviving-parent test of the deferred vertices p.big[0, nb): every warp scans
// a 32-arc slice of the row per step; found[r] (p.tent, zeroed by the warp
// pass) is set by the first warp that sees a surviving parent, and the others
// stop at their next step.
__device__ void grid_parent_probe(const Params& p, uint32_t nb, uint32_t d) {
  const DevAdj& a = p.g.in;
  const int lane = threadIdx.x & 31;
  for (uint32_t r = 0; r < nb; ++r) {
    const uint32_t v = p.big[r];
    uint64_t b, e;
    vxb::base_range(a, v, b, e);
    const uint2 dr = a.drow[v];
    const uint64_t nbase = e - b, total = nbase + dr.y;
    for (uint64_t k0 = (uint64_t)gwarp() * 32; k0 < total; k0 += (uint64_t)nwarps() * 32) {
      if (ld_cg(&p.tent[r])) break;  // one load for the warp: the break is warp-uniform
      const uint64_t k = k0 + lane;
      bool ok = false;
      if (k < total) {
        uint32_t x;
        bool valid = true;
        if (k < nbase) {
          x = a.col[b + k];
          valid = !(x & kTomb);
        } else {
          x = a.darena[dr.x + (uint32_t)(k - nbase)];
        }
        ok = valid && x < p.dist_len && p.dist[x] + 1 == d && !test_bit(p.aff, x);
      }
      if (__any_sync(FULL, ok)) {
        if (lane == 0) atomicExch(&p.tent[r], 1u);
        break;
      }
    }
  }
}

// --------------------------------------------------- pre-batch fixpoint --

// compute_affected_prebatch (bfs.hpp:222-259) level by level: at distance d
// the touched vertices (deletion candidates at d, children of vertices that
// became affected at d-1) are affected iff no shortest parent survives; the
// children of those at d+1 are touched next.  The fallback limit is checked
// after every level (the affected count only grows).
__device__ void repair_pre(const Params& p) {
  BfsCounters* c = p.c;
  const int lane = threadIdx.x & 31;
  const uint32_t F = *p.F;
  for (uint32_t i = gtid(); i < F; i += nthreads()) {
    const uint8_t f = p.ff[i];
    if ((f & kFAdd) || !(f & kFCur)) continue;
    const uint32_t u = p.fu[i], v = p.fv[i];
    if (!is_sp(p, u, v)) continue;
    if (atomicOr(&p.lost[v], 1u) == 0u) {
      const uint32_t slot = atomicAdd(&c->cand_n, 1u);
      p.lst_t[slot] = v;
    }
  }
  if (gtid() == 0) {
    for (int k = 0; k < 3; ++k) {
      c->list_n[k] = 0;
      c->next_seed[k] = kUnreachable;
      c->big_n[k] = 0;
      c->big_t[k] = 0;
    }
    c->seed_min = kUnreachable;
  }
  if (!sync_grid(p)) return;
  const uint32_t ncand = ld_cg(&c->cand_n);
  if (gtid() == 0) {
    c->candidates = ncand;
    c->touched_n = ncand;
  }
  if (ncand == 0) return;
  for (uint32_t i = gtid(); i < ncand; i += nthreads()) atomicMin(&c->seed_min, p.dist[p.lst_t[i]]);
  if (!sync_grid(p)) return;
  uint32_t d = ld_cg(&c->seed_min);
  // level-d work list: candidates at d (and later the children touched at d)
  for (uint32_t i = gtid(); i < ncand; i += nthreads()) {
    const uint32_t v = p.lst_t[i];
    if (p.dist[v] == d) p.q[0][atomicAdd(&c->list_n[0], 1u)] = v;
  }
  if (!sync_grid(p)) return;
  uint32_t a_prev = 0;
  for (uint32_t it = 0;; ++it) {
    if (it > p.dist_len + 1) {
      if (gtid() == 0) atomicOr(&c->err, vxb::kErrLoopBound);
      break;
    }
    const int k = it % 3, k1 = (it + 1) % 3, k2 = (it + 2) % 3;
    const uint32_t np = ld_cg(&c->list_n[k]);
    if (gtid() == 0) {
      c->list_n[k2] = 0;
      c->next_seed[k2] = kUnreachable;
      c->big_n[k2] = 0;
      c->big_t[k2] = 0;
    }
    // every touched vertex at distance d: one warp each, long rows deferred
    for (uint32_t i = gwarp(); i < np; i += nwarps()) {
      const uint32_t v = p.q[k][i];
      if (defer_row(p, p.g.in, v)) {
        if (lane == 0) {
          const uint32_t slot = atomicAdd(&c->big_n[k], 1u);
          p.big[slot] = v;
          p.tent[slot] = 0u;
        }
        continue;
      }
      if (!warp_has_surviving_parent(p, v, d) && lane == 0) mark_affected(p, v);
    }
    if (!sync_grid(p)) return;
    const uint32_t nbp = ld_cg(&c->big_n[k]);
    if (nbp) {
      grid_parent_probe(p, nbp, d);
      if (!sync_grid(p)) return;
      for (uint32_t r = gtid(); r < nbp; r += nthreads())
        if (!ld_cg(&p.tent[r])) mark_affected(p, p.big[r]);
      if (!sync_grid(p)) return;
    }
    const uint32_t a_tot = ld_cg(&c->a_n);
    if (a_tot > p.fallback_limit) {
      if (gtid() == 0) c->fallback = 1;
      break;
    }
    // next level's list: children of the vertices affected at d, candidates
    // at d+1; the nearest deeper candidate level for a jump
    TouchChildren tc{&p, d, p.q[k1], &c->list_n[k1]};
    for (uint32_t i = a_prev + gwarp(); i < a_tot; i += nwarps()) {
      const uint32_t v = p.lst_a[i];
      if (defer_row(p, p.g.out, v)) {
        if (lane == 0) p.big[atomicAdd(&c->big_t[k], 1u)] = v;
        continue;
      }
      warp_row(p.g.out, v, tc);
    }
    for (uint32_t i = gtid(); i < ncand; i += nthreads()) {
      const uint32_t v = p.lst_t[i];
      const uint32_t dv = p.dist[v];
      if (dv == d + 1) p.q[k1][atomicAdd(&c->list_n[k1], 1u)] = v;
      else if (dv != kUnreachable && dv > d + 1) atomicMin(&c->next_seed[k1], dv);
    }
    if (!sync_grid(p)) return;
    const uint32_t nbt = ld_cg(&c->big_t[k]);
    if (nbt) {
      grid_rows(p.g.out, p.big, nbt, tc);
      if (!sync_grid(p)) return;
    }
    a_prev = a_tot;
    const uint32_t nn = ld_cg(&c->list_n[k1]);
    if (nn > 0) {
      ++d;
      continue;
    }
    const uint32_t ns = ld_cg(&c->next_seed[k1]);
    if (ns == kUnreachable) break;
    // every block must have read list_n[k1] == 0 before it is refilled, or a
    // late block would see the refilled count and take the other branch
    if (!sync_grid(p)) return;
    d = ns;  // no touched vertex at d+1: jump to the next candidate level
    for (uint32_t i = gtid(); i < ncand; i += nthreads()) {
      const uint32_t v = p.lst_t[i];
      if (p.dist[v] == d) p.q[k1][atomicAdd(&c->list_n[k1], 1u)] = v;
    }
    if (!sync_grid(p)) return;
  }
  if (gtid() == 0) c->affected = ld_cg(&c->a_n);
}

// -------------------------------------------------- post-batch repair --

__device__ __forceinline__ void reach_add(const Params& p, long long d) {
  if (d) atomicAdd(&p.c->reachable, (unsigned long long)d);
}

__device__ void clear_workspace(const Params& p) {
  const uint32_t nt = ld_cg(&p.c->touched_n), na = ld_cg(&p.c->a_n);
  for (uint32_t i = gtid(); i < nt; i += nthreads()) p.lost[p.lst_t[i]] = 0u;
  for (uint32_t i = gtid(); i < na; i += nthreads()) p.aff[p.lst_a[i] >> 5] = 0u;
}

// Lower dist[x] to cand; on success (INF -> finite counted) queue x once per
// round through the inq bitmap.
__device__ __forceinline__ void lower_and_queue(const Params& p, uint32_t x, uint32_t cand, uint32_t* inq_next,
                                                uint32_t* qn, uint32_t* cnt, long long& reach) {
  if (cand >= ld_cg(&p.dist[x])) return;
  const uint32_t old = atomicMin(&p.dist[x], cand);
  if (old <= cand) return;
  if (old == kUnreachable) ++reach;
  const uint32_t bit = 1u << (x & 31);
  if (!(atomicOr(&inq_next[x >> 5], bit) & bit)) {
    const uint32_t s = atomicAdd(cnt, 1u);
    qn[s] = x;
  }
}

// Bucketed settle: relax affected out-neighbours of level-lvl vertices.
struct SettleVisit {
  const Params* p;
  uint32_t lvl;
  uint32_t* qn;
  uint32_t* cnt;
  long long* reach;
  __device__ __forceinline__ void operator()(bool valid, uint32_t x, uint32_t) {
    bool lowered = false;
    if (valid && test_bit(p->aff, x)) {
      const uint32_t cand = lvl + 1;
      if (cand < ld_cg(&p->dist[x])) {
        const uint32_t old = atomicMin(&p->dist[x], cand);
        if (old > cand) {
          lowered = true;
          if (old == kUnreachable) ++*reach;
        }
      }
    }
    const uint32_t s = vxb::warp_append(lowered, cnt);
    if (lowered) qn[s] = x;
  }
};

// Decrease propagation: relax every out-neighbour of a queued vertex.
struct PropVisit {
  const Params* p;
  uint32_t* inq_next;
  uint32_t* qn;
  uint32_t* cnt;
  long long* reach;
  __device__ __forceinline__ void operator()(bool valid, uint32_t x, uint32_t u) {
    if (!valid) return;
    const uint32_t du = ld_cg(&p->dist[u]);
    if (du == kUnreachable) return;
    lower_and_queue(*p, x, du + 1, inq_next, qn, cnt, *reach);
  }
};

// Warp-uniform minimum of dist+1 over non-affected in-neighbours
// (best_boundary_distance, bfs.hpp:261-269).
struct BoundaryMin {
  const Params* p;
  uint32_t best;
  __device__ __forceinline__ void operator()(bool valid, uint32_t x, uint32_t) {
    if (!valid || x >= p->dist_len || test_bit(p->aff, x)) return;
    const uint32_t dx = p->dist[x];
    if (dx != kUnreachable && dx + 1 < best) best = dx + 1;
  }
};

// Boundary distance of the deferred affected entries p.big[0, nb) (indices
// into lst_a): each warp folds its slices into p.tent[i] by atomicMin.
__device__ void grid_boundary_min(const Params& p, uint32_t nb) {
  const DevAdj& a = p.g.in;
  for (uint32_t r = 0; r < nb; ++r) {
    const uint32_t i = p.big[r];
    const uint32_t v = p.lst_a[i];
    BoundaryMin bm{&p, kUnreachable};
    uint64_t b, e;
    vxb::base_range(a, v, b, e);
    for (uint64_t j0 = b + (uint64_t)gwarp() * 32; j0 < e; j0 += (uint64_t)nwarps() * 32) {
      const uint64_t j = j0 + (threadIdx.x & 31);
      const uint32_t x = j < e ? a.col[j] : kTomb;
      bm(!(x & kTomb), x & kIdMask, v);
    }
    const uint2 dr = a.drow[v];
    for (uint32_t j0 = dr.x + gwarp() * 32; j0 < dr.x + dr.y; j0 += nwarps() * 32) {
      const uint32_t j = j0 + (threadIdx.x & 31);
      const bool ok = j < dr.x + dr.y;
      bm(ok, ok ? a.darena[j] : 0u, v);
    }
    uint32_t best = bm.best;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) best = min(best, __shfl_xor_sync(FULL, best, o));
    if ((threadIdx.x & 31) == 0 && best != kUnreachable) atomicMin(&p.tent[i], best);
  }
}

__device__ void repair_post(const Params& p) {
  BfsCounters* c = p.c;
  const int lane = threadIdx.x & 31;
  if (ld_cg(&c->fallback)) {
    clear_workspace(p);
    if (!sync_grid(p)) return;
    full_bfs(p);
    if (gtid() == 0) c->full = 1;
    return;
  }
  const uint32_t na = ld_cg(&c->a_n);
  long long reach = 0;
  if (na > 0) {
    for (uint32_t i = gtid(); i < na; i += nthreads()) {
      const uint32_t v = p.lst_a[i];
      p.old[i] = p.dist[v];
      p.dist[v] = kUnreachable;
    }
    if (gtid() == 0) {
      reach_add(p, -(long long)na);
      c->seed_min = kUnreachable;
      for (int k = 0; k < 3; ++k) {
        c->list_n[k] = 0;
        c->next_seed[k] = kUnreachable;
        c->big_n[k] = 0;
        c->big_t[k] = 0;
      }
    }
    if (!sync_grid(p)) return;
    // boundary seeds, one warp per affected vertex, long in-rows deferred
    for (uint32_t i = gwarp(); i < na; i += nwarps()) {
      const uint32_t v = p.lst_a[i];
      if (defer_row(p, p.g.in, v)) {
        if (lane == 0) {
          p.tent[i] = kUnreachable;
          p.big[atomicAdd(&c->big_t[0], 1u)] = i;
        }
        continue;
      }
      BoundaryMin bm{&p, kUnreachable};
      warp_row(p.g.in, v, bm);
      uint32_t best = bm.best;
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) best = min(best, __shfl_xor_sync(FULL, best, o));
      if (lane == 0) {
        p.tent[i] = best;
        p.dist[v] = best;
        if (best != kUnreachable) {
          ++reach;
          atomicMin(&c->seed_min, best);
        }
      }
    }
    if (!sync_grid(p)) return;
    const uint32_t nbb = ld_cg(&c->big_t[0]);
    if (nbb) {
      grid_boundary_min(p, nbb);
      if (!sync_grid(p)) return;
      for (uint32_t r = gtid(); r < nbb; r += nthreads()) {
        const uint32_t i = p.big[r];
        const uint32_t best = ld_cg(&p.tent[i]);
        p.dist[p.lst_a[i]] = best;
        if (best != kUnreachable) {
          ++reach;
          atomicMin(&c->seed_min, best);
        }
      }
      if (!sync_grid(p)) return;
    }
    // bucketed settle among affected vertices (unit-weight Dijkstra)
    uint32_t lvl = ld_cg(&c->seed_min);
    if (lvl != kUnreachable) {
      const DevAdj& a = p.g.out;
      for (uint32_t it = 0;; ++it) {
        if (it > p.dist_len + 1) {
          if (gtid() == 0) atomicOr(&c->err, vxb::kErrLoopBound);
          break;
        }
        const int k = it % 3, k1 = (it + 1) % 3, k2 = (it + 2) % 3;
        const uint32_t nr = ld_cg(&c->list_n[k]);
        if (gtid() == 0) {
          c->list_n[k2] = 0;
          c->next_seed[k2] = kUnreachable;
          c->big_n[k2] = 0;
        }
        SettleVisit sv{&p, lvl, p.q[k1], &c->list_n[k1], &reach};
        // items: seeds whose boundary distance is lvl and still hold it, then
        // the vertices relaxed to lvl at the previous level
        for (uint32_t base = gwarp() * 32; base < na + nr; base += nwarps() * 32) {
          const uint32_t i = base + lane;
          bool act = false;
          uint32_t u = 0;
          if (i < na) {
            const uint32_t t = p.tent[i];
            u = p.lst_a[i];
            const uint32_t du = ld_cg(&p.dist[u]);
            act = t == lvl && du == lvl;
            if (!act && t != kUnreachable && t > lvl && du == t) atomicMin(&c->next_seed[k1], t);
          } else if (i < na + nr) {
            u = p.q[k][i - na];
            act = true;
          }
          uint64_t b = 0, e = 0;
          uint2 dr = make_uint2(0, 0);
          if (act) {
            vxb::base_range(a, u, b, e);
            dr = a.drow[u];
          }
          defer_lanes(p, &c->big_n[k], act, u, b, e, dr);
          expand_lanes(a, u, b, e, dr, sv);
        }
        if (!sync_grid(p)) return;
        const uint32_t nbs = ld_cg(&c->big_n[k]);
        if (nbs) {
          grid_rows(a, p.big, nbs, sv);
          if (!sync_grid(p)) return;
        }
        const uint32_t nn = ld_cg(&c->list_n[k1]), ns = ld_cg(&c->next_seed[k1]);
        if (nn > 0) ++lvl;
        else if (ns != kUnreachable) lvl = ns;
        else break;
      }
    }
  }
  // decrease propagation (bfs.hpp:312-318, 91-96, 341-354): seeds are the
  // affected vertices that ended below their old distance and the heads of
  // inserted arcs that relax
  if (gtid() == 0) {
    for (int k = 0; k < 3; ++k) {
      c->list_n[k] = 0;
      c->big_n[k] = 0;
    }
  }
  if (!sync_grid(p)) return;
  for (uint32_t i = gtid(); i < na; i += nthreads()) {
    const uint32_t v = p.lst_a[i];
    const uint32_t dv = ld_cg(&p.dist[v]);
    if (dv != kUnreachable && dv < p.old[i]) {
      const uint32_t bit = 1u << (v & 31);
      if (!(atomicOr(&p.inq[0][v >> 5], bit) & bit)) p.q[0][atomicAdd(&c->list_n[0], 1u)] = v;
    }
  }
  const uint32_t F = *p.F;
  for (uint32_t i = gtid(); i < F; i += nthreads()) {
    if (!(p.ff[i] & kFAdd)) continue;
    const uint32_t u = p.fu[i], v = p.fv[i];
    if (u >= p.dist_len || v >= p.dist_len) continue;
    const uint32_t du = ld_cg(&p.dist[u]);
    if (du == kUnreachable) continue;
    lower_and_queue(p, v, du + 1, p.inq[0], p.q[0], &c->list_n[0], reach);
  }
  if (!sync_grid(p)) return;
  const DevAdj& a = p.g.out;
  for (uint32_t r = 0;; ++r) {
    if (r > p.dist_len + 1) {
      if (gtid() == 0) atomicOr(&c->err, vxb::kErrLoopBound);
      break;
    }
    const int k = r % 3, k1 = (r + 1) % 3, k2 = (r + 2) % 3;
    const uint32_t n = ld_cg(&c->list_n[k]);
    if (n == 0) break;
    if (gtid() == 0) {
      c->list_n[k2] = 0;
      c->big_n[k2] = 0;
    }
    uint32_t* inq_cur = p.inq[r & 1];
    PropVisit pv{&p, p.inq[(r + 1) & 1], p.q[k1], &c->list_n[k1], &reach};
    for (uint32_t base = gwarp() * 32; base < n; base += nwarps() * 32) {
      const uint32_t i = base + lane;
      const bool act = i < n;
      const uint32_t u = act ? p.q[k][i] : 0u;
      uint64_t b = 0, e = 0;
      uint2 dr = make_uint2(0, 0);
      if (act) {
        atomicAnd(&inq_cur[u >> 5], ~(1u << (u & 31)));
        vxb::base_range(a, u, b, e);
        dr = a.drow[u];
      }
      defer_lanes(p, &c->big_n[k], act, u, b, e, dr);
      expand_lanes(a, u, b, e, dr, pv);
    }
    if (!sync_grid(p)) return;
    const uint32_t nbq = ld_cg(&c->big_n[k]);
    if (nbq) {
      grid_rows(a, p.big, nbq, pv);
      if (!sync_grid(p)) return;
    }
  }
  reach = vxb::warp_sum(reach);
  if (lane == 0) reach_add(p, reach);
  clear_workspace(p);
}

__global__ void __launch_bounds__(kThreads, 3) bfs_kernel(Params p, int mode) {
  if (mode == kModeFull) full_bfs(p);
  else if (mode == kModePre) repair_pre(p);
  else repair_post(p);
}

__global__ void reached_arcs_kernel(vxb::DevAdj a, const uint32_t* dist, uint32_t n,
                                    unsigned long long* out) {
  unsigned long long s = 0;
  for (uint32_t v = blockIdx.x * blockDim.x + threadIdx.x; v < n; v += gridDim.x * blockDim.x) {
    if (dist[v] == kUnreachable) continue;
    uint64_t b, e;
    vxb::base_range(a, v, b, e);
    // live arcs: base minus tombstones plus delta
    s += (e - b) - a.tcnt[v] + a.drow[v].y;
  }
  s = vxb::warp_sum(s);
  if ((threadIdx.x & 31) == 0 && s) atomicAdd(out, s);
}

}  // namespace

// ---------------------------------------------------------------- host --

static int ensure_capacity(Bfs* b, size_t V) {
  if (V <= b->cap && b->dist) return 0;
  size_t c = std::max<size_t>(b->cap ? b->cap : 1024, 1024);
  while (c < V) c *= 2;
  const size_t words = (c + 31) / 32 + 1;
  cudaStream_t s = b->g->stream;
  VX_CUDA_TRY(cudaStreamSynchronize(s));
  auto realloc_copy = [&](uint32_t** p, size_t n_new, size_t n_old, int fill) -> int {
    uint32_t* q = nullptr;
    if (cudaMalloc(&q, n_new * sizeof(uint32_t)) != cudaSuccess) {
      set_error("BFS allocation of %zu bytes failed", n_new * 4);
      return -4;
    }
    if (cudaMemset(q, fill, n_new * sizeof(uint32_t)) != cudaSuccess) return -3;
    if (*p && n_old) cudaMemcpy(q, *p, n_old * sizeof(uint32_t), cudaMemcpyDeviceToDevice);
    cudaFree(*p);
    *p = q;
    return 0;
  };
  const size_t oldw = b->cap ? (b->cap + 31) / 32 + 1 : 0;
  int rc = 0;
  rc |= realloc_copy(&b->dist, c, b->cap, 0xFF);
  rc |= realloc_copy(&b->lost, c, b->cap, 0);
  rc |= realloc_copy(&b->vis, words, 0, 0);
  rc |= realloc_copy(&b->aff, words, oldw, 0);
  rc |= realloc_copy(&b->inq[0], words, oldw, 0);
  rc |= realloc_copy(&b->inq[1], words, oldw, 0);
  for (int k = 0; k < 3; ++k) {
    rc |= realloc_copy(&b->fb[k], words, 0, 0);
    rc |= realloc_copy(&b->q[k], c, 0, 0);
  }
  rc |= realloc_copy(&b->big, c, 0, 0);
  rc |= realloc_copy(&b->lst_a, c, 0, 0);
  rc |= realloc_copy(&b->lst_t, c, 0, 0);
  rc |= realloc_copy(&b->old, c, 0, 0);
  rc |= realloc_copy(&b->tent, c, 0, 0);
  if (rc) return -4;
  b->cap = c;
  return 0;
}

static Params make_params(Bfs* b, uint32_t V, uint32_t dist_len) {
  Graph* g = b->g;
  Params p;
  memset(&p, 0, sizeof(p));
  p.g = g->view();
  p.V = V;
  p.dist_len = dist_len;
  p.source = b->source;
  p.dist = b->dist;
  p.vis = b->vis;
  for (int k = 0; k < 3; ++k) {
    p.fb[k] = b->fb[k];
    p.q[k] = b->q[k];
  }
  p.big = b->big;
  p.lst_a = b->lst_a;
  p.lst_t = b->lst_t;
  p.old = b->old;
  p.tent = b->tent;
  p.lost = b->lost;
  p.aff = b->aff;
  p.inq[0] = b->inq[0];
  p.inq[1] = b->inq[1];
  p.fu = g->batch.fu;
  p.fv = g->batch.fv;
  p.ff = g->batch.ff;
  p.F = &g->ctr->final_arcs;
  p.c = b->ctr;
  p.total_arcs = g->adj[0].A;  // estimate for the direction switch
  p.alpha = b->tune.alpha;
  p.beta = b->tune.beta;
  p.large_row = b->tune.large_row;
  p.trace = b->trace;
  p.bar = b->barrier;
  return p;
}

static int launch(Bfs* b, Params& p, int mode) {
  if (!b->grid) {
    int per_sm = 0;
    VX_CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, bfs_kernel, kThreads, 0));
    if (per_sm < 1) {
      set_error("BFS kernel cannot be resident on an SM");
      return -3;
    }
    b->grid = per_sm * sm_count();
  }
  p.nblocks = (uint32_t)b->grid;
  void* args[] = {&p, &mode};
  vxh::count_launch();
  VX_CUDA_TRY(cudaLaunchCooperativeKernel((const void*)bfs_kernel, dim3(b->grid), dim3(kThreads), args, 0,
                                          b->g->stream));
  return 0;
}

int bfs_create(Bfs** out, Graph* g, uint32_t source, double frac) {
  Bfs* b = new Bfs();
  b->g = g;
  b->source = source;
  b->frac = frac;
  if (cudaMalloc(&b->ctr, sizeof(BfsCounters)) != cudaSuccess ||
      cudaMalloc(&b->trace, 2 * (kTraceLevels + 1) * sizeof(unsigned long long)) != cudaSuccess ||
      cudaMalloc(&b->barrier, vxb::kBarrierWords * sizeof(uint32_t)) != cudaSuccess ||
      cudaMalloc(&b->features, 64 * sizeof(float)) != cudaSuccess ||
      cudaMallocHost(&b->hctr, sizeof(BfsCounters)) != cudaSuccess) {
    set_error("BFS counter allocation failed");
    bfs_destroy(b);
    return -4;
  }
  cudaMemsetAsync(b->ctr, 0, sizeof(BfsCounters), g->stream);
  cudaMemsetAsync(b->barrier, 0, vxb::kBarrierWords * sizeof(uint32_t), g->stream);
  memset(b->hctr, 0, sizeof(BfsCounters));
  if (int rc = bfs_recompute(b)) {
    bfs_destroy(b);
    return rc;
  }
  *out = b;
  return 0;
}

void bfs_destroy(Bfs* b) {
  if (!b) return;
  if (b->g && b->g->stream) cudaStreamSynchronize(b->g->stream);
  uint32_t* ptrs[] = {b->dist, b->vis, b->fb[0], b->fb[1], b->fb[2], b->q[0], b->q[1], b->q[2], b->big,
                      b->lst_a, b->lst_t, b->old, b->tent, b->lost, b->aff, b->inq[0], b->inq[1]};
  for (uint32_t* p : ptrs) cudaFree(p);
  cudaFree(b->ctr);
  cudaFree(b->trace);
  cudaFree(b->barrier);
  cudaFree(b->features);
  cudaFreeHost(b->hctr);
  delete b;
}

int bfs_recompute(Bfs* b) {
  Graph* g = b->g;
  const size_t V = g->V;
  if (int rc = ensure_capacity(b, std::max<size_t>(V, 1))) return rc;
  b->dist_len = V;
  VX_CUDA_TRY(cudaMemsetAsync(&b->ctr->candidates, 0, 4 * sizeof(uint32_t), g->stream));
  if (V == 0) {
    VX_CUDA_TRY(cudaMemsetAsync(&b->ctr->reachable, 0, 8, g->stream));
    return 0;
  }
  Params p = make_params(b, (uint32_t)V, (uint32_t)V);
  return launch(b, p, kModeFull);
}

int bfs_stage(Bfs* b, size_t n, size_t vertex_bound) {
  Graph* g = b->g;
  cudaStream_t s = g->stream;
  // last_* counters reset on every apply (bfs.hpp:30-33)
  VX_CUDA_TRY(cudaMemsetAsync(&b->ctr->candidates, 0, 4 * sizeof(uint32_t), s));
  b->staged_ops = n;
  b->staged_V_pre = g->V;
  b->staged_len_pre = b->dist_len;
  if (n == 0) return 0;
  VX_CUDA_TRY(cudaMemsetAsync(&b->ctr->cand_n, 0, 3 * sizeof(uint32_t), s));
  if (int rc = graph_stage_batch(g, n, vertex_bound)) return rc;
  return ensure_capacity(b, std::max<size_t>(g->V, 1));
}

int bfs_repair_staged(Bfs* b) {
  Graph* g = b->g;
  cudaStream_t s = g->stream;
  if (b->staged_ops == 0) return 0;
  const size_t V_pre = b->staged_V_pre, len_pre = b->staged_len_pre;
  const size_t V_post = g->V;
  // fallback limit: max(1, size_t(double(V) * fraction))  (bfs.hpp:225-226)
  unsigned long long lim = (unsigned long long)((double)V_pre * b->frac);
  if (lim < 1) lim = 1;
  // The fixpoint reads the pre-batch graph without the batch's deletions
  // (exactly the arcs the reference's support count and child propagation
  // exclude), so removals are committed first and insertions after it.
  if (int rc = graph_commit_removals(g)) return rc;
  {
    Params p = make_params(b, (uint32_t)V_pre, (uint32_t)len_pre);
    p.fallback_limit = lim;
    if (len_pre > 0)
      if (int rc = launch(b, p, kModePre)) return rc;
  }
  if (int rc = graph_commit_insertions(g)) return rc;
  if (b->dist_len < V_post) {
    VX_CUDA_TRY(cudaMemsetAsync(b->dist + b->dist_len, 0xFF, (V_post - b->dist_len) * 4, s));
    b->dist_len = V_post;
  }
  b->staged_ops = 0;
  Params p = make_params(b, (uint32_t)V_post, (uint32_t)b->dist_len);
  p.fallback_limit = lim;
  return launch(b, p, kModePost);
}

int bfs_full_staged(Bfs* b) {
  if (b->staged_ops == 0) return 0;
  if (int rc = graph_commit_batch(b->g)) return rc;
  b->staged_ops = 0;
  return bfs_recompute(b);
}

int bfs_apply_staged(Bfs* b, size_t n, size_t vertex_bound) {
  if (int rc = bfs_stage(b, n, vertex_bound)) return rc;
  return bfs_repair_staged(b);
}

int bfs_sync(Bfs* b) {
  cudaStream_t s = b->g->stream;
  VX_CUDA_TRY(cudaMemcpyAsync(b->hctr, b->ctr, sizeof(BfsCounters), cudaMemcpyDeviceToHost, s));
  VX_CUDA_TRY(cudaStreamSynchronize(s));
  if (b->hctr->err) {
    set_error("BFS device error word 0x%x", b->hctr->err);
    return -5;
  }
  return 0;
}

int bfs_reached_arcs(Bfs* b, unsigned long long* arcs) {
  cudaStream_t s = b->g->stream;
  unsigned long long* d = &b->ctr->scratch64;
  VX_CUDA_TRY(cudaMemsetAsync(d, 0, 8, s));
  vxh::count_launch();
  reached_arcs_kernel<<<sm_count() * 8, 256, 0, s>>>(b->g->view().out, b->dist, (uint32_t)b->dist_len, d);
  VX_CUDA_TRY(cudaGetLastError());
  VX_CUDA_TRY(cudaMemcpyAsync(b->g->pinned_scalar, d, 8, cudaMemcpyDeviceToHost, s));
  VX_CUDA_TRY(cudaStreamSynchronize(s));
  *arcs = b->g->pinned_scalar[0];
  return 0;
}

}  // namespace vxh

namespace vxh {
int bfs_level_trace(Bfs* b, unsigned long long* out, size_t cap, size_t* n) {
  if (int rc = bfs_sync(b)) return rc;
  const uint32_t levels = std::min<uint32_t>(b->hctr->levels, kTraceLevels - 1);
  *n = 2 * ((size_t)levels + 1);
  const size_t m = std::min(cap, *n);
  if (out && m) VX_CUDA_TRY(cudaMemcpy(out, b->trace, m * sizeof(unsigned long long), cudaMemcpyDeviceToHost));
  return 0;
}
}  // namespace vxh

// ------------------------------------------------ allocation-free full BFS --
//
// Some callers cannot call cudaMalloc: a host framework that owns the whole
// device memory through its own pool (and forbids raw driver allocations),
// or a latency-critical serving loop that must never block on the driver's
// allocator after start-up.  vx_bfs_csr_static serves them: it runs the same
// direction-optimising BFS kernel as recompute() on a CSR the caller already
// holds in device memory, writing distances into the caller's buffer, and
// keeps every other buffer (visited and frontier bitmaps, frontier queues,
// counters, barrier words, the empty delta-row table) in one file-scope
// device array.  It allocates nothing.
//
// Limits and sharing: at most kStaticMaxVertices vertices; every GPU that
// loads this library holds the array (about 6.3 MB) until the process exits;
// all calls share it and it keeps the last call's contents, so calls that
// overlap on the GPU (different streams, different threads) race -- issue
// them one at a time per device.  The first call on a device looks up the
// array's device address for that device; make that first call before any
// stream capture.
namespace vxh {
namespace {

constexpr uint32_t kStaticMaxVertices = 1u << 18;  // 262,144
constexpr uint32_t kStaticWords = kStaticMaxVertices / 32 + 1;

struct StaticBfsScratch {
  uint32_t vis[kStaticWords];
  uint32_t fb[3][kStaticWords];
  uint32_t q[3][kStaticMaxVertices];
  uint32_t big[kStaticMaxVertices];
  uint2 drow[kStaticMaxVertices];  // kept all-zero: a plain CSR has no delta rows
  BfsCounters ctr;
  uint32_t bar[vxb::kBarrierWords];
};

}  // namespace
}  // namespace vxh

static __device__ __align__(256) unsigned char vx_static_bfs_scratch[sizeof(vxh::StaticBfsScratch)];

namespace {
constexpr int kStaticMaxDevices = 64;
void* g_static_scratch_addr[kStaticMaxDevices];  // device address of the array, per device
}  // namespace

extern "C" int vx_bfs_csr_static(const uint64_t* d_out_offsets, const uint32_t* d_out_cols,
                                 const uint64_t* d_in_offsets, const uint32_t* d_in_cols, uint32_t vertices,
                                 uint64_t arcs, uint32_t source, uint32_t* d_dist, void* stream,
                                 uint64_t* reachable) {
  using vxh::StaticBfsScratch;
  if (!d_out_offsets || !d_out_cols || !d_in_offsets || !d_in_cols || !d_dist) {
    vxh::set_error("vx_bfs_csr_static: null argument");
    return -1;
  }
  if (vertices == 0 || vertices > vxh::kStaticMaxVertices) {
    vxh::set_error("vx_bfs_csr_static: %u vertices; the static scratch holds 1..%u", vertices,
                   vxh::kStaticMaxVertices);
    return -2;
  }
  int dev = 0;
  VX_CUDA_TRY(cudaGetDevice(&dev));
  if (dev < 0 || dev >= kStaticMaxDevices) {
    vxh::set_error("vx_bfs_csr_static: device %d beyond the supported %d", dev, kStaticMaxDevices);
    return -2;
  }
  if (!g_static_scratch_addr[dev]) {
    // one-time set-up on this device (the device is current here)
    void* ptr = nullptr;
    const cudaError_t e = cudaGetSymbolAddress(&ptr, vx_static_bfs_scratch);
    if (e != cudaSuccess || !ptr) {
      vxh::set_error("vx_bfs_csr_static: cudaGetSymbolAddress failed: %s", cudaGetErrorString(e));
      return -3;
    }
    g_static_scratch_addr[dev] = ptr;
  }
  StaticBfsScratch* sc = static_cast<StaticBfsScratch*>(g_static_scratch_addr[dev]);
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  // what must start at zero: counters, barrier words, the delta-row table
  VX_CUDA_TRY(cudaMemsetAsync(&sc->ctr, 0, sizeof(vxh::BfsCounters), s));
  VX_CUDA_TRY(cudaMemsetAsync(sc->bar, 0, sizeof(sc->bar), s));
  VX_CUDA_TRY(cudaMemsetAsync(sc->drow, 0, (size_t)vertices * sizeof(uint2), s));
  vxh::Params p;
  memset(&p, 0, sizeof(p));
  auto adj = [&](const uint64_t* off, const uint32_t* col) {
    vxb::DevAdj a;
    memset(&a, 0, sizeof(a));
    a.off = off;
    a.col = const_cast<uint32_t*>(col);
    a.Vb = vertices;
    a.drow = sc->drow;
    return a;
  };
  p.g.out = adj(d_out_offsets, d_out_cols);
  p.g.in = adj(d_in_offsets, d_in_cols);
  p.g.V = vertices;
  p.g.directed = d_in_offsets != d_out_offsets || d_in_cols != d_out_cols;
  p.V = vertices;
  p.dist_len = vertices;
  p.source = source;
  p.dist = d_dist;
  p.vis = sc->vis;
  for (int k = 0; k < 3; ++k) {
    p.fb[k] = sc->fb[k];
    p.q[k] = sc->q[k];
  }
  p.big = sc->big;
  p.c = &sc->ctr;
  p.total_arcs = arcs;
  p.alpha = 14.0f;
  p.beta = 24.0f;
  p.large_row = 1024;
  p.bar = sc->bar;
  int per_sm = 0, sms = 0;
  VX_CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, vxh::bfs_kernel, vxh::kThreads, 0));
  VX_CUDA_TRY(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
  if (per_sm < 1) {
    vxh::set_error("vx_bfs_csr_static: BFS kernel cannot be resident on an SM");
    return -3;
  }
  p.nblocks = (uint32_t)(per_sm * sms);
  int mode = vxh::kModeFull;
  void* args[] = {&p, &mode};
  vxh::count_launch();
  VX_CUDA_TRY(cudaLaunchCooperativeKernel((const void*)vxh::bfs_kernel, dim3(p.nblocks), dim3(vxh::kThreads), args,
                                          0, s));
  uint32_t err = 0;
  unsigned long long reach = 0;
  VX_CUDA_TRY(cudaMemcpyAsync(&err, &sc->ctr.err, sizeof(err), cudaMemcpyDeviceToHost, s));
  VX_CUDA_TRY(cudaMemcpyAsync(&reach, &sc->ctr.reachable, sizeof(reach), cudaMemcpyDeviceToHost, s));
  VX_CUDA_TRY(cudaStreamSynchronize(s));
  if (err) {
    vxh::set_error("vx_bfs_csr_static: device error word 0x%x", err);
    return -5;
  }
  if (reachable) *reachable = reach;
  return 0;
}
