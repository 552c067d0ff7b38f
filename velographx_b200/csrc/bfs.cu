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

namespace vxh {

using vxb::DevAdj;
using vxb::kIdMask;
using vxb::kTomb;
using vxb::kUnreachable;

namespace {

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
};

__device__ __forceinline__ uint32_t ld_cg(const uint32_t* p) { return __ldcg(p); }

__device__ __forceinline__ uint32_t gtid() { return blockIdx.x * blockDim.x + threadIdx.x; }
__device__ __forceinline__ uint32_t nthreads() { return gridDim.x * blockDim.x; }
__device__ __forceinline__ uint32_t gwarp() { return gtid() >> 5; }
__device__ __forceinline__ uint32_t nwarps() { return nthreads() >> 5; }

__device__ __forceinline__ void sync_grid(const Params& p) { vxb::grid_barrier(p.c->bar, p.nblocks, &p.c->err); }

__device__ __forceinline__ bool test_bit(const uint32_t* bm, uint32_t v) { return (bm[v >> 5] >> (v & 31)) & 1u; }

__device__ __forceinline__ uint32_t degree_of(const DevAdj& a, uint32_t u) {
  uint64_t b, e;
  vxb::base_range(a, u, b, e);
  return (uint32_t)(e - b) + a.drow[u].y;
}

// ------------------------------------------------------------ top-down --

struct TdCtx {
  uint32_t level;
  uint32_t* qout;
  uint32_t* fbn;
  uint32_t* cnt_n;
  bool want_deg;
  unsigned long long mloc;
};

// Claim v (if valid) for the next level.  Warp-uniform call.
__device__ __forceinline__ void td_visit(const Params& p, TdCtx& t, bool valid, uint32_t v) {
  bool claim = false;
  const uint32_t bit = 1u << (v & 31);
  if (valid) {
    const uint32_t w = p.vis[v >> 5];
    if (!(w & bit)) claim = !(atomicOr(&p.vis[v >> 5], bit) & bit);
  }
  if (claim) {
    p.dist[v] = t.level + 1;
    atomicOr(&t.fbn[v >> 5], bit);
    if (t.want_deg) t.mloc += degree_of(p.g.out, v);
  }
  const uint32_t slot = vxb::warp_append(claim, t.cnt_n);
  if (claim) t.qout[slot] = v;
}

// Flattened expansion of per-lane segments arr[start, start+len) (len < 32 is
// typical; any length works).  Warp-uniform call.
__device__ __forceinline__ void td_gather(const Params& p, TdCtx& t, const uint32_t* arr, uint64_t start, uint32_t len,
                                          bool tombs) {
  const int lane = threadIdx.x & 31;
  uint32_t incl = len;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const uint32_t y = __shfl_up_sync(0xFFFFFFFFu, incl, o);
    if (lane >= o) incl += y;
  }
  const uint32_t excl = incl - len;
  const uint32_t total = __shfl_sync(0xFFFFFFFFu, incl, 31);
  for (uint32_t k0 = 0; k0 < total; k0 += 32) {
    const uint32_t k = k0 + lane;
    const bool ok = k < total;
    int owner = 0;
#pragma unroll
    for (int step = 16; step >= 1; step >>= 1) {
      const int cand = owner + step;
      const uint32_t ex = __shfl_sync(0xFFFFFFFFu, excl, cand & 31);
      if (cand < 32 && ex <= k) owner = cand;
    }
    const uint64_t st = __shfl_sync(0xFFFFFFFFu, start, owner);
    const uint32_t ex = __shfl_sync(0xFFFFFFFFu, excl, owner);
    const uint32_t x = ok ? arr[st + (k - ex)] : kTomb;
    td_visit(p, t, ok && !(tombs && (x & kTomb)), x & kIdMask);
  }
}

__device__ void td_level(const Params& p, TdCtx& t, const uint32_t* qin, uint32_t n_f, uint32_t* cnt_big) {
  const DevAdj& a = p.g.out;
  const int lane = threadIdx.x & 31;
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
    uint32_t blen = (uint32_t)(e - b), dlen = dr.y;
    const bool big = act && (uint64_t)blen + dlen >= p.large_row;
    const uint32_t slot = vxb::warp_append(big, cnt_big);
    if (big) {
      p.big[slot] = u;
      blen = dlen = 0;
    }
    // medium base rows: whole warp per row
    uint32_t med = __ballot_sync(0xFFFFFFFFu, blen >= 32);
    while (med) {
      const int l = __ffs(med) - 1;
      med &= med - 1;
      const uint64_t bb = __shfl_sync(0xFFFFFFFFu, b, l), ee = __shfl_sync(0xFFFFFFFFu, e, l);
      for (uint64_t j0 = bb; j0 < ee; j0 += 32) {
        const uint64_t j = j0 + lane;
        const uint32_t x = j < ee ? a.col[j] : kTomb;
        td_visit(p, t, !(x & kTomb), x & kIdMask);
      }
    }
    if (blen >= 32) blen = 0;
    td_gather(p, t, a.col, b, blen, true);
    // delta rows
    med = __ballot_sync(0xFFFFFFFFu, dlen >= 32);
    while (med) {
      const int l = __ffs(med) - 1;
      med &= med - 1;
      const uint32_t bb = __shfl_sync(0xFFFFFFFFu, dr.x, l), ee = bb + __shfl_sync(0xFFFFFFFFu, dr.y, l);
      for (uint32_t j0 = bb; j0 < ee; j0 += 32) {
        const uint32_t j = j0 + lane;
        const bool ok = j < ee;
        td_visit(p, t, ok, ok ? a.darena[j] : 0u);
      }
    }
    if (dlen >= 32) dlen = 0;
    td_gather(p, t, a.darena, dr.x, dlen, false);
  }
}

// Rows of at least large_row arcs: every warp of the grid takes a slice.
__device__ void td_big_rows(const Params& p, TdCtx& t, uint32_t nbig) {
  const DevAdj& a = p.g.out;
  const int lane = threadIdx.x & 31;
  for (uint32_t r = 0; r < nbig; ++r) {
    const uint32_t u = p.big[r];
    uint64_t b, e;
    vxb::base_range(a, u, b, e);
    for (uint64_t j0 = b + (uint64_t)gwarp() * 32; j0 < e; j0 += (uint64_t)nwarps() * 32) {
      const uint64_t j = j0 + lane;
      const uint32_t x = j < e ? a.col[j] : kTomb;
      td_visit(p, t, !(x & kTomb), x & kIdMask);
    }
    const uint2 dr = a.drow[u];
    for (uint32_t j0 = dr.x + gwarp() * 32; j0 < dr.x + dr.y; j0 += nwarps() * 32) {
      const uint32_t j = j0 + lane;
      const bool ok = j < dr.x + dr.y;
      td_visit(p, t, ok, ok ? a.darena[j] : 0u);
    }
  }
}

// ----------------------------------------------------------- bottom-up --

__device__ void bu_level(const Params& p, uint32_t level, const uint32_t* fbc, uint32_t* fbn, uint32_t* qout,
                         uint32_t* cnt_n) {
  const DevAdj& a = p.g.in;
  const int lane = threadIdx.x & 31;
  const uint32_t words = (p.V + 31) >> 5;
  for (uint32_t w = gwarp(); w < words; w += nwarps()) {
    const uint32_t visw = p.vis[w];
    if (visw == 0xFFFFFFFFu) continue;
    const uint32_t v = w * 32 + lane;
    bool found = false;
    if (!((visw >> lane) & 1u)) {
      uint64_t b, e;
      vxb::base_range(a, v, b, e);
      for (uint64_t j = b; j < e; ++j) {
        const uint32_t x = a.col[j];
        if (!(x & kTomb) && test_bit(fbc, x)) {
          found = true;
          break;
        }
      }
      if (!found) {
        const uint2 dr = a.drow[v];
        for (uint32_t j = dr.x; j < dr.x + dr.y; ++j) {
          if (test_bit(fbc, a.darena[j])) {
            found = true;
            break;
          }
        }
      }
    }
    const uint32_t newly = __ballot_sync(0xFFFFFFFFu, found);
    if (found) p.dist[v] = level + 1;
    if (lane == 0 && newly) {
      p.vis[w] = visw | newly;
      fbn[w] = newly;
    }
    const uint32_t slot = vxb::warp_append(found, cnt_n);
    if (found) qout[slot] = v;
  }
}

__device__ __forceinline__ void flush_degrees(TdCtx& t, unsigned long long* dst) {
  if (!t.want_deg) return;
  const unsigned long long sum = vxb::warp_sum(t.mloc);
  if ((threadIdx.x & 31) == 0 && sum) atomicAdd(dst, sum);
  t.mloc = 0;
}

// ------------------------------------------------------------ full BFS --

__device__ void full_bfs(const Params& p) {
  BfsCounters* c = p.c;
  const uint32_t V = p.V;
  const uint32_t words = (V + 31) >> 5;
  for (uint32_t i = gtid(); i < V; i += nthreads()) p.dist[i] = kUnreachable;
  for (uint32_t i = gtid(); i < words; i += nthreads()) {
    // bits past V count as visited so bottom-up never scans them
    const uint32_t lo = i * 32;
    p.vis[i] = (lo + 32 <= V) ? 0u : (0xFFFFFFFFu << (V - lo));
    p.fb[0][i] = p.fb[1][i] = p.fb[2][i] = 0u;
  }
  if (gtid() == 0) {
    for (int k = 0; k < 3; ++k) {
      c->lvl_n[k] = 0;
      c->lvl_big[k] = 0;
      c->lvl_m[k] = 0;
    }
  }
  sync_grid(p);
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
  sync_grid(p);
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
    }
    // clear the frontier bitmap of level-1 through its queue
    for (uint32_t i = gtid(); i < prev_n; i += nthreads()) p.fb[clr][p.q[clr][i] >> 5] = 0u;
    if (bottom_up) {
      bu_level(p, level, p.fb[cur], p.fb[nxt], p.q[nxt], &c->lvl_n[nxt]);
      sync_grid(p);
    } else {
      TdCtx t{level, p.q[nxt], p.fb[nxt], &c->lvl_n[nxt], !left_bu, 0ull};
      td_level(p, t, p.q[cur], n_f, &c->lvl_big[cur]);
      flush_degrees(t, &c->lvl_m[nxt]);
      sync_grid(p);
      const uint32_t nbig = ld_cg(&c->lvl_big[cur]);
      if (nbig) {
        td_big_rows(p, t, nbig);
        flush_degrees(t, &c->lvl_m[nxt]);
        sync_grid(p);
      }
    }
    prev_n = n_f;
  }
  if (gtid() == 0) {
    c->reachable = reached;
    c->levels = level;
    c->arcs = m_visited;
  }
}

// ------------------------------------------------------------- helpers --

__device__ __forceinline__ bool is_sp(const Params& p, uint32_t u, uint32_t v) {
  if (u >= p.dist_len || v >= p.dist_len) return false;
  const uint32_t du = p.dist[u], dv = p.dist[v];
  return du != kUnreachable && dv != kUnreachable && du + 1 == dv;
}

// Is (u, v) a final deletion of the staged batch?  fu/fv sorted by (u, v).
__device__ bool is_final_deletion(const Params& p, uint32_t F, uint32_t u, uint32_t v) {
  uint32_t lo = 0, hi = F;
  while (lo < hi) {
    const uint32_t mid = (lo + hi) >> 1;
    const uint32_t mu = p.fu[mid], mv = p.fv[mid];
    if (mu < u || (mu == u && mv < v)) lo = mid + 1;
    else hi = mid;
  }
  return lo < F && p.fu[lo] == u && p.fv[lo] == v && !(p.ff[lo] & kFAdd);
}

// shortest_parent_count (bfs.hpp:211-220) on the current adjacency.
__device__ uint32_t support_of(const Params& p, uint32_t v) {
  const DevAdj& a = p.g.in;
  const uint32_t dv = p.dist[v];
  uint32_t cnt = 0;
  uint64_t b, e;
  vxb::base_range(a, v, b, e);
  for (uint64_t j = b; j < e; ++j) {
    const uint32_t x = a.col[j];
    if (x & kTomb) continue;
    if (x < p.dist_len && p.dist[x] != kUnreachable && p.dist[x] + 1 == dv) ++cnt;
  }
  const uint2 dr = a.drow[v];
  for (uint32_t j = dr.x; j < dr.x + dr.y; ++j) {
    const uint32_t x = a.darena[j];
    if (x < p.dist_len && p.dist[x] != kUnreachable && p.dist[x] + 1 == dv) ++cnt;
  }
  return cnt;
}

__device__ void check_affected(const Params& p, uint32_t v) {
  const uint32_t sup = support_of(p, v);
  if (sup != 0 && p.lost[v] >= sup) {
    atomicOr(&p.aff[v >> 5], 1u << (v & 31));
    const uint32_t slot = atomicAdd(&p.c->a_n, 1u);
    p.lst_a[slot] = v;
  }
}

// --------------------------------------------------- pre-batch fixpoint --

__device__ void repair_pre(const Params& p) {
  BfsCounters* c = p.c;
  const uint32_t F = *p.F;
  // deletion candidates: existing deleted arcs that are shortest-parent arcs
  for (uint32_t i = gtid(); i < F; i += nthreads()) {
    const uint8_t f = p.ff[i];
    if ((f & kFAdd) || !(f & kFCur)) continue;
    const uint32_t u = p.fu[i], v = p.fv[i];
    if (!is_sp(p, u, v)) continue;
    if (atomicAdd(&p.lost[v], 1u) == 0u) {
      const uint32_t slot = atomicAdd(&c->cand_n, 1u);
      p.lst_t[slot] = v;
    }
  }
  if (gtid() == 0) {
    for (int k = 0; k < 3; ++k) {
      c->list_n[k] = 0;
      c->next_seed[k] = kUnreachable;
    }
    c->seed_min = kUnreachable;
  }
  sync_grid(p);
  const uint32_t ncand = ld_cg(&c->cand_n);
  if (gtid() == 0) {
    c->candidates = ncand;
    c->touched_n = ncand;
  }
  if (ncand == 0) return;
  for (uint32_t i = gtid(); i < ncand; i += nthreads()) atomicMin(&c->seed_min, p.dist[p.lst_t[i]]);
  sync_grid(p);
  uint32_t d = ld_cg(&c->seed_min);
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
    }
    // level-d items: candidates at distance d, and children reached at d
    for (uint32_t i = gtid(); i < ncand; i += nthreads()) {
      const uint32_t v = p.lst_t[i];
      const uint32_t dv = p.dist[v];
      if (dv == d) check_affected(p, v);
      else if (dv > d) atomicMin(&c->next_seed[k1], dv);
    }
    for (uint32_t i = gtid(); i < np; i += nthreads()) check_affected(p, p.q[k][i]);
    sync_grid(p);
    const uint32_t a_tot = ld_cg(&c->a_n);
    if (a_tot > p.fallback_limit) {
      if (gtid() == 0) c->fallback = 1;
      break;
    }
    // children of the vertices that became affected at level d
    for (uint32_t i = a_prev + gtid(); i < a_tot; i += nthreads()) {
      const uint32_t u = p.lst_a[i];
      const DevAdj& a = p.g.out;
      uint64_t b, e;
      vxb::base_range(a, u, b, e);
      const uint2 dr = a.drow[u];
      const uint64_t nb = e - b;
      for (uint64_t j = 0; j < nb + dr.y; ++j) {
        uint32_t x;
        if (j < nb) {
          x = a.col[b + j];
          if (x & kTomb) continue;
        } else {
          x = a.darena[dr.x + (j - nb)];
        }
        if (x >= p.dist_len || p.dist[x] != d + 1) continue;
        if (is_final_deletion(p, F, u, x)) continue;
        if (atomicAdd(&p.lost[x], 1u) == 0u) {
          const uint32_t s1 = atomicAdd(&c->list_n[k1], 1u);
          p.q[k1][s1] = x;
          const uint32_t s2 = atomicAdd(&c->touched_n, 1u);
          p.lst_t[s2] = x;
        }
      }
    }
    sync_grid(p);
    a_prev = a_tot;
    const uint32_t nn = ld_cg(&c->list_n[k1]);
    const uint32_t ns = ld_cg(&c->next_seed[k1]);
    if (nn > 0) ++d;
    else if (ns != kUnreachable) d = ns;
    else break;
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

__device__ void repair_post(const Params& p) {
  BfsCounters* c = p.c;
  if (ld_cg(&c->fallback)) {
    clear_workspace(p);
    sync_grid(p);
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
      }
    }
    sync_grid(p);
    // boundary seeds: best non-affected in-neighbour (bfs.hpp:261-269)
    for (uint32_t i = gtid(); i < na; i += nthreads()) {
      const uint32_t v = p.lst_a[i];
      const DevAdj& a = p.g.in;
      uint32_t best = kUnreachable;
      uint64_t b, e;
      vxb::base_range(a, v, b, e);
      const uint2 dr = a.drow[v];
      const uint64_t nb = e - b;
      for (uint64_t j = 0; j < nb + dr.y; ++j) {
        uint32_t x;
        if (j < nb) {
          x = a.col[b + j];
          if (x & kTomb) continue;
        } else {
          x = a.darena[dr.x + (j - nb)];
        }
        if (x >= p.dist_len || test_bit(p.aff, x)) continue;
        const uint32_t dx = p.dist[x];
        if (dx != kUnreachable && dx + 1 < best) best = dx + 1;
      }
      p.tent[i] = best;
      p.dist[v] = best;
      if (best != kUnreachable) {
        ++reach;
        atomicMin(&c->seed_min, best);
      }
    }
    sync_grid(p);
    // bucketed settle among affected vertices (unit-weight Dijkstra)
    uint32_t lvl = ld_cg(&c->seed_min);
    if (lvl != kUnreachable) {
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
        }
        // seeds whose boundary distance is this level and still hold it
        for (uint32_t i = gtid(); i < na + nr; i += nthreads()) {
          uint32_t u;
          if (i < na) {
            const uint32_t t = p.tent[i];
            u = p.lst_a[i];
            const uint32_t du = ld_cg(&p.dist[u]);
            if (t != lvl || du != lvl) {
              if (t != kUnreachable && t > lvl && du == t) atomicMin(&c->next_seed[k1], t);
              continue;
            }
          } else {
            u = p.q[k][i - na];
          }
          const DevAdj& a = p.g.out;
          uint64_t b, e;
          vxb::base_range(a, u, b, e);
          const uint2 dr = a.drow[u];
          const uint64_t nb = e - b;
          for (uint64_t j = 0; j < nb + dr.y; ++j) {
            uint32_t x;
            if (j < nb) {
              x = a.col[b + j];
              if (x & kTomb) continue;
            } else {
              x = a.darena[dr.x + (j - nb)];
            }
            if (!test_bit(p.aff, x)) continue;
            const uint32_t cand = lvl + 1;
            if (cand >= ld_cg(&p.dist[x])) continue;
            const uint32_t old = atomicMin(&p.dist[x], cand);
            if (old > cand) {
              if (old == kUnreachable) ++reach;
              const uint32_t s = atomicAdd(&c->list_n[k1], 1u);
              p.q[k1][s] = x;
            }
          }
        }
        sync_grid(p);
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
    for (int k = 0; k < 3; ++k) c->list_n[k] = 0;
  }
  sync_grid(p);
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
  sync_grid(p);
  for (uint32_t r = 0;; ++r) {
    if (r > p.dist_len + 1) {
      if (gtid() == 0) atomicOr(&c->err, vxb::kErrLoopBound);
      break;
    }
    const int k = r % 3, k1 = (r + 1) % 3, k2 = (r + 2) % 3;
    const uint32_t n = ld_cg(&c->list_n[k]);
    if (n == 0) break;
    if (gtid() == 0) c->list_n[k2] = 0;
    uint32_t* inq_cur = p.inq[r & 1];
    uint32_t* inq_nxt = p.inq[(r + 1) & 1];
    for (uint32_t i = gtid(); i < n; i += nthreads()) {
      const uint32_t u = p.q[k][i];
      atomicAnd(&inq_cur[u >> 5], ~(1u << (u & 31)));
      const uint32_t du = ld_cg(&p.dist[u]);
      if (du == kUnreachable) continue;
      const DevAdj& a = p.g.out;
      uint64_t b, e;
      vxb::base_range(a, u, b, e);
      const uint2 dr = a.drow[u];
      const uint64_t nb = e - b;
      for (uint64_t j = 0; j < nb + dr.y; ++j) {
        uint32_t x;
        if (j < nb) {
          x = a.col[b + j];
          if (x & kTomb) continue;
        } else {
          x = a.darena[dr.x + (j - nb)];
        }
        lower_and_queue(p, x, du + 1, inq_nxt, p.q[k1], &c->list_n[k1], reach);
      }
    }
    sync_grid(p);
  }
  reach = vxb::warp_sum(reach);
  if ((threadIdx.x & 31) == 0) reach_add(p, reach);
  clear_workspace(p);
}

__global__ void __launch_bounds__(kThreads, 2) bfs_kernel(Params p, int mode) {
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
      cudaMallocHost(&b->hctr, sizeof(BfsCounters)) != cudaSuccess) {
    set_error("BFS counter allocation failed");
    bfs_destroy(b);
    return -4;
  }
  cudaMemsetAsync(b->ctr, 0, sizeof(BfsCounters), g->stream);
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

int bfs_apply_staged(Bfs* b, size_t n, size_t vertex_bound) {
  Graph* g = b->g;
  cudaStream_t s = g->stream;
  // last_* counters reset on every apply (bfs.hpp:30-33)
  VX_CUDA_TRY(cudaMemsetAsync(&b->ctr->candidates, 0, 4 * sizeof(uint32_t), s));
  if (n == 0) return 0;
  const size_t V_pre = g->V;
  const size_t len_pre = b->dist_len;
  VX_CUDA_TRY(cudaMemsetAsync(&b->ctr->cand_n, 0, 3 * sizeof(uint32_t), s));
  if (int rc = graph_stage_batch(g, n, vertex_bound)) return rc;
  const size_t V_post = g->V;
  if (int rc = ensure_capacity(b, std::max<size_t>(V_post, 1))) return rc;
  // fallback limit: max(1, size_t(double(V) * fraction))  (bfs.hpp:225-226)
  unsigned long long lim = (unsigned long long)((double)V_pre * b->frac);
  if (lim < 1) lim = 1;
  {
    Params p = make_params(b, (uint32_t)V_pre, (uint32_t)len_pre);
    p.fallback_limit = lim;
    if (len_pre > 0)
      if (int rc = launch(b, p, kModePre)) return rc;
  }
  if (int rc = graph_commit_batch(g)) return rc;
  if (b->dist_len < V_post) {
    VX_CUDA_TRY(cudaMemsetAsync(b->dist + b->dist_len, 0xFF, (V_post - b->dist_len) * 4, s));
    b->dist_len = V_post;
  }
  Params p = make_params(b, (uint32_t)V_post, (uint32_t)b->dist_len);
  p.fallback_limit = lim;
  return launch(b, p, kModePost);
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
  unsigned long long* d = reinterpret_cast<unsigned long long*>(&b->ctr->pad);
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
