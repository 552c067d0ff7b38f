// Full BFS and incremental repair as persistent cooperative kernels.
//
// Two kernels, each a single co-resident grid that synchronises with the
// bounded grid_barrier: bfs_full_kernel runs the full BFS (kModeFull) and
// bfs_kernel the two repair modes.
//
//   kModeFull  recompute (bfs.hpp:100-120) as a direction-optimising BFS:
//              top-down levels expand a frontier queue with warp-cooperative
//              gathers (rows < 32 arcs flattened across the warp, medium rows
//              expanded by the whole warp, rows >= tune.large_row expanded by
//              the whole grid), bottom-up levels scan candidate lists a warp
//              per 32 vertices and stop each scan at the first parent in the
//              frontier bitmap.  Claims are atomicOr on the visited bitmap,
//              frontier queues are appended with warp-aggregated atomics.
//   kModePre   the pre-batch part of apply (bfs.hpp:38-70, 222-259): deletion
//              candidates and the support-count fixpoint, run as one
//              asynchronous cascade over a work ring (no barrier per level).
//   kModePost  the post-batch part (bfs.hpp:72-97, 261-354): either the
//              fallback full BFS, or invalidation and boundary distances of
//              the affected vertices, then one asynchronous label-correcting
//              relaxation from them and from the heads of inserted arcs.
#include <algorithm>
#include <atomic>
#include <cstring>
#include <vector>

#include "bfs.cuh"
#include "vstream.cuh"
#include "graph_dev.cuh"
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
// slots past the vertex count in each candidate list: the per-block segments
// of ceil(V / blocks) slots cover at most V + blocks - 1 (blocks <= 148 * 4)
constexpr uint32_t kListSlack = 1024;

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
  uint32_t* tent;
  uint32_t* bul;      // bottom-up candidate lists A (bul[0, bul_half)) and B (bul[bul_half, 2 * bul_half)),
  uint32_t bul_half;  // each cut into one segment per block (bul_half >= V + blocks)
  unsigned long long* sw;  // support words of the pre-batch cascade (zero between batches)
  unsigned long long* ring;  // work ring of the repair phases (kSent between phases)
  uint32_t ring_mask;
  uint32_t* rq_head;       // ring counters, each on its own 128-byte line: the
  uint32_t* rq_tail;       // idle blocks poll them while the working ones push
  uint32_t* rq_done;
  uint32_t* rq_fin;        // set by the first block that sees the phase finished
  unsigned long long* rq_stat;  // drain statistics of the last phase (own line)
  uint32_t* aff;
  uint32_t* inq[2];
  const uint32_t* fu;
  const uint32_t* fv;
  const uint8_t* ff;
  const uint32_t* F;
  BfsCounters* c;
  unsigned long long total_arcs;
  unsigned long long fallback_limit;
  float handover;        // time budget of a repair phase, in multiples of the last full BFS's time
  uint32_t cascade_bfs;  // the cascade may hand over (the distance vector spans the graph)
  float alpha, beta;
  uint32_t large_row;
  uint32_t nblocks;
  unsigned long long* trace;  // optional per-level {time, n_f | bottom-up << 63}
  // optional accounting of the update launch's algorithmic bytes (null: off):
  // [0] row arcs scanned by the repair, [1] vertices it visited, [2] delta-row
  // entries the commit read and wrote, [3] canonical arcs, [4] batches
  unsigned long long* acct;
  uint32_t* bar;              // grid barrier words
};

constexpr uint32_t kTraceLevels = 256;

// Time budgets of the repair phases.  On a deep graph one batch can move the
// distances of millions of vertices, and the cascade or the relaxation then
// walks them level by level, for far longer than a full BFS takes.  A phase
// that has run longer than handover x the last full BFS's time drops the rest
// of its queue and a BFS finishes its work, so a batch costs at most about
// twice the cheaper of the two; either way the result is the same.  The
// deadline is set by thread 0 before the barrier that precedes the phase's
// drain, which reads it once and compares it with the clock every round.  The cascade's BFS compares distances over every vertex of the
// phase graph, so it may hand over only when the distance vector spans it.
constexpr unsigned long long kNever = ~0ull;

__device__ __forceinline__ void set_deadline(const Params& p) {
  const float h = p.handover;
  const unsigned long long f = p.c->full_ns;
  p.c->deadline = h < 0.0f || (h > 0.0f && f == 0ull)
                      ? kNever
                      : globaltimer() + (unsigned long long)((double)h * (double)f);
}

__device__ __forceinline__ void acct_add(const Params& p, int k, unsigned long long v) {
  if (p.acct && v) atomicAdd(&p.acct[k], v);
}

// Grid barrier; returns false once any block recorded a device error (a
// barrier that gave up waiting, a loop bound), so every persistent loop ends.
__device__ __forceinline__ bool sync_grid(const Params& p) {
  vxb::grid_barrier(p.bar, p.nblocks, &p.c->err);
  return __ldcg(&p.c->err) == 0u;
}


// ------------------------------------------------------------ top-down --

struct TdVisit {
  const Params* p;
  uint32_t* dist;
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
      if (!(w & bit)) {
        // the row length is loaded before the claim, so both are in flight together
        const uint64_t deg = want_deg ? degree_of(p->g.out, x) : 0ull;
        claim = !(atomicOr(&p->vis[x >> 5], bit) & bit);
        if (claim) mloc += deg;
      }
    }
    if (claim) {
      dist[x] = level + 1;
      atomicOr(&fbn[x >> 5], bit);
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

// Appends v where pred holds to a block-private list segment (seg, counter
// n in shared memory), in lane order within the warp.  Warp-uniform.
__device__ __forceinline__ void seg_append(bool pred, uint32_t v, uint32_t* seg, uint32_t* n) {
  const uint32_t m = __ballot_sync(FULL, pred);
  if (!m) return;
  const int lane = threadIdx.x & 31, leader = __ffs(m) - 1;
  uint32_t base = 0;
  if (lane == leader) base = atomicAdd(n, (uint32_t)__popc(m));
  base = __shfl_sync(FULL, base, leader);
  if (pred) seg[base + __popc(m & vxb::lanemask_lt())] = v;
}

// Bottom-up over this block's segment of a candidate list: lin[0, nin) holds
// vertices that may still be reached (unvisited when the list was made,
// in-degree > 0; the first list is every such vertex of the block's range,
// built by the full BFS's initialisation, later ones the previous level's
// misses).  One warp per 32 entries: each lane scans the first kBuHead
// in-arcs of its row, the rest of longer rows is scanned by the whole warp 32
// arcs at a time, every scan stops at the first parent in the frontier
// bitmap.  Entries visited since the list was made are skipped; entries that
// find no parent go to the block's segment of the other list (lout, counter
// nout in shared memory), so isolated vertices cost nothing and a later level
// scans only the vertices still unreached.  Entries are loaded two groups
// ahead and their visited words and row bounds one group ahead, so those
// loads are in flight while a group is scanned.  Block-uniform.
__device__ void bu_list_level(const Params& p, uint32_t* dist, uint32_t level, const uint32_t* fbc, uint32_t* fbn,
                              uint32_t* qout, uint32_t* cnt_n, BlockQueue& bq, const uint32_t* lin, uint32_t nin,
                              uint32_t* lout, uint32_t* nout) {
  const DevAdj& a = p.g.in;
  const int lane = threadIdx.x & 31;
  const uint32_t step = kThreads;  // the block's warps take consecutive 32-entry groups
  uint32_t base = (threadIdx.x >> 5) * 32;
  uint32_t v1 = base + step + lane < nin ? lin[base + step + lane] : kUnreachable;
  uint32_t v0 = base + lane < nin ? lin[base + lane] : kUnreachable;
  uint32_t vis0 = 0;
  uint64_t b0 = 0, e0 = 0;
  uint2 dr0 = make_uint2(0, 0);
  if (v0 != kUnreachable) {
    vis0 = p.vis[v0 >> 5];
    vxb::base_range(a, v0, b0, e0);
    dr0 = a.drow[v0];
  }
  for (; base < nin; base += step) {
    const uint32_t v = v0, visw = vis0;
    uint64_t b = b0, e = e0;
    uint2 dr = dr0;
    // advance the pipeline: row bounds of the next group, entries of the one after
    v0 = v1;
    vis0 = 0;
    b0 = e0 = 0;
    dr0 = make_uint2(0, 0);
    if (v0 != kUnreachable) {
      vis0 = p.vis[v0 >> 5];
      vxb::base_range(a, v0, b0, e0);
      dr0 = a.drow[v0];
    }
    const uint32_t i2 = base + 2 * step + lane;
    v1 = i2 < nin ? lin[i2] : kUnreachable;
    const bool todo = v != kUnreachable && !((visw >> (v & 31)) & 1u);
    if (!todo) {
      b = e = 0;
      dr = make_uint2(0, 0);
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
    if (found) dist[v] = level + 1;
    // visited and next-frontier bits: OR-combined over runs of lanes on the
    // same bitmap word (list entries come in ascending runs), one atomic per
    // run; a word that recurs outside its run is ORed again, which is harmless
    const uint32_t word = v >> 5;
    uint32_t bits = found ? 1u << (v & 31) : 0u;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const uint32_t y = __shfl_up_sync(FULL, bits, o);
      const uint32_t wy = __shfl_up_sync(FULL, word, o);
      if (lane >= o && wy == word) bits |= y;
    }
    const uint32_t wnext = __shfl_down_sync(FULL, word, 1);
    if (bits && (lane == 31 || wnext != word)) {
      atomicOr(&p.vis[word], bits);
      atomicOr(&fbn[word], bits);
    }
    bq_push(bq, found, v, cnt_n, qout);
    seg_append(todo && !found, v, lout, nout);
  }
  bq_flush(bq, cnt_n, qout);
}

// ------------------------------------------------------------ full BFS --

__device__ void full_bfs(const Params& p, BlockQueue& bq, LbStage& lbst, uint32_t* dist,
                         unsigned long long* trace) {
  BfsCounters* c = p.c;
  const unsigned long long t_start = gtid() == 0 ? globaltimer() : 0ull;  // the repair phases' time budget
  __shared__ uint32_t seg_n[2];  // entries of this block's segment of each candidate list
  if (threadIdx.x == 0) bq.cnt = 0;
  const uint32_t V = p.V;
  const uint32_t words = (V + 31) >> 5;
  // one pass sets every vertex unreached and the source at level 0 (bits
  // past V count as visited, so bottom-up never scans them), and lists the
  // bottom-up candidates: every vertex but the source with a nonempty in-row
  // (isolated vertices never enter a bottom-up level).  Each block takes a
  // contiguous range of vertices and lists its candidates in its own segment
  // of list A (shared-memory counter, no global atomics); a bottom-up level
  // scans the block's own segment.
  const uint32_t s = p.source;
  const bool has_source = s < V;
  const uint32_t seg = (V + gridDim.x - 1) / gridDim.x;  // vertices (and list slots) per block
  const uint32_t seg_lo = blockIdx.x * seg, seg_hi = min(V, seg_lo + seg);
  if (threadIdx.x == 0) seg_n[0] = seg_n[1] = 0;
  __syncthreads();
  for (uint32_t i0 = seg_lo; i0 < seg_hi; i0 += kThreads) {
    const uint32_t i = i0 + threadIdx.x;
    bool cand = false;
    if (i < seg_hi) {
      dist[i] = i == s ? 0u : kUnreachable;
      cand = has_source && i != s && degree_of(p.g.in, i) != 0u;
    }
    seg_append(cand, i, p.bul + seg_lo, &seg_n[0]);
  }
  for (uint32_t i = gtid(); i < words; i += nthreads()) {
    const uint32_t lo = i * 32;
    const uint32_t sbit = has_source && i == (s >> 5) ? 1u << (s & 31) : 0u;
    p.vis[i] = ((lo + 32 <= V) ? 0u : (FULL << (V - lo))) | sbit;
    p.fb[0][i] = sbit;
    p.fb[1][i] = p.fb[2][i] = 0u;
  }
  if (gtid() == 0) {
    for (int k = 0; k < 3; ++k) {
      c->lvl_n[k] = 0;
      c->lvl_big[k] = 0;
      c->lvl_m[k] = 0;
    }
    if (has_source) {
      p.q[0][0] = s;
      c->lvl_n[0] = 1;
      c->lvl_m[0] = degree_of(p.g.out, s);
    } else {
      c->reachable = 0;
      c->levels = 0;
      c->arcs = 0;
    }
  }
  if (!sync_grid(p) || !has_source) return;
  unsigned long long m_visited = 0;
  uint32_t reached = 0;
  bool bottom_up = false, left_bu = false;
  uint32_t prev_n = 0;
  uint32_t level = 0;
  // the frontier size and arc count of the current level, read once after the
  // barrier that ends the level before it
  uint32_t n_f = ld_cg(&c->lvl_n[0]);
  unsigned long long m_f = __ldcg(&c->lvl_m[0]);
  // bottom-up candidate lists: the first bottom-up level reads list 0
  uint32_t lin = 0;
  for (;; ++level) {
    if (level > V + 1) {
      if (gtid() == 0) atomicOr(&c->err, vxb::kErrLoopBound);
      break;
    }
    const int cur = level % 3, nxt = (level + 1) % 3, clr = (level + 2) % 3;
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
      if (trace && level < kTraceLevels) {
        trace[2 * level] = globaltimer();
        trace[2 * level + 1] = (unsigned long long)n_f | ((unsigned long long)bottom_up << 63);
      }
    }
    // clear the frontier bitmap of level-1: through its queue when it was
    // small, else word by word (plain stores, no dependent queue loads)
    if ((unsigned long long)prev_n * 8 < words) {
      for (uint32_t i = gtid(); i < prev_n; i += nthreads()) p.fb[clr][p.q[clr][i] >> 5] = 0u;
    } else {
      for (uint32_t i = gtid(); i < words; i += nthreads()) p.fb[clr][i] = 0u;
    }
    if (bottom_up) {
      const uint32_t lout = lin ^ 1u;
      if (threadIdx.x == 0) seg_n[lout] = 0;
      __syncthreads();
      bu_list_level(p, dist, level, p.fb[cur], p.fb[nxt], p.q[nxt], &c->lvl_n[nxt], bq, p.bul + lin * p.bul_half + seg_lo,
                    seg_n[lin], p.bul + lout * p.bul_half + seg_lo, &seg_n[lout]);
      lin = lout;
      if (!sync_grid(p)) return;
      prev_n = n_f;
      n_f = ld_cg(&c->lvl_n[nxt]);
      m_f = __ldcg(&c->lvl_m[nxt]);
    } else {
      TdVisit t{&p, dist, level, p.q[nxt], p.fb[nxt], &c->lvl_n[nxt], !left_bu, 0ull, &bq};
      if (n_f <= kLbMax) td_level_lb(p, t, p.q[cur], n_f, lbst);
      else td_level(p, t, p.q[cur], n_f, &c->lvl_big[cur]);
      t.flush(&c->lvl_m[nxt]);
      bq_flush(bq, &c->lvl_n[nxt], p.q[nxt]);
      if (!sync_grid(p)) return;
      // three independent loads: the next level's figures stand unless hub rows remain
      prev_n = n_f;
      const uint32_t nbig = ld_cg(&c->lvl_big[cur]);
      n_f = ld_cg(&c->lvl_n[nxt]);
      m_f = __ldcg(&c->lvl_m[nxt]);
      if (nbig) {
        grid_rows(p.g.out, p.big, nbig, t);
        t.flush(&c->lvl_m[nxt]);
        bq_flush(bq, &c->lvl_n[nxt], p.q[nxt]);
        if (!sync_grid(p)) return;
        n_f = ld_cg(&c->lvl_n[nxt]);
        m_f = __ldcg(&c->lvl_m[nxt]);
      }
    }
  }
  if (gtid() == 0) {
    c->reachable = reached;
    c->levels = level;
    c->arcs = m_visited;
    c->full_ns = globaltimer() - t_start;
    if (trace && level < kTraceLevels) {
      trace[2 * level] = globaltimer();
      trace[2 * level + 1] = 0;
    }
  }
}

// ------------------------------------------------------------- helpers --

__device__ __forceinline__ bool is_sp(const Params& p, uint32_t u, uint32_t v) {
  if (u >= p.dist_len || v >= p.dist_len) return false;
  const uint32_t du = p.dist[u], dv = p.dist[v];
  return du != kUnreachable && dv != kUnreachable && du + 1 == dv;
}

__device__ __forceinline__ void reach_add(const Params& p, long long d) {
  if (d) atomicAdd(&p.c->reachable, (unsigned long long)d);
}

// ------------------------------------------------- asynchronous work ring --
// The repair phases are dependency chains a few vertices wide and as deep as
// the tree below a deletion or an insertion.  Level-synchronous rounds would
// pay a grid barrier per level; instead each phase drains a work ring: blocks
// claim items, expand their rows, and push the vertices they change, with no
// barrier until the ring is empty.
//
// The ring holds 64-bit items (kSent = empty slot) at slot[i & ring_mask]:
// bits 0-30 a vertex, bit 31 the cascade's expand kind, bits 32-62 the chunk
// of the vertex's row the item covers (rows longer than kChunk arcs are split
// by the block that claims their first chunk, so a hub is spread over
// blocks), bit 63 the cascade's chunk-check kind;
// head / tail / done count claimed, pushed and finished items.  A block ends
// the phase once it sees done == tail (read in that order): every push happens
// while its pusher's item is unfinished, so at that moment nothing is in
// flight.  Every wait is bounded and records kErrDrainTimeout when it gives up.

constexpr unsigned long long kSent = ~0ull;
constexpr uint32_t kChunk = 128;  // arcs of one ring item: a 32-item round stays within 4096 arcs

// Bit test through L2: bits another block sets during a phase.
__device__ __forceinline__ bool test_bit_cg(const uint32_t* bm, uint32_t v) {
  return (__ldcg(&bm[v >> 5]) >> (v & 31)) & 1u;
}
constexpr uint32_t kKindBit = 0x80000000u;  // cascade items: set = expand an affected vertex
constexpr unsigned long long kChunkCheckBit = 1ull << 63;  // cascade items: one chunk of a long check
constexpr uint32_t kDrainIdleLimit = 1u << 20;  // idle rounds of a block (up to 2 us each)

__device__ __forceinline__ void ring_push(const Params& p, bool pred, unsigned long long item) {
  const uint32_t s = vxb::warp_append(pred, p.rq_tail);  // warp-uniform
  if (pred) __stcg(&p.ring[s & p.ring_mask], item);
}

__device__ __forceinline__ uint32_t item_vertex(unsigned long long it) { return (uint32_t)it & ~kKindBit; }
__device__ __forceinline__ uint32_t item_chunk(unsigned long long it) { return (uint32_t)(it >> 32) & 0x7FFFFFFFu; }

// Stages the rows of n <= kThreads items (one per thread; kSent items have no
// row) with their degree prefix in shared memory, then every warp of the block
// takes 32 consecutive arcs of the flattened range per step, so one long row
// is spread over the whole block.  f(valid, x, j) gets the owning item's index
// and is called warp-uniformly.  With 64-bit ring items (p non-null) an item
// covers one kChunk-arc chunk of its row, and the claimer of a row's first
// chunk pushes the rest as items of their own.
template <class T, class F>
__device__ void block_rows(const DevAdj& a, const T* items, uint32_t n, LbStage& st, F& f,
                           const Params* p = nullptr, unsigned long long* acct = nullptr) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  __shared__ uint32_t wsum[kThreads / 32];
  uint32_t len = 0;
  if (threadIdx.x < n) {
    const T it = items[threadIdx.x];
    uint64_t b = 0, e = 0;
    uint2 dr = make_uint2(0, 0);
    if (it != (T)kSent) {
      const uint32_t u = (uint32_t)it & ~kKindBit;
      vxb::base_range(a, u, b, e);
      dr = a.drow[u];
    }
    uint32_t blen = (uint32_t)(e - b), dx = dr.x, dlen = dr.y;
    if (p && it != (T)kSent) {
      const uint32_t total = blen + dlen, c = (uint32_t)((unsigned long long)it >> 32) & 0x7FFFFFFFu;
      const uint32_t lo = c * kChunk, hi = min(total, lo + kChunk);
      if (c == 0 && total > kChunk) {  // hand the other chunks to other blocks
        const uint32_t more = (total - 1) / kChunk;
        const uint32_t s0 = atomicAdd(p->rq_tail, more);
        for (uint32_t k = 0; k < more; ++k)
          __stcg(&p->ring[(s0 + k) & p->ring_mask], ((unsigned long long)it & 0xFFFFFFFFull) |
                                                        ((unsigned long long)(k + 1) << 32));
      }
      const uint32_t bl = lo < blen ? min(blen, hi) - lo : 0u;
      const uint32_t dl = hi > max(lo, blen) ? hi - max(lo, blen) : 0u;
      b += lo < blen ? lo : blen;
      dx += lo > blen ? lo - blen : 0u;
      blen = bl;
      dlen = dl;
    }
    st.base[threadIdx.x] = b;
    st.blen[threadIdx.x] = blen;
    st.dx[threadIdx.x] = dx;
    len = blen + dlen;
  }
  uint32_t incl = len;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const uint32_t y = __shfl_up_sync(FULL, incl, o);
    if (lane >= o) incl += y;
  }
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
  const uint32_t ex = wsum[warp] + incl - len;
  if (threadIdx.x < n) st.pref[threadIdx.x] = ex;
  if (threadIdx.x + 1 == n) st.pref[n] = ex + len;
  __syncthreads();
  const uint32_t M = n ? st.pref[n] : 0u;
  if (acct && threadIdx.x == 0 && M) atomicAdd(&acct[0], (unsigned long long)M);
  for (uint32_t e0 = (uint32_t)warp * 32; e0 < M; e0 += kThreads) {
    const uint32_t e = e0 + lane;
    bool valid = false;
    uint32_t x = 0, j = 0;
    if (e < M) {
      uint32_t lo = 0, hi = n;  // last j with pref[j] <= e
      while (hi - lo > 1) {
        const uint32_t mid = (lo + hi) >> 1;
        if (st.pref[mid] <= e) lo = mid;
        else hi = mid;
      }
      j = lo;
      const uint32_t k = e - st.pref[j];
      if (k < st.blen[j]) {
        x = a.col[st.base[j] + k];
        valid = !(x & kTomb);
        x &= kIdMask;
      } else {
        x = a.darena[st.dx[j] + (k - st.blen[j])];
        valid = true;
      }
    }
    f(valid, x, j);
  }
  __syncthreads();  // st is reused by the next call
}

// Shared memory of one block for the repair phases.
struct RepairSmem {
  unsigned long long items[kThreads];  // claimed ring items
  uint32_t sv[kThreads];     // check items (vertex); boundary chunk vertices
  unsigned long long ex[kThreads];     // expand items (vertex, chunk)
  uint32_t cnt[kThreads];    // chunk + 1 of a chunk-check sv item (0: plain check); boundary minima
  uint32_t d[kThreads];      // distance of each staged item
  uint32_t g0, n, stop, nsv, nex, fallback;
  uint32_t late;     // the round started past the phase's deadline (its items are dropped)
  uint32_t flagged;  // this block has raised the phase's handover flag
};

// Drains the ring; W::process(sm, n) handles sm.items[0, n) block-uniformly,
// with sm.late set for a round that starts at or past the deadline (a
// globaltimer value read once per round by warp 0, no memory access).
//
// A block takes a ticket of kClaim consecutive ring indices (one atomicAdd,
// which never fails) and warp 0 polls the ticket's own slots: items pushed
// into them are processed as they arrive, and the next ticket is taken once
// the current one is used up.  Indices past the tail belong to whichever
// block holds them, so pushes spread over the blocks waiting for work, and no
// two blocks poll the same address.  Every few idle rounds a block checks
// done == tail; the first to see it raises rq_fin, which the other idle
// blocks read every round, and all leave the phase.
constexpr uint32_t kClaim = 32;

template <class W>
__device__ void drain(const Params& p, RepairSmem& sm, W& w, unsigned long long deadline) {
  BfsCounters* c = p.c;
  const int lane = threadIdx.x & 31;
  uint32_t cur = 0, end = 0;  // warp 0's ticket [cur, end), uniform over its lanes
  uint32_t idle = 0;
  if (threadIdx.x == 0) sm.flagged = 0;
  for (;;) {
    if (threadIdx.x < 32) {
      uint32_t n = 0, stop = 0;
      if (ld_cg(&c->err)) {
        stop = 1;
      } else {
        if (cur == end) {
          uint32_t s0 = 0;
          if (lane == 0) {
            s0 = atomicAdd(p.rq_head, kClaim);
            atomicAdd(&p.rq_stat[1], 1ull);
          }
          cur = __shfl_sync(FULL, s0, 0);
          end = cur + kClaim;
        }
        const uint32_t k = cur + lane;
        unsigned long long v = kSent;
        if (k < end) v = __ldcg(&p.ring[k & p.ring_mask]);
        const uint32_t have = __ballot_sync(FULL, v != kSent);
        n = have == FULL ? 32u : (uint32_t)(__ffs(~have) - 1);  // leading filled slots
        if ((uint32_t)lane < n) {
          sm.items[lane] = v;
          __stcg(&p.ring[k & p.ring_mask], kSent);
        }
        cur += n;
        if (n == 0) {
          uint32_t st = 0;
          if (lane == 0) {
            st = ld_cg(p.rq_fin);
            if (!st && (idle & 3) == 3) {
              const uint32_t dn = ld_cg(p.rq_done);
              __threadfence();
              st = dn == ld_cg(p.rq_tail);
              if (st) atomicExch(p.rq_fin, 1u);  // releases the other blocks at their next idle round
              atomicAdd(&p.rq_stat[3], 1ull);
            }
          }
          stop = __shfl_sync(FULL, st, 0);
        }
      }
      if (lane == 0) {
        sm.n = n;
        sm.stop = stop;
        sm.late = n && globaltimer() >= deadline;
      }
    }
    __syncthreads();
    const uint32_t n = sm.n, stop = sm.stop;
    __syncthreads();  // every thread has read the words before warp 0 rewrites them
    if (stop) break;
    if (n == 0) {
      if (threadIdx.x == 0) atomicAdd(&p.rq_stat[2], 1ull);
      if (++idle > kDrainIdleLimit) {
        if (threadIdx.x == 0) atomicOr(&c->err, vxb::kErrDrainTimeout);
        break;
      }
      __nanosleep(32u << min(idle >> 2, 4u));  // back off to 512 ns
      continue;
    }
    idle = 0;
    const long long t0 = clock64();
    w.process(sm, n);
    __syncthreads();
    if (threadIdx.x == 0) {
      acct_add(p, 1, n);
      __threadfence();  // this block's pushes are visible before its items count as done
      atomicAdd(p.rq_done, n);
      atomicAdd(&p.rq_stat[0], 1ull);
      const unsigned long long dt = (unsigned long long)(clock64() - t0);
      atomicAdd(&p.rq_stat[4], dt);
      atomicMax(&p.rq_stat[5], dt);
    }
  }
}

// --------------------------------------------------- pre-batch fixpoint --
//
// compute_affected_prebatch (bfs.hpp:222-259): a touched vertex x at
// distance d is affected iff none of its shortest parents survives -- every
// in-neighbour at d-1 is reached over a deleted arc or is affected itself
// (the reference's lost >= support).  The fixpoint does not depend on the
// order, so it runs as one asynchronous cascade with a witness per vertex:
//
//   check(x)   scan x's in-row from the saved position for the first parent
//              that survives and is not affected; record it as the witness,
//              or mark x affected when the row is exhausted.  Affectedness
//              only grows, so a rescan never goes back.
//   expand(y)  y became affected: its children whose witness is y (or that
//              no check has touched yet) get a check.
//
// In-rows longer than kChunk arcs are checked in chunks by many warps at once
// (chunk_check); their passes always start from the row's beginning.
//
// sw[x] packs bit 63 touched, bits 32-62 witness + 1 (0 = none yet), bits
// 0-31 the scan position.  A check stores its witness, fences, and re-reads
// the witness's affected bit; mark_affected sets the bit and fences before
// the expand item is pushed -- so either the check sees the parent affected
// and scans on, or the expansion sees the witness and asks for a recheck.
// Requests are deduplicated by a bit in inq[1], cleared when a check starts.

constexpr unsigned long long kSwTouched = 1ull << 63;

// Marks v affected once (the affected bit decides); true for the caller that set it.
__device__ __forceinline__ bool mark_affected(const Params& p, uint32_t v) {
  const uint32_t bit = 1u << (v & 31);
  if (atomicOr(&p.aff[v >> 5], bit) & bit) return false;
  const uint32_t slot = atomicAdd(&p.c->a_n, 1u);
  p.lst_a[slot] = v;
  if (slot + 1 > p.fallback_limit) p.c->fallback = 1;
  __threadfence();  // the affected bit is visible before the expand item is
  return true;
}

// Warp-uniform: request a check of x where pred holds (first touch is recorded
// in sw and in the touched list; a pending request is not repeated).  The
// touched-list and ring reservations are one atomic each, both in flight
// before either result is used.
__device__ __forceinline__ void request_check(const Params& p, bool pred, uint32_t x) {
  bool first = false, push = false;
  if (pred) {
    first = !(atomicOr(&p.sw[x], kSwTouched) & kSwTouched);
    const uint32_t bit = 1u << (x & 31);
    push = !(atomicOr(&p.inq[1][x >> 5], bit) & bit);
  }
  const uint32_t mf = __ballot_sync(FULL, first), mp = __ballot_sync(FULL, push);
  if (!(mf | mp)) return;
  const int lane = threadIdx.x & 31;
  const int lf = mf ? __ffs(mf) - 1 : 0, lp = mp ? __ffs(mp) - 1 : 0;
  uint32_t bf = 0, bp = 0;
  if (mf && lane == lf) bf = atomicAdd(&p.c->touched_n, (uint32_t)__popc(mf));
  if (mp && lane == lp) bp = atomicAdd(p.rq_tail, (uint32_t)__popc(mp));
  bf = __shfl_sync(FULL, bf, lf);
  bp = __shfl_sync(FULL, bp, lp);
  const uint32_t lt = vxb::lanemask_lt();
  if (first) p.lst_t[bf + __popc(mf & lt)] = x;
  if (push) __stcg(&p.ring[(bp + __popc(mp & lt)) & p.ring_mask], (unsigned long long)x);
}

// expand(y) for a newly affected y at distance dy, applied to one arc (y, x)
// of y's out-row (warp-uniform): x gets a check if it sits at dy + 1 and its
// witness is y or no check has touched it yet.
constexpr uint32_t kInlineExpand = 64;  // out-rows this short are expanded by the warp that marked y
struct ExpandChildren {
  const Params* p;
  uint32_t y, dy;
  __device__ __forceinline__ void operator()(bool valid, uint32_t x, uint32_t) {
    bool need = false;
    if (valid && x < p->dist_len) {
      const uint32_t dx = p->dist[x];
      const unsigned long long w = __ldcg(&p->sw[x]);
      const uint32_t wit = (uint32_t)(w >> 32) & 0x7FFFFFFFu;
      need = dx == dy + 1 && (!(w & kSwTouched) || wit == y + 1);
    }
    request_check(*p, need, x);
  }
};

// First position k in [lo, hi) of x's in-row (base part [b, b + nb), delta
// part from darena[dx]) whose tail y survives, sits at distance d - 1 and is
// not affected; whole warp, warp-uniform result.  Each step covers 128 arcs:
// every lane issues its four column loads, then the four distance and
// affected-bit loads, so a step costs two dependent round trips however many
// of its arcs are needed.
__device__ __forceinline__ bool find_parent(const Params& p, const DevAdj& a, uint64_t b, uint32_t nb, uint32_t dx,
                                            uint32_t lo, uint32_t hi, uint32_t d, uint32_t& kw, uint32_t& yw) {
  const int lane = threadIdx.x & 31;
  for (uint32_t k0 = lo; k0 < hi; k0 += 128) {
    if (lane == 0) acct_add(p, 0, min(128u, hi - k0));
    uint32_t y[4];
#pragma unroll
    for (int j = 0; j < 4; ++j) {
      const uint32_t k = k0 + 32 * j + lane;
      y[j] = kTomb;  // no arc
      if (k < hi) y[j] = k < nb ? a.col[b + k] : a.darena[dx + (k - nb)];
    }
    uint32_t dy[4], aw[4];
#pragma unroll
    for (int j = 0; j < 4; ++j) {
      const bool live = !(y[j] & kTomb) && y[j] < p.dist_len;
      dy[j] = live ? p.dist[y[j]] : kUnreachable;
      aw[j] = live ? __ldcg(&p.aff[y[j] >> 5]) : 0u;
    }
#pragma unroll
    for (int j = 0; j < 4; ++j) {
      const bool ok = dy[j] != kUnreachable && dy[j] + 1 == d && !((aw[j] >> (y[j] & 31)) & 1u);
      const uint32_t ball = __ballot_sync(FULL, ok);
      if (ball) {
        const int f = __ffs(ball) - 1;
        kw = k0 + 32 * j + (uint32_t)f;
        yw = __shfl_sync(FULL, y[j], f);
        return true;
      }
    }
  }
  return false;
}

// check(x), whole warp.  The scan resumes at the position saved in sw[x]:
// affectedness only grows and distances are fixed during the cascade, so an
// arc that failed once fails again.  In-rows longer than kChunk arcs are
// scanned in place over their first chunk only; when it holds no witness the
// rest goes to a chunked pass (chunk_check), and the saved position kChunk
// tells later checks to go straight to a new pass.
__device__ void check_vertex(const Params& p, uint32_t x) {
  const DevAdj& a = p.g.in;
  const int lane = threadIdx.x & 31;
  // x's distance and row bounds do not change during the cascade: they load
  // together with the clearing of the request bit
  const uint32_t d = p.dist[x];
  uint64_t b, e;
  vxb::base_range(a, x, b, e);
  const uint2 dr = a.drow[x];
  if (lane == 0) atomicAnd(&p.inq[1][x >> 5], ~(1u << (x & 31)));
  __syncwarp();
  __threadfence();  // the request bit is clear before the state (witness, affected bits) is read
  const uint32_t nb = (uint32_t)(e - b), total = nb + dr.y;
  const uint32_t lim = min(total, kChunk);
  uint32_t k0 = (uint32_t)__ldcg(&p.sw[x]);
  bool resolved = false;
  uint32_t kw = 0, yw = 0;
  while (k0 < lim && !resolved) {
    if (!find_parent(p, a, b, nb, dr.x, k0, lim, d, kw, yw)) break;
    bool still = false;
    if (lane == 0) {
      __stcg(&p.sw[x], kSwTouched | ((unsigned long long)(yw + 1) << 32) | kw);
      __threadfence();
      still = !test_bit_cg(p.aff, yw);
    }
    resolved = __shfl_sync(FULL, still, 0);
    k0 = kw + 1;  // the witness turned affected meanwhile: scan on past it
  }
  if (resolved) return;
  if (total > kChunk) {
    // the rest of a long in-row: one chunk-check item per kChunk arcs past the
    // first, scanned by many warps; tent[x] counts the chunks of the pass in
    // flight.  A request that finds a pass in flight is covered by it: the
    // pass clears tent[x] before it verifies its final witness.
    const uint32_t K = (total + kChunk - 1) / kChunk - 1;
    bool start = false;
    if (lane == 0) {
      __stcg(&p.sw[x], kSwTouched | (unsigned long long)kChunk);
      start = atomicCAS(&p.tent[x], 0u, K) == 0u;
    }
    start = __shfl_sync(FULL, start, 0);
    if (start)
      for (uint32_t c0 = 0; c0 < K; c0 += 32)
        ring_push(p, c0 + lane < K, kChunkCheckBit | ((unsigned long long)(c0 + lane + 1) << 32) | x);
    return;
  }
  bool marked = false;
  if (lane == 0) {
    __stcg(&p.sw[x], kSwTouched | (unsigned long long)total);
    marked = mark_affected(p, x);
  }
  marked = __shfl_sync(FULL, marked, 0);
  bool inlined = false;
  if (marked) {
    // a short out-row is expanded here instead of through one more ring round;
    // every lane fences after the affected bit (set and fenced by lane 0)
    // before it reads a child's witness, as the expanding block does after
    // claiming an expand item
    __syncwarp();
    __threadfence();
    // past the fallback limit the block path drops expansions; so does
    // this one (past the deadline its later rounds drop what this pushes)
    const uint32_t odeg = degree_of(p.g.out, x);
    if (odeg <= kInlineExpand && !ld_cg(&p.c->fallback)) {
      if (lane == 0) acct_add(p, 0, odeg);
      ExpandChildren ec{&p, x, d};
      warp_row(p.g.out, x, ec);
      inlined = true;
    }
  }
  ring_push(p, marked && !inlined && lane == 0, (unsigned long long)(x | kKindBit));
}

// One chunk c >= 1 of a long check (whole warp): scan [c * kChunk,
// (c + 1) * kChunk) of x's in-row for a surviving, non-affected parent, unless
// another chunk found one already (kFoundBit in tent[x]).  The last chunk of
// the pass clears tent[x], then either verifies the recorded witness (asking
// for a new check if it turned affected) or, when no chunk found one, marks x
// affected.  Witnesses are recorded with the saved position kChunk (the first
// chunk is known to hold none).
constexpr uint32_t kFoundBit = 0x80000000u;

__device__ void chunk_check(const Params& p, uint32_t x, uint32_t c) {
  const DevAdj& a = p.g.in;
  const int lane = threadIdx.x & 31;
  const uint32_t d = p.dist[x];
  uint64_t b, e;
  vxb::base_range(a, x, b, e);
  const uint2 dr = a.drow[x];
  const uint32_t nb = (uint32_t)(e - b), total = nb + dr.y;
  const uint32_t hi = min(total, (c + 1) * kChunk);
  uint32_t k0 = c * kChunk;
  bool found = (ld_cg(&p.tent[x]) & kFoundBit) != 0u;
  uint32_t kw = 0, yw = 0;
  while (k0 < hi && !found) {
    if (!find_parent(p, a, b, nb, dr.x, k0, hi, d, kw, yw)) break;
    bool good = false;
    if (lane == 0) {
      __stcg(&p.sw[x], kSwTouched | ((unsigned long long)(yw + 1) << 32) | kChunk);
      __threadfence();
      good = !test_bit_cg(p.aff, yw);
      if (good) atomicOr(&p.tent[x], kFoundBit);
    }
    found = __shfl_sync(FULL, good, 0);
    k0 = kw + 1;
  }
  bool recheck = false, aff = false;
  if (lane == 0) {
    __threadfence();
    const uint32_t old = atomicSub(&p.tent[x], 1u);
    if ((old & ~kFoundBit) == 1u) {  // the pass's last chunk
      atomicExch(&p.tent[x], 0u);
      __threadfence();
      if (old & kFoundBit) {
        const uint32_t w1 = (uint32_t)(__ldcg(&p.sw[x]) >> 32) & 0x7FFFFFFFu;
        recheck = w1 == 0u || test_bit_cg(p.aff, w1 - 1);
      } else {
        aff = mark_affected(p, x);
      }
    }
  }
  request_check(p, recheck, x);
  ring_push(p, aff, (unsigned long long)(x | kKindBit));
}

struct Cascade {
  const Params* p;
  LbStage* lb;
  __device__ void process(RepairSmem& sm, uint32_t n) {
    const Params& P = *p;
    BfsCounters* c = P.c;
    const uint32_t t = threadIdx.x;
    if (t == 0) {
      sm.nsv = 0;
      sm.nex = 0;
      // past its deadline the cascade drops the rest of its queue like the
      // fallback does; a BFS then gives the affected set (cascade_by_bfs)
      if (sm.late && !sm.flagged) {
        atomicOr(&c->cbig, 1u);
        sm.flagged = 1;
      }
      sm.fallback = ld_cg(&c->fallback) | sm.late;
    }
    __syncthreads();
    if (t < n) {
      const unsigned long long it = sm.items[t];
      if (it != kSent) {
        if (it & kChunkCheckBit) {
          const uint32_t k = atomicAdd(&sm.nsv, 1u);
          sm.sv[k] = item_vertex(it);
          sm.cnt[k] = item_chunk(it) + 1;
        } else if ((uint32_t)it & kKindBit) {
          sm.ex[atomicAdd(&sm.nex, 1u)] = it;
        } else {
          const uint32_t k = atomicAdd(&sm.nsv, 1u);
          sm.sv[k] = (uint32_t)it;
          sm.cnt[k] = 0u;
        }
      }
    }
    __threadfence();  // expand items were pushed after their affected bits
    __syncthreads();
    if (sm.fallback) {
      // past the fallback limit or the budget: drop the items, keeping the
      // request bits clear
      for (uint32_t i = t; i < sm.nsv; i += kThreads)
        if (sm.cnt[i] == 0u) atomicAnd(&P.inq[1][sm.sv[i] >> 5], ~(1u << (sm.sv[i] & 31)));
      return;
    }
    const uint32_t nsv = sm.nsv, nex = sm.nex;
    for (uint32_t i = t >> 5; i < nsv; i += kThreads / 32) {
      if (sm.cnt[i]) chunk_check(P, sm.sv[i], sm.cnt[i] - 1);
      else check_vertex(P, sm.sv[i]);
    }
    if (nex) {
      if (t < nex) sm.d[t] = P.dist[item_vertex(sm.ex[t])];
      __syncthreads();
      auto expand = [&](bool valid, uint32_t x, uint32_t j) {
        bool need = false;
        if (valid && x < P.dist_len) {  // both loads in flight together
          const uint32_t dx = P.dist[x];
          const unsigned long long w = __ldcg(&P.sw[x]);
          const uint32_t wit = (uint32_t)(w >> 32) & 0x7FFFFFFFu;
          need = dx == sm.d[j] + 1 && (!(w & kSwTouched) || wit == item_vertex(sm.ex[j]) + 1);
        }
        request_check(P, need, x);
      };
      block_rows(P.g.out, sm.ex, nex, *lb, expand, &P, P.acct);
    }
  }
};

__device__ void reset_ring(const Params& p) {
  if (gtid() == 0) {
    *p.rq_head = 0;
    *p.rq_tail = 0;
    *p.rq_done = 0;
    *p.rq_fin = 0;
    for (int k = 0; k < 6; ++k) p.rq_stat[k] = 0;
  }
}

__device__ __forceinline__ void stamp(const Params& p, int k) {
  if (gtid() == 0) p.c->rtrace[k] = globaltimer();
}

// Deletion candidates (bfs.hpp:52-63): heads of deleted shortest-parent arcs.
// The first touch of each records it in the touched list, so the list's
// first cand_n entries are the candidates.  Warp-uniform.
__device__ void register_candidates(const Params& p) {
  BfsCounters* c = p.c;
  const int lane = threadIdx.x & 31;
  const uint32_t F = *p.F;
  for (uint32_t base = gwarp() * 32; base < F; base += nwarps() * 32) {
    const uint32_t i = base + lane;
    bool first = false;
    uint32_t v = 0;
    if (i < F) {
      const uint8_t f = p.ff[i];
      const uint32_t u = p.fu[i];
      v = p.fv[i];
      if (!(f & kFAdd) && (f & kFCur) && is_sp(p, u, v)) first = !(atomicOr(&p.sw[v], kSwTouched) & kSwTouched);
    }
    const uint32_t slot = vxb::warp_append(first, &c->touched_n);
    if (first) p.lst_t[slot] = v;
    vxb::warp_append(first, &c->cand_n);
  }
}

__device__ void clear_workspace(const Params& p);

// The cascade past its time budget (a cut near the root of a deep graph
// leaves millions of vertices affected, and the cascade walks them level by
// level).
// A vertex keeps its distance through the batch's deletions iff one of its
// shortest paths survives them, i.e. iff it has a surviving parent that is not
// affected itself: the affected vertices are exactly those whose distance in
// the graph without the deletions exceeds their old one.  One BFS of that graph
// (the deletions are committed, the insertions not yet) gives them: its
// distances replace the old ones, the count of raised vertices is the batch's
// affected count (and decides the fallback as the cascade's would), and the
// affected list stays empty, so the post-batch repair only relaxes the
// insertions.  The BFS distances go to tent (zero between phases), which the
// comparison pass zeroes again.
__device__ bool cascade_by_bfs(const Params& p, BlockQueue& bq, LbStage& lb) {
  BfsCounters* c = p.c;
  clear_workspace(p);
  reset_ring(p);
  if (!sync_grid(p)) return false;
  unsigned long long arcs = 0;
  uint32_t levels = 0;
  if (gtid() == 0) {  // the last full BFS's figures stand
    arcs = c->arcs;
    levels = c->levels;
    c->touched_n = 0;
    c->a_n = 0;
    c->a_bfs = 0;
  }
  full_bfs(p, bq, lb, p.tent, nullptr);  // also sets the reachable count of the graph without the deletions
  if (!sync_grid(p)) return false;
  uint32_t raised = 0;
  for (uint32_t v = gtid(); v < p.dist_len; v += nthreads()) {
    const uint32_t d0 = p.dist[v], d1 = p.tent[v];
    p.tent[v] = 0u;
    raised += d0 != kUnreachable && d1 > d0;
    p.dist[v] = d1;
  }
  raised = vxb::warp_sum(raised);
  if ((threadIdx.x & 31) == 0 && raised) atomicAdd(&c->a_bfs, raised);
  if (!sync_grid(p)) return false;
  if (gtid() == 0) {
    const uint32_t na = c->a_bfs;
    c->affected = na;
    if (na > p.fallback_limit) c->fallback = 1;  // bfs.hpp:249, 258: more than the limit falls back
    c->arcs = arcs;
    c->levels = levels;
    c->cbig = 0u;
    c->a_bfs = 0u;
    c->handovers[0] += 1;
  }
  return true;
}

// The cascade after the candidates are registered (and the batch's deletions
// committed): every candidate is checked in place, one warp each; the ring
// is drained only when a check left work in it (an affected vertex to expand,
// chunks of a long in-row), which most small batches never do.  Records the
// batch's affected count.
__device__ bool cascade(const Params& p, RepairSmem& sm, LbStage& lb, BlockQueue& bq, uint32_t ncand) {
  if (gtid() == 0) set_deadline(p);
  for (uint32_t i = gwarp(); i < ncand; i += nwarps()) check_vertex(p, p.lst_t[i]);
  if (!sync_grid(p)) return false;
  if (ld_cg(p.rq_tail)) {
    Cascade w{&p, &lb};
    drain(p, sm, w, p.cascade_bfs ? __ldcg(&p.c->deadline) : kNever);
    if (!sync_grid(p)) return false;
  }
  if (gtid() == 0) {  // the drain statistics of the phase trace
    p.c->rtrace[7] = ld_cg(p.rq_tail);
    for (int k = 0; k < 6; ++k) p.c->rtrace[9 + k] = __ldcg(&p.rq_stat[k]);
  }
  if (ld_cg(&p.c->cbig)) return cascade_by_bfs(p, bq, lb);
  if (gtid() == 0) p.c->affected = ld_cg(&p.c->a_n);
  return true;
}

__device__ void repair_pre(const Params& p, RepairSmem& sm, LbStage& lb, BlockQueue& bq) {
  BfsCounters* c = p.c;
  stamp(p, 0);
  reset_ring(p);
  if (!sync_grid(p)) return;
  register_candidates(p);
  if (!sync_grid(p)) return;
  stamp(p, 1);
  const uint32_t ncand = ld_cg(&c->cand_n);
  if (gtid() == 0) c->candidates = ncand;
  if (ncand == 0) return;
  if (!cascade(p, sm, lb, bq, ncand)) return;
  stamp(p, 2);
  reset_ring(p);  // for the post-batch kernel
}

// -------------------------------------------------- post-batch repair --

__device__ void clear_workspace(const Params& p) {
  const uint32_t nt = ld_cg(&p.c->touched_n), na = ld_cg(&p.c->a_n);
  for (uint32_t i = gtid(); i < nt; i += nthreads()) {
    p.sw[p.lst_t[i]] = 0ull;
    p.tent[p.lst_t[i]] = 0u;  // chunk counts left by a pass the fallback dropped
  }
  for (uint32_t i = gtid(); i < na; i += nthreads()) p.aff[p.lst_a[i] >> 5] = 0u;
}

// Lower dist[x] to cand; true when this thread lowered it (INF -> finite
// counted in reach).
__device__ __forceinline__ bool lower(const Params& p, uint32_t x, uint32_t cand, long long& reach) {
  if (cand >= ld_cg(&p.dist[x])) return false;
  const uint32_t old = atomicMin(&p.dist[x], cand);
  if (old <= cand) return false;
  if (old == kUnreachable) ++reach;
  return true;
}

// Queue x unless it is queued already (inq bit; cleared when claimed).
__device__ __forceinline__ void lower_and_push(const Params& p, bool lowered, uint32_t x) {
  bool push = false;
  if (lowered) {
    const uint32_t bit = 1u << (x & 31);
    push = !(atomicOr(&p.inq[0][x >> 5], bit) & bit);
  }
  ring_push(p, push, x);
}

// Per-lane form of a queued push (any lane, no warp aggregation).
__device__ __forceinline__ void push_one(const Params& p, uint32_t x) {
  const uint32_t bit = 1u << (x & 31);
  if (atomicOr(&p.inq[0][x >> 5], bit) & bit) return;
  const uint32_t s = atomicAdd(p.rq_tail, 1u);
  __stcg(&p.ring[s & p.ring_mask], (unsigned long long)x);
}

constexpr uint32_t kInlineRelax = 8;  // rows this short are relaxed where they are lowered

// A seed v just lowered: a short row is relaxed here by its lane (the
// vertices it lowers are queued), a longer one is queued.  Any later lowering
// of v queues v again, so relaxing from the current label loses nothing.
__device__ void seed_relax(const Params& p, bool lowered, uint32_t v, long long& reach) {
  bool queue = false;
  if (lowered) {
    const DevAdj& a = p.g.out;
    uint64_t b, e;
    vxb::base_range(a, v, b, e);
    const uint2 dr = a.drow[v];
    const uint32_t deg = (uint32_t)(e - b) + dr.y;
    if (deg > kInlineRelax) {
      queue = true;
    } else {
      acct_add(p, 0, deg);
      const uint32_t dv = ld_cg(&p.dist[v]);
      for (uint32_t k = 0; k < deg; ++k) {
        uint32_t x;
        if (k < e - b) {
          x = a.col[b + k];
          if (x & kTomb) continue;
        } else {
          x = a.darena[dr.x + (k - (uint32_t)(e - b))];
        }
        if (x < p.dist_len && lower(p, x, dv + 1, reach)) push_one(p, x);
      }
    }
  }
  lower_and_push(p, queue, v);
}

// Label-correcting relaxation (the settle of repair_affected, bfs.hpp:272-310,
// and propagate_decreases, :341-354, as one phase): every label is an upper
// bound of the post-batch distance, and relaxing from every changed label
// until nothing lowers gives the exact distances in any order.
struct Relax {
  const Params* p;
  LbStage* lb;
  long long* reach;
  __device__ void process(RepairSmem& sm, uint32_t n) {
    const Params& P = *p;
    const uint32_t t = threadIdx.x;
    // past its deadline the relaxation drops the rest of its queue: the
    // batch's distances then come from a full BFS of the post-batch graph
    // (the same distances)
    if (t == 0 && sm.late && !sm.flagged) {
      atomicOr(&P.c->rbig, 1u);
      sm.flagged = 1;
    }
    if (t < n) {
      const unsigned long long it = sm.items[t];
      uint32_t du = kUnreachable;
      if (it != kSent) {
        const uint32_t u = item_vertex(it);
        if (item_chunk(it) == 0) atomicAnd(&P.inq[0][u >> 5], ~(1u << (u & 31)));
        if (sm.late) sm.items[t] = kSent;  // dropped
        else du = ld_cg(&P.dist[u]);
      }
      sm.d[t] = du;
    }
    __syncthreads();
    auto relax = [&](bool valid, uint32_t x, uint32_t j) {
      const uint32_t du = sm.d[j];
      const bool lowered = valid && du != kUnreachable && x < P.dist_len && lower(P, x, du + 1, *reach);
      lower_and_push(P, lowered, x);
    };
    block_rows(P.g.out, sm.items, n, *lb, relax, &P, P.acct);
  }
};

// Boundary distances (best_boundary_distance, bfs.hpp:261-269) of the
// affected vertices, a block-sized chunk of them at a time: min of dist + 1
// over non-affected in-neighbours, folded per vertex in shared memory; each
// finite one seeds the relaxation.
constexpr uint32_t kBigBoundary = 4096;  // in-rows this long go to the grid-wide pass

__device__ void boundary_seeds(const Params& p, RepairSmem& sm, LbStage& lb, uint32_t na, long long& reach) {
  const uint32_t per = min((uint32_t)kThreads, max(1u, (na + gridDim.x - 1) / gridDim.x));
  for (uint32_t i0 = blockIdx.x * per; i0 < na; i0 += gridDim.x * per) {
    const uint32_t k = min(per, na - i0);
    if (threadIdx.x < k) {
      uint32_t v = p.lst_a[i0 + threadIdx.x];
      if (degree_of(p.g.in, v) > kBigBoundary) {  // a hub: the whole grid scans it after the barrier
        p.tent[i0 + threadIdx.x] = kUnreachable;
        p.big[atomicAdd(&p.c->big_b, 1u)] = i0 + threadIdx.x;
        v = 0xFFFFFFFFu;  // no row in this pass
      }
      sm.sv[threadIdx.x] = v;
      sm.cnt[threadIdx.x] = kUnreachable;
    }
    __syncthreads();
    auto bmin = [&](bool valid, uint32_t x, uint32_t j) {
      if (!valid || x >= p.dist_len || test_bit(p.aff, x)) return;
      const uint32_t dx = p.dist[x];
      if (dx != kUnreachable) atomicMin(&sm.cnt[j], dx + 1);
    };
    block_rows(p.g.in, sm.sv, k, lb, bmin, nullptr, p.acct);
    bool seed = false;
    uint32_t v = 0;
    if (threadIdx.x < k && sm.sv[threadIdx.x] != 0xFFFFFFFFu) {
      v = sm.sv[threadIdx.x];
      const uint32_t best = sm.cnt[threadIdx.x];
      // by atomicMin: an inserted arc may lower v first
      if (best != kUnreachable) seed = lower(p, v, best, reach);
    }
    seed_relax(p, seed, v, reach);
    __syncthreads();
  }
}

// Boundary distances of the hub entries p.big[0, nb) (indices into lst_a):
// each hub gets its own group of nwarps / nb warps (at least one), which fold
// 32-arc slices of its row into p.tent[i] by atomicMin, so many hubs are
// scanned side by side; the rows' seeds are taken after a barrier.
__device__ void grid_boundary_min(const Params& p, uint32_t nb) {
  const DevAdj& a = p.g.in;
  const int lane = threadIdx.x & 31;
  const uint32_t W = nwarps(), w = gwarp();
  const uint32_t G = max(1u, W / nb), R = W / G;  // warps per hub, hubs per round
  if (w >= R * G) return;
  for (uint32_t r = w / G; r < nb; r += R) {
    const uint32_t i = p.big[r];
    const uint32_t v = p.lst_a[i];
    uint32_t best = kUnreachable;
    uint64_t b, e;
    vxb::base_range(a, v, b, e);
    const uint2 dr = a.drow[v];
    const uint64_t nbase = e - b, total = nbase + dr.y;
    if (w % G == 0 && lane == 0) acct_add(p, 0, total);
    for (uint64_t k = (uint64_t)(w % G) * 32 + lane; k < total; k += (uint64_t)G * 32) {
      uint32_t x;
      if (k < nbase) {
        x = a.col[b + k];
        if (x & kTomb) continue;
      } else {
        x = a.darena[dr.x + (uint32_t)(k - nbase)];
      }
      if (x >= p.dist_len || test_bit(p.aff, x)) continue;
      const uint32_t dx = p.dist[x];
      if (dx != kUnreachable && dx + 1 < best) best = dx + 1;
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) best = min(best, __shfl_xor_sync(FULL, best, o));
    if (lane == 0 && best != kUnreachable) atomicMin(&p.tent[i], best);
  }
}

// The post-batch repair proper (everything but the fallback); true when the
// batch's distances are to come from a full BFS of the post-batch graph
// instead (the relaxation passed its budget), with the workspace cleared.
__device__ bool repair_relax(const Params& p, RepairSmem& sm, LbStage& lb) {
  BfsCounters* c = p.c;
  const int lane = threadIdx.x & 31;
  // the ring counters are zero here: the pre-batch kernel (or the previous
  // batch) left them so, and the first push comes after a barrier of this
  // kernel or a kernel boundary
  stamp(p, 3);
  if (gtid() == 0) set_deadline(p);
  const uint32_t na = ld_cg(&c->a_n);
  if (gtid() == 0) acct_add(p, 1, na);  // invalidated and re-seeded
  long long reach = 0;
  if (na > 0) {
    // invalidate the affected vertices (repair_affected, bfs.hpp:272-283)
    for (uint32_t i = gtid(); i < na; i += nthreads()) p.dist[p.lst_a[i]] = kUnreachable;
    if (gtid() == 0) {
      reach_add(p, -(long long)na);
      c->big_b = 0;
    }
    if (!sync_grid(p)) return false;
    stamp(p, 4);
    boundary_seeds(p, sm, lb, na, reach);
  }
  // inserted arcs relax their heads (bfs.hpp:91-96)
  const uint32_t F = *p.F;
  for (uint32_t base = gwarp() * 32; base < F; base += nwarps() * 32) {
    const uint32_t i = base + lane;
    bool lowered = false;
    uint32_t v = 0;
    if (i < F && (p.ff[i] & kFAdd)) {
      const uint32_t u = p.fu[i];
      v = p.fv[i];
      if (u < p.dist_len && v < p.dist_len) {
        const uint32_t du = ld_cg(&p.dist[u]);
        if (du != kUnreachable) lowered = lower(p, v, du + 1, reach);
      }
    }
    seed_relax(p, lowered, v, reach);
  }
  if (!sync_grid(p)) return false;
  const uint32_t nbig = na ? ld_cg(&c->big_b) : 0u;
  if (nbig) {
    grid_boundary_min(p, nbig);
    if (!sync_grid(p)) return false;
    for (uint32_t base = gwarp() * 32; base < nbig; base += nwarps() * 32) {
      const uint32_t r = base + lane;
      bool seed = false;
      uint32_t v = 0;
      if (r < nbig) {
        const uint32_t i = p.big[r];
        v = p.lst_a[i];
        const uint32_t best = ld_cg(&p.tent[i]);
        p.tent[i] = 0u;  // tent is all-zero between phases (the cascade's chunk counts)
        if (best != kUnreachable) seed = lower(p, v, best, reach);
      }
      seed_relax(p, seed, v, reach);
    }
    if (!sync_grid(p)) return false;
  }
  stamp(p, 5);
  if (ld_cg(p.rq_tail)) {  // the relaxation runs only when a seed left work queued
    Relax w{&p, &lb, &reach};
    drain(p, sm, w, __ldcg(&p.c->deadline));
    if (!sync_grid(p)) return false;
    if (ld_cg(&c->rbig)) {
      // the relaxation passed its budget: a full BFS of the post-batch graph
      // gives the distances and the reachable count (the repair's counters
      // -- candidates, affected, no full recompute -- stand)
      clear_workspace(p);
      reset_ring(p);
      return true;
    }
  }
  stamp(p, 6);
  if (gtid() == 0) {
    c->rtrace[8] = ld_cg(p.rq_tail);
    for (int k = 0; k < 6; ++k) c->rtrace[15 + k] = __ldcg(&p.rq_stat[k]);
  }
  reach = vxb::warp_sum(reach);
  if (lane == 0) reach_add(p, reach);
  clear_workspace(p);
  reset_ring(p);
  return false;
}

// Post-batch repair (bfs.hpp:72-97): the fallback's full BFS or the repair,
// which may itself hand over to a full BFS; one call site serves both.
__device__ void repair_post(const Params& p, RepairSmem& sm, LbStage& lb, BlockQueue& bq) {
  BfsCounters* c = p.c;
  const bool fallback = ld_cg(&c->fallback) != 0u;
  if (fallback) clear_workspace(p);
  else if (!repair_relax(p, sm, lb)) return;
  if (!sync_grid(p)) return;
  full_bfs(p, bq, lb, p.dist, p.trace);
  if (gtid() == 0) {
    if (fallback) {
      c->full = 1;
    } else {
      c->rbig = 0u;
      c->handovers[1] += 1;
    }
  }
}

// ------------------------------------------------------- batched stream --
//
// A whole update stream applied in one persistent launch: the batches' canonical
// arcs come sorted by (batch, u, v) from one stream-wide sort, and every batch
// runs classify + tombstones, delta removals + deletion candidates, the
// cascade, tombstone revivals + delta insertions, and the post-batch repair,
// separated by grid barriers, with no launch or host synchronisation between
// batches.  The result after every batch is the one IncrementalBFS::apply
// gives (bfs.hpp:29-98); an optional per-batch digest of the distances and
// per-batch counters make every batch checkable.

struct StreamArgs {
  const uint32_t* fu;        // canonical arcs of the stream, batch-major
  const uint32_t* fv;
  uint8_t* ff;               // in: desired state (bit 0); out: classification flags
  uint64_t* fpos;
  const uint32_t* boff;      // nb + 1 offsets of the batches' arcs
  const uint32_t* bcnt;      // nb arc counts
  const uint32_t* vpost;     // vertex count after each batch
  uint32_t* scratch;         // one batch's arcs: the insertions of each row run
  unsigned long long* digest;  // nb digests of the distances (optional)
  uint32_t* bstats;          // nb x 4: candidates, affected, full recompute, reachable (optional)
  GraphCounters* gc;
  unsigned long long arena_cap;
  double frac;
  uint32_t nb, V0, len0;
  uint32_t v_single;    // vertex count after the batch when vpost is null (one staged batch)
  uint32_t classified;  // the arcs carry their classification already (a staged batch)
};

// Order-independent 64-bit digest of dist[0, n): sum of splitmix64(v << 32 | dist[v]).
using vxb::mix64;

__device__ void digest_pass(const uint32_t* dist, uint32_t n, unsigned long long* out) {
  unsigned long long h = 0;
  for (uint32_t v = gtid(); v < n; v += nthreads()) h += mix64(((unsigned long long)v << 32) | ld_cg(&dist[v]));
  h = vxb::warp_sum(h);
  if ((threadIdx.x & 31) == 0 && h) atomicAdd(out, h);
}

// End of the row run of canonical arcs starting at s (same u), whole warp.
__device__ __forceinline__ uint32_t run_end(const uint32_t* fu, uint32_t s, uint32_t F) {
  const int lane = threadIdx.x & 31;
  const uint32_t u = fu[s];
  for (uint32_t k = s + 1;; k += 32) {
    const uint32_t i = k + lane;
    const uint32_t m = __ballot_sync(FULL, i >= F || fu[i] != u);
    if (m) return k + (uint32_t)(__ffs(m) - 1);
  }
}

__device__ __forceinline__ bool delta_op(uint8_t f, bool insertion) {
  return !(f & kFInBase) && (f & kFChanged) && (((f & kFAdd) != 0) == insertion);
}

// Delta removals of one row run (whole warp): the row's sorted delta list
// keeps every entry that is not a removal of the run (delta_remove_kernel of
// the per-batch path, on the canonical arcs directly).
__device__ void run_remove(const vxb::DevAdj& a, const uint32_t* fv, const uint8_t* ff, uint32_t s, uint32_t e, uint32_t u,
                           GraphCounters* gc, unsigned long long* acct) {
  const int lane = threadIdx.x & 31;
  bool any = false;
  for (uint32_t k = s + lane; k < e; k += 32) any |= delta_op(ff[k], false);
  if (!__any_sync(FULL, any)) return;
  const uint2 row = a.drow[u];
  uint32_t* A = a.darena + row.x;
  uint32_t written = 0;
  for (uint32_t base = 0; base < row.y; base += 32) {
    const uint32_t j = base + lane;
    const bool in = j < row.y;
    const uint32_t x = in ? A[j] : 0u;
    bool keep = in;
    if (in) {
      const uint32_t q = vxb::lower_bound_u32(fv, s, e, x);
      if (q < e && fv[q] == x && delta_op(ff[q], false)) keep = false;
    }
    const uint32_t mask = __ballot_sync(FULL, keep);
    const uint32_t p = written + __popc(mask & vxb::lanemask_lt());
    __syncwarp();
    if (keep) A[p] = x;
    written += __popc(mask);
    __syncwarp();
  }
  if (lane == 0) {
    a.drow[u].y = written;
    if (acct) atomicAdd(acct, (unsigned long long)(row.y + written));
    atomicAdd(&gc->delta_live[0], (unsigned long long)(-(long long)(row.y - written)));
    gdev::mark_dirty(a.dirty, u, &gc->dirty_rows[0]);
  }
}

// Delta insertions of one row run (whole warp): the run's insertions are
// compacted into scratch[s, s + nB) and merged into the row's delta list, in
// place when its block has room, else into a new power-of-two arena block
// (delta_insert_kernel of the per-batch path).
__device__ void run_insert(const vxb::DevAdj& a, const uint32_t* fv, const uint8_t* ff, uint32_t* scratch, uint32_t s,
                           uint32_t e, uint32_t u, GraphCounters* gc, unsigned long long arena_cap,
                           unsigned long long* acct) {
  const int lane = threadIdx.x & 31;
  uint32_t nB = 0;
  for (uint32_t base = s; base < e; base += 32) {
    const uint32_t k = base + lane;
    const bool ins = k < e && delta_op(ff[k], true);
    const uint32_t m = __ballot_sync(FULL, ins);
    if (ins) scratch[s + nB + __popc(m & vxb::lanemask_lt())] = fv[k];
    nB += __popc(m);
  }
  if (nB == 0) return;
  __syncwarp();
  const uint2 row = a.drow[u];
  const uint32_t cap = a.dcap[u];
  const uint32_t cnew = row.y + nB;
  if (cnew <= cap) {
    gdev::warp_merge_inplace(a.darena + row.x, row.y, scratch + s, nB);
    if (lane == 0) a.drow[u].y = cnew;
  } else {
    uint32_t ncap = 8;
    while (ncap < cnew) ncap <<= 1;
    unsigned long long off = 0;
    if (lane == 0) off = atomicAdd(&gc->arena_top[0], (unsigned long long)ncap);
    off = __shfl_sync(FULL, off, 0);
    if (off + ncap > arena_cap) {
      if (lane == 0) atomicOr(&gc->err, vxb::kErrArenaOverflow);
      return;
    }
    gdev::warp_merge_to(a.darena + off, a.darena + row.x, row.y, scratch + s, nB);
    if (lane == 0) {
      a.drow[u] = make_uint2((uint32_t)off, cnew);
      a.dcap[u] = ncap;
    }
  }
  if (lane == 0) {
    atomicAdd(&gc->delta_live[0], (unsigned long long)nB);
    if (acct) atomicAdd(acct, (unsigned long long)(row.y + cnew));
    gdev::mark_dirty(a.dirty, u, &gc->dirty_rows[0]);
  }
}

// The row runs of the batch's canonical arcs [0, F): delta removals
// (kInsert false) or insertions (true).  A run of one arc whose delta row
// holds at most 7 arcs (8 for a removal) -- most runs of a batch -- is done by
// one lane: the row's block (capacity >= 8, 8-aligned in the arena) is loaded
// as two 16-byte words, edited in registers and stored back; a row without a
// block gets 8 slots from one warp-aggregated arena allocation.  The other
// runs are queued in shared memory and done by the block's warps (run_insert,
// run_remove).  Arcs are dealt round-robin (arc i to block i mod gridDim), so
// a small batch still spreads over every block.  Block-uniform.
template <bool kInsert>
__device__ void commit_runs(const Params& p, const StreamArgs& s, uint32_t off, uint32_t F, RepairSmem& sm) {
  const vxb::DevAdj& a = p.g.out;
  const uint32_t* fu = s.fu + off;
  const uint32_t* fv = s.fv + off;
  const uint8_t* ff = s.ff + off;
  const int lane = threadIdx.x & 31;
  const uint32_t per_round = gridDim.x * kThreads;
  for (uint32_t r0 = 0; r0 < F; r0 += per_round) {
    if (threadIdx.x == 0) sm.nsv = 0;
    __syncthreads();
    const uint32_t i = r0 + threadIdx.x * gridDim.x + blockIdx.x;
    bool job = false, queue = false, need_block = false;
    uint32_t u = 0, v = 0;
    uint2 row = make_uint2(0, 0);
    if (i < F) {
      u = fu[i];
      if (i == 0 || fu[i - 1] != u) {
        if (i + 1 < F && fu[i + 1] == u) {
          queue = true;  // a run of several arcs
        } else if (delta_op(ff[i], kInsert)) {
          v = fv[i];
          row = a.drow[u];
          if (kInsert ? row.y < 8u : row.y <= 8u) {
            job = true;
            need_block = kInsert && a.dcap[u] == 0u;  // no block yet (then the row is empty)
          } else {
            queue = true;
          }
        }
      }
    }
    const uint32_t nm = __ballot_sync(FULL, need_block);
    uint32_t base_off = row.x;
    if (nm) {
      const int leader = __ffs(nm) - 1;
      unsigned long long b0 = 0;
      if (lane == leader) b0 = atomicAdd(&s.gc->arena_top[0], 8ull * (unsigned long long)__popc(nm));
      b0 = __shfl_sync(FULL, b0, leader);
      const unsigned long long o = b0 + 8ull * __popc(nm & vxb::lanemask_lt());
      if (need_block) {
        if (o + 8 > s.arena_cap) {
          atomicOr(&s.gc->err, vxb::kErrArenaOverflow);
          job = false;
        } else {
          base_off = (uint32_t)o;
        }
      }
    }
    long long dlive = 0;
    unsigned long long dirtied = 0;
    if (job) {
      uint32_t x[8] = {0, 0, 0, 0, 0, 0, 0, 0};
      if (row.y) {
        const uint4* src = reinterpret_cast<const uint4*>(a.darena + row.x);
        const uint4 q0 = src[0], q1 = src[1];
        x[0] = q0.x, x[1] = q0.y, x[2] = q0.z, x[3] = q0.w;
        x[4] = q1.x, x[5] = q1.y, x[6] = q1.z, x[7] = q1.w;
      }
      // output k: an insertion takes x[k] below the new arc's position, the arc
      // at it and x[k - 1] above; a removal takes x[k] below the arc, x[k + 1] from it on
      uint32_t pos = 0;
#pragma unroll
      for (int k = 0; k < 8; ++k) pos += ((uint32_t)k < row.y && x[k] < v) ? 1u : 0u;
      auto out = [&](int k) -> uint32_t {
        if (kInsert) return (uint32_t)k < pos ? x[k] : ((uint32_t)k == pos ? v : x[k > 0 ? k - 1 : 0]);
        return (uint32_t)k < pos ? x[k] : x[k < 7 ? k + 1 : 7];
      };
      uint4* dst = reinterpret_cast<uint4*>(a.darena + base_off);
      dst[0] = make_uint4(out(0), out(1), out(2), out(3));
      dst[1] = make_uint4(out(4), out(5), out(6), out(7));
      dlive = kInsert ? 1 : -1;
      acct_add(p, 2, kInsert ? 2ull * row.y + 1 : 2ull * row.y - 1);
      a.drow[u] = make_uint2(base_off, kInsert ? row.y + 1 : row.y - 1);
      if (need_block) a.dcap[u] = 8u;
      const uint32_t bit = 1u << (u & 31);
      dirtied = (atomicOr(&a.dirty[u >> 5], bit) & bit) ? 0ull : 1ull;
    }
    dlive = vxb::warp_sum(dlive);
    dirtied = vxb::warp_sum(dirtied);
    if (lane == 0 && dlive) atomicAdd(&s.gc->delta_live[0], (unsigned long long)dlive);
    if (lane == 0 && dirtied) atomicAdd(&s.gc->dirty_rows[0], dirtied);
    if (queue) sm.sv[atomicAdd(&sm.nsv, 1u)] = i;
    __syncthreads();
    const uint32_t nq = sm.nsv;
    for (uint32_t k = threadIdx.x >> 5; k < nq; k += kThreads / 32) {
      const uint32_t st = sm.sv[k], en = run_end(fu, st, F);
      unsigned long long* ac = p.acct ? p.acct + 2 : nullptr;
      if (kInsert) run_insert(a, fv, ff, s.scratch, st, en, fu[st], s.gc, s.arena_cap, ac);
      else run_remove(a, fv, ff, st, en, fu[st], s.gc, ac);
    }
    __syncthreads();  // the list is rebuilt by the next round
  }
}

__device__ void stream_kernel_body(Params p, const StreamArgs& s, RepairSmem& sm, LbStage& lb, BlockQueue& bq) {
  BfsCounters* c = p.c;
  const int lane = threadIdx.x & 31;
  unsigned long long tmark = globaltimer();
  auto phase = [&](int k) {  // gtid 0 accumulates the time since the previous mark
    if (gtid() == 0) {
      const unsigned long long now = globaltimer();
      c->stream_ns[k] += now - tmark;
      tmark = now;
    }
  };
  if (gtid() == 0) {  // stamps and drain statistics are written by this thread only
    for (int k = 0; k < 6; ++k) c->stream_ns[k] = 0;
    for (int k = 0; k < (int)(sizeof(c->rtrace) / sizeof(c->rtrace[0])); ++k) c->rtrace[k] = 0;
    c->handovers[0] = c->handovers[1] = 0;
  }
  for (uint32_t bi = 0; bi < s.nb; ++bi) {
    const uint32_t off = s.boff ? s.boff[bi] : 0u, F = s.bcnt[bi];
    const uint32_t Vpre = bi ? s.vpost[bi - 1] : s.V0, lpre = bi ? s.vpost[bi - 1] : s.len0;
    const uint32_t Vpost = s.vpost ? s.vpost[bi] : s.v_single;
    Params q = p;
    q.fu = s.fu + off;
    q.fv = s.fv + off;
    q.ff = s.ff + off;
    q.F = &s.bcnt[bi];
    q.V = Vpre;
    q.dist_len = lpre;
    const unsigned long long lim = (unsigned long long)((double)Vpre * s.frac);
    q.fallback_limit = lim < 1 ? 1 : lim;
    if (gtid() == 0) {  // last_* counters and the repair lists start empty (bfs.hpp:30-33)
      c->candidates = c->affected = c->full = c->fallback = 0;
      c->cand_n = c->touched_n = c->a_n = 0;
    }
    stamp(q, 0);
    // A: classification against the pre-batch graph; tombstone the deleted base arcs
    {
      // arcs dealt round-robin over the blocks (arc i to block i mod gridDim),
      // so a small batch's searches spread over every SM
      const vxb::DevAdj& a = p.g.out;
      long long tombs = 0;
      uint32_t dirtied = 0, removals = 0;
      for (uint32_t i = threadIdx.x * gridDim.x + blockIdx.x; i < F; i += nthreads()) {
        uint8_t f = s.ff[off + i];
        if (!s.classified) {
          f = gdev::classify_arc(a, s.fu[off + i], s.fv[off + i], f, s.fpos[off + i]);
          s.ff[off + i] = f;
        }
        removals += !(f & kFAdd) && (f & kFChanged);
        tombs += gdev::tomb_arc(a, s.fu[off + i], f, s.fpos[off + i], 0, dirtied);
      }
      tombs = vxb::warp_sum(tombs);
      dirtied = vxb::warp_sum(dirtied);
      removals = vxb::warp_sum(removals);
      if (lane == 0 && tombs) atomicAdd(&s.gc->tombs[0], (unsigned long long)tombs);
      if (lane == 0 && dirtied) atomicAdd(&s.gc->dirty_rows[0], (unsigned long long)dirtied);
      if (lane == 0 && removals) atomicAdd(&c->rmb[bi & 1], removals);
      if (s.digest && bi > 0) digest_pass(p.dist, lpre, &s.digest[bi - 1]);
    }
    if (!sync_grid(p)) return;
    phase(0);
    // B: delta removals; deletion candidates registered.  A batch without a
    // removal arc has neither, and skips the phase and its barrier.  The other
    // parity's counter was last read before the previous batch's later
    // barriers: it is cleared here for the next batch.
    const uint32_t nrm = ld_cg(&c->rmb[bi & 1]);
    if (gtid() == 0) c->rmb[(bi + 1) & 1] = 0u;
    if (nrm) {
      commit_runs<false>(q, s, off, F, sm);
      register_candidates(q);
      if (!sync_grid(p)) return;
    }
    phase(1);
    stamp(q, 1);
    // C: the cascade over the graph without the batch's deletions
    const uint32_t ncand = ld_cg(&c->cand_n);
    if (gtid() == 0) {
      c->candidates = ncand;
      acct_add(p, 1, ncand + F);  // candidate checks, heads of the canonical arcs
      acct_add(p, 3, F);
      acct_add(p, 4, 1);
    }
    if (ncand) {
      q.cascade_bfs = lpre == Vpre;
      if (!cascade(q, sm, lb, bq, ncand)) return;
      reset_ring(q);
    }
    phase(2);
    stamp(q, 2);
    // D: revive re-added base arcs, delta insertions; new vertices start unreachable
    {
      const vxb::DevAdj& a = p.g.out;
      long long tombs = 0;
      uint32_t dirtied = 0;
      for (uint32_t i = threadIdx.x * gridDim.x + blockIdx.x; i < F; i += nthreads())
        tombs += gdev::tomb_arc(a, s.fu[off + i], s.ff[off + i], s.fpos[off + i], 1, dirtied);
      tombs = vxb::warp_sum(tombs);
      dirtied = vxb::warp_sum(dirtied);
      if (lane == 0 && tombs) atomicAdd(&s.gc->tombs[0], (unsigned long long)tombs);
      if (lane == 0 && dirtied) atomicAdd(&s.gc->dirty_rows[0], (unsigned long long)dirtied);
      for (uint32_t v = lpre + gtid(); v < Vpost; v += nthreads()) p.dist[v] = kUnreachable;
    }
    commit_runs<true>(q, s, off, F, sm);
    if (!sync_grid(p)) return;
    phase(3);
    // E: the post-batch repair (or the fallback full BFS) on the new graph
    q.V = Vpost;
    q.dist_len = Vpost;
    repair_post(q, sm, lb, bq);
    if (ld_cg(&c->err)) return;
    phase(4);
    // every block's counter updates are in before they are recorded, and
    // recorded before the next batch resets them (same thread)
    if (!sync_grid(p)) return;
    phase(5);
    if (gtid() == 0 && s.bstats) {
      s.bstats[4 * bi + 0] = ld_cg(&c->candidates);
      s.bstats[4 * bi + 1] = ld_cg(&c->affected);
      s.bstats[4 * bi + 2] = ld_cg(&c->full);
      s.bstats[4 * bi + 3] = (uint32_t)__ldcg(&c->reachable);
    }
  }
  if (s.digest && s.nb) digest_pass(p.dist, s.vpost[s.nb - 1], &s.digest[s.nb - 1]);
  // every read of the removal counters came before the last end-of-batch barrier
  if (gtid() == 0) c->rmb[0] = c->rmb[1] = 0u;
}

// The full BFS has a kernel of its own, so that its registers are allocated
// apart from the repair phases' (the repair kernel runs it too, for the
// fallback and the budget handovers).
__global__ void __launch_bounds__(kThreads, 3) bfs_full_kernel(Params p) {
  __shared__ BlockQueue bq;
  __shared__ LbStage lb;
  full_bfs(p, bq, lb, p.dist, p.trace);
}

__global__ void __launch_bounds__(kThreads, 3) bfs_kernel(Params p, int mode) {
  __shared__ BlockQueue bq;
  __shared__ LbStage lb;
  __shared__ RepairSmem sm;
  if (mode == kModePre) repair_pre(p, sm, lb, bq);
  else repair_post(p, sm, lb, bq);
}

__global__ void __launch_bounds__(kThreads, 2) bfs_stream_kernel(Params p, StreamArgs s) {
  __shared__ BlockQueue bq;
  __shared__ LbStage lb;
  __shared__ RepairSmem sm;
  stream_kernel_body(p, s, sm, lb, bq);
}

// Stream canonicalisation: both arcs of every non-self-loop op keyed by
// (batch, u, v) with the op's stream index as the value; a stable sort then
// leaves each batch's ops for one arc in order, and the last one wins.
__global__ void stream_keys_kernel(const uint32_t* src, const uint32_t* dst, const uint8_t* add,
                                   const uint64_t* boff, uint32_t nb, size_t n, int b, uint64_t* keys,
                                   uint32_t* vals) {
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
    uint32_t lo = 0, hi = nb;  // the batch t with boff[t] <= i < boff[t + 1]
    while (hi - lo > 1) {
      const uint32_t mid = (lo + hi) >> 1;
      if (boff[mid] <= i) lo = mid;
      else hi = mid;
    }
    const uint64_t t = (uint64_t)lo << (2 * b);
    const uint32_t u = src[i], v = dst[i];
    const uint32_t val = ((uint32_t)i << 1) | (add[i] ? 1u : 0u);
    const bool ok = u != v;
    keys[2 * i] = ok ? (t | ((uint64_t)u << b) | v) : ~0ull;
    keys[2 * i + 1] = ok ? (t | ((uint64_t)v << b) | u) : ~0ull;
    vals[2 * i] = val;
    vals[2 * i + 1] = val;
  }
}

__global__ void stream_last_kernel(const uint64_t* keys, size_t m, uint32_t* flag) {
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < m; i += (size_t)gridDim.x * blockDim.x) {
    const uint64_t k = keys[i];
    flag[i] = (k != ~0ull) && (i + 1 == m || keys[i + 1] != k);
  }
}

__global__ void stream_compact_kernel(const uint64_t* keys, const uint32_t* vals, const uint32_t* flag,
                                      const uint32_t* pos, size_t m, int b, uint32_t* fu, uint32_t* fv, uint8_t* ff,
                                      uint32_t* bid) {
  const uint64_t mask = ((uint64_t)1 << b) - 1;
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < m; i += (size_t)gridDim.x * blockDim.x) {
    if (!flag[i]) continue;
    const uint32_t q = pos[i];
    const uint64_t k = keys[i];
    fu[q] = (uint32_t)((k >> b) & mask);
    fv[q] = (uint32_t)(k & mask);
    ff[q] = (uint8_t)(vals[i] & 1u);
    bid[q] = (uint32_t)(k >> (2 * b));
  }
}

// boff[t] = first canonical arc of batch t (t <= nb), bcnt[t] = its arc count.
__global__ void stream_bounds_kernel(const uint32_t* bid, const uint32_t* total, uint32_t nb, uint32_t* boff,
                                     uint32_t* bcnt) {
  const uint32_t F = *total;
  for (uint32_t t = blockIdx.x * blockDim.x + threadIdx.x; t <= nb; t += gridDim.x * blockDim.x) {
    uint32_t lo = 0, hi = F;
    while (lo < hi) {
      const uint32_t mid = (lo + hi) >> 1;
      if (bid[mid] < t) lo = mid + 1;
      else hi = mid;
    }
    boff[t] = lo;
    uint32_t lo2 = lo, hi2 = F;
    while (lo2 < hi2) {
      const uint32_t mid = (lo2 + hi2) >> 1;
      if (bid[mid] <= t) lo2 = mid + 1;
      else hi2 = mid;
    }
    if (t < nb) bcnt[t] = lo2 - lo;
  }
}

__global__ void digest_kernel(const uint32_t* dist, uint32_t n, unsigned long long* out) {
  unsigned long long h = 0;
  for (uint32_t v = blockIdx.x * blockDim.x + threadIdx.x; v < n; v += gridDim.x * blockDim.x)
    h += mix64(((unsigned long long)v << 32) | dist[v]);
  h = vxb::warp_sum(h);
  if ((threadIdx.x & 31) == 0 && h) atomicAdd(out, h);
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
  // fills and copies go on the graph's (non-blocking) stream, ahead of the
  // kernels that use the new buffers; the old buffers are freed once the
  // stream has finished copying out of them
  std::vector<uint32_t*> old;
  auto realloc_copy = [&](uint32_t** p, size_t n_new, size_t n_old, int fill) -> int {
    uint32_t* q = nullptr;
    if (cudaMalloc(&q, n_new * sizeof(uint32_t)) != cudaSuccess) {
      set_error("BFS allocation of %zu bytes failed", n_new * 4);
      return -4;
    }
    if (cudaMemsetAsync(q, fill, n_new * sizeof(uint32_t), s) != cudaSuccess) return -3;
    if (*p && n_old && cudaMemcpyAsync(q, *p, n_old * sizeof(uint32_t), cudaMemcpyDeviceToDevice, s) != cudaSuccess)
      return -3;
    if (*p) old.push_back(*p);
    *p = q;
    return 0;
  };
  const size_t oldw = b->cap ? (b->cap + 31) / 32 + 1 : 0;
  int rc = 0;
  rc |= realloc_copy(&b->dist, c, b->cap, 0xFF);
  rc |= realloc_copy(&b->sw, 2 * c, 0, 0);
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
  rc |= realloc_copy(&b->tent, c, 0, 0);
  rc |= realloc_copy(&b->bul, 2 * (c + kListSlack), 0, 0);
  const cudaError_t e = cudaStreamSynchronize(s);
  for (uint32_t* p : old) cudaFree(p);
  if (rc) return -4;
  VX_CUDA_TRY(e);
  b->cap = c;
  return 0;
}

// The work ring holds at most one pending item per vertex plus the extra
// chunks of long rows (one per kChunk arcs), so it is sized for capacity +
// arcs / kChunk, with the delta arena counted at its allocated size (so a
// reserved arena needs no growth mid-stream); made with the object and
// checked before every staged batch.
static int ensure_ring(Bfs* b) {
  const Adjacency& a = b->g->adj[0];
  // + the tickets blocks hold past the tail (kClaim each) and slack
  const size_t need = b->cap + (size_t)((a.A + std::max<uint64_t>(a.arena_bound, a.arena_cap)) / kChunk) +
                      (size_t)kThreads * 1024;
  size_t slots = 1;
  while (slots < need) slots <<= 1;
  if (slots <= b->ring_slots) return 0;
  VX_CUDA_TRY(cudaStreamSynchronize(b->g->stream));
  cudaFree(b->ring);
  b->ring = nullptr;
  b->ring_slots = 0;
  if (cudaMalloc(&b->ring, slots * sizeof(unsigned long long)) != cudaSuccess) {
    set_error("BFS work ring allocation of %zu bytes failed", slots * 8);
    return -4;
  }
  // on the graph's stream, so the first launch that drains the ring sees every
  // slot empty (the graph's stream is non-blocking: a legacy-stream memset
  // would not be ordered before it)
  VX_CUDA_TRY(cudaMemsetAsync(b->ring, 0xFF, slots * sizeof(unsigned long long), b->g->stream));
  b->ring_slots = slots;
  return 0;
}

static Params make_params(Bfs* b, uint32_t V, uint32_t dist_len) {
  Graph* g = b->g;
  Params p;
  memset(&p, 0, sizeof(p));
  p.g = g->view();
  p.V = V;
  // a full BFS reads every arc once; a relaxation that has processed this
  // many items is past the point where one would have been cheaper on a
  // deep graph
  p.handover = b->tune.handover;
  p.cascade_bfs = dist_len == V;
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
  p.tent = b->tent;
  p.bul = b->bul;
  p.bul_half = (uint32_t)(b->cap + kListSlack);
  p.sw = reinterpret_cast<unsigned long long*>(b->sw);
  p.ring = b->ring;
  p.ring_mask = b->ring_slots ? (uint32_t)(b->ring_slots - 1) : 0u;
  p.rq_head = b->rq;
  p.rq_tail = b->rq + 32;
  p.rq_done = b->rq + 64;
  p.rq_fin = b->rq + 128;
  p.rq_stat = reinterpret_cast<unsigned long long*>(b->rq + 96);
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
  p.acct = b->acct_on ? b->acct : nullptr;
  p.bar = b->barrier;
  return p;
}

// Every co-resident block of the kernel, once per object.
static int grid_of(const void* kernel, int* grid) {
  if (*grid) return 0;
  int per_sm = 0;
  VX_CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kernel, kThreads, 0));
  if (per_sm < 1) {
    set_error("BFS kernel cannot be resident on an SM");
    return -3;
  }
  *grid = per_sm * sm_count();
  return 0;
}

static int launch(Bfs* b, Params& p, int mode) {
  const bool full = mode == kModeFull;
  const void* kernel = full ? (const void*)bfs_full_kernel : (const void*)bfs_kernel;
  int* grid = full ? &b->full_grid : &b->grid;
  if (int rc = grid_of(kernel, grid)) return rc;
  p.nblocks = (uint32_t)*grid;
  void* args[] = {&p, &mode};  // the full-BFS kernel takes p alone
  vxh::count_launch();
  VX_CUDA_TRY(cudaLaunchCooperativeKernel(kernel, dim3(*grid), dim3(kThreads), args, 0, b->g->stream));
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
      cudaMalloc(&b->rq, 160 * sizeof(uint32_t)) != cudaSuccess ||
      cudaMallocHost(&b->hctr, sizeof(BfsCounters)) != cudaSuccess) {
    set_error("BFS counter allocation failed");
    bfs_destroy(b);
    return -4;
  }
  cudaMemsetAsync(b->ctr, 0, sizeof(BfsCounters), g->stream);
  cudaMemsetAsync(b->barrier, 0, vxb::kBarrierWords * sizeof(uint32_t), g->stream);
  cudaMemsetAsync(b->rq, 0, 160 * sizeof(uint32_t), g->stream);
  memset(b->hctr, 0, sizeof(BfsCounters));
  int rc = bfs_recompute(b);
  if (!rc) rc = ensure_ring(b);  // before the first batch, which would otherwise allocate it
  if (rc) {
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
                      b->lst_a, b->lst_t, b->tent, b->bul, b->sw, b->aff, b->inq[0], b->inq[1]};
  for (uint32_t* p : ptrs) cudaFree(p);
  cudaFree(b->ctr);
  cudaFree(b->acct);
  cudaFree(b->trace);
  cudaFree(b->barrier);
  cudaFree(b->features);
  cudaFree(b->rq);
  cudaFree(b->ring);
  b->sb.free_all();
  delete b->vb;
  cudaFreeHost(b->hctr);
  delete b;
}

int bfs_ensure_capacity(Bfs* b, size_t V) { return ensure_capacity(b, V); }

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

// The direction switch and the grid-expanded row length of the full BFS,
// picked by timing: every candidate (alpha, beta, large_row) of a small grid
// runs a full BFS from each of the given roots (CUDA events on the graph's
// stream, one untimed warm-up per candidate), the median over the roots
// decides, and the best candidate stays set on b.  The distances from b's
// own source are recomputed afterwards.
int bfs_autotune(Bfs* b, const uint32_t* roots, size_t k, float* chosen) {
  static const float kAlpha[] = {4.f, 14.f, 40.f, 120.f};
  static const float kBeta[] = {8.f, 24.f, 96.f};
  static const uint32_t kLarge[] = {512u, 1024u, 4096u};
  Graph* g = b->g;
  cudaStream_t s = g->stream;
  const uint32_t source = b->source;
  const BfsTuning keep = b->tune;
  cudaEvent_t e0, e1;
  VX_CUDA_TRY(cudaEventCreate(&e0));
  VX_CUDA_TRY(cudaEventCreate(&e1));
  float best = -1.f;
  BfsTuning pick = keep;
  std::vector<float> ts(k);
  int rc = 0;
  for (float al : kAlpha)
    for (float be : kBeta)
      for (uint32_t lr : kLarge) {
        b->tune.alpha = al;
        b->tune.beta = be;
        b->tune.large_row = lr;
        // each root timed twice, the faster run kept (a single run now and
        // then lands several percent slow); the candidate's score is the
        // mean over the roots
        for (size_t r = 0; r < k && !rc; ++r) {
          b->source = roots[r];
          if (r == 0) rc = bfs_recompute(b);  // warm-up of this candidate
          ts[r] = -1.f;
          for (int rep = 0; rep < 2 && !rc; ++rep) {
            float t = 0.f;
            if (cudaEventRecord(e0, s) != cudaSuccess) rc = -3;
            if (!rc) rc = bfs_recompute(b);
            if (!rc && cudaEventRecord(e1, s) != cudaSuccess) rc = -3;
            if (!rc && cudaEventSynchronize(e1) != cudaSuccess) rc = -3;
            if (!rc && cudaEventElapsedTime(&t, e0, e1) != cudaSuccess) rc = -3;
            if (!rc && (ts[r] < 0.f || t < ts[r])) ts[r] = t;
          }
        }
        if (rc) break;
        float mean = 0.f;
        for (float t : ts) mean += t;
        mean /= (float)k;
        if (best < 0.f || mean < best) {
          best = mean;
          pick = b->tune;
        }
      }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  b->source = source;
  b->tune = rc ? keep : pick;
  if (rc) {
    set_error("autotune: timing failed");
    return rc;
  }
  if (chosen) {
    chosen[0] = pick.alpha;
    chosen[1] = pick.beta;
    chosen[2] = (float)pick.large_row;
    chosen[3] = best;
  }
  return bfs_recompute(b);
}

int bfs_set_accounting(Bfs* b, int on) {
  if (on && !b->acct && cudaMalloc(&b->acct, 8 * sizeof(unsigned long long)) != cudaSuccess) {
    set_error("accounting counter allocation failed");
    return -4;
  }
  if (on) VX_CUDA_TRY(cudaMemsetAsync(b->acct, 0, 8 * sizeof(unsigned long long), b->g->stream));
  b->acct_on = on != 0;
  return 0;
}

int bfs_accounting(Bfs* b, unsigned long long* out5) {
  memset(out5, 0, 5 * sizeof(unsigned long long));
  if (!b->acct) return 0;
  VX_CUDA_TRY(cudaMemcpyAsync(out5, b->acct, 5 * sizeof(unsigned long long), cudaMemcpyDeviceToHost, b->g->stream));
  VX_CUDA_TRY(cudaStreamSynchronize(b->g->stream));
  return 0;
}

int bfs_stage(Bfs* b, size_t n, size_t vertex_bound, bool classify) {
  Graph* g = b->g;
  cudaStream_t s = g->stream;
  b->staged_ops = n;
  b->staged_V_pre = g->V;
  b->staged_len_pre = b->dist_len;
  if (n == 0) {  // last_* counters reset on every apply (bfs.hpp:30-33)
    VX_CUDA_TRY(cudaMemsetAsync(&b->ctr->candidates, 0, 4 * sizeof(uint32_t), s));
    return 0;
  }
  // a non-empty batch resets them (and the repair lists) in whichever path
  // consumes it: the fused launch in its first phase, the per-phase and full
  // paths on the host before their kernels
  b->staged_classified = classify;
  if (int rc = graph_stage_batch(g, n, vertex_bound, classify)) return rc;
  if (int rc = ensure_capacity(b, std::max<size_t>(g->V, 1))) return rc;
  return ensure_ring(b);
}

static int launch_stream(Bfs* b, Params& p, StreamArgs& sa) {
  if (!b->stream_grid) {
    int per_sm = 0;
    VX_CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, bfs_stream_kernel, kThreads, 0));
    if (per_sm < 1) {
      set_error("stream kernel cannot be resident on an SM");
      return -3;
    }
    b->stream_grid = per_sm * sm_count();
  }
  // one block per SM by default: against two per SM (every co-resident
  // block) the grid barriers and the work ring's polling are cheaper, and the
  // update step measured 13% faster at R-MAT 22 and R-MAT 20
  const uint32_t want = b->tune.update_blocks ? b->tune.update_blocks : (uint32_t)sm_count();
  p.nblocks = want < (uint32_t)b->stream_grid ? want : (uint32_t)b->stream_grid;
  void* args[] = {&p, &sa};
  count_launch();
  VX_CUDA_TRY(cudaLaunchCooperativeKernel((const void*)bfs_stream_kernel, dim3(p.nblocks), dim3(kThreads), args,
                                          0, b->g->stream));
  return 0;
}

// The staged batch of an undirected graph as a one-batch stream: tombstones,
// delta removals, the cascade, delta insertions and the post-batch repair in
// one persistent launch (the arcs were classified when they were staged).
static int repair_fused(Bfs* b) {
  Graph* g = b->g;
  const size_t n = b->staged_ops, m = 2 * n;
  StreamArgs sa;
  memset(&sa, 0, sizeof(sa));
  sa.fu = g->batch.fu;
  sa.fv = g->batch.fv;
  sa.ff = g->batch.ff;
  sa.fpos = g->batch.fpos;
  sa.bcnt = &g->ctr->final_arcs;
  sa.scratch = g->batch.lu;
  sa.gc = g->ctr;
  sa.arena_cap = g->adj[0].arena_cap;
  sa.frac = b->frac;
  sa.nb = 1;
  sa.V0 = (uint32_t)b->staged_V_pre;
  sa.len0 = (uint32_t)b->staged_len_pre;
  sa.v_single = (uint32_t)g->V;
  sa.classified = b->staged_classified ? 1u : 0u;
  Params p = make_params(b, (uint32_t)g->V, (uint32_t)g->V);
  if (int rc = launch_stream(b, p, sa)) return rc;
  g->adj[0].arena_bound += 8ull * m + 8;  // the bound the staging reserved for
  ++g->version;
  b->dist_len = std::max<size_t>(b->dist_len, g->V);
  b->staged_ops = 0;
  return 0;
}

int bfs_repair_staged(Bfs* b) {
  Graph* g = b->g;
  cudaStream_t s = g->stream;
  if (b->staged_ops == 0) return 0;
  if (!g->directed && b->tune.fused) return repair_fused(b);
  VX_CUDA_TRY(cudaMemsetAsync(&b->ctr->candidates, 0, 4 * sizeof(uint32_t), s));
  VX_CUDA_TRY(cudaMemsetAsync(&b->ctr->cand_n, 0, 3 * sizeof(uint32_t), s));
  VX_CUDA_TRY(cudaMemsetAsync(b->ctr->rtrace, 0, sizeof(b->ctr->rtrace), s));
  VX_CUDA_TRY(cudaMemsetAsync(b->ctr->handovers, 0, sizeof(b->ctr->handovers), s));
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
  VX_CUDA_TRY(cudaMemsetAsync(b->ctr->rtrace, 0, sizeof(b->ctr->rtrace), b->g->stream));
  VX_CUDA_TRY(cudaMemsetAsync(b->ctr->handovers, 0, sizeof(b->ctr->handovers), b->g->stream));
  return bfs_recompute(b);
}

int bfs_apply_staged(Bfs* b, size_t n, size_t vertex_bound) {
  // the fused repair classifies the arcs itself; the per-phase path needs them classified
  const bool fused = !b->g->directed && b->tune.fused;
  if (int rc = bfs_stage(b, n, vertex_bound, !fused)) return rc;
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

int bfs_phase_trace(Bfs* b, unsigned long long* out, size_t cap, size_t* n) {
  if (int rc = bfs_sync(b)) return rc;
  constexpr size_t kR = sizeof(b->hctr->rtrace) / sizeof(b->hctr->rtrace[0]);
  constexpr size_t kS = sizeof(b->hctr->stream_ns) / sizeof(b->hctr->stream_ns[0]);
  constexpr size_t kH = sizeof(b->hctr->handovers) / sizeof(b->hctr->handovers[0]);
  *n = kR + kS + kH;
  for (size_t i = 0; i < std::min(cap, kR); ++i) out[i] = b->hctr->rtrace[i];
  for (size_t i = kR; i < std::min(cap, kR + kS); ++i) out[i] = b->hctr->stream_ns[i - kR];
  for (size_t i = kR + kS; i < std::min(cap, kR + kS + kH); ++i) out[i] = b->hctr->handovers[i - kR - kS];
  return 0;
}

// ------------------------------------------------------- batched stream --

void StreamBufs::free_all() {
  void* ptrs[] = {src, dst, add, off, keys, keys_alt, vals, vals_alt, flag, pos, fu, fv, bid, ff, fpos,
                  boff, bcnt, vpost, total, scratch, digest, bstats};
  for (void* q : ptrs) cudaFree(q);
  *this = StreamBufs();
}

int StreamBufs::ensure(size_t n, size_t nb, size_t maxf) {
  if (n <= ops_cap && nb <= nb_cap && maxf <= maxf_cap) return 0;
  const size_t N = std::max(n, ops_cap), B = std::max(nb, nb_cap), MF = std::max(maxf, maxf_cap);
  free_all();
  const size_t m = 2 * std::max<size_t>(N, 1);
  bool ok = true;
  auto al = [&](auto** q, size_t count, size_t size) {
    if (ok && cudaMalloc((void**)q, std::max<size_t>(count, 1) * size) != cudaSuccess) ok = false;
  };
  al(&src, N, 4);
  al(&dst, N, 4);
  al(&add, N, 1);
  al(&off, B + 1, 8);
  al(&keys, m, 8);
  al(&keys_alt, m, 8);
  al(&vals, m, 4);
  al(&vals_alt, m, 4);
  al(&flag, m, 4);
  al(&pos, m, 4);
  al(&fu, m, 4);
  al(&fv, m, 4);
  al(&bid, m, 4);
  al(&ff, m, 1);
  al(&fpos, m, 8);
  al(&boff, B + 1, 4);
  al(&bcnt, B, 4);
  al(&vpost, B, 4);
  al(&total, 1, 4);
  al(&scratch, MF, 4);
  al(&digest, B, 8);
  al(&bstats, 4 * B, 4);
  if (!ok) {
    free_all();
    set_error("stream buffer allocation failed");
    return -4;
  }
  ops_cap = N;
  nb_cap = B;
  maxf_cap = MF;
  return 0;
}

int bfs_apply_stream(Bfs* b, const uint32_t* hs, const uint32_t* hd, const uint8_t* ha, const uint64_t* hoff,
                     size_t nb, uint64_t* digests, uint32_t* stats, size_t* applied) {
  Graph* g = b->g;
  cudaStream_t st = g->stream;
  *applied = 0;
  if (nb == 0) return 0;
  if (hoff[0] != 0) {
    set_error("batch offsets must start at 0");
    return -1;
  }
  const size_t n = hoff[nb];
  const size_t Vbefore = g->V;
  // vertex count after every batch (the graph grows to max id + 1 over the
  // non-self-loop ops, dynamic_graph.hpp:717-733) and the arena bound
  std::vector<uint32_t> vpost(nb);
  size_t V = g->V, maxf = 1;
  uint64_t bound = 0;
  size_t nonempty = 0;
  for (size_t t = 0; t < nb; ++t) {
    if (hoff[t + 1] < hoff[t]) {
      set_error("batch offsets must not decrease");
      return -1;
    }
    for (uint64_t i = hoff[t]; i < hoff[t + 1]; ++i)
      if (hs[i] != hd[i]) V = std::max<size_t>(V, (size_t)std::max(hs[i], hd[i]) + 1);
    if (V > vxb::kMaxVertices) {
      set_error("vertex id beyond the supported maximum (2^31 - 1)");
      return -2;
    }
    vpost[t] = (uint32_t)V;
    const size_t m = 2 * (size_t)(hoff[t + 1] - hoff[t]);
    if (m) {
      bound += 8ull * m + 8;
      ++nonempty;
    }
    maxf = std::max(maxf, m);
  }
  int bbits = 1;
  while (bbits < 32 && ((size_t)1 << bbits) < std::max<size_t>(V, 2)) ++bbits;
  int tbits = 1;
  while (tbits < 40 && ((size_t)1 << tbits) < nb) ++tbits;
  const uint32_t window = std::min<uint32_t>(b->tune.stream_window, kMaxVersions);
  if (!stats && window && !g->directed && nb >= 2 && 2 * bbits + 8 <= 64 && n < (1ull << 31)) {
    // every batch but the last in version-parallel windows
    StreamBufs& S = b->sb;
    if (int rc = S.ensure(n, nb, maxf)) return rc;
    VX_CUDA_TRY(cudaMemcpyAsync(S.src, hs, n * 4, cudaMemcpyHostToDevice, st));
    VX_CUDA_TRY(cudaMemcpyAsync(S.dst, hd, n * 4, cudaMemcpyHostToDevice, st));
    VX_CUDA_TRY(cudaMemcpyAsync(S.add, ha, n, cudaMemcpyHostToDevice, st));
    // every window's buffers up front, so that no window allocates
    size_t wops = 0;
    for (size_t t0 = 0; t0 + 1 < nb; t0 += window)
      wops = std::max<size_t>(wops, hoff[std::min<size_t>(t0 + window, nb - 1)] - hoff[t0]);
    if (int rc = stream_versions_reserve(b, wops, std::max<size_t>(b->dist_len, vpost[nb - 2]),
                                         std::min<size_t>(window, nb - 1)))
      return rc;
    for (size_t t0 = 0; t0 + 1 < nb; t0 += window) {
      const size_t t1 = std::min<size_t>(t0 + window, nb - 1);
      if (int rc = stream_versions(b, S.src, S.dst, S.add, hoff, vpost.data(), t0, t1, digests)) return rc;
      *applied = t1;
    }
    const uint64_t tail[2] = {0, hoff[nb] - hoff[nb - 1]};
    const uint64_t lo = hoff[nb - 1];
    size_t last = 0;
    if (int rc = bfs_apply_stream(b, hs + lo, hd + lo, ha + lo, tail, 1, digests ? digests + nb - 1 : nullptr,
                                  nullptr, &last))
      return rc;
    *applied += last;
    return 0;
  }
  // the persistent path covers undirected graphs whose (batch, u, v) keys fit
  // 64 bits and whose arena takes the whole stream; the caller loops otherwise
  if (g->directed || 2 * bbits + tbits > 64 || n >= (1ull << 31)) return 0;
  int fits = 0;
  if (int rc = graph_reserve_stream(g, bound, &fits)) return rc;
  if (!fits) return 0;
  if (int rc = graph_grow(g, V)) return rc;
  const uint32_t len0 = (uint32_t)b->dist_len;
  if (int rc = ensure_capacity(b, std::max<size_t>(V, 1))) return rc;
  Adjacency& a = g->adj[0];
  a.arena_bound += bound;
  if (int rc = ensure_ring(b)) return rc;
  StreamBufs& S = b->sb;
  if (int rc = S.ensure(n, nb, maxf)) return rc;
  VX_CUDA_TRY(cudaMemcpyAsync(S.src, hs, n * 4, cudaMemcpyHostToDevice, st));
  VX_CUDA_TRY(cudaMemcpyAsync(S.dst, hd, n * 4, cudaMemcpyHostToDevice, st));
  VX_CUDA_TRY(cudaMemcpyAsync(S.add, ha, n, cudaMemcpyHostToDevice, st));
  VX_CUDA_TRY(cudaMemcpyAsync(S.off, hoff, (nb + 1) * 8, cudaMemcpyHostToDevice, st));
  VX_CUDA_TRY(cudaMemcpyAsync(S.vpost, vpost.data(), nb * 4, cudaMemcpyHostToDevice, st));
  const size_t m = 2 * n;
  const unsigned grid_n = (unsigned)std::max<size_t>(1, std::min<size_t>((n + 255) / 256, (size_t)sm_count() * 32));
  const unsigned grid_m = (unsigned)std::max<size_t>(1, std::min<size_t>((m + 255) / 256, (size_t)sm_count() * 32));
  count_launch();
  stream_keys_kernel<<<grid_n, 256, 0, st>>>(S.src, S.dst, S.add, S.off, (uint32_t)nb, n, bbits, S.keys, S.vals);
  VX_CUDA_TRY(cudaGetLastError());
  bool in_alt = false;
  if (int rc = radix_sort_u64(S.keys, S.keys_alt, S.vals, S.vals_alt, m, 2 * bbits + tbits, &in_alt, g->scratch, st))
    return rc;
  uint64_t* keys = in_alt ? S.keys_alt : S.keys;
  uint32_t* vals = in_alt ? S.vals_alt : S.vals;
  count_launch();
  stream_last_kernel<<<grid_m, 256, 0, st>>>(keys, m, S.flag);
  if (int rc = scan_exclusive_u32(S.flag, S.pos, m, S.total, g->scratch, st)) return rc;
  count_launch();
  stream_compact_kernel<<<grid_m, 256, 0, st>>>(keys, vals, S.flag, S.pos, m, bbits, S.fu, S.fv, S.ff, S.bid);
  count_launch();
  stream_bounds_kernel<<<(unsigned)((nb + 256) / 256), 256, 0, st>>>(S.bid, S.total, (uint32_t)nb, S.boff, S.bcnt);
  VX_CUDA_TRY(cudaGetLastError());
  if (digests) VX_CUDA_TRY(cudaMemsetAsync(S.digest, 0, nb * 8, st));
  StreamArgs sa;
  memset(&sa, 0, sizeof(sa));
  sa.fu = S.fu;
  sa.fv = S.fv;
  sa.ff = S.ff;
  sa.fpos = S.fpos;
  sa.boff = S.boff;
  sa.bcnt = S.bcnt;
  sa.vpost = S.vpost;
  sa.scratch = S.scratch;
  sa.digest = digests ? S.digest : nullptr;
  sa.bstats = stats ? S.bstats : nullptr;
  sa.gc = g->ctr;
  sa.arena_cap = a.arena_cap;
  sa.frac = b->frac;
  sa.nb = (uint32_t)nb;
  sa.V0 = (uint32_t)Vbefore;
  sa.len0 = len0;
  Params p = make_params(b, (uint32_t)V, (uint32_t)V);
  if (int rc = launch_stream(b, p, sa)) return rc;
  g->version += nonempty;
  b->dist_len = V;
  b->staged_ops = 0;
  if (digests) VX_CUDA_TRY(cudaMemcpyAsync(digests, S.digest, nb * 8, cudaMemcpyDeviceToHost, st));
  if (stats) VX_CUDA_TRY(cudaMemcpyAsync(stats, S.bstats, nb * 16, cudaMemcpyDeviceToHost, st));
  if (digests || stats) VX_CUDA_TRY(cudaStreamSynchronize(st));
  *applied = nb;
  return 0;
}

int bfs_digest(Bfs* b, uint64_t* out) {
  cudaStream_t st = b->g->stream;
  unsigned long long* d = &b->ctr->scratch64;
  VX_CUDA_TRY(cudaMemsetAsync(d, 0, 8, st));
  if (b->dist_len) {
    count_launch();
    digest_kernel<<<sm_count() * 8, 256, 0, st>>>(b->dist, (uint32_t)b->dist_len, d);
    VX_CUDA_TRY(cudaGetLastError());
  }
  VX_CUDA_TRY(cudaMemcpyAsync(b->g->pinned_scalar, d, 8, cudaMemcpyDeviceToHost, st));
  VX_CUDA_TRY(cudaStreamSynchronize(st));
  *out = b->g->pinned_scalar[0];
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
// loads this library holds the array (about 8.5 MB) until the process exits;
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
  uint32_t bul[2 * (kStaticMaxVertices + kListSlack)];  // the bottom-up candidate lists
  uint2 drow[kStaticMaxVertices];  // kept all-zero: a plain CSR has no delta rows
  BfsCounters ctr;
  uint32_t bar[vxb::kBarrierWords];
};

}  // namespace
}  // namespace vxh

static __device__ __align__(256) unsigned char vx_static_bfs_scratch[sizeof(vxh::StaticBfsScratch)];

namespace {
constexpr int kStaticMaxDevices = 64;
// device address of the array, per device; two host threads making their
// first call on one device at once both look it up and store the same value
std::atomic<void*> g_static_scratch_addr[kStaticMaxDevices];
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
  void* addr = g_static_scratch_addr[dev].load(std::memory_order_acquire);
  if (!addr) {
    // one-time set-up on this device (the device is current here)
    const cudaError_t e = cudaGetSymbolAddress(&addr, vx_static_bfs_scratch);
    if (e != cudaSuccess || !addr) {
      vxh::set_error("vx_bfs_csr_static: cudaGetSymbolAddress failed: %s", cudaGetErrorString(e));
      return -3;
    }
    g_static_scratch_addr[dev].store(addr, std::memory_order_release);
  }
  StaticBfsScratch* sc = static_cast<StaticBfsScratch*>(addr);
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
  p.bul = sc->bul;
  p.bul_half = vxh::kStaticMaxVertices + vxh::kListSlack;
  p.c = &sc->ctr;
  p.total_arcs = arcs;
  p.alpha = 14.0f;
  p.beta = 24.0f;
  p.large_row = 1024;
  p.bar = sc->bar;
  int per_sm = 0, sms = 0;
  VX_CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, vxh::bfs_full_kernel, vxh::kThreads, 0));
  VX_CUDA_TRY(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
  if (per_sm < 1) {
    vxh::set_error("vx_bfs_csr_static: BFS kernel cannot be resident on an SM");
    return -3;
  }
  p.nblocks = (uint32_t)(per_sm * sms);
  void* args[] = {&p};
  vxh::count_launch();
  VX_CUDA_TRY(cudaLaunchCooperativeKernel((const void*)vxh::bfs_full_kernel, dim3(p.nblocks), dim3(vxh::kThreads),
                                          args, 0, s));
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
