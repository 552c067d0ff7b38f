// Device BFS state: the B200 counterpart of BasicIncrementalBFS<DynamicGraph>
// (include/velographx/incremental/bfs.hpp:13-383).
#pragma once

#include <cstddef>
#include <cstdint>

#include "graph.cuh"

namespace vxh {

struct BfsCounters {
  unsigned long long reachable;   // finite distances
  unsigned long long arcs;        // sum of out-degrees of reached vertices (full BFS)
  uint32_t levels;
  uint32_t candidates;            // last_deletion_candidates
  uint32_t affected;              // last_affected_vertices
  uint32_t full;                  // last_used_full_recompute
  uint32_t fallback;              // fixpoint exceeded the fallback limit
  uint32_t err;
  // per-level counters of the persistent loops (3-way rotation)
  uint32_t lvl_n[3];
  uint32_t lvl_big[3];
  unsigned long long lvl_m[3];
  // repair bookkeeping
  uint32_t cand_n;       // deletion candidates (distinct heads)
  uint32_t touched_n;    // vertices whose support word is non-zero (lst_t)
  uint32_t a_n;          // affected list length
  uint32_t big_b;        // affected hubs whose boundary the whole grid computes
  unsigned long long scratch64;  // single-value readbacks
  // globaltimer stamps of the last repair: pre entry, after its seeds, after
  // its cascade; post entry, after the boundary distances, after its seeds,
  // after the relaxation; then the items pushed by the cascade and by the
  // relaxation; then the drain statistics of the cascade and of the
  // relaxation (claims, failed claims, idle rounds, slot waits, cycles
  // spent processing summed over blocks, and the longest processing round)
  unsigned long long rtrace[21];
  // time spent by the last stream launch in each of its per-batch phases
  // (classify + tombstones, removals + candidates, cascade, insertions,
  // post-batch repair, end-of-batch barrier), summed over its batches, ns
  unsigned long long stream_ns[6];
  // removal arcs of the update launch's current batch (two slots, by batch
  // parity; zero between launches): a batch without any skips the removal
  // phase and its barrier
  uint32_t rmb[2];
  // the post-batch relaxation passed its time budget and the batch's
  // distances come from a full BFS (zero between batches)
  uint32_t rbig;
  // the cascade passed its time budget and the affected set comes from a BFS
  // of the graph without the batch's deletions (zero between batches), and
  // the number of vertices whose distance that BFS raised
  uint32_t cbig;
  uint32_t a_bfs;
  // globaltimer ns the last full BFS took, and the time at which the running
  // repair phase hands over to a BFS (~0: never)
  unsigned long long full_ns;
  unsigned long long deadline;
  // batches of the last apply or stream launch whose cascade [0] or
  // relaxation [1] handed over to a BFS
  unsigned long long handovers[2];
};

struct BfsTuning {
  float alpha = 14.0f;       // top-down -> bottom-up when m_f * alpha > m_u
  float beta = 24.0f;        // bottom-up -> top-down when n_f * beta < V (shrinking)
  uint32_t large_row = 1024; // rows this long are expanded by the whole grid
  bool fused = true;         // undirected batches: one persistent launch after staging
  uint32_t update_blocks = 0;  // blocks of the update launch (0: every co-resident block)
  // batches per version-parallel window of a stream whose per-batch repair
  // counters are not asked for (0: every batch by the update launch)
  uint32_t stream_window = 256;
  // a window traversal's level pulls when its frontier holds more than this
  // fraction of the vertices
  float window_pull_frac = 0.02f;
  // a repair phase (the cascade, the relaxation) that has run longer than this
  // multiple of the last full BFS's time hands over to a BFS (0: at its first
  // work-ring round; negative: never)
  float handover = 1.0f;
};

struct VersionBufs;

// Device buffers of the batched stream path (kept between calls).
struct StreamBufs {
  size_t ops_cap = 0, nb_cap = 0, maxf_cap = 0;
  uint32_t *src = nullptr, *dst = nullptr;
  uint8_t* add = nullptr;
  uint64_t* off = nullptr;
  uint64_t *keys = nullptr, *keys_alt = nullptr;
  uint32_t *vals = nullptr, *vals_alt = nullptr, *flag = nullptr, *pos = nullptr;
  uint32_t *fu = nullptr, *fv = nullptr, *bid = nullptr;
  uint8_t* ff = nullptr;
  uint64_t* fpos = nullptr;
  uint32_t *boff = nullptr, *bcnt = nullptr, *vpost = nullptr, *total = nullptr, *scratch = nullptr;
  unsigned long long* digest = nullptr;
  uint32_t* bstats = nullptr;
  int ensure(size_t ops, size_t batches, size_t max_batch_arcs);
  void free_all();
};

struct Bfs {
  Graph* g = nullptr;
  uint32_t source = 0;
  double frac = 0.35;
  size_t dist_len = 0;  // the reference's dist_.size()
  size_t cap = 0;       // allocated per-vertex capacity
  uint32_t* dist = nullptr;
  uint32_t* vis = nullptr;
  uint32_t* fb[3] = {nullptr, nullptr, nullptr};
  uint32_t* q[3] = {nullptr, nullptr, nullptr};
  uint32_t* big = nullptr;
  uint32_t* lst_a = nullptr;  // affected list
  uint32_t* lst_t = nullptr;  // touched (lost > 0) list
  uint32_t* tent = nullptr;   // boundary seed distance of each affected entry
  uint32_t* bul = nullptr;    // two bottom-up candidate lists of cap entries each (full BFS)
  uint32_t* sw = nullptr;     // 64-bit support words, as pairs of u32 (zero between batches)
  unsigned long long* ring = nullptr;  // work ring of the repair phases (ring_slots, a power of two)
  size_t ring_slots = 0;
  uint32_t* rq = nullptr;     // ring counters head / tail / done, one 128-byte line each
  uint32_t* aff = nullptr;    // affected bitmap (zero between batches)
  uint32_t* inq[2] = {nullptr, nullptr};  // queued bitmaps of the decrease propagation
  BfsCounters* ctr = nullptr;
  BfsCounters* hctr = nullptr;
  unsigned long long* trace = nullptr;  // per-level timestamps of the last full BFS
  uint32_t* barrier = nullptr;          // grid barrier words (vxb::kBarrierWords)
  float* features = nullptr;            // selector features of the staged batch
  size_t staged_ops = 0, staged_V_pre = 0, staged_len_pre = 0;  // batch staged by bfs_stage
  bool staged_classified = true;
  BfsTuning tune;
  int grid = 0;       // blocks of the repair kernel
  int full_grid = 0;  // blocks of the full-BFS kernel
  int stream_grid = 0;
  unsigned long long* acct = nullptr;  // algorithmic-byte accounting (5 counters), when on
  bool acct_on = false;
  StreamBufs sb;
  VersionBufs* vb = nullptr;  // version-parallel stream buffers, made on first use
};

int bfs_create(Bfs** out, Graph* g, uint32_t source, double frac);
void bfs_destroy(Bfs* b);
int bfs_recompute(Bfs* b);
// Algorithmic-byte accounting of the update launches: on != 0 allocates and
// zeroes the counters and turns it on; counters are {row arcs scanned by the
// repair, vertices visited, delta-row entries read and written, canonical
// arcs, batches} summed since it was turned on.
int bfs_set_accounting(Bfs* b, int on);
int bfs_accounting(Bfs* b, unsigned long long* out5);
// Times a grid of (alpha, beta, large_row) on full BFS from the k roots and
// keeps the fastest (median over the roots); chosen = {alpha, beta,
// large_row, median ms}.  Recomputes b's own distances afterwards.
int bfs_autotune(Bfs* b, const uint32_t* roots, size_t k, float* chosen);
// Incremental apply of the batch in b->g->batch (ops already on device):
// bfs_stage (canonicalise + classify on the pre-batch graph) followed by
// bfs_repair_staged (the reference's apply) or bfs_full_staged (graph apply +
// recompute, the explicit full arm of the reference's selector harness).
int bfs_apply_staged(Bfs* b, size_t n, size_t vertex_bound);
int bfs_stage(Bfs* b, size_t n, size_t vertex_bound, bool classify = true);
int bfs_repair_staged(Bfs* b);
int bfs_full_staged(Bfs* b);
int bfs_sync(Bfs* b);  // copies counters to hctr (synchronises the stream)
int bfs_reached_arcs(Bfs* b, unsigned long long* arcs);  // sum of degrees of reached vertices
// Per-level trace of the last full BFS: pairs {globaltimer ns, n_f | bottom_up << 63}
// for every level, then a closing timestamp.  Writes up to cap u64 values.
int bfs_level_trace(Bfs* b, unsigned long long* out, size_t cap, size_t* n);
int bfs_phase_trace(Bfs* b, unsigned long long* out, size_t cap, size_t* n);
// The batches [hoff[t], hoff[t+1]) of host arrays (hoff[0] == 0) applied in
// order.  Undirected streams: without stats, every batch but the last in
// version-parallel windows of tune.stream_window batches, the last one (so
// that the object's repair counters are its own) by the update launch;
// otherwise all of them in one persistent update launch.  *applied = the
// number of leading batches applied; the caller applies the rest one by one
// (directed graphs, keys past 64 bits, an arena the stream does not fit).
// digests / stats (optional, host) receive the distance digest and
// {candidates, affected, full, reachable} after every batch.
int bfs_apply_stream(Bfs* b, const uint32_t* hs, const uint32_t* hd, const uint8_t* ha, const uint64_t* hoff,
                     size_t nb, uint64_t* digests, uint32_t* stats, size_t* applied);
// Distance, bitmap and list buffers for V vertices.
int bfs_ensure_capacity(Bfs* b, size_t V);
// Order-independent digest of the current distances: the sum over v of
// splitmix64(v << 32 | dist[v]) modulo 2^64.
int bfs_digest(Bfs* b, uint64_t* out);

}  // namespace vxh
