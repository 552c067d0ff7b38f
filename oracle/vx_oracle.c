/*
 * CPU oracle: plain-C restatement of VeloGraphX's dynamic-BFS path.
 *
 * TEST INFRASTRUCTURE ONLY -- the checker, never the product.  Only tests/,
 * __graft_entry__.smoke() and bench.py's CPU-baseline leg load this library.
 *
 * Every function names the reference lines it restates (paths relative to the
 * VeloGraphX project root).  The restatement keeps the reference's observable
 * semantics -- the logical adjacency, the overlay/compaction counters, the
 * order-sensitive counters of IncrementalBFS -- while using its own storage:
 * each base row (base CSR row or compacted patch) is one sorted array, and the
 * delta overlay is one sorted (dst, present) array per row.
 */
#include "vx_oracle.h"

#include <stdlib.h>
#include <string.h>

/* ------------------------------------------------------------------ rows -- */

typedef struct {
  uint32_t* v;
  size_t n, cap;
} row_t;

typedef struct {
  uint32_t* v;
  uint8_t* p;
  size_t n, cap;
} orow_t;

typedef struct {
  uint32_t* v;
  size_t n, cap;
} vec_t;

static void vec_push(vec_t* a, uint32_t x) {
  if (a->n == a->cap) {
    a->cap = a->cap ? a->cap * 2 : 16;
    a->v = (uint32_t*)realloc(a->v, a->cap * sizeof(uint32_t));
  }
  a->v[a->n++] = x;
}

static void row_reserve(row_t* r, size_t need) {
  if (r->cap >= need) return;
  size_t c = r->cap ? r->cap : 4;
  while (c < need) c *= 2;
  r->v = (uint32_t*)realloc(r->v, c * sizeof(uint32_t));
  r->cap = c;
}

static void orow_reserve(orow_t* r, size_t need) {
  if (r->cap >= need) return;
  size_t c = r->cap ? r->cap : 4;
  while (c < need) c *= 2;
  r->v = (uint32_t*)realloc(r->v, c * sizeof(uint32_t));
  r->p = (uint8_t*)realloc(r->p, c);
  r->cap = c;
}

static size_t lower_bound_u32(const uint32_t* a, size_t n, uint32_t x) {
  size_t lo = 0, hi = n;
  while (lo < hi) {
    size_t mid = lo + (hi - lo) / 2;
    if (a[mid] < x) lo = mid + 1;
    else hi = mid;
  }
  return lo;
}

static int cmp_u32(const void* a, const void* b) {
  uint32_t x = *(const uint32_t*)a, y = *(const uint32_t*)b;
  return x < y ? -1 : (x > y);
}

static int cmp_u64(const void* a, const void* b) {
  uint64_t x = *(const uint64_t*)a, y = *(const uint64_t*)b;
  return x < y ? -1 : (x > y);
}

/* ------------------------------------------------------- delta overlay -- */
/* PackedDeltaStore (dynamic_graph.hpp:221-446): per-row sorted overlay with
 * live/present/absent counters. */
typedef struct {
  orow_t* rows;
  size_t live, present, absent;
} dstore_t;

/* set_if_changed  dynamic_graph.hpp:261-308 */
static int ds_set_if_changed(dstore_t* d, uint32_t u, uint32_t v, int desired, int base) {
  orow_t* r = &d->rows[u];
  size_t pos = lower_bound_u32(r->v, r->n, v);
  int found = pos < r->n && r->v[pos] == v;
  int current = found ? r->p[pos] : base;
  if (current == desired) return 0;
  if (desired == base) {
    if (!found) return 0;
    if (r->p[pos]) --d->present;
    else --d->absent;
    memmove(r->v + pos, r->v + pos + 1, (r->n - pos - 1) * sizeof(uint32_t));
    memmove(r->p + pos, r->p + pos + 1, (r->n - pos - 1));
    --r->n;
    --d->live;
    return 1;
  }
  if (found) {
    if (r->p[pos]) { --d->present; ++d->absent; }
    else { --d->absent; ++d->present; }
    r->p[pos] = (uint8_t)desired;
    return 1;
  }
  orow_reserve(r, r->n + 1);
  memmove(r->v + pos + 1, r->v + pos, (r->n - pos) * sizeof(uint32_t));
  memmove(r->p + pos + 1, r->p + pos, (r->n - pos));
  r->v[pos] = v;
  r->p[pos] = (uint8_t)desired;
  ++r->n;
  ++d->live;
  if (desired) ++d->present;
  else ++d->absent;
  return 1;
}

/* erase  dynamic_graph.hpp:423-439 */
static void ds_erase(dstore_t* d, uint32_t u, uint32_t v) {
  orow_t* r = &d->rows[u];
  if (r->n == 0) return;
  size_t pos = lower_bound_u32(r->v, r->n, v);
  if (pos == r->n || r->v[pos] != v) return;
  if (r->p[pos]) --d->present;
  else --d->absent;
  memmove(r->v + pos, r->v + pos + 1, (r->n - pos - 1) * sizeof(uint32_t));
  memmove(r->p + pos, r->p + pos + 1, (r->n - pos - 1));
  --r->n;
  --d->live;
}

/* upsert  dynamic_graph.hpp:391-421 */
static void ds_upsert(dstore_t* d, uint32_t u, uint32_t v, int present) {
  orow_t* r = &d->rows[u];
  size_t pos = lower_bound_u32(r->v, r->n, v);
  if (pos < r->n && r->v[pos] == v) {
    if (r->p[pos] != present) {
      if (r->p[pos]) { --d->present; ++d->absent; }
      else { --d->absent; ++d->present; }
      r->p[pos] = (uint8_t)present;
    }
    return;
  }
  orow_reserve(r, r->n + 1);
  memmove(r->v + pos + 1, r->v + pos, (r->n - pos) * sizeof(uint32_t));
  memmove(r->p + pos + 1, r->p + pos, (r->n - pos));
  r->v[pos] = v;
  r->p[pos] = (uint8_t)present;
  ++r->n;
  ++d->live;
  if (present) ++d->present;
  else ++d->absent;
}

/* set  dynamic_graph.hpp:255-259 */
static void ds_set(dstore_t* d, uint32_t u, uint32_t v, int desired, int base) {
  if (desired == base) ds_erase(d, u, v);
  else ds_upsert(d, u, v, desired);
}

/* clear_range for one row  dynamic_graph.hpp:322-334 */
static void ds_clear_row(dstore_t* d, uint32_t u) {
  orow_t* r = &d->rows[u];
  for (size_t i = 0; i < r->n; ++i) {
    if (r->p[i]) --d->present;
    else --d->absent;
  }
  d->live -= r->n;
  r->n = 0;
}

/* ----------------------------------------------------------------- graph -- */

struct vxo_graph {
  int directed;
  size_t V, Vcap;
  row_t* base_out; /* SegmentedCsr rows with CompactRowPatches applied */
  row_t* base_in;
  dstore_t delta_out, delta_in;
  vec_t dirty_out, dirty_in;
  size_t compact_out_edges, compact_in_edges;
  uint64_t version;
};

/* ensure_vertex / resize_vertices  dynamic_graph.hpp:493-500, 54-70, 228-230 */
static void g_grow(vxo_graph* g, size_t n) {
  if (n <= g->V) return;
  if (n > g->Vcap) {
    size_t c = g->Vcap ? g->Vcap : 16;
    while (c < n) c *= 2;
    g->base_out = (row_t*)realloc(g->base_out, c * sizeof(row_t));
    g->base_in = (row_t*)realloc(g->base_in, c * sizeof(row_t));
    g->delta_out.rows = (orow_t*)realloc(g->delta_out.rows, c * sizeof(orow_t));
    g->delta_in.rows = (orow_t*)realloc(g->delta_in.rows, c * sizeof(orow_t));
    memset(g->base_out + g->Vcap, 0, (c - g->Vcap) * sizeof(row_t));
    memset(g->base_in + g->Vcap, 0, (c - g->Vcap) * sizeof(row_t));
    memset(g->delta_out.rows + g->Vcap, 0, (c - g->Vcap) * sizeof(orow_t));
    memset(g->delta_in.rows + g->Vcap, 0, (c - g->Vcap) * sizeof(orow_t));
    g->Vcap = c;
  }
  g->V = n;
}

vxo_graph* vxo_graph_create(size_t vertices, int directed) {
  vxo_graph* g = (vxo_graph*)calloc(1, sizeof(vxo_graph));
  g->directed = directed != 0;
  g_grow(g, vertices);
  return g;
}

void vxo_graph_destroy(vxo_graph* g) {
  if (!g) return;
  for (size_t i = 0; i < g->Vcap; ++i) {
    free(g->base_out[i].v);
    free(g->base_in[i].v);
    free(g->delta_out.rows[i].v);
    free(g->delta_out.rows[i].p);
    free(g->delta_in.rows[i].v);
    free(g->delta_in.rows[i].p);
  }
  free(g->base_out);
  free(g->base_in);
  free(g->delta_out.rows);
  free(g->delta_in.rows);
  free(g->dirty_out.v);
  free(g->dirty_in.v);
  free(g);
}

size_t vxo_graph_vertex_count(const vxo_graph* g) { return g->V; }
uint64_t vxo_graph_version(const vxo_graph* g) { return g->version; }
int vxo_graph_directed(const vxo_graph* g) { return g->directed; }

static int base_contains(const row_t* r, uint32_t v) {
  size_t pos = lower_bound_u32(r->v, r->n, v);
  return pos < r->n && r->v[pos] == v;
}

/* Merge iterator over base row + overlay row, skipping absent entries:
 * for_each_effective_row  dynamic_graph.hpp:659-681. */
typedef struct {
  const uint32_t* b;
  size_t bn, i;
  const uint32_t* ov;
  const uint8_t* op;
  size_t on, j;
} nbr_it;

static void it_init(nbr_it* it, const row_t* base, const orow_t* ov) {
  it->b = base->v;
  it->bn = base->n;
  it->i = 0;
  it->ov = ov->v;
  it->op = ov->p;
  it->on = ov->n;
  it->j = 0;
}

static int it_next(nbr_it* it, uint32_t* out) {
  while (it->i < it->bn || it->j < it->on) {
    if (it->j == it->on || (it->i < it->bn && it->b[it->i] < it->ov[it->j])) {
      *out = it->b[it->i++];
      return 1;
    } else if (it->i == it->bn || it->ov[it->j] < it->b[it->i]) {
      int pr = it->op[it->j];
      uint32_t x = it->ov[it->j++];
      if (pr) { *out = x; return 1; }
    } else {
      int pr = it->op[it->j];
      uint32_t x = it->b[it->i];
      ++it->i;
      ++it->j;
      if (pr) { *out = x; return 1; }
    }
  }
  return 0;
}

static int out_it(const vxo_graph* g, uint32_t u, nbr_it* it) {
  if (u >= g->V) return 0;
  it_init(it, &g->base_out[u], &g->delta_out.rows[u]);
  return 1;
}

static int in_it(const vxo_graph* g, uint32_t v, nbr_it* it) {
  if (v >= g->V) return 0;
  it_init(it, &g->base_in[v], &g->delta_in.rows[v]);
  return 1;
}

/* materialize_row  dynamic_graph.hpp:683-708 */
static size_t materialize(const row_t* base, const orow_t* ov, uint32_t* out, size_t cap) {
  nbr_it it;
  it_init(&it, base, ov);
  size_t n = 0;
  uint32_t x;
  while (it_next(&it, &x)) {
    if (n < cap) out[n] = x;
    ++n;
  }
  return n;
}

size_t vxo_graph_neighbors(const vxo_graph* g, uint32_t u, uint32_t* out, size_t cap) {
  if (u >= g->V) return 0;
  return materialize(&g->base_out[u], &g->delta_out.rows[u], out, cap);
}

size_t vxo_graph_in_neighbors(const vxo_graph* g, uint32_t v, uint32_t* out, size_t cap) {
  if (v >= g->V) return 0;
  return materialize(&g->base_in[v], &g->delta_in.rows[v], out, cap);
}

/* has_edge  dynamic_graph.hpp:583-587 */
int vxo_graph_has_edge(const vxo_graph* g, uint32_t u, uint32_t v) {
  if (u >= g->V) return 0;
  const orow_t* r = &g->delta_out.rows[u];
  size_t pos = lower_bound_u32(r->v, r->n, v);
  if (pos < r->n && r->v[pos] == v) return r->p[pos];
  return base_contains(&g->base_out[u], v);
}

/* edge_count_directed  dynamic_graph.hpp:589-591 */
size_t vxo_graph_edge_count_directed(const vxo_graph* g) {
  return g->compact_out_edges + g->delta_out.present - g->delta_out.absent;
}

size_t vxo_graph_delta_edge_count(const vxo_graph* g) { return g->delta_out.live; }

/* base_edge_count_directed  dynamic_graph.hpp:593-595 */
size_t vxo_graph_base_edge_count_directed(const vxo_graph* g) { return g->compact_out_edges; }

/* ensure_vertex  dynamic_graph.hpp:493-500 (no version change) */
void vxo_graph_ensure_vertex(vxo_graph* g, uint32_t v) { g_grow(g, (size_t)v + 1); }

/* compact_neighbors / compact_in_neighbors  dynamic_graph.hpp:573-581: the
 * base-or-patch row without the overlay */
static size_t copy_row(const row_t* r, uint32_t* out, size_t cap) {
  const size_t m = r->n < cap ? r->n : cap;
  if (out && m) memcpy(out, r->v, m * sizeof(uint32_t));
  return r->n;
}
size_t vxo_graph_compact_neighbors(const vxo_graph* g, uint32_t u, uint32_t* out, size_t cap) {
  return u < g->V ? copy_row(&g->base_out[u], out, cap) : 0;
}
size_t vxo_graph_compact_in_neighbors(const vxo_graph* g, uint32_t v, uint32_t* out, size_t cap) {
  return v < g->V ? copy_row(&g->base_in[v], out, cap) : 0;
}

int vxo_graph_is_compact(const vxo_graph* g) {
  return g->delta_out.live == 0 && g->delta_in.live == 0;
}

/* normalize_dirty  dynamic_graph.hpp:735-738 */
static void normalize_dirty(vec_t* rows) {
  if (rows->n == 0) return;
  qsort(rows->v, rows->n, sizeof(uint32_t), cmp_u32);
  size_t w = 1;
  for (size_t i = 1; i < rows->n; ++i)
    if (rows->v[i] != rows->v[w - 1]) rows->v[w++] = rows->v[i];
  rows->n = w;
}

static size_t unique_count(const vec_t* rows) {
  if (rows->n == 0) return 0;
  uint32_t* c = (uint32_t*)malloc(rows->n * sizeof(uint32_t));
  memcpy(c, rows->v, rows->n * sizeof(uint32_t));
  qsort(c, rows->n, sizeof(uint32_t), cmp_u32);
  size_t w = 1;
  for (size_t i = 1; i < rows->n; ++i)
    if (c[i] != c[i - 1]) ++w;
  free(c);
  return w;
}

/* dirty_out_segment_count / dirty_in_segment_count  dynamic_graph.hpp:612-618
 * (counts unique dirty rows) */
size_t vxo_graph_dirty_out_count(const vxo_graph* g) { return unique_count(&g->dirty_out); }
size_t vxo_graph_dirty_in_count(const vxo_graph* g) { return unique_count(&g->dirty_in); }

/* compact_one_row  dynamic_graph.hpp:740-752 */
static void compact_one_row(row_t* base, dstore_t* d, uint32_t u, size_t* compact_edges) {
  orow_t* ov = &d->rows[u];
  if (ov->n == 0) return;
  size_t old_size = base[u].n;
  size_t n = materialize(&base[u], ov, NULL, 0);
  uint32_t* merged = (uint32_t*)malloc((n ? n : 1) * sizeof(uint32_t));
  materialize(&base[u], ov, merged, n);
  free(base[u].v);
  base[u].v = merged;
  base[u].n = n;
  base[u].cap = n ? n : 1;
  ds_clear_row(d, u);
  *compact_edges = *compact_edges - old_size + n;
}

/* compact_marked_rows  dynamic_graph.hpp:754-762 */
static void compact_marked(row_t* base, dstore_t* d, vec_t* dirty, size_t* ce) {
  normalize_dirty(dirty);
  for (size_t i = 0; i < dirty->n; ++i) compact_one_row(base, d, dirty->v[i], ce);
  dirty->n = 0;
}

/* compact_dense_rows  dynamic_graph.hpp:764-789 */
static int compact_dense(row_t* base, dstore_t* d, vec_t* dirty, size_t* ce, double threshold) {
  normalize_dirty(dirty);
  int compacted = 0;
  size_t w = 0;
  for (size_t i = 0; i < dirty->n; ++i) {
    uint32_t u = dirty->v[i];
    size_t overlay = d->rows[u].n;
    if (overlay == 0) continue;
    size_t base_size = base[u].n;
    size_t budget = base_size > 8 ? base_size : 8;
    double density = (double)overlay / (double)budget;
    if (density < threshold) {
      dirty->v[w++] = u;
      continue;
    }
    compact_one_row(base, d, u, ce);
    compacted = 1;
  }
  dirty->n = w;
  return compacted;
}

/* maybe_compact  dynamic_graph.hpp:620-631 (arena repack is a storage-layout
 * detail with no observable effect on the logical graph or the counters). */
int vxo_graph_maybe_compact(vxo_graph* g, double threshold) {
  int c = 0;
  c |= compact_dense(g->base_out, &g->delta_out, &g->dirty_out, &g->compact_out_edges, threshold);
  c |= compact_dense(g->base_in, &g->delta_in, &g->dirty_in, &g->compact_in_edges, threshold);
  return c;
}

/* compact  dynamic_graph.hpp:633-639 */
void vxo_graph_compact(vxo_graph* g) {
  if (vxo_graph_is_compact(g)) return;
  compact_marked(g->base_out, &g->delta_out, &g->dirty_out, &g->compact_out_edges);
  compact_marked(g->base_in, &g->delta_in, &g->dirty_in, &g->compact_in_edges);
}

/* automatic_storage_maintenance  dynamic_graph.hpp:791-803 */
static void auto_maintenance(vxo_graph* g) {
  const size_t kMinDelta = 65536;
  const double kGlobalRatio = 0.01;
  const double kRowDensity = 0.50;
  size_t denom = g->compact_out_edges > 1 ? g->compact_out_edges : 1;
  double ratio = (double)g->delta_out.live / (double)denom;
  if (g->delta_out.live >= kMinDelta && ratio >= kGlobalRatio)
    (void)vxo_graph_maybe_compact(g, kRowDensity);
}

/* apply_arc  dynamic_graph.hpp:726-733 */
static void apply_arc(vxo_graph* g, uint32_t u, uint32_t v, int present) {
  int base_present = base_contains(&g->base_out[u], v);
  if (!ds_set_if_changed(&g->delta_out, u, v, present, base_present)) return;
  ds_set(&g->delta_in, v, u, present, base_present);
  vec_push(&g->dirty_out, u);
  vec_push(&g->dirty_in, v);
}

/* apply_unversioned  dynamic_graph.hpp:717-724 */
static void apply_op(vxo_graph* g, uint32_t s, uint32_t d, int add) {
  if (s == d) return;
  g_grow(g, (size_t)(s > d ? s : d) + 1);
  apply_arc(g, s, d, add);
  if (!g->directed) apply_arc(g, d, s, add);
}

/* apply  dynamic_graph.hpp:543-549 */
int vxo_graph_apply(vxo_graph* g, const uint32_t* src, const uint32_t* dst,
                    const uint8_t* add, size_t n) {
  for (size_t i = 0; i < n; ++i) apply_op(g, src[i], dst[i], add[i] != 0);
  if (n) {
    ++g->version;
    auto_maintenance(g);
  }
  return 0;
}

/* Build sorted, unique rows from packed (u<<32|v) arcs: SegmentedCsr::build
 * dynamic_graph.hpp:79-111 (sort + unique + counting placement). */
static void build_rows(row_t* rows, size_t V, uint64_t* arcs, size_t n) {
  for (size_t i = 0; i < V; ++i) rows[i].n = 0;
  if (n == 0) return;
  qsort(arcs, n, sizeof(uint64_t), cmp_u64);
  size_t prev_ok = 0;
  for (size_t i = 0; i < n; ++i) {
    if (i && arcs[i] == arcs[prev_ok]) continue;
    prev_ok = i;
    uint32_t u = (uint32_t)(arcs[i] >> 32), v = (uint32_t)arcs[i];
    row_reserve(&rows[u], rows[u].n + 1);
    rows[u].v[rows[u].n++] = v;
  }
}

/* bulk_load_edges  dynamic_graph.hpp:502-529 (+ build_transpose_from :147-178) */
int vxo_graph_bulk_load(vxo_graph* g, const uint32_t* uv, size_t n) {
  uint32_t max_vertex = 0;
  int saw = 0;
  uint64_t* arcs = (uint64_t*)malloc((2 * n + 1) * sizeof(uint64_t));
  size_t na = 0;
  for (size_t i = 0; i < n; ++i) {
    uint32_t u = uv[2 * i], v = uv[2 * i + 1];
    if (u == v) continue;
    if (u > max_vertex) max_vertex = u;
    if (v > max_vertex) max_vertex = v;
    saw = 1;
    arcs[na++] = ((uint64_t)u << 32) | v;
    if (!g->directed) arcs[na++] = ((uint64_t)v << 32) | u;
  }
  if (saw) g_grow(g, (size_t)max_vertex + 1);
  build_rows(g->base_out, g->V, arcs, na);
  /* transpose */
  for (size_t i = 0; i < na; ++i) {
    uint64_t a = arcs[i];
    arcs[i] = ((a & 0xFFFFFFFFull) << 32) | (a >> 32);
  }
  build_rows(g->base_in, g->V, arcs, na);
  free(arcs);
  size_t edges = 0;
  for (size_t i = 0; i < g->V; ++i) edges += g->base_out[i].n;
  g->compact_out_edges = edges;
  g->compact_in_edges = edges;
  for (size_t i = 0; i < g->V; ++i) {
    g->delta_out.rows[i].n = 0;
    g->delta_in.rows[i].n = 0;
  }
  g->delta_out.live = g->delta_out.present = g->delta_out.absent = 0;
  g->delta_in.live = g->delta_in.present = g->delta_in.absent = 0;
  g->dirty_out.n = g->dirty_in.n = 0;
  ++g->version;
  return 0;
}

/* ------------------------------------------------------- incremental BFS -- */

/* ReusableKeySet  bfs.hpp:123-176: generation-stamped open-addressing set */
typedef struct {
  uint64_t* keys;
  uint32_t* stamps;
  size_t mask;
  uint32_t gen;
} keyset_t;

static uint64_t key_hash(uint64_t x) {
  x ^= x >> 33;
  x *= 0xff51afd7ed558ccdULL;
  x ^= x >> 33;
  x *= 0xc4ceb9fe1a85ec53ULL;
  x ^= x >> 33;
  return x;
}

static void ks_reset(keyset_t* s, size_t expected) {
  size_t req = 8, target = expected * 2 + 1;
  while (req < target) req <<= 1;
  if (s->mask + 1 < req || s->keys == NULL) {
    free(s->keys);
    free(s->stamps);
    s->keys = (uint64_t*)calloc(req, sizeof(uint64_t));
    s->stamps = (uint32_t*)calloc(req, sizeof(uint32_t));
    s->mask = req - 1;
    s->gen = 1;
    return;
  }
  if (++s->gen == 0) {
    memset(s->stamps, 0, (s->mask + 1) * sizeof(uint32_t));
    s->gen = 1;
  }
}

static int ks_insert(keyset_t* s, uint64_t key) {
  size_t slot = (size_t)key_hash(key) & s->mask;
  while (s->stamps[slot] == s->gen) {
    if (s->keys[slot] == key) return 0;
    slot = (slot + 1) & s->mask;
  }
  s->keys[slot] = key;
  s->stamps[slot] = s->gen;
  return 1;
}

static int ks_contains(const keyset_t* s, uint64_t key) {
  if (!s->keys) return 0;
  size_t slot = (size_t)key_hash(key) & s->mask;
  while (s->stamps[slot] == s->gen) {
    if (s->keys[slot] == key) return 1;
    slot = (slot + 1) & s->mask;
  }
  return 0;
}

typedef struct {
  uint32_t* u;
  uint32_t* v;
  size_t n, cap;
} pairs_t;

static void pairs_push(pairs_t* p, uint32_t u, uint32_t v) {
  if (p->n == p->cap) {
    p->cap = p->cap ? p->cap * 2 : 16;
    p->u = (uint32_t*)realloc(p->u, p->cap * sizeof(uint32_t));
    p->v = (uint32_t*)realloc(p->v, p->cap * sizeof(uint32_t));
  }
  p->u[p->n] = u;
  p->v[p->n] = v;
  ++p->n;
}

typedef struct {
  uint64_t* a; /* (dist << 32) | vertex, min-heap */
  size_t n, cap;
} heap_t;

static void heap_push(heap_t* h, uint64_t x) {
  if (h->n == h->cap) {
    h->cap = h->cap ? h->cap * 2 : 64;
    h->a = (uint64_t*)realloc(h->a, h->cap * sizeof(uint64_t));
  }
  size_t i = h->n++;
  while (i > 0) {
    size_t p = (i - 1) / 2;
    if (h->a[p] <= x) break;
    h->a[i] = h->a[p];
    i = p;
  }
  h->a[i] = x;
}

static uint64_t heap_pop(heap_t* h) {
  uint64_t top = h->a[0];
  uint64_t x = h->a[--h->n];
  size_t i = 0;
  for (;;) {
    size_t l = 2 * i + 1;
    if (l >= h->n) break;
    size_t c = (l + 1 < h->n && h->a[l + 1] < h->a[l]) ? l + 1 : l;
    if (h->a[c] >= x) break;
    h->a[i] = h->a[c];
    i = c;
  }
  if (h->n) h->a[i] = x;
  return top;
}

struct vxo_bfs {
  vxo_graph* g;
  uint32_t source;
  double frac;
  uint32_t* dist;
  size_t dist_len, dist_cap;
  size_t reachable;
  uint8_t* affected;
  uint32_t* lost;
  uint32_t* spc;
  size_t ws;
  vec_t touched;
  keyset_t seen, del_keys;
  pairs_t final_add, final_del, existing_del;
  vec_t candidates, affected_list, old_aff, invalidate, queue;
  heap_t heap;
  size_t last_candidates, last_affected;
  int last_full;
};

/* ensure_workspace  bfs.hpp:183-187 */
static void ensure_ws(vxo_bfs* b, size_t n) {
  if (b->ws >= n) return;
  b->affected = (uint8_t*)realloc(b->affected, n);
  b->lost = (uint32_t*)realloc(b->lost, n * sizeof(uint32_t));
  b->spc = (uint32_t*)realloc(b->spc, n * sizeof(uint32_t));
  memset(b->affected + b->ws, 0, n - b->ws);
  memset(b->lost + b->ws, 0, (n - b->ws) * sizeof(uint32_t));
  memset(b->spc + b->ws, 0, (n - b->ws) * sizeof(uint32_t));
  b->ws = n;
}

static void dist_resize(vxo_bfs* b, size_t n) {
  if (n > b->dist_cap) {
    b->dist = (uint32_t*)realloc(b->dist, (n ? n : 1) * sizeof(uint32_t));
    b->dist_cap = n;
  }
  for (size_t i = b->dist_len; i < n; ++i) b->dist[i] = VXO_UNREACHABLE;
  b->dist_len = n;
}

/* edge_key  bfs.hpp:178-181 */
static uint64_t edge_key(const vxo_bfs* b, uint32_t u, uint32_t v) {
  if (!b->g->directed && v < u) { uint32_t t = u; u = v; v = t; }
  return ((uint64_t)u << 32) | v;
}

/* is_shortest_parent  bfs.hpp:206-209 */
static int is_sp(const vxo_bfs* b, uint32_t u, uint32_t v) {
  return u < b->dist_len && v < b->dist_len && b->dist[u] != VXO_UNREACHABLE &&
         b->dist[v] != VXO_UNREACHABLE && b->dist[u] + 1 == b->dist[v];
}

/* shortest_parent_count  bfs.hpp:211-220 */
static uint32_t sp_count(vxo_bfs* b, uint32_t v) {
  if (v >= b->dist_len || v == b->source || b->dist[v] == VXO_UNREACHABLE) return 0;
  if (b->spc[v] != 0) return b->spc[v];
  uint32_t count = 0, p;
  nbr_it it;
  if (in_it(b->g, v, &it))
    while (it_next(&it, &p))
      if (is_sp(b, p, v)) ++count;
  b->spc[v] = count;
  return count;
}

/* recompute  bfs.hpp:100-120 */
void vxo_bfs_recompute(vxo_bfs* b) {
  size_t V = b->g->V;
  b->dist_len = 0;
  dist_resize(b, V);
  b->reachable = 0;
  ensure_ws(b, V);
  if (b->source >= V) return;
  b->queue.n = 0;
  b->dist[b->source] = 0;
  vec_push(&b->queue, b->source);
  size_t head = 0;
  while (head < b->queue.n) {
    uint32_t u = b->queue.v[head++], v;
    nbr_it it;
    out_it(b->g, u, &it);
    while (it_next(&it, &v)) {
      if (b->dist[v] == VXO_UNREACHABLE) {
        b->dist[v] = b->dist[u] + 1;
        vec_push(&b->queue, v);
      }
    }
  }
  b->reachable = b->queue.n;
}

vxo_bfs* vxo_bfs_create(vxo_graph* g, uint32_t source, double frac) {
  vxo_bfs* b = (vxo_bfs*)calloc(1, sizeof(vxo_bfs));
  b->g = g;
  b->source = source;
  b->frac = frac;
  vxo_bfs_recompute(b);
  return b;
}

void vxo_bfs_destroy(vxo_bfs* b) {
  if (!b) return;
  free(b->dist);
  free(b->affected);
  free(b->lost);
  free(b->spc);
  free(b->touched.v);
  free(b->seen.keys);
  free(b->seen.stamps);
  free(b->del_keys.keys);
  free(b->del_keys.stamps);
  free(b->final_add.u);
  free(b->final_add.v);
  free(b->final_del.u);
  free(b->final_del.v);
  free(b->existing_del.u);
  free(b->existing_del.v);
  free(b->candidates.v);
  free(b->affected_list.v);
  free(b->old_aff.v);
  free(b->invalidate.v);
  free(b->queue.v);
  free(b->heap.a);
  free(b);
}

/* record_parent_loss  bfs.hpp:229-240 */
static void record_loss(vxo_bfs* b, uint32_t v) {
  if (v >= b->dist_len || v == b->source || b->dist[v] == VXO_UNREACHABLE || b->affected[v])
    return;
  if (b->lost[v] == 0) vec_push(&b->touched, v);
  ++b->lost[v];
  uint32_t support = sp_count(b, v);
  if (support != 0 && b->lost[v] >= support) {
    b->affected[v] = 1;
    vec_push(&b->affected_list, v);
    vec_push(&b->invalidate, v);
    ++b->last_affected;
  }
}

/* compute_affected_prebatch  bfs.hpp:222-259 */
static int compute_affected_prebatch(vxo_bfs* b) {
  size_t lim = (size_t)((double)b->g->V * b->frac);
  if (lim < 1) lim = 1;
  for (size_t i = 0; i < b->existing_del.n; ++i) {
    uint32_t u = b->existing_del.u[i], v = b->existing_del.v[i];
    if (is_sp(b, u, v)) record_loss(b, v);
    if (!b->g->directed && is_sp(b, v, u)) record_loss(b, u);
  }
  size_t head = 0;
  while (head < b->invalidate.n) {
    if (b->last_affected > lim) return 0;
    uint32_t u = b->invalidate.v[head++], v;
    if (u >= b->dist_len || b->dist[u] == VXO_UNREACHABLE) continue;
    nbr_it it;
    out_it(b->g, u, &it);
    while (it_next(&it, &v)) {
      if (v >= b->dist_len || b->dist[v] != b->dist[u] + 1) continue;
      if (ks_contains(&b->del_keys, edge_key(b, u, v))) continue;
      record_loss(b, v);
    }
  }
  return b->last_affected <= lim;
}

/* best_boundary_distance  bfs.hpp:261-269 */
static uint32_t best_boundary(const vxo_bfs* b, uint32_t v) {
  uint32_t best = VXO_UNREACHABLE, p;
  nbr_it it;
  if (!in_it(b->g, v, &it)) return best;
  while (it_next(&it, &p)) {
    if (p >= b->dist_len || p >= b->ws || b->affected[p] || b->dist[p] == VXO_UNREACHABLE)
      continue;
    uint32_t c = b->dist[p] + 1;
    if (c < best) best = c;
  }
  return best;
}

/* propagate_decreases  bfs.hpp:341-354 */
static void propagate(vxo_bfs* b) {
  size_t head = 0;
  while (head < b->queue.n) {
    uint32_t u = b->queue.v[head++], v;
    if (b->dist[u] == VXO_UNREACHABLE) continue;
    nbr_it it;
    out_it(b->g, u, &it);
    while (it_next(&it, &v)) {
      if (b->dist[u] + 1 < b->dist[v]) {
        if (b->dist[v] == VXO_UNREACHABLE) ++b->reachable;
        b->dist[v] = b->dist[u] + 1;
        vec_push(&b->queue, v);
      }
    }
  }
}

/* repair_affected  bfs.hpp:271-319 */
static void repair_affected(vxo_bfs* b) {
  for (size_t i = 0; i < b->affected_list.n; ++i) {
    uint32_t v = b->affected_list.v[i];
    if (v < b->dist_len && b->dist[v] != VXO_UNREACHABLE) {
      b->dist[v] = VXO_UNREACHABLE;
      --b->reachable;
    }
  }
  b->heap.n = 0;
  for (size_t i = 0; i < b->affected_list.n; ++i) {
    uint32_t v = b->affected_list.v[i];
    uint32_t best = best_boundary(b, v);
    if (best != VXO_UNREACHABLE) {
      if (b->dist[v] == VXO_UNREACHABLE) ++b->reachable;
      b->dist[v] = best;
      heap_push(&b->heap, ((uint64_t)best << 32) | v);
    }
  }
  while (b->heap.n) {
    uint64_t top = heap_pop(&b->heap);
    uint32_t du = (uint32_t)(top >> 32), u = (uint32_t)top, v;
    if (u >= b->dist_len || du != b->dist[u]) continue;
    nbr_it it;
    out_it(b->g, u, &it);
    while (it_next(&it, &v)) {
      if (v >= b->ws || !b->affected[v]) continue;
      uint32_t c = du + 1;
      if (c < b->dist[v]) {
        if (b->dist[v] == VXO_UNREACHABLE) ++b->reachable;
        b->dist[v] = c;
        heap_push(&b->heap, ((uint64_t)c << 32) | v);
      }
    }
  }
  b->queue.n = 0;
  for (size_t i = 0; i < b->affected_list.n; ++i) {
    uint32_t v = b->affected_list.v[i];
    uint32_t old = i < b->old_aff.n ? b->old_aff.v[i] : VXO_UNREACHABLE;
    if (v < b->dist_len && b->dist[v] != VXO_UNREACHABLE && b->dist[v] < old)
      vec_push(&b->queue, v);
  }
  propagate(b);
}

/* clear_workspace  bfs.hpp:321-330 */
static void clear_ws(vxo_bfs* b) {
  for (size_t i = 0; i < b->affected_list.n; ++i) {
    uint32_t v = b->affected_list.v[i];
    if (v < b->ws) b->affected[v] = 0;
  }
  for (size_t i = 0; i < b->touched.n; ++i) {
    uint32_t v = b->touched.v[i];
    if (v < b->ws) {
      b->lost[v] = 0;
      b->spc[v] = 0;
    }
  }
  b->touched.n = 0;
}

/* relax_edge  bfs.hpp:332-339 */
static void relax(vxo_bfs* b, uint32_t u, uint32_t v) {
  if (u >= b->dist_len || v >= b->dist_len || b->dist[u] == VXO_UNREACHABLE) return;
  if (b->dist[u] + 1 < b->dist[v]) {
    if (b->dist[v] == VXO_UNREACHABLE) ++b->reachable;
    b->dist[v] = b->dist[u] + 1;
    vec_push(&b->queue, v);
  }
}

/* apply  bfs.hpp:29-98 */
int vxo_bfs_apply(vxo_bfs* b, const uint32_t* src, const uint32_t* dst,
                  const uint8_t* add, size_t n) {
  vxo_graph* g = b->g;
  b->last_candidates = 0;
  b->last_affected = 0;
  b->last_full = 0;
  if (n == 0) return 0;
  ensure_ws(b, g->V);
  /* prepare_batch_workspace  bfs.hpp:189-204 */
  ks_reset(&b->seen, n);
  ks_reset(&b->del_keys, n);
  b->final_add.n = b->final_del.n = b->existing_del.n = 0;
  b->candidates.n = b->affected_list.n = b->old_aff.n = b->invalidate.n = 0;
  b->touched.n = 0;

  /* final-state dedupe, last op per normalised edge wins  bfs.hpp:38-50 */
  for (size_t k = n; k-- > 0;) {
    uint64_t key = edge_key(b, src[k], dst[k]);
    if (!ks_insert(&b->seen, key)) continue;
    if (add[k]) {
      pairs_push(&b->final_add, src[k], dst[k]);
    } else {
      pairs_push(&b->final_del, src[k], dst[k]);
      ks_insert(&b->del_keys, key);
    }
  }
  /* deletion candidates  bfs.hpp:52-63 */
  for (size_t i = 0; i < b->final_del.n; ++i) {
    uint32_t u = b->final_del.u[i], v = b->final_del.v[i];
    if (!vxo_graph_has_edge(g, u, v)) continue;
    pairs_push(&b->existing_del, u, v);
    if (is_sp(b, u, v)) vec_push(&b->candidates, v);
    if (!g->directed && is_sp(b, v, u)) vec_push(&b->candidates, u);
  }
  normalize_dirty(&b->candidates);
  b->last_candidates = b->candidates.n;

  int fallback = 0;
  if (b->candidates.n) fallback = !compute_affected_prebatch(b);

  /* apply_updates + resize  bfs.hpp:72-74 */
  vxo_graph_apply(g, src, dst, add, n);
  if (b->dist_len < g->V) dist_resize(b, g->V);
  ensure_ws(b, g->V);

  if (fallback) { /* bfs.hpp:76-81 */
    clear_ws(b);
    vxo_bfs_recompute(b);
    b->last_full = 1;
    return 0;
  }
  if (b->affected_list.n) { /* bfs.hpp:83-89 */
    for (size_t i = 0; i < b->affected_list.n; ++i) {
      uint32_t v = b->affected_list.v[i];
      vec_push(&b->old_aff, v < b->dist_len ? b->dist[v] : VXO_UNREACHABLE);
    }
    repair_affected(b);
  }
  /* insertion relax + propagation  bfs.hpp:91-96 */
  b->queue.n = 0;
  for (size_t i = 0; i < b->final_add.n; ++i) {
    relax(b, b->final_add.u[i], b->final_add.v[i]);
    if (!g->directed) relax(b, b->final_add.v[i], b->final_add.u[i]);
  }
  propagate(b);
  clear_ws(b);
  return 0;
}

size_t vxo_bfs_distances(const vxo_bfs* b, uint32_t* out, size_t cap) {
  size_t m = b->dist_len < cap ? b->dist_len : cap;
  if (out && m) memcpy(out, b->dist, m * sizeof(uint32_t));
  return b->dist_len;
}

size_t vxo_bfs_reachable_count(const vxo_bfs* b) { return b->reachable; }
size_t vxo_bfs_last_deletion_candidates(const vxo_bfs* b) { return b->last_candidates; }
size_t vxo_bfs_last_affected_vertices(const vxo_bfs* b) { return b->last_affected; }
int vxo_bfs_last_used_full_recompute(const vxo_bfs* b) { return b->last_full; }

/* bfs_distances  src/algorithms.cpp:11-27 */
int vxo_csr_bfs(const uint64_t* offsets, const uint32_t* cols, size_t V,
                uint32_t source, uint32_t* dist) {
  if (source >= V) return -1;
  for (size_t i = 0; i < V; ++i) dist[i] = VXO_UNREACHABLE;
  uint32_t* q = (uint32_t*)malloc(V * sizeof(uint32_t));
  size_t head = 0, tail = 0;
  dist[source] = 0;
  q[tail++] = source;
  while (head < tail) {
    uint32_t u = q[head++];
    for (uint64_t e = offsets[u]; e < offsets[u + 1]; ++e) {
      uint32_t v = cols[e];
      if (dist[v] == VXO_UNREACHABLE) {
        dist[v] = dist[u] + 1;
        q[tail++] = v;
      }
    }
  }
  free(q);
  return 0;
}
