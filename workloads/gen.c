/*
 * Seeded synthetic graph generators for the benchmarks and tests (host code,
 * multi-threaded).  Not part of the product library: the bench's reference
 * arm and the tests load this file's shared object without loading the GPU
 * library.
 *
 * Every edge is a pure function of (seed, edge index), so the output does not
 * depend on the thread count.  R-MAT follows the Graph500-style recursive
 * quadrant choice with initiator (a, b, c, 1-a-b-c) and no vertex permutation,
 * matching in distribution the reference's publication generator
 * (scripts/prepare_publication_datasets.py:80-111).
 *
 * Outputs are (u, v) pairs, row-major; self-loops and duplicates are kept (the
 * graph loaders drop them, as DynamicGraph::bulk_load_edges does).
 */
#include <pthread.h>
#include <stdint.h>
#include <stdlib.h>
#include <unistd.h>

static inline uint64_t mix64(uint64_t x) { /* splitmix64 finaliser */
  x += 0x9E3779B97F4A7C15ull;
  x = (x ^ (x >> 30)) * 0xBF58476D1CE4E5B9ull;
  x = (x ^ (x >> 27)) * 0x94D049BB133111EBull;
  return x ^ (x >> 31);
}

static inline double unit01(uint64_t x) { return (double)(x >> 11) * (1.0 / 9007199254740992.0); }

typedef struct {
  int kind; /* 0 rmat, 1 uniform, 2 lattice */
  uint64_t lo, hi;
  uint32_t* out;
  /* rmat */
  uint32_t scale;
  double a, ab, abc;
  uint64_t s0;
  /* uniform */
  uint32_t vertices;
  /* lattice */
  uint64_t cols, horiz;
} job_t;

static void rmat_range(const job_t* j) {
  for (uint64_t i = j->lo; i < j->hi; ++i) {
    uint32_t u = 0, v = 0;
    const uint64_t base = mix64(j->s0 + i);
    for (uint32_t l = 0; l < j->scale; ++l) {
      const double r = unit01(mix64(base + 0xD1B54A32D192ED03ull * (l + 1)));
      const uint32_t bu = r >= j->ab ? 1u : 0u;
      const uint32_t bv = ((r >= j->a && r < j->ab) || r >= j->abc) ? 1u : 0u;
      u = (u << 1) | bu;
      v = (v << 1) | bv;
    }
    j->out[2 * i] = u;
    j->out[2 * i + 1] = v;
  }
}

static void uniform_range(const job_t* j) {
  for (uint64_t i = j->lo; i < j->hi; ++i) {
    const uint64_t h = mix64(j->s0 + i);
    j->out[2 * i] = (uint32_t)(((h & 0xFFFFFFFFull) * j->vertices) >> 32);
    j->out[2 * i + 1] = (uint32_t)(((h >> 32) * j->vertices) >> 32);
  }
}

static void lattice_range(const job_t* j) {
  for (uint64_t i = j->lo; i < j->hi; ++i) {
    uint32_t u, v;
    if (i < j->horiz) {
      const uint64_t r = i / (j->cols - 1), c = i % (j->cols - 1);
      u = (uint32_t)(r * j->cols + c);
      v = u + 1;
    } else {
      u = (uint32_t)(i - j->horiz);
      v = (uint32_t)(i - j->horiz + j->cols);
    }
    j->out[2 * i] = u;
    j->out[2 * i + 1] = v;
  }
}

static void* run_job(void* arg) {
  const job_t* j = (const job_t*)arg;
  if (j->kind == 0) rmat_range(j);
  else if (j->kind == 1) uniform_range(j);
  else lattice_range(j);
  return NULL;
}

/* Splits [0, n) over up to 64 threads (one below 65,536 items). */
static void parallel_run(const job_t* proto, uint64_t n) {
  long hw = sysconf(_SC_NPROCESSORS_ONLN);
  unsigned t = hw < 1 ? 1u : (hw > 64 ? 64u : (unsigned)hw);
  if (n < 65536) t = 1;
  job_t jobs[64];
  pthread_t th[64];
  int started[64] = {0};
  const uint64_t chunk = (n + t - 1) / t;
  for (unsigned k = 0; k < t; ++k) {
    jobs[k] = *proto;
    jobs[k].lo = k * chunk;
    jobs[k].hi = jobs[k].lo + chunk < n ? jobs[k].lo + chunk : n;
    if (jobs[k].lo >= jobs[k].hi) break;
    started[k] = t > 1 && pthread_create(&th[k], NULL, run_job, &jobs[k]) == 0;
    if (!started[k]) run_job(&jobs[k]);
  }
  for (unsigned k = 0; k < t; ++k)
    if (started[k]) pthread_join(th[k], NULL);
}

int vxg_rmat(uint32_t scale, uint32_t edge_factor, double a, double b, double c, uint64_t seed, uint32_t* uv_out) {
  if (!uv_out || scale == 0 || scale > 31 || a < 0 || b < 0 || c < 0 || a + b + c > 1.0) return -1;
  job_t j = {0};
  j.kind = 0;
  j.out = uv_out;
  j.scale = scale;
  j.a = a;
  j.ab = a + b;
  j.abc = a + b + c;
  j.s0 = mix64(seed ^ 0x5241544D524D4154ull);
  parallel_run(&j, (uint64_t)edge_factor << scale);
  return 0;
}

int vxg_uniform(uint32_t vertices, uint64_t n, uint64_t seed, uint32_t* uv_out) {
  if (!uv_out || vertices == 0) return -1;
  job_t j = {0};
  j.kind = 1;
  j.out = uv_out;
  j.vertices = vertices;
  j.s0 = mix64(seed ^ 0x554E49464F524D31ull);
  parallel_run(&j, n);
  return 0;
}

uint64_t vxg_grid_edge_count(uint32_t rows, uint32_t cols, uint64_t extra) {
  return (uint64_t)rows * (cols - 1) + (uint64_t)(rows - 1) * cols + extra;
}

int vxg_grid(uint32_t rows, uint32_t cols, uint64_t extra, uint64_t seed, uint32_t* uv_out) {
  if (!uv_out || rows == 0 || cols == 0 || (uint64_t)rows * cols > 0x7FFFFFFFull) return -1;
  job_t j = {0};
  j.kind = 2;
  j.out = uv_out;
  j.cols = cols;
  j.horiz = (uint64_t)rows * (cols - 1);
  parallel_run(&j, j.horiz + (uint64_t)(rows - 1) * cols);
  if (extra) vxg_uniform(rows * cols, extra, seed, uv_out + 2 * vxg_grid_edge_count(rows, cols, 0));
  return 0;
}
