// Seeded synthetic graph generators (host code, multi-threaded).
//
// Every edge is a pure function of (seed, edge index), so the output does not
// depend on the thread count.  R-MAT follows the Graph500-style recursive
// quadrant choice with initiator (a, b, c, 1-a-b-c) and no vertex permutation,
// matching in distribution the reference's publication generator
// (scripts/prepare_publication_datasets.py:80-111).
#include <algorithm>
#include <cstdint>
#include <thread>
#include <vector>

#include "../../include/vx_workloads.h"

namespace {

inline uint64_t mix64(uint64_t x) {  // splitmix64 finaliser
  x += 0x9E3779B97F4A7C15ull;
  x = (x ^ (x >> 30)) * 0xBF58476D1CE4E5B9ull;
  x = (x ^ (x >> 27)) * 0x94D049BB133111EBull;
  return x ^ (x >> 31);
}

inline double unit(uint64_t x) { return (double)(x >> 11) * (1.0 / 9007199254740992.0); }

template <class Fn>
void parallel_for(uint64_t n, Fn fn) {
  unsigned t = std::max(1u, std::min(64u, std::thread::hardware_concurrency()));
  if (n < 65536) t = 1;
  std::vector<std::thread> pool;
  const uint64_t chunk = (n + t - 1) / t;
  for (unsigned k = 0; k < t; ++k) {
    const uint64_t lo = k * chunk, hi = std::min(n, lo + chunk);
    if (lo >= hi) break;
    pool.emplace_back([=] {
      for (uint64_t i = lo; i < hi; ++i) fn(i);
    });
  }
  for (auto& th : pool) th.join();
}

}  // namespace

extern "C" {

int vx_gen_rmat(uint32_t scale, uint32_t edge_factor, double a, double b, double c, uint64_t seed,
                uint32_t* uv_out) {
  if (!uv_out || scale == 0 || scale > 31 || a < 0 || b < 0 || c < 0 || a + b + c > 1.0) return -1;
  const uint64_t n = (uint64_t)edge_factor << scale;
  const double ab = a + b, abc = a + b + c;
  const uint64_t s0 = mix64(seed ^ 0x5241544D524D4154ull);
  parallel_for(n, [&](uint64_t i) {
    uint32_t u = 0, v = 0;
    const uint64_t base = mix64(s0 + i);
    for (uint32_t l = 0; l < scale; ++l) {
      const double r = unit(mix64(base + 0xD1B54A32D192ED03ull * (l + 1)));
      const uint32_t bu = r >= ab ? 1u : 0u;
      const uint32_t bv = (r >= a && r < ab) || r >= abc ? 1u : 0u;
      u = (u << 1) | bu;
      v = (v << 1) | bv;
    }
    uv_out[2 * i] = u;
    uv_out[2 * i + 1] = v;
  });
  return 0;
}

int vx_gen_uniform(uint32_t vertices, uint64_t n, uint64_t seed, uint32_t* uv_out) {
  if (!uv_out || vertices == 0) return -1;
  const uint64_t s0 = mix64(seed ^ 0x554E49464F524D31ull);
  parallel_for(n, [&](uint64_t i) {
    const uint64_t h = mix64(s0 + i);
    uv_out[2 * i] = (uint32_t)(((h & 0xFFFFFFFFull) * vertices) >> 32);
    uv_out[2 * i + 1] = (uint32_t)(((h >> 32) * vertices) >> 32);
  });
  return 0;
}

int vx_gen_grid(uint32_t rows, uint32_t cols, uint64_t extra, uint64_t seed, uint32_t* uv_out) {
  if (!uv_out || rows == 0 || cols == 0 || (uint64_t)rows * cols > 0x7FFFFFFFull) return -1;
  const uint64_t horiz = (uint64_t)rows * (cols - 1), vert = (uint64_t)(rows - 1) * cols;
  parallel_for(horiz + vert, [&](uint64_t i) {
    uint32_t u, v;
    if (i < horiz) {
      const uint64_t r = i / (cols - 1), cidx = i % (cols - 1);
      u = (uint32_t)(r * cols + cidx);
      v = u + 1;
    } else {
      const uint64_t j = i - horiz;
      u = (uint32_t)j;
      v = (uint32_t)(j + cols);
    }
    uv_out[2 * i] = u;
    uv_out[2 * i + 1] = v;
  });
  if (extra) vx_gen_uniform(rows * cols, extra, seed, uv_out + 2 * (horiz + vert));
  return 0;
}

uint64_t vx_gen_grid_edge_count(uint32_t rows, uint32_t cols, uint64_t extra) {
  return (uint64_t)rows * (cols - 1) + (uint64_t)(rows - 1) * cols + extra;
}

}  // extern "C"
