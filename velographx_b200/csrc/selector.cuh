// Repair-vs-recompute selector state (features, MLP, heuristic fallback).
#pragma once

#include <cstddef>
#include <cstdint>
#include <cuda_runtime.h>

namespace vxh {

struct Bfs;

constexpr int kSelFeatures = 16;
constexpr int kSelParams = 64 * 16 + 64 + 64 * 64 + 64 + 2 * 64 + 2;  // 5,378

// Host-provided inputs of the feature kernel.
struct SelInputs {
  unsigned long long ops;    // ops in the batch
  unsigned long long edges;  // edge_count_directed before the batch
  uint32_t vertices;
  uint32_t levels;           // BFS depth of the last full BFS
  float reachable_fraction;
  float prev_affected_fraction;
};

struct Selector {
  float* params = nullptr;
  float* adam_m = nullptr;
  float* adam_v = nullptr;
  float* grad = nullptr;
  float* scalar = nullptr;
  cudaStream_t stream = nullptr;
};

int selector_create(Selector** out, uint64_t seed);
void selector_destroy(Selector* s);
int selector_train(Selector* s, const float* X, const float* Y, size_t n, uint32_t epochs, uint32_t batch, float lr,
                   uint32_t seed, float* loss);
int selector_gradients(Selector* s, const float* X, const float* Y, size_t n, float* grad, float* loss);
int selector_predict(Selector* s, const float* X, size_t n, float* Y);
int selector_set_params(Selector* s, const float* p);
int selector_get_params(Selector* s, float* p);
// Features of the batch staged on b's graph (pre-batch state); synchronises.
int batch_features(Bfs* b, size_t n, const SelInputs& in, float* host16);

// The reference's adaptive selector state (publication_policy_bfs.cpp:78-95).
struct HeuristicState {
  bool large_scale = false;
  bool first_batch = true;
  double initial_reachable_fraction = 0.0;
  double previous_affected_fraction = 0.0;
  double ema_incremental_us = 0.0, ema_full_us = 0.0;
  double last_incremental_update_fraction = 0.0;
  double ema_incremental_rel_error = 0.0, ema_full_rel_error = 0.0;
  bool have_incremental_error = false, have_full_error = false;
  bool have_incremental = false, have_full = true;
  size_t incremental_age = 5, full_age = 0;
  double update_fraction = 0.0;
  double predicted_incremental_us = 0.0, predicted_full_us = 0.0;
};

bool heuristic_decide(HeuristicState& h, double update_fraction, double shallow_fraction);
void heuristic_observe(HeuristicState& h, bool observed_full, double execution_us, double affected_fraction);

}  // namespace vxh
