// Repair-vs-recompute selector: batch features, a 16-64-64-2 MLP trained and
// evaluated by the project's own kernels, and the reference's hand-tuned
// heuristic as the fallback.
//
// The reference picks the arm outside the library, in its benchmark harnesses
// (benchmarks/publication_policy_bfs.cpp:163-235 decision, :285-320 EMA
// updates, benchmarks/adaptive_policy_bfs.cpp:21-31 constants).  Here the
// features come straight from the staged batch on the device (the same pass
// that classifies every canonical arc), the network predicts log execution
// time of both arms, and the cheaper arm runs.  Both arms are exact, so a
// wrong choice costs time, never correctness.
//
// MLP parameter layout (fp32, kParams = 5,378):
//   W1[64][16] b1[64] W2[64][64] b2[64] W3[2][64] b3[2]
// Targets are standardised log(us) of (repair, full).
#include <cmath>
#include <cstring>

#include "bfs.cuh"
#include "selector.cuh"

namespace vxh {

namespace {

constexpr int kIn = kSelFeatures, kH = 64, kOut = 2;
constexpr int oW1 = 0, oB1 = oW1 + kH * kIn, oW2 = oB1 + kH, oB2 = oW2 + kH * kH, oW3 = oB2 + kH,
              oB3 = oW3 + kOut * kH;
static_assert(oB3 + kOut == kSelParams, "parameter layout");

// ------------------------------------------------------------ features --

// One CTA of 1024 threads reduces over the F canonical arcs of the staged
// batch (pre-batch distances, current degrees).
__global__ void __launch_bounds__(1024) features_kernel(vxb::DevAdj a, const uint32_t* fu, const uint32_t* fv,
                                                        const uint8_t* ff, const uint32_t* count,
                                                        const uint32_t* dist, uint32_t dist_len, SelInputs in,
                                                        float* out) {
  __shared__ float red[32][11];
  const uint32_t F = *count;
  float s[8] = {0, 0, 0, 0, 0, 0, 0, 0};
  float mxdeg = 0.f, mxdepth = 0.f, mndepth = 1e30f;
  const float depth = (float)(in.levels + 1);
  for (uint32_t i = threadIdx.x; i < F; i += blockDim.x) {
    const uint32_t u = fu[i], v = fv[i];
    const uint8_t f = ff[i];
    const bool add = f & kFAdd, cur = f & kFCur;
    const uint32_t du = u < dist_len ? dist[u] : vxb::kUnreachable;
    const uint32_t dv = v < dist_len ? dist[v] : vxb::kUnreachable;
    uint64_t b, e;
    vxb::base_range(a, v, b, e);
    const float lg = log2f(1.0f + (float)(e - b) + (float)a.drow[v].y);
    s[7] += lg;
    mxdeg = fmaxf(mxdeg, lg);
    if (!add) {
      s[0] += 1.f;  // final deletions
      if (cur) {
        s[1] += 1.f;  // existing deletions
        if (du != vxb::kUnreachable && dv != vxb::kUnreachable && du + 1 == dv) {
          s[2] += 1.f;  // shortest-parent (tree) deletions
          if (dv <= 3) s[3] += 1.f;  // shallow, as kShallowDeletionDepth (adaptive_policy_bfs.cpp:28)
          s[4] += (float)dv / depth;
          s[5] += lg;
          mndepth = fminf(mndepth, (float)dv / depth);
          mxdepth = fmaxf(mxdepth, (float)dv / depth);
        }
      }
    } else if (du != vxb::kUnreachable) {
      if (dv == vxb::kUnreachable) s[6] += 1.f;  // insertion reaches an unreachable vertex
      else if (du + 1 < dv) s[6] += 0.5f;       // insertion shortens a path
    }
  }
  // block reduction
  float vals[11] = {s[0], s[1], s[2], s[3], s[4], s[5], s[6], s[7], mxdeg, mxdepth, mndepth};
#pragma unroll
  for (int k = 0; k < 11; ++k) {
    float x = vals[k];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
      const float y = __shfl_xor_sync(0xFFFFFFFFu, x, o);
      x = k < 8 ? x + y : (k == 10 ? fminf(x, y) : fmaxf(x, y));
    }
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5][k] = x;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    float t[11];
    for (int k = 0; k < 11; ++k) t[k] = red[0][k];
    for (int w = 1; w < (int)(blockDim.x >> 5); ++w)
      for (int k = 0; k < 11; ++k)
        t[k] = k < 8 ? t[k] + red[w][k] : (k == 10 ? fminf(t[k], red[w][k]) : fmaxf(t[k], red[w][k]));
    const float Fn = fmaxf(1.f, (float)F);
    const float trees = fmaxf(1.f, t[2]);
    out[0] = log1pf((float)in.ops) / 16.f;
    out[1] = log1pf(1000.f * (float)in.ops / fmaxf(1.f, (float)in.edges)) / 10.f;
    out[2] = t[0] / Fn;
    out[3] = t[1] / Fn;
    out[4] = t[2] / Fn;
    out[5] = t[3] / Fn;
    out[6] = t[2] > 0.f ? t[4] / trees : 0.f;
    out[7] = t[2] > 0.f ? t[10] : 1.f;
    out[8] = t[9];
    out[9] = t[6] / Fn;
    out[10] = t[2] > 0.f ? t[5] / trees / 32.f : 0.f;
    out[11] = t[8] / 32.f;
    out[12] = t[7] / Fn / 32.f;
    out[13] = in.reachable_fraction;
    out[14] = in.prev_affected_fraction;
    out[15] = log2f(1.f + (float)in.edges) / 32.f;  // graph size; grows with the stream
  }
}

// ------------------------------------------------------------------ MLP --

// Forward pass of one sample by one warp (64 hidden units: 2 per lane).
__device__ void mlp_forward_warp(const float* P, const float* x, float* h1, float* h2, float* y) {
  const int lane = threadIdx.x & 31;
  for (int j = lane; j < kH; j += 32) {
    float acc = P[oB1 + j];
#pragma unroll
    for (int k = 0; k < kIn; ++k) acc += P[oW1 + j * kIn + k] * x[k];
    h1[j] = fmaxf(acc, 0.f);
  }
  __syncwarp();
  for (int j = lane; j < kH; j += 32) {
    float acc = P[oB2 + j];
    for (int k = 0; k < kH; ++k) acc += P[oW2 + j * kH + k] * h1[k];
    h2[j] = fmaxf(acc, 0.f);
  }
  __syncwarp();
  for (int o = 0; o < kOut; ++o) {
    float acc = 0.f;
    for (int k = lane; k < kH; k += 32) acc += P[oW3 + o * kH + k] * h2[k];
#pragma unroll
    for (int s = 16; s > 0; s >>= 1) acc += __shfl_xor_sync(0xFFFFFFFFu, acc, s);
    if (lane == 0) y[o] = acc + P[oB3 + o];
  }
  __syncwarp();
}

// Inference for n samples: one warp per sample.
__global__ void mlp_predict_kernel(const float* P, const float* X, uint32_t n, float* Y) {
  __shared__ float buf[8][2 * kH + kIn];
  __shared__ float out[8][kOut];
  const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
  for (uint32_t i = blockIdx.x * (blockDim.x >> 5) + w; i < n; i += gridDim.x * (blockDim.x >> 5)) {
    float* x = buf[w] + 2 * kH;
    for (int k = lane; k < kIn; k += 32) x[k] = X[i * kIn + k];
    __syncwarp();
    mlp_forward_warp(P, x, buf[w], buf[w] + kH, out[w]);
    if (lane < kOut) Y[i * kOut + lane] = out[w][lane];
    __syncwarp();
  }
}

// Gradients of the mean squared error over a minibatch, one CTA of 256
// threads.  P, G in global memory; activations staged in shared memory.
constexpr int kTrainThreads = 256;
constexpr int kMaxBatch = 64;

struct TrainSmem {
  float x[kMaxBatch][kIn];
  float h1[kMaxBatch][kH];
  float h2[kMaxBatch][kH];
  float dy[kMaxBatch][kOut];
  float d2[kMaxBatch][kH];
  float d1[kMaxBatch][kH];
};

__device__ float batch_grad(const float* P, const float* X, const float* Y, const uint32_t* idx, int B, float* G,
                            TrainSmem& sm) {
  const int t = threadIdx.x;
  for (int i = t; i < B * kIn; i += kTrainThreads) sm.x[i / kIn][i % kIn] = X[idx[i / kIn] * kIn + i % kIn];
  __syncthreads();
  for (int i = t; i < B * kH; i += kTrainThreads) {
    const int s = i / kH, j = i % kH;
    float acc = P[oB1 + j];
#pragma unroll
    for (int k = 0; k < kIn; ++k) acc += P[oW1 + j * kIn + k] * sm.x[s][k];
    sm.h1[s][j] = fmaxf(acc, 0.f);
  }
  __syncthreads();
  for (int i = t; i < B * kH; i += kTrainThreads) {
    const int s = i / kH, j = i % kH;
    float acc = P[oB2 + j];
    for (int k = 0; k < kH; ++k) acc += P[oW2 + j * kH + k] * sm.h1[s][k];
    sm.h2[s][j] = fmaxf(acc, 0.f);
  }
  __syncthreads();
  __shared__ float loss_part[kTrainThreads];
  float lsum = 0.f;
  for (int i = t; i < B * kOut; i += kTrainThreads) {
    const int s = i / kOut, o = i % kOut;
    float acc = P[oB3 + o];
    for (int k = 0; k < kH; ++k) acc += P[oW3 + o * kH + k] * sm.h2[s][k];
    const float d = acc - Y[idx[s] * kOut + o];
    lsum += d * d;
    sm.dy[s][o] = 2.f * d / (float)(B * kOut);
  }
  loss_part[t] = lsum;
  __syncthreads();
  // d2 = W3^T dy * relu'(h2)
  for (int i = t; i < B * kH; i += kTrainThreads) {
    const int s = i / kH, j = i % kH;
    float acc = 0.f;
#pragma unroll
    for (int o = 0; o < kOut; ++o) acc += P[oW3 + o * kH + j] * sm.dy[s][o];
    sm.d2[s][j] = sm.h2[s][j] > 0.f ? acc : 0.f;
  }
  __syncthreads();
  // d1 = W2^T d2 * relu'(h1)
  for (int i = t; i < B * kH; i += kTrainThreads) {
    const int s = i / kH, k = i % kH;
    float acc = 0.f;
    for (int j = 0; j < kH; ++j) acc += P[oW2 + j * kH + k] * sm.d2[s][j];
    sm.d1[s][k] = sm.h1[s][k] > 0.f ? acc : 0.f;
  }
  __syncthreads();
  // parameter gradients (sums over the minibatch)
  for (int p = t; p < kSelParams; p += kTrainThreads) {
    float g = 0.f;
    if (p < oB1) {
      const int j = p / kIn, k = p % kIn;
      for (int s = 0; s < B; ++s) g += sm.d1[s][j] * sm.x[s][k];
    } else if (p < oW2) {
      const int j = p - oB1;
      for (int s = 0; s < B; ++s) g += sm.d1[s][j];
    } else if (p < oB2) {
      const int j = (p - oW2) / kH, k = (p - oW2) % kH;
      for (int s = 0; s < B; ++s) g += sm.d2[s][j] * sm.h1[s][k];
    } else if (p < oW3) {
      const int j = p - oB2;
      for (int s = 0; s < B; ++s) g += sm.d2[s][j];
    } else if (p < oB3) {
      const int o = (p - oW3) / kH, k = (p - oW3) % kH;
      for (int s = 0; s < B; ++s) g += sm.dy[s][o] * sm.h2[s][k];
    } else {
      const int o = p - oB3;
      for (int s = 0; s < B; ++s) g += sm.dy[s][o];
    }
    G[p] = g;
  }
  __syncthreads();
  if (t == 0) {
    float l = 0.f;
    for (int i = 0; i < kTrainThreads; ++i) l += loss_part[i];
    loss_part[0] = l / (float)(B * kOut);
  }
  __syncthreads();
  const float loss = loss_part[0];
  __syncthreads();
  return loss;
}

__global__ void __launch_bounds__(kTrainThreads) mlp_grad_kernel(const float* P, const float* X, const float* Y,
                                                                 const uint32_t* idx, int B, float* G, float* loss) {
  extern __shared__ __align__(16) unsigned char raw[];
  TrainSmem& sm = *reinterpret_cast<TrainSmem*>(raw);
  const float l = batch_grad(P, X, Y, idx, B, G, sm);
  if (threadIdx.x == 0) *loss = l;
}

__device__ __forceinline__ uint32_t lcg(uint32_t& s) {
  s = s * 1664525u + 1013904223u;
  return s;
}

// Adam over shuffled minibatches for `epochs` passes; one CTA.
__global__ void __launch_bounds__(kTrainThreads) mlp_train_kernel(float* P, float* M, float* Vv, float* G,
                                                                  const float* X, const float* Y, uint32_t n,
                                                                  uint32_t* perm, uint32_t epochs, int B, float lr,
                                                                  uint32_t seed, float* loss_out) {
  extern __shared__ __align__(16) unsigned char raw[];
  TrainSmem& sm = *reinterpret_cast<TrainSmem*>(raw);
  const int t = threadIdx.x;
  const float b1 = 0.9f, b2 = 0.999f, eps = 1e-8f;
  uint32_t step = 0;
  float last = 0.f;
  for (uint32_t i = t; i < n; i += kTrainThreads) perm[i] = i;
  __syncthreads();
  for (uint32_t ep = 0; ep < epochs; ++ep) {
    if (t == 0) {  // Fisher-Yates shuffle with a fixed-seed LCG
      uint32_t s = seed ^ (ep * 2654435761u);
      for (uint32_t i = n - 1; i > 0; --i) {
        const uint32_t j = lcg(s) % (i + 1);
        const uint32_t tmp = perm[i];
        perm[i] = perm[j];
        perm[j] = tmp;
      }
    }
    __syncthreads();
    float ep_loss = 0.f;
    uint32_t nb = 0;
    for (uint32_t base = 0; base < n; base += B) {
      const int bs = (int)min((uint32_t)B, n - base);
      const float l = batch_grad(P, X, Y, perm + base, bs, G, sm);
      ep_loss += l;
      ++nb;
      ++step;
      const float c1 = 1.f - powf(b1, (float)step), c2 = 1.f - powf(b2, (float)step);
      for (int p = t; p < kSelParams; p += kTrainThreads) {
        const float g = G[p];
        M[p] = b1 * M[p] + (1.f - b1) * g;
        Vv[p] = b2 * Vv[p] + (1.f - b2) * g * g;
        P[p] -= lr * (M[p] / c1) / (sqrtf(Vv[p] / c2) + eps);
      }
      __syncthreads();
    }
    last = ep_loss / (float)max(nb, 1u);
  }
  if (t == 0) *loss_out = last;
}

}  // namespace

// ---------------------------------------------------------------- host --

int selector_create(Selector** out, uint64_t seed) {
  Selector* s = new Selector();
  if (cudaMalloc(&s->params, kSelParams * 4) != cudaSuccess || cudaMalloc(&s->adam_m, kSelParams * 4) != cudaSuccess ||
      cudaMalloc(&s->adam_v, kSelParams * 4) != cudaSuccess || cudaMalloc(&s->grad, kSelParams * 4) != cudaSuccess ||
      cudaMalloc(&s->scalar, 64) != cudaSuccess ||
      cudaStreamCreateWithFlags(&s->stream, cudaStreamNonBlocking) != cudaSuccess) {
    set_error("selector allocation failed");
    selector_destroy(s);
    return -4;
  }
  // He-style uniform initialisation from a fixed-seed splitmix stream
  float* h = new float[kSelParams];
  uint64_t st = seed ^ 0x53454C4543544F52ull;
  auto next = [&]() {
    st += 0x9E3779B97F4A7C15ull;
    uint64_t z = st;
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    z ^= z >> 31;
    return (float)((z >> 11) * (1.0 / 9007199254740992.0)) * 2.f - 1.f;
  };
  for (int i = 0; i < kSelParams; ++i) h[i] = 0.f;
  for (int i = oW1; i < oB1; ++i) h[i] = next() * std::sqrt(6.f / kIn);
  for (int i = oW2; i < oB2; ++i) h[i] = next() * std::sqrt(6.f / kH);
  for (int i = oW3; i < oB3; ++i) h[i] = next() * std::sqrt(3.f / kH);
  // uploads and fills go on the selector's (non-blocking) stream, ahead of its
  // kernels; the copy from pageable memory is staged before this returns
  cudaError_t e = cudaMemcpyAsync(s->params, h, kSelParams * 4, cudaMemcpyHostToDevice, s->stream);
  if (e == cudaSuccess) e = cudaMemsetAsync(s->adam_m, 0, kSelParams * 4, s->stream);
  if (e == cudaSuccess) e = cudaMemsetAsync(s->adam_v, 0, kSelParams * 4, s->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(s->stream);
  delete[] h;
  if (e != cudaSuccess) {
    set_error("selector initialisation failed");
    selector_destroy(s);
    return -3;
  }
  *out = s;
  return 0;
}

void selector_destroy(Selector* s) {
  if (!s) return;
  cudaFree(s->params);
  cudaFree(s->adam_m);
  cudaFree(s->adam_v);
  cudaFree(s->grad);
  cudaFree(s->scalar);
  if (s->stream) cudaStreamDestroy(s->stream);
  delete s;
}

// Device copy of a host array, ordered on `stream` before the kernels that read it.
static int upload(const void* host, size_t bytes, void** dev, cudaStream_t stream) {
  if (cudaMalloc(dev, bytes ? bytes : 4) != cudaSuccess) {
    set_error("selector staging allocation failed");
    return -4;
  }
  if (bytes && host) {
    const cudaError_t e = cudaMemcpyAsync(*dev, host, bytes, cudaMemcpyHostToDevice, stream);
    if (e != cudaSuccess) {
      set_error("selector staging copy failed: %s", cudaGetErrorString(e));
      cudaFree(*dev);
      *dev = nullptr;
      return -3;
    }
  }
  return 0;
}

int selector_train(Selector* s, const float* X, const float* Y, size_t n, uint32_t epochs, uint32_t batch, float lr,
                   uint32_t seed, float* loss) {
  if (n == 0 || batch == 0 || batch > (uint32_t)kMaxBatch) {
    set_error("training needs n > 0 and 1 <= batch <= %d", kMaxBatch);
    return -1;
  }
  void *dx = nullptr, *dy = nullptr, *perm = nullptr;
  int rc = upload(X, n * kIn * 4, &dx, s->stream);
  if (!rc) rc = upload(Y, n * kOut * 4, &dy, s->stream);
  if (!rc) rc = upload(nullptr, n * 4, &perm, s->stream);
  if (!rc) {
    static bool attr = false;
    if (!attr) {
      cudaFuncSetAttribute(mlp_train_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sizeof(TrainSmem));
      attr = true;
    }
    count_launch();
    mlp_train_kernel<<<1, kTrainThreads, sizeof(TrainSmem), s->stream>>>(
        s->params, s->adam_m, s->adam_v, s->grad, (const float*)dx, (const float*)dy, (uint32_t)n,
        (uint32_t*)perm, epochs, (int)batch, lr, seed, s->scalar);
    if (cudaGetLastError() != cudaSuccess || cudaStreamSynchronize(s->stream) != cudaSuccess) {
      set_error("selector training kernel failed");
      rc = -3;
    } else if (loss) {
      cudaMemcpy(loss, s->scalar, 4, cudaMemcpyDeviceToHost);
    }
  }
  cudaFree(dx);
  cudaFree(dy);
  cudaFree(perm);
  return rc;
}

int selector_gradients(Selector* s, const float* X, const float* Y, size_t n, float* grad, float* loss) {
  if (n == 0 || n > (size_t)kMaxBatch) {
    set_error("gradients take 1..%d samples", kMaxBatch);
    return -1;
  }
  uint32_t idx[kMaxBatch];
  for (size_t i = 0; i < n; ++i) idx[i] = (uint32_t)i;
  void *dx = nullptr, *dy = nullptr, *di = nullptr;
  int rc = upload(X, n * kIn * 4, &dx, s->stream);
  if (!rc) rc = upload(Y, n * kOut * 4, &dy, s->stream);
  if (!rc) rc = upload(idx, n * 4, &di, s->stream);
  if (!rc) {
    static bool attr = false;
    if (!attr) {
      cudaFuncSetAttribute(mlp_grad_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sizeof(TrainSmem));
      attr = true;
    }
    count_launch();
    mlp_grad_kernel<<<1, kTrainThreads, sizeof(TrainSmem), s->stream>>>(
        s->params, (const float*)dx, (const float*)dy, (const uint32_t*)di, (int)n, s->grad, s->scalar);
    if (cudaGetLastError() != cudaSuccess || cudaStreamSynchronize(s->stream) != cudaSuccess) {
      set_error("selector gradient kernel failed");
      rc = -3;
    } else {
      cudaMemcpy(grad, s->grad, kSelParams * 4, cudaMemcpyDeviceToHost);
      if (loss) cudaMemcpy(loss, s->scalar, 4, cudaMemcpyDeviceToHost);
    }
  }
  cudaFree(dx);
  cudaFree(dy);
  cudaFree(di);
  return rc;
}

int selector_predict(Selector* s, const float* X, size_t n, float* Y) {
  void *dx = nullptr, *dy = nullptr;
  int rc = upload(X, n * kIn * 4, &dx, s->stream);
  if (!rc) rc = upload(nullptr, n * kOut * 4, &dy, s->stream);
  if (!rc && n) {
    count_launch();
    const unsigned blocks = (unsigned)std::min<size_t>((n + 7) / 8, 1024);
    mlp_predict_kernel<<<blocks, 256, 0, s->stream>>>(s->params, (const float*)dx, (uint32_t)n, (float*)dy);
    if (cudaGetLastError() != cudaSuccess || cudaStreamSynchronize(s->stream) != cudaSuccess) {
      set_error("selector inference kernel failed");
      rc = -3;
    } else {
      cudaMemcpy(Y, dy, n * kOut * 4, cudaMemcpyDeviceToHost);
    }
  }
  cudaFree(dx);
  cudaFree(dy);
  return rc;
}

int selector_set_params(Selector* s, const float* p) {
  VX_CUDA_TRY(cudaMemcpyAsync(s->params, p, kSelParams * 4, cudaMemcpyHostToDevice, s->stream));
  VX_CUDA_TRY(cudaMemsetAsync(s->adam_m, 0, kSelParams * 4, s->stream));
  VX_CUDA_TRY(cudaMemsetAsync(s->adam_v, 0, kSelParams * 4, s->stream));
  VX_CUDA_TRY(cudaStreamSynchronize(s->stream));
  return 0;
}

int selector_get_params(Selector* s, float* p) {
  VX_CUDA_TRY(cudaMemcpyAsync(p, s->params, kSelParams * 4, cudaMemcpyDeviceToHost, s->stream));
  VX_CUDA_TRY(cudaStreamSynchronize(s->stream));
  return 0;
}

int batch_features(Bfs* b, size_t n, const SelInputs& in, float* host16) {
  Graph* g = b->g;
  cudaStream_t st = g->stream;
  float* d = reinterpret_cast<float*>(b->features);
  count_launch();
  features_kernel<<<1, 1024, 0, st>>>(g->view().out, g->batch.fu, g->batch.fv, g->batch.ff, &g->ctr->final_arcs,
                                      b->dist, (uint32_t)b->dist_len, in, d);
  VX_CUDA_TRY(cudaGetLastError());
  VX_CUDA_TRY(cudaMemcpyAsync(host16, d, kSelFeatures * 4, cudaMemcpyDeviceToHost, st));
  VX_CUDA_TRY(cudaStreamSynchronize(st));
  (void)n;
  return 0;
}

// ------------------------------------------------------------ heuristic --
// The reference's adaptive selector (publication_policy_bfs.cpp:163-235,
// EMA updates :285-320; constants adaptive_policy_bfs.cpp:21-31).

bool heuristic_decide(HeuristicState& h, double update_fraction, double shallow_fraction) {
  const double kPreflightFullUpdate = 0.05, kVerySparseReach = 0.02, kSparseReach = 0.20,
               kSparseReachFullUpdate = 0.0025, kLearnedFullMargin = 1.25;
  const size_t kFreshAge = 4;
  h.update_fraction = update_fraction;
  if (h.large_scale) {
    const double normalized = h.have_incremental
                                  ? std::sqrt((update_fraction + 1e-12) / (h.last_incremental_update_fraction + 1e-12))
                                  : 1.0;
    const double bounded = std::min(2.5, std::max(0.5, normalized));
    const double pred_inc = h.have_incremental ? h.ema_incremental_us * bounded * (1.0 + 3.0 * h.previous_affected_fraction)
                                               : 0.0;
    const double pred_full = h.ema_full_us;
    const double inc_unc = h.have_incremental_error ? std::min(0.35, std::max(0.05, h.ema_incremental_rel_error)) : 0.35;
    const double full_unc = h.have_full_error ? std::min(0.35, std::max(0.05, h.ema_full_rel_error)) : 0.20;
    h.predicted_incremental_us = pred_inc;
    h.predicted_full_us = pred_full;
    const bool shallow_cold = h.first_batch && shallow_fraction > 0.0;
    if (update_fraction >= kPreflightFullUpdate) return true;
    if (shallow_cold) return true;
    if (!h.have_incremental) return false;
    return pred_inc * (1.0 - inc_unc) > pred_full * (1.0 + full_unc);
  }
  const double pred_inc = h.have_incremental ? h.ema_incremental_us * (1.0 + 2.0 * h.previous_affected_fraction) : 0.0;
  const double pred_full = h.have_full ? h.ema_full_us : 0.0;
  h.predicted_incremental_us = pred_inc;
  h.predicted_full_us = pred_full;
  const bool fresh = h.have_incremental && h.have_full && h.incremental_age <= kFreshAge && h.full_age <= kFreshAge;
  if (update_fraction >= kPreflightFullUpdate) return true;
  if (h.initial_reachable_fraction <= kVerySparseReach) return true;
  if (h.initial_reachable_fraction < kSparseReach && update_fraction >= kSparseReachFullUpdate) return true;
  if (fresh && pred_inc > pred_full * kLearnedFullMargin) return true;
  return false;
}

void heuristic_observe(HeuristicState& h, bool observed_full, double execution_us, double affected_fraction) {
  const double a = 0.25;  // kEmaAlpha
  ++h.incremental_age;
  ++h.full_age;
  if (h.large_scale && h.predicted_incremental_us > 0.0 && h.predicted_full_us > 0.0) {
    if (observed_full) {
      const double rel = std::abs(execution_us - h.predicted_full_us) / std::max(1.0, h.predicted_full_us);
      h.ema_full_rel_error = h.have_full_error ? (1 - a) * h.ema_full_rel_error + a * rel : rel;
      h.have_full_error = true;
    } else {
      const double rel = std::abs(execution_us - h.predicted_incremental_us) / std::max(1.0, h.predicted_incremental_us);
      h.ema_incremental_rel_error = h.have_incremental_error ? (1 - a) * h.ema_incremental_rel_error + a * rel : rel;
      h.have_incremental_error = true;
    }
  }
  if (observed_full) {
    h.ema_full_us = h.have_full ? (1 - a) * h.ema_full_us + a * execution_us : execution_us;
    h.have_full = true;
    h.full_age = 0;
    h.previous_affected_fraction = 0.0;
  } else {
    h.ema_incremental_us = h.have_incremental ? (1 - a) * h.ema_incremental_us + a * execution_us : execution_us;
    h.have_incremental = true;
    h.incremental_age = 0;
    h.last_incremental_update_fraction = h.update_fraction;
    h.previous_affected_fraction = affected_fraction;
  }
  h.first_batch = false;
}

}  // namespace vxh
