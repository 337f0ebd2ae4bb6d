// Learned schedule policy: graph features -> MLP 24 -> 64 -> 64 -> 3 -> (log2
// delta multiplier, log2 bucket-fusion threshold, log2 push/pull switch point
// of the heavy pass).
//
// No reference counterpart (the reference picks delta with the Near-Far rule,
// Charlotte_oneshot/sssp_hip.cpp:59-81, and adapts it in hip_adds).  The
// policy only chooses the schedule; distances are the same for every choice,
// and without an active policy the Near-Far delta is used.
//
// Numerics: weights are stored in BF16 for the forward and backward passes
// (FP32 master copy for the optimizer), every dot product accumulates in
// FP32.  Forward/backward run one 64-thread block per sample; per-sample
// gradients are written to a [batch x params] buffer and summed in a fixed
// order by a second kernel, so a training step is deterministic.
// Loss per sample: sum over the three outputs of (y - t)^2 (every output is a
// base-2 logarithm, so the loss weighs relative errors).
// Decoding (policy_decide): delta = Near-Far delta x 2^clamp(y0, -4, 6)
// (|y0| under the dead zone keeps the Near-Far delta); fusion threshold =
// 2^clamp(y1, 7, 14) frontier entries, off when y1 < 7; the heavy pass may
// pull when the bucket's heavy out-edges exceed 2^clamp(y2, 0, 7) x n, push
// only when y2 > 7.
#include <cuda_bf16.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <mutex>
#include <vector>

#include "b2_common.cuh"
#include "b2_internal.hpp"

namespace b2 {
namespace {

constexpr int kIn = 24, kH = 64, kOut = 3;
constexpr int oW1 = 0, oB1 = oW1 + kH * kIn, oW2 = oB1 + kH, oB2 = oW2 + kH * kH, oW3 = oB2 + kH,
              oB3 = oW3 + kOut * kH, kParams = oB3 + kOut;   // 5955
static_assert(kParams == 5955, "parameter count");

__device__ __forceinline__ float bf(const __nv_bfloat16* p, int i) { return __bfloat162float(p[i]); }

// forward for one sample; h1/h2 in shared memory
__device__ void mlp_forward(const __nv_bfloat16* __restrict__ w, const float* x, float* h1, float* h2, float* y) {
  const int j = threadIdx.x;   // 64 threads
  float a = bf(w, oB1 + j);
#pragma unroll 4
  for (int k = 0; k < kIn; ++k) a = fmaf(bf(w, oW1 + j * kIn + k), x[k], a);
  h1[j] = fmaxf(a, 0.0f);
  __syncthreads();
  float b = bf(w, oB2 + j);
#pragma unroll 8
  for (int k = 0; k < kH; ++k) b = fmaf(bf(w, oW2 + j * kH + k), h1[k], b);
  h2[j] = fmaxf(b, 0.0f);
  __syncthreads();
  if (j < kOut) {
    float c = bf(w, oB3 + j);
#pragma unroll 8
    for (int k = 0; k < kH; ++k) c = fmaf(bf(w, oW3 + j * kH + k), h2[k], c);
    y[j] = c;
  }
  __syncthreads();
}

__global__ void k_mlp_forward(const __nv_bfloat16* __restrict__ w, const float* __restrict__ X, int B,
                              float* __restrict__ Y) {
  __shared__ float x[kIn], h1[kH], h2[kH], y[kOut];
  for (int s = blockIdx.x; s < B; s += gridDim.x) {
    if (threadIdx.x < kIn) x[threadIdx.x] = X[s * kIn + threadIdx.x];
    __syncthreads();
    mlp_forward(w, x, h1, h2, y);
    if (threadIdx.x < kOut) Y[s * kOut + threadIdx.x] = y[threadIdx.x];
    __syncthreads();
  }
}


// per-sample loss and gradient of the mean loss (divided by B) -> G[s * kParams ...]
__global__ void k_mlp_backward(const __nv_bfloat16* __restrict__ w, const float* __restrict__ X,
                               const float* __restrict__ T, int B, float* __restrict__ G, float* __restrict__ L) {
  __shared__ float x[kIn], h1[kH], h2[kH], y[kOut], dy[kOut], dh2[kH], dh1[kH];
  const int j = threadIdx.x;
  const float inv_b = 1.0f / (float)B;
  for (int s = blockIdx.x; s < B; s += gridDim.x) {
    if (j < kIn) x[j] = X[s * kIn + j];
    __syncthreads();
    mlp_forward(w, x, h1, h2, y);
    if (j == 0) {
      float loss = 0.0f;
      for (int k = 0; k < kOut; ++k) {
        const float e = y[k] - T[s * kOut + k];
        loss = fmaf(e, e, loss);
        dy[k] = 2.0f * e * inv_b;
      }
      L[s] = loss;
    }
    __syncthreads();
    float* g = G + (size_t)s * kParams;
    // layer 3
    if (j < kOut) g[oB3 + j] = dy[j];
    for (int t = 0; t < kOut; ++t) g[oW3 + t * kH + j] = dy[t] * h2[j];
    float a = 0.0f;
    for (int t = 0; t < kOut; ++t) a = fmaf(bf(w, oW3 + t * kH + j), dy[t], a);
    dh2[j] = h2[j] > 0.0f ? a : 0.0f;
    __syncthreads();
    // layer 2
    g[oB2 + j] = dh2[j];
    for (int k = 0; k < kH; ++k) g[oW2 + j * kH + k] = dh2[j] * h1[k];
    float b = 0.0f;
    for (int i = 0; i < kH; ++i) b = fmaf(bf(w, oW2 + i * kH + j), dh2[i], b);
    dh1[j] = h1[j] > 0.0f ? b : 0.0f;
    __syncthreads();
    // layer 1
    g[oB1 + j] = dh1[j];
    for (int k = 0; k < kIn; ++k) g[oW1 + j * kIn + k] = dh1[j] * x[k];
    __syncthreads();
  }
}

// G_sum[p] = sum_s G[s][p] in sample order (deterministic)
__global__ void k_reduce_grads(const float* __restrict__ G, int B, float* __restrict__ out) {
  for (int p = blockIdx.x * blockDim.x + threadIdx.x; p < kParams; p += gridDim.x * blockDim.x) {
    float acc = 0.0f;
    for (int s = 0; s < B; ++s) acc += G[(size_t)s * kParams + p];
    out[p] = acc;
  }
}

// AdamW step (decoupled weight decay wd) on the FP32 master copy; refreshes the BF16 copy.
__global__ void k_adam(float* __restrict__ master, __nv_bfloat16* __restrict__ w, const float* __restrict__ g,
                       float* __restrict__ m, float* __restrict__ v, float lr, float b1, float b2, float eps,
                       float c1, float c2, float wd) {
  for (int p = blockIdx.x * blockDim.x + threadIdx.x; p < kParams; p += gridDim.x * blockDim.x) {
    const float gp = g[p];
    const float mp = b1 * m[p] + (1.0f - b1) * gp;
    const float vp = b2 * v[p] + (1.0f - b2) * gp * gp;
    m[p] = mp;
    v[p] = vp;
    const float upd = lr * ((mp / c1) / (sqrtf(vp / c2) + eps) + wd * master[p]);
    const float np = master[p] - upd;
    master[p] = np;
    w[p] = __float2bfloat16(np);
  }
}

__global__ void k_to_bf16(const float* __restrict__ src, __nv_bfloat16* __restrict__ dst, int n) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
    dst[i] = __float2bfloat16(src[i]);
}

// deterministic samples for the feature extractor
__device__ __forceinline__ uint64_t mix64d(uint64_t z) {
  z += 0x9E3779B97F4A7C15ull;
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
  return z ^ (z >> 31);
}
__global__ void k_sample(int64_t n, int64_t m, const uint64_t* __restrict__ rowptr, const uint2* __restrict__ edges,
                         int S, uint32_t* __restrict__ vid, uint32_t* __restrict__ deg, uint32_t* __restrict__ wb) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < S; i += gridDim.x * blockDim.x) {
    const uint64_t v = n <= S ? (uint64_t)i % (uint64_t)n : mix64d(0x5eed0000ull + i) % (uint64_t)n;
    const uint64_t d = rowptr[v + 1] - rowptr[v];
    vid[i] = (uint32_t)v;
    deg[i] = (uint32_t)(d > 0xFFFFFFFFull ? 0xFFFFFFFFull : d);
    if (m > 0) {
      const uint64_t e = m <= S ? (uint64_t)i % (uint64_t)m : mix64d(0xfeed0000ull + i) % (uint64_t)m;
      wb[i] = edges[e].y;
    } else {
      wb[i] = 0;
    }
  }
}

}  // namespace

struct PolicyState {
  float* master = nullptr;          // FP32 parameters
  __nv_bfloat16* w = nullptr;       // BF16 working copy
  float* m = nullptr;
  float* v = nullptr;
  float* grad = nullptr;
  float mu[kIn];
  float sigma[kIn];
  // raw features are clamped to the range seen in training before they are
  // normalized, so a graph past the training sizes is scored like the
  // nearest training graphs rather than extrapolated
  float lo[kIn];
  float hi[kIn];
  int has_range = 0;
  float dead_zone = 0.0f;   // |predicted log2 delta multiplier| below this keeps the Near-Far delta
  int step = 0;
};

}  // namespace b2

struct b2_policy_s {
  b2::PolicyState s;
};

namespace b2 {
namespace {
std::mutex g_pol_mu;
b2_policy g_active = nullptr;
uint64_t g_generation = 1;   // bumped whenever the active policy or its weights change

b2_status upload_params(b2_policy p, const float* host) {
  B2_CUDA_TRY(cudaMemcpy(p->s.master, host, kParams * sizeof(float), cudaMemcpyHostToDevice));
  k_to_bf16<<<24, 256>>>(p->s.master, p->s.w, kParams);
  B2_CUDA_TRY(cudaGetLastError());
  B2_CUDA_TRY(cudaDeviceSynchronize());
  return B2_SUCCESS;
}

void normalize(const b2_policy p, const float* raw, float* out, int B) {
  for (int s = 0; s < B; ++s)
    for (int k = 0; k < kIn; ++k) {
      float x = raw[s * kIn + k];
      if (p->s.has_range) x = std::min(std::max(x, p->s.lo[k]), p->s.hi[k]);
      out[s * kIn + k] = (x - p->s.mu[k]) / p->s.sigma[k];
    }
}

constexpr int kSample = 65536;
constexpr double kLog2MultMin = -4.0, kLog2MultMax = 6.0;   // clamp of output y0
constexpr double kFusionOffBelow = 7.0, kFusionLog2Max = 14.0;   // output y1
constexpr double kPullOffAbove = 7.0, kPullLog2Min = 0.0;       // output y2
constexpr int kDepthCap = 256;   // hop-depth probe: at most this many Bellman-Ford rounds
constexpr float kRangeMargin = 0.1f;   // out-of-range tolerance, as a fraction of each feature's training span

// The 24 features: size (log n, log m, m/n, log max degree), out-degree
// quantiles of a vertex sample, weight quantiles of an edge sample (relative
// to the mean weight), weight spread, Near-Far delta and the light-edge share
// under it, and the hop depth of a bounded Bellman-Ford solve from the
// highest-degree sampled vertex (rounds until no label changes, capped).
b2_status graph_features(b2_graph g, float* f) {
  const int S = kSample;
  uint32_t* dbuf = nullptr;
  B2_CUDA_TRY(cudaMalloc((void**)&dbuf, (size_t)3 * S * 4));
  k_sample<<<64, 256>>>(g->n, g->m, g->rowptr, g->edges, S, dbuf, dbuf + S, dbuf + 2 * S);
  std::vector<uint32_t> h((size_t)3 * S);
  cudaError_t e = cudaGetLastError();
  if (e == cudaSuccess) e = cudaMemcpy(h.data(), dbuf, h.size() * 4, cudaMemcpyDeviceToHost);
  cudaFree(dbuf);
  if (e != cudaSuccess) return from_cuda(e);
  const uint32_t* vid = h.data();
  std::vector<uint32_t> deg(h.begin() + S, h.begin() + 2 * S);
  const uint32_t* wb = h.data() + 2 * S;
  uint32_t src = vid[0], best = deg[0];
  for (int i = 1; i < S; ++i)
    if (deg[i] > best) { best = deg[i]; src = vid[i]; }
  const bool isf = g->weight_type == B2_W_F32;
  std::vector<double> w(S);
  for (int i = 0; i < S; ++i) {
    if (isf) {
      float x;
      memcpy(&x, &wb[i], 4);
      w[i] = std::isfinite(x) ? (double)x : 0.0;
    } else {
      w[i] = (double)wb[i];
    }
  }
  std::sort(deg.begin(), deg.end());
  std::sort(w.begin(), w.end());
  auto dq = [&](double q) { return std::log2(1.0 + (double)deg[(size_t)std::min<double>(S - 1, q * S)]); };
  const double mw = std::max(1e-12, g->mean_weight);
  auto wq = [&](double q) { return w[(size_t)std::min<double>(S - 1, q * S)] / mw; };
  double mean = 0, var = 0;
  for (double x : w) mean += x;
  mean /= S;
  for (double x : w) var += (x - mean) * (x - mean);
  var /= S;
  size_t zero = 0;
  for (uint32_t d : deg) zero += d == 0;
  double nf = 1.0;
  b2_delta_heuristic(g, 16.0, &nf);
  size_t light = 0;
  for (double x : w) light += x <= nf;
  double depth = kDepthCap;
  {
    b2_sssp_opts o;
    b2_sssp_opts_default(&o);
    o.max_iters = kDepthCap;
    b2_stats st;
    void* d = nullptr;
    B2_CUDA_TRY(cudaMalloc(&d, (size_t)g->n * 4));
    uint32_t src_in = src;   // sampled ids are internal; solves take input ids
    if (g->perm) cudaMemcpy(&src_in, g->perm + src, 4, cudaMemcpyDeviceToHost);
    b2_status s = b2_sssp_bf(g, src_in, d, nullptr, &o, 0, &st);
    cudaFree(d);
    if (s != B2_SUCCESS) return s;
    if (st.converged) depth = (double)st.iterations_used;
  }
  const double n = (double)g->n, m = (double)std::max<int64_t>(1, g->m);
  const float feats[kIn] = {
      (float)std::log2(n), (float)std::log2(m), (float)(m / n), (float)std::log2(1.0 + g->max_degree),
      (float)dq(0.25), (float)dq(0.5), (float)dq(0.75), (float)dq(0.9), (float)dq(0.99),
      (float)((double)zero / S),
      (float)wq(0.1), (float)wq(0.25), (float)wq(0.5), (float)wq(0.75), (float)wq(0.9),
      (float)std::log2(mw), (float)(std::sqrt(var) / mw), (float)std::log2(1.0 + depth),
      (float)std::log2(nf), (float)((double)light / S), isf ? 1.0f : 0.0f,
      (float)(depth >= kDepthCap ? 1.0f : 0.0f), (float)wq(0.99), (float)std::log2(1.0 + m / n)};
  memcpy(f, feats, sizeof(feats));
  return B2_SUCCESS;
}

b2_status features_cached(b2_graph g) {
  if (g->features_valid) return B2_SUCCESS;
  b2_status s = graph_features(g, g->features);
  if (s == B2_SUCCESS) g->features_valid = true;
  return s;
}

b2_status run_forward(b2_policy p, const float* xn_host, int B, float* y_host) {
  float* d = nullptr;
  B2_CUDA_TRY(cudaMalloc((void**)&d, (size_t)B * (kIn + kOut) * 4));
  cudaError_t e = cudaMemcpy(d, xn_host, (size_t)B * kIn * 4, cudaMemcpyHostToDevice);
  if (e == cudaSuccess) {
    k_mlp_forward<<<std::min(B, 1024), kH>>>(p->s.w, d, B, d + (size_t)B * kIn);
    e = cudaGetLastError();
  }
  if (e == cudaSuccess) e = cudaMemcpy(y_host, d + (size_t)B * kIn, (size_t)B * kOut * 4, cudaMemcpyDeviceToHost);
  cudaFree(d);
  return from_cuda(e);
}
}  // namespace

b2_status policy_decide(b2_graph g, double* delta_mult, uint32_t* fusion_threshold, float* pull_fraction) {
  std::lock_guard<std::mutex> lock(g_pol_mu);
  if (!g_active) return B2_NOT_SUPPORTED;
  if (g->pol_version != g_generation) {
    b2_status s = features_cached(g);
    if (s != B2_SUCCESS) return s;
    // a graph past the training graphs' range (by more than a tenth of the
    // range in any feature) keeps the fixed schedule: the network was never
    // shown such a graph and its guess there is not evidence
    g->pol_outside = false;
    if (g_active->s.has_range)
      for (int k = 0; k < kIn; ++k) {
        const float span = g_active->s.hi[k] - g_active->s.lo[k];
        const float x = g->features[k];
        if (x < g_active->s.lo[k] - kRangeMargin * span || x > g_active->s.hi[k] + kRangeMargin * span)
          g->pol_outside = true;
      }
    float xn[kIn], y[kOut];
    normalize(g_active, g->features, xn, 1);
    s = run_forward(g_active, xn, 1, y);
    if (s != B2_SUCCESS) return s;
    double lm = std::max(kLog2MultMin, std::min(kLog2MultMax, (double)y[0]));
    if (std::fabs(lm) < (double)g_active->s.dead_zone) lm = 0.0;
    g->pol_mult = std::exp2(lm);
    g->pol_fusion = (double)y[1] < kFusionOffBelow
                        ? 0u
                        : (uint32_t)std::lround(std::exp2(std::min(kFusionLog2Max, (double)y[1])));
    g->pol_pull = (double)y[2] > kPullOffAbove ? 0.0f
                                               : (float)std::exp2(std::max(kPullLog2Min, (double)y[2]));
    g->pol_version = g_generation;
  }
  if (g->pol_outside) return B2_NOT_SUPPORTED;   // the caller runs the fixed Near-Far schedule
  *delta_mult = g->pol_mult;
  *fusion_threshold = g->pol_fusion;
  *pull_fraction = g->pol_pull;
  return B2_SUCCESS;
}

}  // namespace b2

using namespace b2;

extern "C" int32_t b2_policy_param_count(void) { return kParams; }

extern "C" b2_status b2_policy_create(uint64_t seed, b2_policy* out) {
  if (!out) return B2_INVALID_ARGUMENT;
  b2_policy p = new b2_policy_s();
  auto fail = [&](cudaError_t e) {
    b2_policy_destroy(p);
    return from_cuda(e);
  };
  cudaError_t e = cudaMalloc((void**)&p->s.master, kParams * 4);
  if (e == cudaSuccess) e = cudaMalloc((void**)&p->s.w, kParams * 2);
  if (e == cudaSuccess) e = cudaMalloc((void**)&p->s.m, kParams * 4);
  if (e == cudaSuccess) e = cudaMalloc((void**)&p->s.v, kParams * 4);
  if (e == cudaSuccess) e = cudaMalloc((void**)&p->s.grad, kParams * 4);
  if (e != cudaSuccess) return fail(e);
  cudaMemset(p->s.m, 0, kParams * 4);
  cudaMemset(p->s.v, 0, kParams * 4);
  // He-uniform initial weights from a counter hash (deterministic), zero biases
  std::vector<float> h(kParams, 0.0f);
  uint64_t st = seed ^ 0x2545F4914F6CDD1Dull;
  auto u01 = [&]() {
    st += 0x9E3779B97F4A7C15ull;
    uint64_t z = st;
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    z ^= z >> 31;
    return (double)(z >> 11) * (1.0 / 9007199254740992.0);
  };
  auto fill = [&](int off, int count, int fan_in) {
    const double a = std::sqrt(6.0 / fan_in);
    for (int i = 0; i < count; ++i) h[off + i] = (float)((2.0 * u01() - 1.0) * a);
  };
  fill(oW1, kH * kIn, kIn);
  fill(oW2, kH * kH, kH);
  fill(oW3, kOut * kH, kH);
  for (int k = 0; k < kIn; ++k) { p->s.mu[k] = 0.0f; p->s.sigma[k] = 1.0f; }
  b2_status s = upload_params(p, h.data());
  if (s != B2_SUCCESS) { b2_policy_destroy(p); return s; }
  *out = p;
  return B2_SUCCESS;
}

extern "C" b2_status b2_policy_destroy(b2_policy p) {
  if (!p) return B2_INVALID_ARGUMENT;
  {
    std::lock_guard<std::mutex> lock(g_pol_mu);
    if (g_active == p) {
      g_active = nullptr;
      ++g_generation;
    }
  }
  cudaFree(p->s.master);
  cudaFree(p->s.w);
  cudaFree(p->s.m);
  cudaFree(p->s.v);
  cudaFree(p->s.grad);
  delete p;
  return B2_SUCCESS;
}

extern "C" b2_status b2_policy_set_params(b2_policy p, const float* params, const float* mu, const float* sigma) {
  if (!p || !params) return B2_INVALID_ARGUMENT;
  if (mu && sigma)
    for (int k = 0; k < kIn; ++k) {
      p->s.mu[k] = mu[k];
      p->s.sigma[k] = sigma[k] > 0.0f ? sigma[k] : 1.0f;
    }
  std::lock_guard<std::mutex> lock(g_pol_mu);
  ++g_generation;
  return upload_params(p, params);
}

// Range of the raw features seen in training (lo/hi null: no clamping).
extern "C" b2_status b2_policy_set_feature_range(b2_policy p, const float* lo, const float* hi) {
  if (!p || (!lo) != (!hi)) return B2_INVALID_ARGUMENT;
  if (lo)
    for (int k = 0; k < kIn; ++k)
      if (!(lo[k] <= hi[k])) return B2_INVALID_ARGUMENT;
  std::lock_guard<std::mutex> lock(g_pol_mu);
  if (lo) {
    memcpy(p->s.lo, lo, sizeof(p->s.lo));
    memcpy(p->s.hi, hi, sizeof(p->s.hi));
  }
  p->s.has_range = lo ? 1 : 0;
  ++g_generation;
  return B2_SUCCESS;
}

extern "C" b2_status b2_policy_set_dead_zone(b2_policy p, float log2_dead_zone) {
  if (!p || !(log2_dead_zone >= 0.0f)) return B2_INVALID_ARGUMENT;
  std::lock_guard<std::mutex> lock(g_pol_mu);
  p->s.dead_zone = log2_dead_zone;
  ++g_generation;
  return B2_SUCCESS;
}

extern "C" b2_status b2_policy_get_params(b2_policy p, float* params, float* mu, float* sigma) {
  if (!p || !params) return B2_INVALID_ARGUMENT;
  B2_CUDA_TRY(cudaMemcpy(params, p->s.master, kParams * 4, cudaMemcpyDeviceToHost));
  if (mu) memcpy(mu, p->s.mu, sizeof(p->s.mu));
  if (sigma) memcpy(sigma, p->s.sigma, sizeof(p->s.sigma));
  return B2_SUCCESS;
}

// X: B x 24 raw features (normalized here with the policy's mu/sigma).
extern "C" b2_status b2_policy_forward(b2_policy p, const float* X, int32_t B, float* Y) {
  if (!p || !X || !Y || B <= 0) return B2_INVALID_ARGUMENT;
  std::vector<float> xn((size_t)B * kIn);
  normalize(p, X, xn.data(), B);
  return run_forward(p, xn.data(), B, Y);
}

// Gradient of the mean loss over the batch at the current BF16 weights
// (grad: 5955 floats, loss: mean loss).  Features are normalized first.
extern "C" b2_status b2_policy_gradient(b2_policy p, const float* X, const float* T, int32_t B, float* grad,
                                       float* loss) {
  if (!p || !X || !T || B <= 0) return B2_INVALID_ARGUMENT;
  std::vector<float> xn((size_t)B * kIn);
  normalize(p, X, xn.data(), B);
  float *dx = nullptr, *dt = nullptr, *dg = nullptr, *dl = nullptr;
  cudaError_t e = cudaMalloc((void**)&dx, xn.size() * 4);
  if (e == cudaSuccess) e = cudaMalloc((void**)&dt, (size_t)B * kOut * 4);
  if (e == cudaSuccess) e = cudaMalloc((void**)&dg, (size_t)B * kParams * 4);
  if (e == cudaSuccess) e = cudaMalloc((void**)&dl, (size_t)B * 4);
  if (e == cudaSuccess) e = cudaMemcpy(dx, xn.data(), xn.size() * 4, cudaMemcpyHostToDevice);
  if (e == cudaSuccess) e = cudaMemcpy(dt, T, (size_t)B * kOut * 4, cudaMemcpyHostToDevice);
  if (e == cudaSuccess) {
    k_mlp_backward<<<std::min(B, 4096), kH>>>(p->s.w, dx, dt, B, dg, dl);
    k_reduce_grads<<<24, 256>>>(dg, B, p->s.grad);
    e = cudaGetLastError();
  }
  std::vector<float> hl((size_t)B);
  if (e == cudaSuccess && grad) e = cudaMemcpy(grad, p->s.grad, kParams * 4, cudaMemcpyDeviceToHost);
  if (e == cudaSuccess) e = cudaMemcpy(hl.data(), dl, (size_t)B * 4, cudaMemcpyDeviceToHost);
  cudaFree(dx);
  cudaFree(dt);
  cudaFree(dg);
  cudaFree(dl);
  if (e != cudaSuccess) return from_cuda(e);
  if (loss) {
    double s = 0;
    for (float x : hl) s += x;
    *loss = (float)(s / B);
  }
  return B2_SUCCESS;
}

// Full-batch AdamW on the GPU.  Sets the feature normalization from X on the
// first call (step 0).  loss_out: mean loss after the last epoch.
extern "C" b2_status b2_policy_train(b2_policy p, const float* X, const float* T, int32_t B, int32_t epochs,
                                    float lr, float weight_decay, float* loss_out) {
  if (!p || !X || !T || B <= 0 || epochs < 0 || !(lr > 0.0f) || !(weight_decay >= 0.0f))
    return B2_INVALID_ARGUMENT;
  {
    std::lock_guard<std::mutex> lock(g_pol_mu);
    ++g_generation;
  }
  if (p->s.step == 0) {
    for (int k = 0; k < kIn; ++k) {
      double m = 0, v = 0;
      float lo = X[k], hi = X[k];
      for (int s = 0; s < B; ++s) {
        m += X[s * kIn + k];
        lo = std::min(lo, X[s * kIn + k]);
        hi = std::max(hi, X[s * kIn + k]);
      }
      m /= B;
      for (int s = 0; s < B; ++s) v += (X[s * kIn + k] - m) * (X[s * kIn + k] - m);
      v /= B;
      p->s.mu[k] = (float)m;
      p->s.sigma[k] = v > 1e-12 ? (float)std::sqrt(v) : 1.0f;
      p->s.lo[k] = lo;
      p->s.hi[k] = hi;
    }
    p->s.has_range = 1;
  }
  std::vector<float> xn((size_t)B * kIn);
  normalize(p, X, xn.data(), B);
  float *dx = nullptr, *dt = nullptr, *dg = nullptr, *dl = nullptr;
  cudaError_t e = cudaMalloc((void**)&dx, xn.size() * 4);
  if (e == cudaSuccess) e = cudaMalloc((void**)&dt, (size_t)B * kOut * 4);
  if (e == cudaSuccess) e = cudaMalloc((void**)&dg, (size_t)B * kParams * 4);
  if (e == cudaSuccess) e = cudaMalloc((void**)&dl, (size_t)B * 4);
  if (e == cudaSuccess) e = cudaMemcpy(dx, xn.data(), xn.size() * 4, cudaMemcpyHostToDevice);
  if (e == cudaSuccess) e = cudaMemcpy(dt, T, (size_t)B * kOut * 4, cudaMemcpyHostToDevice);
  const float b1 = 0.9f, b2v = 0.999f;
  for (int ep = 0; ep < epochs && e == cudaSuccess; ++ep) {
    k_mlp_backward<<<std::min(B, 4096), kH>>>(p->s.w, dx, dt, B, dg, dl);
    k_reduce_grads<<<24, 256>>>(dg, B, p->s.grad);
    ++p->s.step;
    const float c1 = 1.0f - std::pow(b1, (float)p->s.step), c2 = 1.0f - std::pow(b2v, (float)p->s.step);
    k_adam<<<24, 256>>>(p->s.master, p->s.w, p->s.grad, p->s.m, p->s.v, lr, b1, b2v, 1e-8f, c1, c2,
                        weight_decay);
    e = cudaGetLastError();
  }
  if (e == cudaSuccess && loss_out) {
    k_mlp_backward<<<std::min(B, 4096), kH>>>(p->s.w, dx, dt, B, dg, dl);
    std::vector<float> hl((size_t)B);
    e = cudaMemcpy(hl.data(), dl, (size_t)B * 4, cudaMemcpyDeviceToHost);
    double s = 0;
    for (float x : hl) s += x;
    *loss_out = (float)(s / B);
  }
  cudaFree(dx);
  cudaFree(dt);
  cudaFree(dg);
  cudaFree(dl);
  return from_cuda(e);
}

// The policy used by solves run with opts.policy = 1 (NULL deactivates).
extern "C" b2_status b2_policy_activate(b2_policy p) {
  std::lock_guard<std::mutex> lock(g_pol_mu);
  g_active = p;
  ++g_generation;
  return B2_SUCCESS;
}

extern "C" b2_status b2_graph_features(b2_graph g, float* features) {
  if (!g || !features) return B2_INVALID_ARGUMENT;
  b2_status s;
  {
    std::lock_guard<std::mutex> lock(g_pol_mu);
    s = features_cached(g);
  }
  if (s != B2_SUCCESS) return s;
  memcpy(features, g->features, sizeof(float) * kIn);
  return B2_SUCCESS;
}
