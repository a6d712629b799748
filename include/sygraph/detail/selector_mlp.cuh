// Parameter layout of the strategy-selector MLP and its device-side forward
// pass for one feature vector (one warp), used inside the traversal engines.
//
// 12 features -> 32 (ReLU) -> 32 (ReLU) -> 6 predicted log-times, one per
// strategy: 0 push/warp, 1 push/CTA, 2 pull/warp, 3 pull/CTA, 4 pull_all/warp,
// 5 pull_all/CTA.  Inputs are standardised with the training set's mean and
// 1/std; lo/hi bound the training range (a feature outside it means the
// network is not trusted and the caller falls back to the heuristic).
#pragma once

#include <cstdint>

namespace sygraph {
namespace detail {

constexpr int kMlpIn = 12;
constexpr int kMlpHidden = 32;
constexpr int kMlpOut = 6;

struct MlpParams {
  // trainable block first (gradients and optimiser state cover only these)
  float w1[kMlpHidden][kMlpIn];
  float b1[kMlpHidden];
  float w2[kMlpHidden][kMlpHidden];
  float b2[kMlpHidden];
  float w3[kMlpOut][kMlpHidden];
  float b3[kMlpOut];
  // input standardisation and trusted range
  float mean[kMlpIn];
  float inv_std[kMlpIn];
  float lo[kMlpIn];
  float hi[kMlpIn];
};

constexpr int kMlpTrainableCount =
    kMlpHidden * kMlpIn + kMlpHidden + kMlpHidden * kMlpHidden + kMlpHidden + kMlpOut * kMlpHidden + kMlpOut;
constexpr int kMlpParamCount = (int)(sizeof(MlpParams) / sizeof(float));
static_assert(kMlpParamCount == kMlpTrainableCount + 4 * kMlpIn, "MlpParams must be packed floats");

#ifdef __CUDACC__
// Shared-memory copy of the parameters for inference inside the traversal
// engines: the two hidden-layer matrices transposed, so that lane j reads
// element j of a row (no bank conflicts), and no global load on the path.
struct __align__(16) MlpStaged {
  float w1t[kMlpIn][kMlpHidden];
  float b1[kMlpHidden];
  float w2t[kMlpHidden][kMlpHidden];
  float b2[kMlpHidden];
  float w3[kMlpOut][kMlpHidden];
  float b3[kMlpOut];
  float mean[kMlpIn];
  float inv_std[kMlpIn];
  float lo[kMlpIn];
  float hi[kMlpIn];
  float pad[2];  // a whole number of 16-byte chunks
};
constexpr int kMlpStagedChunks = (int)(sizeof(MlpStaged) / 16);
static_assert(sizeof(MlpStaged) % 16 == 0, "the staged image is copied in 16-byte chunks");

// Block-cooperative copy from the parameters; the caller synchronises the
// block afterwards.  (Also builds the staged image in global memory.)
__device__ __forceinline__ void mlp_stage(const MlpParams* __restrict__ g, MlpStaged* s) {
  for (int t = threadIdx.x; t < kMlpIn * kMlpHidden; t += blockDim.x)
    s->w1t[t / kMlpHidden][t % kMlpHidden] = g->w1[t % kMlpHidden][t / kMlpHidden];
  for (int t = threadIdx.x; t < kMlpHidden * kMlpHidden; t += blockDim.x)
    s->w2t[t / kMlpHidden][t % kMlpHidden] = g->w2[t % kMlpHidden][t / kMlpHidden];
  for (int t = threadIdx.x; t < kMlpOut * kMlpHidden; t += blockDim.x) s->w3[t / kMlpHidden][t % kMlpHidden] =
      g->w3[t / kMlpHidden][t % kMlpHidden];
  for (int t = threadIdx.x; t < kMlpHidden; t += blockDim.x) {
    s->b1[t] = g->b1[t];
    s->b2[t] = g->b2[t];
  }
  for (int t = threadIdx.x; t < kMlpIn; t += blockDim.x) {
    s->mean[t] = g->mean[t];
    s->inv_std[t] = g->inv_std[t];
    s->lo[t] = g->lo[t];
    s->hi[t] = g->hi[t];
  }
  for (int t = threadIdx.x; t < kMlpOut; t += blockDim.x) s->b3[t] = g->b3[t];
  if (threadIdx.x < 2) s->pad[threadIdx.x] = 0.f;
}

// Asynchronous copy of a staged image (already in the MlpStaged layout in
// global memory) into shared memory: every thread issues at most one or two
// 16-byte cp.async copies and goes on; mlp_stage_wait() completes them.
__device__ __forceinline__ void mlp_stage_async(const MlpStaged* __restrict__ image, MlpStaged* s) {
  const char* src = reinterpret_cast<const char*>(image);
  const uint32_t dst = static_cast<uint32_t>(__cvta_generic_to_shared(s));
  for (int t = threadIdx.x; t < kMlpStagedChunks; t += blockDim.x)
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(dst + 16u * t), "l"(src + 16 * t) : "memory");
  asm volatile("cp.async.commit_group;" ::: "memory");
}
// Waits for this thread's copies; the block must synchronise before any
// thread reads the staged parameters.
__device__ __forceinline__ void mlp_stage_wait() { asm volatile("cp.async.wait_all;" ::: "memory"); }

// Forward pass by one full warp, laid out for latency (it sits between a grid
// barrier and the next level): lane i < 12 holds feature i and checks and
// standardises it; lane j computes hidden unit j of both hidden layers (the
// inputs of layer 1 come by shuffles, the layer-1 activations through
// `scratch`, 32 floats of shared memory); the six outputs are butterfly sums
// over the lanes, so every lane ends with all six and picks locally.  Returns
// the strategy with the smallest predicted time among the set bits of
// `allowed` (lowest index on ties) -- unless `fallback` (the heuristic's
// choice, when allowed) is predicted within `margin` of it in log-time, which
// keeps the fallback -- or -1 when a feature lies outside the trusted range.
// Lanes may differ in the last bit of an output (each sums in its own order);
// callers take lane 0's answer, which is the same in every CTA.
__device__ __forceinline__ int mlp_choose(const MlpStaged* __restrict__ P, float f, uint32_t allowed, float* scratch,
                                          int fallback = -1, float margin = 0.f) {
  constexpr uint32_t kAll = 0xffffffffu;
  const uint32_t lane = threadIdx.x & 31;
  const bool mine = lane < (uint32_t)kMlpIn;
  const uint32_t li = mine ? lane : 0u;
  const bool out_of_range = mine && (f < P->lo[li] || f > P->hi[li]);
  if (__any_sync(kAll, out_of_range)) return -1;
  const float x = mine ? (f - P->mean[li]) * P->inv_std[li] : 0.f;
  // layer 1; independent partial sums break the dependent FMA chains
  float a0 = P->b1[lane], a1 = 0.f;
#pragma unroll
  for (int i = 0; i < kMlpIn; i += 2) {
    a0 += P->w1t[i][lane] * __shfl_sync(kAll, x, i);
    a1 += P->w1t[i + 1][lane] * __shfl_sync(kAll, x, i + 1);
  }
  const float h1 = a0 + a1;
  scratch[lane] = h1 > 0.f ? h1 : 0.f;
  __syncwarp();
  float c[4] = {P->b2[lane], 0.f, 0.f, 0.f};
#pragma unroll
  for (int i = 0; i < kMlpHidden; i += 4)
#pragma unroll
    for (int k = 0; k < 4; k++) c[k] += P->w2t[i + k][lane] * scratch[i + k];
  const float h2 = (c[0] + c[1]) + (c[2] + c[3]);
  const float r2 = h2 > 0.f ? h2 : 0.f;
  __syncwarp();  // scratch is rewritten by the next call
  // layer 3: the products of this lane's hidden unit, summed over the warp
  float y[kMlpOut];
#pragma unroll
  for (int o = 0; o < kMlpOut; o++) y[o] = P->w3[o][lane] * r2;
#pragma unroll
  for (int d = 16; d > 0; d >>= 1)
#pragma unroll
    for (int o = 0; o < kMlpOut; o++) y[o] += __shfl_xor_sync(kAll, y[o], d);
  float best = 3.4e38f, y_fallback = 3.4e38f;
  int arg = -1;
#pragma unroll
  for (int o = 0; o < kMlpOut; o++) {
    y[o] += P->b3[o];
    if (((allowed >> o) & 1u) && y[o] < best) {
      best = y[o];
      arg = o;
    }
    if (o == fallback) y_fallback = y[o];
  }
  if (arg < 0) return -1;
  if (fallback >= 0 && ((allowed >> fallback) & 1u) && y_fallback - best <= margin) arg = fallback;
  return arg;
}
#endif

}  // namespace detail
}  // namespace sygraph
