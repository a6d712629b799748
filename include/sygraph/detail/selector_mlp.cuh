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

// Forward pass by one full warp: lane j computes hidden unit j; the hidden
// activations go through `scratch` (64 floats of shared memory) so that every
// lane reads them with independent broadcast loads, and lanes 0-5 compute the
// six outputs.  Returns, in every lane, the strategy with the smallest
// predicted time among the set bits of `allowed` (lowest index on ties) --
// unless `fallback` (the heuristic's choice, when allowed) is predicted within
// `margin` of it in log-time, which keeps the fallback -- or -1 when a
// feature lies outside the trusted range.
__device__ __forceinline__ int mlp_choose(const MlpStaged* __restrict__ P, const float* f, uint32_t allowed,
                                          float* scratch, int fallback = -1, float margin = 0.f) {
  const uint32_t lane = threadIdx.x & 31;
  bool out_of_range = false;
  float x[kMlpIn];
#pragma unroll
  for (int i = 0; i < kMlpIn; i++) {
    out_of_range |= f[i] < P->lo[i] || f[i] > P->hi[i];
    x[i] = (f[i] - P->mean[i]) * P->inv_std[i];
  }
  if (out_of_range) return -1;
  // independent partial sums break the dependent FMA chains
  float a0 = P->b1[lane], a1 = 0.f;
#pragma unroll
  for (int i = 0; i < kMlpIn; i += 2) {
    a0 += P->w1t[i][lane] * x[i];
    a1 += P->w1t[i + 1][lane] * x[i + 1];
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
  scratch[kMlpHidden + lane] = h2 > 0.f ? h2 : 0.f;
  __syncwarp();
  float y = 3.4e38f;
  if (lane < (uint32_t)kMlpOut) {
    float d[4] = {P->b3[lane], 0.f, 0.f, 0.f};
#pragma unroll
    for (int i = 0; i < kMlpHidden; i += 4)
#pragma unroll
      for (int k = 0; k < 4; k++) d[k] += P->w3[lane][i + k] * scratch[kMlpHidden + i + k];
    y = (d[0] + d[1]) + (d[2] + d[3]);
  }
  __syncwarp();
  const float y_fallback = __shfl_sync(0xffffffffu, y, fallback >= 0 ? fallback : 0);
  // argmin over lanes 0-7 (the six outputs; the others hold +inf)
  float best = (lane < (uint32_t)kMlpOut && ((allowed >> lane) & 1u)) ? y : 3.4e38f;
  int arg = best < 3.4e38f ? (int)lane : 32;
#pragma unroll
  for (int dd = 4; dd > 0; dd >>= 1) {
    const float ob = __shfl_xor_sync(0xffffffffu, best, dd);
    const int oa = __shfl_xor_sync(0xffffffffu, arg, dd);
    if (ob < best || (ob == best && oa < arg)) {
      best = ob;
      arg = oa;
    }
  }
  best = __shfl_sync(0xffffffffu, best, 0);
  arg = __shfl_sync(0xffffffffu, arg, 0);
  if (arg >= kMlpOut) return -1;
  if (fallback >= 0 && ((allowed >> fallback) & 1u) && y_fallback - best <= margin) arg = fallback;
  return arg;
}
#endif

}  // namespace detail
}  // namespace sygraph
