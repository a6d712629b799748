// Learned strategy selector: a 12 -> 32 -> 32 -> 6 MLP (ReLU, FP32) that
// predicts the log-time of one traversal level under each of the six
// strategies (push / pull / pull_all x warp- / CTA-mapped) from twelve
// frontier features.  Training, gradients and inference are this file's own
// kernels: forward over a batch, backward with per-CTA gradient sums, Adam.
// The traversal engines run the same forward pass on the device at every
// level end (sygraph/detail/selector_mlp.cuh).
#include <cmath>
#include <cstring>
#include <vector>

#include "internal.cuh"
#include "sygraph/detail/selector_mlp.cuh"

namespace sgb {
namespace sel {

using sygraph::detail::MlpParams;
using sygraph::detail::kMlpIn;
using sygraph::detail::kMlpHidden;
using sygraph::detail::kMlpOut;
using sygraph::detail::kMlpParamCount;

// Forward pass of one sample held by one thread; activations kept for backward.
struct Acts {
  float x[kMlpIn];
  float h1[kMlpHidden];
  float h2[kMlpHidden];
  float y[kMlpOut];
};

__device__ __forceinline__ void forward_one(const float* __restrict__ p, const float* x, Acts& a) {
  const MlpParams& P = *reinterpret_cast<const MlpParams*>(p);
  for (int i = 0; i < kMlpIn; i++) a.x[i] = (x[i] - P.mean[i]) * P.inv_std[i];
  for (int j = 0; j < kMlpHidden; j++) {
    float s = P.b1[j];
    for (int i = 0; i < kMlpIn; i++) s += P.w1[j][i] * a.x[i];
    a.h1[j] = s > 0.f ? s : 0.f;
  }
  for (int j = 0; j < kMlpHidden; j++) {
    float s = P.b2[j];
    for (int i = 0; i < kMlpHidden; i++) s += P.w2[j][i] * a.h1[i];
    a.h2[j] = s > 0.f ? s : 0.f;
  }
  for (int j = 0; j < kMlpOut; j++) {
    float s = P.b3[j];
    for (int i = 0; i < kMlpHidden; i++) s += P.w3[j][i] * a.h2[i];
    a.y[j] = s;
  }
}

__global__ void __launch_bounds__(128) mlp_forward_kernel(const float* __restrict__ params,
                                                         const float* __restrict__ X, uint32_t n,
                                                         float* __restrict__ Y) {
  for (uint32_t r = blockIdx.x * blockDim.x + threadIdx.x; r < n; r += gridDim.x * blockDim.x) {
    Acts a;
    forward_one(params, X + (size_t)r * kMlpIn, a);
    for (int j = 0; j < kMlpOut; j++) Y[(size_t)r * kMlpOut + j] = a.y[j];
  }
}

// Loss = mean over samples and outputs of 0.5 * m * (y - t)^2, with mask m
// (0 where a strategy's time is unknown).  Gradients of the weights and
// biases (not of the normalisation) are summed per thread, reduced per CTA in
// shared memory and added to grad[] with one atomic per parameter per CTA.
__global__ void __launch_bounds__(128) mlp_backward_kernel(const float* __restrict__ params,
                                                          const float* __restrict__ X, const float* __restrict__ T,
                                                          const float* __restrict__ M, uint32_t n, float scale,
                                                          float* __restrict__ grad, float* __restrict__ loss) {
  __shared__ float s_grad[kMlpParamCount];
  for (int i = threadIdx.x; i < kMlpParamCount; i += blockDim.x) s_grad[i] = 0.f;
  __syncthreads();
  const MlpParams& P = *reinterpret_cast<const MlpParams*>(params);
  MlpParams& G = *reinterpret_cast<MlpParams*>(s_grad);
  float my_loss = 0.f;
  for (uint32_t r = blockIdx.x * blockDim.x + threadIdx.x; r < n; r += gridDim.x * blockDim.x) {
    Acts a;
    forward_one(params, X + (size_t)r * kMlpIn, a);
    float dy[kMlpOut], dh2[kMlpHidden], dh1[kMlpHidden];
    for (int j = 0; j < kMlpOut; j++) {
      const float mk = M[(size_t)r * kMlpOut + j];
      const float d = a.y[j] - T[(size_t)r * kMlpOut + j];
      my_loss += 0.5f * mk * d * d;
      dy[j] = mk * d * scale;
    }
    for (int i = 0; i < kMlpHidden; i++) dh2[i] = 0.f;
    for (int j = 0; j < kMlpOut; j++) {
      atomicAdd(&G.b3[j], dy[j]);
      for (int i = 0; i < kMlpHidden; i++) {
        atomicAdd(&G.w3[j][i], dy[j] * a.h2[i]);
        dh2[i] += P.w3[j][i] * dy[j];
      }
    }
    for (int i = 0; i < kMlpHidden; i++) {
      dh2[i] = a.h2[i] > 0.f ? dh2[i] : 0.f;
      dh1[i] = 0.f;
    }
    for (int j = 0; j < kMlpHidden; j++) {
      if (dh2[j] == 0.f) continue;
      atomicAdd(&G.b2[j], dh2[j]);
      for (int i = 0; i < kMlpHidden; i++) {
        atomicAdd(&G.w2[j][i], dh2[j] * a.h1[i]);
        dh1[i] += P.w2[j][i] * dh2[j];
      }
    }
    for (int j = 0; j < kMlpHidden; j++) {
      const float d = a.h1[j] > 0.f ? dh1[j] : 0.f;
      if (d == 0.f) continue;
      atomicAdd(&G.b1[j], d);
      for (int i = 0; i < kMlpIn; i++) atomicAdd(&G.w1[j][i], d * a.x[i]);
    }
  }
  __syncthreads();
  // normalisation entries carry no gradient
  for (int i = threadIdx.x; i < sygraph::detail::kMlpTrainableCount; i += blockDim.x)
    if (s_grad[i] != 0.f) atomicAdd(grad + i, s_grad[i]);
  // loss: warp reduce then one atomic per warp
  for (int d = 16; d > 0; d >>= 1) my_loss += __shfl_xor_sync(0xffffffffu, my_loss, d);
  if ((threadIdx.x & 31) == 0 && loss) atomicAdd(loss, my_loss * scale);
}

// Adam on the trainable prefix of the parameter block.
__global__ void adam_kernel(float* __restrict__ params, const float* __restrict__ grad, float* __restrict__ m1,
                            float* __restrict__ m2, uint32_t count, float lr, float b1, float b2, float eps,
                            float bc1, float bc2, float weight_decay) {
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < count; i += gridDim.x * blockDim.x) {
    const float g = grad[i] + weight_decay * params[i];
    m1[i] = b1 * m1[i] + (1.f - b1) * g;
    m2[i] = b2 * m2[i] + (1.f - b2) * g * g;
    params[i] -= lr * (m1[i] / bc1) / (sqrtf(m2[i] / bc2) + eps);
  }
}

}  // namespace sel
}  // namespace sgb

using namespace sgb;
using sygraph::detail::kMlpHidden;
using sygraph::detail::kMlpIn;
using sygraph::detail::kMlpOut;

struct sg_mlp_s {
  float* params = nullptr;  // kMlpParamCount
  // the parameters in the layout the traversal engines read them in (hidden
  // matrices transposed), rebuilt after every change of the parameters
  sygraph::detail::MlpStaged* image = nullptr;
  float* grad = nullptr;
  float* m1 = nullptr;
  float* m2 = nullptr;
  float* loss = nullptr;
  uint64_t step = 0;
};

namespace sgb {
const void* mlp_device_params(sg_mlp h) { return h ? h->params : nullptr; }
const void* mlp_device_image(sg_mlp h) { return h ? h->image : nullptr; }
}  // namespace sgb

__global__ void mlp_image_kernel(const sygraph::detail::MlpParams* __restrict__ p, sygraph::detail::MlpStaged* image) {
  sygraph::detail::mlp_stage(p, image);
}

// Rebuilds the staged image from the parameters and waits for it (the
// engines read it from any stream).
static sg_status mlp_refresh_image(sg_mlp h) {
  mlp_image_kernel<<<1, 256>>>(reinterpret_cast<const sygraph::detail::MlpParams*>(h->params), h->image);
  SG_CHECK_LAUNCH();
  SG_CUDA(cudaStreamSynchronize(0));
  return SG_OK;
}

static void mlp_release(sg_mlp h) {
  if (!h) return;
  dev_free(h->params);
  dev_free(h->image);
  dev_free(h->grad);
  dev_free(h->m1);
  dev_free(h->m2);
  dev_free(h->loss);
  delete h;
}

extern "C" {

uint32_t sg_mlp_param_count(void) { return sygraph::detail::kMlpParamCount; }

sg_status sg_mlp_create(const float* host_params, sg_mlp* out) {
  clear_error();
  SG_REQUIRE(out, SG_ERR_INVALID, "out is NULL");
  *out = nullptr;
  sg_mlp h = new sg_mlp_s();
  const uint32_t P = sygraph::detail::kMlpParamCount;
  sg_status s;
  if ((s = dev_alloc(&h->params, P)) || (s = dev_alloc(&h->grad, P)) || (s = dev_alloc(&h->m1, P)) ||
      (s = dev_alloc(&h->m2, P)) || (s = dev_alloc(&h->loss, 1)) || (s = dev_alloc(&h->image, 1))) {
    mlp_release(h);
    return s;
  }
  std::vector<float> init(P, 0.f);
  if (host_params) {
    memcpy(init.data(), host_params, sizeof(float) * P);
  } else {
    // He-style initialisation from a fixed generator; identity normalisation
    sygraph::detail::MlpParams* p = reinterpret_cast<sygraph::detail::MlpParams*>(init.data());
    uint64_t st = 0x2545f4914f6cdd1dull;
    auto rnd = [&]() {
      st ^= st >> 12;
      st ^= st << 25;
      st ^= st >> 27;
      return (double)((st * 0x2545f4914f6cdd1dull) >> 11) * (1.0 / 9007199254740992.0) * 2.0 - 1.0;
    };
    for (int j = 0; j < kMlpHidden; j++)
      for (int i = 0; i < kMlpIn; i++) p->w1[j][i] = (float)(rnd() * std::sqrt(6.0 / kMlpIn));
    for (int j = 0; j < kMlpHidden; j++)
      for (int i = 0; i < kMlpHidden; i++) p->w2[j][i] = (float)(rnd() * std::sqrt(6.0 / kMlpHidden));
    for (int j = 0; j < kMlpOut; j++)
      for (int i = 0; i < kMlpHidden; i++) p->w3[j][i] = (float)(rnd() * std::sqrt(3.0 / kMlpHidden));
    for (int i = 0; i < kMlpIn; i++) {
      p->mean[i] = 0.f;
      p->inv_std[i] = 1.f;
      p->lo[i] = -1e30f;
      p->hi[i] = 1e30f;
    }
  }
  cudaError_t e = cudaMemcpy(h->params, init.data(), sizeof(float) * P, cudaMemcpyHostToDevice);
  if (e == cudaSuccess) e = cudaMemset(h->m1, 0, sizeof(float) * P);
  if (e == cudaSuccess) e = cudaMemset(h->m2, 0, sizeof(float) * P);
  if (e != cudaSuccess) {
    mlp_release(h);
    return cuda_fail(e, "mlp init", __FILE__, __LINE__);
  }
  if ((s = mlp_refresh_image(h)) != SG_OK) {
    mlp_release(h);
    return s;
  }
  *out = h;
  return SG_OK;
}

sg_status sg_mlp_destroy(sg_mlp h) {
  mlp_release(h);
  return SG_OK;
}

sg_status sg_mlp_get_params(sg_mlp h, float* host_params) {
  SG_REQUIRE(h && host_params, SG_ERR_INVALID, "NULL argument");
  SG_CUDA(cudaMemcpy(host_params, h->params, sizeof(float) * sygraph::detail::kMlpParamCount, cudaMemcpyDeviceToHost));
  return SG_OK;
}

sg_status sg_mlp_set_params(sg_mlp h, const float* host_params) {
  SG_REQUIRE(h && host_params, SG_ERR_INVALID, "NULL argument");
  SG_CUDA(cudaMemcpy(h->params, host_params, sizeof(float) * sygraph::detail::kMlpParamCount, cudaMemcpyHostToDevice));
  return mlp_refresh_image(h);
}

sg_status sg_mlp_forward(sg_mlp h, const float* dev_x, uint32_t n, float* dev_y) {
  SG_REQUIRE(h && dev_x && dev_y, SG_ERR_INVALID, "NULL argument");
  if (!n) return SG_OK;
  sel::mlp_forward_kernel<<<grid_for(n, 128, 8), 128>>>(h->params, dev_x, n, dev_y);
  SG_CHECK_LAUNCH();
  SG_CUDA(cudaDeviceSynchronize());
  return SG_OK;
}

sg_status sg_mlp_gradient(sg_mlp h, const float* dev_x, const float* dev_t, const float* dev_mask, uint32_t n,
                          float* host_grad, float* host_loss) {
  SG_REQUIRE(h && dev_x && dev_t && dev_mask && host_grad, SG_ERR_INVALID, "NULL argument");
  const uint32_t P = sygraph::detail::kMlpParamCount;
  SG_CUDA(cudaMemset(h->grad, 0, sizeof(float) * P));
  SG_CUDA(cudaMemset(h->loss, 0, sizeof(float)));
  const float scale = n ? 1.0f / ((float)n * kMlpOut) : 0.f;
  sel::mlp_backward_kernel<<<grid_for(n, 128, 4), 128>>>(h->params, dev_x, dev_t, dev_mask, n, scale, h->grad,
                                                        h->loss);
  SG_CHECK_LAUNCH();
  SG_CUDA(cudaMemcpy(host_grad, h->grad, sizeof(float) * P, cudaMemcpyDeviceToHost));
  if (host_loss) SG_CUDA(cudaMemcpy(host_loss, h->loss, sizeof(float), cudaMemcpyDeviceToHost));
  return SG_OK;
}

sg_status sg_mlp_train(sg_mlp h, const float* dev_x, const float* dev_t, const float* dev_mask, uint32_t n,
                       uint32_t steps, float lr, float weight_decay, float* host_final_loss) {
  SG_REQUIRE(h && dev_x && dev_t && dev_mask, SG_ERR_INVALID, "NULL argument");
  SG_REQUIRE(n > 0, SG_ERR_INVALID, "empty training set");
  const uint32_t P = sygraph::detail::kMlpParamCount, T = sygraph::detail::kMlpTrainableCount;
  const float scale = 1.0f / ((float)n * kMlpOut);
  const float b1 = 0.9f, b2 = 0.999f, eps = 1e-8f;
  for (uint32_t s = 0; s < steps; s++) {
    SG_CUDA(cudaMemsetAsync(h->grad, 0, sizeof(float) * P));
    SG_CUDA(cudaMemsetAsync(h->loss, 0, sizeof(float)));
    sel::mlp_backward_kernel<<<grid_for(n, 128, 4), 128>>>(h->params, dev_x, dev_t, dev_mask, n, scale, h->grad,
                                                          h->loss);
    SG_CHECK_LAUNCH();
    h->step++;
    const float bc1 = 1.f - powf(b1, (float)h->step), bc2 = 1.f - powf(b2, (float)h->step);
    sel::adam_kernel<<<grid_for(T, 256), 256>>>(h->params, h->grad, h->m1, h->m2, T, lr, b1, b2, eps, bc1, bc2,
                                               weight_decay);
    SG_CHECK_LAUNCH();
  }
  if (host_final_loss) SG_CUDA(cudaMemcpy(host_final_loss, h->loss, sizeof(float), cudaMemcpyDeviceToHost));
  SG_CUDA(cudaDeviceSynchronize());
  return mlp_refresh_image(h);
}

}  // extern "C"
