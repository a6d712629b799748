// Two-level bitmap frontier (FrontierMLB, frontier/impls/mlb_frontier.hpp:155-449):
// create / clear / insert / remove / check / empty / size / merge /
// intersect / swap / save / load, and the bitmap -> word-list compaction
// computeActiveFrontier(invert) (mlb:388-442) as a warp-ballot kernel.
#include <algorithm>
#include <vector>

#include "internal.cuh"
#include "sygraph/detail/advance_kernels.cuh"

namespace sgb {

using sygraph::detail::kFullMask;
using sygraph::detail::ld_cg;
using sygraph::detail::MLBDev;

MLBDev mlb_dev(const sg_frontier_s* f) {
  MLBDev d;
  d.num_elems = f->num_elems;
  d.words0 = f->words0;
  d.words1 = f->words1;
  d.l0 = f->level0;
  d.l1 = f->level1;
  d.offsets = f->offsets;
  d.offsets_size = f->offsets_size;
  return d;
}

// One lane per level-0 word.  Push lists words with any bit set; pull
// (invert) lists words with a clear bit inside [0, num_elems), i.e. words
// that still hold candidates.  Warp ballot + one atomic per warp.
__global__ void __launch_bounds__(256) mlb_compact_kernel(MLBDev f, int invert) {
  const uint32_t lane = threadIdx.x & 31;
  const uint32_t gwarp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const uint32_t nwarps = (gridDim.x * blockDim.x) >> 5;
  const uint32_t rem = f.num_elems & 31u;
  for (uint32_t base = gwarp * 32; base < f.words0; base += nwarps * 32) {
    const uint32_t w = base + lane;
    bool keep = false;
    if (w < f.words0) {
      const uint32_t bits = ld_cg(f.l0 + w);
      if (!invert) {
        keep = bits != 0;
      } else {
        const uint32_t full = (w == f.words0 - 1 && rem) ? ((1u << rem) - 1u) : 0xffffffffu;
        keep = (bits & full) != full;
      }
    }
    const uint32_t pos = sygraph::detail::warp_append(keep, f.offsets_size);
    if (keep) f.offsets[pos] = (int32_t)w;
  }
}

__global__ void mlb_insert_one(MLBDev f, uint32_t idx) { f.insert(idx); }
__global__ void mlb_remove_one(MLBDev f, uint32_t idx) { f.remove(idx); }

__global__ void __launch_bounds__(256) mlb_insert_list(MLBDev f, const uint32_t* ids, uint64_t count) {
  for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < count; i += (uint64_t)gridDim.x * blockDim.x)
    f.insert(ids[i]);
}

// Level-1 bits recomputed from level 0 (bit j of word k set iff level-0 word
// 32k+j is non-zero).  One lane per level-0 word.
__global__ void __launch_bounds__(256) mlb_rebuild_level1(MLBDev f) {
  const uint32_t lane = threadIdx.x & 31;
  const uint32_t gwarp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const uint32_t nwarps = (gridDim.x * blockDim.x) >> 5;
  for (uint32_t k = gwarp; k < f.words1; k += nwarps) {
    const uint32_t w = k * 32 + lane;
    const bool nz = w < f.words0 && ld_cg(f.l0 + w) != 0;
    const uint32_t bits = __ballot_sync(kFullMask, nz);
    if (lane == 0) f.l1[k] = bits;
  }
}

// op 0: a |= b (both levels); op 1: a &= b (level 0); op 2: out = a & b (level 0)
__global__ void __launch_bounds__(256) mlb_bitwise(uint32_t* dst, const uint32_t* a, const uint32_t* b, uint32_t words,
                                                   int op) {
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < words; i += gridDim.x * blockDim.x) {
    const uint32_t x = ld_cg(a + i), y = ld_cg(b + i);
    dst[i] = op == 0 ? (x | y) : (x & y);
  }
}

// Population count of level 0 and any-non-zero flag.
__global__ void __launch_bounds__(256) mlb_count(MLBDev f, unsigned long long* out) {
  __shared__ unsigned long long s_red[32];
  unsigned long long c = 0;
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < f.words0; i += gridDim.x * blockDim.x)
    c += __popc(ld_cg(f.l0 + i));
  c = sygraph::detail::block_sum(c, s_red);
  if (threadIdx.x == 0 && c) atomicAdd(out, c);
}

__global__ void __launch_bounds__(256) mlb_any(MLBDev f, unsigned long long* out) {
  bool any = false;
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < f.words0 && !any; i += gridDim.x * blockDim.x)
    any = ld_cg(f.l0 + i) != 0;
  if (__any_sync(kFullMask, any) && (threadIdx.x & 31) == 0) atomicOr(out, 1ull);
}

sg_status frontier_compact(sg_frontier f, int invert, cudaStream_t stream) {
  SG_CUDA(cudaMemsetAsync(f->offsets_size, 0, sizeof(uint32_t), stream));
  mlb_compact_kernel<<<grid_for(f->words0, 256), 256, 0, stream>>>(mlb_dev(f), invert);
  SG_CHECK_LAUNCH();
  return SG_OK;
}

sg_status frontier_clear(sg_frontier f, cudaStream_t stream) {
  SG_CUDA(cudaMemsetAsync(f->level0, 0, sizeof(uint32_t) * f->words0, stream));
  SG_CUDA(cudaMemsetAsync(f->level1, 0, sizeof(uint32_t) * f->words1, stream));
  SG_CUDA(cudaMemsetAsync(f->offsets_size, 0, sizeof(uint32_t), stream));
  return SG_OK;
}

sg_status frontier_rebuild_level1(sg_frontier f, cudaStream_t stream) {
  mlb_rebuild_level1<<<grid_for((uint64_t)f->words1 * 32, 256), 256, 0, stream>>>(mlb_dev(f));
  SG_CHECK_LAUNCH();
  return SG_OK;
}

sg_status frontier_and(sg_frontier out, sg_frontier a, sg_frontier b, cudaStream_t stream) {
  mlb_bitwise<<<grid_for(out->words0, 256), 256, 0, stream>>>(out->level0, a->level0, b->level0, out->words0, 1);
  SG_CHECK_LAUNCH();
  SG_CUDA(cudaMemsetAsync(out->offsets_size, 0, sizeof(uint32_t), stream));
  return frontier_rebuild_level1(out, stream);
}

}  // namespace sgb

using namespace sgb;

static void frontier_release(sg_frontier f) {
  if (!f) return;
  dev_free(f->level0);
  dev_free(f->level1);
  dev_free(f->offsets);
  dev_free(f->offsets_size);
  dev_free(f->scratch);
  delete f;
}

extern "C" {

sg_status sg_frontier_create(uint32_t num_elems, void* stream, sg_frontier* out) {
  clear_error();
  SG_REQUIRE(out, SG_ERR_INVALID, "out is NULL");
  *out = nullptr;
  sg_frontier f = new sg_frontier_s();
  f->num_elems = num_elems;
  f->words0 = div_up(num_elems, 32);
  f->words1 = div_up(f->words0, 32);
  f->stream = (cudaStream_t)stream;
  sg_status s;
  if ((s = dev_alloc(&f->level0, f->words0)) || (s = dev_alloc(&f->level1, f->words1)) ||
      (s = dev_alloc(&f->offsets, f->words0)) || (s = dev_alloc(&f->offsets_size, 1)) ||
      (s = dev_alloc(&f->scratch, 1)) || (s = frontier_clear(f, f->stream))) {
    frontier_release(f);
    return s;
  }
  *out = f;
  return SG_OK;
}

sg_status sg_frontier_destroy(sg_frontier f) {
  if (f) {
    cudaStreamSynchronize(f->stream);
    frontier_release(f);
  }
  return SG_OK;
}

sg_status sg_frontier_device_view(sg_frontier f, sg_frontier_view* view) {
  SG_REQUIRE(f && view, SG_ERR_INVALID, "NULL argument");
  *view = f->view();
  return SG_OK;
}

sg_status sg_frontier_num_elems(sg_frontier f, uint32_t* num_elems) {
  SG_REQUIRE(f && num_elems, SG_ERR_INVALID, "NULL argument");
  *num_elems = f->num_elems;
  return SG_OK;
}

sg_status sg_frontier_clear(sg_frontier f) {
  SG_REQUIRE(f, SG_ERR_INVALID, "frontier is NULL");
  return frontier_clear(f, f->stream);
}

sg_status sg_frontier_insert(sg_frontier f, uint32_t idx) {
  SG_REQUIRE(f, SG_ERR_INVALID, "frontier is NULL");
  SG_REQUIRE(idx < f->num_elems, SG_ERR_INVALID, "index out of range");
  mlb_insert_one<<<1, 1, 0, f->stream>>>(mlb_dev(f), idx);
  SG_CHECK_LAUNCH();
  return SG_OK;
}

sg_status sg_frontier_remove(sg_frontier f, uint32_t idx) {
  SG_REQUIRE(f, SG_ERR_INVALID, "frontier is NULL");
  SG_REQUIRE(idx < f->num_elems, SG_ERR_INVALID, "index out of range");
  mlb_remove_one<<<1, 1, 0, f->stream>>>(mlb_dev(f), idx);
  SG_CHECK_LAUNCH();
  return SG_OK;
}

sg_status sg_frontier_check(sg_frontier f, uint32_t idx, int* present) {
  SG_REQUIRE(f && present, SG_ERR_INVALID, "NULL argument");
  SG_REQUIRE(idx < f->num_elems, SG_ERR_INVALID, "index out of range");
  uint32_t w = 0;
  SG_CUDA(cudaMemcpyAsync(&w, f->level0 + (idx >> 5), sizeof(w), cudaMemcpyDeviceToHost, f->stream));
  SG_CUDA(cudaStreamSynchronize(f->stream));
  *present = (w >> (idx & 31)) & 1u;
  return SG_OK;
}

sg_status sg_frontier_insert_list(sg_frontier f, const uint32_t* host_ids, uint64_t count) {
  SG_REQUIRE(f, SG_ERR_INVALID, "frontier is NULL");
  if (count == 0) return SG_OK;
  SG_REQUIRE(host_ids, SG_ERR_INVALID, "ids is NULL");
  for (uint64_t i = 0; i < count; i++) SG_REQUIRE(host_ids[i] < f->num_elems, SG_ERR_INVALID, "index out of range");
  uint32_t* d = nullptr;
  SG_TRY(dev_alloc(&d, count));
  cudaError_t e = cudaMemcpyAsync(d, host_ids, sizeof(uint32_t) * count, cudaMemcpyHostToDevice, f->stream);
  if (e == cudaSuccess) {
    mlb_insert_list<<<grid_for(count, 256), 256, 0, f->stream>>>(mlb_dev(f), d, count);
    e = cudaGetLastError();
    count_launch();
  }
  cudaError_t e2 = cudaStreamSynchronize(f->stream);
  cudaFree(d);
  if (e != cudaSuccess) return cuda_fail(e, "insert_list", __FILE__, __LINE__);
  if (e2 != cudaSuccess) return cuda_fail(e2, "insert_list", __FILE__, __LINE__);
  return SG_OK;
}

sg_status sg_frontier_empty(sg_frontier f, int* empty) {
  SG_REQUIRE(f && empty, SG_ERR_INVALID, "NULL argument");
  SG_CUDA(cudaMemsetAsync(f->scratch, 0, sizeof(uint64_t), f->stream));
  mlb_any<<<grid_for(f->words0, 256), 256, 0, f->stream>>>(mlb_dev(f), (unsigned long long*)f->scratch);
  SG_CHECK_LAUNCH();
  uint64_t any = 0;
  SG_CUDA(cudaMemcpyAsync(&any, f->scratch, sizeof(any), cudaMemcpyDeviceToHost, f->stream));
  SG_CUDA(cudaStreamSynchronize(f->stream));
  *empty = any ? 0 : 1;
  return SG_OK;
}

sg_status sg_frontier_size(sg_frontier f, uint64_t* size) {
  SG_REQUIRE(f && size, SG_ERR_INVALID, "NULL argument");
  SG_CUDA(cudaMemsetAsync(f->scratch, 0, sizeof(uint64_t), f->stream));
  mlb_count<<<grid_for(f->words0, 256), 256, 0, f->stream>>>(mlb_dev(f), (unsigned long long*)f->scratch);
  SG_CHECK_LAUNCH();
  SG_CUDA(cudaMemcpyAsync(size, f->scratch, sizeof(uint64_t), cudaMemcpyDeviceToHost, f->stream));
  SG_CUDA(cudaStreamSynchronize(f->stream));
  return SG_OK;
}

sg_status sg_frontier_merge(sg_frontier f, sg_frontier other) {
  SG_REQUIRE(f && other, SG_ERR_INVALID, "NULL argument");
  SG_REQUIRE(f->num_elems == other->num_elems, SG_ERR_INVALID, "frontier sizes differ");
  mlb_bitwise<<<grid_for(f->words0, 256), 256, 0, f->stream>>>(f->level0, f->level0, other->level0, f->words0, 0);
  SG_CHECK_LAUNCH();
  mlb_bitwise<<<grid_for(f->words1, 256), 256, 0, f->stream>>>(f->level1, f->level1, other->level1, f->words1, 0);
  SG_CHECK_LAUNCH();
  return SG_OK;
}

sg_status sg_frontier_intersect(sg_frontier f, sg_frontier other) {
  SG_REQUIRE(f && other, SG_ERR_INVALID, "NULL argument");
  SG_REQUIRE(f->num_elems == other->num_elems, SG_ERR_INVALID, "frontier sizes differ");
  mlb_bitwise<<<grid_for(f->words0, 256), 256, 0, f->stream>>>(f->level0, f->level0, other->level0, f->words0, 1);
  SG_CHECK_LAUNCH();
  return frontier_rebuild_level1(f, f->stream);
}

sg_status sg_frontier_swap(sg_frontier a, sg_frontier b) {
  SG_REQUIRE(a && b, SG_ERR_INVALID, "NULL argument");
  SG_REQUIRE(a->num_elems == b->num_elems, SG_ERR_INVALID, "frontier sizes differ");
  std::swap(a->level0, b->level0);
  std::swap(a->level1, b->level1);
  std::swap(a->offsets, b->offsets);
  std::swap(a->offsets_size, b->offsets_size);
  std::swap(a->scratch, b->scratch);
  return SG_OK;
}

sg_status sg_frontier_compact(sg_frontier f, int invert, uint32_t* host_active_words) {
  SG_REQUIRE(f, SG_ERR_INVALID, "frontier is NULL");
  SG_TRY(frontier_compact(f, invert, f->stream));
  if (host_active_words) {
    SG_CUDA(cudaMemcpyAsync(host_active_words, f->offsets_size, sizeof(uint32_t), cudaMemcpyDeviceToHost, f->stream));
    SG_CUDA(cudaStreamSynchronize(f->stream));
  }
  return SG_OK;
}

sg_status sg_frontier_save(sg_frontier f, uint32_t* host_level0, uint32_t* host_level1) {
  SG_REQUIRE(f && host_level0 && host_level1, SG_ERR_INVALID, "NULL argument");
  SG_CUDA(cudaMemcpyAsync(host_level0, f->level0, sizeof(uint32_t) * f->words0, cudaMemcpyDeviceToHost, f->stream));
  SG_CUDA(cudaMemcpyAsync(host_level1, f->level1, sizeof(uint32_t) * f->words1, cudaMemcpyDeviceToHost, f->stream));
  SG_CUDA(cudaStreamSynchronize(f->stream));
  return SG_OK;
}

sg_status sg_frontier_load(sg_frontier f, const uint32_t* host_level0, const uint32_t* host_level1) {
  SG_REQUIRE(f && host_level0 && host_level1, SG_ERR_INVALID, "NULL argument");
  SG_CUDA(cudaMemcpyAsync(f->level0, host_level0, sizeof(uint32_t) * f->words0, cudaMemcpyHostToDevice, f->stream));
  SG_CUDA(cudaMemcpyAsync(f->level1, host_level1, sizeof(uint32_t) * f->words1, cudaMemcpyHostToDevice, f->stream));
  SG_CUDA(cudaStreamSynchronize(f->stream));
  return SG_OK;
}

sg_status sg_frontier_to_flags(sg_frontier f, uint8_t* host_flags) {
  SG_REQUIRE(f && host_flags, SG_ERR_INVALID, "NULL argument");
  std::vector<uint32_t> w(f->words0 ? f->words0 : 1);
  SG_CUDA(cudaMemcpyAsync(w.data(), f->level0, sizeof(uint32_t) * f->words0, cudaMemcpyDeviceToHost, f->stream));
  SG_CUDA(cudaStreamSynchronize(f->stream));
  for (uint32_t i = 0; i < f->num_elems; i++) host_flags[i] = (w[i >> 5] >> (i & 31)) & 1u;
  return SG_OK;
}

}  // extern "C"
