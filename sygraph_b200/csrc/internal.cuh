// Internal declarations of libsygraph_b200.so: handle types, status plumbing
// and launch helpers.  Not installed; the public surface is
// include/sygraph_b200.h.
#pragma once

#include <cuda_runtime.h>

#include <atomic>
#include <cstdint>
#include <mutex>
#include <cstdio>
#include <string>

#include "sygraph_b200.h"
#include "sygraph/detail/primitives.cuh"

namespace sgb {

// ------------------------------------------------------------------ status --
void set_error(const std::string& msg);
void clear_error();
sg_status fail(sg_status s, const std::string& msg);
sg_status cuda_fail(cudaError_t e, const char* what, const char* file, int line);
// Host CSR structure check (host_graph.cpp): offsets start at 0, never
// decrease and end at m; every column is below n.
sg_status check_csr(const uint32_t* ro, const uint32_t* col, uint32_t n, uint64_t m);

// Every launch goes through this counter so callers can report how many of
// this library's kernels ran in a timed region.
extern std::atomic<uint64_t> g_launches;
inline void count_launch(uint64_t k = 1) { g_launches.fetch_add(k, std::memory_order_relaxed); }

#define SG_CUDA(call)                                                         \
  do {                                                                        \
    cudaError_t _e = (call);                                                  \
    if (_e != cudaSuccess) return ::sgb::cuda_fail(_e, #call, __FILE__, __LINE__); \
  } while (0)

#define SG_CHECK_LAUNCH()                                                     \
  do {                                                                        \
    cudaError_t _e = cudaGetLastError();                                      \
    if (_e != cudaSuccess) return ::sgb::cuda_fail(_e, "kernel launch", __FILE__, __LINE__); \
    ::sgb::count_launch();                                                    \
  } while (0)

#define SG_REQUIRE(cond, status, msg)                                         \
  do {                                                                        \
    if (!(cond)) return ::sgb::fail((status), (msg));                         \
  } while (0)

#define SG_TRY(call)                                                          \
  do {                                                                        \
    sg_status _s = (call);                                                    \
    if (_s != SG_OK) return _s;                                               \
  } while (0)

// Device properties of the current device, cached.
struct DeviceProps {
  int device = -1;
  int sm_count = 0;
  int max_threads_per_sm = 0;
  size_t smem_per_block_optin = 0;
};
const DeviceProps& device_props();

template <typename T>
inline sg_status dev_alloc(T** p, uint64_t count) {
  *p = nullptr;
  if (count == 0) count = 1;
  cudaError_t e = cudaMalloc(reinterpret_cast<void**>(p), sizeof(T) * count);
  if (e != cudaSuccess) {
    cudaGetLastError();
    return fail(SG_ERR_NOMEM, std::string("cudaMalloc of ") + std::to_string(sizeof(T) * count) + " bytes failed: " +
                                  cudaGetErrorString(e));
  }
  return SG_OK;
}
template <typename T>
inline void dev_free(T*& p) {
  if (p) cudaFree(p);
  p = nullptr;
}

inline uint32_t div_up(uint64_t a, uint64_t b) { return (uint32_t)((a + b - 1) / b); }

// Grid for a grid-stride kernel: enough blocks to fill every SM `per_sm`
// times, never more than the work needs.
inline unsigned grid_for(uint64_t work_items, unsigned block, unsigned per_sm = 4) {
  const auto& p = device_props();
  uint64_t need = (work_items + block - 1) / block;
  uint64_t cap = (uint64_t)p.sm_count * per_sm;
  if (need < 1) need = 1;
  return (unsigned)(need < cap ? need : cap);
}

// Device address of an sg_mlp's parameter block (selector.cu).
const void* mlp_device_params(sg_mlp h);
// The parameters in the engines' shared-memory layout (MlpStaged), kept in
// device memory and rebuilt whenever the parameters change.
const void* mlp_device_image(sg_mlp h);
// Frees a graph and every device array it owns.
void release_graph(sg_graph g);
// Builds g->wcol / g->wval once (weighted graphs only).
sg_status graph_weight_sorted(sg_graph g);
// SG_ERR_TIMEOUT when the last launch of the instance left its grid barrier's
// error flag set (read after its stream completed; used by the server).
sg_status bfs_launch_status(sg_bfs b);
sg_status msbfs_launch_status(sg_msbfs h);
sg_status sssp_launch_status(sg_sssp s);

// ------------------------------------------------------------------ handles --
struct GraphDir {
  uint32_t* ro = nullptr;
  uint32_t* col = nullptr;
  void* val = nullptr;
};

}  // namespace sgb

struct sg_graph_s {
  // forward adjacency with each row sorted by (weight, column): the light /
  // heavy edge split of delta-stepping reads a prefix / suffix of a row;
  // built on first use (graph_weight_sorted), row offsets are fwd.ro
  uint32_t* wcol = nullptr;
  void* wval = nullptr;
  // set with wcol: rows sorted by column and every edge (u, v, w) has its
  // reverse (v, u, w), so a row also lists the vertex's in-edges
  bool wsym = false;
  std::mutex wsort_mu;
  uint32_t n = 0;
  uint64_t m = 0;
  uint32_t flags = 0;
  int value_type = SG_WEIGHT_NONE;
  cudaStream_t stream = nullptr;
  sgb::GraphDir fwd;
  sgb::GraphDir inv;  // aliases fwd when the graph is undirected
  bool owns_inverse = false;
  uint64_t bytes = 0;
  sg_graph_view view(bool inverse) const {
    const sgb::GraphDir& d = inverse ? inv : fwd;
    sg_graph_view v;
    v.n = n;
    v.m = m;
    v.row_offsets = d.ro;
    v.column_indices = d.col;
    v.values = d.val;
    v.value_type = value_type;
    return v;
  }
};

struct sg_frontier_s {
  uint32_t num_elems = 0;
  uint32_t words0 = 0;
  uint32_t words1 = 0;
  uint32_t* level0 = nullptr;
  uint32_t* level1 = nullptr;
  int32_t* offsets = nullptr;
  uint32_t* offsets_size = nullptr;
  uint64_t* scratch = nullptr;  // device scalar for reductions
  cudaStream_t stream = nullptr;
  sg_frontier_view view() const {
    sg_frontier_view v;
    v.num_elems = num_elems;
    v.words0 = words0;
    v.words1 = words1;
    v.level0 = level0;
    v.level1 = level1;
    v.offsets = offsets;
    v.offsets_size = offsets_size;
    return v;
  }
};
