// Status plumbing, device helpers and the device CSR graph
// (graph::build::fromCSR / GraphCSR, graph/build.hpp:31-41,
// graph/impls/graph_csr.hpp:158-439).
#include <algorithm>
#include <cstring>
#include <mutex>
#include <vector>

#include "internal.cuh"
#include "sygraph/detail/primitives.cuh"

namespace sgb {

std::atomic<uint64_t> g_launches{0};

static thread_local std::string t_last_error;

void set_error(const std::string& msg) { t_last_error = msg; }
void clear_error() { t_last_error.clear(); }
sg_status fail(sg_status s, const std::string& msg) {
  set_error(msg);
  return s;
}
sg_status cuda_fail(cudaError_t e, const char* what, const char* file, int line) {
  cudaGetLastError();  // clear sticky-free errors so the context stays usable
  char buf[512];
  snprintf(buf, sizeof(buf), "%s failed: %s (%s:%d)", what, cudaGetErrorString(e), file, line);
  set_error(buf);
  if (e == cudaErrorMemoryAllocation) return SG_ERR_NOMEM;
  return SG_ERR_CUDA;
}

const DeviceProps& device_props() {
  static thread_local DeviceProps props;
  int dev = 0;
  cudaGetDevice(&dev);
  if (props.device != dev) {
    cudaDeviceProp p;
    if (cudaGetDeviceProperties(&p, dev) == cudaSuccess) {
      props.device = dev;
      props.sm_count = p.multiProcessorCount;
      props.max_threads_per_sm = p.maxThreadsPerMultiProcessor;
      props.smem_per_block_optin = p.sharedMemPerBlockOptin;
    } else {
      cudaGetLastError();
      props.sm_count = 148;
    }
  }
  return props;
}

// Transpose on the device: count in-degrees, exclusive scan on the host side
// of the copy, then a stable scatter per source row (one thread per source
// row walks its sorted list, so each inverse list comes out sorted by source
// id exactly as formats::CSR::invert builds it, formats/csr.hpp:179-209).
__global__ void k_indegree(const uint32_t* __restrict__ col, uint64_t m, uint32_t* __restrict__ cnt) {
  for (uint64_t e = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; e < m; e += (uint64_t)gridDim.x * blockDim.x)
    atomicAdd(cnt + col[e], 1u);
}

}  // namespace sgb

// Diagnostic of the bounded grid barrier: every block but `skip_block`
// (none when it is >= the grid) waits at one barrier with `limit` polls;
// blocks whose wait ran out count themselves in *out.
__global__ void barrier_check_kernel(sygraph::detail::GridBarrier* bar, uint32_t skip_block, uint64_t limit,
                                     uint32_t* out) {
  if (blockIdx.x == skip_block) return;  // never arrives
  const bool ok = sygraph::detail::grid_sync(bar, limit);
  if (threadIdx.x == 0 && !ok) atomicAdd(out, 1u);
}

using namespace sgb;

void sgb::release_graph(sg_graph g) {
  if (!g) return;
  dev_free(g->wcol);
  if (g->wval) cudaFree(g->wval);
  if (g->owns_inverse) {
    dev_free(g->inv.ro);
    dev_free(g->inv.col);
    if (g->inv.val) cudaFree(g->inv.val);
  }
  dev_free(g->fwd.ro);
  dev_free(g->fwd.col);
  if (g->fwd.val) cudaFree(g->fwd.val);
  delete g;
}

extern "C" {

const char* sg_last_error(void) { return t_last_error.c_str(); }

const char* sg_status_string(sg_status s) {
  switch (s) {
    case SG_OK: return "SG_OK";
    case SG_ERR_INVALID: return "SG_ERR_INVALID";
    case SG_ERR_CUDA: return "SG_ERR_CUDA";
    case SG_ERR_NOMEM: return "SG_ERR_NOMEM";
    case SG_ERR_TIMEOUT: return "SG_ERR_TIMEOUT";
    case SG_ERR_UNSUPPORTED: return "SG_ERR_UNSUPPORTED";
    case SG_ERR_NOT_INITIALIZED: return "SG_ERR_NOT_INITIALIZED";
    default: return "SG_ERR_UNKNOWN";
  }
}

const char* sg_version(void) { return "sygraph_b200 0.1 (sm_100a)"; }

uint64_t sg_kernel_launch_count(void) { return g_launches.load(); }

sg_status sg_device_count(int* count) {
  SG_REQUIRE(count, SG_ERR_INVALID, "count is NULL");
  SG_CUDA(cudaGetDeviceCount(count));
  return SG_OK;
}

sg_status sg_set_device(int device) {
  SG_CUDA(cudaSetDevice(device));
  return SG_OK;
}

sg_status sg_device_info(int* sm_count, uint64_t* free_bytes, uint64_t* total_bytes) {
  size_t f = 0, t = 0;
  SG_CUDA(cudaMemGetInfo(&f, &t));
  if (sm_count) *sm_count = device_props().sm_count;
  if (free_bytes) *free_bytes = f;
  if (total_bytes) *total_bytes = t;
  return SG_OK;
}

sg_status sg_malloc_device(uint64_t bytes, void** dev_ptr) {
  SG_REQUIRE(dev_ptr, SG_ERR_INVALID, "dev_ptr is NULL");
  return dev_alloc(reinterpret_cast<uint8_t**>(dev_ptr), bytes);
}

sg_status sg_free_device(void* dev_ptr) {
  if (dev_ptr) SG_CUDA(cudaFree(dev_ptr));
  return SG_OK;
}

sg_status sg_malloc_host_pinned(uint64_t bytes, void** host_ptr) {
  SG_REQUIRE(host_ptr, SG_ERR_INVALID, "host_ptr is NULL");
  cudaError_t e = cudaMallocHost(host_ptr, bytes ? bytes : 1);
  if (e != cudaSuccess) {
    cudaGetLastError();
    return fail(SG_ERR_NOMEM, "cudaMallocHost failed");
  }
  return SG_OK;
}

sg_status sg_free_host_pinned(void* host_ptr) {
  if (host_ptr) SG_CUDA(cudaFreeHost(host_ptr));
  return SG_OK;
}

sg_status sg_memcpy(void* dst, const void* src, uint64_t bytes, int kind, void* stream) {
  if (bytes == 0) return SG_OK;
  SG_REQUIRE(dst && src, SG_ERR_INVALID, "NULL pointer in sg_memcpy");
  cudaMemcpyKind k = kind == 0 ? cudaMemcpyHostToDevice
                     : kind == 1 ? cudaMemcpyDeviceToHost
                     : kind == 2 ? cudaMemcpyDeviceToDevice
                                 : cudaMemcpyDefault;
  SG_CUDA(cudaMemcpyAsync(dst, src, bytes, k, (cudaStream_t)stream));
  if (kind == 1 || kind == 3) SG_CUDA(cudaStreamSynchronize((cudaStream_t)stream));
  return SG_OK;
}

sg_status sg_memcpy_async(void* dst, const void* src, uint64_t bytes, int kind, void* stream) {
  if (bytes == 0) return SG_OK;
  SG_REQUIRE(dst && src, SG_ERR_INVALID, "NULL pointer in sg_memcpy_async");
  SG_REQUIRE(kind >= 0 && kind <= 3, SG_ERR_INVALID, "kind must be 0-3");
  const cudaMemcpyKind k = kind == 0   ? cudaMemcpyHostToDevice
                           : kind == 1 ? cudaMemcpyDeviceToHost
                           : kind == 2 ? cudaMemcpyDeviceToDevice
                                       : cudaMemcpyDefault;
  SG_CUDA(cudaMemcpyAsync(dst, src, bytes, k, (cudaStream_t)stream));
  return SG_OK;
}

sg_status sg_memset(void* dev_ptr, int value, uint64_t bytes, void* stream) {
  if (bytes == 0) return SG_OK;
  SG_REQUIRE(dev_ptr, SG_ERR_INVALID, "NULL pointer in sg_memset");
  SG_CUDA(cudaMemsetAsync(dev_ptr, value, bytes, (cudaStream_t)stream));
  return SG_OK;
}

sg_status sg_debug_barrier_check(uint32_t blocks, uint32_t skip_block, uint64_t spin_limit, uint32_t* timed_out,
                                 uint32_t* error_flag) {
  clear_error();
  SG_REQUIRE(timed_out && error_flag, SG_ERR_INVALID, "NULL argument");
  SG_REQUIRE(blocks >= 1 && blocks <= 64, SG_ERR_INVALID, "blocks must be in [1, 64]");
  SG_REQUIRE(spin_limit >= 1 && spin_limit <= (1ull << 20), SG_ERR_INVALID, "spin_limit must be in [1, 2^20]");
  int coop = 0, dev = 0;
  SG_CUDA(cudaGetDevice(&dev));
  SG_CUDA(cudaDeviceGetAttribute(&coop, cudaDevAttrCooperativeLaunch, dev));
  SG_REQUIRE(coop, SG_ERR_UNSUPPORTED, "device cannot launch cooperative kernels");
  sygraph::detail::GridBarrier* bar = nullptr;
  uint32_t* out = nullptr;
  SG_TRY(dev_alloc(&bar, 1));
  sg_status st = dev_alloc(&out, 1);
  cudaError_t e = cudaSuccess;
  if (st == SG_OK) {
    e = cudaMemset(bar, 0, sizeof(*bar));
    if (e == cudaSuccess) e = cudaMemset(out, 0, sizeof(uint32_t));
    void* args[] = {&bar, &skip_block, &spin_limit, &out};
    if (e == cudaSuccess)
      e = cudaLaunchCooperativeKernel((const void*)barrier_check_kernel, dim3(blocks), dim3(64), args, 0, nullptr);
    if (e == cudaSuccess) e = cudaDeviceSynchronize();
    sygraph::detail::GridBarrier hb = {};
    if (e == cudaSuccess) e = cudaMemcpy(&hb, bar, sizeof(hb), cudaMemcpyDeviceToHost);
    if (e == cudaSuccess) e = cudaMemcpy(timed_out, out, sizeof(uint32_t), cudaMemcpyDeviceToHost);
    *error_flag = hb.error;
    if (e != cudaSuccess) st = cuda_fail(e, "barrier check", __FILE__, __LINE__);
  }
  dev_free(bar);
  dev_free(out);
  return st;
}

sg_status sg_event_record(void* stream, void** event) {
  clear_error();
  SG_REQUIRE(event, SG_ERR_INVALID, "NULL argument");
  cudaEvent_t e = nullptr;
  SG_CUDA(cudaEventCreate(&e));
  const cudaError_t r = cudaEventRecord(e, (cudaStream_t)stream);
  if (r != cudaSuccess) {
    cudaEventDestroy(e);
    return cuda_fail(r, "cudaEventRecord", __FILE__, __LINE__);
  }
  *event = e;
  return SG_OK;
}

sg_status sg_event_elapsed_ms(void* start, void* end, float* ms) {
  clear_error();
  SG_REQUIRE(start && end && ms, SG_ERR_INVALID, "NULL argument");
  SG_CUDA(cudaEventSynchronize((cudaEvent_t)end));
  SG_CUDA(cudaEventElapsedTime(ms, (cudaEvent_t)start, (cudaEvent_t)end));
  return SG_OK;
}

sg_status sg_event_destroy(void* event) {
  if (event) cudaEventDestroy((cudaEvent_t)event);
  return SG_OK;
}

sg_status sg_stream_create(void** stream) {
  clear_error();
  SG_REQUIRE(stream, SG_ERR_INVALID, "NULL argument");
  cudaStream_t st = nullptr;
  SG_CUDA(cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking));
  *stream = st;
  return SG_OK;
}

sg_status sg_stream_destroy(void* stream) {
  if (stream) SG_CUDA(cudaStreamDestroy((cudaStream_t)stream));
  return SG_OK;
}

sg_status sg_stream_synchronize(void* stream) {
  SG_CUDA(cudaStreamSynchronize((cudaStream_t)stream));
  return SG_OK;
}

sg_status sg_device_synchronize(void) {
  SG_CUDA(cudaDeviceSynchronize());
  return SG_OK;
}

// ------------------------------------------------------------------- graph --

static sg_status build_inverse(sg_graph g, const uint32_t* h_ro, const uint32_t* h_col, const void* h_val) {
  // Host transpose, the same construction as formats::CSR::invert
  // (formats/csr.hpp:179-209): counting pass, prefix sum, then rows in
  // increasing order append themselves to their columns' lists.
  const uint32_t n = g->n;
  const uint64_t m = g->m;
  std::vector<uint32_t> iro((size_t)n + 1, 0);
  for (uint64_t e = 0; e < m; e++) {
    if (h_col[e] >= n) return fail(SG_ERR_INVALID, "column index out of range");
    iro[(size_t)h_col[e] + 1]++;
  }
  for (uint32_t v = 0; v < n; v++) iro[v + 1] += iro[v];
  std::vector<uint32_t> icol(m ? m : 1);
  std::vector<uint32_t> ival(h_val ? (m ? m : 1) : 0);
  std::vector<uint32_t> cursor(iro.begin(), iro.end() - 1);
  const uint32_t* hv = reinterpret_cast<const uint32_t*>(h_val);
  for (uint32_t r = 0; r < n; r++) {
    for (uint32_t e = h_ro[r]; e < h_ro[r + 1]; e++) {
      uint32_t c = h_col[e];
      uint32_t d = cursor[c]++;
      icol[d] = r;
      if (hv) ival[d] = hv[e];
    }
  }
  SG_TRY(dev_alloc(&g->inv.ro, (uint64_t)n + 1));
  SG_TRY(dev_alloc(&g->inv.col, m));
  SG_CUDA(cudaMemcpyAsync(g->inv.ro, iro.data(), sizeof(uint32_t) * ((uint64_t)n + 1), cudaMemcpyHostToDevice, g->stream));
  SG_CUDA(cudaMemcpyAsync(g->inv.col, icol.data(), sizeof(uint32_t) * m, cudaMemcpyHostToDevice, g->stream));
  if (hv) {
    uint32_t* d = nullptr;
    SG_TRY(dev_alloc(&d, m));
    g->inv.val = d;
    SG_CUDA(cudaMemcpyAsync(d, ival.data(), sizeof(uint32_t) * m, cudaMemcpyHostToDevice, g->stream));
  }
  SG_CUDA(cudaStreamSynchronize(g->stream));
  g->owns_inverse = true;
  g->bytes += sizeof(uint32_t) * ((uint64_t)n + 1 + m + (hv ? m : 0));
  return SG_OK;
}


sg_status sg_graph_create_csr(const uint32_t* host_row_offsets, const uint32_t* host_column_indices,
                              const void* host_values, int value_type, uint32_t n, uint64_t m, uint32_t flags,
                              void* stream, sg_graph* out) {
  clear_error();
  SG_REQUIRE(out, SG_ERR_INVALID, "out is NULL");
  *out = nullptr;
  SG_REQUIRE(host_row_offsets, SG_ERR_INVALID, "row_offsets is NULL");
  SG_REQUIRE(m == 0 || host_column_indices, SG_ERR_INVALID, "column_indices is NULL");
  SG_REQUIRE(m < (1ull << 32), SG_ERR_INVALID, "edge count must fit uint32 offsets");
  SG_REQUIRE(n < 0xffffffffu, SG_ERR_INVALID, "vertex count must be below 2^32-1");
  SG_REQUIRE(value_type == SG_WEIGHT_NONE || value_type == SG_WEIGHT_F32 || value_type == SG_WEIGHT_U32,
             SG_ERR_INVALID, "unknown value_type");
  SG_TRY(check_csr(host_row_offsets, host_column_indices, n, m));
  sg_graph g = new sg_graph_s();
  g->n = n;
  g->m = m;
  g->flags = flags;
  g->stream = (cudaStream_t)stream;
  // Unweighted input still carries a value array of ones so every functor
  // sees a weight, as fromMM does for pattern matrices (io/read_csr.hpp:121-124).
  g->value_type = value_type == SG_WEIGHT_NONE ? SG_WEIGHT_U32 : value_type;
  std::vector<uint32_t> ones;
  const void* vals = host_values;
  if (!vals || value_type == SG_WEIGHT_NONE) {
    ones.assign(m ? m : 1, 1u);
    if (value_type == SG_WEIGHT_F32) {
      float one = 1.0f;
      uint32_t bits;
      memcpy(&bits, &one, 4);
      for (auto& x : ones) x = bits;
    }
    vals = ones.data();
  }
  sg_status s = SG_OK;
  do {
    if ((s = dev_alloc(&g->fwd.ro, (uint64_t)n + 1)) != SG_OK) break;
    if ((s = dev_alloc(&g->fwd.col, m)) != SG_OK) break;
    uint32_t* dv = nullptr;
    if ((s = dev_alloc(&dv, m)) != SG_OK) break;
    g->fwd.val = dv;
    cudaError_t e;
    if ((e = cudaMemcpyAsync(g->fwd.ro, host_row_offsets, sizeof(uint32_t) * ((uint64_t)n + 1), cudaMemcpyHostToDevice,
                             g->stream)) != cudaSuccess ||
        (m && (e = cudaMemcpyAsync(g->fwd.col, host_column_indices, sizeof(uint32_t) * m, cudaMemcpyHostToDevice,
                                   g->stream)) != cudaSuccess) ||
        (m && (e = cudaMemcpyAsync(dv, vals, sizeof(uint32_t) * m, cudaMemcpyHostToDevice, g->stream)) != cudaSuccess) ||
        (e = cudaStreamSynchronize(g->stream)) != cudaSuccess) {
      s = cuda_fail(e, "graph upload", __FILE__, __LINE__);
      break;
    }
    g->bytes = sizeof(uint32_t) * ((uint64_t)n + 1 + 2 * m);
    if (flags & SG_GRAPH_DIRECTED) {
      if ((s = build_inverse(g, host_row_offsets, host_column_indices, vals)) != SG_OK) break;
    } else {
      g->inv = g->fwd;
      g->owns_inverse = false;
    }
  } while (0);
  if (s != SG_OK) {
    release_graph(g);
    return s;
  }
  *out = g;
  return SG_OK;
}

sg_status sg_graph_destroy(sg_graph g) {
  if (g) {
    cudaStreamSynchronize(g->stream);
    release_graph(g);
  }
  return SG_OK;
}

sg_status sg_graph_info(sg_graph g, uint32_t* n, uint64_t* m, uint32_t* flags, int* value_type) {
  SG_REQUIRE(g, SG_ERR_INVALID, "graph is NULL");
  if (n) *n = g->n;
  if (m) *m = g->m;
  if (flags) *flags = g->flags;
  if (value_type) *value_type = g->value_type;
  return SG_OK;
}

sg_status sg_graph_device_view(sg_graph g, int inverse, sg_graph_view* view) {
  SG_REQUIRE(g && view, SG_ERR_INVALID, "NULL argument");
  *view = g->view(inverse != 0);
  return SG_OK;
}

sg_status sg_graph_set_stream(sg_graph g, void* stream) {
  SG_REQUIRE(g, SG_ERR_INVALID, "graph is NULL");
  g->stream = (cudaStream_t)stream;
  return SG_OK;
}

sg_status sg_graph_copy_csr(sg_graph g, int inverse, uint32_t* host_row_offsets, uint32_t* host_column_indices,
                            void* host_values) {
  SG_REQUIRE(g, SG_ERR_INVALID, "graph is NULL");
  const GraphDir& d = inverse ? g->inv : g->fwd;
  if (host_row_offsets)
    SG_CUDA(cudaMemcpyAsync(host_row_offsets, d.ro, sizeof(uint32_t) * ((uint64_t)g->n + 1), cudaMemcpyDeviceToHost,
                            g->stream));
  if (host_column_indices && g->m)
    SG_CUDA(cudaMemcpyAsync(host_column_indices, d.col, sizeof(uint32_t) * g->m, cudaMemcpyDeviceToHost, g->stream));
  if (host_values && g->m)
    SG_CUDA(cudaMemcpyAsync(host_values, d.val, sizeof(uint32_t) * g->m, cudaMemcpyDeviceToHost, g->stream));
  SG_CUDA(cudaStreamSynchronize(g->stream));
  return SG_OK;
}

sg_status sg_graph_degree(sg_graph g, uint32_t v, uint32_t* degree) {
  SG_REQUIRE(g && degree, SG_ERR_INVALID, "NULL argument");
  SG_REQUIRE(v < g->n, SG_ERR_INVALID, "vertex out of range");
  uint32_t r[2];
  SG_CUDA(cudaMemcpyAsync(r, g->fwd.ro + v, sizeof(r), cudaMemcpyDeviceToHost, g->stream));
  SG_CUDA(cudaStreamSynchronize(g->stream));
  *degree = r[1] - r[0];
  return SG_OK;
}

sg_status sg_graph_memory_bytes(sg_graph g, uint64_t* bytes) {
  SG_REQUIRE(g && bytes, SG_ERR_INVALID, "NULL argument");
  *bytes = g->bytes;
  return SG_OK;
}

}  // extern "C"
