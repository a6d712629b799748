// Exact triangle counting, TC::run + getNumTriangles (algorithms/tc.hpp:67-138).
//
// The reference runs, for every edge (u,v) with u < v, a serial merge of the
// full adjacency lists and adds its running count inside the merge loop
// (tc.hpp:104), which over-counts.  Here:
//   1. orient every edge from the endpoint with the smaller (degree, id) key
//      (the degree-ordered DAG, out-degree O(sqrt m)); lists stay sorted;
//   2. for every DAG edge (u,v), |N+(u) n N+(v)| by walking the shorter list
//      and binary-searching the longer one (segmented intersection);
//   3. each triangle is found exactly once; the total is a uint64 sum.
// The reference's per-vertex convention (for every edge (u,v), u < v,
// |N(u) n N(v)| is added to u) is recovered from the same enumeration: a
// triangle a < b < c adds 2 to a and 1 to b.
#include "internal.cuh"

namespace sgb {
namespace {

using sygraph::detail::block_sum;

__device__ __forceinline__ bool dag_before(uint32_t du, uint32_t u, uint32_t dv, uint32_t v) {
  return du < dv || (du == dv && u < v);
}

__global__ void __launch_bounds__(256) dag_count_kernel(const uint32_t* __restrict__ ro, const uint32_t* __restrict__ col,
                                                        uint32_t n, uint32_t* __restrict__ cnt) {
  for (uint32_t u = blockIdx.x * blockDim.x + threadIdx.x; u < n; u += gridDim.x * blockDim.x) {
    const uint32_t b = ro[u], e = ro[u + 1], du = e - b;
    uint32_t c = 0;
    for (uint32_t i = b; i < e; i++) {
      const uint32_t v = col[i];
      if (dag_before(du, u, ro[v + 1] - ro[v], v)) c++;
    }
    cnt[u] = c;
  }
}

__global__ void __launch_bounds__(256) dag_fill_kernel(const uint32_t* __restrict__ ro, const uint32_t* __restrict__ col,
                                                       uint32_t n, const uint32_t* __restrict__ dro,
                                                       uint32_t* __restrict__ dcol, uint32_t* __restrict__ dsrc) {
  for (uint32_t u = blockIdx.x * blockDim.x + threadIdx.x; u < n; u += gridDim.x * blockDim.x) {
    const uint32_t b = ro[u], e = ro[u + 1], du = e - b;
    uint32_t p = dro[u];
    for (uint32_t i = b; i < e; i++) {
      const uint32_t v = col[i];
      if (dag_before(du, u, ro[v + 1] - ro[v], v)) {
        dcol[p] = v;
        dsrc[p] = u;
        p++;
      }
    }
  }
}

// Exclusive scan in three passes: per-block sums, a scan of those, then the
// per-block scan with its offset.  kItems values per block.
constexpr uint32_t kScanThreads = 256, kScanItems = 8, kScanTile = kScanThreads * kScanItems;

__global__ void __launch_bounds__(kScanThreads) scan_tile_sums(const uint32_t* in, uint32_t n, uint32_t* tile_sums) {
  __shared__ unsigned long long s_red[32];
  const uint32_t base = blockIdx.x * kScanTile;
  unsigned long long s = 0;
  for (uint32_t i = threadIdx.x; i < kScanTile; i += kScanThreads)
    if (base + i < n) s += in[base + i];
  s = block_sum(s, s_red);
  if (threadIdx.x == 0) tile_sums[blockIdx.x] = (uint32_t)s;
}

__global__ void __launch_bounds__(1024) scan_tile_offsets(uint32_t* tile_sums, uint32_t tiles) {
  __shared__ uint32_t s_scan[32];
  __shared__ uint32_t s_carry;
  if (threadIdx.x == 0) s_carry = 0;
  __syncthreads();
  for (uint32_t base = 0; base < tiles; base += blockDim.x) {
    const uint32_t i = base + threadIdx.x;
    const uint32_t v = i < tiles ? tile_sums[i] : 0u;
    uint32_t total;
    const uint32_t ex = sygraph::detail::block_excl_scan(v, &total, s_scan);
    if (i < tiles) tile_sums[i] = s_carry + ex;
    __syncthreads();
    if (threadIdx.x == 0) s_carry += total;
    __syncthreads();
  }
}

__global__ void __launch_bounds__(kScanThreads) scan_tiles(const uint32_t* in, uint32_t n, const uint32_t* tile_off,
                                                           uint32_t* out) {
  __shared__ uint32_t s_scan[32];
  const uint32_t base = blockIdx.x * kScanTile + threadIdx.x * kScanItems;
  uint32_t v[kScanItems], s = 0;
#pragma unroll
  for (uint32_t k = 0; k < kScanItems; k++) {
    v[k] = base + k < n ? in[base + k] : 0u;
    s += v[k];
  }
  uint32_t total;
  uint32_t run = tile_off[blockIdx.x] + sygraph::detail::block_excl_scan(s, &total, s_scan);
#pragma unroll
  for (uint32_t k = 0; k < kScanItems; k++) {
    if (base + k < n) out[base + k] = run;
    run += v[k];
  }
}

template <bool kPerVertex>
__global__ void __launch_bounds__(256) tc_count_kernel(const uint32_t* __restrict__ dro,
                                                       const uint32_t* __restrict__ dcol,
                                                       const uint32_t* __restrict__ dsrc, uint64_t dm,
                                                       unsigned long long* total,
                                                       unsigned long long* __restrict__ per_vertex) {
  __shared__ unsigned long long s_red[32];
  unsigned long long acc = 0;
  for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < dm; i += (uint64_t)gridDim.x * blockDim.x) {
    const uint32_t u = dsrc[i], v = dcol[i];
    uint32_t xb = dro[u], xe = dro[u + 1], yb = dro[v], ye = dro[v + 1];
    if (xe - xb > ye - yb) {
      uint32_t t = xb; xb = yb; yb = t;
      t = xe; xe = ye; ye = t;
    }
    uint32_t lo = yb;
    for (uint32_t e = xb; e < xe && lo < ye; e++) {
      const uint32_t key = dcol[e];
      uint32_t l = lo, h = ye;
      while (l < h) {
        const uint32_t mid = (l + h) >> 1;
        if (dcol[mid] < key)
          l = mid + 1;
        else
          h = mid;
      }
      if (l < ye && dcol[l] == key) {
        acc++;
        if (kPerVertex) {
          uint32_t a = u, b = v, c = key, t;
          if (a > b) { t = a; a = b; b = t; }
          if (b > c) { t = b; b = c; c = t; }
          if (a > b) { t = a; a = b; b = t; }
          atomicAdd(per_vertex + a, 2ull);
          atomicAdd(per_vertex + b, 1ull);
        }
        l++;
      }
      lo = l;
    }
  }
  acc = block_sum(acc, s_red);
  if (threadIdx.x == 0 && acc) atomicAdd(total, acc);
}

}  // namespace

sg_status exclusive_scan_u32(const uint32_t* in, uint32_t n, uint32_t* out, cudaStream_t s) {
  const uint32_t tiles = div_up(n ? n : 1, kScanTile);
  uint32_t* tile = nullptr;
  SG_TRY(dev_alloc(&tile, tiles));
  scan_tile_sums<<<tiles, kScanThreads, 0, s>>>(in, n, tile);
  scan_tile_offsets<<<1, 1024, 0, s>>>(tile, tiles);
  scan_tiles<<<tiles, kScanThreads, 0, s>>>(in, n, tile, out);
  cudaError_t e = cudaGetLastError();
  count_launch(3);
  cudaStreamSynchronize(s);
  cudaFree(tile);
  if (e != cudaSuccess) return cuda_fail(e, "scan launch", __FILE__, __LINE__);
  return SG_OK;
}

}  // namespace sgb

using namespace sgb;

extern "C" {

sg_status sg_tc(sg_graph g, uint64_t* total, uint64_t* host_per_vertex) {
  clear_error();
  SG_REQUIRE(g && total, SG_ERR_INVALID, "NULL argument");
  const uint32_t n = g->n;
  cudaStream_t s = g->stream;
  uint32_t *cnt = nullptr, *dro = nullptr, *dcol = nullptr, *dsrc = nullptr;
  unsigned long long *tot = nullptr, *pv = nullptr;
  sg_status st = SG_OK;
  do {
    if ((st = dev_alloc(&cnt, (uint64_t)n + 1)) || (st = dev_alloc(&dro, (uint64_t)n + 1)) ||
        (st = dev_alloc(&tot, 1)))
      break;
    cudaError_t e = cudaMemsetAsync(cnt, 0, sizeof(uint32_t) * ((uint64_t)n + 1), s);
    if (e != cudaSuccess) { st = cuda_fail(e, "memset", __FILE__, __LINE__); break; }
    dag_count_kernel<<<grid_for(n, 256, 16), 256, 0, s>>>(g->fwd.ro, g->fwd.col, n, cnt);
    if ((e = cudaGetLastError()) != cudaSuccess) { st = cuda_fail(e, "dag count", __FILE__, __LINE__); break; }
    count_launch();
    if ((st = exclusive_scan_u32(cnt, n + 1, dro, s))) break;
    uint32_t dm = 0;
    e = cudaMemcpy(&dm, dro + n, sizeof(uint32_t), cudaMemcpyDeviceToHost);
    if (e != cudaSuccess) { st = cuda_fail(e, "dag size", __FILE__, __LINE__); break; }
    if ((st = dev_alloc(&dcol, dm)) || (st = dev_alloc(&dsrc, dm))) break;
    dag_fill_kernel<<<grid_for(n, 256, 16), 256, 0, s>>>(g->fwd.ro, g->fwd.col, n, dro, dcol, dsrc);
    if ((e = cudaGetLastError()) != cudaSuccess) { st = cuda_fail(e, "dag fill", __FILE__, __LINE__); break; }
    count_launch();
    if ((e = cudaMemsetAsync(tot, 0, sizeof(*tot), s)) != cudaSuccess) { st = cuda_fail(e, "memset", __FILE__, __LINE__); break; }
    if (host_per_vertex) {
      if ((st = dev_alloc(&pv, n))) break;
      if ((e = cudaMemsetAsync(pv, 0, sizeof(*pv) * n, s)) != cudaSuccess) { st = cuda_fail(e, "memset", __FILE__, __LINE__); break; }
      tc_count_kernel<true><<<grid_for(dm, 256, 16), 256, 0, s>>>(dro, dcol, dsrc, dm, tot, pv);
    } else {
      tc_count_kernel<false><<<grid_for(dm, 256, 16), 256, 0, s>>>(dro, dcol, dsrc, dm, tot, nullptr);
    }
    if ((e = cudaGetLastError()) != cudaSuccess) { st = cuda_fail(e, "tc count", __FILE__, __LINE__); break; }
    count_launch();
    unsigned long long t = 0;
    if ((e = cudaMemcpyAsync(&t, tot, sizeof(t), cudaMemcpyDeviceToHost, s)) != cudaSuccess ||
        (host_per_vertex && (e = cudaMemcpyAsync(host_per_vertex, pv, sizeof(*pv) * n, cudaMemcpyDeviceToHost, s)) != cudaSuccess) ||
        (e = cudaStreamSynchronize(s)) != cudaSuccess) {
      st = cuda_fail(e, "tc copy", __FILE__, __LINE__);
      break;
    }
    *total = t;
  } while (0);
  cudaStreamSynchronize(s);
  dev_free(cnt);
  dev_free(dro);
  dev_free(dcol);
  dev_free(dsrc);
  dev_free(tot);
  dev_free(pv);
  return st;
}

}  // extern "C"
