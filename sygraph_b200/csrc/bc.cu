// Fused Brandes betweenness centrality, BC::run (algorithms/bc.hpp:118-200),
// one persistent kernel per source.
//
// Forward: the push level loop with the reference's functor (bc.hpp:144-153):
//   CAS labels[dst] from invalid to labels[src]+1; if dst sits on the next
//   level, sigma[dst] += sigma[src]; dst joins the next frontier when this
//   edge discovered it.
// Backward: levels in reverse, as the reference's replay of the saved
//   frontiers (bc.hpp:167-194), but as a gather instead of atomics: each
//   vertex v at depth d sums sigma[v]/sigma[u]*(1+delta[u]) over its
//   neighbours u at depth d+1, then bc[v] += delta[v].  The level of a
//   vertex is its label, so no frontier history leaves the device.
#include <vector>

#include "push_engine.cuh"

namespace sgb {
namespace {

using namespace eng;

struct BcParams {
  PushLoop L;
  uint32_t source;
  uint32_t* labels;
  float* sigma;
  float* delta;
  float* bc;
  unsigned long long* result;
};

struct BcForwardVisitor : NextFrontier {
  using src_t = float;
  uint32_t* labels;
  float* sigma;
  uint32_t next_label;
  __device__ __forceinline__ float src(uint32_t v) const { return ld_cg(sigma + v); }
  __device__ __forceinline__ bool visit(uint32_t u, uint32_t, float sv, uint32_t) {
    uint32_t lbl = ld_cg(labels + u);
    bool won = false;
    if (lbl == 0xffffffffu) {
      const uint32_t old = atomicCAS(labels + u, 0xffffffffu, next_label);
      won = old == 0xffffffffu;
      lbl = won ? next_label : old;
    }
    if (lbl == next_label) atomicAdd(sigma + u, sv);
    return won;
  }
};

__global__ void __launch_bounds__(kThreads, 2) bc_kernel(BcParams P) {
  __shared__ uint32_t s_scan[32];
  __shared__ unsigned long long s_red[32];
  const uint32_t gtid = blockIdx.x * blockDim.x + threadIdx.x, nthreads = gridDim.x * blockDim.x;
  const uint32_t lane = threadIdx.x & 31, gwarp = gtid >> 5, nwarps = nthreads >> 5;
  const uint32_t n = P.L.n, w0 = P.L.w0, src = P.source;
  for (uint32_t i = gtid; i < n; i += nthreads) {
    st_cg(P.labels + i, i == src ? 0u : 0xffffffffu);
    st_cg(P.sigma + i, i == src ? 1.0f : 0.0f);
    st_cg(P.delta + i, 0.0f);
  }
  for (uint32_t i = gtid; i < w0; i += nthreads) {
    st_cg(P.L.fb + i, (i == (src >> 5)) ? (1u << (src & 31)) : 0u);
    st_cg(P.L.fb + w0 + i, 0u);
    st_cg(P.L.fb + 2 * w0 + i, 0u);
  }
  if (gtid < 3) {
    Counters z = {};
    P.L.cnt[gtid] = z;
  }
  if (!grid_sync(P.L.bar)) return;
  const uint32_t levels = push_levels(
      P.L,
      [&](uint32_t level, uint32_t* fb_next) {
        BcForwardVisitor v;
        v.fb_next = fb_next;
        v.labels = P.labels;
        v.sigma = P.sigma;
        v.next_label = level + 1;
        return v;
      },
      s_scan, s_red);
  if (levels == 0) return;
  // Deepest label is levels-1; its vertices have no successors (delta = 0).
  for (int d = (int)levels - 2; d >= 1; d--) {
    const uint32_t du = (uint32_t)d;
    for (uint32_t wi = gwarp; wi < w0; wi += nwarps) {
      const uint32_t v = wi * 32 + lane;
      const bool mine = v < n && ld_cg(P.labels + v) == du;
      if (!__any_sync(kFullMask, mine)) continue;
      float acc = 0.0f;
      uint32_t e = 0, end = 0;
      float sv = 0.0f;
      if (mine) {
        e = P.L.ro[v];
        end = P.L.ro[v + 1];
        sv = ld_cg(P.sigma + v);
        const uint32_t lim = min(end, e + kPullSerial);
        for (; e < lim; e++) {
          const uint32_t u = P.L.col[e];
          if (ld_cg(P.labels + u) == du + 1) acc += sv / ld_cg(P.sigma + u) * (1.0f + ld_cg(P.delta + u));
        }
      }
      uint32_t left = __ballot_sync(kFullMask, mine && e < end);
      while (left) {
        const uint32_t j = __ffs(left) - 1;
        left &= left - 1;
        const uint32_t jb = __shfl_sync(kFullMask, e, j), je = __shfl_sync(kFullMask, end, j);
        const float sj = __shfl_sync(kFullMask, sv, j);
        float part = 0.0f;
        for (uint32_t eb = jb; eb < je; eb += 32) {
          const uint32_t ee = eb + lane;
          if (ee < je) {
            const uint32_t u = P.L.col[ee];
            if (ld_cg(P.labels + u) == du + 1) part += sj / ld_cg(P.sigma + u) * (1.0f + ld_cg(P.delta + u));
          }
        }
        part = sygraph::detail::warp_sum(part);
        if (lane == j) acc += part;
      }
      if (mine) {
        st_cg(P.delta + v, acc);
        P.bc[v] += acc;
      }
    }
    if (!grid_sync(P.L.bar)) return;
  }
  if (gtid == 0) P.result[0] = levels;
}

}  // namespace

struct BcWorkspace {
  uint32_t w0 = 0;
  uint32_t* fb = nullptr;
  Queues q{};
  Counters* cnt = nullptr;
  GridBarrier* bar = nullptr;
  unsigned long long* result = nullptr;
  uint32_t* labels = nullptr;
  float* sigma = nullptr;
  float* delta = nullptr;
  float* bc = nullptr;
  sg_status alloc(uint32_t n) {
    w0 = div_up(n, 32);
    sg_status s;
    if ((s = dev_alloc(&fb, 3ull * w0)) || (s = dev_alloc(&q.small, n)) || (s = dev_alloc(&q.big, n)) ||
        (s = dev_alloc(&q.big_start, n)) || (s = dev_alloc(&cnt, 3)) || (s = dev_alloc(&bar, 1)) ||
        (s = dev_alloc(&result, 4)) || (s = dev_alloc(&labels, n)) || (s = dev_alloc(&sigma, n)) ||
        (s = dev_alloc(&delta, n)) || (s = dev_alloc(&bc, n)))
      return s;
    return SG_OK;
  }
  void release() {
    dev_free(fb);
    dev_free(q.small);
    dev_free(q.big);
    dev_free(q.big_start);
    dev_free(cnt);
    dev_free(bar);
    dev_free(result);
    dev_free(labels);
    dev_free(sigma);
    dev_free(delta);
    dev_free(bc);
  }
};

}  // namespace sgb

using namespace sgb;

extern "C" {

sg_status sg_bc(sg_graph g, const uint32_t* host_sources, uint32_t k, float* host_bc) {
  clear_error();
  SG_REQUIRE(g && host_bc, SG_ERR_INVALID, "NULL argument");
  SG_REQUIRE(k == 0 || host_sources, SG_ERR_INVALID, "sources is NULL");
  SG_REQUIRE(g->n > 0, SG_ERR_INVALID, "graph has no vertices");
  for (uint32_t i = 0; i < k; i++) SG_REQUIRE(host_sources[i] < g->n, SG_ERR_INVALID, "source out of range");
  BcWorkspace ws;
  sg_status st = ws.alloc(g->n);
  cudaStream_t s = g->stream;
  if (st == SG_OK) {
    cudaError_t e = cudaMemsetAsync(ws.bc, 0, sizeof(float) * g->n, s);
    if (e == cudaSuccess) e = cudaMemsetAsync(ws.bar, 0, sizeof(GridBarrier), s);
    if (e != cudaSuccess) st = cuda_fail(e, "memset", __FILE__, __LINE__);
  }
  for (uint32_t i = 0; i < k && st == SG_OK; i++) {
    // the arrival count restarts per launch; the error flag persists
    cudaError_t e = cudaMemsetAsync(&ws.bar->count, 0, sizeof(ws.bar->count), s);
    if (e != cudaSuccess) {
      st = cuda_fail(e, "memset", __FILE__, __LINE__);
      break;
    }
    PushLoop L;
    L.n = g->n;
    L.w0 = ws.w0;
    L.ro = g->fwd.ro;
    L.col = g->fwd.col;
    L.fb = ws.fb;
    L.q = ws.q;
    L.cnt = ws.cnt;
    L.bar = ws.bar;
    BcParams P{L, host_sources[i], ws.labels, ws.sigma, ws.delta, ws.bc, ws.result};
    st = launch_persistent(bc_kernel, P, 2, s);
  }
  if (st == SG_OK) {
    GridBarrier b;
    cudaError_t e = cudaMemcpyAsync(&b, ws.bar, sizeof(b), cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaMemcpyAsync(host_bc, ws.bc, sizeof(float) * g->n, cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    if (e != cudaSuccess) st = cuda_fail(e, "bc copy", __FILE__, __LINE__);
    else if (b.error) st = fail(SG_ERR_TIMEOUT, "BC engine: a grid barrier wait ran out");
  }
  cudaStreamSynchronize(s);
  ws.release();
  return st;
}

}  // extern "C"
