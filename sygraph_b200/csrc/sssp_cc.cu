// Fused SSSP (algorithms/sssp.hpp:152-210) and CC (algorithms/cc.hpp:103-169)
// engines on the shared push level loop.
//
// SSSP: frontier Bellman-Ford.  A frontier vertex v relaxes each out-edge
//   with nd = d[v] + w and atomicMin on d[u] (non-negative floats compare as
//   their bit patterns); u joins the next frontier when its distance dropped
//   (sssp.hpp:180-189).  The reference's filter::external after each advance
//   (sssp.hpp:192-196) only de-duplicates, which the bitmap does.  Every
//   relaxation order reaches the same least fixed point, so distances match
//   Dijkstra bit for bit.
// CC: labels[v] = v, then every vertex pushes its label along its out-edges
//   with atomicMax; a vertex whose label grew joins the next frontier
//   (cc.hpp:135-168).  The fixed point is the maximum id over the vertices
//   that reach v.
#include "push_engine.cuh"

namespace sgb {
namespace {

using namespace eng;

// Near-far bookkeeping of one refill pass (three rotating slots).
struct Refill {
  unsigned long long moved, remaining;
  uint32_t far_min;  // bit pattern of the smallest distance left in the far set
  uint32_t pad[3];
};

template <typename W>
struct SsspParams {
  PushLoop L;
  uint32_t source;
  W* dist;
  const W* w;
  unsigned long long* result;
  uint32_t* far;  // w0 words: improved vertices at or beyond the threshold
  Refill* refill;
  W delta;        // 0: plain frontier Bellman-Ford (every improved vertex is near)
};

// Non-negative floats and unsigned integers both order like their bits.
template <typename W>
__device__ __forceinline__ uint32_t order_bits(W x) {
  if constexpr (sizeof(W) == 4 && W(0.5) != W(0))
    return __float_as_uint(x);
  else
    return (uint32_t)x;
}
template <typename W>
__device__ __forceinline__ W from_order_bits(uint32_t b) {
  if constexpr (sizeof(W) == 4 && W(0.5) != W(0))
    return __uint_as_float(b);
  else
    return (W)b;
}

template <typename W>
struct SsspVisitor : NextFrontier {
  using src_t = W;
  W* dist;
  const W* w;
  uint32_t* far;
  W threshold;
  bool bucketed;
  __device__ __forceinline__ W src(uint32_t v) const { return ld_cg(dist + v); }
  __device__ __forceinline__ bool visit(uint32_t u, uint32_t e, W dv, uint32_t) {
    const W nd = dv + w[e];
    if (!(nd < ld_cg(dist + u))) return false;
    if (!(nd < sygraph::detail::atomic_min_nonneg(dist + u, nd))) return false;
    if (bucketed && !(nd < threshold)) {
      atomicOr(far + (u >> 5), 1u << (u & 31));
      return false;
    }
    return true;
  }
};

template <typename W>
__global__ void __launch_bounds__(kThreads, 2) sssp_kernel(SsspParams<W> P) {
  __shared__ uint32_t s_scan[32];
  __shared__ unsigned long long s_red[32];
  const uint32_t gtid = blockIdx.x * blockDim.x + threadIdx.x, nthreads = gridDim.x * blockDim.x;
  const uint32_t n = P.L.n, w0 = P.L.w0, src = P.source;
  const W inf = (W)(n + 1);  // (weight_t)(size + 1), sssp.hpp:43
  for (uint32_t i = gtid; i < n; i += nthreads) st_cg(P.dist + i, i == src ? (W)0 : inf);
  for (uint32_t i = gtid; i < w0; i += nthreads) {
    st_cg(P.L.fb + i, (i == (src >> 5)) ? (1u << (src & 31)) : 0u);
    st_cg(P.L.fb + w0 + i, 0u);
    st_cg(P.L.fb + 2 * w0 + i, 0u);
  }
  if (gtid < 3) {
    Counters z = {};
    P.L.cnt[gtid] = z;
  }
  const bool bucketed = P.delta > W(0);
  if (bucketed) {
    for (uint32_t i = gtid; i < w0; i += nthreads) st_cg(P.far + i, 0u);
    if (gtid < 3) {
      Refill z = {};
      z.far_min = 0xffffffffu;
      P.refill[gtid] = z;
    }
  }
  if (!grid_sync(P.L.bar)) return;
  // Near-far: vertices improved to a distance below the threshold stay in the
  // frontier, the others wait in the far set; when the near frontier is empty
  // the threshold moves up by delta (or to the far set's minimum) and the far
  // vertices below it become the next frontier.  Every improved vertex is
  // relaxed again before the end, so the fixed point is Bellman-Ford's.
  W threshold = P.delta;
  unsigned long long total = 0;
  uint32_t pass = 0;
  PushLoop loop = P.L;
  for (;;) {
    loop.log_base = (uint32_t)min(total, (unsigned long long)kMaxLog);
    const uint32_t levels = push_levels(
        loop,
        [&](uint32_t, uint32_t* fb_next) {
          SsspVisitor<W> v;
          v.fb_next = fb_next;
          v.dist = P.dist;
          v.w = P.w;
          v.far = P.far;
          v.threshold = threshold;
          v.bucketed = bucketed;
          return v;
        },
        s_scan, s_red);
    if (!levels) return;
    total += levels;
    if (!bucketed) break;
    bool refilled = false;
    for (;;) {
      // far vertices below the new threshold become fb[0]; fb[1], fb[2] cleared
      Refill* R = P.refill + (pass % 3);
      if (gtid == 0) {
        Refill z = {};
        z.far_min = 0xffffffffu;
        P.refill[(pass + 1) % 3] = z;
      }
      if (gtid < 3) {
        Counters z = {};
        P.L.cnt[gtid] = z;
      }
      const W next_t = threshold + P.delta;
      unsigned long long moved = 0, remaining = 0;
      uint32_t fmin = 0xffffffffu;
      for (uint32_t i = gtid; i < w0; i += nthreads) {
        const uint32_t f = ld_cg(P.far + i);
        uint32_t near = 0;
        for (uint32_t b = f; b; b &= b - 1) {
          const uint32_t bit = __ffs(b) - 1;
          const W d = ld_cg(P.dist + i * 32 + bit);
          if (d < next_t)
            near |= 1u << bit;
          else
            fmin = min(fmin, order_bits<W>(d));
        }
        st_cg(P.L.fb + i, near);
        st_cg(P.L.fb + w0 + i, 0u);
        st_cg(P.L.fb + 2 * w0 + i, 0u);
        if (f) st_cg(P.far + i, f & ~near);
        moved += __popc(near);
        remaining += __popc(f & ~near);
      }
      const unsigned long long mv = block_sum<unsigned long long>(moved, s_red);
      const unsigned long long rm = block_sum<unsigned long long>(remaining, s_red);
      fmin = sygraph::detail::warp_min(fmin);
      if ((threadIdx.x & 31) == 0 && fmin != 0xffffffffu) atomicMin(&R->far_min, fmin);
      if (threadIdx.x == 0) {
        if (mv) atomicAdd(&R->moved, mv);
        if (rm) atomicAdd(&R->remaining, rm);
      }
      if (!grid_sync(P.L.bar)) return;
      pass++;
      threshold = next_t;
      if (ld_cg(&R->moved)) {
        refilled = true;
        break;
      }
      if (!ld_cg(&R->remaining)) break;
      // nothing below the new threshold: jump to the far set's minimum
      const W m = from_order_bits<W>(ld_cg(&R->far_min));
      if (threshold < m) threshold = m;
    }
    if (!refilled) break;
  }
  if (gtid == 0) {
    P.result[0] = total;
    P.result[1] = pass;
  }
}

struct CcParams {
  PushLoop L;
  uint32_t* labels;
  unsigned long long* result;
};

struct CcVisitor : NextFrontier {
  using src_t = uint32_t;
  uint32_t* labels;
  __device__ __forceinline__ uint32_t src(uint32_t v) const { return ld_cg(labels + v); }
  __device__ __forceinline__ bool visit(uint32_t u, uint32_t, uint32_t sl, uint32_t) {
    if (ld_cg(labels + u) >= sl) return false;
    return atomicMax(labels + u, sl) < sl;
  }
};

__global__ void __launch_bounds__(kThreads, 2) cc_kernel(CcParams P) {
  __shared__ uint32_t s_scan[32];
  __shared__ unsigned long long s_red[32];
  const uint32_t gtid = blockIdx.x * blockDim.x + threadIdx.x, nthreads = gridDim.x * blockDim.x;
  const uint32_t n = P.L.n, w0 = P.L.w0;
  // labels[i] = i (cc.hpp:121-128); the first level pushes from every vertex,
  // which is the reference's advance::vertices pass (cc.hpp:135-145).
  for (uint32_t i = gtid; i < n; i += nthreads) st_cg(P.labels + i, i);
  for (uint32_t i = gtid; i < w0; i += nthreads) {
    st_cg(P.L.fb + i, valid_bits(i, w0, n));
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
      [&](uint32_t, uint32_t* fb_next) {
        CcVisitor v;
        v.fb_next = fb_next;
        v.labels = P.labels;
        return v;
      },
      s_scan, s_red);
  if (gtid == 0) P.result[0] = levels;
}

}  // namespace

// Workspace shared by the push engines: rotating bitmaps, queues, counters.
struct PushWorkspace {
  uint32_t w0 = 0;
  uint32_t* fb = nullptr;
  Queues q{};
  Counters* cnt = nullptr;
  GridBarrier* bar = nullptr;
  unsigned long long* result = nullptr;
  sg_status alloc(uint32_t n) {
    w0 = div_up(n, 32);
    sg_status s;
    if ((s = dev_alloc(&fb, 3ull * w0)) || (s = dev_alloc(&q.small, n)) || (s = dev_alloc(&q.big, n)) ||
        (s = dev_alloc(&q.big_start, n)) || (s = dev_alloc(&cnt, 3)) || (s = dev_alloc(&bar, 1)) ||
        (s = dev_alloc(&result, 4)))
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
  }
  PushLoop loop(sg_graph g) const {
    PushLoop L;
    L.n = g->n;
    L.w0 = w0;
    L.ro = g->fwd.ro;
    L.col = g->fwd.col;
    L.fb = fb;
    L.q = q;
    L.cnt = cnt;
    L.bar = bar;
    return L;
  }
  sg_status finish(cudaStream_t s, uint64_t* levels) {
    unsigned long long r = 0;
    GridBarrier b;
    SG_CUDA(cudaMemcpyAsync(&r, result, sizeof(r), cudaMemcpyDeviceToHost, s));
    SG_CUDA(cudaMemcpyAsync(&b, bar, sizeof(b), cudaMemcpyDeviceToHost, s));
    SG_CUDA(cudaStreamSynchronize(s));
    if (b.error) return fail(SG_ERR_TIMEOUT, "engine: a grid barrier wait ran out");
    if (levels) *levels = r;
    return SG_OK;
  }
};

}  // namespace sgb

using namespace sgb;

struct sg_sssp_s {
  sg_graph g = nullptr;
  cudaStream_t stream = nullptr;
  uint32_t max_ctas = 0;
  uint32_t source = 0;
  bool initialised = false;
  bool fresh = false;  // initialised but not run: distances not written yet
  void* dist = nullptr;
  sg_level_record* log = nullptr;
  uint32_t* far = nullptr;
  Refill* refill = nullptr;
  double delta = 0.0;  // near-far threshold step; 0 = the reference's frontier Bellman-Ford
  PushWorkspace ws;
};

template <typename W>
__global__ void fill_dist_kernel(W* dist, uint32_t n, uint32_t src) {
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
    dist[i] = i == src ? (W)0 : (W)(n + 1);
}

// SSSPInstance ctor state (sssp.hpp:392-405), written only when distances are
// read before a run.
static sg_status sssp_materialise(sg_sssp s) {
  if (!s->fresh) return SG_OK;
  sg_graph g = s->g;
  if (g->value_type == SG_WEIGHT_F32)
    fill_dist_kernel<float><<<grid_for(g->n, 256), 256, 0, s->stream>>>((float*)s->dist, g->n, s->source);
  else
    fill_dist_kernel<uint32_t><<<grid_for(g->n, 256), 256, 0, s->stream>>>((uint32_t*)s->dist, g->n, s->source);
  SG_CHECK_LAUNCH();
  s->fresh = false;
  return SG_OK;
}

static sg_status sssp_launch(sg_sssp s) {
  sg_graph g = s->g;
  SG_CUDA(cudaMemsetAsync(s->ws.bar, 0, sizeof(GridBarrier), s->stream));
  PushLoop L = s->ws.loop(g);
  L.log = s->log;
  if (g->value_type == SG_WEIGHT_F32) {
    SsspParams<float> P{L, s->source, (float*)s->dist, (const float*)g->fwd.val, s->ws.result,
                        s->far, s->refill, (float)s->delta};
    return launch_persistent(sssp_kernel<float>, P, 2, s->stream, s->max_ctas);
  }
  const uint32_t d = s->delta > 0.0 ? (uint32_t)std::max(1.0, std::min(s->delta, 4294967295.0)) : 0u;
  SsspParams<uint32_t> P{L, s->source, (uint32_t*)s->dist, (const uint32_t*)g->fwd.val, s->ws.result,
                         s->far, s->refill, d};
  return launch_persistent(sssp_kernel<uint32_t>, P, 2, s->stream, s->max_ctas);
}

extern "C" {

sg_status sg_sssp_create(sg_graph g, sg_sssp* out) {
  clear_error();
  SG_REQUIRE(g && out, SG_ERR_INVALID, "NULL argument");
  SG_REQUIRE(g->n > 0, SG_ERR_INVALID, "graph has no vertices");
  *out = nullptr;
  sg_sssp s = new sg_sssp_s();
  s->g = g;
  s->stream = g->stream;
  uint32_t* d = nullptr;
  sg_status st = dev_alloc(&d, g->n);
  s->dist = d;
  if (st == SG_OK) st = s->ws.alloc(g->n);
  if (st == SG_OK) st = dev_alloc(&s->far, div_up(g->n, 32));
  if (st == SG_OK) st = dev_alloc(&s->refill, 3);
  if (st == SG_OK) st = dev_alloc(&s->log, SG_MAX_LOGGED_LEVELS);
  if (st != SG_OK) {
    s->ws.release();
    cudaFree(s->dist);
    dev_free(s->far);
    dev_free(s->refill);
    dev_free(s->log);
    delete s;
    return st;
  }
  *out = s;
  return SG_OK;
}

sg_status sg_sssp_destroy(sg_sssp s) {
  if (s) {
    cudaStreamSynchronize(s->stream);
    s->ws.release();
    cudaFree(s->dist);
    dev_free(s->far);
    dev_free(s->refill);
    dev_free(s->log);
    delete s;
  }
  return SG_OK;
}

sg_status sg_sssp_level_records(sg_sssp s, sg_level_record* host_records, uint32_t cap, uint32_t* count) {
  SG_REQUIRE(s && count, SG_ERR_INVALID, "NULL argument");
  SG_CUDA(cudaStreamSynchronize(s->stream));
  unsigned long long it = 0;
  SG_CUDA(cudaMemcpy(&it, s->ws.result, sizeof(it), cudaMemcpyDeviceToHost));
  uint32_t k = (uint32_t)(it < SG_MAX_LOGGED_LEVELS ? it : SG_MAX_LOGGED_LEVELS);
  if (k > cap) k = cap;
  if (host_records && k) SG_CUDA(cudaMemcpy(host_records, s->log, sizeof(sg_level_record) * k, cudaMemcpyDeviceToHost));
  *count = k;
  return SG_OK;
}

sg_status sg_sssp_set_launch(sg_sssp s, void* stream, uint32_t max_ctas) {
  clear_error();
  SG_REQUIRE(s, SG_ERR_INVALID, "sssp is NULL");
  SG_CUDA(cudaStreamSynchronize(s->stream));
  s->stream = stream ? (cudaStream_t)stream : s->g->stream;
  s->max_ctas = max_ctas;
  return SG_OK;
}

sg_status sg_sssp_set_delta(sg_sssp s, double delta) {
  clear_error();
  SG_REQUIRE(s, SG_ERR_INVALID, "sssp is NULL");
  SG_REQUIRE(delta >= 0.0 && delta < 1e30, SG_ERR_INVALID, "delta must be finite and non-negative");
  s->delta = delta;
  return SG_OK;
}

sg_status sg_sssp_init(sg_sssp s, uint32_t source) {
  clear_error();
  SG_REQUIRE(s, SG_ERR_INVALID, "sssp is NULL");
  SG_REQUIRE(source < s->g->n, SG_ERR_INVALID, "source out of range");
  s->source = source;
  s->initialised = true;
  s->fresh = true;
  return SG_OK;
}

sg_status sg_sssp_run_async(sg_sssp s) {
  clear_error();
  SG_REQUIRE(s, SG_ERR_INVALID, "sssp is NULL");
  SG_REQUIRE(s->initialised, SG_ERR_NOT_INITIALIZED, "SSSP instance not initialized");
  s->fresh = false;
  return sssp_launch(s);
}

sg_status sg_sssp_run(sg_sssp s, uint64_t* iterations) {
  SG_TRY(sg_sssp_run_async(s));
  return s->ws.finish(s->stream, iterations);
}

sg_status sg_sssp_get_distances(sg_sssp s, void* host_dist) {
  SG_REQUIRE(s && host_dist, SG_ERR_INVALID, "NULL argument");
  SG_REQUIRE(s->initialised, SG_ERR_NOT_INITIALIZED, "SSSP instance not initialized");
  SG_TRY(sssp_materialise(s));
  SG_CUDA(cudaMemcpyAsync(host_dist, s->dist, sizeof(uint32_t) * s->g->n, cudaMemcpyDeviceToHost, s->stream));
  SG_CUDA(cudaStreamSynchronize(s->stream));
  return SG_OK;
}

sg_status sg_sssp_distances_device(sg_sssp s, const void** dev_dist) {
  SG_REQUIRE(s && dev_dist, SG_ERR_INVALID, "NULL argument");
  if (s->initialised) SG_TRY(sssp_materialise(s));
  *dev_dist = s->dist;
  return SG_OK;
}

sg_status sg_run_sssp(sg_graph g, uint32_t source, void* host_dist, uint64_t* iterations) {
  sg_sssp s = nullptr;
  SG_TRY(sg_sssp_create(g, &s));
  sg_status st = sg_sssp_init(s, source);
  if (st == SG_OK) st = sg_sssp_run(s, iterations);
  if (st == SG_OK && host_dist) st = sg_sssp_get_distances(s, host_dist);
  sg_sssp_destroy(s);
  return st;
}

sg_status sg_cc(sg_graph g, uint32_t* host_labels, uint64_t* iterations) {
  clear_error();
  SG_REQUIRE(g, SG_ERR_INVALID, "graph is NULL");
  SG_REQUIRE(g->n > 0, SG_ERR_INVALID, "graph has no vertices");
  PushWorkspace ws;
  uint32_t* labels = nullptr;
  sg_status st = ws.alloc(g->n);
  if (st == SG_OK) st = dev_alloc(&labels, g->n);
  if (st == SG_OK) {
    cudaError_t e = cudaMemsetAsync(ws.bar, 0, sizeof(GridBarrier), g->stream);
    if (e != cudaSuccess) st = cuda_fail(e, "memset", __FILE__, __LINE__);
  }
  if (st == SG_OK) {
    CcParams P{ws.loop(g), labels, ws.result};
    st = launch_persistent(cc_kernel, P, 2, g->stream);
  }
  if (st == SG_OK) st = ws.finish(g->stream, iterations);
  if (st == SG_OK && host_labels) {
    cudaError_t e = cudaMemcpy(host_labels, labels, sizeof(uint32_t) * g->n, cudaMemcpyDeviceToHost);
    if (e != cudaSuccess) st = cuda_fail(e, "labels copy", __FILE__, __LINE__);
  }
  cudaStreamSynchronize(g->stream);
  ws.release();
  dev_free(labels);
  return st;
}

}  // extern "C"
