// Fused direction-optimising BFS: BFS::run (algorithms/bfs.hpp:153-238) with
// its push functor (:185-191), pull functor (:201-207) and hybrid heuristic
// (:284-350), as one persistent cooperative kernel.
//
// Per level L (frontier F_L as bitmap fb[L%3]):
//   push: compact F_L into queues | barrier | degree-bucketed expansion that
//         claims each unvisited neighbour with one atomicOr on the visited
//         bitmap, writes depth L+1 and sets its bit in fb[(L+1)%3] | barrier
//   pull: one warp per 32 unvisited vertices; each lane scans its in-edges
//         for a neighbour in F_L (short-circuit), the warp helps long lists,
//         then writes the visited / next-frontier words with plain stores | barrier
// After each level every CTA reads the same counters (|F_{L+1}|, sum of
// degrees) and takes the same direction decision, so no host round trip is
// needed until the traversal ends.  fb[(L+2)%3] is cleared during level L.
#include <cstring>
#include <vector>

#include "engine_common.cuh"

namespace sgb {
namespace bfs {

using namespace eng;

struct Params {
  uint32_t n, w0;
  uint64_t m;
  const uint32_t* ro;   // forward CSR
  const uint32_t* col;
  const uint32_t* iro;  // inverse CSR (aliases forward when undirected)
  const uint32_t* icol;
  uint32_t source;
  int mode;             // SG_BFS_PUSH / PULL / HYBRID
  int pull_all;         // pull without short-circuit
  float alpha, beta;
  uint32_t* depth;
  uint32_t* visited;
  uint32_t* fb;  // 3 * w0
  Queues q;
  Counters* cnt;  // 3
  GridBarrier* bar;
  sg_level_record* log;
  unsigned long long* result;  // [iterations, push, pull, visited_vertices, visited_edges]
  const int* schedule;         // optional forced direction per level (0 push, 1 pull), -1 = heuristic
  uint32_t schedule_len;
};

struct BfsVisitor {
  using src_t = uint32_t;
  uint32_t* visited;
  uint32_t* depth;
  uint32_t* fb_next;
  const uint32_t* ro;
  uint32_t next_depth;
  uint32_t n_new = 0;
  unsigned long long deg_new = 0;
  __device__ __forceinline__ uint32_t src(uint32_t) const { return 0u; }
  __device__ __forceinline__ bool visit(uint32_t u, uint32_t, uint32_t, uint32_t) {
    return sygraph::detail::bit_set_once(visited, u);
  }
  __device__ __forceinline__ void mark(uint32_t u) {
    st_cg(depth + u, next_depth);
    atomicOr(fb_next + (u >> 5), 1u << (u & 31));
    n_new++;
    deg_new += ro[u + 1] - ro[u];
  }
};

__global__ void __launch_bounds__(kThreads, 2) bfs_kernel(Params P) {
  __shared__ uint32_t s_scan[32];
  __shared__ unsigned long long s_red[32];
  const uint32_t gtid = blockIdx.x * blockDim.x + threadIdx.x;
  const uint32_t nthreads = gridDim.x * blockDim.x;
  const uint32_t lane = threadIdx.x & 31;
  const uint32_t gwarp = gtid >> 5, nwarps = nthreads >> 5;
  const uint32_t n = P.n, w0 = P.w0, src = P.source, inf = n + 1;

  // ---- init: depth = n+1 except the source, bitmaps cleared, F_0 = {source}
  for (uint32_t i = gtid; i < n; i += nthreads) st_cg(P.depth + i, i == src ? 0u : inf);
  for (uint32_t i = gtid; i < w0; i += nthreads) {
    const uint32_t b = (i == (src >> 5)) ? (1u << (src & 31)) : 0u;
    st_cg(P.visited + i, b);
    st_cg(P.fb + i, b);
    st_cg(P.fb + w0 + i, 0u);
    st_cg(P.fb + 2 * w0 + i, 0u);
  }
  if (gtid < 3) {
    Counters z = {};
    P.cnt[gtid] = z;
  }
  if (!grid_sync(P.bar)) return;

  const uint32_t deg_src = P.ro[src + 1] - P.ro[src];
  unsigned long long unexplored = P.m - deg_src;
  unsigned long long frontier_size = 1, frontier_deg = deg_src;
  unsigned long long visited_vertices = 1;
  unsigned long long n_push = 0, n_pull = 0;
  int pull = P.mode == SG_BFS_PULL;

  uint32_t level = 0;
  for (;; level++) {
    if (P.schedule && level < P.schedule_len && P.schedule[level] >= 0) pull = P.schedule[level];
    Counters* C = P.cnt + (level % 3);
    uint32_t* fb_cur = P.fb + (size_t)(level % 3) * w0;
    uint32_t* fb_next = P.fb + (size_t)((level + 1) % 3) * w0;
    uint32_t* fb_zero = P.fb + (size_t)((level + 2) % 3) * w0;
    if (gtid == 0) {
      Counters z = {};
      P.cnt[(level + 1) % 3] = z;
    }
    const uint64_t t0 = gtid == 0 ? sygraph::detail::global_timer_ns() : 0;

    BfsVisitor vis{P.visited, P.depth, fb_next, P.ro, level + 1};
    if (!pull) {
      n_push++;
      compact_frontier(fb_cur, w0, P.ro, C, P.q, s_scan);
      if (!grid_sync(P.bar)) return;
      const uint32_t ns = ld_cg(&C->small_tail);
      const unsigned long long bp = ld_cg(&C->big_packed);
      push_expand(P.ro, P.col, P.q, ns, (uint32_t)(bp >> 32), (uint32_t)bp, vis);
    } else {
      n_pull++;
      const bool same = P.iro == P.ro;
      for (uint32_t wi = gwarp; wi < w0; wi += nwarps) {
        const uint32_t vw = ld_cg(P.visited + wi);
        const uint32_t cand = ~vw & valid_bits(wi, w0, n);
        if (!cand) continue;
        const uint32_t v = wi * 32 + lane;
        const bool mine = (cand >> lane) & 1u;
        const uint32_t beg = mine ? P.iro[v] : 0u;
        const uint32_t end = mine ? P.iro[v + 1] : 0u;
        bool found = false;
        uint32_t e = beg;
        if (P.pull_all) {
          for (; e < end; e++)
            if (bit_test(fb_cur, P.icol[e])) found = true;
        } else {
          const uint32_t lim = min(end, beg + kPullSerial);
          for (; e < lim; e++)
            if (bit_test(fb_cur, P.icol[e])) {
              found = true;
              break;
            }
          // long lists that are still unresolved: the whole warp scans them
          uint32_t left = __ballot_sync(kFullMask, mine && !found && e < end);
          while (left) {
            const uint32_t j = __ffs(left) - 1;
            left &= left - 1;
            const uint32_t jb = __shfl_sync(kFullMask, e, j);
            const uint32_t je = __shfl_sync(kFullMask, end, j);
            bool hit = false;
            for (uint32_t eb = jb; eb < je; eb += 32) {
              const uint32_t ee = eb + lane;
              const bool h = ee < je && bit_test(fb_cur, P.icol[ee]);
              if (__any_sync(kFullMask, h)) {
                hit = true;
                break;
              }
            }
            if (lane == j) found = hit;
          }
        }
        const uint32_t fmask = __ballot_sync(kFullMask, found);
        if (fmask) {
          if (found) {
            st_cg(P.depth + v, level + 1);
            vis.n_new++;
            vis.deg_new += same ? (end - beg) : (P.ro[v + 1] - P.ro[v]);
          }
          if (lane == 0) {
            st_cg(P.visited + wi, vw | fmask);
            st_cg(fb_next + wi, fmask);
          }
        }
      }
    }
    for (uint32_t i = gtid; i < w0; i += nthreads) st_cg(fb_zero + i, 0u);
    // one atomic per CTA for the level totals
    {
      const unsigned long long c = block_sum<unsigned long long>(vis.n_new, s_red);
      const unsigned long long d = block_sum<unsigned long long>(vis.deg_new, s_red);
      if (threadIdx.x == 0) {
        if (c) atomicAdd(&C->new_count, c);
        if (d) atomicAdd(&C->new_deg, d);
      }
    }
    if (!grid_sync(P.bar)) return;

    const unsigned long long next_size = ld_cg(&C->new_count);
    const unsigned long long next_deg = ld_cg(&C->new_deg);
    unexplored -= next_deg;
    visited_vertices += next_size;
    if (gtid == 0 && level < kMaxLog) {
      sg_level_record r;
      r.level = level;
      r.strategy = pull ? (P.pull_all ? 4u : 2u) : 0u;
      r.frontier_size = (uint32_t)frontier_size;
      r.next_size = (uint32_t)next_size;
      r.frontier_degree = frontier_deg;
      r.next_degree = next_deg;
      r.unexplored_degree = unexplored;
      r.t_start_ns = t0;
      r.t_end_ns = sygraph::detail::global_timer_ns();
      P.log[level] = r;
    }
    // BFS::evaluateHeuristic (bfs.hpp:325-350), same float arithmetic.
    if (P.mode == SG_BFS_HYBRID) {
      if (!pull) {
        if ((float)(uint32_t)next_deg > (float)(uint32_t)unexplored / P.alpha) pull = 1;
      } else {
        if ((float)next_size < (float)n / P.beta) pull = 0;
      }
    }
    frontier_size = next_size;
    frontier_deg = next_deg;
    if (next_size == 0) break;
  }
  if (gtid == 0) {
    P.result[0] = level + 1;
    P.result[1] = n_push;
    P.result[2] = n_pull;
    P.result[3] = visited_vertices;
    P.result[4] = P.m - unexplored;
  }
}

__global__ void fill_depth_kernel(uint32_t* depth, uint32_t n, uint32_t src) {
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
    depth[i] = i == src ? 0u : n + 1;
}

}  // namespace bfs
}  // namespace sgb

using namespace sgb;

struct sg_bfs_s {
  sg_graph g = nullptr;
  uint32_t source = 0;
  bool initialised = false;
  uint32_t w0 = 0;
  uint32_t* depth = nullptr;
  uint32_t* visited = nullptr;
  uint32_t* fb = nullptr;
  eng::Queues q{};
  eng::Counters* cnt = nullptr;
  sygraph::detail::GridBarrier* bar = nullptr;
  sg_level_record* log = nullptr;
  unsigned long long* result = nullptr;
  int* schedule = nullptr;
  uint32_t schedule_len = 0;
  uint32_t last_iterations = 0;
};

static void bfs_release(sg_bfs b) {
  if (!b) return;
  dev_free(b->depth);
  dev_free(b->visited);
  dev_free(b->fb);
  dev_free(b->q.small);
  dev_free(b->q.big);
  dev_free(b->q.big_start);
  dev_free(b->cnt);
  dev_free(b->bar);
  dev_free(b->log);
  dev_free(b->result);
  dev_free(b->schedule);
  delete b;
}

static sg_status bfs_launch(sg_bfs b, int direction, float alpha, float beta, int pull_all) {
  sg_graph g = b->g;
  bfs::Params P;
  P.n = g->n;
  P.w0 = b->w0;
  P.m = g->m;
  P.ro = g->fwd.ro;
  P.col = g->fwd.col;
  P.iro = g->inv.ro;
  P.icol = g->inv.col;
  P.source = b->source;
  P.mode = direction;
  P.pull_all = pull_all;
  P.alpha = alpha;
  P.beta = beta;
  P.depth = b->depth;
  P.visited = b->visited;
  P.fb = b->fb;
  P.q = b->q;
  P.cnt = b->cnt;
  P.bar = b->bar;
  P.log = b->log;
  P.result = b->result;
  P.schedule = b->schedule_len ? b->schedule : nullptr;
  P.schedule_len = b->schedule_len;
  SG_CUDA(cudaMemsetAsync(b->bar, 0, sizeof(*b->bar), g->stream));
  return eng::launch_persistent(bfs::bfs_kernel, P, 2, g->stream);
}

static sg_status bfs_collect(sg_bfs b, sg_bfs_details* details) {
  unsigned long long res[5];
  sygraph::detail::GridBarrier bar;
  SG_CUDA(cudaMemcpyAsync(res, b->result, sizeof(res), cudaMemcpyDeviceToHost, b->g->stream));
  SG_CUDA(cudaMemcpyAsync(&bar, b->bar, sizeof(bar), cudaMemcpyDeviceToHost, b->g->stream));
  SG_CUDA(cudaStreamSynchronize(b->g->stream));
  if (bar.error) return fail(SG_ERR_TIMEOUT, "BFS engine: a grid barrier wait ran out");
  b->last_iterations = (uint32_t)res[0];
  if (details) {
    memset(details, 0, sizeof(*details));
    details->iterations = res[0];
    details->push_steps = res[1];
    details->pull_steps = res[2];
    details->visited_vertices = res[3];
    details->visited_edges = res[4];
    const uint32_t nlog = res[0] < SG_MAX_LOGGED_LEVELS ? (uint32_t)res[0] : SG_MAX_LOGGED_LEVELS;
    std::vector<sg_level_record> recs(nlog ? nlog : 1);
    if (nlog) {
      SG_CUDA(cudaMemcpy(recs.data(), b->log, sizeof(sg_level_record) * nlog, cudaMemcpyDeviceToHost));
      for (uint32_t i = 0; i < nlog; i++) details->step_is_pull[i] = recs[i].strategy != 0;
    }
  }
  return SG_OK;
}

extern "C" {

sg_status sg_bfs_create(sg_graph g, sg_bfs* out) {
  clear_error();
  SG_REQUIRE(g && out, SG_ERR_INVALID, "NULL argument");
  *out = nullptr;
  SG_REQUIRE(g->n > 0, SG_ERR_INVALID, "graph has no vertices");
  sg_bfs b = new sg_bfs_s();
  b->g = g;
  b->w0 = div_up(g->n, 32);
  const uint64_t n = g->n;
  sg_status s = SG_OK;
  if ((s = dev_alloc(&b->depth, n)) || (s = dev_alloc(&b->visited, b->w0)) || (s = dev_alloc(&b->fb, 3ull * b->w0)) ||
      (s = dev_alloc(&b->q.small, n)) || (s = dev_alloc(&b->q.big, n)) || (s = dev_alloc(&b->q.big_start, n)) ||
      (s = dev_alloc(&b->cnt, 3)) || (s = dev_alloc(&b->bar, 1)) || (s = dev_alloc(&b->log, SG_MAX_LOGGED_LEVELS)) ||
      (s = dev_alloc(&b->result, 8))) {
    bfs_release(b);
    return s;
  }
  *out = b;
  return SG_OK;
}

sg_status sg_bfs_destroy(sg_bfs b) {
  if (b) {
    cudaStreamSynchronize(b->g->stream);
    bfs_release(b);
  }
  return SG_OK;
}

sg_status sg_bfs_init(sg_bfs b, uint32_t source) {
  clear_error();
  SG_REQUIRE(b, SG_ERR_INVALID, "bfs is NULL");
  SG_REQUIRE(source < b->g->n, SG_ERR_INVALID, "source out of range");
  b->source = source;
  b->initialised = true;
  bfs::fill_depth_kernel<<<grid_for(b->g->n, 256), 256, 0, b->g->stream>>>(b->depth, b->g->n, source);
  SG_CHECK_LAUNCH();
  return SG_OK;
}

sg_status sg_bfs_reset(sg_bfs b) {
  SG_REQUIRE(b, SG_ERR_INVALID, "bfs is NULL");
  b->initialised = false;
  return SG_OK;
}

sg_status sg_bfs_run_async(sg_bfs b, int direction, float alpha, float beta) {
  clear_error();
  SG_REQUIRE(b, SG_ERR_INVALID, "bfs is NULL");
  SG_REQUIRE(b->initialised, SG_ERR_NOT_INITIALIZED, "BFS instance not initialized");
  SG_REQUIRE(direction >= SG_BFS_PUSH && direction <= SG_BFS_HYBRID, SG_ERR_INVALID, "unknown BFS direction");
  return bfs_launch(b, direction, alpha, beta, 0);
}

sg_status sg_bfs_run(sg_bfs b, int direction, float alpha, float beta, sg_bfs_details* details) {
  SG_TRY(sg_bfs_run_async(b, direction, alpha, beta));
  return bfs_collect(b, details);
}

sg_status sg_bfs_get_distances(sg_bfs b, uint32_t* host_depth) {
  SG_REQUIRE(b && host_depth, SG_ERR_INVALID, "NULL argument");
  SG_REQUIRE(b->initialised, SG_ERR_NOT_INITIALIZED, "BFS instance not initialized");
  SG_CUDA(cudaMemcpyAsync(host_depth, b->depth, sizeof(uint32_t) * b->g->n, cudaMemcpyDeviceToHost, b->g->stream));
  SG_CUDA(cudaStreamSynchronize(b->g->stream));
  return SG_OK;
}

sg_status sg_bfs_distances_device(sg_bfs b, const uint32_t** dev_depth) {
  SG_REQUIRE(b && dev_depth, SG_ERR_INVALID, "NULL argument");
  *dev_depth = b->depth;
  return SG_OK;
}

sg_status sg_bfs_level_records(sg_bfs b, sg_level_record* host_records, uint32_t cap, uint32_t* count) {
  SG_REQUIRE(b && count, SG_ERR_INVALID, "NULL argument");
  SG_CUDA(cudaStreamSynchronize(b->g->stream));
  unsigned long long it = 0;
  SG_CUDA(cudaMemcpy(&it, b->result, sizeof(it), cudaMemcpyDeviceToHost));
  uint32_t k = (uint32_t)(it < SG_MAX_LOGGED_LEVELS ? it : SG_MAX_LOGGED_LEVELS);
  if (k > cap) k = cap;
  if (host_records && k) SG_CUDA(cudaMemcpy(host_records, b->log, sizeof(sg_level_record) * k, cudaMemcpyDeviceToHost));
  *count = k;
  return SG_OK;
}

sg_status sg_run_bfs(sg_graph g, uint32_t source, int direction, float alpha, float beta, uint32_t* host_depth,
                 sg_bfs_details* details) {
  sg_bfs b = nullptr;
  SG_TRY(sg_bfs_create(g, &b));
  sg_status s = sg_bfs_init(b, source);
  if (s == SG_OK) s = sg_bfs_run(b, direction, alpha, beta, details);
  if (s == SG_OK && host_depth) s = sg_bfs_get_distances(b, host_depth);
  sg_bfs_destroy(b);
  return s;
}

}  // extern "C"
