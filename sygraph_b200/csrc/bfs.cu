// Fused direction-optimising BFS: BFS::run (algorithms/bfs.hpp:153-238) with
// its push functor (:185-191), pull functor (:201-207) and hybrid heuristic
// (:284-350), as one persistent cooperative kernel.
//
// Frontier F_L lives in bitmap fb[L%3] with a summary sm[L%3] (bit j of
// summary word k set iff fb word 32k+j is non-zero); vertices of degree >=
// kHeavy are also listed, with their first chunk index, in heavy[L&1] as they
// are discovered.  Per level, one of six strategies (bfs_strategies.cuh):
//   push (warp- or CTA-mapped): each unvisited neighbour of F_L is claimed
//         with one atomicOr on the visited bitmap; the winner writes depth L+1
//         and sets its fb / summary bits; heavy vertices go in chunks.
//   pull / pull_all (warp- or CTA-mapped): every unvisited vertex scans its
//         in-edges for a neighbour in F_L (pull stops at the first); the
//         owner stores the visited and next-frontier words.
//   then: fb / summary of F_{L-1} are cleared, per-CTA totals are added,
//         one grid barrier, and every CTA takes the same decision for the
//         next level from the same counters: the reference heuristic, a
//         forced schedule, or the learned selector (bfs_engine.cuh).
// One grid barrier per level; no host round trip until the traversal ends.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <memory>
#include <mutex>
#include <vector>

#include "bfs_strategies.cuh"

namespace sgb {
namespace bfs {

using namespace eng;

__global__ void __launch_bounds__(kBfsThreads, 2) bfs_kernel(Params P) {
  __shared__ Shared S;
  const uint32_t gtid = blockIdx.x * blockDim.x + threadIdx.x;
  const uint32_t nthreads = gridDim.x * blockDim.x;
  const uint32_t gwarp = gtid >> 5, nwarps = nthreads >> 5;
  const uint32_t lane = threadIdx.x & 31;
  const uint32_t n = P.n, w0 = P.w0, w1 = P.w1, src = P.source, inf = n + 1;
  const uint32_t deg_src = P.ro[src + 1] - P.ro[src];

  // ---- init: F_0 = {source}; vertices that no edge reaches are pre-marked
  // visited so pull never scans them.  Depths are write-only in the
  // traversal: a vertex's depth is stored when it is discovered, and the
  // unreached ones get n+1 after the last level (the same time as filling all
  // n depths first on RMAT-22, with less traffic).
  // learned mode: the staged parameters arrive by asynchronous copies while
  // the bitmaps are initialised; the init barrier publishes them
  const bool learned = P.mode == kLearned && P.mlp;
  if (learned) sygraph::detail::mlp_stage_async(P.mlp_image, &S.mlp);
  if (gtid == 0) st_cg(P.depth + src, 0u);
  for (uint32_t i = gtid; i < w0; i += nthreads) {
    const uint32_t b = (i == (src >> 5)) ? (1u << (src & 31)) : 0u;
    st_cg(P.visited + i, P.no_in_edges[i] | b);
    st_cg(P.fb + i, b);
    st_cg(P.fb + w0 + i, 0u);
    st_cg(P.fb + 2 * w0 + i, 0u);
  }
  for (uint32_t i = gtid; i < w1; i += nthreads) {
    st_cg(P.sm + i, i == (src >> 10) ? (1u << ((src >> 5) & 31)) : 0u);
    st_cg(P.sm + w1 + i, 0u);
    st_cg(P.sm + 2 * w1 + i, 0u);
  }
  if (gtid < 3) {
    LevelCounters z = {};
    if (gtid == 2 && deg_src >= kHeavy) {
      z.heavy_packed = (1ull << 32) | bfs_chunks(deg_src);
      P.heavy_v[0] = src;
      P.heavy_s[0] = 0;
    }
    P.cnt[gtid] = z;
  }
  if (threadIdx.x == 0) {
    S.hn = 0;
    S.acc[0] = S.acc[1] = 0ull;
  }
  if (threadIdx.x == 0) S.fk = feature_const(P.n, P.m, P.w0, P.w1);
  if (learned) sygraph::detail::mlp_stage_wait();
  if (!grid_sync(P.bar)) return;

  // heavy list of the frontier being expanded, read with the level's other
  // counters right after each barrier
  unsigned long long heavy_packed = ld_cg(&P.cnt[2].heavy_packed);
  unsigned long long unexplored = P.m - deg_src;
  unsigned long long frontier_size = 1, frontier_deg = deg_src, prev_size = 1;
  unsigned long long visited_vertices = 1;
  unsigned long long n_push = 0, n_pull = 0;
  // level 0: the mode's first choice (the reference starts in push unless pull-only)
  int strategy = P.mode == SG_BFS_PULL ? 2 : 0;
  {
    FeatureInputs x{1.0, (double)deg_src, (double)unexplored, 1.0, 1.0, 0};
    const int d = decide(P, S, 0, x, 0, 0.f, 1.f, 1);
    if (P.mode == kLearned) strategy = d;
  }

  uint32_t level = 0;
  for (;; level++) {
    if (P.schedule && level < P.schedule_len && P.schedule[level] >= 0) strategy = P.schedule[level];
    LevelCounters* C = P.cnt + (level % 3);
    const uint32_t* fb_cur = P.fb + (size_t)(level % 3) * w0;
    uint32_t* fb_zero = P.fb + (size_t)((level + 2) % 3) * w0;
    const uint32_t* sm_cur = P.sm + (size_t)(level % 3) * w1;
    uint32_t* sm_zero = P.sm + (size_t)((level + 2) % 3) * w1;
    const uint32_t par = level & 1;
    if (gtid == 0) {
      LevelCounters z = {};
      P.cnt[(level + 1) % 3] = z;
    }
    const uint64_t t0 = gtid == 0 ? sygraph::detail::global_timer_ns() : 0;

    Level L{&P, &S, C, P.fb + (size_t)((level + 1) % 3) * w0, P.sm + (size_t)((level + 1) % 3) * w1,
            P.heavy_v + (size_t)(par ^ 1) * P.heavy_cap, P.heavy_s + (size_t)(par ^ 1) * P.heavy_cap, level + 1,
            frontier_deg < kDirectClaimDeg};
    if (strategy < 2) {
      n_push++;
      const uint32_t n_heavy = (uint32_t)(heavy_packed >> 32), n_chunks = (uint32_t)heavy_packed;
      const uint32_t* hv = P.heavy_v + (size_t)par * P.heavy_cap;
      const uint32_t* hs = P.heavy_s + (size_t)par * P.heavy_cap;
      if (strategy == 0)
        push_warp(L, fb_cur, sm_cur, fb_zero, sm_zero, hv, hs, n_heavy, n_chunks);
      else
        push_cta(L, fb_cur, sm_cur, hv, hs, n_heavy, n_chunks);
    } else {
      n_pull++;
      const bool sc = strategy < 4;
      if (strategy & 1)
        pull_cta(L, fb_cur, sc);
      else
        pull_warp(L, fb_cur, sc, level < 64 && ((P.pull_reverse >> level) & 1ull));
    }
    // clear F_{L-1}: push/warp and the warp-mapped pulls cleared its words in
    // their own word loops (their summary words here, no load needed); the
    // CTA-mapped strategies clear the words its summary flags
    if (strategy == 2 || strategy == 4) {
      for (uint32_t j = gtid; j < w1; j += nthreads) st_cg(sm_zero + j, 0u);
    } else if (strategy != 0) {
      for (uint32_t j = gwarp; j < w1; j += nwarps) {
        const uint32_t s = ld_cg(sm_zero + j);
        if (!s) continue;
        if ((s >> lane) & 1u) st_cg(fb_zero + j * 32 + lane, 0u);
        if (lane == 0) st_cg(sm_zero + j, 0u);
      }
    }
    // level totals: warp sums into shared accumulators, one global atomic per
    // counter and CTA after the barrier below
    {
      unsigned long long v2[2] = {L.n_new, L.deg_new};
#pragma unroll
      for (int k = 0; k < 2; k++) {
        v2[k] = sygraph::detail::warp_sum(v2[k]);
        if (lane == 0 && v2[k]) atomicAdd(&S.acc[k], v2[k]);
      }
    }
    // staged heavy vertices: one atomic per CTA reserves entries and chunks
    __syncthreads();
    if (threadIdx.x == 0) {
      if (S.acc[0]) atomicAdd(&C->new_count, S.acc[0]);
      if (S.acc[1]) atomicAdd(&C->new_deg, S.acc[1]);
      S.acc[0] = S.acc[1] = 0ull;  // next added to after the grid barrier
    }
    if (const uint32_t nb = min(S.hn, kHeavyBuf)) {  // block-uniform; most levels stage none
      const uint32_t k0 = 2 * threadIdx.x;
      uint32_t my = 0;
      if (k0 < nb) my += bfs_chunks(S.hd[k0]);
      if (k0 + 1 < nb) my += bfs_chunks(S.hd[k0 + 1]);
      uint32_t total;
      const uint32_t ex = sygraph::detail::block_excl_scan(my, &total, S.scan);
      if (threadIdx.x == 0 && nb) {
        const unsigned long long old = atomicAdd(&C->heavy_packed, ((unsigned long long)nb << 32) | total);
        S.base_e = (uint32_t)(old >> 32);
        S.base_c = (uint32_t)old;
      }
      __syncthreads();
      if (nb) {
        uint32_t pc = S.base_c + ex;
        for (uint32_t k = k0; k < k0 + 2 && k < nb; k++) {
          L.hv_next[S.base_e + k] = S.hv[k];
          L.hs_next[S.base_e + k] = pc;
          pc += bfs_chunks(S.hd[k]);
        }
      }
      if (threadIdx.x == 0) S.hn = 0;
    }
    if (!grid_sync(P.bar)) return;

    const unsigned long long next_size = ld_cg(&C->new_count);
    const unsigned long long next_deg = ld_cg(&C->new_deg);
    heavy_packed = ld_cg(&C->heavy_packed);
    unexplored -= next_deg;
    visited_vertices += next_size;
    if (gtid == 0 && level < kMaxLog) {
      sg_level_record r;
      r.level = level;
      r.strategy = (uint32_t)strategy;
      r.frontier_size = (uint32_t)frontier_size;
      r.next_size = (uint32_t)next_size;
      r.frontier_degree = frontier_deg;
      r.next_degree = next_deg;
      r.unexplored_degree = unexplored;
      r.t_start_ns = t0;
      r.t_end_ns = sygraph::detail::global_timer_ns();
      P.log[level] = r;
    }
    prev_size = frontier_size;
    frontier_size = next_size;
    frontier_deg = next_deg;
    if (next_size == 0) break;
    FeatureInputs x{(double)next_size, (double)next_deg, (double)unexplored, (double)visited_vertices,
                    (double)prev_size, strategy >= 2};
    // (float)(uint32) casts: the reference's uint32 degree sums (bfs.hpp:327-330)
    strategy = decide(P, S, strategy, x, level + 1, (float)(uint32_t)next_deg, (float)(uint32_t)unexplored,
                      next_size);
  }
  if (gtid == 0) {
    P.result[0] = level + 1;
    P.result[1] = n_push;
    P.result[2] = n_pull;
    P.result[3] = visited_vertices;
    P.result[4] = P.m - unexplored;
  }
  {
    // n+1 for every vertex not reached: reached = visited, minus the vertices
    // pre-marked for having no in-edge, plus the source.  Four vertices per
    // thread (one 16-byte store when none of them was reached).
    const bool vec = (reinterpret_cast<uintptr_t>(P.depth) & 15) == 0;
    const uint32_t nq = (n + 3) / 4;
    for (uint32_t q = gtid; q < nq; q += nthreads) {
      const uint32_t wi = q >> 3;
      uint32_t reached = ld_cg(P.visited + wi) & ~P.no_in_edges[wi];
      if (wi == (src >> 5)) reached |= 1u << (src & 31);
      const uint32_t nib = (reached >> ((q & 7) * 4)) & 0xfu;
      if (nib == 0xfu) continue;
      const uint32_t v0 = 4 * q;
      if (vec && nib == 0 && v0 + 3 < n) {
        st_cg(reinterpret_cast<uint4*>(P.depth) + q, make_uint4(inf, inf, inf, inf));
        continue;
      }
      for (uint32_t k = 0; k < 4 && v0 + k < n; k++)
        if (!((nib >> k) & 1u)) st_cg(P.depth + v0 + k, inf);
    }
  }
  sygraph::detail::grid_exit(P.bar);
}

__global__ void fill_depth_kernel(uint32_t* depth, uint32_t n, uint32_t src) {
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
    depth[i] = i == src ? 0u : n + 1;
}

// First in-neighbour of every vertex (0 for a vertex with none, which is
// never a pull candidate).
__global__ void first_in_kernel(const uint32_t* __restrict__ iro, const uint32_t* __restrict__ icol, uint32_t n,
                                uint32_t* __restrict__ out) {
  for (uint32_t v = blockIdx.x * blockDim.x + threadIdx.x; v < n; v += gridDim.x * blockDim.x) {
    const uint32_t b = iro[v];
    out[v] = b < iro[v + 1] ? icol[b] : 0u;
  }
}

// Bitmap of the vertices with no incoming edge (inverse degree 0).
__global__ void no_in_edges_kernel(const uint32_t* __restrict__ iro, uint32_t n, uint32_t w0, uint32_t* out) {
  const uint32_t lane = threadIdx.x & 31;
  for (uint32_t base = (blockIdx.x * blockDim.x + threadIdx.x) & ~31u; base < (uint64_t)w0 * 32;
       base += gridDim.x * blockDim.x) {
    const uint32_t v = base + lane;
    const bool z = v < n && iro[v + 1] == iro[v];
    const uint32_t m = __ballot_sync(kFullMask, z);
    if (lane == 0) out[base >> 5] = m;
  }
}

}  // namespace bfs
}  // namespace sgb

using namespace sgb;

struct sg_bfs_s {
  sg_graph g = nullptr;
  cudaStream_t stream = nullptr;  // launches and copies (the graph's stream unless set)
  uint32_t max_ctas = 0;          // 0: the whole GPU
  uint32_t source = 0;
  bool initialised = false;
  uint32_t w0 = 0;
  uint32_t* depth = nullptr;
  uint32_t* visited = nullptr;
  uint32_t w1 = 0;
  uint32_t* fb = nullptr;
  uint32_t* sm = nullptr;
  uint32_t* no_in = nullptr;
  uint32_t* first_in = nullptr;  // first in-neighbour of each vertex (the pull's first probe)
  uint32_t* heavy_v = nullptr;
  uint32_t* heavy_s = nullptr;
  uint32_t heavy_cap = 0;
  bfs::LevelCounters* cnt = nullptr;
  sygraph::detail::GridBarrier* bar = nullptr;
  sg_level_record* log = nullptr;
  unsigned long long* result = nullptr;
  int* schedule = nullptr;
  uint32_t schedule_len = 0;
  const sygraph::detail::MlpParams* mlp = nullptr;  // not owned
  uint32_t allowed = 0x3f;
  float margin = 0.05f;
  float min_frontier = 1e-3f;  // learned mode: frontiers below this fraction of n keep the heuristic
  float max_frontier = 1.0f;   // ... and frontiers above this one
  const void* mlp_image = nullptr;  // the MLP's staged image
  // learned mode: the MLP is consulted only on graphs whose mean-degree
  // feature log2(1 + m/n) / 8 lies in [graph_lo, graph_hi]
  float graph_lo = -INFINITY, graph_hi = INFINITY;
  unsigned long long pull_reverse = 0;  // levels whose pull probes in-neighbours from the back
  uint32_t pull_words = bfs::kDefaultPullWords;  // short-circuit pull form (bfs_engine.cuh)
  float* features = nullptr;
  uint32_t last_iterations = 0;
  bool fresh = false;  // initialised but not run: depths not written yet
  // the grid barrier needs a reset before the next launch: set at creation
  // and when a launch reported a barrier timeout (a completed launch resets
  // it itself, grid_exit)
  bool bar_reset = true;
};

static sg_status bfs_materialise(sg_bfs b) {
  if (!b->fresh) return SG_OK;
  bfs::fill_depth_kernel<<<grid_for(b->g->n, 256), 256, 0, b->stream>>>(b->depth, b->g->n, b->source);
  SG_CHECK_LAUNCH();
  b->fresh = false;
  return SG_OK;
}

static void bfs_release(sg_bfs b) {
  if (!b) return;
  dev_free(b->depth);
  dev_free(b->visited);
  dev_free(b->fb);
  dev_free(b->sm);
  dev_free(b->no_in);
  dev_free(b->first_in);
  dev_free(b->heavy_v);
  dev_free(b->heavy_s);
  dev_free(b->cnt);
  dev_free(b->bar);
  dev_free(b->log);
  dev_free(b->result);
  dev_free(b->schedule);
  dev_free(b->features);
  delete b;
}

static sg_status bfs_launch(sg_bfs b, int direction, float alpha, float beta) {
  sg_graph g = b->g;
  bfs::Params P;
  P.n = g->n;
  P.w0 = b->w0;
  P.w1 = b->w1;
  P.m = g->m;
  P.ro = g->fwd.ro;
  P.col = g->fwd.col;
  P.iro = g->inv.ro;
  P.icol = g->inv.col;
  P.source = b->source;
  P.mode = direction;
  P.alpha = alpha;
  P.beta = beta;
  // outside the model's graph range the launch runs without the MLP (no
  // staging, no inference: the heuristic decides every level), as on graphs
  // where the model never overruled the heuristic in training
  const float f9 = log2f(1.f + (float)(g->m ? g->m : 1) / (float)g->n) / 8.f;
  P.mlp = (b->mlp && f9 >= b->graph_lo && f9 <= b->graph_hi) ? b->mlp : nullptr;
  P.allowed = b->allowed;
  P.margin = b->margin;
  P.min_frontier = b->min_frontier;
  P.max_frontier = b->max_frontier;
  P.mlp_image = static_cast<const sygraph::detail::MlpStaged*>(b->mlp_image);
  P.pull_reverse = b->pull_reverse;
  P.pull_words = b->pull_words;
  P.features = b->features;
  P.depth = b->depth;
  P.visited = b->visited;
  P.no_in_edges = b->no_in;
  P.first_in = b->first_in;
  P.fb = b->fb;
  P.sm = b->sm;
  P.heavy_v = b->heavy_v;
  P.heavy_s = b->heavy_s;
  P.heavy_cap = b->heavy_cap;
  P.cnt = b->cnt;
  P.bar = b->bar;
  P.log = b->log;
  P.result = b->result;
  P.schedule = b->schedule_len ? b->schedule : nullptr;
  P.schedule_len = b->schedule_len;
  if (b->bar_reset) {
    SG_CUDA(cudaMemsetAsync(b->bar, 0, sizeof(*b->bar), b->stream));
    b->bar_reset = false;
  }
  return eng::launch_persistent(bfs::bfs_kernel, P, 2, b->stream, b->max_ctas, nullptr, bfs::kBfsThreads);
}

static sg_status bfs_collect(sg_bfs b, sg_bfs_details* details) {
  unsigned long long res[5];
  sygraph::detail::GridBarrier bar;
  SG_CUDA(cudaMemcpyAsync(res, b->result, sizeof(res), cudaMemcpyDeviceToHost, b->stream));
  SG_CUDA(cudaMemcpyAsync(&bar, b->bar, sizeof(bar), cudaMemcpyDeviceToHost, b->stream));
  SG_CUDA(cudaStreamSynchronize(b->stream));
  if (bar.error) {
    b->bar_reset = true;
    return fail(SG_ERR_TIMEOUT, "BFS engine: a grid barrier wait ran out");
  }
  b->last_iterations = (uint32_t)res[0];
  if (details) {
    memset(details, 0, sizeof(*details));
    details->iterations = res[0];
    details->push_steps = res[1];
    details->pull_steps = res[2];
    details->visited_vertices = res[3];
    details->visited_edges = res[4];
    const uint32_t nlog = res[0] < SG_MAX_LOGGED_LEVELS ? (uint32_t)res[0] : SG_MAX_LOGGED_LEVELS;
    // (a std::vector of this C struct trips an internal error of nvcc 12.9's
    // front end under -std=c++20)
    std::unique_ptr<sg_level_record[]> recs(new sg_level_record[nlog ? nlog : 1]);
    if (nlog) {
      SG_CUDA(cudaMemcpy(recs.get(), b->log, sizeof(sg_level_record) * nlog, cudaMemcpyDeviceToHost));
      for (uint32_t i = 0; i < nlog; i++) details->step_is_pull[i] = recs[i].strategy >= 2;
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
  b->stream = g->stream;
  b->w0 = div_up(g->n, 32);
  b->w1 = div_up(b->w0, 32);
  const uint64_t n = g->n;
  // at most m / kHeavy vertices have degree >= kHeavy
  b->heavy_cap = (uint32_t)std::min<uint64_t>(n, g->m / bfs::kHeavy + 1);
  sg_status s = SG_OK;
  if ((s = dev_alloc(&b->depth, n)) || (s = dev_alloc(&b->visited, b->w0)) || (s = dev_alloc(&b->fb, 3ull * b->w0)) ||
      (s = dev_alloc(&b->sm, 3ull * b->w1)) || (s = dev_alloc(&b->no_in, b->w0)) || (s = dev_alloc(&b->first_in, n)) ||
      (s = dev_alloc(&b->heavy_v, 2ull * b->heavy_cap)) || (s = dev_alloc(&b->heavy_s, 2ull * b->heavy_cap)) ||
      (s = dev_alloc(&b->cnt, 3)) || (s = dev_alloc(&b->bar, 1)) || (s = dev_alloc(&b->log, SG_MAX_LOGGED_LEVELS)) ||
      (s = dev_alloc(&b->result, 8))) {
    bfs_release(b);
    return s;
  }
  bfs::no_in_edges_kernel<<<grid_for((uint64_t)b->w0 * 32, 256), 256, 0, g->stream>>>(g->inv.ro, g->n, b->w0,
                                                                                       b->no_in);
  bfs::first_in_kernel<<<grid_for(n, 256), 256, 0, g->stream>>>(g->inv.ro, g->inv.col, g->n, b->first_in);
  if (cudaGetLastError() != cudaSuccess) {
    bfs_release(b);
    return fail(SG_ERR_CUDA, "BFS set-up kernel failed to launch");
  }
  count_launch();
  *out = b;
  return SG_OK;
}

sg_status sg_bfs_destroy(sg_bfs b) {
  if (b) {
    cudaStreamSynchronize(b->stream);
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
  // The traversal kernel writes every depth itself; the initial state
  // (BFSInstance ctor, bfs.hpp:60-73) is materialised only if distances are
  // read before a run.
  b->fresh = true;
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
  SG_REQUIRE(direction >= SG_BFS_PUSH && direction <= SG_BFS_LEARNED, SG_ERR_INVALID, "unknown BFS direction");
  SG_REQUIRE(direction != SG_BFS_LEARNED || b->mlp, SG_ERR_NOT_INITIALIZED,
             "learned mode needs a selector (sg_bfs_set_selector)");
  b->fresh = false;
  return bfs_launch(b, direction, alpha, beta);
}

sg_status sg_bfs_set_launch(sg_bfs b, void* stream, uint32_t max_ctas) {
  clear_error();
  SG_REQUIRE(b, SG_ERR_INVALID, "bfs is NULL");
  SG_CUDA(cudaStreamSynchronize(b->stream));  // set-up work queued on the old stream
  b->stream = stream ? (cudaStream_t)stream : b->g->stream;
  b->max_ctas = max_ctas;
  return SG_OK;
}

sg_status sg_bfs_set_schedule(sg_bfs b, const int* host_strategies, uint32_t len) {
  clear_error();
  SG_REQUIRE(b, SG_ERR_INVALID, "bfs is NULL");
  SG_REQUIRE(len == 0 || host_strategies, SG_ERR_INVALID, "strategies is NULL");
  for (uint32_t i = 0; i < len; i++)
    SG_REQUIRE(host_strategies[i] >= -1 && host_strategies[i] <= 5, SG_ERR_INVALID, "strategy codes are -1..5");
  dev_free(b->schedule);
  b->schedule_len = 0;
  if (len) {
    SG_TRY(dev_alloc(&b->schedule, len));
    SG_CUDA(cudaMemcpy(b->schedule, host_strategies, sizeof(int) * len, cudaMemcpyHostToDevice));
    b->schedule_len = len;
  }
  return SG_OK;
}

}  // extern "C"

sg_status sgb::bfs_launch_status(sg_bfs b) {
  uint32_t err = 0;
  SG_CUDA(cudaMemcpyAsync(&err, &b->bar->error, sizeof(err), cudaMemcpyDeviceToHost, b->stream));
  SG_CUDA(cudaStreamSynchronize(b->stream));
  if (err) b->bar_reset = true;
  return err ? fail(SG_ERR_TIMEOUT, "BFS engine: a grid barrier wait ran out") : SG_OK;
}

extern "C" {

sg_status sg_bfs_set_pull_order(sg_bfs b, uint64_t reverse_levels) {
  clear_error();
  SG_REQUIRE(b, SG_ERR_INVALID, "bfs is NULL");
  b->pull_reverse = reverse_levels;
  return SG_OK;
}

sg_status sg_bfs_set_pull_words(sg_bfs b, uint32_t words) {
  clear_error();
  SG_REQUIRE(b, SG_ERR_INVALID, "bfs is NULL");
  SG_REQUIRE(words == 0 || words == 2 || words == 4, SG_ERR_INVALID,
             "0 (ranked candidates) or 2 or 4 words per warp step");
  b->pull_words = words;
  return SG_OK;
}

sg_status sg_bfs_set_selector_graph_range(sg_bfs b, float lo, float hi) {
  clear_error();
  SG_REQUIRE(b, SG_ERR_INVALID, "bfs is NULL");
  SG_REQUIRE(!(lo != lo) && !(hi != hi), SG_ERR_INVALID, "graph range bounds must be numbers");
  b->graph_lo = lo;
  b->graph_hi = hi;
  return SG_OK;
}

sg_status sg_bfs_set_selector_max_frontier(sg_bfs b, float fraction) {
  clear_error();
  SG_REQUIRE(b, SG_ERR_INVALID, "bfs is NULL");
  SG_REQUIRE(fraction >= 0.f && fraction <= 1.f, SG_ERR_INVALID, "fraction must be in [0, 1]");
  b->max_frontier = fraction;
  return SG_OK;
}

sg_status sg_bfs_set_selector_min_frontier(sg_bfs b, float fraction) {
  clear_error();
  SG_REQUIRE(b, SG_ERR_INVALID, "bfs is NULL");
  SG_REQUIRE(fraction >= 0.f && fraction <= 1.f, SG_ERR_INVALID, "fraction must be in [0, 1]");
  b->min_frontier = fraction;
  return SG_OK;
}

sg_status sg_bfs_set_selector_margin(sg_bfs b, float margin) {
  clear_error();
  SG_REQUIRE(b, SG_ERR_INVALID, "bfs is NULL");
  SG_REQUIRE(margin >= 0.f && margin < 100.f, SG_ERR_INVALID, "margin must be in [0, 100)");
  b->margin = margin;
  return SG_OK;
}

sg_status sg_bfs_set_selector(sg_bfs b, sg_mlp mlp, uint32_t allowed) {
  clear_error();
  SG_REQUIRE(b, SG_ERR_INVALID, "bfs is NULL");
  SG_REQUIRE(!mlp || (allowed & 0x3fu), SG_ERR_INVALID, "no strategy allowed");
  b->mlp = mlp ? static_cast<const sygraph::detail::MlpParams*>(mlp_device_params(mlp)) : nullptr;
  b->mlp_image = mlp ? mlp_device_image(mlp) : nullptr;
  b->allowed = allowed & 0x3fu;
  return SG_OK;
}

sg_status sg_bfs_log_features(sg_bfs b, int enable) {
  clear_error();
  SG_REQUIRE(b, SG_ERR_INVALID, "bfs is NULL");
  if (enable && !b->features) SG_TRY(dev_alloc(&b->features, 12ull * SG_MAX_LOGGED_LEVELS));
  if (!enable) dev_free(b->features);
  return SG_OK;
}

sg_status sg_bfs_level_features(sg_bfs b, float* host_features, uint32_t cap_levels, uint32_t* count) {
  SG_REQUIRE(b && count, SG_ERR_INVALID, "NULL argument");
  SG_REQUIRE(b->features, SG_ERR_NOT_INITIALIZED, "feature logging is off (sg_bfs_log_features)");
  SG_CUDA(cudaStreamSynchronize(b->stream));
  unsigned long long it = 0;
  SG_CUDA(cudaMemcpy(&it, b->result, sizeof(it), cudaMemcpyDeviceToHost));
  uint32_t k = (uint32_t)(it < SG_MAX_LOGGED_LEVELS ? it : SG_MAX_LOGGED_LEVELS);
  if (k > cap_levels) k = cap_levels;
  if (host_features && k)
    SG_CUDA(cudaMemcpy(host_features, b->features, sizeof(float) * 12 * k, cudaMemcpyDeviceToHost));
  *count = k;
  return SG_OK;
}

sg_status sg_bfs_run(sg_bfs b, int direction, float alpha, float beta, sg_bfs_details* details) {
  SG_TRY(sg_bfs_run_async(b, direction, alpha, beta));
  return bfs_collect(b, details);
}

sg_status sg_bfs_get_distances(sg_bfs b, uint32_t* host_depth) {
  SG_REQUIRE(b && host_depth, SG_ERR_INVALID, "NULL argument");
  SG_REQUIRE(b->initialised, SG_ERR_NOT_INITIALIZED, "BFS instance not initialized");
  SG_TRY(bfs_materialise(b));
  SG_CUDA(cudaMemcpyAsync(host_depth, b->depth, sizeof(uint32_t) * b->g->n, cudaMemcpyDeviceToHost, b->stream));
  SG_CUDA(cudaStreamSynchronize(b->stream));
  return SG_OK;
}

sg_status sg_bfs_distances_device(sg_bfs b, const uint32_t** dev_depth) {
  SG_REQUIRE(b && dev_depth, SG_ERR_INVALID, "NULL argument");
  if (b->initialised) SG_TRY(bfs_materialise(b));
  *dev_depth = b->depth;
  return SG_OK;
}

sg_status sg_bfs_level_records(sg_bfs b, sg_level_record* host_records, uint32_t cap, uint32_t* count) {
  SG_REQUIRE(b && count, SG_ERR_INVALID, "NULL argument");
  SG_CUDA(cudaStreamSynchronize(b->stream));
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

// ---------------------------------------------------------------------------
// BFS without any allocation.
//
// Some callers cannot allocate device memory at the moment they need a
// traversal: host code that runs inside a region where the CUDA allocator must
// not be entered (cudaMalloc can synchronise the whole device and take
// milliseconds, which a latency-critical query loop cannot afford), or a
// plug-in embedded in a host application that owns every byte of device
// memory and hands the plug-in only its input and output buffers.  For them,
// sg_bfs_noalloc runs the same traversal kernel as sg_bfs_run with all of its
// working memory in one statically sized device array of this library.
//
// The array is kNoAllocScratchBytes long (about 11 MB) and every GPU that
// loads the library holds it until the process exits.  It bounds the graphs
// this entry point accepts: at most kNoAllocMaxVertices vertices and
// kNoAllocMaxEdges edges; larger graphs are rejected with SG_ERR_INVALID.
// ---------------------------------------------------------------------------
namespace sgb {
namespace bfs_noalloc {

constexpr uint64_t kNoAllocMaxVertices = 1ull << 22;
constexpr uint64_t kNoAllocMaxEdges = 1ull << 27;
constexpr uint64_t kMaxW0 = kNoAllocMaxVertices / 32;
constexpr uint64_t kMaxW1 = kMaxW0 / 32;
constexpr uint64_t kMaxHeavy = kNoAllocMaxEdges / bfs::kHeavy + 1;

constexpr uint64_t align256(uint64_t x) { return (x + 255) & ~255ull; }
// Byte offsets of each region inside the static array.
constexpr uint64_t kOffVisited = 0;
constexpr uint64_t kOffNoIn = kOffVisited + align256(4 * kMaxW0);
constexpr uint64_t kOffFb = kOffNoIn + align256(4 * kMaxW0);
constexpr uint64_t kOffSm = kOffFb + align256(3 * 4 * kMaxW0);
constexpr uint64_t kOffHeavyV = kOffSm + align256(3 * 4 * kMaxW1);
constexpr uint64_t kOffHeavyS = kOffHeavyV + align256(2 * 4 * kMaxHeavy);
constexpr uint64_t kOffCnt = kOffHeavyS + align256(2 * 4 * kMaxHeavy);
constexpr uint64_t kOffBar = kOffCnt + align256(3 * sizeof(bfs::LevelCounters));
constexpr uint64_t kOffLog = kOffBar + align256(sizeof(sygraph::detail::GridBarrier));
constexpr uint64_t kOffResult = kOffLog + align256(SG_MAX_LOGGED_LEVELS * sizeof(sg_level_record));
constexpr uint64_t kNoAllocScratchBytes = kOffResult + align256(8 * sizeof(unsigned long long));

// Working memory of sg_bfs_noalloc; shared by every call on a device.
static __device__ __align__(256) unsigned char g_noalloc_scratch[kNoAllocScratchBytes];

// Device address of g_noalloc_scratch per device, looked up once per device.
static std::mutex g_noalloc_mutex;
static void* g_noalloc_base[64] = {};

static sg_status scratch_base(unsigned char** out) {
  int dev = 0;
  SG_CUDA(cudaGetDevice(&dev));
  SG_REQUIRE(dev >= 0 && dev < 64, SG_ERR_UNSUPPORTED, "device index out of range for the static scratch table");
  std::lock_guard<std::mutex> lock(g_noalloc_mutex);
  if (!g_noalloc_base[dev]) {
    void* p = nullptr;
    cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (e != cudaSuccess) return cuda_fail(e, "cudaGetSymbolAddress(static BFS scratch)", __FILE__, __LINE__);
    SG_REQUIRE(p, SG_ERR_CUDA, "cudaGetSymbolAddress returned NULL for the static BFS scratch");
    g_noalloc_base[dev] = p;
  }
  *out = static_cast<unsigned char*>(g_noalloc_base[dev]);
  return SG_OK;
}

}  // namespace bfs_noalloc
}  // namespace sgb

extern "C" {

sg_status sg_bfs_noalloc(const uint32_t* dev_row_offsets, const uint32_t* dev_column_indices,
                         const uint32_t* dev_inv_row_offsets, const uint32_t* dev_inv_column_indices, uint32_t n,
                         uint64_t m, uint32_t source, int direction, float alpha, float beta, uint32_t* dev_depth,
                         uint64_t* host_iterations, void* stream) {
  using namespace sgb::bfs_noalloc;
  clear_error();
  SG_REQUIRE(dev_row_offsets && dev_depth, SG_ERR_INVALID, "row offsets and depth output are required");
  SG_REQUIRE(m == 0 || dev_column_indices, SG_ERR_INVALID, "column indices are required");
  SG_REQUIRE(n > 0, SG_ERR_INVALID, "graph has no vertices");
  SG_REQUIRE(n <= kNoAllocMaxVertices, SG_ERR_INVALID,
             "sg_bfs_noalloc: vertex count exceeds its static scratch limit of 4194304 (2^22) vertices");
  SG_REQUIRE(m <= kNoAllocMaxEdges, SG_ERR_INVALID,
             "sg_bfs_noalloc: edge count exceeds its static scratch limit of 134217728 (2^27) edges");
  SG_REQUIRE(source < n, SG_ERR_INVALID, "source out of range");
  SG_REQUIRE(direction >= SG_BFS_PUSH && direction <= SG_BFS_HYBRID, SG_ERR_INVALID, "unknown BFS direction");
  if (!dev_inv_row_offsets) {  // an undirected graph is its own inverse
    dev_inv_row_offsets = dev_row_offsets;
    dev_inv_column_indices = dev_column_indices;
  }
  unsigned char* base = nullptr;
  SG_TRY(scratch_base(&base));
  cudaStream_t s = (cudaStream_t)stream;
  // The heavy-vertex lists in the static array are sized from m: a caller's
  // m below the graph's real edge count would let them overflow into the
  // regions after them, so m must be row_offsets[n] of both CSRs.
  {
    uint32_t last[2] = {0, 0};
    SG_CUDA(cudaMemcpyAsync(&last[0], dev_row_offsets + n, sizeof(uint32_t), cudaMemcpyDeviceToHost, s));
    SG_CUDA(cudaMemcpyAsync(&last[1], dev_inv_row_offsets + n, sizeof(uint32_t), cudaMemcpyDeviceToHost, s));
    SG_CUDA(cudaStreamSynchronize(s));
    SG_REQUIRE(last[0] == m && last[1] == m, SG_ERR_INVALID,
               "sg_bfs_noalloc: m must equal row_offsets[n] of the forward and the inverse CSR");
  }
  const uint32_t w0 = div_up(n, 32), w1 = div_up(w0, 32);
  bfs::Params P;
  P.n = n;
  P.w0 = w0;
  P.w1 = w1;
  P.m = m;
  P.ro = dev_row_offsets;
  P.col = dev_column_indices;
  P.iro = dev_inv_row_offsets;
  P.icol = dev_inv_column_indices;
  P.source = source;
  P.mode = direction;
  P.mlp = nullptr;
  P.allowed = 0x3f;
  P.margin = 0.f;
  P.min_frontier = 0.f;
  P.max_frontier = 1.f;
  P.mlp_image = nullptr;
  P.pull_reverse = 0;
  P.pull_words = bfs::kDefaultPullWords;  // the instance default of sg_bfs_create
  P.features = nullptr;
  P.alpha = alpha;
  P.beta = beta;
  P.depth = dev_depth;
  P.visited = reinterpret_cast<uint32_t*>(base + kOffVisited);
  uint32_t* no_in = reinterpret_cast<uint32_t*>(base + kOffNoIn);
  P.no_in_edges = no_in;
  P.first_in = nullptr;  // (no room in the static workspace: read through the offsets)
  P.fb = reinterpret_cast<uint32_t*>(base + kOffFb);
  P.sm = reinterpret_cast<uint32_t*>(base + kOffSm);
  P.heavy_cap = (uint32_t)std::min<uint64_t>(n, m / bfs::kHeavy + 1);
  P.heavy_v = reinterpret_cast<uint32_t*>(base + kOffHeavyV);
  P.heavy_s = reinterpret_cast<uint32_t*>(base + kOffHeavyS);
  P.cnt = reinterpret_cast<bfs::LevelCounters*>(base + kOffCnt);
  P.bar = reinterpret_cast<sygraph::detail::GridBarrier*>(base + kOffBar);
  P.log = reinterpret_cast<sg_level_record*>(base + kOffLog);
  P.result = reinterpret_cast<unsigned long long*>(base + kOffResult);
  P.schedule = nullptr;
  P.schedule_len = 0;
  // The previous call's contents stay in the array: the barrier must start at
  // zero (the kernel initialises every other region it reads).
  SG_CUDA(cudaMemsetAsync(P.bar, 0, sizeof(sygraph::detail::GridBarrier), s));
  bfs::no_in_edges_kernel<<<grid_for((uint64_t)w0 * 32, 256), 256, 0, s>>>(dev_inv_row_offsets, n, w0, no_in);
  SG_CHECK_LAUNCH();
  SG_TRY(eng::launch_persistent(bfs::bfs_kernel, P, 2, s, 0, nullptr, bfs::kBfsThreads));
  unsigned long long it = 0;
  uint32_t err = 0;
  SG_CUDA(cudaMemcpyAsync(&it, P.result, sizeof(it), cudaMemcpyDeviceToHost, s));
  SG_CUDA(cudaMemcpyAsync(&err, &P.bar->error, sizeof(err), cudaMemcpyDeviceToHost, s));
  SG_CUDA(cudaStreamSynchronize(s));
  if (err) return fail(SG_ERR_TIMEOUT, "sg_bfs_noalloc: a grid barrier wait ran out");
  if (host_iterations) *host_iterations = it;
  return SG_OK;
}

}  // extern "C"
