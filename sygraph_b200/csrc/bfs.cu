// Fused direction-optimising BFS: BFS::run (algorithms/bfs.hpp:153-238) with
// its push functor (:185-191), pull functor (:201-207) and hybrid heuristic
// (:284-350), as one persistent cooperative kernel.
//
// Frontier F_L lives in bitmap fb[L%3] with a summary sm[L%3] (bit j of
// summary word k set iff fb word 32k+j is non-zero); vertices of degree >=
// kHeavy are also listed, with their first chunk index, in heavy[L&1] as they
// are discovered.  Per level:
//   push: warps take summary words (skipping empty regions) and expand the
//         light vertices found there 32 at a time, edge-parallel by a shuffle
//         scan; heavy vertices are expanded kChunk edges per warp.  Each
//         unvisited neighbour is claimed with one atomicOr on the visited
//         bitmap; the winner writes depth L+1 and sets its fb / summary bits.
//   pull: one warp per 32 unvisited vertices; each lane scans its in-edges,
//         four at a time, for a neighbour in F_L and stops at the first (the
//         warp takes over long lists); the warp stores the visited and
//         next-frontier words.
//   then: fb / summary of F_{L-1} are cleared, per-CTA totals are added,
//         one grid barrier, and every CTA takes the same direction decision
//         from the same counters.
// One grid barrier per level; no host round trip until the traversal ends.
#include <algorithm>
#include <cstring>
#include <mutex>
#include <vector>

#include "engine_common.cuh"

namespace sgb {
namespace bfs {

using namespace eng;

constexpr uint32_t kHeavy = 256;      // degree from which a vertex is expanded in kChunk-edge chunks
constexpr uint32_t kHeavyBuf = 1024;  // per-CTA staging of newly discovered heavy vertices

struct LevelCounters {
  unsigned long long heavy_packed;  // (entries << 32) | chunks of the heavy list being built
  unsigned long long new_count;
  unsigned long long new_deg;
  unsigned long long pad;
};

struct Params {
  uint32_t n, w0, w1;
  uint64_t m;
  const uint32_t* ro;  // forward CSR
  const uint32_t* col;
  const uint32_t* iro;  // inverse CSR (aliases forward when undirected)
  const uint32_t* icol;
  uint32_t source;
  int mode;      // SG_BFS_PUSH / PULL / HYBRID
  int pull_all;  // pull without short-circuit
  float alpha, beta;
  uint32_t* depth;
  uint32_t* visited;
  const uint32_t* no_in_edges;  // bitmap of vertices no edge reaches: never candidates
  uint32_t* fb;                 // 3 * w0
  uint32_t* sm;                 // 3 * w1
  uint32_t* heavy_v;            // 2 * heavy_cap
  uint32_t* heavy_s;            // 2 * heavy_cap
  uint32_t heavy_cap;
  LevelCounters* cnt;  // 3
  GridBarrier* bar;
  sg_level_record* log;
  unsigned long long* result;  // [iterations, push, pull, visited_vertices, visited_edges]
  const int* schedule;         // optional forced direction per level (0 push, 1 pull), -1 = heuristic
  uint32_t schedule_len;
};

struct Shared {
  uint32_t scan[32];
  unsigned long long red[32];
  uint32_t hv[kHeavyBuf];
  uint32_t hd[kHeavyBuf];
  uint32_t hn;
  uint32_t base_e, base_c;
};

// Per-thread state of one level's expansion.
struct Level {
  const Params* P;
  Shared* S;
  LevelCounters* C;
  uint32_t* fb_next;
  uint32_t* sm_next;
  uint32_t* hv_next;
  uint32_t* hs_next;
  uint32_t next_depth;
  uint32_t n_new = 0;
  unsigned long long deg_new = 0;

  __device__ __forceinline__ void add_heavy(uint32_t u, uint32_t du) {
    const uint32_t i = atomicAdd(&S->hn, 1u);
    if (i < kHeavyBuf) {
      S->hv[i] = u;
      S->hd[i] = du;
    } else {
      const unsigned long long old = atomicAdd(&C->heavy_packed, (1ull << 32) | chunks_of(du));
      hv_next[old >> 32] = u;
      hs_next[old >> 32] = (uint32_t)old;
    }
  }
  // u was discovered at this level (forward degree du); fb bit set by the caller.
  __device__ __forceinline__ void discovered(uint32_t u, uint32_t du) {
    st_cg(P->depth + u, next_depth);
    n_new++;
    deg_new += du;
    if (du >= kHeavy) add_heavy(u, du);
  }
  // push: claim u through the visited bitmap
  __device__ __forceinline__ void visit_push(uint32_t u) {
    if (!sygraph::detail::bit_set_once(P->visited, u)) return;
    const uint32_t du = P->ro[u + 1] - P->ro[u];
    const uint32_t b = 1u << (u & 31);
    if (atomicOr(fb_next + (u >> 5), b) == 0) atomicOr(sm_next + (u >> 10), 1u << ((u >> 5) & 31));
    discovered(u, du);
  }
};

// Expands 32 (vertex, beg, deg) triples of a warp edge-parallel.
__device__ __forceinline__ void expand_group(Level& L, uint32_t beg, uint32_t deg) {
  const uint32_t lane = threadIdx.x & 31;
  const uint32_t incl = warp_inclusive_scan(deg);
  const uint32_t total = __shfl_sync(kFullMask, incl, 31);
  const uint32_t excl = incl - deg;
  for (uint32_t r0 = 0; r0 < total; r0 += 32) {
    const uint32_t r = r0 + lane;
    const bool act = r < total;
    const uint32_t o = warp_owner_of_rank(incl, act ? r : total - 1);
    const uint32_t ob = __shfl_sync(kFullMask, beg, o);
    const uint32_t oe = __shfl_sync(kFullMask, excl, o);
    if (act) L.visit_push(L.P->col[ob + (r - oe)]);
  }
}

__global__ void __launch_bounds__(kThreads, 2) bfs_kernel(Params P) {
  __shared__ Shared S;
  const uint32_t gtid = blockIdx.x * blockDim.x + threadIdx.x;
  const uint32_t nthreads = gridDim.x * blockDim.x;
  const uint32_t lane = threadIdx.x & 31;
  const uint32_t gwarp = gtid >> 5, nwarps = nthreads >> 5;
  const uint32_t n = P.n, w0 = P.w0, w1 = P.w1, src = P.source, inf = n + 1;
  const uint32_t deg_src = P.ro[src + 1] - P.ro[src];

  // ---- init: depth = n+1 except the source; F_0 = {source}; vertices that no
  // edge reaches are pre-marked visited so pull never scans them.
  for (uint32_t i = gtid; i < n; i += nthreads) st_cg(P.depth + i, i == src ? 0u : inf);
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
      z.heavy_packed = (1ull << 32) | chunks_of(deg_src);
      P.heavy_v[0] = src;
      P.heavy_s[0] = 0;
    }
    P.cnt[gtid] = z;
  }
  if (threadIdx.x == 0) S.hn = 0;
  if (!grid_sync(P.bar)) return;

  unsigned long long unexplored = P.m - deg_src;
  unsigned long long frontier_size = 1, frontier_deg = deg_src;
  unsigned long long visited_vertices = 1;
  unsigned long long n_push = 0, n_pull = 0;
  int pull = P.mode == SG_BFS_PULL;

  uint32_t level = 0;
  for (;; level++) {
    if (P.schedule && level < P.schedule_len && P.schedule[level] >= 0) pull = P.schedule[level];
    LevelCounters* C = P.cnt + (level % 3);
    const LevelCounters* Cprev = P.cnt + ((level + 2) % 3);
    uint32_t* fb_cur = P.fb + (size_t)(level % 3) * w0;
    uint32_t* fb_next = P.fb + (size_t)((level + 1) % 3) * w0;
    uint32_t* fb_zero = P.fb + (size_t)((level + 2) % 3) * w0;
    uint32_t* sm_cur = P.sm + (size_t)(level % 3) * w1;
    uint32_t* sm_next = P.sm + (size_t)((level + 1) % 3) * w1;
    uint32_t* sm_zero = P.sm + (size_t)((level + 2) % 3) * w1;
    const uint32_t par = level & 1;
    if (gtid == 0) {
      LevelCounters z = {};
      P.cnt[(level + 1) % 3] = z;
    }
    const uint64_t t0 = gtid == 0 ? sygraph::detail::global_timer_ns() : 0;

    Level L{&P, &S, C, fb_next, sm_next, P.heavy_v + (size_t)(par ^ 1) * P.heavy_cap,
            P.heavy_s + (size_t)(par ^ 1) * P.heavy_cap, level + 1};
    if (!pull) {
      n_push++;
      const unsigned long long hp = ld_cg(&Cprev->heavy_packed);
      const uint32_t n_heavy = (uint32_t)(hp >> 32), n_chunks = (uint32_t)hp;
      const uint32_t* hv_cur = P.heavy_v + (size_t)par * P.heavy_cap;
      const uint32_t* hs_cur = P.heavy_s + (size_t)par * P.heavy_cap;
      const uint32_t units = w1 + n_chunks;
      for (uint32_t unit = gwarp; unit < units; unit += nwarps) {
        if (unit < w1) {
          const uint32_t s = ld_cg(sm_cur + unit);
          if (!s) continue;
          const uint32_t bits = ((s >> lane) & 1u) ? ld_cg(fb_cur + unit * 32 + lane) : 0u;
          const uint32_t c = __popc(bits);
          const uint32_t incl = warp_inclusive_scan(c);
          const uint32_t total = __shfl_sync(kFullMask, incl, 31);
          const uint32_t excl = incl - c;
          for (uint32_t r0 = 0; r0 < total; r0 += 32) {
            const uint32_t r = r0 + lane;
            const bool act = r < total;
            const uint32_t o = warp_owner_of_rank(incl, act ? r : total - 1);
            const uint32_t ob = __shfl_sync(kFullMask, bits, o);
            const uint32_t oe = __shfl_sync(kFullMask, excl, o);
            uint32_t beg = 0, deg = 0;
            if (act) {
              const uint32_t v = (unit * 32 + o) * 32 + select_bit(ob, r - oe);
              beg = P.ro[v];
              deg = P.ro[v + 1] - beg;
              if (deg >= kHeavy) deg = 0;  // expanded through the heavy list
            }
            expand_group(L, beg, deg);
          }
        } else {
          const uint32_t c = unit - w1;
          const uint32_t ent = find_chunk_owner(hs_cur, n_heavy, c);
          const uint32_t v = ld_cg(hv_cur + ent);
          const uint32_t first = ld_cg(hs_cur + ent);
          const uint32_t cb = P.ro[v] + (c - first) * kChunk;
          const uint32_t ce = min(P.ro[v + 1], cb + kChunk);
          for (uint32_t eb = cb; eb < ce; eb += 32) {
            const uint32_t e = eb + lane;
            if (e < ce) L.visit_push(P.col[e]);
          }
        }
      }
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
        const uint32_t lim = P.pull_all ? end : min(end, beg + kPullSerial);
        // four independent column loads and bitmap probes per step
        while (e < lim && (P.pull_all || !found)) {
          const uint32_t c0 = P.icol[e];
          const uint32_t c1 = e + 1 < lim ? P.icol[e + 1] : c0;
          const uint32_t c2 = e + 2 < lim ? P.icol[e + 2] : c0;
          const uint32_t c3 = e + 3 < lim ? P.icol[e + 3] : c0;
          const bool h = bit_test(fb_cur, c0) | bit_test(fb_cur, c1) | bit_test(fb_cur, c2) | bit_test(fb_cur, c3);
          found |= h;
          e += 4;
        }
        if (e > lim) e = lim;
        if (!P.pull_all) {
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
          if (found) L.discovered(v, same ? (end - beg) : (P.ro[v + 1] - P.ro[v]));
          if (lane == 0) {
            st_cg(P.visited + wi, vw | fmask);
            st_cg(fb_next + wi, fmask);
            atomicOr(sm_next + (wi >> 5), 1u << (wi & 31));
          }
        }
      }
    }
    // clear F_{L-1}: only the words its summary flags
    for (uint32_t j = gwarp; j < w1; j += nwarps) {
      const uint32_t s = ld_cg(sm_zero + j);
      if (!s) continue;
      if ((s >> lane) & 1u) st_cg(fb_zero + j * 32 + lane, 0u);
      if (lane == 0) st_cg(sm_zero + j, 0u);
    }
    // staged heavy vertices: one atomic per CTA reserves entries and chunks
    __syncthreads();
    {
      const uint32_t nb = min(S.hn, kHeavyBuf);
      const uint32_t k0 = 2 * threadIdx.x;
      uint32_t my = 0;
      if (k0 < nb) my += chunks_of(S.hd[k0]);
      if (k0 + 1 < nb) my += chunks_of(S.hd[k0 + 1]);
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
          pc += chunks_of(S.hd[k]);
        }
      }
      if (threadIdx.x == 0) S.hn = 0;
    }
    {
      const unsigned long long c = block_sum<unsigned long long>(L.n_new, S.red);
      const unsigned long long d = block_sum<unsigned long long>(L.deg_new, S.red);
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
  uint32_t source = 0;
  bool initialised = false;
  uint32_t w0 = 0;
  uint32_t* depth = nullptr;
  uint32_t* visited = nullptr;
  uint32_t w1 = 0;
  uint32_t* fb = nullptr;
  uint32_t* sm = nullptr;
  uint32_t* no_in = nullptr;
  uint32_t* heavy_v = nullptr;
  uint32_t* heavy_s = nullptr;
  uint32_t heavy_cap = 0;
  bfs::LevelCounters* cnt = nullptr;
  sygraph::detail::GridBarrier* bar = nullptr;
  sg_level_record* log = nullptr;
  unsigned long long* result = nullptr;
  int* schedule = nullptr;
  uint32_t schedule_len = 0;
  uint32_t last_iterations = 0;
  bool fresh = false;  // initialised but not run: depths not written yet
};

static sg_status bfs_materialise(sg_bfs b) {
  if (!b->fresh) return SG_OK;
  bfs::fill_depth_kernel<<<grid_for(b->g->n, 256), 256, 0, b->g->stream>>>(b->depth, b->g->n, b->source);
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
  dev_free(b->heavy_v);
  dev_free(b->heavy_s);
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
  P.w1 = b->w1;
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
  P.no_in_edges = b->no_in;
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
  b->w1 = div_up(b->w0, 32);
  const uint64_t n = g->n;
  // at most m / kHeavy vertices have degree >= kHeavy
  b->heavy_cap = (uint32_t)std::min<uint64_t>(n, g->m / bfs::kHeavy + 1);
  sg_status s = SG_OK;
  if ((s = dev_alloc(&b->depth, n)) || (s = dev_alloc(&b->visited, b->w0)) || (s = dev_alloc(&b->fb, 3ull * b->w0)) ||
      (s = dev_alloc(&b->sm, 3ull * b->w1)) || (s = dev_alloc(&b->no_in, b->w0)) ||
      (s = dev_alloc(&b->heavy_v, 2ull * b->heavy_cap)) || (s = dev_alloc(&b->heavy_s, 2ull * b->heavy_cap)) ||
      (s = dev_alloc(&b->cnt, 3)) || (s = dev_alloc(&b->bar, 1)) || (s = dev_alloc(&b->log, SG_MAX_LOGGED_LEVELS)) ||
      (s = dev_alloc(&b->result, 8))) {
    bfs_release(b);
    return s;
  }
  bfs::no_in_edges_kernel<<<grid_for((uint64_t)b->w0 * 32, 256), 256, 0, g->stream>>>(g->inv.ro, g->n, b->w0,
                                                                                       b->no_in);
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
  SG_REQUIRE(direction >= SG_BFS_PUSH && direction <= SG_BFS_HYBRID, SG_ERR_INVALID, "unknown BFS direction");
  b->fresh = false;
  return bfs_launch(b, direction, alpha, beta, 0);
}

sg_status sg_bfs_run(sg_bfs b, int direction, float alpha, float beta, sg_bfs_details* details) {
  SG_TRY(sg_bfs_run_async(b, direction, alpha, beta));
  return bfs_collect(b, details);
}

sg_status sg_bfs_get_distances(sg_bfs b, uint32_t* host_depth) {
  SG_REQUIRE(b && host_depth, SG_ERR_INVALID, "NULL argument");
  SG_REQUIRE(b->initialised, SG_ERR_NOT_INITIALIZED, "BFS instance not initialized");
  SG_TRY(bfs_materialise(b));
  SG_CUDA(cudaMemcpyAsync(host_depth, b->depth, sizeof(uint32_t) * b->g->n, cudaMemcpyDeviceToHost, b->g->stream));
  SG_CUDA(cudaStreamSynchronize(b->g->stream));
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
  P.pull_all = 0;
  P.alpha = alpha;
  P.beta = beta;
  P.depth = dev_depth;
  P.visited = reinterpret_cast<uint32_t*>(base + kOffVisited);
  uint32_t* no_in = reinterpret_cast<uint32_t*>(base + kOffNoIn);
  P.no_in_edges = no_in;
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
  SG_TRY(eng::launch_persistent(bfs::bfs_kernel, P, 2, s));
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
