// Brandes betweenness centrality, BC::run (algorithms/bc.hpp:118-200), one
// source at a time.
//
// Depths: the direction-optimising BFS engine (bfs.cu; hybrid, alpha 15,
//   beta 24) -- the reference's forward sweep labels every vertex with its
//   level (bc.hpp:144-153).
// sigma: level by level, every vertex v at depth L gathers the sum of
//   sigma[w] over its in-neighbours w at depth L-1 (the reference adds
//   sigma[src] into sigma[dst] with an atomic for every such edge).  The sum
//   runs in adjacency order, so it is the same bits on every run, and no
//   hub's counter is hit by an atomic per in-edge.
// delta: levels in reverse, as the reference's replay of the saved frontiers
//   (bc.hpp:167-194), as a gather: each vertex v at depth d sums
//   (1+delta[u])/sigma[u] over its out-neighbours u at depth d+1 and
//   multiplies by sigma[v] (the reference's sigma[v]/sigma[u]*(1+delta[u])
//   per edge, with the common factor taken out), then bc[v] += delta[v].
// The depths stay on the device (the reference saves the frontier bitmaps
// of every level to the host).  One kernel does sigma and delta, a grid
// barrier between levels.
#include <vector>

#include "engine_common.cuh"

namespace sgb {
namespace {

using namespace eng;

constexpr uint32_t kBcHeavy = 1024;  // edges per chunk; lists this long are split across the grid

struct BcParams {
  uint32_t n, w0;
  const uint32_t* ro;   // out-edges (successors)
  const uint32_t* col;
  const uint32_t* iro;  // in-edges (predecessors; the forward CSR again when undirected)
  const uint32_t* icol;
  uint32_t source;
  const uint32_t* depth;  // BFS depths, n+1 for unreached vertices
  float* sigma;
  float* delta;
  float* bc;
  uint32_t* max_depth;           // zeroed before the launch
  unsigned long long* heavy_ctr;  // 2: (entries << 32) | chunks of a level's long lists, zeroed before the launch
  uint32_t* heavy_v;              // the level's long-list vertices
  uint32_t* heavy_c;              // their first chunk (increasing with the entry)
  float* partial;                 // one partial sum per chunk
  GridBarrier* bar;
  unsigned long long* result;
};

__device__ __forceinline__ uint32_t bc_chunks(uint32_t deg) { return (deg + kBcHeavy - 1) / kBcHeavy; }

// Sum of term(u) over the vertices u of the edge lists of a warp's lanes
// (lane: [e, end), fewer than kBcHeavy edges) whose depth is `want`: each lane
// walks the first kPullSerial edges of its own list, and the rest of every
// longer list is walked by the whole warp, 32 edges per step (term depends
// on u only, so any lane can evaluate it).  The sums run in a fixed order,
// so repeated runs give the same bits.
template <class Term>
__device__ __forceinline__ float gather_depth(const BcParams& P, const uint32_t* col, bool mine, uint32_t e,
                                              uint32_t end, uint32_t want, Term term) {
  const uint32_t lane = threadIdx.x & 31;
  float acc = 0.0f;
  if (mine) {
    const uint32_t lim = min(end, e + kPullSerial);
    for (; e < lim; e++) {
      const uint32_t u = col[e];
      if (ld_cg(P.depth + u) == want) acc += term(u);
    }
  }
  for (uint32_t left = __ballot_sync(kFullMask, mine && e < end); left; left &= left - 1) {
    const uint32_t j = __ffs(left) - 1;
    const uint32_t jb = __shfl_sync(kFullMask, e, j), je = __shfl_sync(kFullMask, end, j);
    float part = 0.0f;
    for (uint32_t eb = jb; eb < je; eb += 32) {
      const uint32_t ee = eb + lane;
      if (ee < je) {
        const uint32_t u = col[ee];
        if (ld_cg(P.depth + u) == want) part += term(u);
      }
    }
    part = sygraph::detail::warp_sum(part);
    if (lane == j) acc += part;
  }
  return acc;
}

// One level of the sigma sweep (kSigma: v at depth L gathers sigma over its
// in-neighbours at L-1) or of the delta sweep (v at depth L gathers
// (1 + delta[u]) / sigma[u] over its out-neighbours at L+1).  Lists shorter
// than kBcHeavy are done by the warp that owns v; longer ones are deferred
// to a grid-wide list (one atomic reserves the entry and its chunks), their
// chunks summed by all warps into one partial each after a barrier, and
// after another barrier one warp per vertex adds its chunks' partials in
// chunk order.  `ctr` is this level's list counter, `ctr_next` the next
// level's (zeroed here).  Ends with a grid barrier; false when one timed out.
template <bool kSigma>
__device__ __forceinline__ bool bc_level(const BcParams& P, uint32_t L, unsigned long long* ctr,
                                         unsigned long long* ctr_next) {
  const uint32_t gtid = blockIdx.x * blockDim.x + threadIdx.x, nthreads = gridDim.x * blockDim.x;
  const uint32_t lane = threadIdx.x & 31, gwarp = gtid >> 5, nwarps = nthreads >> 5;
  const uint32_t* ro = kSigma ? P.iro : P.ro;
  const uint32_t* col = kSigma ? P.icol : P.col;
  const uint32_t want = kSigma ? L - 1 : L + 1;
  auto term = [&](uint32_t u) -> float {
    return kSigma ? ld_cg(P.sigma + u) : (1.0f + ld_cg(P.delta + u)) / ld_cg(P.sigma + u);
  };
  auto finish = [&](uint32_t v, float q) {
    if (kSigma) {
      st_cg(P.sigma + v, q);
    } else {  // delta[v] = sigma[v] * sum over successors of (1 + delta[u]) / sigma[u]
      const float acc = ld_cg(P.sigma + v) * q;
      st_cg(P.delta + v, acc);
      P.bc[v] += acc;
    }
  };
  for (uint32_t wi = gwarp; wi < P.w0; wi += nwarps) {
    const uint32_t v = wi * 32 + lane;
    const bool mine = v < P.n && ld_cg(P.depth + v) == L;
    if (!__any_sync(kFullMask, mine)) continue;
    const uint32_t b = mine ? ro[v] : 0u, e = mine ? ro[v + 1] : 0u;
    const bool heavy = mine && e - b >= kBcHeavy;
    if (heavy) {
      const unsigned long long o = atomicAdd(ctr, (1ull << 32) | bc_chunks(e - b));
      st_cg(P.heavy_v + (uint32_t)(o >> 32), v);
      st_cg(P.heavy_c + (uint32_t)(o >> 32), (uint32_t)o);
    }
    const bool light = mine && !heavy;
    const float q = gather_depth(P, col, light, b, e, want, term);
    if (light) finish(v, q);
  }
  if (gtid == 0) *ctr_next = 0ull;  // the next level's list starts empty (nobody reads it this level)
  if (!grid_sync(P.bar)) return false;
  const unsigned long long hp = ld_cg(ctr);
  const uint32_t nh = (uint32_t)(hp >> 32), nc = (uint32_t)hp;
  if (nh == 0) return true;  // uniform: every block read the same counter
  for (uint32_t c = gwarp; c < nc; c += nwarps) {
    const uint32_t ent = warp_find_owner(P.heavy_c, nh, c);
    const uint32_t v = ld_cg(P.heavy_v + ent);
    const uint32_t cb = ro[v] + (c - ld_cg(P.heavy_c + ent)) * kBcHeavy;
    const uint32_t ce = min(ro[v + 1], cb + kBcHeavy);
    float part = 0.0f;
    for (uint32_t x = cb + lane; x < ce; x += 32) {
      const uint32_t u = col[x];
      if (ld_cg(P.depth + u) == want) part += term(u);
    }
    part = sygraph::detail::warp_sum(part);
    if (lane == 0) st_cg(P.partial + c, part);
  }
  if (!grid_sync(P.bar)) return false;
  for (uint32_t j = gwarp; j < nh; j += nwarps) {
    const uint32_t v = ld_cg(P.heavy_v + j), first = ld_cg(P.heavy_c + j);
    const uint32_t cnt = bc_chunks(ro[v + 1] - ro[v]);
    float q = 0.0f;
    for (uint32_t k = lane; k < cnt; k += 32) q += ld_cg(P.partial + first + k);
    q = sygraph::detail::warp_sum(q);
    if (lane == 0) finish(v, q);
  }
  return grid_sync(P.bar);
}

__global__ void __launch_bounds__(kThreads, 2) bc_kernel(BcParams P) {
  const uint32_t gtid = blockIdx.x * blockDim.x + threadIdx.x, nthreads = gridDim.x * blockDim.x;
  const uint32_t lane = threadIdx.x & 31;
  const uint32_t n = P.n, src = P.source, inf = n + 1;
  // delta = 0 everywhere (the deepest level keeps it); the deepest level reached
  uint32_t dmax = 0;
  for (uint32_t i = gtid; i < n; i += nthreads) {
    st_cg(P.delta + i, 0.0f);
    const uint32_t d = ld_cg(P.depth + i);
    if (d != inf && d > dmax) dmax = d;
  }
  dmax = __reduce_max_sync(kFullMask, dmax);
  if (lane == 0 && dmax) atomicMax(P.max_depth, dmax);
  if (gtid == 0) st_cg(P.sigma + src, 1.0f);
  if (!grid_sync(P.bar)) return;
  const uint32_t D = ld_cg(P.max_depth);
  uint32_t step = 0;  // alternates the long-list counters
  // sigma, level by level from depth 1: predecessors are at depth L-1
  for (uint32_t L = 1; L <= D; L++, step++)
    if (!bc_level<true>(P, L, P.heavy_ctr + (step & 1), P.heavy_ctr + ((step + 1) & 1))) return;
  // delta, levels in reverse: successors are at depth L+1 (the deepest level
  // has none; the source, at depth 0, gets no share)
  for (int d = (int)D - 1; d >= 1; d--, step++)
    if (!bc_level<false>(P, (uint32_t)d, P.heavy_ctr + (step & 1), P.heavy_ctr + ((step + 1) & 1))) return;
  if (gtid == 0) P.result[0] = D + 1;
}

}  // namespace

struct BcWorkspace {
  uint32_t* small = nullptr;  // max_depth
  unsigned long long* heavy_ctr = nullptr;
  uint32_t* heavy_v = nullptr;
  uint32_t* heavy_c = nullptr;
  float* partial = nullptr;
  GridBarrier* bar = nullptr;
  unsigned long long* result = nullptr;
  float* sigma = nullptr;
  float* delta = nullptr;
  float* bc = nullptr;
  sg_status alloc(uint32_t n, uint64_t m) {
    // a level's long lists: at most m / kBcHeavy vertices, chunks at most
    // twice that (each list has fewer than two chunks per kBcHeavy edges)
    const uint64_t hv = m / kBcHeavy + 1, hc = 2 * (m / kBcHeavy) + 1;
    sg_status s;
    if ((s = dev_alloc(&small, 1)) || (s = dev_alloc(&heavy_ctr, 2)) || (s = dev_alloc(&heavy_v, hv)) ||
        (s = dev_alloc(&heavy_c, hv)) || (s = dev_alloc(&partial, hc)) || (s = dev_alloc(&bar, 1)) ||
        (s = dev_alloc(&result, 4)) || (s = dev_alloc(&sigma, n)) || (s = dev_alloc(&delta, n)) ||
        (s = dev_alloc(&bc, n)))
      return s;
    return SG_OK;
  }
  void release() {
    dev_free(small);
    dev_free(heavy_ctr);
    dev_free(heavy_v);
    dev_free(heavy_c);
    dev_free(partial);
    dev_free(bar);
    dev_free(result);
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
  sg_bfs bfs = nullptr;
  const uint32_t* depth = nullptr;
  sg_status st = ws.alloc(g->n, g->m);
  if (st == SG_OK) st = sg_bfs_create(g, &bfs);
  if (st == SG_OK) st = sg_bfs_distances_device(bfs, &depth);
  cudaStream_t s = g->stream;
  if (st == SG_OK) {
    cudaError_t e = cudaMemsetAsync(ws.bc, 0, sizeof(float) * g->n, s);
    if (e == cudaSuccess) e = cudaMemsetAsync(ws.bar, 0, sizeof(GridBarrier), s);
    if (e != cudaSuccess) st = cuda_fail(e, "memset", __FILE__, __LINE__);
  }
  for (uint32_t i = 0; i < k && st == SG_OK; i++) {
    // depths of this source (the BFS instance runs on the graph's stream)
    if ((st = sg_bfs_init(bfs, host_sources[i])) != SG_OK) break;
    if ((st = sg_bfs_run_async(bfs, SG_BFS_HYBRID, 15.0f, 24.0f)) != SG_OK) break;
    // the arrival count and the depth maximum restart per launch; the error flag persists
    cudaError_t e = cudaMemsetAsync(&ws.bar->count, 0, sizeof(ws.bar->count), s);
    if (e == cudaSuccess) e = cudaMemsetAsync(ws.small, 0, sizeof(uint32_t), s);
    if (e == cudaSuccess) e = cudaMemsetAsync(ws.heavy_ctr, 0, 2 * sizeof(unsigned long long), s);
    if (e != cudaSuccess) {
      st = cuda_fail(e, "memset", __FILE__, __LINE__);
      break;
    }
    BcParams P{g->n,       div_up(g->n, 32), g->fwd.ro,  g->fwd.col, g->inv.ro,  g->inv.col,
               host_sources[i], depth,      ws.sigma,   ws.delta,   ws.bc,      ws.small,
               ws.heavy_ctr, ws.heavy_v,    ws.heavy_c, ws.partial, ws.bar,     ws.result};
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
  if (bfs) sg_bfs_destroy(bfs);
  ws.release();
  return st;
}

}  // extern "C"
