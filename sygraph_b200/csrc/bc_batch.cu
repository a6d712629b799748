// Batched Brandes betweenness centrality: up to 64 sources per launch as
// bit-parallel frontiers (bit s of a vertex's uint64 mask = source s), one
// persistent cooperative kernel for the forward and backward sweeps.
// Per source the arithmetic is BC::run (algorithms/bc.hpp:118-200): sigma by
// forward levels, delta_s(v) = sum over successors u of
// sigma_s(v)/sigma_s(u) * (1 + delta_s(u)), bc[v] += delta_s(v) for v != s.
//
// Layout: hist[L][v] = sources for which v has depth L (one uint64 array per
// level, kept for the backward sweep), seen[v] = OR of hist[0..L][v], and
// sigma / q as vertex-major rows of 64 floats (row v is 256 bytes: lane l of
// a warp holds sources 2l and 2l+1, so a row is one coalesced load), with
// q_s(v) = (1 + delta_s(v)) / sigma_s(v), the one row a successor contributes.
//
// Forward level L, one fused pull pass without atomics: every candidate u
// (a vertex some source has not reached) scans its in-neighbours w in
// adjacency order; m = hist[L][w] & ~seen[u] are the sources reaching u
// through w at depth L+1; u's new mask is the OR of the m's and sigma_s(u)
// the sum of sigma_s(w) over the w with bit s in m, added in adjacency order.
// When the frontier's out-degree is small against the in-degree of the
// vertices not yet done, a mark pass first flags the out-neighbours of the
// frontier and only those are candidates (one more barrier, far less work).
// Light vertices take a warp each (lanes over 32 edges, then over sources,
// with up to kUnroll row loads in flight); vertices of degree >= kCtaDeg take
// a whole CTA whose warps split the list and add their partial sums in warp
// order.  So every sum has a fixed order: results do not depend on scheduling.
//
// Backward level L (from the deepest down to 1): every v with hist[L][v] != 0
// gathers over its out-neighbours u with m = hist[L+1][u] & hist[L][v]:
// acc_s += q_s(u); delta_s(v) = sigma_s(v) * acc_s, q_s(v) is stored and
// bc[v] += the warp's fixed-order sum of delta_s(v) over s in hist[L][v].
//
// One grid barrier per level in each sweep (two on marked forward levels).
// When the depth exceeds the history capacity the kernel stops with a flag
// and the host enlarges the history and runs again.
#include <algorithm>
#include <vector>

#include "engine_common.cuh"

namespace sgb {
namespace bcb {

using namespace eng;
using u64 = unsigned long long;

constexpr uint32_t kCtaDeg = 1024;    // degree from which a vertex is gathered in chunks by many warps
constexpr uint32_t kChunkE = 1024;    // edges per chunk of such a vertex (one warp)
constexpr uint32_t kMarkDeg = 256;    // frontier out-degree from which the whole grid marks its edges
constexpr uint32_t kRow = 64;         // floats per sigma / q row
constexpr uint32_t kUnroll = 8;       // row loads a warp keeps in flight
constexpr uint32_t kSparseRatio = 4;  // mark pass when frontier out-degree * ratio < undone in-degree
constexpr uint32_t kBackwardLog = 7;  // strategy code of backward levels in the level log

struct Counters {
  u64 new_count;  // vertices that gained a source this level
  u64 reached;    // sum over (source, newly reached vertex) of its out-degree
  u64 new_deg;    // out-degree sum of the vertices that gained a source
  u64 done_in;    // in-degree sum of the vertices every source has now reached
  u64 big_packed; // (entries << 32) | chunks of this phase's chunked vertices
  uint32_t mark;       // high-degree vertices of the next frontier (mark list)
  uint32_t next_word;  // words of a dense level handed out so far
  u64 pad[2];
};

struct Params {
  uint32_t n, w0, k;
  uint64_t m;
  const uint32_t* ro;   // out-edges (mark pass, backward sweep, reached-edge counts)
  const uint32_t* col;
  const uint32_t* iro;  // in-edges (forward pull); alias ro / col when undirected
  const uint32_t* icol;
  const uint32_t* sources;
  u64 all;
  u64* seen;
  u64* hist;            // cap_levels * n
  uint32_t cap_levels;
  uint32_t* act;        // cap_levels * w0: hist[L] != 0
  uint32_t* done;       // w0: every source reached (or no in-edge)
  uint32_t* cand;       // w0: marked candidates of a sparse level (zero between levels)
  uint32_t* big;        // big_cap: chunked vertices of the current phase
  uint32_t* big_first;  // big_cap: their first chunk index
  float* part;          // chunk_cap * 64: per-chunk partial sums
  u64* part_mask;       // chunk_cap: per-chunk source masks (forward)
  uint32_t chunk_cap;
  uint32_t* mark;       // 2 * big_cap: frontier vertices of out-degree >= kMarkDeg, by level parity
  uint32_t big_cap;     // > (number of edges) / kMarkDeg
  const uint32_t* no_in_edges;
  float* sigma;         // n * 64
  float* q;             // n * 64
  float* bc;            // n
  int accumulate;       // add into bc instead of overwriting
  Counters* cnt;        // 3 rotating slots
  GridBarrier* bar;
  sg_level_record* log;
  u64* result;          // [forward levels, overflow, reached_edges, log entries]
};

// Levels whose sizes are kept for the backward sweep's choice of word order.
constexpr uint32_t kSizedLevels = 64;

struct Shared {
  uint32_t scan[32];
  u64 red[32];
  uint32_t level_size[kSizedLevels];  // vertices active at each depth (same in every block)
};

// Words of a dense level are handed out one at a time from a per-level
// counter, the next one requested before the current one is processed (its
// latency overlaps the work), so that warps drawing heavy words do not hold
// up the level's barrier.  Levels with few candidates keep the static
// interleaving: most of their words are empty and an atomic per word would
// cost more.
template <class Fn>
__device__ __forceinline__ void for_each_word(bool dynamic, uint32_t* counter, uint32_t w0, uint32_t gwarp,
                                              uint32_t nwarps, Fn&& fn) {
  if (!dynamic) {
    for (uint32_t wi = gwarp; wi < w0; wi += nwarps) fn(wi);
    return;
  }
  const uint32_t lane = threadIdx.x & 31u;
  uint32_t mine = lane == 0 ? atomicAdd(counter, 1u) : 0u;
  uint32_t wi = __shfl_sync(kFullMask, mine, 0);
  while (wi < w0) {
    if (lane == 0) mine = atomicAdd(counter, 1u);
    fn(wi);
    wi = __shfl_sync(kFullMask, mine, 0);
  }
}

struct Local {
  u64 new_count = 0, reached = 0, new_deg = 0, done_in = 0;
};

__device__ __forceinline__ u64 shfl64(u64 x, uint32_t src) {
  const uint32_t lo = __shfl_sync(kFullMask, (uint32_t)x, src);
  const uint32_t hi = __shfl_sync(kFullMask, (uint32_t)(x >> 32), src);
  return ((u64)hi << 32) | lo;
}

__device__ __forceinline__ u64 warp_or64(u64 x) {
#pragma unroll
  for (int d = 16; d > 0; d >>= 1) x |= shfl64(x, (threadIdx.x & 31) ^ d);
  return x;
}

// The two floats of row w that lane `lane` owns (sources 2*lane, 2*lane+1).
// Rows are written in earlier levels by other SMs: loaded through L2.
__device__ __forceinline__ float2 row2(const float* rows, uint32_t w, uint32_t lane) {
  return __ldcg(reinterpret_cast<const float2*>(rows + (size_t)w * kRow) + lane);
}

// Adds, in lane order, the rows of the lanes set in `ball` (warp-uniform):
// lane j of the ballot contributes row x_j to the sources of its mask m_j.
// Up to kUnroll independent row loads are issued before their additions.
__device__ __forceinline__ void add_rows(const float* rows, uint32_t ball, uint32_t x, u64 m, float& a0, float& a1) {
  const uint32_t lane = threadIdx.x & 31;
  while (ball) {
    float2 r[kUnroll];
    uint32_t bs[kUnroll];
#pragma unroll
    for (uint32_t t = 0; t < kUnroll; t++) {
      bs[t] = 0u;
      r[t] = make_float2(0.f, 0.f);
      if (ball) {
        const uint32_t j = __ffs(ball) - 1;
        ball &= ball - 1;
        const uint32_t xj = __shfl_sync(kFullMask, x, j);
        const u64 mj = shfl64(m, j);
        bs[t] = (uint32_t)(mj >> (2 * lane)) & 3u;
        if (bs[t]) r[t] = row2(rows, xj, lane);
      }
    }
#pragma unroll
    for (uint32_t t = 0; t < kUnroll; t++) {
      if (bs[t] & 1u) a0 += r[t].x;
      if (bs[t] & 2u) a1 += r[t].y;
    }
  }
}

// Forward gather over in-edges [beg, end) of u for level L: ORs the masks
// m = hist_L[w] & ~su and adds sigma rows.  Returns the OR (in every lane).
__device__ __forceinline__ u64 forward_gather(const Params& P, const u64* hist_L, uint32_t beg, uint32_t end, u64 su,
                                              float& a0, float& a1) {
  const uint32_t lane = threadIdx.x & 31;
  u64 acc_mask = 0;
  for (uint32_t eb = beg; eb < end; eb += 32) {
    const uint32_t e = eb + lane;
    uint32_t w = 0;
    u64 mw = 0;
    if (e < end) {
      w = P.icol[e];
      mw = __ldcg(hist_L + w) & ~su;
    }
    acc_mask |= mw;
    add_rows(P.sigma, __ballot_sync(kFullMask, mw != 0), w, mw, a0, a1);
  }
  return warp_or64(acc_mask);
}

// Backward gather over out-edges [beg, end) of v: acc_s += q_s(u) for the u
// with bit s in hist_next[u] & fv.
__device__ __forceinline__ void backward_gather(const Params& P, const u64* hist_next, uint32_t beg, uint32_t end,
                                                u64 fv, float& a0, float& a1) {
  const uint32_t lane = threadIdx.x & 31;
  for (uint32_t eb = beg; eb < end; eb += 32) {
    const uint32_t e = eb + lane;
    uint32_t u = 0;
    u64 mu = 0;
    if (e < end) {
      u = P.col[e];
      mu = __ldcg(hist_next + u) & fv;
    }
    add_rows(P.q, __ballot_sync(kFullMask, mu != 0), u, mu, a0, a1);
  }
}

// Forward result of vertex u: seen, hist[L+1], sigma entries of its new
// sources, the act / done bits.  Every lane calls; nm is warp-uniform.
__device__ __forceinline__ void forward_finish(const Params& P, u64* hist_N, uint32_t* act_N, uint32_t* mark_N,
                                               Counters* C, uint32_t u, u64 su, u64 nm, float a0, float a1,
                                               Local& loc) {
  const uint32_t lane = threadIdx.x & 31;
  if (!nm) return;
  const uint32_t b = (uint32_t)(nm >> (2 * lane)) & 3u;
  float* row = P.sigma + (size_t)u * kRow + 2 * lane;
  if (b == 3u) {
    __stcg(reinterpret_cast<float2*>(row), make_float2(a0, a1));
  } else if (b == 1u) {
    __stcg(row, a0);
  } else if (b == 2u) {
    __stcg(row + 1, a1);
  }
  if (lane == 0) {
    const uint32_t dout = P.ro[u + 1] - P.ro[u];
    st_cg(P.seen + u, su | nm);
    st_cg(hist_N + u, nm);
    atomicOr(act_N + (u >> 5), 1u << (u & 31));
    if ((su | nm) == P.all) {
      atomicOr(P.done + (u >> 5), 1u << (u & 31));
      loc.done_in += P.iro[u + 1] - P.iro[u];
    }
    loc.new_count++;
    loc.new_deg += dout;
    if (dout >= kMarkDeg) mark_N[atomicAdd(&C->mark, 1u)] = u;
    loc.reached += (u64)__popcll(nm) * dout;
  }
}

// Backward result of vertex v: delta_s(v) = sigma_s(v) * acc_s for its
// sources at this level, q_s(v) = (1 + delta_s(v)) / sigma_s(v) stored for
// its predecessors, and bc[v] += the fixed-order sum of the deltas.
__device__ __forceinline__ void backward_finish(const Params& P, uint32_t v, u64 fv, float a0, float a1) {
  const uint32_t lane = threadIdx.x & 31;
  const uint32_t b = (uint32_t)(fv >> (2 * lane)) & 3u;
  float d0 = 0.f, d1 = 0.f;
  if (b) {
    const float2 s = row2(P.sigma, v, lane);
    float* row = P.q + (size_t)v * kRow + 2 * lane;
    if (b & 1u) {
      d0 = s.x * a0;
      __stcg(row, (1.0f + d0) / s.x);
    }
    if (b & 2u) {
      d1 = s.y * a1;
      __stcg(row + 1, (1.0f + d1) / s.y);
    }
  }
  float t = d0 + d1;
#pragma unroll
  for (int d = 16; d > 0; d >>= 1) t += __shfl_xor_sync(kFullMask, t, d);
  if (lane == 0) st_cg(P.bc + v, ld_cg(P.bc + v) + t);
}

// Chunked vertices (degree >= kCtaDeg): every warp of the grid takes chunks
// of kChunkE edges (its first owner by a warp-wide search, then the next
// ones), gathers each into its own partial sums; after a grid barrier one
// warp per vertex adds the partials in chunk order (a fixed order, so
// repeated runs give the same bits) and finishes the vertex.
template <bool kForward>
__device__ __forceinline__ void gather_chunks(const Params& P, const u64* hist_src, const u64* hist_N, uint32_t n_big,
                                              uint32_t n_chunks) {
  const uint32_t lane = threadIdx.x & 31;
  const uint32_t gwarp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const uint32_t nwarps = (gridDim.x * blockDim.x) >> 5;
  for (uint32_t c = gwarp; c < n_chunks; c += nwarps) {
    const uint32_t ent = warp_find_owner(P.big_first, n_big, c);
    const uint32_t x = ld_cg(P.big + ent);
    const uint32_t first = ld_cg(P.big_first + ent);
    const uint32_t beg = kForward ? P.iro[x] : P.ro[x];
    const uint32_t end = kForward ? P.iro[x + 1] : P.ro[x + 1];
    const uint32_t cb = beg + (c - first) * kChunkE, ce = min(end, cb + kChunkE);
    const u64 sx = kForward ? ld_cg(P.seen + x) : ld_cg(hist_src + x);
    float a0 = 0.f, a1 = 0.f;
    u64 mk = 0;
    if (kForward)
      mk = forward_gather(P, hist_src, cb, ce, sx, a0, a1);
    else
      backward_gather(P, hist_N, cb, ce, sx, a0, a1);
    __stcg(reinterpret_cast<float2*>(P.part + (size_t)c * kRow) + lane, make_float2(a0, a1));
    if (lane == 0) st_cg(P.part_mask + c, mk);
  }
}

template <bool kForward>
__device__ __forceinline__ void finish_chunked(const Params& P, const u64* hist_src, u64* hist_N, uint32_t* act_N,
                                               uint32_t* mark_N, Counters* C, uint32_t n_big, uint32_t n_chunks,
                                               Local& loc) {
  const uint32_t lane = threadIdx.x & 31;
  const uint32_t gwarp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const uint32_t nwarps = (gridDim.x * blockDim.x) >> 5;
  for (uint32_t ent = gwarp; ent < n_big; ent += nwarps) {
    const uint32_t x = ld_cg(P.big + ent);
    const uint32_t c0 = ld_cg(P.big_first + ent);
    const uint32_t c1 = ent + 1 < n_big ? ld_cg(P.big_first + ent + 1) : n_chunks;
    float t0 = 0.f, t1 = 0.f;
    u64 all = 0;
    for (uint32_t c = c0; c < c1; c++) {
      const float2 pr = __ldcg(reinterpret_cast<const float2*>(P.part + (size_t)c * kRow) + lane);
      t0 += pr.x;
      t1 += pr.y;
      if (kForward) all |= ld_cg(P.part_mask + c);
    }
    if (kForward)
      forward_finish(P, hist_N, act_N, mark_N, C, x, ld_cg(P.seen + x), all, t0, t1, loc);
    else
      backward_finish(P, x, ld_cg(hist_src + x), t0, t1);
  }
}

__device__ __forceinline__ void block_add(Local& loc, Shared& S, Counters* C) {
  const u64 a = block_sum<u64>(loc.new_count, S.red);
  const u64 b = block_sum<u64>(loc.reached, S.red);
  const u64 c = block_sum<u64>(loc.new_deg, S.red);
  const u64 d = block_sum<u64>(loc.done_in, S.red);
  if (threadIdx.x == 0) {
    if (a) atomicAdd(&C->new_count, a);
    if (b) atomicAdd(&C->reached, b);
    if (c) atomicAdd(&C->new_deg, c);
    if (d) atomicAdd(&C->done_in, d);
  }
}

// Appends vertex x of degree >= kCtaDeg, with its first chunk index, to the
// phase's chunked list (one atomic reserves the entry and its chunks, so the
// first-chunk indices increase with the entries); true when deferred.
// Warp-uniform.
__device__ __forceinline__ bool defer_big(const Params& P, Counters* C, uint32_t x, uint32_t deg) {
  if (deg < kCtaDeg) return false;
  if ((threadIdx.x & 31) == 0) {
    const u64 old = atomicAdd(&C->big_packed, (1ull << 32) | ((deg + kChunkE - 1) / kChunkE));
    P.big[old >> 32] = x;
    P.big_first[old >> 32] = (uint32_t)old;
  }
  return true;
}

__device__ __forceinline__ void mark_one(const Params& P, uint32_t u) {
  const uint32_t b = 1u << (u & 31);
  if ((ld_cg(P.done + (u >> 5)) & b) || (ld_cg(P.cand + (u >> 5)) & b)) return;
  atomicOr(P.cand + (u >> 5), b);
}

// Mark pass of a sparse level: out-neighbours of the frontier that some
// source has not reached become candidates (idempotent bit sets).  Frontier
// vertices of out-degree < kMarkDeg take a warp each; the others, listed when
// they joined the frontier, take a CTA each, round-robin over the grid.
__device__ __forceinline__ void mark_candidates(const Params& P, const uint32_t* act_L, const uint32_t* mark_L,
                                                uint32_t n_mark) {
  const uint32_t lane = threadIdx.x & 31;
  const uint32_t gwarp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const uint32_t nwarps = (gridDim.x * blockDim.x) >> 5;
  for (uint32_t wi = gwarp; wi < P.w0; wi += nwarps) {
    uint32_t word = ld_cg(act_L + wi);
    while (word) {
      const uint32_t v = wi * 32 + (__ffs(word) - 1);
      word &= word - 1;
      const uint32_t beg = P.ro[v], end = P.ro[v + 1];
      if (end - beg >= kMarkDeg) continue;
      for (uint32_t e = beg + lane; e < end; e += 32) mark_one(P, P.col[e]);
    }
  }
  for (uint32_t i = blockIdx.x; i < n_mark; i += gridDim.x) {
    const uint32_t v = ld_cg(mark_L + i);
    const uint32_t beg = P.ro[v], end = P.ro[v + 1];
    for (uint32_t e = beg + threadIdx.x; e < end; e += blockDim.x) mark_one(P, P.col[e]);
  }
}

__global__ void __launch_bounds__(kThreads, 2) bc_batch_kernel(Params P) {
  __shared__ Shared S;
  const uint32_t gtid = blockIdx.x * blockDim.x + threadIdx.x;
  const uint32_t nthreads = gridDim.x * blockDim.x;
  const uint32_t gwarp = gtid >> 5, nwarps = nthreads >> 5;
  const uint32_t n = P.n, w0 = P.w0;

  // ---- clear: seen, hist[0..1], act[0..1], cand, done = no in-edges, bc
  for (uint32_t i = gtid; i < n; i += nthreads) {
    st_cg(P.seen + i, 0ull);
    st_cg(P.hist + i, 0ull);
    st_cg(P.hist + (size_t)n + i, 0ull);
    if (!P.accumulate) st_cg(P.bc + i, 0.f);
  }
  for (uint32_t i = gtid; i < w0; i += nthreads) {
    st_cg(P.act + i, 0u);
    st_cg(P.act + w0 + i, 0u);
    st_cg(P.cand + i, 0u);
    st_cg(P.done + i, P.no_in_edges[i]);
  }
  if (gtid < 3) {
    Counters z = {};
    P.cnt[gtid] = z;
  }
  if (!grid_sync(P.bar)) return;
  // ---- sources: depth 0, sigma 1; high-degree sources go on the level-0 mark list
  u64 reached_total = 0, frontier_deg = 0;
  for (uint32_t i = 0; i < P.k; i++) {
    const uint32_t d = P.ro[P.sources[i] + 1] - P.ro[P.sources[i]];
    reached_total += d;
    bool first = true;
    for (uint32_t j = 0; j < i; j++) first &= P.sources[j] != P.sources[i];
    if (first) frontier_deg += d;
  }
  if (gtid == 0) {
    uint32_t nm = 0;
    for (uint32_t i = 0; i < P.k; i++) {
      const uint32_t s = P.sources[i];
      const u64 before = P.seen[s];
      const u64 now = before | (1ull << i);
      P.seen[s] = now;
      P.hist[s] = now;
      P.act[s >> 5] |= 1u << (s & 31);
      if (now == P.all) P.done[s >> 5] |= 1u << (s & 31);
      P.sigma[(size_t)s * kRow + i] = 1.0f;
      if (!before && P.ro[s + 1] - P.ro[s] >= kMarkDeg) P.mark[nm++] = s;
    }
    P.cnt[2].mark = nm;
    __threadfence();
  }
  if (!grid_sync(P.bar)) return;

  u64 undone_in = P.m;  // in-degree of the vertices some source has not reached
  uint32_t n_log = 0, phase = 0;

  // ---- forward sweep
  uint32_t L = 0;
  bool overflow = false;
  for (;; L++, phase++) {
    if (L + 1 >= P.cap_levels) {
      overflow = true;
      break;
    }
    Counters* C = P.cnt + (phase % 3);
    const Counters* Cprev = P.cnt + ((phase + 2) % 3);
    if (gtid == 0) {
      Counters z = {};
      P.cnt[(phase + 1) % 3] = z;
    }
    const uint64_t t0 = gtid == 0 ? sygraph::detail::global_timer_ns() : 0;
    const u64* hist_L = P.hist + (size_t)L * n;
    u64* hist_N = P.hist + (size_t)(L + 1) * n;
    uint32_t* act_N = P.act + (size_t)(L + 1) * w0;
    uint32_t* mark_N = P.mark + (size_t)((L + 1) & 1) * P.big_cap;
    if (L + 2 < P.cap_levels) {  // hist / act of level L+2 start empty
      u64* h2 = P.hist + (size_t)(L + 2) * n;
      for (uint32_t i = gtid; i < n; i += nthreads) st_cg(h2 + i, 0ull);
      uint32_t* a2 = P.act + (size_t)(L + 2) * w0;
      for (uint32_t i = gtid; i < w0; i += nthreads) st_cg(a2 + i, 0u);
    }
    const bool sparse = frontier_deg * kSparseRatio < undone_in;
    if (sparse) {
      mark_candidates(P, P.act + (size_t)L * w0, P.mark + (size_t)(L & 1) * P.big_cap, ld_cg(&Cprev->mark));
      if (!grid_sync(P.bar)) return;
    }
    Local loc;
    // a sparse level whose frontier has many out-edges marks candidates in
    // most words (RMAT-20: 450 K from 4869 vertices): balanced as well
    for_each_word(!sparse || frontier_deg > w0, &C->next_word, w0, gwarp, nwarps, [&](uint32_t wi) {
      uint32_t cand = ~ld_cg(P.done + wi) & valid_bits(wi, w0, n);
      if (sparse) {
        const uint32_t c = ld_cg(P.cand + wi);
        if (c) st_cg(P.cand + wi, 0u);  // the mark bitmap is zero again for the next level
        cand &= c;
      }
      while (cand) {
        const uint32_t u = wi * 32 + (__ffs(cand) - 1);
        cand &= cand - 1;
        const uint32_t beg = P.iro[u], end = P.iro[u + 1];
        if (defer_big(P, C, u, end - beg)) continue;
        const u64 su = ld_cg(P.seen + u);
        float a0 = 0.f, a1 = 0.f;
        const u64 nm = forward_gather(P, hist_L, beg, end, su, a0, a1);
        forward_finish(P, hist_N, act_N, mark_N, C, u, su, nm, a0, a1, loc);
      }
    });
    if (!grid_sync(P.bar)) return;
    {
      const u64 bp = ld_cg(&C->big_packed);
      const uint32_t nbig = (uint32_t)(bp >> 32), nch = (uint32_t)bp;
      if (nbig) {  // grid-uniform
        gather_chunks<true>(P, hist_L, nullptr, nbig, nch);
        if (!grid_sync(P.bar)) return;
        finish_chunked<true>(P, hist_L, hist_N, act_N, mark_N, C, nbig, nch, loc);
      }
    }
    block_add(loc, S, C);
    if (!grid_sync(P.bar)) return;
    const u64 next = ld_cg(&C->new_count);
    if (threadIdx.x == 0 && L + 1 < kSizedLevels) S.level_size[L + 1] = (uint32_t)min(next, (u64)0xffffffffu);
    reached_total += ld_cg(&C->reached);
    frontier_deg = ld_cg(&C->new_deg);
    undone_in -= ld_cg(&C->done_in);
    if (gtid == 0 && n_log < kMaxLog) {
      sg_level_record r = {};
      r.level = L;
      r.strategy = sparse ? 0u : 2u;
      r.next_size = (uint32_t)next;
      r.next_degree = frontier_deg;
      r.unexplored_degree = undone_in;
      r.t_start_ns = t0;
      r.t_end_ns = sygraph::detail::global_timer_ns();
      P.log[n_log] = r;
    }
    n_log++;
    if (next == 0) break;
  }
  if (overflow) {
    if (gtid == 0) {
      P.result[0] = L + 1;
      P.result[1] = 1;
      P.result[3] = min(n_log, kMaxLog);
    }
    return;
  }
  phase++;
  // ---- backward sweep: levels Lmax .. 1 (Lmax is the deepest non-empty level)
  const uint32_t Lmax = L;
  for (uint32_t Lb = Lmax; Lb >= 1; Lb--, phase++) {
    Counters* C = P.cnt + (phase % 3);
    if (gtid == 0) {
      Counters z = {};
      P.cnt[(phase + 1) % 3] = z;
    }
    const uint64_t t0 = gtid == 0 ? sygraph::detail::global_timer_ns() : 0;
    const u64* hist_B = P.hist + (size_t)Lb * n;
    const u64* hist_next = Lb < Lmax ? P.hist + (size_t)(Lb + 1) * n : nullptr;
    const uint32_t* act_B = P.act + (size_t)Lb * w0;
    Local unused;
    const bool dense = Lb < kSizedLevels && S.level_size[Lb] > w0;  // block- and grid-uniform
    for_each_word(dense, &C->next_word, w0, gwarp, nwarps, [&](uint32_t wi) {
      uint32_t word = ld_cg(act_B + wi);
      while (word) {
        const uint32_t v = wi * 32 + (__ffs(word) - 1);
        word &= word - 1;
        const uint32_t beg = P.ro[v], end = P.ro[v + 1];
        if (hist_next && defer_big(P, C, v, end - beg)) continue;
        const u64 fv = ld_cg(hist_B + v);
        float a0 = 0.f, a1 = 0.f;
        if (hist_next) backward_gather(P, hist_next, beg, end, fv, a0, a1);
        backward_finish(P, v, fv, a0, a1);
      }
    });
    if (!grid_sync(P.bar)) return;
    {
      const u64 bp = ld_cg(&C->big_packed);
      const uint32_t nbig = (uint32_t)(bp >> 32), nch = (uint32_t)bp;
      if (nbig) {  // grid-uniform
        gather_chunks<false>(P, hist_B, hist_next, nbig, nch);
        if (!grid_sync(P.bar)) return;
        finish_chunked<false>(P, hist_B, nullptr, nullptr, nullptr, C, nbig, nch, unused);
        if (!grid_sync(P.bar)) return;
      }
    }
    if (gtid == 0 && n_log < kMaxLog) {
      sg_level_record r = {};
      r.level = Lb;
      r.strategy = kBackwardLog;
      r.t_start_ns = t0;
      r.t_end_ns = sygraph::detail::global_timer_ns();
      P.log[n_log] = r;
    }
    n_log++;
  }
  if (gtid == 0) {
    P.result[0] = Lmax + 1;
    P.result[1] = 0;
    P.result[2] = reached_total;
    P.result[3] = min(n_log, kMaxLog);
  }
}

__global__ void no_in_edges_kernel(const uint32_t* __restrict__ iro, uint32_t n, uint32_t w0, uint32_t* out) {
  const uint32_t lane = threadIdx.x & 31;
  for (uint32_t base = (blockIdx.x * blockDim.x + threadIdx.x) & ~31u; base < (uint64_t)w0 * 32;
       base += gridDim.x * blockDim.x) {
    const uint32_t v = base + lane;
    const bool z = v < n && iro[v + 1] == iro[v];
    const uint32_t msk = __ballot_sync(kFullMask, z);
    if (lane == 0) out[base >> 5] = msk;
  }
}

}  // namespace bcb
}  // namespace sgb

using namespace sgb;

struct sg_bc_batch_s {
  sg_graph g = nullptr;
  cudaStream_t stream = nullptr;  // launches and copies (the graph's stream unless set)
  uint32_t max_ctas = 0;
  uint32_t w0 = 0, cap_levels = 0, last_k = 0;
  unsigned long long* seen = nullptr;
  unsigned long long* hist = nullptr;
  uint32_t *act = nullptr, *done = nullptr, *no_in = nullptr, *sources = nullptr;
  uint32_t* cand = nullptr;
  uint32_t *big = nullptr, *big_first = nullptr, *mark = nullptr, big_cap = 0;
  float* part = nullptr;                // chunk partial sums of degree >= kCtaDeg vertices
  unsigned long long* part_mask = nullptr;
  uint32_t chunk_cap = 0;
  float *sigma = nullptr, *q = nullptr, *bc = nullptr;
  bcb::Counters* cnt = nullptr;
  sygraph::detail::GridBarrier* bar = nullptr;
  sg_level_record* log = nullptr;
  unsigned long long* result = nullptr;
};

namespace {

void bcb_release(sg_bc_batch h) {
  if (!h) return;
  dev_free(h->seen);
  dev_free(h->hist);
  dev_free(h->act);
  dev_free(h->done);
  dev_free(h->no_in);
  dev_free(h->sources);
  dev_free(h->sigma);
  dev_free(h->q);
  dev_free(h->cand);
  dev_free(h->big);
  dev_free(h->big_first);
  dev_free(h->part);
  dev_free(h->part_mask);
  dev_free(h->mark);
  dev_free(h->bc);
  dev_free(h->cnt);
  dev_free(h->bar);
  dev_free(h->log);
  dev_free(h->result);
  delete h;
}

uint64_t level_bytes(sg_bc_batch h) { return 8ull * h->g->n + 4ull * h->w0; }

// History of `levels` levels (frontier masks + activity words).
sg_status bcb_history(sg_bc_batch h, uint32_t levels) {
  dev_free(h->hist);
  dev_free(h->act);
  h->cap_levels = 0;
  SG_TRY(dev_alloc(&h->hist, (uint64_t)levels * h->g->n));
  SG_TRY(dev_alloc(&h->act, (uint64_t)levels * h->w0));
  h->cap_levels = levels;
  return SG_OK;
}

// Levels that fit in a quarter of the free device memory.
uint32_t bcb_max_levels(sg_bc_batch h) {
  size_t f = 0, t = 0;
  if (cudaMemGetInfo(&f, &t) != cudaSuccess) return h->cap_levels;
  const uint64_t have = (uint64_t)h->cap_levels * level_bytes(h);
  const uint64_t lv = (f / 4 + have) / level_bytes(h);
  return (uint32_t)std::min<uint64_t>(lv, 1u << 20);
}

sg_status bcb_launch(sg_bc_batch h, uint32_t k, int accumulate) {
  sg_graph g = h->g;
  SG_CUDA(cudaMemsetAsync(h->bar, 0, sizeof(*h->bar), h->stream));
  SG_CUDA(cudaMemsetAsync(h->result, 0, 4 * sizeof(unsigned long long), h->stream));
  bcb::Params P;
  P.n = g->n;
  P.w0 = h->w0;
  P.k = k;
  P.m = g->m;
  P.ro = g->fwd.ro;
  P.col = g->fwd.col;
  P.iro = g->inv.ro;
  P.icol = g->inv.col;
  P.sources = h->sources;
  P.all = k == 64 ? ~0ull : ((1ull << k) - 1ull);
  P.seen = h->seen;
  P.hist = h->hist;
  P.cap_levels = h->cap_levels;
  P.act = h->act;
  P.done = h->done;
  P.no_in_edges = h->no_in;
  P.sigma = h->sigma;
  P.q = h->q;
  P.cand = h->cand;
  P.big = h->big;
  P.big_first = h->big_first;
  P.part = h->part;
  P.part_mask = h->part_mask;
  P.chunk_cap = h->chunk_cap;
  P.mark = h->mark;
  P.big_cap = h->big_cap;
  P.bc = h->bc;
  P.accumulate = accumulate;
  P.cnt = h->cnt;
  P.bar = h->bar;
  P.log = h->log;
  P.result = h->result;
  return eng::launch_persistent(bcb::bc_batch_kernel, P, 2, h->stream, h->max_ctas);
}

}  // namespace

extern "C" {

sg_status sg_bc_batch_create(sg_graph g, uint32_t history_levels, sg_bc_batch* out) {
  clear_error();
  SG_REQUIRE(g && out, SG_ERR_INVALID, "NULL argument");
  SG_REQUIRE(g->n > 0, SG_ERR_INVALID, "graph has no vertices");
  *out = nullptr;
  sg_bc_batch h = new sg_bc_batch_s();
  h->g = g;
  h->stream = g->stream;
  h->w0 = div_up(g->n, 32);
  // at most m / kMarkDeg vertices have a degree >= kMarkDeg (>= kCtaDeg too)
  h->big_cap = (uint32_t)std::min<uint64_t>(g->n, g->m / bcb::kMarkDeg + 2);
  // chunks of the vertices of degree >= kCtaDeg: at most m / kChunkE + one per vertex
  h->chunk_cap = (uint32_t)std::min<uint64_t>(0xffffffffu, g->m / bcb::kChunkE + h->big_cap);
  const uint64_t n = g->n;
  uint32_t levels = history_levels;
  if (!levels) levels = (uint32_t)std::max<uint64_t>(16, std::min<uint64_t>(256, (2ull << 30) / level_bytes(h)));
  levels = std::max<uint32_t>(levels, 2);
  sg_status s;
  if ((s = dev_alloc(&h->seen, n)) || (s = dev_alloc(&h->done, h->w0)) || (s = dev_alloc(&h->no_in, h->w0)) ||
      (s = dev_alloc(&h->sources, 64)) || (s = dev_alloc(&h->sigma, n * bcb::kRow)) ||
      (s = dev_alloc(&h->q, n * bcb::kRow)) || (s = dev_alloc(&h->cand, h->w0)) ||
      (s = dev_alloc(&h->big, h->big_cap)) || (s = dev_alloc(&h->big_first, h->big_cap)) ||
      (s = dev_alloc(&h->part, (uint64_t)h->chunk_cap * bcb::kRow)) || (s = dev_alloc(&h->part_mask, h->chunk_cap)) ||
      (s = dev_alloc(&h->mark, 2ull * h->big_cap)) || (s = dev_alloc(&h->bc, n)) || (s = dev_alloc(&h->cnt, 3)) ||
      (s = dev_alloc(&h->bar, 1)) || (s = dev_alloc(&h->log, SG_MAX_LOGGED_LEVELS)) ||
      (s = dev_alloc(&h->result, 4)) || (s = bcb_history(h, levels))) {
    bcb_release(h);
    return s;
  }
  bcb::no_in_edges_kernel<<<grid_for((uint64_t)h->w0 * 32, 256), 256, 0, g->stream>>>(g->inv.ro, g->n, h->w0, h->no_in);
  if (cudaGetLastError() != cudaSuccess) {
    bcb_release(h);
    return fail(SG_ERR_CUDA, "batched BC set-up kernel failed to launch");
  }
  count_launch();
  if (cudaMemsetAsync(h->bc, 0, sizeof(float) * n, g->stream) != cudaSuccess) {
    bcb_release(h);
    return fail(SG_ERR_CUDA, "batched BC set-up failed");
  }
  *out = h;
  return SG_OK;
}

sg_status sg_bc_batch_destroy(sg_bc_batch h) {
  if (h) {
    cudaStreamSynchronize(h->stream);
    bcb_release(h);
  }
  return SG_OK;
}

sg_status sg_bc_batch_run_async(sg_bc_batch h, const uint32_t* host_sources, uint32_t k, int accumulate) {
  clear_error();
  SG_REQUIRE(h && host_sources, SG_ERR_INVALID, "NULL argument");
  SG_REQUIRE(k >= 1 && k <= 64, SG_ERR_INVALID, "a batch holds 1 to 64 sources");
  for (uint32_t i = 0; i < k; i++) SG_REQUIRE(host_sources[i] < h->g->n, SG_ERR_INVALID, "source out of range");
  SG_CUDA(cudaMemcpyAsync(h->sources, host_sources, sizeof(uint32_t) * k, cudaMemcpyHostToDevice, h->stream));
  h->last_k = k;
  return bcb_launch(h, k, accumulate);
}

sg_status sg_bc_batch_run(sg_bc_batch h, const uint32_t* host_sources, uint32_t k, int accumulate,
                          sg_bc_batch_details* details) {
  SG_TRY(sg_bc_batch_run_async(h, host_sources, k, accumulate));
  uint32_t retries = 0;
  for (;;) {
    unsigned long long r[4];
    sygraph::detail::GridBarrier b;
    SG_CUDA(cudaMemcpyAsync(r, h->result, sizeof(r), cudaMemcpyDeviceToHost, h->stream));
    SG_CUDA(cudaMemcpyAsync(&b, h->bar, sizeof(b), cudaMemcpyDeviceToHost, h->stream));
    SG_CUDA(cudaStreamSynchronize(h->stream));
    if (b.error) return fail(SG_ERR_TIMEOUT, "batched BC: a grid barrier wait ran out");
    if (r[1]) {
      // deeper than the history: enlarge it (bc is untouched before the backward sweep) and run again
      const uint32_t want = std::min<uint32_t>(bcb_max_levels(h), h->cap_levels * 4);
      SG_REQUIRE(want > h->cap_levels, SG_ERR_NOMEM, "batched BC: the traversal is deeper than the history that fits");
      SG_TRY(bcb_history(h, want));
      SG_TRY(bcb_launch(h, k, accumulate));
      retries++;
      continue;
    }
    if (details) {
      details->iterations = r[0];
      details->reached_edges = r[2];
      details->history_levels = h->cap_levels;
      details->history_retries = retries;
    }
    return SG_OK;
  }
}

sg_status sg_bc_batch_set_launch(sg_bc_batch h, void* stream, uint32_t max_ctas) {
  clear_error();
  SG_REQUIRE(h, SG_ERR_INVALID, "NULL argument");
  SG_CUDA(cudaStreamSynchronize(h->stream));
  h->stream = stream ? (cudaStream_t)stream : h->g->stream;
  h->max_ctas = max_ctas;
  return SG_OK;
}

sg_status sg_bc_batch_get(sg_bc_batch h, float* host_bc) {
  SG_REQUIRE(h && host_bc, SG_ERR_INVALID, "NULL argument");
  SG_CUDA(cudaMemcpyAsync(host_bc, h->bc, sizeof(float) * h->g->n, cudaMemcpyDeviceToHost, h->stream));
  SG_CUDA(cudaStreamSynchronize(h->stream));
  return SG_OK;
}

sg_status sg_bc_batch_bc_device(sg_bc_batch h, const float** dev_bc) {
  SG_REQUIRE(h && dev_bc, SG_ERR_INVALID, "NULL argument");
  *dev_bc = h->bc;
  return SG_OK;
}

sg_status sg_bc_batch_level_records(sg_bc_batch h, sg_level_record* host_records, uint32_t cap, uint32_t* count) {
  SG_REQUIRE(h && count, SG_ERR_INVALID, "NULL argument");
  SG_CUDA(cudaStreamSynchronize(h->stream));
  unsigned long long it = 0;
  if (h->last_k) SG_CUDA(cudaMemcpy(&it, h->result + 3, sizeof(it), cudaMemcpyDeviceToHost));
  uint32_t k = (uint32_t)(it < SG_MAX_LOGGED_LEVELS ? it : SG_MAX_LOGGED_LEVELS);
  if (k > cap) k = cap;
  if (host_records && k) SG_CUDA(cudaMemcpy(host_records, h->log, sizeof(sg_level_record) * k, cudaMemcpyDeviceToHost));
  *count = k;
  return SG_OK;
}

sg_status sg_bc_batched(sg_graph g, const uint32_t* host_sources, uint32_t k, float* host_bc) {
  clear_error();
  SG_REQUIRE(g && host_bc, SG_ERR_INVALID, "NULL argument");
  SG_REQUIRE(k == 0 || host_sources, SG_ERR_INVALID, "sources is NULL");
  sg_bc_batch h = nullptr;
  SG_TRY(sg_bc_batch_create(g, 0, &h));
  sg_status s = SG_OK;
  for (uint32_t i = 0; i < k && s == SG_OK; i += 64)
    s = sg_bc_batch_run(h, host_sources + i, std::min<uint32_t>(64, k - i), i > 0, nullptr);
  if (s == SG_OK) s = sg_bc_batch_get(h, host_bc);
  sg_bc_batch_destroy(h);
  return s;
}

}  // extern "C"
