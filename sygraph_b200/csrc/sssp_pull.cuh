// Pull sweep of the SSSP engine: every vertex takes the minimum of
// d[v] + w over its in-neighbours v in the current frontier (no atomics for
// the light ones), for the dense iterations where pushing would issue an
// atomicMin per improving edge.  The minimum is exact and order-independent,
// so a pull iteration reaches the same fixed point as a push iteration.
//
//   light vertex (in-degree < kPullHeavy): a warp per bitmap word; the
//       in-lists of the word's 32 vertices are walked edge-parallel (a warp
//       scan of their degrees maps lanes to consecutive edges, so column and
//       weight loads are coalesced) and each candidate goes into the owner's
//       shared-memory slot by atomicMin on order-preserving bits; only the
//       owner writes d[u].
//   heavy vertex: its in-list is cut into kPullChunk-edge chunks (a static
//       list built when the instance is created); warps take chunks
//       grid-stride and finish each with one atomicMin on d[u].
#pragma once

#include "engine_common.cuh"

namespace sgb {
namespace eng {

constexpr uint32_t kPullHeavy = 256;  // in-degree from which a vertex is pulled in chunks
constexpr uint32_t kPullChunk = 256;  // in-edges per chunk

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

// A threshold above every distance (+inf for floats).
template <typename W>
__device__ __forceinline__ W max_weight() {
  if constexpr (sizeof(W) == 4 && W(0.5) != W(0))
    return __uint_as_float(0x7f800000u);
  else
    return (W)0xffffffffu;
}

template <typename W>
__device__ __forceinline__ W warp_min_w(W x) {
#pragma unroll
  for (int d = 16; d > 0; d >>= 1) {
    const W y = __shfl_xor_sync(kFullMask, x, d);
    x = y < x ? y : x;
  }
  return x;
}

template <typename W>
struct PullArgs {
  uint32_t n, w0;
  const uint32_t* ro;      // out-degrees (frontier degree bookkeeping)
  const uint32_t* iro;
  const uint32_t* icol;
  const W* iw;             // weights of the in-edges
  W* dist;
  uint32_t* far;
  const uint32_t* heavy_v;      // vertices of in-degree >= kPullHeavy
  const uint32_t* heavy_first;  // first chunk index of each, increasing
  uint32_t n_heavy, n_chunks;
};

// Marks u improved to distance nd: next frontier when below the threshold
// (or not bucketed), far set otherwise.  Counts a vertex the first time its
// next-frontier bit is set.
template <typename W>
__device__ __forceinline__ void pull_mark(const PullArgs<W>& A, uint32_t* fb_next, uint32_t u, W nd, W threshold,
                                          bool bucketed, unsigned long long& n_new, unsigned long long& deg_new) {
  const uint32_t b = 1u << (u & 31);
  if (!bucketed || nd < threshold) {
    if (!(atomicOr(fb_next + (u >> 5), b) & b)) {
      n_new++;
      deg_new += A.ro[u + 1] - A.ro[u];
    }
  } else {
    atomicOr(A.far + (u >> 5), b);
  }
}

// s_best: one uint32 per thread of the block (the warp's 32 owner slots).
template <typename W>
__device__ __forceinline__ void sssp_pull_sweep(const PullArgs<W>& A, const uint32_t* fb_cur, uint32_t* fb_next,
                                                W threshold, bool bucketed, unsigned long long& n_new,
                                                unsigned long long& deg_new, uint32_t* s_best) {
  const uint32_t lane = threadIdx.x & 31;
  const uint32_t gwarp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const uint32_t nwarps = (gridDim.x * blockDim.x) >> 5;
  uint32_t* best_slot = s_best + (threadIdx.x & ~31u);
  for (uint32_t wi = gwarp; wi < A.w0; wi += nwarps) {
    const uint32_t v = wi * 32 + lane;
    const bool in = v < A.n;
    const uint32_t beg = in ? A.iro[v] : 0u, end = in ? A.iro[v + 1] : 0u;
    const bool light = in && end - beg < kPullHeavy;
    const uint32_t dg = light ? end - beg : 0u;
    const uint32_t incl = warp_inclusive_scan(dg);
    const uint32_t total = __shfl_sync(kFullMask, incl, 31);
    if (!total) continue;
    const uint32_t excl = incl - dg;
    const W d0 = light ? ld_cg(A.dist + v) : W(0);
    best_slot[lane] = light ? order_bits<W>(d0) : 0xffffffffu;
    __syncwarp();
    for (uint32_t r0 = 0; r0 < total; r0 += 32) {
      const uint32_t r = r0 + lane;
      const bool act = r < total;
      const uint32_t o = warp_owner_of_rank(incl, act ? r : total - 1);
      const uint32_t ob = __shfl_sync(kFullMask, beg, o);
      const uint32_t oe = __shfl_sync(kFullMask, excl, o);
      if (act) {
        const uint32_t e = ob + (r - oe);
        const uint32_t c = A.icol[e];
        if (bit_test_ro(fb_cur, c)) atomicMin(best_slot + o, order_bits<W>(ld_cg(A.dist + c) + A.iw[e]));
      }
    }
    __syncwarp();
    const W best = from_order_bits<W>(best_slot[lane]);
    __syncwarp();
    if (light && best < d0) {
      st_cg(A.dist + v, best);
      pull_mark(A, fb_next, v, best, threshold, bucketed, n_new, deg_new);
    }
  }
  // heavy vertices, chunk by chunk
  for (uint32_t c = gwarp; c < A.n_chunks; c += nwarps) {
    const uint32_t ent = find_chunk_owner(A.heavy_first, A.n_heavy, c);
    const uint32_t v = A.heavy_v[ent];
    const uint32_t cb = A.iro[v] + (c - A.heavy_first[ent]) * kPullChunk;
    const uint32_t ce = min(A.iro[v + 1], cb + kPullChunk);
    W part = ld_cg(A.dist + v);
    const W d_seen = part;
    for (uint32_t e = cb + lane; e < ce; e += 32) {
      const uint32_t s = A.icol[e];
      if (bit_test_ro(fb_cur, s)) {
        const W cand = ld_cg(A.dist + s) + A.iw[e];
        part = cand < part ? cand : part;
      }
    }
    part = warp_min_w(part);
    if (lane == 0 && part < d_seen) {
      const W old = sygraph::detail::atomic_min_nonneg(A.dist + v, part);
      if (part < old) pull_mark(A, fb_next, v, part, threshold, bucketed, n_new, deg_new);
    }
  }
}

}  // namespace eng
}  // namespace sgb
