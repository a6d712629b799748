// Pull sweep of the SSSP engine: every vertex takes the minimum of
// d[v] + w over its in-neighbours v in the current frontier (no atomics for
// the light ones), for the dense iterations where pushing would issue an
// atomicMin per improving edge.  The minimum is exact and order-independent,
// so a pull iteration reaches the same fixed point as a push iteration.
//
//   light vertex (in-degree < kPullHeavy): a warp per bitmap word; lists of
//       at most 32 in-neighbours are scanned by their lane (next column index
//       loaded while the current frontier bit is tested), longer ones by the
//       whole warp with a min-reduction; only the owner writes d[u].
//   heavy vertex: its in-list is cut into kPullChunk-edge chunks (a static
//       list built when the instance is created); warps take chunks
//       grid-stride and finish each with one atomicMin on d[u].
#pragma once

#include "engine_common.cuh"

namespace sgb {
namespace eng {

constexpr uint32_t kPullHeavy = 256;  // in-degree from which a vertex is pulled in chunks
constexpr uint32_t kPullChunk = 256;  // in-edges per chunk

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

template <typename W>
__device__ __forceinline__ void sssp_pull_sweep(const PullArgs<W>& A, const uint32_t* fb_cur, uint32_t* fb_next,
                                                W threshold, bool bucketed, unsigned long long& n_new,
                                                unsigned long long& deg_new) {
  const uint32_t lane = threadIdx.x & 31;
  const uint32_t gwarp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const uint32_t nwarps = (gridDim.x * blockDim.x) >> 5;
  for (uint32_t wi = gwarp; wi < A.w0; wi += nwarps) {
    const uint32_t v = wi * 32 + lane;
    const bool in = v < A.n;
    const uint32_t beg = in ? A.iro[v] : 0u, end = in ? A.iro[v + 1] : 0u;
    const uint32_t deg = end - beg;
    const bool light = in && deg < kPullHeavy;
    const W d0 = light ? ld_cg(A.dist + v) : W(0);
    W best = d0;
    if (light && deg <= 32) {
      uint32_t e = beg;
      uint32_t c = e < end ? A.icol[e] : 0u;
      while (e < end) {
        const uint32_t cn = e + 1 < end ? A.icol[e + 1] : 0u;
        if (bit_test_ro(fb_cur, c)) {
          const W cand = ld_cg(A.dist + c) + A.iw[e];
          best = cand < best ? cand : best;
        }
        c = cn;
        e++;
      }
    }
    // medium lists: the warp scans each with a min-reduction
    uint32_t med = __ballot_sync(kFullMask, light && deg > 32);
    while (med) {
      const uint32_t j = __ffs(med) - 1;
      med &= med - 1;
      const uint32_t jb = __shfl_sync(kFullMask, beg, j), je = __shfl_sync(kFullMask, end, j);
      W part = __shfl_sync(kFullMask, best, j);
      for (uint32_t eb = jb; eb < je; eb += 32) {
        const uint32_t e = eb + lane;
        if (e < je) {
          const uint32_t c = A.icol[e];
          if (bit_test_ro(fb_cur, c)) {
            const W cand = ld_cg(A.dist + c) + A.iw[e];
            part = cand < part ? cand : part;
          }
        }
      }
      part = warp_min_w(part);
      if (lane == j) best = part;
    }
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
