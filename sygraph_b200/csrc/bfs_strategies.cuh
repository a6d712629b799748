// The expansion strategies of the BFS engine (bfs.cu), one call per level.
//   push/warp : warps take summary words, expand the frontier's light vertices
//               32 at a time, edge-parallel by a shuffle scan
//   push/CTA  : a CTA takes one frontier word per warp (16 words, 512
//               candidates), scans their
//               degrees across the block and walks the combined edge range
//               (shared-memory binary search from edge rank to source)
//   pull/warp : a warp takes four bitmap words (128 unvisited candidates,
//               first probes of all four in flight together), each lane scans
//               its own in-edges with the next column index prefetched; the
//               warp helps with long lists
//   pull/CTA  : a CTA takes one word per warp of unvisited candidates and walks all their
//               in-edges edge-parallel, with a per-candidate done flag
// Heavy vertices (degree >= kHeavy) of a push level are expanded from the
// heavy list in kBfsChunk-edge chunks by both push strategies.
#pragma once

#include "bfs_engine.cuh"

namespace sgb {
namespace bfs {

__device__ __forceinline__ uint32_t smem_upper_bound(const uint32_t* a, uint32_t n, uint32_t r) {
  uint32_t lo = 0, hi = n;
  while (lo < hi) {
    const uint32_t mid = (lo + hi) >> 1;
    if (a[mid] <= r)
      lo = mid + 1;
    else
      hi = mid;
  }
  return lo;
}

// Expands 32 (beg, deg) ranges of a warp edge-parallel.
__device__ __forceinline__ void expand_group(Level& L, uint32_t beg, uint32_t deg) {
  const uint32_t lane = threadIdx.x & 31;
  const uint32_t incl = warp_inclusive_scan(deg);
  const uint32_t total = __shfl_sync(kFullMask, incl, 31);
  const uint32_t excl = incl - deg;
  for (uint32_t r0 = 0; r0 < total; r0 += 64) {
    uint32_t u[2], act = 0;
#pragma unroll
    for (int k = 0; k < 2; k++) {
      const uint32_t r = r0 + k * 32 + lane;
      const bool a = r < total;
      const uint32_t o = warp_owner_of_rank(incl, a ? r : total - 1);
      const uint32_t ob = __shfl_sync(kFullMask, beg, o);
      const uint32_t oe = __shfl_sync(kFullMask, excl, o);
      u[k] = a ? L.P->col[ob + (r - oe)] : 0u;
      act |= (uint32_t)a << k;
    }
    L.visit_push_n<2>(u, act);
  }
}

// Heavy-vertex chunks, warp-strided from `first_warp`.
__device__ __forceinline__ void push_heavy(Level& L, const uint32_t* hv, const uint32_t* hs, uint32_t n_heavy,
                                           uint32_t n_chunks, uint32_t first_unit, uint32_t units_end) {
  const Params& P = *L.P;
  const uint32_t lane = threadIdx.x & 31;
  const uint32_t gwarp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const uint32_t nwarps = (gridDim.x * blockDim.x) >> 5;
  for (uint32_t unit = gwarp; unit < units_end; unit += nwarps) {
    if (unit < first_unit) continue;
    const uint32_t c = unit - first_unit;
    const uint32_t ent = warp_find_owner(hs, n_heavy, c);
    const uint32_t v = ld_cg(hv + ent);
    const uint32_t first = ld_cg(hs + ent);
    const uint32_t cb = P.ro[v] + (c - first) * kBfsChunk;
    const uint32_t ce = min(P.ro[v + 1], cb + kBfsChunk);
    for (uint32_t eb = cb; eb < ce; eb += 64) {
      uint32_t u[2], act = 0;
#pragma unroll
      for (int k = 0; k < 2; k++) {
        const uint32_t e = eb + k * 32 + lane;
        u[k] = e < ce ? P.col[e] : 0u;
        act |= (uint32_t)(e < ce) << k;
      }
      L.visit_push_n<2>(u, act);
    }
  }
  (void)n_chunks;
}

// A warp takes a summary unit of 32 bitmap words and loads the words
// directly (one round trip, not summary then words: the 128-byte load costs
// the same when the unit is empty), and clears the unit of F_{L-1} (fb_zero
// / sm_zero) with plain stores.
__device__ __forceinline__ void push_warp(Level& L, const uint32_t* fb_cur, const uint32_t* sm_cur,
                                          uint32_t* fb_zero, uint32_t* sm_zero, const uint32_t* hv,
                                          const uint32_t* hs, uint32_t n_heavy, uint32_t n_chunks) {
  const Params& P = *L.P;
  const uint32_t lane = threadIdx.x & 31;
  const uint32_t gwarp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const uint32_t nwarps = (gridDim.x * blockDim.x) >> 5;
  const uint32_t w0 = P.w0, w1 = P.w1;
  (void)sm_cur;
  for (uint32_t unit = gwarp; unit < w1; unit += nwarps) {
    const uint32_t wi = unit * 32 + lane;
    const uint32_t bits = wi < w0 ? ld_cg(fb_cur + wi) : 0u;
    if (wi < w0) st_cg(fb_zero + wi, 0u);
    if (lane == 0) st_cg(sm_zero + unit, 0u);
    if (!__any_sync(kFullMask, bits)) continue;
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
  }
  // heavy chunks continue the warp numbering after the summary words
  push_heavy(L, hv, hs, n_heavy, n_chunks, w1, w1 + n_chunks);
}

__device__ __forceinline__ void push_cta(Level& L, const uint32_t* fb_cur, const uint32_t* sm_cur, const uint32_t* hv,
                                         const uint32_t* hs, uint32_t n_heavy, uint32_t n_chunks) {
  const Params& P = *L.P;
  Shared& S = *L.S;
  const uint32_t t = threadIdx.x, lane = t & 31, wl = t >> 5;
  // a CTA takes as many bitmap words as it has warps (16 or 32: a group never
  // straddles a summary word)
  const uint32_t wg = blockDim.x >> 5;
  const uint32_t ngroups = (P.w0 + wg - 1) / wg;
  for (uint32_t g = blockIdx.x; g < ngroups; g += gridDim.x) {
    const uint32_t first = g * wg;
    const uint32_t sg = (ld_cg(sm_cur + (first >> 5)) >> (first & 31)) & (wg == 32 ? 0xffffffffu : ((1u << wg) - 1u));
    if (!sg) continue;  // the same for every thread of the CTA
    const uint32_t w = first + wl;
    const uint32_t word = (((sg >> wl) & 1u) && w < P.w0) ? ld_cg(fb_cur + w) : 0u;
    const bool act = (word >> lane) & 1u;
    const uint32_t v = w * 32 + lane;
    const uint32_t beg = act ? P.ro[v] : 0u;
    uint32_t deg = act ? P.ro[v + 1] - beg : 0u;
    if (deg >= kHeavy) deg = 0;
    uint32_t total;
    const uint32_t excl = sygraph::detail::block_excl_scan(deg, &total, S.scan);
    S.beg[t] = beg;
    S.incl[t] = excl + deg;
    __syncthreads();
    for (uint32_t r = t; r < total; r += blockDim.x) {
      const uint32_t slot = smem_upper_bound(S.incl, blockDim.x, r);
      const uint32_t before = slot ? S.incl[slot - 1] : 0u;
      L.visit_push(P.col[S.beg[slot] + (r - before)]);
    }
    __syncthreads();
  }
  push_heavy(L, hv, hs, n_heavy, n_chunks, 0, n_chunks);
}

// Position of the k-th in-neighbour probed (from the front, or from the back
// of the sorted list when `reverse`).
__device__ __forceinline__ uint32_t probe_pos(uint32_t beg, uint32_t end, uint32_t k, bool reverse) {
  return reverse ? end - 1 - k : beg + k;
}

// Short-circuit pull of the still-open lists of one bitmap word, after the
// serial probes: the lanes' remaining in-neighbours are ranked across the
// warp and scanned kPullWin windows of 32 at a time (coalesced column loads,
// then the frontier tests); a hit marks its owner (one warp OR-reduction per
// window batch), edges of owners already found are not loaded, and the scan
// ends once every open list has a hit.  Returns this lane's result.
__device__ __forceinline__ bool pull_word_scan(const Params& P, const uint32_t* fb_cur, bool open, uint32_t b,
                                               uint32_t e, bool reverse) {
  const uint32_t lane = threadIdx.x & 31;
  const uint32_t rem = open ? e - b - kPullProbes : 0u;  // open: more than kPullProbes in-neighbours
  const uint32_t incl = warp_inclusive_scan(rem);
  const uint32_t total = __shfl_sync(kFullMask, incl, 31);
  const uint32_t excl = incl - rem;
  const uint32_t need = __ballot_sync(kFullMask, open);
  uint32_t hitm = 0;
  for (uint32_t r0 = 0; r0 < total; r0 += 32 * kPullWin) {
    uint32_t col[kPullWin], own[kPullWin];
    bool act[kPullWin];
#pragma unroll
    for (int k = 0; k < kPullWin; k++) {
      const uint32_t r = r0 + k * 32 + lane;
      const bool in = r < total;
      const uint32_t o = warp_owner_of_rank(incl, in ? r : total - 1);
      const uint32_t ob = __shfl_sync(kFullMask, b, o);
      const uint32_t oe = __shfl_sync(kFullMask, e, o);
      const uint32_t ox = __shfl_sync(kFullMask, excl, o);
      own[k] = o;
      act[k] = in && !((hitm >> o) & 1u);
      col[k] = act[k] ? P.icol[probe_pos(ob, oe, kPullProbes + (r - ox), reverse)] : 0u;
    }
    uint32_t bits = 0;
#pragma unroll
    for (int k = 0; k < kPullWin; k++)
      if (act[k] && bit_test_ro(fb_cur, col[k])) bits |= 1u << own[k];
    hitm |= __reduce_or_sync(kFullMask, bits);
    if ((hitm & need) == need) break;
  }
  return (hitm >> lane) & 1u;
}

// Short-circuit pull, U bitmap words per warp step.  Every candidate first
// probes up to kPullProbes in-neighbours serially, the probes of all U words
// issued together (U column loads in flight per lane); vertices still open
// after that (mostly those with no frontier neighbour at all, whose whole
// list must be read) are finished edge-parallel, word by word.
// F_{L-1}, the frontier bitmap two levels back (rotating buffers).
__device__ __forceinline__ uint32_t* old_frontier(const Level& L) {
  return L.P->fb + (size_t)((L.next_depth + 1) % 3) * L.P->w0;
}

// Also clears F_{L-1}: every word is visited once, and the store needs no
// load of the old summary.  PB in-neighbours of each candidate are probed per
// round (2 and 4 measured no faster than 1 on RMAT-22: after the first probe
// the columns come from L1).
template <int U, int PB = 1>
__device__ __forceinline__ void pull_words(Level& L, const uint32_t* fb_cur, bool reverse) {
  static_assert(kPullProbes % PB == 0, "the probe batch must divide the serial probes");
  const Params& P = *L.P;
  const uint32_t lane = threadIdx.x & 31;
  const uint32_t gwarp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const uint32_t nwarps = (gridDim.x * blockDim.x) >> 5;
  const bool same = P.iro == P.ro;
  for (uint32_t wbase = gwarp; wbase < P.w0; wbase += U * nwarps) {
    if (lane < (uint32_t)U && wbase + lane * nwarps < P.w0) st_cg(old_frontier(L) + wbase + lane * nwarps, 0u);
    uint32_t vw[U], cd[U], b[U], e[U];
    bool f[U];
    uint32_t any = 0;
#pragma unroll
    for (int k = 0; k < U; k++) {
      const uint32_t w = wbase + k * nwarps;
      vw[k] = w < P.w0 ? ld_cg(P.visited + w) : 0xffffffffu;
      cd[k] = w < P.w0 ? (~vw[k] & valid_bits(w, P.w0, P.n)) : 0u;
      any |= cd[k];
    }
    if (!any) continue;
#pragma unroll
    for (int k = 0; k < U; k++) {
      const uint32_t v = (wbase + k * nwarps) * 32 + lane;
      const bool m = (cd[k] >> lane) & 1u;
      b[k] = m ? P.iro[v] : 0u;
      e[k] = m ? P.iro[v + 1] : 0u;
      f[k] = false;
    }
    for (uint32_t j = 0; j < kPullProbes; j += PB) {
      uint32_t x[U][PB];
      bool a[U][PB];
#pragma unroll
      for (int k = 0; k < U; k++)
#pragma unroll
        for (int q = 0; q < PB; q++) {
          a[k][q] = !f[k] && b[k] + j + q < e[k];
          x[k][q] = a[k][q] ? P.icol[probe_pos(b[k], e[k], j + q, reverse)] : 0u;
        }
      uint32_t w[U][PB];
#pragma unroll
      for (int k = 0; k < U; k++)
#pragma unroll
        for (int q = 0; q < PB; q++) w[k][q] = a[k][q] ? fb_cur[x[k][q] >> 5] : 0u;  // as bit_test_ro
      bool more = false;
#pragma unroll
      for (int k = 0; k < U; k++) {
#pragma unroll
        for (int q = 0; q < PB; q++) f[k] = f[k] || (a[k][q] && ((w[k][q] >> (x[k][q] & 31)) & 1u));
        more |= !f[k] && b[k] + j + PB < e[k];
      }
      if (!__any_sync(kFullMask, more)) break;
    }
#pragma unroll
    for (int k = 0; k < U; k++) {
      if (!cd[k]) continue;  // uniform
      const uint32_t w = wbase + k * nwarps;
      const bool open = !f[k] && e[k] - b[k] > kPullProbes;
      if (__any_sync(kFullMask, open)) f[k] = pull_word_scan(P, fb_cur, open, b[k], e[k], reverse) || f[k];
      const uint32_t fmask = __ballot_sync(kFullMask, f[k]);
      if (fmask) {
        const uint32_t v = w * 32 + lane;
        if (f[k]) L.discovered(v, same ? e[k] - b[k] : (P.ro[v + 1] - P.ro[v]));
        if (lane == 0) L.publish_word(w, vw[k], fmask);
      }
    }
  }
}

// Short-circuit pull with the candidates ranked across the warp (the
// default).  A warp owns the bitmap words gwarp + k * nwarps; it loads 32 of
// them at once (one per lane), ranks their unvisited vertices and hands them
// to its lanes kRanked at a time, so every lane has kRanked candidates in
// flight whatever the density of the words: a level whose candidates are
// sparse costs the warp a few round trips, not one chain of round trips per
// group of words.  Each candidate probes its first kPullProbes in-neighbours
// serially (after the first, the columns mostly come from the same sector,
// in L1); a list still open after that -- no frontier neighbour yet and more
// in-neighbours left -- is scanned by the whole warp, kPullWin windows of 32
// edges at a time, until a hit or its end.  (Ranking the open lists' edges
// across the warp after one or two serial probes measured slower: 0.198
// against 0.157 ms per RMAT-22 traversal.)  Hits are gathered per word in
// shared memory and each lane publishes its own word (the owner of a word is
// its only writer in a pull level).  Also clears F_{L-1}.
constexpr int kRanked = 4;

__device__ __forceinline__ void pull_ranked(Level& L, const uint32_t* fb_cur, bool reverse) {
  const Params& P = *L.P;
  const uint32_t lane = threadIdx.x & 31;
  const uint32_t gwarp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const uint32_t nwarps = (gridDim.x * blockDim.x) >> 5;
  const bool same = P.iro == P.ro;
  uint32_t* found = L.S->pull_found[threadIdx.x >> 5];
  uint32_t* oldf = old_frontier(L);
  for (uint64_t k0 = 0; gwarp + k0 * nwarps < P.w0; k0 += 32) {
    const uint64_t w64 = gwarp + (k0 + lane) * nwarps;
    const bool wok = w64 < P.w0;
    const uint32_t w = wok ? (uint32_t)w64 : 0u;
    const uint32_t vw = wok ? ld_cg(P.visited + w) : 0xffffffffu;
    if (wok) st_cg(oldf + w, 0u);
    const uint32_t cand = wok ? (~vw & valid_bits(w, P.w0, P.n)) : 0u;
    found[lane] = 0u;
    __syncwarp();
    const uint32_t incl = warp_inclusive_scan((uint32_t)__popc(cand));
    const uint32_t total = __shfl_sync(kFullMask, incl, 31);
    const uint32_t excl = incl - (uint32_t)__popc(cand);
    for (uint32_t r0 = 0; r0 < total; r0 += 32 * kRanked) {
      uint32_t v[kRanked], b[kRanked], e[kRanked], own[kRanked];
      bool act[kRanked], f[kRanked];
#pragma unroll
      for (int k = 0; k < kRanked; k++) {
        const uint32_t r = r0 + k * 32 + lane;
        act[k] = r < total;
        const uint32_t o = warp_owner_of_rank(incl, act[k] ? r : total - 1);
        const uint32_t ob = __shfl_sync(kFullMask, cand, o);
        const uint32_t oe = __shfl_sync(kFullMask, excl, o);
        const uint32_t ow = __shfl_sync(kFullMask, w, o);
        own[k] = o;
        v[k] = ow * 32 + select_bit(ob, act[k] ? r - oe : 0u);
      }
      // the first probe from the first-in-neighbour array when there is one
      // (every candidate has an in-edge: the others are pre-marked visited),
      // its load issued with the offsets' and not after them
      const bool first = P.first_in && !reverse;
      uint32_t x0[kRanked];
#pragma unroll
      for (int k = 0; k < kRanked; k++) x0[k] = (first && act[k]) ? P.first_in[v[k]] : 0u;
#pragma unroll
      for (int k = 0; k < kRanked; k++) {
        b[k] = act[k] ? P.iro[v[k]] : 0u;
        e[k] = act[k] ? P.iro[v[k] + 1] : 0u;
        f[k] = false;
      }
      if (first) {
        uint32_t fw0[kRanked];
#pragma unroll
        for (int k = 0; k < kRanked; k++) fw0[k] = act[k] ? fb_cur[x0[k] >> 5] : 0u;  // as bit_test_ro
#pragma unroll
        for (int k = 0; k < kRanked; k++) f[k] = act[k] && ((fw0[k] >> (x0[k] & 31)) & 1u);
      }
      for (uint32_t j = first ? 1u : 0u; j < kPullProbes; j++) {
        uint32_t x[kRanked], fw[kRanked];
        bool a[kRanked];
#pragma unroll
        for (int k = 0; k < kRanked; k++) {
          a[k] = !f[k] && b[k] + j < e[k];
          x[k] = a[k] ? P.icol[probe_pos(b[k], e[k], j, reverse)] : 0u;
        }
#pragma unroll
        for (int k = 0; k < kRanked; k++) fw[k] = a[k] ? fb_cur[x[k] >> 5] : 0u;  // as bit_test_ro
        bool more = false;
#pragma unroll
        for (int k = 0; k < kRanked; k++) {
          f[k] = f[k] || (a[k] && ((fw[k] >> (x[k] & 31)) & 1u));
          more |= !f[k] && b[k] + j + 1 < e[k];
        }
        if (!__any_sync(kFullMask, more)) break;
      }
      // lists still open after the serial probes: the whole warp, one at a time
#pragma unroll
      for (int k = 0; k < kRanked; k++) {
        for (uint32_t om = __ballot_sync(kFullMask, act[k] && !f[k] && e[k] - b[k] > kPullProbes); om;
             om &= om - 1) {
          const uint32_t o = __ffs(om) - 1;
          const uint32_t ob = __shfl_sync(kFullMask, b[k], o), oe = __shfl_sync(kFullMask, e[k], o);
          bool hit = false;
          for (uint32_t x0 = ob + kPullProbes; x0 < oe && !hit; x0 += 32 * kPullWin) {
            uint32_t cc[kPullWin];
            bool ca[kPullWin];
#pragma unroll
            for (int q = 0; q < kPullWin; q++) {
              const uint32_t x = x0 + q * 32 + lane;
              ca[q] = x < oe;
              cc[q] = ca[q] ? P.icol[probe_pos(ob, oe, x - ob, reverse)] : 0u;
            }
            bool h = false;
#pragma unroll
            for (int q = 0; q < kPullWin; q++) h |= ca[q] && bit_test_ro(fb_cur, cc[q]);
            hit = __any_sync(kFullMask, h);
          }
          if (lane == o) f[k] = hit;
        }
      }
#pragma unroll
      for (int k = 0; k < kRanked; k++)
        if (act[k] && f[k]) {
          atomicOr(found + own[k], 1u << (v[k] & 31));
          L.discovered(v[k], same ? e[k] - b[k] : (P.ro[v[k] + 1] - P.ro[v[k]]));
        }
    }
    __syncwarp();
    const uint32_t fm = found[lane];
    __syncwarp();  // found[] is cleared again by the next chunk
    if (fm) L.publish_word(w, vw, fm);
  }
}

__device__ __forceinline__ void pull_warp(Level& L, const uint32_t* fb_cur, bool short_circuit, bool reverse) {
  const Params& P = *L.P;
  const uint32_t lane = threadIdx.x & 31;
  const uint32_t gwarp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const uint32_t nwarps = (gridDim.x * blockDim.x) >> 5;
  const bool same = P.iro == P.ro;
  if (short_circuit) {
    if (P.pull_words == 4)
      pull_words<4>(L, fb_cur, reverse);
    else if (P.pull_words == 2)
      pull_words<2>(L, fb_cur, reverse);
    else
      pull_ranked(L, fb_cur, reverse);
    return;
  }
  // pull_all: every in-neighbour of every unvisited vertex is scanned
  for (uint32_t wi = gwarp; wi < P.w0; wi += nwarps) {
    if (lane == 0) st_cg(old_frontier(L) + wi, 0u);
    const uint32_t vw = ld_cg(P.visited + wi);
    const uint32_t cand = ~vw & valid_bits(wi, P.w0, P.n);
    if (!cand) continue;
    const uint32_t v = wi * 32 + lane;
    const bool mine = (cand >> lane) & 1u;
    const uint32_t beg = mine ? P.iro[v] : 0u;
    const uint32_t end = mine ? P.iro[v + 1] : 0u;
    bool found = false;
    uint32_t e = beg;
    uint32_t c = e < end ? P.icol[e] : 0u;
    while (e < end) {
      const uint32_t cn = e + 1 < end ? P.icol[e + 1] : 0u;
      found |= bit_test_ro(fb_cur, c);
      c = cn;
      e++;
    }
    const uint32_t fmask = __ballot_sync(kFullMask, found);
    if (fmask) {
      if (found) L.discovered(v, same ? (end - beg) : (P.ro[v + 1] - P.ro[v]));
      if (lane == 0) L.publish_word(wi, vw, fmask);
    }
  }
}

__device__ __forceinline__ void pull_cta(Level& L, const uint32_t* fb_cur, bool short_circuit) {
  const Params& P = *L.P;
  Shared& S = *L.S;
  const uint32_t t = threadIdx.x, lane = t & 31, wl = t >> 5;
  const uint32_t wg = blockDim.x >> 5;
  const uint32_t ngroups = (P.w0 + wg - 1) / wg;
  const bool same = P.iro == P.ro;
  volatile uint32_t* flag = S.flag;
  for (uint32_t g = blockIdx.x; g < ngroups; g += gridDim.x) {
    const uint32_t w = g * wg + wl;
    const uint32_t vw = w < P.w0 ? ld_cg(P.visited + w) : 0xffffffffu;
    const uint32_t cand = w < P.w0 ? (~vw & valid_bits(w, P.w0, P.n)) : 0u;
    if (!__syncthreads_or(cand != 0)) continue;
    const bool mine = (cand >> lane) & 1u;
    const uint32_t v = w * 32 + lane;
    const uint32_t beg = mine ? P.iro[v] : 0u;
    const uint32_t deg = mine ? P.iro[v + 1] - beg : 0u;
    uint32_t total;
    const uint32_t excl = sygraph::detail::block_excl_scan(deg, &total, S.scan);
    S.beg[t] = beg;
    S.incl[t] = excl + deg;
    flag[t] = 0u;
    __syncthreads();
    for (uint32_t r = t; r < total; r += blockDim.x) {
      const uint32_t slot = smem_upper_bound(S.incl, blockDim.x, r);
      if (short_circuit && flag[slot]) continue;
      const uint32_t before = slot ? S.incl[slot - 1] : 0u;
      if (bit_test_ro(fb_cur, P.icol[S.beg[slot] + (r - before)])) flag[slot] = 1u;
    }
    __syncthreads();
    const bool found = mine && flag[t];
    const uint32_t fmask = __ballot_sync(kFullMask, found);
    if (found) L.discovered(v, same ? deg : (P.ro[v + 1] - P.ro[v]));
    if (lane == 0 && fmask) L.publish_word(w, vw, fmask);
    __syncthreads();
  }
}

}  // namespace bfs
}  // namespace sgb
