// Generic advance kernels: advance::frontier<Direction, Lb, InView, OutView>
// (operators/advance/advance.hpp:116-218) for any device functor
// bool f(src, dst, edge, weight).  The C ABI instantiates them with its
// built-in functors; the C++ header API instantiates them with user lambdas.
//
// Semantics kept from operators/advance/common.hpp:49-75:
//   candidates   push: vertices in the input frontier; pull / pull_all: the
//                vertices NOT in it; graph view: every vertex < limit
//   neighbours   push: every out-edge; pull: in-edges (the inverse graph)
//                whose endpoint is in the input frontier
//   insert       push: dst; pull: src (the candidate)
//   short-circuit (pull only): a candidate stops at its first successful edge
//
// Candidate vertices are enumerated through the input frontier's compacted
// word list (offsets[0 .. *offsets_size), written by the compaction kernel);
// the count is read on the device, so no launch needs a host round trip.
#pragma once

#include <cstdint>

#include "primitives.cuh"

namespace sygraph {
namespace detail {

enum AdvDir : int { kPush = 0, kPull = 1, kPullAll = 2 };
enum AdvView : int { kViewGraph = 0, kViewVertex = 1, kViewEdge = 2, kViewNone = 3 };

// Device view of a two-level bitmap frontier (MLBDevice,
// frontier/impls/mlb_frontier.hpp:58-153): level 0 has one bit per element,
// level 1 one bit per level-0 word.
struct MLBDev {
  uint32_t num_elems;
  uint32_t words0;
  uint32_t words1;
  uint32_t* l0;
  uint32_t* l1;
  int32_t* offsets;
  uint32_t* offsets_size;

  __device__ __forceinline__ bool check(uint32_t i) const { return (ld_cg(l0 + (i >> 5)) >> (i & 31)) & 1u; }
  // MLBDevice::insert (mlb:86-97): read first, atomicOr only when the bit is clear.
  __device__ __forceinline__ void insert(uint32_t i) const {
    const uint32_t b0 = 1u << (i & 31);
    uint32_t* w0 = l0 + (i >> 5);
    if (!(ld_cg(w0) & b0)) atomicOr(w0, b0);
    const uint32_t j = i >> 5;
    const uint32_t b1 = 1u << (j & 31);
    uint32_t* w1 = l1 + (j >> 5);
    if (!(ld_cg(w1) & b1)) atomicOr(w1, b1);
  }
  // MLBDevice::remove (mlb:99-103): level 0 only.
  __device__ __forceinline__ void remove(uint32_t i) const { atomicAnd(l0 + (i >> 5), ~(1u << (i & 31))); }
};

template <typename W>
struct GraphDev {
  uint32_t n;
  uint64_t m;
  const uint32_t* ro;
  const uint32_t* col;
  const W* val;
};

struct AdvanceArgs {
  int in_view;
  int out_view;
  uint32_t limit;  // number of vertices
  MLBDev in;
  MLBDev out;

  __device__ __forceinline__ uint32_t num_words() const {
    return in_view == kViewVertex ? ld_cg(in.offsets_size) : (limit + 31) / 32;
  }
  __device__ __forceinline__ uint32_t word_at(uint32_t i) const {
    return in_view == kViewVertex ? (uint32_t)ld_cg(in.offsets + i) : i;
  }
  template <int Dir>
  __device__ __forceinline__ bool check(uint32_t v) const {
    if (v >= limit) return false;
    if (in_view == kViewGraph) return true;
    if (in_view != kViewVertex) return false;
    return (Dir == kPush) == in.check(v);
  }
  template <int Dir>
  __device__ __forceinline__ bool valid_neighbor(uint32_t u) const {
    return Dir == kPush ? true : in.check(u);
  }
  template <int Dir>
  __device__ __forceinline__ void insert(uint32_t v, uint32_t u) const {
    if (out_view == kViewVertex) out.insert(Dir == kPush ? u : v);
  }
};

// ---- work-item mapped: one thread per candidate vertex, serial neighbour loop
template <int Dir, typename W, typename F>
__global__ void __launch_bounds__(256) advance_workitem_kernel(GraphDev<W> g, AdvanceArgs a, F f) {
  const uint64_t total = (uint64_t)a.num_words() * 32;
  for (uint64_t t = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; t < total; t += (uint64_t)gridDim.x * blockDim.x) {
    const uint32_t v = a.word_at((uint32_t)(t >> 5)) * 32 + (uint32_t)(t & 31);
    if (!a.template check<Dir>(v)) continue;
    const uint32_t end = g.ro[v + 1];
    for (uint32_t e = g.ro[v]; e < end; e++) {
      const uint32_t u = g.col[e];
      if (!a.template valid_neighbor<Dir>(u)) continue;
      if (!f(v, u, e, g.val[e])) continue;
      a.template insert<Dir>(v, u);
      if (Dir == kPull) break;
    }
  }
}

// ---- sub-group mapped: a warp walks each candidate of its word in turn,
// 32 neighbours per step (coalesced column loads).
template <int Dir, typename W, typename F>
__global__ void __launch_bounds__(256) advance_subgroup_kernel(GraphDev<W> g, AdvanceArgs a, F f) {
  const uint32_t lane = threadIdx.x & 31;
  const uint32_t nw = a.num_words();
  const uint32_t gwarp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const uint32_t nwarps = (gridDim.x * blockDim.x) >> 5;
  for (uint32_t wi = gwarp; wi < nw; wi += nwarps) {
    const uint32_t v0 = a.word_at(wi) * 32;
    uint32_t cand = __ballot_sync(kFullMask, a.template check<Dir>(v0 + lane));
    while (cand) {
      const uint32_t v = v0 + __ffs(cand) - 1;
      cand &= cand - 1;
      const uint32_t b = g.ro[v], en = g.ro[v + 1];
      for (uint32_t eb = b; eb < en; eb += 32) {
        const uint32_t e = eb + lane;
        bool ok = false;
        if (e < en) {
          const uint32_t u = g.col[e];
          if (a.template valid_neighbor<Dir>(u) && f(v, u, e, g.val[e])) {
            a.template insert<Dir>(v, u);
            ok = true;
          }
        }
        if (Dir == kPull && __any_sync(kFullMask, ok)) break;
      }
    }
  }
}

// ---- work-group mapped: a 256-thread CTA takes 8 words (256 candidates),
// scans their degrees, and walks the combined edge range; each thread finds
// its source by binary search over the inclusive degree scan in shared memory.
template <int Dir, typename W, typename F>
__global__ void __launch_bounds__(256) advance_workgroup_kernel(GraphDev<W> g, AdvanceArgs a, F f) {
  constexpr uint32_t kB = 256;
  __shared__ uint32_t s_v[kB], s_beg[kB], s_incl[kB], s_scan[32];
  __shared__ volatile uint32_t s_done[kB];
  const uint32_t t = threadIdx.x, lane = t & 31, warp = t >> 5;
  const uint32_t nw = a.num_words();
  for (uint32_t chunk = blockIdx.x; chunk * (kB / 32) < nw; chunk += gridDim.x) {
    const uint32_t wi = chunk * (kB / 32) + warp;
    uint32_t v = 0xffffffffu;
    bool act = false;
    if (wi < nw) {
      v = a.word_at(wi) * 32 + lane;
      act = a.template check<Dir>(v);
    }
    const uint32_t beg = act ? g.ro[v] : 0u;
    const uint32_t deg = act ? g.ro[v + 1] - beg : 0u;
    uint32_t total;
    const uint32_t excl = block_excl_scan(deg, &total, s_scan);
    s_v[t] = v;
    s_beg[t] = beg;
    s_incl[t] = excl + deg;
    s_done[t] = 0;
    __syncthreads();
    for (uint32_t r = t; r < total; r += kB) {
      uint32_t lo = 0, hi = kB;
      while (lo < hi) {
        const uint32_t mid = (lo + hi) >> 1;
        if (s_incl[mid] <= r)
          lo = mid + 1;
        else
          hi = mid;
      }
      const uint32_t slot = lo;
      if (Dir == kPull && s_done[slot]) continue;
      const uint32_t before = slot ? s_incl[slot - 1] : 0u;
      const uint32_t e = s_beg[slot] + (r - before);
      const uint32_t src = s_v[slot];
      const uint32_t u = g.col[e];
      if (!a.template valid_neighbor<Dir>(u)) continue;
      if (!f(src, u, e, g.val[e])) continue;
      a.template insert<Dir>(src, u);
      if (Dir == kPull) s_done[slot] = 1;
    }
    __syncthreads();
  }
}

// ---- bucketing: each candidate by degree goes to its lane (< 32), its warp
// (< kCtaDegree) or the whole CTA (the rest).
template <int Dir, typename W, typename F>
__global__ void __launch_bounds__(256) advance_bucketing_kernel(GraphDev<W> g, AdvanceArgs a, F f) {
  constexpr uint32_t kB = 256, kCtaDegree = 2048;
  __shared__ uint32_t s_big[kB];
  __shared__ uint32_t s_nbig;
  __shared__ volatile uint32_t s_claimed;
  const uint32_t t = threadIdx.x, lane = t & 31, warp = t >> 5;
  const uint32_t nw = a.num_words();
  for (uint32_t chunk = blockIdx.x; chunk * (kB / 32) < nw; chunk += gridDim.x) {
    if (t == 0) s_nbig = 0;
    __syncthreads();
    const uint32_t wi = chunk * (kB / 32) + warp;
    uint32_t v = 0;
    bool act = false;
    if (wi < nw) {
      v = a.word_at(wi) * 32 + lane;
      act = a.template check<Dir>(v);
    }
    const uint32_t beg = act ? g.ro[v] : 0u;
    const uint32_t deg = act ? g.ro[v + 1] - beg : 0u;
    const bool big = act && deg >= kCtaDegree;
    const bool mid = act && !big && deg >= 32;
    const bool small = act && deg < 32;
    if (big) s_big[atomicAdd(&s_nbig, 1u)] = v;
    // warp bucket
    uint32_t mids = __ballot_sync(kFullMask, mid);
    while (mids) {
      const uint32_t j = __ffs(mids) - 1;
      mids &= mids - 1;
      const uint32_t vj = __shfl_sync(kFullMask, v, j);
      const uint32_t bj = __shfl_sync(kFullMask, beg, j);
      const uint32_t ej = bj + __shfl_sync(kFullMask, deg, j);
      for (uint32_t eb = bj; eb < ej; eb += 32) {
        const uint32_t e = eb + lane;
        bool ok = false;
        if (e < ej) {
          const uint32_t u = g.col[e];
          if (a.template valid_neighbor<Dir>(u) && f(vj, u, e, g.val[e])) {
            a.template insert<Dir>(vj, u);
            ok = true;
          }
        }
        if (Dir == kPull && __any_sync(kFullMask, ok)) break;
      }
    }
    // lane bucket: serial, stops at the first success in pull mode
    if (small) {
      for (uint32_t e = beg; e < beg + deg; e++) {
        const uint32_t u = g.col[e];
        if (!a.template valid_neighbor<Dir>(u)) continue;
        if (!f(v, u, e, g.val[e])) continue;
        a.template insert<Dir>(v, u);
        if (Dir == kPull) break;
      }
    }
    __syncthreads();
    // CTA bucket
    const uint32_t nbig = s_nbig;
    for (uint32_t i = 0; i < nbig; i++) {
      const uint32_t vb = s_big[i];
      const uint32_t b = g.ro[vb], en = g.ro[vb + 1];
      if (t == 0) s_claimed = 0;
      __syncthreads();
      for (uint32_t e = b + t; e < en; e += kB) {
        if (Dir == kPull && s_claimed) break;
        const uint32_t u = g.col[e];
        if (!a.template valid_neighbor<Dir>(u)) continue;
        if (!f(vb, u, e, g.val[e])) continue;
        a.template insert<Dir>(vb, u);
        if (Dir == kPull) s_claimed = 1;
      }
      __syncthreads();
    }
  }
}

// Host launcher; lb follows operators/config.hpp (0 workitem, 1 subgroup,
// 2 workgroup, 3 bucketing).  Returns the CUDA launch status.
template <int Dir, typename W, typename F>
inline cudaError_t launch_advance(int lb, const GraphDev<W>& g, const AdvanceArgs& a, const F& f, unsigned grid,
                                  cudaStream_t stream) {
  switch (lb) {
    case 0: advance_workitem_kernel<Dir, W, F><<<grid, 256, 0, stream>>>(g, a, f); break;
    case 1: advance_subgroup_kernel<Dir, W, F><<<grid, 256, 0, stream>>>(g, a, f); break;
    case 2: advance_workgroup_kernel<Dir, W, F><<<grid, 256, 0, stream>>>(g, a, f); break;
    case 3: advance_bucketing_kernel<Dir, W, F><<<grid, 256, 0, stream>>>(g, a, f); break;
    default: return cudaErrorInvalidValue;
  }
  return cudaGetLastError();
}

// ---- frontier-wide helpers used by filter / compute (one thread per
// candidate of the compacted input).
template <typename P>
__global__ void __launch_bounds__(256) filter_external_kernel(MLBDev in, MLBDev out, uint32_t limit, P pred) {
  const uint64_t total = (uint64_t)ld_cg(in.offsets_size) * 32;
  for (uint64_t t = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; t < total; t += (uint64_t)gridDim.x * blockDim.x) {
    const uint32_t v = (uint32_t)ld_cg(in.offsets + (t >> 5)) * 32 + (uint32_t)(t & 31);
    if (v < limit && in.check(v) && pred(v)) out.insert(v);
  }
}

template <typename P>
__global__ void __launch_bounds__(256) filter_inplace_kernel(MLBDev f, uint32_t limit, P pred) {
  const uint64_t total = (uint64_t)ld_cg(f.offsets_size) * 32;
  for (uint64_t t = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; t < total; t += (uint64_t)gridDim.x * blockDim.x) {
    const uint32_t v = (uint32_t)ld_cg(f.offsets + (t >> 5)) * 32 + (uint32_t)(t & 31);
    if (v < limit && f.check(v) && pred(v)) f.remove(v);
  }
}

template <typename Fn>
__global__ void __launch_bounds__(256) compute_execute_kernel(MLBDev f, uint32_t limit, Fn fn) {
  const uint64_t total = (uint64_t)ld_cg(f.offsets_size) * 32;
  for (uint64_t t = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; t < total; t += (uint64_t)gridDim.x * blockDim.x) {
    const uint32_t v = (uint32_t)ld_cg(f.offsets + (t >> 5)) * 32 + (uint32_t)(t & 31);
    if (v < limit && f.check(v)) fn(v);
  }
}

// Sum of fn(v) over the active vertices; one atomic per CTA.
template <typename Fn>
__global__ void __launch_bounds__(256) compute_reduce_kernel(MLBDev f, uint32_t limit, Fn fn,
                                                             unsigned long long* out) {
  __shared__ unsigned long long s_red[32];
  const uint64_t total = (uint64_t)ld_cg(f.offsets_size) * 32;
  unsigned long long acc = 0;
  for (uint64_t t = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; t < total; t += (uint64_t)gridDim.x * blockDim.x) {
    const uint32_t v = (uint32_t)ld_cg(f.offsets + (t >> 5)) * 32 + (uint32_t)(t & 31);
    if (v < limit && f.check(v)) acc += fn(v);
  }
  acc = block_sum(acc, s_red);
  if (threadIdx.x == 0 && acc) atomicAdd(out, acc);
}

}  // namespace detail
}  // namespace sygraph
