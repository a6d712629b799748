// Building blocks of the fused traversal engines (BFS, SSSP, CC, BC): one
// persistent cooperative kernel walks every level of a traversal with the
// frontier kept as a bitmap, a per-level bitmap -> queue compaction, and a
// degree-bucketed push expansion.  The reference runs each of these stages as
// its own launch followed by a host wait (computeActiveFrontier + D2H size
// fetch + advance + empty() + clear(), operators/advance/common.hpp:89-135,
// frontier/impls/mlb_frontier.hpp:216-246, 367-442); here they are phases
// separated by a bounded grid barrier.
#pragma once

#include "internal.cuh"

namespace sgb {
namespace eng {

using sygraph::detail::bit_test;
using sygraph::detail::bit_test_ro;
using sygraph::detail::GridBarrier;
using sygraph::detail::grid_sync;
using sygraph::detail::kFullMask;
using sygraph::detail::ld_cg;
using sygraph::detail::st_cg;
using sygraph::detail::warp_inclusive_scan;
using sygraph::detail::warp_owner_of_rank;

constexpr uint32_t kThreads = 512;     // threads per engine CTA
constexpr uint32_t kSmallDeg = 64;     // degree below which a vertex joins a 32-vertex warp group
constexpr uint32_t kChunk = 256;       // edges per work chunk of a high-degree vertex (one warp)
constexpr uint32_t kPullSerial = 32;   // edges a pull lane scans alone before the warp helps (per-source BC)
constexpr uint32_t kPullProbes = 8;    // in-neighbours a BFS pull lane probes alone before the warp scans the rest
constexpr int kPullWin = 4;            // 32-edge windows in flight in a warp's edge-parallel pull scan
constexpr uint32_t kMaxLog = SG_MAX_LOGGED_LEVELS;

// Per-level counters, three rotating slots (a slot is reset two levels
// before it is written again, after every CTA has read it).
struct Counters {
  uint32_t small_tail;
  uint32_t pad0;
  unsigned long long big_packed;  // (entries << 32) | chunks: one atomic keeps both in order
  unsigned long long new_count;   // vertices that joined the next frontier
  unsigned long long new_deg;     // sum of their (forward) degrees
  unsigned long long frontier_deg;  // push loop: out-degree sum of the frontier being expanded
};

// Frontier as queues, rebuilt from the bitmap when a push step needs them.
struct Queues {
  uint32_t* small;      // vertices of degree < kSmallDeg
  uint32_t* big;        // vertices of degree >= kSmallDeg
  uint32_t* big_start;  // first chunk index of big[i]; increasing in i
};

template <uint32_t kC = kChunk>
__device__ __forceinline__ uint32_t chunks_of(uint32_t deg) { return (deg + kC - 1) / kC; }

// Position of the k-th (0-based) set bit of x.
__device__ __forceinline__ uint32_t select_bit(uint32_t x, uint32_t k) {
  uint32_t pos = 0;
#pragma unroll
  for (uint32_t s = 16; s > 0; s >>= 1) {
    const uint32_t low = __popc(x & ((1u << s) - 1u));
    if (k >= low) {
      k -= low;
      x >>= s;
      pos += s;
    }
  }
  return pos;
}

using sygraph::detail::block_excl_scan;
using sygraph::detail::block_sum;

// Edge range [lo[v], hi[v + shift]) of vertex v in a push step: the whole row
// (lo = hi = row offsets, shift 1) or a prefix / suffix of it.
struct RowRange {
  const uint32_t* lo;
  const uint32_t* hi;
  uint32_t shift;
  __device__ __forceinline__ uint32_t beg(uint32_t v) const { return lo[v]; }
  __device__ __forceinline__ uint32_t end(uint32_t v) const { return hi[v + shift]; }
};

// Bitmap -> queues.  Each CTA owns a contiguous range of bitmap words and
// takes them 32 words per warp: the warp ranks the set bits of its words and
// every lane takes every 32nd rank, so the row-range loads of a dense word go
// out together instead of one latency per set bit.  A first pass counts each
// lane's vertices by class; one block scan and one atomic per list reserve
// the slots; a second pass repeats the same rank walk and writes them.  When
// `accumulate` is given, each word is also OR-ed into it (one thread per
// word).
template <uint32_t kC = kChunk>  // edges per chunk of a big vertex
__device__ __forceinline__ void compact_frontier(const uint32_t* __restrict__ fb, uint32_t w0, RowRange R,
                                                 Counters* C, Queues q, uint32_t* s_scan,
                                                 uint32_t* accumulate = nullptr) {
  __shared__ uint32_t s_base_small, s_base_big, s_base_chunk;
  const uint32_t lane = threadIdx.x & 31;
  const uint32_t per_block = (w0 + gridDim.x - 1) / gridDim.x;
  const uint32_t wbeg = blockIdx.x * per_block;
  const uint32_t wend = min(w0, wbeg + per_block);
  for (uint32_t base = wbeg; base < wend; base += blockDim.x) {
    const uint32_t wi = base + threadIdx.x;
    const uint32_t bits = wi < wend ? ld_cg(fb + wi) : 0u;
    if (accumulate && bits) st_cg(accumulate + wi, ld_cg(accumulate + wi) | bits);
    // words all empty across the block (most blocks of a small frontier):
    // nothing to rank, count or reserve, so one barrier instead of the scans
    if (!__syncthreads_or(bits != 0u)) continue;
    const uint32_t c = __popc(bits);
    const uint32_t incl = warp_inclusive_scan(c);
    const uint32_t total = __shfl_sync(kFullMask, incl, 31);
    const uint32_t excl = incl - c;
    const uint32_t w_first = base + (threadIdx.x & ~31u);  // the warp's first word
    // vertex of rank r (< total) among the warp's set bits
    auto vertex_of = [&](uint32_t r) {
      const uint32_t o = warp_owner_of_rank(incl, r);
      const uint32_t ob = __shfl_sync(kFullMask, bits, o);
      const uint32_t oe = __shfl_sync(kFullMask, excl, o);
      return (w_first + o) * 32 + select_bit(ob, r - oe);
    };
    uint32_t n_small = 0, n_big = 0, n_chunk = 0;
    unsigned long long fdeg = 0;
    for (uint32_t r0 = 0; r0 < total; r0 += 32) {
      const uint32_t r = r0 + lane;
      const uint32_t v = vertex_of(min(r, total - 1));
      if (r < total) {
        const uint32_t d = R.end(v) - R.beg(v);
        fdeg += d;
        if (d < kSmallDeg) {
          n_small++;
        } else {
          n_big++;
          n_chunk += chunks_of<kC>(d);
        }
      }
    }
    uint32_t t_pack, t_chunk;
    const uint32_t e_pack = block_excl_scan(n_small | (n_big << 16), &t_pack, s_scan);
    const uint32_t e_chunk = block_excl_scan(n_chunk, &t_chunk, s_scan);
    fdeg = sygraph::detail::warp_sum(fdeg);
    if (lane == 0 && fdeg) atomicAdd(&C->frontier_deg, fdeg);
    if (threadIdx.x == 0) {
      const uint32_t ts = t_pack & 0xffffu, tb = t_pack >> 16;
      s_base_small = ts ? atomicAdd(&C->small_tail, ts) : 0u;
      if (tb) {
        const unsigned long long old = atomicAdd(&C->big_packed, ((unsigned long long)tb << 32) | t_chunk);
        s_base_big = (uint32_t)(old >> 32);
        s_base_chunk = (uint32_t)old;
      }
    }
    __syncthreads();
    uint32_t ps = s_base_small + (e_pack & 0xffffu);
    uint32_t pb = s_base_big + (e_pack >> 16);
    uint32_t pc = s_base_chunk + e_chunk;
    for (uint32_t r0 = 0; r0 < total; r0 += 32) {
      const uint32_t r = r0 + lane;
      const uint32_t v = vertex_of(min(r, total - 1));
      if (r < total) {
        const uint32_t d = R.end(v) - R.beg(v);
        if (d < kSmallDeg) {
          q.small[ps++] = v;
        } else {
          q.big[pb] = v;
          q.big_start[pb] = pc;
          pb++;
          pc += chunks_of<kC>(d);
        }
      }
    }
    __syncthreads();
  }
}

// Index of the big-list entry that owns chunk c (big_start is increasing).
__device__ __forceinline__ uint32_t find_chunk_owner(const uint32_t* big_start, uint32_t entries, uint32_t c) {
  uint32_t lo = 0, hi = entries - 1;
  while (lo < hi) {
    const uint32_t mid = (lo + hi + 1) >> 1;
    if (ld_cg(big_start + mid) <= c)
      lo = mid;
    else
      hi = mid - 1;
  }
  return lo;
}

// Last entry of the increasing list start[0, n) that is <= c (start[0] <=
// c): a warp-wide 32-ary search, one load per lane per round (one round for
// up to 32 entries).  Called by the whole warp.
__device__ __forceinline__ uint32_t warp_find_owner(const uint32_t* start, uint32_t n, uint32_t c) {
  const uint32_t lane = threadIdx.x & 31;
  uint32_t lo = 0, hi = n;
  while (hi - lo > 1) {
    const uint32_t step = (hi - lo + 31) / 32;
    const uint32_t idx = lo + lane * step;
    const bool le = idx < hi && ld_cg(start + idx) <= c;
    const uint32_t m = __ballot_sync(kFullMask, le);  // a prefix of the lanes; lane 0 always
    lo += (31 - __clz(m)) * step;
    hi = min(hi, lo + step);
  }
  return lo;
}

// Degree-bucketed push expansion over the queues of one frontier.  Work units
// are 32-vertex groups of small vertices (edge-parallel inside the warp by a
// shuffle scan) and kChunk-edge chunks of big vertices; warps take units
// grid-stride.  Visitor::src(v) loads per-source state once; Visitor::visit
// (u, e, src_state, v) relaxes one edge and returns true when u must join the
// next frontier; Visitor::mark(u) is then called by that lane.
template <class Visitor>
__device__ __forceinline__ void push_expand(RowRange R, const uint32_t* __restrict__ col, Queues q, uint32_t n_small,
                                            uint32_t n_big, uint32_t n_chunks, Visitor& vis) {
  const uint32_t lane = threadIdx.x & 31;
  const uint32_t gwarp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const uint32_t nwarps = (gridDim.x * blockDim.x) >> 5;
  const uint32_t n_groups = (n_small + 31) / 32;
  const uint32_t units = n_groups + n_chunks;
  using S = typename Visitor::src_t;
  for (uint32_t unit = gwarp; unit < units; unit += nwarps) {
    if (unit < n_groups) {
      const uint32_t idx = unit * 32 + lane;
      const bool valid = idx < n_small;
      const uint32_t v = valid ? ld_cg(q.small + idx) : 0u;
      const uint32_t beg = valid ? R.beg(v) : 0u;
      const uint32_t deg = valid ? R.end(v) - beg : 0u;
      const S sv = valid ? vis.src(v) : S();
      const uint32_t incl = warp_inclusive_scan(deg);
      const uint32_t total = __shfl_sync(kFullMask, incl, 31);
      const uint32_t excl = incl - deg;
      for (uint32_t r0 = 0; r0 < total; r0 += 32) {
        const uint32_t r = r0 + lane;
        const bool act = r < total;
        const uint32_t o = warp_owner_of_rank(incl, act ? r : total - 1);
        const uint32_t ob = __shfl_sync(kFullMask, beg, o);
        const uint32_t oe = __shfl_sync(kFullMask, excl, o);
        const uint32_t ov = __shfl_sync(kFullMask, v, o);
        const S os = __shfl_sync(kFullMask, sv, o);
        if (act) {
          const uint32_t e = ob + (r - oe);
          const uint32_t u = col[e];
          if (vis.visit(u, e, os, ov)) vis.mark(u);
        }
      }
    } else {
      const uint32_t c = unit - n_groups;
      const uint32_t ent = find_chunk_owner(q.big_start, n_big, c);
      const uint32_t v = ld_cg(q.big + ent);
      const uint32_t first = ld_cg(q.big_start + ent);
      const uint32_t vb = R.beg(v), ve = R.end(v);
      const uint32_t cb = vb + (c - first) * kChunk;
      const uint32_t ce = min(ve, cb + kChunk);
      const S sv = vis.src(v);
      for (uint32_t eb = cb; eb < ce; eb += 32) {
        const uint32_t e = eb + lane;
        if (e < ce) {
          const uint32_t u = col[e];
          if (vis.visit(u, e, sv, v)) vis.mark(u);
        }
      }
    }
  }
}

__device__ __forceinline__ void compact_frontier(const uint32_t* __restrict__ fb, uint32_t w0,
                                                 const uint32_t* __restrict__ ro, Counters* C, Queues q,
                                                 uint32_t* s_scan) {
  compact_frontier(fb, w0, RowRange{ro, ro, 1}, C, q, s_scan);
}

template <class Visitor>
__device__ __forceinline__ void push_expand(const uint32_t* __restrict__ ro, const uint32_t* __restrict__ col,
                                            Queues q, uint32_t n_small, uint32_t n_big, uint32_t n_chunks,
                                            Visitor& vis) {
  push_expand(RowRange{ro, ro, 1}, col, q, n_small, n_big, n_chunks, vis);
}

__device__ __forceinline__ uint32_t valid_bits(uint32_t wi, uint32_t w0, uint32_t n) {
  const uint32_t rem = n & 31u;
  return (wi == w0 - 1 && rem) ? ((1u << rem) - 1u) : 0xffffffffu;
}

// Cooperative launch with a grid that fills every SM `blocks_per_sm` times,
// or at most `max_grid` CTAs (a share of the GPU, so that launches on other
// streams can be resident at the same time).
template <typename Params>
inline sg_status launch_persistent(void (*kernel)(Params), const Params& p, int blocks_per_sm, cudaStream_t stream,
                                   unsigned max_grid = 0, unsigned* grid_out = nullptr, unsigned threads = kThreads) {
  // the cooperative-launch attribute and the kernel's occupancy are queried
  // once per (kernel, device, block size) and thread, so a launch costs the
  // host one cudaGetDevice and the launch itself
  static thread_local int cached_dev = -1, cached_occ = 0;
  static thread_local unsigned cached_threads = 0;
  static thread_local void (*cached_kernel)(Params) = nullptr;
  int dev = 0;
  SG_CUDA(cudaGetDevice(&dev));
  if (dev != cached_dev || threads != cached_threads || kernel != cached_kernel) {
    int coop = 0, o = 0;
    SG_CUDA(cudaDeviceGetAttribute(&coop, cudaDevAttrCooperativeLaunch, dev));
    SG_REQUIRE(coop, SG_ERR_UNSUPPORTED, "device does not support cooperative launch");
    SG_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&o, kernel, (int)threads, 0));
    cached_dev = dev;
    cached_threads = threads;
    cached_kernel = kernel;
    cached_occ = o;
  }
  const int occ = cached_occ;
  SG_REQUIRE(occ > 0, SG_ERR_CUDA, "engine kernel does not fit on an SM");
  const int per_sm = occ < blocks_per_sm ? occ : blocks_per_sm;
  unsigned grid = (unsigned)(per_sm * device_props().sm_count);
  if (max_grid && max_grid < grid) grid = max_grid;
  void* args[] = {(void*)&p};
  SG_CUDA(cudaLaunchCooperativeKernel((const void*)kernel, dim3(grid), dim3(threads), args, 0, stream));
  count_launch();
  if (grid_out) *grid_out = grid;
  return SG_OK;
}

}  // namespace eng
}  // namespace sgb
