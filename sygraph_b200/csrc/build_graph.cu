// Graph construction on the device: edge list -> CSR (forward, and the
// inverse for directed graphs).  The reference builds on the host:
// io::csr::fromCOO (io/read_csr.hpp:260-300), formats::CSR::invert
// (formats/csr.hpp:179-209) and the upload of GraphCSR
// (graph/impls/graph_csr.hpp:394-426); sg_csr_from_edges is that host path.
// Here one persistent cooperative kernel does it all:
//   fill    entry 2i / 2i+1 (or i) = (u, v) / (v, u) of edge i as the key
//           u * 2^b + v (2^b > n); a dropped entry (a self-loop when they are
//           dropped, the reverse of a self-loop) gets the all-ones key, which
//           sorts after every edge
//   sort    LSD radix sort of (key, value) pairs, 8 bits per pass.  Each CTA
//           owns one contiguous range of the array in every pass: it counts
//           its digits, and after a grid barrier scatters its range in order,
//           one thread per entry and 512 entries per round, equal digits
//           ranked by warp match groups -- a stable sort, so equal keys keep
//           their insertion order
//   compact the first entry of every run of equal keys (every entry without
//           de-duplication) is kept, in order: columns, values, and the row
//           offset of each non-empty row; empty rows take the next row's
//           offset by a backward minimum scan
// The result is bit-identical to the host path's (stable sort by key, keep
// the first of equal keys).
#include <algorithm>
#include <cstring>
#include <mutex>
#include <vector>

#include "engine_common.cuh"

namespace sgb {
namespace gb {

using namespace eng;
using u64 = unsigned long long;

constexpr u64 kNone = ~0ull;
constexpr uint32_t kWarps = kThreads / 32;

struct BuildParams {
  const uint32_t* src;
  const uint32_t* dst;
  const uint32_t* val;  // nullptr: every value is `one`
  uint64_t count;
  uint32_t n;
  uint32_t b;  // bits per endpoint (2^b > n)
  uint32_t one;
  int symmetrize, dedupe, drop_self_loops;
  uint64_t entries;
  uint32_t passes;
  u64* k0;
  u64* k1;
  uint32_t* v0;
  uint32_t* v1;
  uint32_t* hist;   // 256 * gridDim.x
  u64* csum;        // gridDim.x
  uint32_t* ro;     // n + 1
  uint32_t* col;    // compacted columns (entries)
  uint32_t* oval;   // compacted values (entries)
  u64* m_out;
  uint32_t* bad;    // an endpoint was >= n
  GridBarrier* bar;
};

struct Shared {
  uint32_t hist[256];
  uint32_t base[256];
  uint32_t tot[256];
  uint32_t cnt[kWarps][256];
  uint32_t scan[32];
  uint32_t wmin[kWarps];
  u64 red[32];
};

// Suffix minimum of x over the block's threads (thread t gets min of x over
// t..blockDim-1).
__device__ __forceinline__ uint32_t block_suffix_min(uint32_t x, Shared& S) {
  const uint32_t lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
#pragma unroll
  for (int d = 1; d < 32; d <<= 1) {
    const uint32_t y = __shfl_down_sync(kFullMask, x, d);
    if (lane + d < 32) x = min(x, y);
  }
  if (lane == 0) S.wmin[warp] = x;
  __syncthreads();
  uint32_t later = 0xffffffffu;
  for (uint32_t w = warp + 1; w < nw; w++) later = min(later, S.wmin[w]);
  __syncthreads();
  return min(x, later);
}

// LSD radix sort of (key, value) pairs, `passes` digits of 8 bits from bit
// `shift0` up.  CTA c owns [lo, hi) of the array in every pass: it counts its
// digits, and after a grid barrier scatters its range in order, one thread
// per entry and blockDim entries per round, equal digits ranked by warp match
// groups -- a stable sort.  On return kin / vin hold the sorted pairs (the
// pointers are swapped after every pass).  False when a barrier wait ran out.
__device__ __forceinline__ bool radix_sort_pairs(Shared& S, GridBarrier* bar, uint32_t* ghist, u64*& kin,
                                                 u64*& kout, uint32_t*& vin, uint32_t*& vout, uint64_t lo,
                                                 uint64_t hi, uint32_t shift0, uint32_t passes) {
  const uint32_t G = gridDim.x, c = blockIdx.x, t = threadIdx.x, lane = t & 31, warp = t >> 5;
  for (uint32_t p = 0; p < passes; p++) {
    const uint32_t sh = shift0 + 8 * p;
    if (t < 256) S.hist[t] = 0;
    __syncthreads();
    for (uint64_t i = lo + t; i < hi; i += blockDim.x) atomicAdd(&S.hist[(uint32_t)(kin[i] >> sh) & 255u], 1u);
    __syncthreads();
    if (t < 256) ghist[(size_t)t * G + c] = S.hist[t];
    if (!grid_sync(bar)) return false;
    uint32_t tot = 0, before = 0;
    if (t < 256) {
      for (uint32_t cc = 0; cc < G; cc++) {
        const uint32_t x = ld_cg(ghist + (size_t)t * G + cc);
        tot += x;
        if (cc < c) before += x;
      }
    }
    uint32_t all;
    const uint32_t dbase = sygraph::detail::block_excl_scan(t < 256 ? tot : 0u, &all, S.scan);
    if (t < 256) S.base[t] = dbase + before;
    __syncthreads();
    for (uint64_t r0 = lo; r0 < hi; r0 += blockDim.x) {
      const uint64_t i = r0 + t;
      const bool in = i < hi;
      const u64 k = in ? kin[i] : 0ull;
      const uint32_t vv = in ? vin[i] : 0u;
      const uint32_t d = in ? ((uint32_t)(k >> sh) & 255u) : 256u;
      for (uint32_t x = t; x < kWarps * 256; x += blockDim.x) (&S.cnt[0][0])[x] = 0u;
      __syncthreads();
      const uint32_t grp = __match_any_sync(kFullMask, d);
      const uint32_t rank = __popc(grp & ((1u << lane) - 1u));
      if (in && rank == 0) S.cnt[warp][d] = __popc(grp);
      __syncthreads();
      if (t < 256) {
        uint32_t run = 0;
        for (uint32_t w = 0; w < kWarps; w++) {
          const uint32_t x = S.cnt[w][t];
          S.cnt[w][t] = run;
          run += x;
        }
        S.tot[t] = run;
      }
      __syncthreads();
      if (in) {
        const uint32_t pos = S.base[d] + S.cnt[warp][d] + rank;
        kout[pos] = k;
        vout[pos] = vv;
      }
      __syncthreads();
      if (t < 256) S.base[t] += S.tot[t];
    }
    u64* tk = kin;
    kin = kout;
    kout = tk;
    uint32_t* tv = vin;
    vin = vout;
    vout = tv;
    if (!grid_sync(bar)) return false;
  }
  return true;
}

__global__ void __launch_bounds__(kThreads, 2) build_kernel(BuildParams P) {
  __shared__ Shared S;
  const uint32_t G = gridDim.x, c = blockIdx.x, t = threadIdx.x, lane = t & 31, warp = t >> 5;
  const uint64_t nth = (uint64_t)G * blockDim.x;
  const uint64_t gtid = (uint64_t)c * blockDim.x + t;
  const uint64_t E = P.entries;
  const uint64_t per = (E + G - 1) / G;
  const uint64_t lo = min(E, (uint64_t)c * per), hi = min(E, lo + per);
  const uint32_t bmask = (1u << P.b) - 1u;

  // ---- fill
  for (uint64_t i = gtid; i < E; i += nth) {
    const uint64_t j = P.symmetrize ? i >> 1 : i;
    const bool rev = P.symmetrize && (i & 1);
    const uint32_t u = P.src[j], v = P.dst[j];
    bool drop = (P.drop_self_loops && u == v) || (rev && u == v);
    if (u >= P.n || v >= P.n) {
      atomicOr(P.bad, 1u);
      drop = true;
    }
    const uint32_t a = rev ? v : u, z = rev ? u : v;
    P.k0[i] = drop ? kNone : (((u64)a << P.b) | z);
    P.v0[i] = P.val ? P.val[j] : P.one;
  }
  for (uint64_t v = gtid; v <= P.n; v += nth) P.ro[v] = 0xffffffffu;
  if (!grid_sync(P.bar)) return;

  // ---- sort
  u64* kin = P.k0;
  u64* kout = P.k1;
  uint32_t* vin = P.v0;
  uint32_t* vout = P.v1;
  if (!radix_sort_pairs(S, P.bar, P.hist, kin, kout, vin, vout, lo, hi, 0, P.passes)) return;

  // ---- compact: kept entries in order, and the row start of each non-empty row
  auto keep = [&](uint64_t i, u64 k) {
    return k != kNone && (!P.dedupe || i == 0 || kin[i - 1] != k);
  };
  u64 mine = 0;
  for (uint64_t i = lo + t; i < hi; i += blockDim.x) mine += keep(i, kin[i]) ? 1u : 0u;
  const u64 csum = sygraph::detail::block_sum<u64>(mine, S.red);
  if (t == 0) P.csum[c] = csum;
  if (!grid_sync(P.bar)) return;
  u64 base = 0, m = 0;
  for (uint32_t cc = 0; cc < G; cc++) {
    const u64 x = ld_cg(P.csum + cc);
    m += x;
    if (cc < c) base += x;
  }
  for (uint64_t r0 = lo; r0 < hi; r0 += blockDim.x) {
    const uint64_t i = r0 + t;
    const u64 k = i < hi ? kin[i] : kNone;
    const bool kp = i < hi && keep(i, k);
    uint32_t total;
    const uint32_t ex = sygraph::detail::block_excl_scan(kp ? 1u : 0u, &total, S.scan);
    if (kp) {
      const uint32_t pos = (uint32_t)(base + ex);
      const uint32_t s = (uint32_t)(k >> P.b);
      P.col[pos] = (uint32_t)k & bmask;
      P.oval[pos] = vin[i];
      // first kept entry of row s: nothing before it in the sorted order
      // shares its row (a duplicate of the same key shares it and is not kept)
      if (i == 0 || (kin[i - 1] >> P.b) != (u64)s) P.ro[s] = pos;
    }
    base += total;
    __syncthreads();
  }
  if (gtid == 0) {
    P.ro[P.n] = (uint32_t)m;
    *P.m_out = m;
  }
  if (!grid_sync(P.bar)) return;

  // ---- empty rows take the offset of the next non-empty row: backward
  // minimum over ro (ro[n] = m is always set)
  const uint64_t nr = (uint64_t)P.n + 1;
  const uint64_t rper = (nr + G - 1) / G;
  const uint64_t rlo = min(nr, (uint64_t)c * rper), rhi = min(nr, rlo + rper);
  uint32_t mn = 0xffffffffu;
  for (uint64_t v = rlo + t; v < rhi; v += blockDim.x) mn = min(mn, P.ro[v]);
  mn = block_suffix_min(mn, S);  // thread 0 holds the range's minimum
  if (t == 0) P.csum[c] = mn;
  if (!grid_sync(P.bar)) return;
  uint32_t carry = 0xffffffffu;
  for (uint32_t cc = c + 1; cc < G; cc++) carry = min(carry, (uint32_t)ld_cg(P.csum + cc));
  if (rhi > rlo) {
    for (uint64_t e0 = rhi; e0 > rlo;) {
      const uint64_t b0 = e0 - rlo > blockDim.x ? e0 - blockDim.x : rlo;
      const uint64_t v = b0 + t;
      const uint32_t x = v < e0 ? P.ro[v] : 0xffffffffu;
      const uint32_t y = min(block_suffix_min(x, S), carry);
      if (v < e0) P.ro[v] = y;
      // the chunk's minimum (thread 0's suffix) carries to the chunk before
      if (t == 0) S.scan[0] = y;
      __syncthreads();
      carry = S.scan[0];
      __syncthreads();
      e0 = b0;
    }
  }
}


// ---- weight-sorted adjacency (delta-stepping SSSP) ---------------------------
//
// Every row of the forward CSR sorted by weight, on the device: the pairs
// (row << 32 | weight bits, column) of all edges, filled in row order, are
// radix-sorted on the weight digits and then the row digits (stable, so equal
// weights keep their column order); weights are non-negative float32 or
// uint32, whose bit patterns order like the values.  The same pass checks
// whether the weighted adjacency is symmetric (each row strictly increasing
// in column, every edge's reverse present with the same weight), which the
// pull phases of delta-stepping need.
constexpr uint32_t kWsBig = 256;  // rows at least this long are filled by a whole warp

struct WsortParams {
  const uint32_t* ro;
  const uint32_t* col;
  const uint32_t* val;
  uint32_t n;
  uint64_t m;
  uint32_t passes;  // 4 weight digits + the row digits
  u64* k0;
  u64* k1;
  uint32_t* v0;
  uint32_t* v1;
  uint32_t* hist;       // 256 * gridDim.x
  uint32_t* big;        // rows of at least kWsBig edges (n entries)
  uint32_t* big_count;
  uint32_t* asym;       // set when the adjacency is not symmetric with sorted rows
  uint32_t* wval;       // out: sorted weights (m)
  GridBarrier* bar;
};

// Edge i of row v: its sort pair, and whether it breaks symmetry.
__device__ __forceinline__ bool ws_edge(const WsortParams& P, uint32_t v, uint64_t i, uint64_t e) {
  const uint32_t u = P.col[i], w = P.val[i];
  P.k0[i] = ((u64)v << 32) | w;
  P.v0[i] = u;
  if (i + 1 < e && u >= P.col[i + 1]) return true;
  uint32_t lo = P.ro[u], hi = P.ro[u + 1];  // v in row u (sorted): lower bound
  while (lo < hi) {
    const uint32_t mid = (lo + hi) >> 1;
    if (P.col[mid] < v)
      lo = mid + 1;
    else
      hi = mid;
  }
  return lo == P.ro[u + 1] || P.col[lo] != v || P.val[lo] != w;
}

__global__ void __launch_bounds__(kThreads, 2) wsort_kernel(WsortParams P) {
  __shared__ Shared S;
  const uint32_t G = gridDim.x, c = blockIdx.x, lane = threadIdx.x & 31;
  const uint64_t nth = (uint64_t)G * blockDim.x;
  const uint64_t gtid = (uint64_t)c * blockDim.x + threadIdx.x;
  bool bad = false;
  // ---- fill: short rows one thread each, long rows listed for whole warps
  for (uint64_t v = gtid; v < P.n; v += nth) {
    const uint32_t b = P.ro[v], e = P.ro[v + 1];
    if (e - b >= kWsBig) {
      P.big[atomicAdd(P.big_count, 1u)] = (uint32_t)v;
      continue;
    }
    for (uint32_t i = b; i < e; i++) bad |= ws_edge(P, (uint32_t)v, i, e);
  }
  if (!grid_sync(P.bar)) return;
  const uint32_t nbig = ld_cg(P.big_count);
  for (uint64_t j = gtid >> 5; j < nbig; j += nth >> 5) {
    const uint32_t v = ld_cg(P.big + j);
    const uint32_t b = P.ro[v], e = P.ro[v + 1];
    for (uint32_t i = b + lane; i < e; i += 32) bad |= ws_edge(P, v, i, e);
  }
  if (__any_sync(kFullMask, bad) && lane == 0) atomicOr(P.asym, 1u);
  if (!grid_sync(P.bar)) return;
  // ---- sort: weight digits (bits 0-31), then row digits
  const uint64_t per = (P.m + G - 1) / G;
  const uint64_t lo = min(P.m, (uint64_t)c * per), hi = min(P.m, lo + per);
  u64* kin = P.k0;
  u64* kout = P.k1;
  uint32_t* vin = P.v0;
  uint32_t* vout = P.v1;
  if (!radix_sort_pairs(S, P.bar, P.hist, kin, kout, vin, vout, lo, hi, 0, P.passes)) return;
  // ---- the sorted weights (the sorted columns stay in vin)
  for (uint64_t i = gtid; i < P.m; i += nth) P.wval[i] = (uint32_t)kin[i];
}

}  // namespace gb

namespace {

uint32_t bit_length(uint32_t x) { return x ? 32u - (uint32_t)__builtin_clz(x) : 1u; }

}  // namespace

// Builds g->wcol / g->wval (rows of the forward CSR sorted by weight) and
// g->wsym once per graph, on the device (wsort_kernel).
sg_status graph_weight_sorted(sg_graph g) {
  std::lock_guard<std::mutex> lk(g->wsort_mu);
  if (g->wcol) return SG_OK;
  SG_REQUIRE(g->fwd.val && g->value_type != SG_WEIGHT_NONE, SG_ERR_INVALID, "the graph has no weights");
  const uint32_t n = g->n;
  const uint64_t m = g->m;
  cudaStream_t st = g->stream;
  gb::WsortParams P = {};
  P.ro = g->fwd.ro;
  P.col = g->fwd.col;
  P.val = reinterpret_cast<const uint32_t*>(g->fwd.val);
  P.n = n;
  P.m = m;
  P.passes = 4 + (bit_length(n - 1) + 7) / 8;
  const uint64_t grid = 2ull * device_props().sm_count;
  const uint64_t ma = m ? m : 1;
  uint32_t* wv = nullptr;
  uint32_t* flags = nullptr;  // big_count, asym
  sg_status s = SG_OK;
  do {
    if ((s = dev_alloc(&P.k0, ma)) || (s = dev_alloc(&P.k1, ma)) || (s = dev_alloc(&P.v0, ma)) ||
        (s = dev_alloc(&P.v1, ma)) || (s = dev_alloc(&P.hist, 256 * grid)) || (s = dev_alloc(&P.big, (uint64_t)n)) ||
        (s = dev_alloc(&flags, 2)) || (s = dev_alloc(&P.bar, 1)) || (s = dev_alloc(&wv, ma)))
      break;
    P.big_count = flags;
    P.asym = flags + 1;
    P.wval = wv;
    cudaError_t e = cudaMemsetAsync(P.bar, 0, sizeof(*P.bar), st);
    if (e == cudaSuccess) e = cudaMemsetAsync(flags, 0, 2 * sizeof(uint32_t), st);
    if (e != cudaSuccess) {
      s = cuda_fail(e, "memset", __FILE__, __LINE__);
      break;
    }
    if ((s = eng::launch_persistent(gb::wsort_kernel, P, 2, st)) != SG_OK) break;
    uint32_t hf[2] = {0, 0};
    sygraph::detail::GridBarrier hb;
    e = cudaMemcpyAsync(hf, flags, sizeof(hf), cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaMemcpyAsync(&hb, P.bar, sizeof(hb), cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    if (e != cudaSuccess) {
      s = cuda_fail(e, "weight sort", __FILE__, __LINE__);
      break;
    }
    if (hb.error) {
      s = fail(SG_ERR_TIMEOUT, "weight sort: a grid barrier wait ran out");
      break;
    }
    // after an even number of passes the sorted columns are in v0, else v1
    uint32_t*& sorted_col = P.passes % 2 == 0 ? P.v0 : P.v1;
    g->wcol = sorted_col;
    sorted_col = nullptr;
    g->wval = wv;
    wv = nullptr;
    g->wsym = hf[1] == 0;
    g->bytes += 8ull * m;
  } while (0);
  dev_free(P.k0);
  dev_free(P.k1);
  dev_free(P.v0);
  dev_free(P.v1);
  dev_free(P.hist);
  dev_free(P.big);
  dev_free(flags);
  dev_free(P.bar);
  dev_free(wv);
  return s;
}

namespace {

// One direction (forward, or with src / dst swapped the inverse) of a build;
// out gets device arrays ro (n+1), col and val (m each).
sg_status build_direction(const uint32_t* dsrc, const uint32_t* ddst, const uint32_t* dval, uint64_t count,
                          uint32_t n, uint32_t one, int symmetrize, int dedupe, int drop_self_loops,
                          cudaStream_t stream, GraphDir* out, uint64_t* m_out) {
  const uint64_t E = symmetrize ? 2 * count : count;
  gb::BuildParams P = {};
  P.src = dsrc;
  P.dst = ddst;
  P.val = dval;
  P.count = count;
  P.n = n;
  P.b = bit_length(n);
  P.one = one;
  P.symmetrize = symmetrize;
  P.dedupe = dedupe;
  P.drop_self_loops = drop_self_loops;
  P.entries = E;
  P.passes = (2 * P.b + 7) / 8;
  const uint64_t grid = 2ull * device_props().sm_count;  // at least the launch's grid
  const uint64_t Ea = E ? E : 1;
  sg_status s = SG_OK;
  uint32_t* ro = nullptr;
  uint32_t* col = nullptr;
  uint32_t* val = nullptr;
  do {
    if ((s = dev_alloc(&P.k0, Ea)) || (s = dev_alloc(&P.k1, Ea)) || (s = dev_alloc(&P.v0, Ea)) ||
        (s = dev_alloc(&P.v1, Ea)) || (s = dev_alloc(&P.hist, 256 * grid)) || (s = dev_alloc(&P.csum, grid)) ||
        (s = dev_alloc(&ro, (uint64_t)n + 1)) || (s = dev_alloc(&P.m_out, 1)) || (s = dev_alloc(&P.bad, 1)) ||
        (s = dev_alloc(&P.bar, 1)))
      break;
    P.ro = ro;
    // compacted columns / row ids / values go to the sort buffers that the
    // last pass leaves free (the pass count decides which ones)
    const bool even = P.passes % 2 == 0;
    P.col = reinterpret_cast<uint32_t*>(even ? P.k1 : P.k0);
    P.oval = even ? P.v1 : P.v0;
    cudaError_t e = cudaMemsetAsync(P.bar, 0, sizeof(*P.bar), stream);
    if (e == cudaSuccess) e = cudaMemsetAsync(P.bad, 0, sizeof(uint32_t), stream);
    if (e != cudaSuccess) {
      s = cuda_fail(e, "memset", __FILE__, __LINE__);
      break;
    }
    if ((s = eng::launch_persistent(gb::build_kernel, P, 2, stream)) != SG_OK) break;
    uint64_t m = 0;
    uint32_t bad = 0;
    sygraph::detail::GridBarrier hb;
    e = cudaMemcpyAsync(&m, P.m_out, sizeof(m), cudaMemcpyDeviceToHost, stream);
    if (e == cudaSuccess) e = cudaMemcpyAsync(&bad, P.bad, sizeof(bad), cudaMemcpyDeviceToHost, stream);
    if (e == cudaSuccess) e = cudaMemcpyAsync(&hb, P.bar, sizeof(hb), cudaMemcpyDeviceToHost, stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(stream);
    if (e != cudaSuccess) {
      s = cuda_fail(e, "graph build", __FILE__, __LINE__);
      break;
    }
    if (hb.error) {
      s = fail(SG_ERR_TIMEOUT, "graph build: a grid barrier wait ran out");
      break;
    }
    if (bad) {
      s = fail(SG_ERR_INVALID, "edge endpoint out of range");
      break;
    }
    if (m >= (1ull << 32)) {
      s = fail(SG_ERR_INVALID, "edge count must fit uint32 offsets");
      break;
    }
    if ((s = dev_alloc(&col, m ? m : 1)) || (s = dev_alloc(&val, m ? m : 1))) break;
    if (m) {
      e = cudaMemcpyAsync(col, P.col, sizeof(uint32_t) * m, cudaMemcpyDeviceToDevice, stream);
      if (e == cudaSuccess) e = cudaMemcpyAsync(val, P.oval, sizeof(uint32_t) * m, cudaMemcpyDeviceToDevice, stream);
      if (e == cudaSuccess) e = cudaStreamSynchronize(stream);
      if (e != cudaSuccess) {
        s = cuda_fail(e, "graph build copy", __FILE__, __LINE__);
        break;
      }
    }
    out->ro = ro;
    out->col = col;
    out->val = val;
    *m_out = m;
    ro = col = val = nullptr;
  } while (0);
  dev_free(P.k0);
  dev_free(P.k1);
  dev_free(P.v0);
  dev_free(P.v1);
  dev_free(P.hist);
  dev_free(P.csum);
  dev_free(P.m_out);
  dev_free(P.bad);
  dev_free(P.bar);
  dev_free(ro);
  dev_free(col);
  dev_free(val);
  return s;
}

}  // namespace
}  // namespace sgb

using namespace sgb;

extern "C" {

sg_status sg_graph_create_coo(const uint32_t* src, const uint32_t* dst, const void* values, int value_type,
                              uint32_t n, uint64_t count, int symmetrize, int dedupe, int drop_self_loops,
                              int device_pointers, void* stream, sg_graph* out) {
  clear_error();
  SG_REQUIRE(out, SG_ERR_INVALID, "out is NULL");
  *out = nullptr;
  SG_REQUIRE(count == 0 || (src && dst), SG_ERR_INVALID, "NULL edge array");
  SG_REQUIRE(n > 0 && n < 0x7fffffffu, SG_ERR_INVALID, "vertex count must be in [1, 2^31)");
  SG_REQUIRE(value_type == SG_WEIGHT_NONE || value_type == SG_WEIGHT_F32 || value_type == SG_WEIGHT_U32,
             SG_ERR_INVALID, "unknown value_type");
  SG_REQUIRE((symmetrize ? 2 * count : count) < (1ull << 32), SG_ERR_INVALID,
             "edge entries (twice the edges when symmetrised) must be below 2^32");
  cudaStream_t st = (cudaStream_t)stream;
  const bool weighted = value_type != SG_WEIGHT_NONE && values;
  // missing weights are ones, as sg_graph_create_csr stores them
  uint32_t one = 1u;
  if (value_type == SG_WEIGHT_F32) {
    const float f = 1.0f;
    memcpy(&one, &f, 4);
  }
  const uint32_t* dsrc = src;
  const uint32_t* ddst = dst;
  const uint32_t* dval = weighted ? (const uint32_t*)values : nullptr;
  uint32_t* own[3] = {nullptr, nullptr, nullptr};
  sg_status s = SG_OK;
  if (!device_pointers && count) {
    if ((s = dev_alloc(&own[0], count)) || (s = dev_alloc(&own[1], count)) ||
        (weighted && (s = dev_alloc(&own[2], count)))) {
      for (auto* p : own) dev_free(p);
      return s;
    }
    cudaError_t e = cudaMemcpyAsync(own[0], src, 4 * count, cudaMemcpyHostToDevice, st);
    if (e == cudaSuccess) e = cudaMemcpyAsync(own[1], dst, 4 * count, cudaMemcpyHostToDevice, st);
    if (e == cudaSuccess && weighted) e = cudaMemcpyAsync(own[2], values, 4 * count, cudaMemcpyHostToDevice, st);
    if (e != cudaSuccess) {
      for (auto* p : own) dev_free(p);
      return cuda_fail(e, "edge upload", __FILE__, __LINE__);
    }
    dsrc = own[0];
    ddst = own[1];
    dval = weighted ? own[2] : nullptr;
  }
  sg_graph g = new sg_graph_s();
  g->n = n;
  g->flags = (symmetrize ? 0u : SG_GRAPH_DIRECTED) | (value_type != SG_WEIGHT_NONE ? SG_GRAPH_WEIGHTED : 0u);
  g->stream = st;
  g->value_type = value_type == SG_WEIGHT_NONE ? SG_WEIGHT_U32 : value_type;
  uint64_t m = 0;
  s = build_direction(dsrc, ddst, dval, count, n, one, symmetrize, dedupe, drop_self_loops, st, &g->fwd, &m);
  if (s == SG_OK) {
    g->m = m;
    g->bytes = sizeof(uint32_t) * ((uint64_t)n + 1 + 2 * m);
    if (symmetrize) {
      g->inv = g->fwd;
      g->owns_inverse = false;
    } else {
      uint64_t mi = 0;
      s = build_direction(ddst, dsrc, dval, count, n, one, 0, dedupe, drop_self_loops, st, &g->inv, &mi);
      if (s == SG_OK) {
        g->owns_inverse = true;
        g->bytes *= 2;
      }
    }
  }
  for (auto* p : own) dev_free(p);
  if (s != SG_OK) {
    release_graph(g);
    return s;
  }
  *out = g;
  return SG_OK;
}

sg_status sg_graph_weight_sorted(sg_graph g, uint32_t* host_column_indices, void* host_values, int* symmetric) {
  clear_error();
  SG_REQUIRE(g, SG_ERR_INVALID, "graph is NULL");
  SG_TRY(graph_weight_sorted(g));
  if (host_column_indices && g->m)
    SG_CUDA(cudaMemcpyAsync(host_column_indices, g->wcol, sizeof(uint32_t) * g->m, cudaMemcpyDeviceToHost, g->stream));
  if (host_values && g->m)
    SG_CUDA(cudaMemcpyAsync(host_values, g->wval, sizeof(uint32_t) * g->m, cudaMemcpyDeviceToHost, g->stream));
  SG_CUDA(cudaStreamSynchronize(g->stream));
  if (symmetric) *symmetric = g->wsym ? 1 : 0;
  return SG_OK;
}

}  // extern "C"
