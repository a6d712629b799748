// Exact triangle counting, TC::run + getNumTriangles (algorithms/tc.hpp:67-138).
//
// The reference runs, for every edge (u,v) with u < v, a serial merge of the
// full adjacency lists and adds its running count inside the merge loop
// (tc.hpp:104), which over-counts.  Here:
//   1. orient every edge from the endpoint with the smaller (degree, id) key
//      (the degree-ordered DAG, out-degree at most sqrt(m)): one keep bit per
//      edge, a scan of the per-word counts, and a stable compaction;
//   2. every DAG edge a -> b needs |N+(a) n N+(b)|.  It is counted at the
//      endpoint x with the longer row: x's row N+(x) goes into a
//      shared-memory hash set (four-slot buckets, at most half a key per
//      bucket, one in a warp's table for 129..256 keys) and the shorter
//      row is streamed against it by whole warps
//      (coalesced, eight loads in flight per lane).  So x streams its
//      out-neighbours' rows no longer than its own, and the rows of the
//      in-neighbours y with d+(y) < d+(x) (the reverse lists, built by a
//      count, a scan and a fill);
//   3. each triangle is found exactly once, through the edge between its two
//      lowest DAG vertices; the total is a uint64 sum.
// On RMAT-20 this streams sum over DAG edges of min(d+(a), d+(b)) = 1.97 G
// elements instead of sum of d+(b) = 4.42 G.  The per-vertex convention of
// the reference (for every edge (u,v), u < v, |N(u) n N(v)| is added to u)
// is recovered from the same enumeration: a triangle a < b < c adds 2 to a
// and 1 to b.
//
// Work lists by an upper bound of each vertex's probes: the big ones (or
// d+(x) > 256) are counted by a whole 256-thread block (one 2048-bucket
// table; the flattened rows in 8 equal shares, one per warp), the rest by
// single warps (256-bucket tables, up to one key per bucket), medium before
// small so that the long counts start first; five blocks share an SM.  A vertex with d+(x) > 1024
// is counted in pieces of 1024 keys, each piece against all of x's rows.  The count is that of a graph without parallel
// edges (the reference's sorted-list merge assumes none either); self-loops
// are no DAG edges.
#include "internal.cuh"

namespace sgb {
namespace {

using sygraph::detail::block_sum;

constexpr uint32_t kTcThreads = 256, kTcWarps = kTcThreads / 32;
constexpr uint32_t kTcBlocksPerSm = 5;  // 5 x 41 KB of shared memory, 48 registers
constexpr uint32_t kWarpBuckets = 256;                       // one warp's table: 256 x 4 slots, 4 KB
constexpr uint32_t kBlockBuckets = kWarpBuckets * kTcWarps;  // the block's table: 2048 buckets, 32 KB
constexpr uint32_t kWarpMaxDeg = kWarpBuckets;               // d+(u) counted by one warp (<= 1 key per bucket)
constexpr uint64_t kWarpMaxWork = 1ull << 17;                // probe bound counted by one warp
constexpr uint64_t kSmallMaxWork = 1ull << 11;               // medium above, small below
constexpr uint32_t kBlockMaxDeg = kBlockBuckets / 2;  // keys of one block table
constexpr uint32_t kBlockRows = 4 * kTcThreads;       // rows per balanced block pass
constexpr uint32_t kEmptySlot = 0xffffffffu;          // never a vertex id (n < 2^32)
constexpr uint32_t kRowUnroll = 8;                    // row loads in flight per lane

struct TcCounters {
  uint32_t n_list[3];  // heavy, medium, small
  uint32_t next[3];    // next unclaimed entry of each list
  unsigned long long total;
};

__device__ __forceinline__ bool dag_before(uint32_t du, uint32_t u, uint32_t dv, uint32_t v) {
  return du < dv || (du == dv && u < v);
}

// Keep bit of every edge, one thread per 32-edge word: the thread finds the
// source of its first edge by binary search on the row offsets (kept in
// wsrc for the compaction), loads the word's 32 columns and their 32 degrees
// with every load in flight, then walks the rows.
__global__ void __launch_bounds__(256) dag_flags_kernel(const uint32_t* __restrict__ ro,
                                                        const uint32_t* __restrict__ col, uint32_t n, uint32_t m,
                                                        uint32_t nw, uint32_t* __restrict__ keep,
                                                        uint32_t* __restrict__ cnt, uint32_t* __restrict__ wsrc) {
  const uint32_t tid = blockIdx.x * blockDim.x + threadIdx.x;
  if (tid == 0) cnt[nw] = 0;  // the scan's last input: its output is the DAG size
  for (uint32_t w = tid; w < nw; w += gridDim.x * blockDim.x) {
    const uint32_t e0 = w * 32u, ne = (uint32_t)min((uint64_t)m - e0, (uint64_t)32u);
    uint32_t v[32], dv[32];
    if (ne == 32u) {  // col + e0 is 128-byte aligned
      const uint4* c4 = reinterpret_cast<const uint4*>(col + e0);
#pragma unroll
      for (uint32_t k = 0; k < 8; k++) {
        const uint4 t = c4[k];
        v[4 * k] = t.x;
        v[4 * k + 1] = t.y;
        v[4 * k + 2] = t.z;
        v[4 * k + 3] = t.w;
      }
    } else {
#pragma unroll
      for (uint32_t i = 0; i < 32; i++) v[i] = i < ne ? col[e0 + i] : 0u;
    }
    uint32_t lo = 0, hi = n - 1;  // last u with ro[u] <= e0: the source of edge e0
    while (lo < hi) {
      const uint32_t mid = lo + ((hi - lo + 1) >> 1);
      if (ro[mid] <= e0)
        lo = mid;
      else
        hi = mid - 1;
    }
#pragma unroll
    for (uint32_t i = 0; i < 32; i++) dv[i] = i < ne ? ro[v[i] + 1] - ro[v[i]] : 0u;
    wsrc[w] = lo;
    uint32_t u = lo, rb = ro[u], re = ro[u + 1], bits = 0;
#pragma unroll
    for (uint32_t i = 0; i < 32; i++) {
      if (i < ne) {
        while (re <= e0 + i) {  // rows without edges are skipped
          u++;
          rb = re;
          re = ro[u + 1];
        }
        if (dag_before(re - rb, u, dv[i], v[i])) bits |= 1u << i;
      }
    }
    keep[w] = bits;
    cnt[w] = __popc(bits);
  }
}

// Number of DAG edges among the first e edges of the input CSR.
__device__ __forceinline__ uint32_t dag_prefix(const uint32_t* keep, const uint32_t* wpre, uint32_t e) {
  const uint32_t r = e & 31u;
  return wpre[e >> 5] + (r ? __popc(keep[e >> 5] & ((1u << r) - 1u)) : 0u);
}

// Stable compaction of the kept edges into the DAG's columns (and each
// edge's source) and the DAG's row offsets; zeroes the reverse counts.
__global__ void __launch_bounds__(256) dag_fill_kernel(const uint32_t* __restrict__ ro, const uint32_t* __restrict__ col,
                                                       uint32_t n, uint32_t nw, const uint32_t* __restrict__ keep,
                                                       const uint32_t* __restrict__ wpre,
                                                       const uint32_t* __restrict__ wsrc, uint32_t* __restrict__ dro,
                                                       uint32_t* __restrict__ dcol, uint32_t* __restrict__ dsrc,
                                                       uint32_t* __restrict__ rcnt) {
  const uint32_t tid = blockIdx.x * blockDim.x + threadIdx.x, nthreads = gridDim.x * blockDim.x;
  for (uint32_t w = tid; w < nw; w += nthreads) {
    uint32_t bits = keep[w], p = wpre[w];
    if (!bits) continue;
    const uint32_t e0 = w * 32u;
    uint32_t u = wsrc[w], re = ro[u + 1];
    while (bits) {
      const uint32_t j = __ffs(bits) - 1u;
      bits &= bits - 1u;
      while (re <= e0 + j) re = ro[++u + 1];  // rows without edges are skipped
      dcol[p] = col[e0 + j];
      dsrc[p++] = u;
    }
  }
  for (uint32_t u = tid; u <= n; u += nthreads) {
    dro[u] = dag_prefix(keep, wpre, ro[u]);
    rcnt[u] = 0;
  }
}

// The reverse lists: for every DAG edge y -> x with d+(y) < d+(x), y joins
// x's list (the edge's shorter row N+(y) is then streamed against x's set).
// One thread per DAG edge; kFill = false counts, kFill = true places (rcnt
// counted down to zero).
template <bool kFill>
__global__ void __launch_bounds__(256) rev_kernel(const uint32_t* __restrict__ dro, const uint32_t* __restrict__ dcol,
                                                  const uint32_t* __restrict__ dsrc, const uint32_t* dm_ptr,
                                                  uint32_t* __restrict__ rcnt, const uint32_t* __restrict__ rro,
                                                  uint32_t* __restrict__ rcol) {
  const uint32_t dm = *dm_ptr;  // DAG edges
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < dm; i += gridDim.x * blockDim.x) {
    const uint32_t y = dsrc[i], x = dcol[i];
    if (dro[y + 1] - dro[y] < dro[x + 1] - dro[x]) {
      if (kFill)
        rcol[rro[x] + atomicSub(rcnt + x, 1u) - 1u] = y;
      else
        atomicAdd(rcnt + x, 1u);
    }
  }
}

// Work lists by an upper bound of the probes, (d+(x) + reverse count) *
// d+(x): heavy (block) when d+(x) > kWarpMaxDeg or the bound exceeds
// kWarpMaxWork, medium above kSmallMaxWork, small otherwise; d+(x) < 2 has
// no triangle to count.  Warp-aggregated appends.
__global__ void __launch_bounds__(256) classify_kernel(const uint32_t* __restrict__ dro, const uint32_t* __restrict__ rro,
                                                       uint32_t n, uint32_t* __restrict__ lists,
                                                       TcCounters* __restrict__ C) {
  const uint32_t tid = blockIdx.x * blockDim.x + threadIdx.x, lane = threadIdx.x & 31u;
  for (uint32_t base = tid - lane; base < n; base += gridDim.x * blockDim.x) {  // whole warps, for the ballots
    const uint32_t x = base + lane;
    int kind = -1;
    if (x < n) {
      const uint64_t d = dro[x + 1] - dro[x], r = rro[x + 1] - rro[x], bound = (d + r) * d;
      if (d >= 2) kind = (d > kWarpMaxDeg || bound > kWarpMaxWork) ? 0 : bound > kSmallMaxWork ? 1 : 2;
    }
#pragma unroll
    for (int k = 0; k < 3; k++) {
      const uint32_t mask = __ballot_sync(0xffffffffu, kind == k);
      if (!mask) continue;
      const uint32_t leader = __ffs(mask) - 1u;
      uint32_t at = 0;
      if (lane == leader) at = atomicAdd(&C->n_list[k], (uint32_t)__popc(mask));
      at = __shfl_sync(0xffffffffu, at, leader);
      if (kind == k) lists[(uint64_t)k * n + at + __popc(mask & ((1u << lane) - 1u))] = x;
    }
  }
}

// Exclusive scan in three passes: per-tile sums, a scan of those, then the
// per-tile scan with its offset.  kScanItems values per thread.
constexpr uint32_t kScanThreads = 256, kScanItems = 8, kScanTile = kScanThreads * kScanItems;

__global__ void __launch_bounds__(kScanThreads) scan_tile_sums(const uint32_t* in, uint32_t n, uint32_t* tile_sums) {
  __shared__ unsigned long long s_red[32];
  const uint32_t base = blockIdx.x * kScanTile;
  unsigned long long s = 0;
  for (uint32_t i = threadIdx.x; i < kScanTile; i += kScanThreads)
    if (base + i < n) s += in[base + i];
  s = block_sum(s, s_red);
  if (threadIdx.x == 0) tile_sums[blockIdx.x] = (uint32_t)s;
}

__global__ void __launch_bounds__(1024) scan_tile_offsets(uint32_t* tile_sums, uint32_t tiles) {
  __shared__ uint32_t s_scan[32];
  __shared__ uint32_t s_carry;
  if (threadIdx.x == 0) s_carry = 0;
  __syncthreads();
  for (uint32_t base = 0; base < tiles; base += blockDim.x) {
    const uint32_t i = base + threadIdx.x;
    const uint32_t v = i < tiles ? tile_sums[i] : 0u;
    uint32_t total;
    const uint32_t ex = sygraph::detail::block_excl_scan(v, &total, s_scan);
    if (i < tiles) tile_sums[i] = s_carry + ex;
    __syncthreads();
    if (threadIdx.x == 0) s_carry += total;
    __syncthreads();
  }
}

__global__ void __launch_bounds__(kScanThreads) scan_tiles(const uint32_t* in, uint32_t n, const uint32_t* tile_off,
                                                           uint32_t* out) {
  __shared__ uint32_t s_scan[32];
  const uint32_t base = blockIdx.x * kScanTile + threadIdx.x * kScanItems;
  uint32_t v[kScanItems], s = 0;
#pragma unroll
  for (uint32_t k = 0; k < kScanItems; k++) {
    v[k] = base + k < n ? in[base + k] : 0u;
    s += v[k];
  }
  uint32_t total;
  uint32_t run = tile_off[blockIdx.x] + sygraph::detail::block_excl_scan(s, &total, s_scan);
#pragma unroll
  for (uint32_t k = 0; k < kScanItems; k++) {
    if (base + k < n) out[base + k] = run;
    run += v[k];
  }
}

// Hash set in shared memory: buckets of four slots, read with one 16-byte
// load.  A key goes to the first empty slot at or after the first slot of
// its bucket (linear probing over slots), so every bucket fills as a prefix:
// a bucket whose last slot is empty ends a lookup.  At most half a key per
// bucket (one in a warp's table holding 129 to 256 keys), so a few lookups
// in a thousand read a second bucket.
__device__ __forceinline__ uint32_t bucket_of(uint32_t key, uint32_t shift) { return (key * 0x9E3779B1u) >> shift; }

__device__ __forceinline__ void set_insert(uint4* tab, uint32_t key, uint32_t shift, uint32_t bmask) {
  uint32_t h = bucket_of(key, shift);
  for (;;) {  // ends: at most one key per bucket, a quarter of the slots
    uint32_t* slot = reinterpret_cast<uint32_t*>(tab + h);
#pragma unroll
    for (uint32_t i = 0; i < 4; i++) {
      const uint32_t prev = atomicCAS(slot + i, kEmptySlot, key);
      if (prev == kEmptySlot || prev == key) return;
    }
    h = (h + 1u) & bmask;
  }
}

__device__ __forceinline__ bool set_has(const uint4* tab, uint32_t key, uint32_t shift, uint32_t bmask) {
  uint32_t h = bucket_of(key, shift);
  for (;;) {
    const uint4 x = tab[h];
    if ((x.x == key) | (x.y == key) | (x.z == key) | (x.w == key)) return true;
    if (x.w == kEmptySlot) return false;
    h = (h + 1u) & bmask;
  }
}

// log2 of the bucket count for `keys` keys: at least two buckets per key,
// at least eight buckets, at most 2^max_log2.
__device__ __forceinline__ uint32_t log2_buckets(uint32_t keys, uint32_t max_log2) {
  const uint32_t want = keys <= 4u ? 8u : 2u * keys;
  const uint32_t lg = 32u - __clz(want - 1u);
  return lg < max_log2 ? lg : max_log2;
}

__device__ __forceinline__ void set_clear(uint4* tab, uint32_t buckets, uint32_t first, uint32_t step) {
  for (uint32_t s = first; s < buckets; s += step) tab[s] = make_uint4(kEmptySlot, kEmptySlot, kEmptySlot, kEmptySlot);
}

struct TcParams {
  const uint32_t* dro;
  const uint32_t* dcol;
  const uint32_t* rro;
  const uint32_t* rcol;
  const uint32_t* lists;
  TcCounters* C;
  unsigned long long* per_vertex;
  uint32_t n;
  uint32_t shorter;  // 1: an out-row longer than x's own is left to its head's reverse list
};

template <bool kPerVertex>
__device__ __forceinline__ void add_triangle(unsigned long long* pv, uint32_t a, uint32_t b, uint32_t c) {
  if (kPerVertex) {
    uint32_t t;
    if (a > b) { t = a; a = b; b = t; }
    if (b > c) { t = b; b = c; c = t; }
    if (a > b) { t = a; a = b; b = t; }
    atomicAdd(pv + a, 2ull);
    atomicAdd(pv + b, 1ull);
  }
}

// Lookups of the row segment dcol[sb, se) (warp-uniform bounds), one
// element per lane and chunk of 32, kRowUnroll loads in flight; the last
// chunks are skipped by uniform branches.  A hit w closes the triangle
// {x, y, w}.
template <bool kPerVertex>
__device__ __forceinline__ uint32_t probe_segment(const TcParams& P, const uint4* tab, uint32_t shift, uint32_t bmask,
                                                  uint32_t x, uint32_t y, uint32_t sb, uint32_t se) {
  const uint32_t lane = threadIdx.x & 31u, part = (se - sb) & 31u;  // lanes of the partial last chunk
  uint32_t full = (se - sb) >> 5, e = sb + lane, hits = 0;
  for (; full >= kRowUnroll; full -= kRowUnroll, e += 32u * kRowUnroll) {
    uint32_t w[kRowUnroll];
#pragma unroll
    for (uint32_t q = 0; q < kRowUnroll; q++) w[q] = P.dcol[e + 32u * q];
#pragma unroll
    for (uint32_t q = 0; q < kRowUnroll; q++) {
      if (set_has(tab, w[q], shift, bmask)) {
        hits++;
        add_triangle<kPerVertex>(P.per_vertex, x, y, w[q]);
      }
    }
  }
  // fewer than kRowUnroll full chunks left, then the partial one (q == full)
  uint32_t w[kRowUnroll];
#pragma unroll
  for (uint32_t q = 0; q < kRowUnroll; q++) {
    if (q > full) break;
    w[q] = (q < full || lane < part) ? P.dcol[e + 32u * q] : 0u;
  }
#pragma unroll
  for (uint32_t q = 0; q < kRowUnroll; q++) {
    if (q > full) break;
    if ((q < full || lane < part) && set_has(tab, w[q], shift, bmask)) {
      hits++;
      add_triangle<kPerVertex>(P.per_vertex, x, y, w[q]);
    }
  }
  return hits;
}

// The rows x streams: the out-neighbours y of x with d+(y) <= d+(x) (row
// index j < d), then x's reverse list (j >= d, d+(y) < d+(x) already).
__device__ __forceinline__ uint32_t row_vertex(const TcParams& P, uint32_t b, uint32_t d, uint32_t rb, uint32_t j) {
  return j < d ? P.dcol[b + j] : P.rcol[rb + (j - d)];
}

// One warp streams the rows j = j0, j0 + jstride, ... < rows of x against
// the table, 32 row bounds loaded at a time; returns its lane's hits.
template <bool kPerVertex>
__device__ __forceinline__ uint32_t count_rows(const TcParams& P, const uint4* tab, uint32_t shift, uint32_t bmask,
                                               uint32_t x, uint32_t b, uint32_t d, uint32_t rb, uint32_t rows,
                                               uint32_t j0, uint32_t jstride) {
  const uint32_t lane = threadIdx.x & 31u;
  uint32_t hits = 0;
  for (uint32_t jb = j0; jb < rows; jb += 32u * jstride) {
    const uint32_t j = jb + lane * jstride;
    uint32_t y = 0, vb = 0, ve = 0;
    if (j < rows) {
      y = row_vertex(P, b, d, rb, j);
      vb = P.dro[y];
      ve = P.dro[y + 1];
      if (P.shorter && j < d && ve - vb > d) ve = vb;  // the edge's shorter row is x's own
    }
    for (uint32_t live = __ballot_sync(0xffffffffu, ve > vb); live; live &= live - 1u) {
      const uint32_t k = __ffs(live) - 1u;
      const uint32_t sb = __shfl_sync(0xffffffffu, vb, k), se = __shfl_sync(0xffffffffu, ve, k);
      const uint32_t sy = kPerVertex ? __shfl_sync(0xffffffffu, y, k) : 0u;
      hits += probe_segment<kPerVertex>(P, tab, shift, bmask, x, sy, sb, se);
    }
  }
  return hits;
}

// Shared memory of the counting kernel: the table (the block's for heavy
// vertices, 32 warp slices otherwise), then the row starts and the prefix of
// the row lengths of one balanced pass.
constexpr size_t kTcSmem = sizeof(uint4) * kBlockBuckets + sizeof(uint32_t) * (2 * kBlockRows + 1);

template <bool kPerVertex>
__global__ void __launch_bounds__(kTcThreads, kTcBlocksPerSm) tc_hash_kernel(TcParams P) {
  extern __shared__ uint4 s_tab[];  // kBlockBuckets, then s_vb and s_pre
  uint32_t* s_vb = reinterpret_cast<uint32_t*>(s_tab + kBlockBuckets);
  uint32_t* s_pre = s_vb + kBlockRows;
  __shared__ uint32_t s_next, s_scan[32];
  __shared__ unsigned long long s_red[32];
  const uint32_t lane = threadIdx.x & 31u, warp = threadIdx.x >> 5;
  unsigned long long acc = 0;
  // heavy vertices: one block each, the whole table
  const uint32_t n_heavy = P.C->n_list[0];
  for (;;) {
    if (threadIdx.x == 0) s_next = atomicAdd(&P.C->next[0], 1u);
    __syncthreads();
    const uint32_t i = s_next;
    if (i >= n_heavy) break;
    const uint32_t x = P.lists[i], b = P.dro[x], d = P.dro[x + 1] - b;
    const uint32_t rb = P.rro[x], rows = d + (P.rro[x + 1] - rb);
    // the table holds N+(x), in pieces of kBlockMaxDeg keys when longer
    for (uint32_t off = 0; off < d; off += kBlockMaxDeg) {
      const uint32_t kd = min(kBlockMaxDeg, d - off);
      const uint32_t lg = log2_buckets(kd, 11u), shift = 32u - lg, bmask = (1u << lg) - 1u;
      set_clear(s_tab, 1u << lg, threadIdx.x, kTcThreads);
      __syncthreads();
      for (uint32_t j = threadIdx.x; j < kd; j += kTcThreads) set_insert(s_tab, P.dcol[b + off + j], shift, bmask);
      // passes of kBlockRows rows: their flattened lengths in kTcWarps equal shares
      for (uint32_t c0 = 0; c0 < rows; c0 += kBlockRows) {
        const uint32_t cr = min(kBlockRows, rows - c0);
        uint32_t len[4], sum = 0;
#pragma unroll
        for (uint32_t q = 0; q < 4; q++) {
          const uint32_t jj = 4u * threadIdx.x + q;
          len[q] = 0;
          if (jj < cr) {
            const uint32_t j = c0 + jj, y = row_vertex(P, b, d, rb, j), vb = P.dro[y];
            len[q] = P.dro[y + 1] - vb;
            if (P.shorter && j < d && len[q] > d) len[q] = 0;
            s_vb[jj] = vb;
          }
          sum += len[q];
        }
        uint32_t total;  // block_excl_scan synchronises: the inserts above are complete after it
        uint32_t run = sygraph::detail::block_excl_scan(sum, &total, s_scan);
#pragma unroll
        for (uint32_t q = 0; q < 4; q++) {
          const uint32_t jj = 4u * threadIdx.x + q;
          if (jj < cr) s_pre[jj] = run;
          run += len[q];
        }
        if (threadIdx.x == 0) s_pre[cr] = total;
        __syncthreads();
        const uint32_t lo = (uint32_t)((uint64_t)total * warp / kTcWarps);
        const uint32_t hi = (uint32_t)((uint64_t)total * (warp + 1) / kTcWarps);
        if (lo < hi) {
          uint32_t r = 0, top = cr;  // last row with s_pre[r] <= lo
          while (r < top) {
            const uint32_t mid = (r + top + 1) >> 1;
            if (s_pre[mid] <= lo)
              r = mid;
            else
              top = mid - 1;
          }
          for (uint32_t pos = lo; pos < hi;) {
            while (s_pre[r + 1] <= pos) r++;  // rows left out or without out-edges
            const uint32_t rend = min(hi, s_pre[r + 1]);
            const uint32_t base = s_vb[r] - s_pre[r];  // dcol index of flattened position 0 of row r (mod 2^32)
            const uint32_t ry = kPerVertex ? row_vertex(P, b, d, rb, c0 + r) : 0u;
            acc += probe_segment<kPerVertex>(P, s_tab, shift, bmask, x, ry, base + pos, base + rend);
            pos = rend;
          }
        }
        __syncthreads();  // s_vb and s_pre are reused
      }
    }
  }
  // medium, then small vertices: one warp each, a 256-bucket slice of the table
  uint4* tab = s_tab + warp * kWarpBuckets;
#pragma unroll 1
  for (uint32_t k = 1; k < 3; k++) {
    const uint32_t cnt = P.C->n_list[k], grab = k == 1 ? 1u : 8u;
    const uint32_t* list = P.lists + (uint64_t)k * P.n;
    for (;;) {
      uint32_t i0 = 0;
      if (lane == 0) i0 = atomicAdd(&P.C->next[k], grab);
      i0 = __shfl_sync(0xffffffffu, i0, 0);
      if (i0 >= cnt) break;
      const uint32_t i1 = min(i0 + grab, cnt);
      for (uint32_t i = i0; i < i1; i++) {
        const uint32_t x = list[i], b = P.dro[x], d = P.dro[x + 1] - b;
        const uint32_t rb = P.rro[x], rows = d + (P.rro[x + 1] - rb);
        const uint32_t lg = log2_buckets(d, 8u), shift = 32u - lg, bmask = (1u << lg) - 1u;
        __syncwarp();  // the previous vertex's lookups are done
        set_clear(tab, 1u << lg, lane, 32u);
        __syncwarp();
        for (uint32_t j = lane; j < d; j += 32u) set_insert(tab, P.dcol[b + j], shift, bmask);
        __syncwarp();
        acc += count_rows<kPerVertex>(P, tab, shift, bmask, x, b, d, rb, rows, 0u, 1u);
      }
    }
  }
  acc = block_sum(acc, s_red);
  if (threadIdx.x == 0 && acc) atomicAdd(&P.C->total, acc);
}

template <bool kPerVertex>
sg_status launch_count(const TcParams& P, cudaStream_t s) {
  // once per kernel (thread-safe static initialisation)
  static const cudaError_t configured =
      cudaFuncSetAttribute(tc_hash_kernel<kPerVertex>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kTcSmem);
  SG_CUDA(configured);
  int occ = 0;
  SG_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, tc_hash_kernel<kPerVertex>, (int)kTcThreads, kTcSmem));
  SG_REQUIRE(occ > 0, SG_ERR_CUDA, "triangle-count kernel does not fit on an SM");
  tc_hash_kernel<kPerVertex><<<(unsigned)(occ * device_props().sm_count), kTcThreads, kTcSmem, s>>>(P);
  SG_CUDA(cudaGetLastError());
  count_launch();
  return SG_OK;
}

}  // namespace

// Exclusive scan of n values into out, with tile_sums holding
// div_up(n, 2048) words; enqueued on s only.
sg_status exclusive_scan_u32(const uint32_t* in, uint32_t n, uint32_t* out, uint32_t* tile_sums, cudaStream_t s) {
  const uint32_t tiles = div_up(n ? n : 1, kScanTile);
  scan_tile_sums<<<tiles, kScanThreads, 0, s>>>(in, n, tile_sums);
  scan_tile_offsets<<<1, 1024, 0, s>>>(tile_sums, tiles);
  scan_tiles<<<tiles, kScanThreads, 0, s>>>(in, n, tile_sums, out);
  count_launch(3);
  SG_CUDA(cudaGetLastError());
  return SG_OK;
}

}  // namespace sgb

using namespace sgb;

struct sg_tc_s {
  sg_graph g = nullptr;
  cudaStream_t stream = nullptr;
  uint32_t nw = 0;  // 32-edge words of the input CSR
  uint32_t* keep = nullptr;
  uint32_t* wsrc = nullptr;  // nw: source of each word's first edge
  uint32_t* cnt = nullptr;   // nw + 1
  uint32_t* wpre = nullptr;  // nw + 1
  uint32_t* tiles = nullptr;
  uint32_t* dro = nullptr;   // n + 1
  uint32_t* dcol = nullptr;  // up to m
  uint32_t* dsrc = nullptr;  // up to m
  uint32_t* rcnt = nullptr;  // n + 1
  uint32_t* rro = nullptr;   // n + 1
  uint32_t* rcol = nullptr;  // up to m
  uint32_t* rtiles = nullptr;
  uint32_t* lists = nullptr; // 3 n
  TcCounters* counters = nullptr;
  unsigned long long* pv = nullptr;  // n, allocated on the first per-vertex run
  bool ran = false, ran_per_vertex = false;
  bool shorter = true;  // stream each DAG edge's shorter row
};

extern "C" {

sg_status sg_tc_destroy(sg_tc_handle t) {
  if (t) {
    cudaStreamSynchronize(t->stream);
    dev_free(t->keep);
    dev_free(t->wsrc);
    dev_free(t->cnt);
    dev_free(t->wpre);
    dev_free(t->tiles);
    dev_free(t->dro);
    dev_free(t->dcol);
    dev_free(t->dsrc);
    dev_free(t->rcnt);
    dev_free(t->rro);
    dev_free(t->rcol);
    dev_free(t->rtiles);
    dev_free(t->lists);
    dev_free(t->counters);
    dev_free(t->pv);
    delete t;
  }
  return SG_OK;
}

sg_status sg_tc_create(sg_graph g, sg_tc_handle* out) {
  clear_error();
  SG_REQUIRE(g && out, SG_ERR_INVALID, "NULL argument");
  SG_REQUIRE(g->n > 0, SG_ERR_INVALID, "graph has no vertices");
  *out = nullptr;
  sg_tc_handle t = new sg_tc_s();
  t->g = g;
  t->stream = g->stream;
  const uint64_t n = g->n, m = g->m;
  t->nw = (uint32_t)div_up(m, 32);
  sg_status st;
  if ((st = dev_alloc(&t->keep, t->nw)) || (st = dev_alloc(&t->wsrc, t->nw)) || (st = dev_alloc(&t->cnt, (uint64_t)t->nw + 1)) ||
      (st = dev_alloc(&t->wpre, (uint64_t)t->nw + 1)) ||
      (st = dev_alloc(&t->tiles, div_up((uint64_t)t->nw + 1, kScanTile))) || (st = dev_alloc(&t->dro, n + 1)) ||
      (st = dev_alloc(&t->dcol, m)) || (st = dev_alloc(&t->dsrc, m)) || (st = dev_alloc(&t->rcnt, n + 1)) || (st = dev_alloc(&t->rro, n + 1)) ||
      (st = dev_alloc(&t->rcol, m)) || (st = dev_alloc(&t->rtiles, div_up(n + 1, kScanTile))) ||
      (st = dev_alloc(&t->lists, 3 * n)) || (st = dev_alloc(&t->counters, 1))) {
    sg_tc_destroy(t);
    return st;
  }
  *out = t;
  return SG_OK;
}

sg_status sg_tc_run_async(sg_tc_handle t, int per_vertex) {
  clear_error();
  SG_REQUIRE(t, SG_ERR_INVALID, "tc is NULL");
  const sg_graph g = t->g;
  const uint32_t n = g->n, m = (uint32_t)g->m;
  cudaStream_t s = t->stream;
  if (per_vertex && !t->pv) SG_TRY(dev_alloc(&t->pv, n));
  SG_CUDA(cudaMemsetAsync(t->counters, 0, sizeof(TcCounters), s));
  dag_flags_kernel<<<grid_for(t->nw ? t->nw : 1, 256, 8), 256, 0, s>>>(g->fwd.ro, g->fwd.col, n, m, t->nw, t->keep,
                                                                       t->cnt, t->wsrc);
  SG_CUDA(cudaGetLastError());
  count_launch();
  SG_TRY(exclusive_scan_u32(t->cnt, t->nw + 1, t->wpre, t->tiles, s));
  const unsigned vgrid = grid_for((uint64_t)n + 1, 256, 8), egrid = grid_for(m ? m : 1, 256, 8);
  dag_fill_kernel<<<grid_for(std::max<uint64_t>(t->nw, (uint64_t)n + 1), 256, 8), 256, 0, s>>>(
      g->fwd.ro, g->fwd.col, n, t->nw, t->keep, t->wpre, t->wsrc, t->dro, t->dcol, t->dsrc, t->rcnt);
  SG_CUDA(cudaGetLastError());
  count_launch();
  if (t->shorter) {  // the DAG size is read on the device: dro[n]
    rev_kernel<false><<<egrid, 256, 0, s>>>(t->dro, t->dcol, t->dsrc, t->dro + n, t->rcnt, nullptr, nullptr);
    SG_CUDA(cudaGetLastError());
    count_launch();
  }
  SG_TRY(exclusive_scan_u32(t->rcnt, n + 1, t->rro, t->rtiles, s));
  if (t->shorter) {
    rev_kernel<true><<<egrid, 256, 0, s>>>(t->dro, t->dcol, t->dsrc, t->dro + n, t->rcnt, t->rro, t->rcol);
    SG_CUDA(cudaGetLastError());
    count_launch();
  }
  classify_kernel<<<vgrid, 256, 0, s>>>(t->dro, t->rro, n, t->lists, t->counters);
  SG_CUDA(cudaGetLastError());
  count_launch();
  TcParams P{t->dro, t->dcol, t->rro, t->rcol, t->lists, t->counters, t->pv, n, t->shorter ? 1u : 0u};
  if (per_vertex) {
    SG_CUDA(cudaMemsetAsync(t->pv, 0, sizeof(unsigned long long) * n, s));
    SG_TRY(launch_count<true>(P, s));
  } else {
    SG_TRY(launch_count<false>(P, s));
  }
  t->ran = true;
  t->ran_per_vertex = per_vertex != 0;
  return SG_OK;
}

sg_status sg_tc_set_shorter_rows(sg_tc_handle t, int shorter) {
  clear_error();
  SG_REQUIRE(t, SG_ERR_INVALID, "tc is NULL");
  t->shorter = shorter != 0;
  return SG_OK;
}

sg_status sg_tc_get_total(sg_tc_handle t, uint64_t* total) {
  clear_error();
  SG_REQUIRE(t && total, SG_ERR_INVALID, "NULL argument");
  SG_REQUIRE(t->ran, SG_ERR_NOT_INITIALIZED, "triangle count not run");
  unsigned long long v = 0;
  SG_CUDA(cudaMemcpyAsync(&v, &t->counters->total, sizeof(v), cudaMemcpyDeviceToHost, t->stream));
  SG_CUDA(cudaStreamSynchronize(t->stream));
  *total = v;
  return SG_OK;
}

sg_status sg_tc_run(sg_tc_handle t, int per_vertex, uint64_t* total) {
  SG_TRY(sg_tc_run_async(t, per_vertex));
  if (total) return sg_tc_get_total(t, total);
  SG_CUDA(cudaStreamSynchronize(t->stream));
  return SG_OK;
}

sg_status sg_tc_get_per_vertex(sg_tc_handle t, uint64_t* host_per_vertex) {
  clear_error();
  SG_REQUIRE(t && host_per_vertex, SG_ERR_INVALID, "NULL argument");
  SG_REQUIRE(t->ran_per_vertex, SG_ERR_NOT_INITIALIZED, "no per-vertex triangle count run");
  SG_CUDA(cudaMemcpyAsync(host_per_vertex, t->pv, sizeof(uint64_t) * t->g->n, cudaMemcpyDeviceToHost, t->stream));
  SG_CUDA(cudaStreamSynchronize(t->stream));
  return SG_OK;
}

sg_status sg_tc(sg_graph g, uint64_t* total, uint64_t* host_per_vertex) {
  clear_error();
  SG_REQUIRE(g && total, SG_ERR_INVALID, "NULL argument");
  sg_tc_handle t = nullptr;
  SG_TRY(sg_tc_create(g, &t));
  sg_status st = sg_tc_run(t, host_per_vertex != nullptr, total);
  if (st == SG_OK && host_per_vertex) st = sg_tc_get_per_vertex(t, host_per_vertex);
  sg_tc_destroy(t);
  return st;
}

}  // extern "C"
