// Fused SSSP (algorithms/sssp.hpp:152-210) and CC (algorithms/cc.hpp:103-169)
// engines on the shared push level loop.
//
// SSSP: frontier Bellman-Ford.  A frontier vertex v relaxes each out-edge
//   with nd = d[v] + w and atomicMin on d[u] (non-negative floats compare as
//   their bit patterns); u joins the next frontier when its distance dropped
//   (sssp.hpp:180-189).  The reference's filter::external after each advance
//   (sssp.hpp:192-196) only de-duplicates, which the bitmap does.  Every
//   relaxation order reaches the same least fixed point, so distances match
//   Dijkstra bit for bit.
// CC: labels[v] = v, then every vertex pushes its label along its out-edges
//   with atomicMax; a vertex whose label grew joins the next frontier
//   (cc.hpp:135-168).  The fixed point is the maximum id over the vertices
//   that reach v.
#include <vector>

#include "push_engine.cuh"
#include "selector_features.cuh"
#include "sssp_pull.cuh"
#include "sygraph/detail/selector_mlp.cuh"

namespace sgb {
namespace {

using namespace eng;

// Near-far bookkeeping of one refill pass (three rotating slots).
struct Refill {
  unsigned long long moved, remaining;
  uint32_t far_min;  // bit pattern of the smallest distance left in the far set
  uint32_t pad;
};

template <typename W>
struct SsspParams {
  PushLoop L;
  uint32_t source;
  W* dist;
  const W* w;
  unsigned long long* result;
  uint32_t* far;     // w0 words: improved vertices at or beyond the threshold
  uint32_t* bucket;  // w0 words: vertices expanded in the current bucket (their heavy edges wait)
  Refill* refill;
  W delta;        // 0: plain frontier Bellman-Ford (every improved vertex is near)
  PullArgs<W> pull;
  uint32_t pull_ratio;  // pull when the frontier's out-degree * pull_ratio > m (0: push only)
  unsigned long long m;
  const uint32_t* split;  // delta-stepping: first edge of weight >= delta in each weight-sorted row
  const uint32_t* wcol;   // weight-sorted rows (same row offsets)
  const W* wval;
  uint32_t tail;  // far set below this many vertices: the rest runs as plain Bellman-Ford
  // heavy phase by pull when its push would relax more than m / heavy_pull
  // edges (0: always push); only where a row's out-edges are its in-edges
  uint32_t heavy_pull;
  // light iteration by pull when its frontier holds more than n / light_pull
  // vertices (0: always push); same condition on the graph
  uint32_t light_pull;
  // learned heavy phase: the selector's staged image (nullptr: the ratio
  // rule above decides), asked at every heavy phase when pull is possible
  const sygraph::detail::MlpStaged* mlp_image;
  float margin;      // log-time gain the MLP must predict to overrule the rule
  float heavy_lo, heavy_hi;  // heavy edges of the buckets (fraction of m) on which the MLP is asked
  bool pull_ok;      // the weighted rows are symmetric: a heavy phase may pull
  float* features;   // optional log: 12 floats per heavy phase
};

// Shared state of the learned heavy-phase choice.
struct HeavySelect {
  sygraph::detail::MlpStaged mlp;
  float scratch[sygraph::detail::kMlpHidden];
  FeatureConst fk;
  int choice;
};

// Direction of a bucket's heavy phase (true = pull), identical in every CTA:
// the MLP's choice between push and pull (warp 0 of each CTA; outputs 0 and
// 2) on the bucket's features, where the model is attached, pull is possible
// and the bucket's heavy edges are within [heavy_lo, heavy_hi] * m (near the
// rule's own threshold, where the rule was wrong in training; elsewhere an
// inference costs more than it saves), the ratio rule's `h_pull` unless the
// model predicts it `margin` slower in log-time or outside the trusted
// feature range; logs the features when asked.  Features: the bucket's vertices and heavy edges, the heavy
// edges not yet relaxed, the vertices settled, the previous bucket's size
// and the previous heavy phase's direction.
template <typename W>
__device__ __forceinline__ bool heavy_decide(const SsspParams<W>& P, HeavySelect& S, bool h_pull,
                                             const FeatureInputs& x, uint32_t phase) {
  const bool log = P.features && blockIdx.x == 0 && phase < kMaxLog;
  const bool infer = P.mlp_image && P.pull_ok && (float)x.nd >= P.heavy_lo * (float)P.m &&
                     (float)x.nd <= P.heavy_hi * (float)P.m;
  if (!infer && !log) return h_pull;
  if (threadIdx.x < 32) {
    const float f = feature_of_lane(threadIdx.x, P.L.n, S.fk, x);
    if (log && threadIdx.x < 12) P.features[(size_t)phase * 12 + threadIdx.x] = f;
    if (infer) {
      const int c = sygraph::detail::mlp_choose(&S.mlp, f, (1u << 0) | (1u << 2), S.scratch, h_pull ? 2 : 0,
                                                P.margin);
      if (threadIdx.x == 0) S.choice = c;
    }
  }
  __syncthreads();
  const bool out = (infer && S.choice >= 0) ? S.choice == 2 : h_pull;
  __syncthreads();  // S.choice is written again at the next heavy phase
  return out;
}

// Edge relaxation of the SSSP push steps, kU edges per lane at a time: the
// column and weight loads of all kU edges go out together, then their
// distance probes, then the atomicMins that improve, then the bitmap marks,
// so a warp waits about four memory latencies per 32 * kU edges instead of
// four per 32.  nd = d[v] + w with atomicMin on d[u] (non-negative floats
// order as their bit patterns); an improved u joins the next frontier, or,
// under near-far bucketing with nd at or beyond the threshold, the far set.
constexpr int kU = 4;
// Edges per chunk of a big vertex in SSSP push steps: half the push
// engines' (more warps share a hub's edges; a step with few frontier
// vertices is a few dependent round trips per chunk): on RMAT-22 the
// reference schedule 5.40 -> 5.04 ms per source, delta-stepping 1.99 ->
// 1.95 ms; 64-edge chunks lose on the reference schedule (6.0 ms).
constexpr uint32_t kSsspChunk = 128;

template <typename W>
struct SsspRelax {
  W* dist;
  const W* w;
  const uint32_t* col;
  uint32_t* far;
  uint32_t* fb_next;
  const uint32_t* ro;
  W threshold;
  bool bucketed;
  bool want_deg;  // sum the out-degree of new frontier vertices (only a pull decision reads it)
  // count each newly set frontier bit once; otherwise the marks do not wait
  // for the old bitmap word and n_new counts marks (zero exactly when no bit
  // was set, which is all that termination reads)
  bool exact = true;
  uint32_t n_new = 0;
  unsigned long long deg_new = 0;

  __device__ __forceinline__ void relax(const uint32_t (&e)[kU], const W (&dv)[kU], uint32_t act) {
    uint32_t u[kU];
    W nd[kU], cur[kU], old[kU];
#pragma unroll
    for (int k = 0; k < kU; k++) {
      u[k] = 0;
      nd[k] = W(0);
      if ((act >> k) & 1u) {
        u[k] = col[e[k]];
        nd[k] = dv[k] + w[e[k]];
      }
    }
#pragma unroll
    for (int k = 0; k < kU; k++) cur[k] = ((act >> k) & 1u) ? ld_cg(dist + u[k]) : W(0);
    uint32_t imp = 0;
#pragma unroll
    for (int k = 0; k < kU; k++)
      if (((act >> k) & 1u) && nd[k] < cur[k]) imp |= 1u << k;
    if (!imp) return;
#pragma unroll
    for (int k = 0; k < kU; k++) old[k] = ((imp >> k) & 1u) ? sygraph::detail::atomic_min_nonneg(dist + u[k], nd[k]) : W(0);
    if (!exact) {
#pragma unroll
      for (int k = 0; k < kU; k++)
        if (((imp >> k) & 1u) && nd[k] < old[k]) {
          const uint32_t b = 1u << (u[k] & 31);
          if (bucketed && !(nd[k] < threshold)) {
            atomicOr(far + (u[k] >> 5), b);
          } else {
            atomicOr(fb_next + (u[k] >> 5), b);
            n_new++;
          }
        }
      return;
    }
    uint32_t prev[kU];
    uint32_t marked = 0;
#pragma unroll
    for (int k = 0; k < kU; k++) {
      prev[k] = 0;
      if (((imp >> k) & 1u) && nd[k] < old[k]) {
        const uint32_t b = 1u << (u[k] & 31);
        if (bucketed && !(nd[k] < threshold)) {
          atomicOr(far + (u[k] >> 5), b);
        } else {
          prev[k] = atomicOr(fb_next + (u[k] >> 5), b);
          marked |= 1u << k;
        }
      }
    }
#pragma unroll
    for (int k = 0; k < kU; k++)
      if (((marked >> k) & 1u) && !(prev[k] & (1u << (u[k] & 31)))) {
        n_new++;
        if (want_deg) deg_new += ro[u[k] + 1] - ro[u[k]];
      }
  }
};

// Push expansion of one SSSP step over the compacted queues.  Small vertices
// (row range < kSmallDeg) go 32 per warp, their edges ranked across the warp;
// big vertices are cut in kSsspChunk-edge chunks, and each warp takes a
// contiguous run of chunks: one owner search, then the owners advance.
template <typename W>
__device__ __forceinline__ void sssp_expand(RowRange R, Queues q, uint32_t n_small, uint32_t n_big, uint32_t n_chunks,
                                            SsspRelax<W>& X) {
  const uint32_t lane = threadIdx.x & 31;
  const uint32_t gwarp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const uint32_t nwarps = (gridDim.x * blockDim.x) >> 5;
  const uint32_t n_groups = (n_small + 31) / 32;
  for (uint32_t unit = gwarp; unit < n_groups; unit += nwarps) {
    const uint32_t idx = unit * 32 + lane;
    const bool valid = idx < n_small;
    const uint32_t v = valid ? ld_cg(q.small + idx) : 0u;
    const uint32_t beg = valid ? R.beg(v) : 0u;
    const uint32_t deg = valid ? R.end(v) - beg : 0u;
    const W dv = valid ? ld_cg(X.dist + v) : W(0);
    const uint32_t incl = warp_inclusive_scan(deg);
    const uint32_t total = __shfl_sync(kFullMask, incl, 31);
    const uint32_t excl = incl - deg;
    for (uint32_t r0 = 0; r0 < total; r0 += 32 * kU) {
      uint32_t e[kU];
      W d[kU];
      uint32_t act = 0;
#pragma unroll
      for (int k = 0; k < kU; k++) {
        const uint32_t r = r0 + k * 32 + lane;
        const bool a = r < total;
        const uint32_t o = warp_owner_of_rank(incl, a ? r : total - 1);
        const uint32_t ob = __shfl_sync(kFullMask, beg, o);
        const uint32_t oe = __shfl_sync(kFullMask, excl, o);
        d[k] = __shfl_sync(kFullMask, dv, o);
        e[k] = ob + (r - oe);
        act |= (uint32_t)a << k;
      }
      X.relax(e, d, act);
    }
  }
  if (!n_chunks) return;
  // the chunk runs start at the first warp without a small group, so that
  // on a small frontier no warp walks a group and then a chunk (two chains
  // of dependent loads one after the other)
  const uint32_t bw = (gwarp + nwarps - (n_groups % nwarps)) % nwarps;
  const uint32_t per = (n_chunks + nwarps - 1) / nwarps;
  const uint32_t c_lo = bw * per;
  const uint32_t c_hi = min(n_chunks, c_lo + per);
  if (c_lo >= c_hi) return;
  uint32_t ent = warp_find_owner(q.big_start, n_big, c_lo);
  uint32_t v = ld_cg(q.big + ent);
  uint32_t first = ld_cg(q.big_start + ent);
  uint32_t next = ent + 1 < n_big ? ld_cg(q.big_start + ent + 1) : n_chunks;
  uint32_t vb = R.beg(v), ve = R.end(v);
  W dv = ld_cg(X.dist + v);
  for (uint32_t c = c_lo; c < c_hi; c++) {
    while (c >= next) {  // the run crossed into the next big vertex
      ent++;
      v = ld_cg(q.big + ent);
      first = next;
      next = ent + 1 < n_big ? ld_cg(q.big_start + ent + 1) : n_chunks;
      vb = R.beg(v);
      ve = R.end(v);
      dv = ld_cg(X.dist + v);
    }
    const uint32_t cb = vb + (c - first) * kSsspChunk;
    const uint32_t ce = min(ve, cb + kSsspChunk);
    for (uint32_t eb = cb; eb < ce; eb += 32 * kU) {
      uint32_t e[kU];
      W d[kU];
      uint32_t act = 0;
#pragma unroll
      for (int k = 0; k < kU; k++) {
        e[k] = eb + k * 32 + lane;
        d[k] = dv;
        act |= (uint32_t)(e[k] < ce) << k;
      }
      X.relax(e, d, act);
    }
  }
}

// Pull steps of near-far bucketing, for graphs whose rows list in-edges as
// well as out-edges (undirected, symmetric weights), over the bucket [lo,
// threshold).  Every candidate vertex u takes the minimum of d[c] + w over
// its neighbours c in a member bitmap, scanning its weight-sorted row from
// the lightest edge; since d[c] >= lo for every member, the scan stops at the
// first weight with lo + w >= best (rounding is monotone: no later edge
// gives less).  u alone writes d[u]: no atomics on distances.
//   heavy phase (kLight false): members = the bucket, candidates = vertices
//     beyond the threshold, the whole row.  Only an edge of weight >= delta
//     can improve u (the bucket's light edges were relaxed while it ran);
//     improved vertices join the far set.
//   light iteration (kLight true): members = the frontier, candidates =
//     vertices above lo, the light prefix of the row (weights < delta);
//     improved vertices join the next frontier below the threshold, the far
//     set otherwise, and the frontier joins the bucket.  The frontier's own
//     distances may drop during the sweep: any value read is an upper bound,
//     and a vertex that dropped is in the next frontier, so its neighbours
//     see the final value then.
// Lanes scan their own rows kP edges per step; rows of kPullLong edges or
// more are walked by the whole warp, 32 edges per step.
constexpr uint32_t kP = 4;
constexpr uint32_t kPullLong = 256;

template <typename W, bool kLight>
__device__ __forceinline__ uint32_t sssp_pull_scan(const SsspParams<W>& P, const uint32_t* member, uint32_t* fb_next,
                                                   W lo, W threshold) {
  const uint32_t lane = threadIdx.x & 31;
  const uint32_t gwarp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const uint32_t nwarps = (gridDim.x * blockDim.x) >> 5;
  const uint32_t n = P.L.n, w0 = P.L.w0;
  const uint32_t* ro = P.L.ro;
  uint32_t n_new = 0;
  for (uint32_t wi = gwarp; wi < w0; wi += nwarps) {
    if (kLight && lane == 0) {  // the frontier joins the bucket (its heavy edges wait)
      const uint32_t fw = ld_cg(member + wi);
      if (fw) st_cg(P.bucket + wi, ld_cg(P.bucket + wi) | fw);
    }
    const uint32_t u = wi * 32 + lane;
    const W d0 = u < n ? ld_cg(P.dist + u) : W(0);
    const bool cand = u < n && (kLight ? lo < d0 : threshold < d0);
    if (!__any_sync(kFullMask, cand)) continue;
    const uint32_t beg = cand ? ro[u] : 0u;
    const uint32_t end = cand ? (kLight ? P.split[u] : ro[u + 1]) : 0u;
    const bool is_long = end - beg >= kPullLong;
    W best = d0;
    uint32_t e = beg;
    bool open = cand && !is_long && beg < end;
    while (__any_sync(kFullMask, open)) {
      if (open) {
        W wv[kP], dc[kP];
        uint32_t cv[kP];
        bool inb[kP];
#pragma unroll
        for (uint32_t k = 0; k < kP; k++) {
          const bool ok = e + k < end;
          wv[k] = ok ? P.wval[e + k] : W(0);
          cv[k] = ok ? P.wcol[e + k] : 0u;
          inb[k] = ok;
        }
#pragma unroll
        for (uint32_t k = 0; k < kP; k++) inb[k] = inb[k] && lo + wv[k] < best && bit_test_ro(member, cv[k]);
#pragma unroll
        for (uint32_t k = 0; k < kP; k++) dc[k] = inb[k] ? ld_cg(P.dist + cv[k]) : W(0);
#pragma unroll
        for (uint32_t k = 0; k < kP; k++)
          if (inb[k]) {
            const W c = dc[k] + wv[k];
            if (c < best) best = c;
          }
        e += kP;
        open = e < end && lo + wv[kP - 1] < best;
      }
    }
    // long rows: one at a time, the warp's 32 lanes on consecutive edges
    for (uint32_t lm = __ballot_sync(kFullMask, cand && is_long); lm; lm &= lm - 1) {
      const uint32_t o = __ffs(lm) - 1;
      const uint32_t ob = __shfl_sync(kFullMask, beg, o), oe = __shfl_sync(kFullMask, end, o);
      W ob_best = __shfl_sync(kFullMask, best, o);
      for (uint32_t eb = ob; eb < oe; eb += 32) {
        const uint32_t x = eb + lane;
        const W w = x < oe ? P.wval[x] : W(0);
        W c = max_weight<W>();
        if (x < oe && lo + w < ob_best) {
          const uint32_t cc = P.wcol[x];
          if (bit_test_ro(member, cc)) c = ld_cg(P.dist + cc) + w;
        }
        c = warp_min_w(c);
        if (c < ob_best) ob_best = c;
        // the step's heaviest edge (lane 31; the row's last when it ends here)
        const W w_last = __shfl_sync(kFullMask, w, min(31u, oe - 1 - eb));
        if (!(lo + w_last < ob_best)) break;  // uniform: every lane holds the same values
      }
      if (lane == o) best = ob_best;
    }
    const bool improved = cand && best < d0;
    if (improved) st_cg(P.dist + u, best);
    const bool near = kLight && improved && best < threshold;
    const uint32_t fm = __ballot_sync(kFullMask, improved && !near);
    const uint32_t nm = __ballot_sync(kFullMask, near);
    if (lane == 0) {
      if (fm) atomicOr(P.far + wi, fm);
      if (nm) {
        st_cg(fb_next + wi, nm);  // cleared before this step; this warp is its only writer
        n_new += __popc(nm);
      }
    }
  }
  return n_new;
}

// The SSSP level loop: per iteration, push (compact the frontier, expand it
// with atomicMin relaxations) or, when the frontier's out-degree is a large
// part of the edges, one pull sweep.  Returns the number of iterations, or 0
// when a barrier timed out.  `fdeg0` is the out-degree of the first frontier.
template <typename W>
__device__ __forceinline__ uint32_t sssp_levels(const SsspParams<W>& P, const PushLoop& S, W lo, W threshold,
                                                bool bucketed, unsigned long long fdeg0, unsigned long long fsize0,
                                                uint32_t* s_scan, unsigned long long* s_red, uint32_t* s_best) {
  const uint32_t gtid = blockIdx.x * blockDim.x + threadIdx.x;
  const uint32_t nthreads = gridDim.x * blockDim.x;
  for (uint32_t level = 0;; level++) {
    Counters* C = S.cnt + (level % 3);
    const Counters* Cprev = S.cnt + ((level + 2) % 3);
    uint32_t* fb_cur = S.fb + (size_t)(level % 3) * S.w0;
    uint32_t* fb_next = S.fb + (size_t)((level + 1) % 3) * S.w0;
    uint32_t* fb_zero = S.fb + (size_t)((level + 2) % 3) * S.w0;
    const unsigned long long fdeg = level ? ld_cg(&Cprev->new_deg) : fdeg0;
    const unsigned long long fsize = level ? ld_cg(&Cprev->new_count) : fsize0;
    if (gtid == 0) {
      Counters z = {};
      S.cnt[(level + 1) % 3] = z;
    }
    const uint64_t t0 = (S.log && gtid == 0) ? sygraph::detail::global_timer_ns() : 0;
    // pull sweeps relax every edge: not with the light / heavy split
    const bool pull = !bucketed && P.pull_ratio && fdeg * P.pull_ratio > P.m;
    // a large frontier of a bucket: its light edges by pull, one barrier
    const bool pull_light = bucketed && P.light_pull && fsize * P.light_pull > S.n;
    unsigned long long n_new = 0, deg_new = 0;
    uint32_t ns = 0;
    unsigned long long bp = 0;
    if (pull_light) {
      n_new = sssp_pull_scan<W, true>(P, fb_cur, fb_next, lo, threshold);
    } else if (!pull) {
      // bucketed: light edges only, the prefix of each weight-sorted row
      const RowRange R = bucketed ? RowRange{S.ro, P.split, 0} : RowRange{S.ro, S.ro, 1};
      compact_frontier<kSsspChunk>(fb_cur, S.w0, R, C, S.q, s_scan, bucketed ? P.bucket : nullptr);
      if (!grid_sync(S.bar)) return 0;
      ns = ld_cg(&C->small_tail);
      bp = ld_cg(&C->big_packed);
      SsspRelax<W> X;
      X.dist = P.dist;
      X.w = bucketed ? P.wval : P.w;
      X.col = bucketed ? P.wcol : S.col;
      X.far = P.far;
      X.fb_next = fb_next;
      X.ro = S.ro;
      X.threshold = threshold;
      X.bucketed = bucketed;
      X.want_deg = !bucketed && P.pull_ratio;
      // delta-stepping's light iterations need only termination from the
      // count, unless a light pull decision reads the frontier size (the
      // frontier Bellman-Ford ran slower without the returned word: RMAT-22
      // 4.97 -> 5.11 ms, delta 0.1 1.89 -> 1.85 ms)
      X.exact = !bucketed || X.want_deg || P.light_pull;
      sssp_expand(R, S.q, ns, (uint32_t)(bp >> 32), (uint32_t)bp, X);
      n_new = X.n_new;
      deg_new = X.deg_new;
    } else {
      sssp_pull_sweep(P.pull, fb_cur, fb_next, threshold, bucketed, n_new, deg_new, s_best);
    }
    for (uint32_t i = gtid; i < S.w0; i += nthreads) st_cg(fb_zero + i, 0u);
    const unsigned long long c = block_sum<unsigned long long>(n_new, s_red);
    const unsigned long long d = block_sum<unsigned long long>(deg_new, s_red);
    if (threadIdx.x == 0) {
      if (c) atomicAdd(&C->new_count, c);
      if (d) atomicAdd(&C->new_deg, d);
    }
    if (!grid_sync(S.bar)) return 0;
    if (S.log && gtid == 0 && S.log_base + level < kMaxLog) {
      sg_level_record r = {};
      r.level = S.log_base + level;
      r.strategy = (pull || pull_light) ? 2u : 0u;
      r.frontier_size = pull ? 0u : pull_light ? (uint32_t)fsize : ns + (uint32_t)(bp >> 32);
      r.frontier_degree = fdeg;
      r.next_size = (uint32_t)ld_cg(&C->new_count);
      r.t_start_ns = t0;
      r.t_end_ns = sygraph::detail::global_timer_ns();
      S.log[S.log_base + level] = r;
    }
    if (ld_cg(&C->new_count) == 0) return level + 1;
  }
}

template <typename W>
__global__ void __launch_bounds__(kThreads, 2) sssp_kernel(SsspParams<W> P) {
  __shared__ uint32_t s_scan[32];
  __shared__ unsigned long long s_red[32];
  __shared__ uint32_t s_best[kThreads];
  __shared__ HeavySelect s_sel;
  const uint32_t gtid = blockIdx.x * blockDim.x + threadIdx.x, nthreads = gridDim.x * blockDim.x;
  const uint32_t n = P.L.n, w0 = P.L.w0, src = P.source;
  // learned heavy phases: the staged parameters arrive while the state is
  // initialised; the init barrier publishes them
  const bool staging = P.mlp_image && P.pull_ok;
  if (staging) sygraph::detail::mlp_stage_async(P.mlp_image, &s_sel.mlp);
  if (threadIdx.x == 0) s_sel.fk = feature_const(n, P.m, w0, (w0 + 31) / 32);
  const W inf = (W)(n + 1);  // (weight_t)(size + 1), sssp.hpp:43
  for (uint32_t i = gtid; i < n; i += nthreads) st_cg(P.dist + i, i == src ? (W)0 : inf);
  for (uint32_t i = gtid; i < w0; i += nthreads) {
    st_cg(P.L.fb + i, (i == (src >> 5)) ? (1u << (src & 31)) : 0u);
    st_cg(P.L.fb + w0 + i, 0u);
    st_cg(P.L.fb + 2 * w0 + i, 0u);
  }
  if (gtid < 3) {
    Counters z = {};
    P.L.cnt[gtid] = z;
  }
  const bool bucketed = P.delta > W(0);
  if (bucketed) {
    for (uint32_t i = gtid; i < w0; i += nthreads) {
      st_cg(P.far + i, 0u);
      st_cg(P.bucket + i, 0u);
    }
    if (gtid < 3) {
      Refill z = {};
      z.far_min = 0xffffffffu;
      P.refill[gtid] = z;
    }
  }
  if (staging) sygraph::detail::mlp_stage_wait();
  if (!grid_sync(P.L.bar)) return;
  // Near-far: vertices improved to a distance below the threshold stay in the
  // frontier, the others wait in the far set; when the near frontier is empty
  // the threshold moves up by delta (or to the far set's minimum) and the far
  // vertices below it become the next frontier.  Once half the vertices are
  // settled and a refill leaves fewer than P.tail vertices in the far set, the
  // next refill takes all of them and the rest runs as plain frontier
  // Bellman-Ford (every edge, no far set): the last, sparse stretch of
  // distances then costs a few iterations instead of one bucket per delta.  Every improved vertex is relaxed again before the
  // end, so the fixed point is Bellman-Ford's.
  W threshold = P.delta;
  W lo = W(0);  // the current bucket is [lo, threshold)
  unsigned long long total = 0;
  uint32_t pass = 0;
  PushLoop loop = P.L;
  unsigned long long fdeg0 = P.L.ro[src + 1] - P.L.ro[src];
  unsigned long long fsize0 = 1;  // vertices of the first frontier of the next bucket
  bool near_far = bucketed;
  unsigned long long far_left = ~0ull;  // far vertices the last refill left
  unsigned long long settled = 0;       // vertices of finished buckets
  uint32_t records = 0;                 // log entries written: iterations, heavy phases, refills
  uint32_t phases = 0;                  // heavy phases run
  unsigned long long heavy_done = 0;    // heavy edges of the buckets before this one
  unsigned long long prev_bucket = 1;   // vertices of the previous bucket
  bool prev_pull = false;               // direction of the previous heavy phase
  // one log entry for a heavy phase (strategy 4) or a refill pass (5)
  auto log_phase = [&](uint32_t kind, uint64_t t0, unsigned long long size, unsigned long long next) {
    if (P.L.log && gtid == 0 && records < kMaxLog) {
      sg_level_record r = {};
      r.level = records;
      r.strategy = kind;
      r.frontier_size = (uint32_t)size;
      r.next_size = (uint32_t)next;
      r.t_start_ns = t0;
      r.t_end_ns = sygraph::detail::global_timer_ns();
      P.L.log[records] = r;
    }
    records++;
  };
  for (;;) {
    loop.log_base = min(records, kMaxLog);
    const uint32_t levels = sssp_levels(P, loop, lo, threshold, near_far, fdeg0, fsize0, s_scan, s_red, s_best);
    if (!levels) return;
    total += levels;
    records += levels;
    if (!near_far) break;
    {
      const uint64_t t0 = (P.L.log && gtid == 0) ? sygraph::detail::global_timer_ns() : 0;
      // heavy edges (w >= delta) of the bucket's vertices, relaxed once with
      // their final distances: they land at or beyond the threshold (far)
      Counters* Ch = P.L.cnt + (levels % 3);  // zeroed by the last level, unused since
      const RowRange Rh{P.split, P.L.ro, 1};   // the suffix of each weight-sorted row
      compact_frontier<kSsspChunk>(P.bucket, w0, Rh, Ch, P.L.q, s_scan);
      if (!grid_sync(P.L.bar)) return;
      const uint32_t ns = ld_cg(&Ch->small_tail);
      const unsigned long long bp = ld_cg(&Ch->big_packed);
      const unsigned long long bsize = ns + (bp >> 32), hdeg = ld_cg(&Ch->frontier_deg);
      settled += bsize;
      // pull when the push would relax a large share of the edges (or as the
      // learned selector says)
      const bool h_pull = P.heavy_pull && hdeg * P.heavy_pull > P.m;
      const FeatureInputs x{(double)bsize, (double)hdeg, (double)(P.m - min(P.m, heavy_done)), (double)settled,
                            (double)prev_bucket, prev_pull};
      const bool pull_heavy = heavy_decide(P, s_sel, h_pull, x, phases);
      phases++;
      heavy_done += hdeg;
      prev_bucket = bsize;
      prev_pull = pull_heavy;
      if (pull_heavy) {
        sssp_pull_scan<W, false>(P, P.bucket, nullptr, lo, threshold);
      } else {
        SsspRelax<W> X;
        X.dist = P.dist;
        X.w = P.wval;
        X.col = P.wcol;
        X.far = P.far;
        X.fb_next = P.L.fb + (size_t)((levels + 1) % 3) * w0;
        X.ro = P.L.ro;
        X.threshold = threshold;
        X.bucketed = true;
        X.want_deg = false;
        X.exact = false;
        sssp_expand(Rh, P.L.q, ns, (uint32_t)(bp >> 32), (uint32_t)bp, X);
      }
      // the bucket bitmap is cleared by the refill (the pull reads it until the barrier)
      if (!grid_sync(P.L.bar)) return;
      log_phase(pull_heavy ? 6 : 4, t0, ns + (bp >> 32), 0);
    }
    bool refilled = false;
    for (;;) {
      // far vertices below the new threshold become fb[0]; fb[1], fb[2] cleared
      Refill* R = P.refill + (pass % 3);
      if (gtid == 0) {
        Refill z = {};
        z.far_min = 0xffffffffu;
        P.refill[(pass + 1) % 3] = z;
      }
      if (gtid < 3) {
        Counters z = {};
        P.L.cnt[gtid] = z;
      }
      // (only once half the vertices are settled: early on the far set is
      // small because little has been reached yet)
      const bool tail = far_left < P.tail && 2 * settled >= n;
      const uint64_t t0 = (P.L.log && gtid == 0) ? sygraph::detail::global_timer_ns() : 0;
      const W next_t = tail ? max_weight<W>() : threshold + P.delta;
      unsigned long long moved = 0, remaining = 0;
      uint32_t fmin = 0xffffffffu;
      for (uint32_t i = gtid; i < w0; i += nthreads) {
        const uint32_t f = ld_cg(P.far + i);
        uint32_t near = 0;
        // the word's far distances, 16 loads in flight at a time
#pragma unroll
        for (uint32_t h = 0; h < 32; h += 16) {
          const uint32_t fh = (f >> h) & 0xffffu;
          if (!fh) continue;
          W d[16];
#pragma unroll
          for (uint32_t k = 0; k < 16; k++) d[k] = ((fh >> k) & 1u) ? ld_cg(P.dist + i * 32 + h + k) : W(0);
#pragma unroll
          for (uint32_t k = 0; k < 16; k++) {
            if (!((fh >> k) & 1u)) continue;
            if (d[k] < next_t)
              near |= 1u << (h + k);
            else
              fmin = min(fmin, order_bits<W>(d[k]));
          }
        }
        st_cg(P.L.fb + i, near);
        st_cg(P.L.fb + w0 + i, 0u);
        st_cg(P.L.fb + 2 * w0 + i, 0u);
        st_cg(P.bucket + i, 0u);
        if (f) st_cg(P.far + i, f & ~near);
        moved += __popc(near);
        remaining += __popc(f & ~near);
      }
      const unsigned long long mv = block_sum<unsigned long long>(moved, s_red);
      const unsigned long long rm = block_sum<unsigned long long>(remaining, s_red);
      fmin = sygraph::detail::warp_min(fmin);
      if ((threadIdx.x & 31) == 0 && fmin != 0xffffffffu) atomicMin(&R->far_min, fmin);
      if (threadIdx.x == 0) {
        if (mv) atomicAdd(&R->moved, mv);
        if (rm) atomicAdd(&R->remaining, rm);
      }
      if (!grid_sync(P.L.bar)) return;
      pass++;
      lo = threshold;
      threshold = next_t;
      far_left = ld_cg(&R->remaining);
      log_phase(5, t0, ld_cg(&R->moved), far_left);
      if (tail) near_far = false;
      if (ld_cg(&R->moved)) {
        fdeg0 = 0;  // not summed: only a pull decision reads it, and pull is off with the light / heavy split
        fsize0 = ld_cg(&R->moved);
        refilled = true;
        break;
      }
      if (!far_left) break;
      // nothing below the new threshold: jump to the far set's minimum
      const W m = from_order_bits<W>(ld_cg(&R->far_min));
      if (threshold < m) threshold = m;
    }
    if (!refilled) break;
  }
  if (gtid == 0) {
    P.result[0] = total;
    P.result[1] = pass;
    P.result[2] = records;
    P.result[3] = phases;
  }
}

struct CcParams {
  PushLoop L;
  uint32_t* labels;
  unsigned long long* result;
};

struct CcVisitor : NextFrontier {
  using src_t = uint32_t;
  uint32_t* labels;
  __device__ __forceinline__ uint32_t src(uint32_t v) const { return ld_cg(labels + v); }
  __device__ __forceinline__ bool visit(uint32_t u, uint32_t, uint32_t sl, uint32_t) {
    if (ld_cg(labels + u) >= sl) return false;
    return atomicMax(labels + u, sl) < sl;
  }
};

__global__ void __launch_bounds__(kThreads, 2) cc_kernel(CcParams P) {
  __shared__ uint32_t s_scan[32];
  __shared__ unsigned long long s_red[32];
  const uint32_t gtid = blockIdx.x * blockDim.x + threadIdx.x, nthreads = gridDim.x * blockDim.x;
  const uint32_t n = P.L.n, w0 = P.L.w0;
  // labels[i] = i (cc.hpp:121-128); the first level pushes from every vertex,
  // which is the reference's advance::vertices pass (cc.hpp:135-145).
  for (uint32_t i = gtid; i < n; i += nthreads) st_cg(P.labels + i, i);
  for (uint32_t i = gtid; i < w0; i += nthreads) {
    st_cg(P.L.fb + i, valid_bits(i, w0, n));
    st_cg(P.L.fb + w0 + i, 0u);
    st_cg(P.L.fb + 2 * w0 + i, 0u);
  }
  if (gtid < 3) {
    Counters z = {};
    P.L.cnt[gtid] = z;
  }
  if (!grid_sync(P.L.bar)) return;
  const uint32_t levels = push_levels(
      P.L,
      [&](uint32_t, uint32_t* fb_next) {
        CcVisitor v;
        v.fb_next = fb_next;
        v.labels = P.labels;
        return v;
      },
      s_scan, s_red);
  if (gtid == 0) P.result[0] = levels;
}

// Connected components of an undirected graph by lock-free union-find, then
// the largest id of each component as its label (the label propagation's
// result).  Links put the larger root under the smaller, so a component's
// root is its smallest id: on a power-law graph a hub, which stops changing
// early, and every link CASes the thread's own root instead of a shared
// one.  A failed link means another thread linked that root first, so every
// retry follows progress of the whole grid: no thread waits on another.
// Every access to the parent array that races with the links is a strong
// relaxed one (coherent with the atomics), and the memory clobber keeps the
// compiler from reusing or moving it.
__device__ __forceinline__ uint32_t ld_relaxed(const uint32_t* p) {
  uint32_t v;
  asm volatile("ld.relaxed.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
  return v;
}

__device__ __forceinline__ void st_relaxed(uint32_t* p, uint32_t v) {
  asm volatile("st.relaxed.gpu.global.u32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}

__device__ __forceinline__ uint32_t uf_find(uint32_t* parent, uint32_t x) {
  for (;;) {
    const uint32_t p = ld_relaxed(parent + x);
    if (p == x) return x;
    const uint32_t gp = ld_relaxed(parent + p);
    if (gp != p) st_relaxed(parent + x, gp);  // path halving: gp is an ancestor of x
    x = gp;
  }
}

__device__ __forceinline__ void uf_unite(uint32_t* parent, uint32_t u, uint32_t v) {
  for (;;) {
    u = uf_find(parent, u);
    v = uf_find(parent, v);
    if (u == v) return;
    if (u < v) {
      const uint32_t t = u;
      u = v;
      v = t;
    }
    if (atomicCAS(parent + u, u, v) == u) return;  // larger root under the smaller
  }
}

__global__ void __launch_bounds__(256) uf_init_kernel(uint32_t* __restrict__ parent, uint32_t* __restrict__ top,
                                                      uint32_t n) {
  for (uint32_t v = blockIdx.x * blockDim.x + threadIdx.x; v < n; v += gridDim.x * blockDim.x) {
    parent[v] = v;
    top[v] = v;
  }
}

// Afforest-style order: every vertex first unites with its first kSampled
// neighbours (one round per neighbour index; one round measured best on
// RMAT-20 and RMAT-22, a second cost 18% on RMAT-22), the trees are
// flattened, and
// the root shared by most of 1024 sampled vertices is taken as the giant
// component's; then only vertices outside it unite with their other
// neighbours.  An edge skipped at an endpoint inside the giant component is
// united from its other endpoint (the rows hold every edge both ways) unless
// that endpoint is inside too.
constexpr uint32_t kSampled = 1, kGiantSamples = 1024;

__global__ void __launch_bounds__(256) uf_sample_kernel(const uint32_t* __restrict__ ro, const uint32_t* __restrict__ col,
                                                        uint32_t n, uint32_t r, uint32_t* parent) {
  for (uint32_t u = blockIdx.x * blockDim.x + threadIdx.x; u < n; u += gridDim.x * blockDim.x) {
    const uint32_t b = ro[u];
    if (ro[u + 1] - b > r) uf_unite(parent, u, col[b + r]);
  }
}

// One block of kGiantSamples threads: the most frequent root among the
// samples (ties to the larger id); the trees are flat when it runs.
__global__ void __launch_bounds__(kGiantSamples) uf_giant_kernel(const uint32_t* parent, uint32_t n,
                                                                 uint32_t* __restrict__ giant) {
  __shared__ uint32_t s_root[kGiantSamples];
  __shared__ unsigned long long s_best;
  const uint32_t i = threadIdx.x;
  s_root[i] = ld_relaxed(parent + (uint32_t)(((uint64_t)i * 2654435761u) % n));
  if (i == 0) s_best = 0;
  __syncthreads();
  uint32_t c = 0;
  for (uint32_t j = 0; j < kGiantSamples; j++) c += s_root[j] == s_root[i];
  atomicMax(&s_best, ((unsigned long long)c << 32) | s_root[i]);
  __syncthreads();
  if (i == 0) *giant = (uint32_t)s_best;
}

__global__ void __launch_bounds__(256) uf_rest_kernel(const uint32_t* __restrict__ ro, const uint32_t* __restrict__ col,
                                                      uint32_t n, const uint32_t* __restrict__ giant, uint32_t* parent) {
  const uint32_t g = *giant;
  for (uint32_t u = blockIdx.x * blockDim.x + threadIdx.x; u < n; u += gridDim.x * blockDim.x) {
    if (ld_relaxed(parent + u) == g) continue;
    const uint32_t e = ro[u + 1];
    for (uint32_t i = ro[u] + kSampled; i < e; i++) uf_unite(parent, u, col[i]);
  }
}

// Flattening: every vertex's parent becomes its root.  The walk only reads:
// a path-halving store here could land after another vertex's root and
// replace it with an ancestor short of the root.  The only stores are roots,
// so every value read is still an ancestor.
__global__ void __launch_bounds__(256) uf_flatten_kernel(uint32_t* parent, uint32_t n) {
  for (uint32_t v = blockIdx.x * blockDim.x + threadIdx.x; v < n; v += gridDim.x * blockDim.x) {
    uint32_t x = v;
    for (uint32_t p = ld_relaxed(parent + x); p != x; p = ld_relaxed(parent + x)) x = p;
    st_relaxed(parent + v, x);
  }
}

// top[root] = largest id of the root's (flat) tree: one atomicMax per root
// and warp, and for the giant component's root one per block (through
// shared memory), since most vertices carry it.
__global__ void __launch_bounds__(256) uf_top_kernel(const uint32_t* __restrict__ parent, uint32_t* top, uint32_t n,
                                                     const uint32_t* __restrict__ giant) {
  __shared__ uint32_t s_giant_max;
  const uint32_t lane = threadIdx.x & 31u, gr = *giant;
  if (threadIdx.x == 0) s_giant_max = 0;
  __syncthreads();
  for (uint32_t base = blockIdx.x * blockDim.x + threadIdx.x - lane; base < n; base += gridDim.x * blockDim.x) {
    const uint32_t v = base + lane;
    const bool ok = v < n;
    const uint32_t r = ok ? parent[v] : 0xffffffffu;
    const uint32_t same = __match_any_sync(0xffffffffu, r);
    const uint32_t mx = __reduce_max_sync(same, ok ? v : 0u);
    if (ok && lane == __ffs(same) - 1u) {
      if (r == gr)
        atomicMax(&s_giant_max, mx);
      else
        atomicMax(top + r, mx);
    }
  }
  __syncthreads();
  if (threadIdx.x == 0 && s_giant_max) atomicMax(top + gr, s_giant_max);
}

// labels[v] = top[root(v)]; in place: each thread reads only its own parent.
__global__ void __launch_bounds__(256) uf_label_kernel(uint32_t* parent, const uint32_t* __restrict__ top, uint32_t n) {
  for (uint32_t v = blockIdx.x * blockDim.x + threadIdx.x; v < n; v += gridDim.x * blockDim.x) parent[v] = top[parent[v]];
}

}  // namespace

// Workspace shared by the push engines: rotating bitmaps, queues, counters.
struct PushWorkspace {
  uint32_t w0 = 0;
  uint32_t* fb = nullptr;
  Queues q{};
  Counters* cnt = nullptr;
  GridBarrier* bar = nullptr;
  unsigned long long* result = nullptr;
  sg_status alloc(uint32_t n) {
    w0 = div_up(n, 32);
    sg_status s;
    if ((s = dev_alloc(&fb, 3ull * w0)) || (s = dev_alloc(&q.small, n)) || (s = dev_alloc(&q.big, n)) ||
        (s = dev_alloc(&q.big_start, n)) || (s = dev_alloc(&cnt, 3)) || (s = dev_alloc(&bar, 1)) ||
        (s = dev_alloc(&result, 4)))
      return s;
    return SG_OK;
  }
  void release() {
    dev_free(fb);
    dev_free(q.small);
    dev_free(q.big);
    dev_free(q.big_start);
    dev_free(cnt);
    dev_free(bar);
    dev_free(result);
  }
  PushLoop loop(sg_graph g) const {
    PushLoop L;
    L.n = g->n;
    L.w0 = w0;
    L.ro = g->fwd.ro;
    L.col = g->fwd.col;
    L.fb = fb;
    L.q = q;
    L.cnt = cnt;
    L.bar = bar;
    return L;
  }
  sg_status finish(cudaStream_t s, uint64_t* levels) {
    unsigned long long r = 0;
    GridBarrier b;
    SG_CUDA(cudaMemcpyAsync(&r, result, sizeof(r), cudaMemcpyDeviceToHost, s));
    SG_CUDA(cudaMemcpyAsync(&b, bar, sizeof(b), cudaMemcpyDeviceToHost, s));
    SG_CUDA(cudaStreamSynchronize(s));
    if (b.error) return fail(SG_ERR_TIMEOUT, "engine: a grid barrier wait ran out");
    if (levels) *levels = r;
    return SG_OK;
  }
};

}  // namespace sgb

using namespace sgb;

struct sg_cc_s {
  sg_graph g = nullptr;
  cudaStream_t stream = nullptr;
  uint32_t* labels = nullptr;
  bool ran = false;
  int method = SG_CC_AUTO;
  bool used_union_find = false;
  PushWorkspace ws;
};

struct sg_sssp_s {
  sg_graph g = nullptr;
  cudaStream_t stream = nullptr;
  uint32_t max_ctas = 0;
  uint32_t source = 0;
  bool initialised = false;
  bool fresh = false;  // initialised but not run: distances not written yet
  void* dist = nullptr;
  sg_level_record* log = nullptr;
  uint32_t* far = nullptr;
  uint32_t* bucket = nullptr;
  uint32_t* split = nullptr;  // for split_delta
  double split_delta = -1.0;
  Refill* refill = nullptr;
  double delta = 0.0;  // near-far threshold step; 0 = the reference's frontier Bellman-Ford
  double tail = 0.25;  // far-set fraction of n below which the rest runs as plain Bellman-Ford
  uint32_t heavy_pull = 8;  // heavy phase by pull when its push would relax more than m / heavy_pull edges
  // light iteration by pull when its frontier holds more than n / light_pull
  // vertices; off by default: on RMAT-22 the warps holding the low-id hubs'
  // long light prefixes made each pull iteration take milliseconds
  uint32_t light_pull = 0;
  uint32_t pull_ratio = 0;  // pull iterations when frontier out-degree * ratio > m; 0 = push only
  uint32_t* heavy_v = nullptr;      // vertices of in-degree >= kPullHeavy
  uint32_t* heavy_first = nullptr;  // their first chunk index
  uint32_t n_heavy = 0, n_chunks = 0;
  const void* mlp_image = nullptr;  // learned heavy phases: the selector's staged image (owned by the sg_mlp)
  float margin = 0.05f;
  float heavy_lo = 0.f, heavy_hi = 1e30f;
  float* features = nullptr;  // feature log, 12 floats per heavy phase
  PushWorkspace ws;
};

// First edge of weight >= delta in each weight-sorted row (binary search).
template <typename W>
__global__ void split_kernel(const uint32_t* __restrict__ ro, const W* __restrict__ wval, uint32_t n, W delta,
                             uint32_t* __restrict__ split) {
  for (uint32_t v = blockIdx.x * blockDim.x + threadIdx.x; v < n; v += gridDim.x * blockDim.x) {
    uint32_t lo = ro[v], hi = ro[v + 1];
    while (lo < hi) {
      const uint32_t mid = lo + ((hi - lo) >> 1);
      if (wval[mid] < delta)
        lo = mid + 1;
      else
        hi = mid;
    }
    split[v] = lo;
  }
}

template <typename W>
__global__ void fill_dist_kernel(W* dist, uint32_t n, uint32_t src) {
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
    dist[i] = i == src ? (W)0 : (W)(n + 1);
}

// SSSPInstance ctor state (sssp.hpp:392-405), written only when distances are
// read before a run.
static sg_status sssp_materialise(sg_sssp s) {
  if (!s->fresh) return SG_OK;
  sg_graph g = s->g;
  if (g->value_type == SG_WEIGHT_F32)
    fill_dist_kernel<float><<<grid_for(g->n, 256), 256, 0, s->stream>>>((float*)s->dist, g->n, s->source);
  else
    fill_dist_kernel<uint32_t><<<grid_for(g->n, 256), 256, 0, s->stream>>>((uint32_t*)s->dist, g->n, s->source);
  SG_CHECK_LAUNCH();
  s->fresh = false;
  return SG_OK;
}

static sg_status sssp_launch(sg_sssp s) {
  sg_graph g = s->g;
  if (s->delta > 0.0 && s->split_delta != s->delta) {
    // delta-stepping reads the weight-sorted rows: their light prefix / heavy suffix
    SG_TRY(graph_weight_sorted(g));
    if (!s->split) SG_TRY(dev_alloc(&s->split, g->n));
    if (g->value_type == SG_WEIGHT_F32)
      split_kernel<float><<<grid_for(g->n, 256), 256, 0, s->stream>>>(g->fwd.ro, (const float*)g->wval, g->n,
                                                                       (float)s->delta, s->split);
    else
      split_kernel<uint32_t><<<grid_for(g->n, 256), 256, 0, s->stream>>>(
          g->fwd.ro, (const uint32_t*)g->wval, g->n,
          (uint32_t)std::max(1.0, std::min(s->delta, 4294967295.0)), s->split);
    SG_CHECK_LAUNCH();
    s->split_delta = s->delta;
  }
  SG_CUDA(cudaMemsetAsync(s->ws.bar, 0, sizeof(GridBarrier), s->stream));
  PushLoop L = s->ws.loop(g);
  L.log = s->log;
  if (g->value_type == SG_WEIGHT_F32) {
    SsspParams<float> P{L, s->source, (float*)s->dist, (const float*)g->fwd.val, s->ws.result,
                        s->far, s->bucket, s->refill, (float)s->delta};
    P.pull = PullArgs<float>{g->n, L.w0, g->fwd.ro, g->inv.ro, g->inv.col, (const float*)g->inv.val,
                             (float*)s->dist, s->far, s->heavy_v, s->heavy_first, s->n_heavy, s->n_chunks};
    P.pull_ratio = s->pull_ratio;
    P.m = g->m;
    P.split = s->split;
    P.wcol = g->wcol;
    P.wval = (const float*)g->wval;
    P.tail = (uint32_t)(s->tail * g->n);
    P.heavy_pull = g->wsym ? s->heavy_pull : 0u;
    P.light_pull = g->wsym ? s->light_pull : 0u;
    P.mlp_image = static_cast<const sygraph::detail::MlpStaged*>(s->delta > 0.0 ? s->mlp_image : nullptr);
    P.margin = s->margin;
    P.heavy_lo = s->heavy_lo;
    P.heavy_hi = s->heavy_hi;
    P.pull_ok = g->wsym;
    P.features = s->features;
    return launch_persistent(sssp_kernel<float>, P, 2, s->stream, s->max_ctas);
  }
  const uint32_t d = s->delta > 0.0 ? (uint32_t)std::max(1.0, std::min(s->delta, 4294967295.0)) : 0u;
  SsspParams<uint32_t> P{L, s->source, (uint32_t*)s->dist, (const uint32_t*)g->fwd.val, s->ws.result,
                         s->far, s->bucket, s->refill, d};
  P.pull = PullArgs<uint32_t>{g->n, L.w0, g->fwd.ro, g->inv.ro, g->inv.col, (const uint32_t*)g->inv.val,
                              (uint32_t*)s->dist, s->far, s->heavy_v, s->heavy_first, s->n_heavy, s->n_chunks};
  P.pull_ratio = s->pull_ratio;
  P.m = g->m;
  P.split = s->split;
  P.wcol = g->wcol;
  P.wval = (const uint32_t*)g->wval;
  P.tail = (uint32_t)(s->tail * g->n);
  P.heavy_pull = g->wsym ? s->heavy_pull : 0u;
  P.light_pull = g->wsym ? s->light_pull : 0u;
  P.mlp_image = static_cast<const sygraph::detail::MlpStaged*>(s->delta > 0.0 ? s->mlp_image : nullptr);
  P.margin = s->margin;
  P.heavy_lo = s->heavy_lo;
  P.heavy_hi = s->heavy_hi;
  P.pull_ok = g->wsym;
  P.features = s->features;
  return launch_persistent(sssp_kernel<uint32_t>, P, 2, s->stream, s->max_ctas);
}

extern "C" {

sg_status sg_sssp_create(sg_graph g, sg_sssp* out) {
  clear_error();
  SG_REQUIRE(g && out, SG_ERR_INVALID, "NULL argument");
  SG_REQUIRE(g->n > 0, SG_ERR_INVALID, "graph has no vertices");
  *out = nullptr;
  sg_sssp s = new sg_sssp_s();
  s->g = g;
  s->stream = g->stream;
  uint32_t* d = nullptr;
  sg_status st = dev_alloc(&d, g->n);
  s->dist = d;
  if (st == SG_OK) st = s->ws.alloc(g->n);
  if (st == SG_OK) st = dev_alloc(&s->far, div_up(g->n, 32));
  if (st == SG_OK) st = dev_alloc(&s->bucket, div_up(g->n, 32));
  if (st == SG_OK) st = dev_alloc(&s->refill, 3);
  if (st == SG_OK) st = dev_alloc(&s->log, SG_MAX_LOGGED_LEVELS);
  if (st == SG_OK) {
    // static chunk list of the vertices pulled in chunks (in-degree >= kPullHeavy)
    std::vector<uint32_t> iro((size_t)g->n + 1), hv, hf;
    if (cudaMemcpy(iro.data(), g->inv.ro, sizeof(uint32_t) * iro.size(), cudaMemcpyDeviceToHost) != cudaSuccess) {
      cudaGetLastError();
      st = fail(SG_ERR_CUDA, "SSSP set-up: reading the in-edge offsets failed");
    }
    uint32_t chunks = 0;
    for (uint32_t v = 0; st == SG_OK && v < g->n; v++) {
      const uint32_t d = iro[v + 1] - iro[v];
      if (d >= eng::kPullHeavy) {
        hv.push_back(v);
        hf.push_back(chunks);
        chunks += (d + eng::kPullChunk - 1) / eng::kPullChunk;
      }
    }
    if (st == SG_OK && !hv.empty()) {
      st = dev_alloc(&s->heavy_v, hv.size());
      if (st == SG_OK) st = dev_alloc(&s->heavy_first, hf.size());
      if (st == SG_OK && (cudaMemcpy(s->heavy_v, hv.data(), 4 * hv.size(), cudaMemcpyHostToDevice) != cudaSuccess ||
                          cudaMemcpy(s->heavy_first, hf.data(), 4 * hf.size(), cudaMemcpyHostToDevice) != cudaSuccess)) {
        cudaGetLastError();
        st = fail(SG_ERR_CUDA, "SSSP set-up: uploading the chunk list failed");
      }
      s->n_heavy = (uint32_t)hv.size();
      s->n_chunks = chunks;
    }
  }
  if (st != SG_OK) {
    s->ws.release();
    cudaFree(s->dist);
    dev_free(s->far);
    dev_free(s->bucket);
    dev_free(s->split);
    dev_free(s->refill);
    dev_free(s->log);
    dev_free(s->heavy_v);
    dev_free(s->heavy_first);
    delete s;
    return st;
  }
  *out = s;
  return SG_OK;
}

sg_status sg_sssp_destroy(sg_sssp s) {
  if (s) {
    cudaStreamSynchronize(s->stream);
    s->ws.release();
    cudaFree(s->dist);
    dev_free(s->far);
    dev_free(s->bucket);
    dev_free(s->split);
    dev_free(s->refill);
    dev_free(s->log);
    dev_free(s->heavy_v);
    dev_free(s->heavy_first);
    dev_free(s->features);
    delete s;
  }
  return SG_OK;
}

sg_status sg_sssp_set_pull(sg_sssp s, uint32_t ratio) {
  clear_error();
  SG_REQUIRE(s, SG_ERR_INVALID, "sssp is NULL");
  s->pull_ratio = ratio;
  return SG_OK;
}

sg_status sg_sssp_set_selector(sg_sssp s, sg_mlp mlp, float margin, float min_heavy, float max_heavy) {
  clear_error();
  SG_REQUIRE(s, SG_ERR_INVALID, "sssp is NULL");
  SG_REQUIRE(margin >= 0.f && min_heavy >= 0.f && min_heavy <= max_heavy, SG_ERR_INVALID,
             "margin >= 0 and 0 <= min_heavy <= max_heavy");
  SG_CUDA(cudaStreamSynchronize(s->stream));  // a queued launch may still read the old image
  s->mlp_image = mlp ? mlp_device_image(mlp) : nullptr;
  s->margin = margin;
  s->heavy_lo = min_heavy;
  s->heavy_hi = max_heavy;
  return SG_OK;
}

sg_status sg_sssp_log_features(sg_sssp s, int enable) {
  clear_error();
  SG_REQUIRE(s, SG_ERR_INVALID, "sssp is NULL");
  SG_CUDA(cudaStreamSynchronize(s->stream));
  if (enable && !s->features) SG_TRY(dev_alloc(&s->features, 12ull * SG_MAX_LOGGED_LEVELS));
  if (!enable) dev_free(s->features);
  return SG_OK;
}

sg_status sg_sssp_level_features(sg_sssp s, float* host_features, uint32_t cap, uint32_t* count) {
  SG_REQUIRE(s && count, SG_ERR_INVALID, "NULL argument");
  SG_REQUIRE(s->features, SG_ERR_NOT_INITIALIZED, "feature logging is off (sg_sssp_log_features)");
  SG_CUDA(cudaStreamSynchronize(s->stream));
  unsigned long long r[4] = {0, 0, 0, 0};
  SG_CUDA(cudaMemcpy(r, s->ws.result, sizeof(r), cudaMemcpyDeviceToHost));
  uint32_t k = (uint32_t)(r[3] < SG_MAX_LOGGED_LEVELS ? r[3] : SG_MAX_LOGGED_LEVELS);
  if (k > cap) k = cap;
  if (host_features && k)
    SG_CUDA(cudaMemcpy(host_features, s->features, sizeof(float) * 12 * k, cudaMemcpyDeviceToHost));
  *count = k;
  return SG_OK;
}

}  // extern "C"

sg_status sgb::sssp_launch_status(sg_sssp s) {
  uint32_t err = 0;
  SG_CUDA(cudaMemcpyAsync(&err, &s->ws.bar->error, sizeof(err), cudaMemcpyDeviceToHost, s->stream));
  SG_CUDA(cudaStreamSynchronize(s->stream));
  return err ? fail(SG_ERR_TIMEOUT, "SSSP engine: a grid barrier wait ran out") : SG_OK;
}

extern "C" {

sg_status sg_sssp_level_records(sg_sssp s, sg_level_record* host_records, uint32_t cap, uint32_t* count) {
  SG_REQUIRE(s && count, SG_ERR_INVALID, "NULL argument");
  SG_CUDA(cudaStreamSynchronize(s->stream));
  unsigned long long it = 0;  // log entries of the last run
  SG_CUDA(cudaMemcpy(&it, s->ws.result + 2, sizeof(it), cudaMemcpyDeviceToHost));
  uint32_t k = (uint32_t)(it < SG_MAX_LOGGED_LEVELS ? it : SG_MAX_LOGGED_LEVELS);
  if (k > cap) k = cap;
  if (host_records && k) SG_CUDA(cudaMemcpy(host_records, s->log, sizeof(sg_level_record) * k, cudaMemcpyDeviceToHost));
  *count = k;
  return SG_OK;
}

sg_status sg_sssp_set_launch(sg_sssp s, void* stream, uint32_t max_ctas) {
  clear_error();
  SG_REQUIRE(s, SG_ERR_INVALID, "sssp is NULL");
  SG_CUDA(cudaStreamSynchronize(s->stream));
  s->stream = stream ? (cudaStream_t)stream : s->g->stream;
  s->max_ctas = max_ctas;
  return SG_OK;
}

sg_status sg_sssp_set_heavy_pull(sg_sssp s, uint32_t ratio) {
  clear_error();
  SG_REQUIRE(s, SG_ERR_INVALID, "sssp is NULL");
  s->heavy_pull = ratio;
  return SG_OK;
}

sg_status sg_sssp_set_light_pull(sg_sssp s, uint32_t ratio) {
  clear_error();
  SG_REQUIRE(s, SG_ERR_INVALID, "sssp is NULL");
  s->light_pull = ratio;
  return SG_OK;
}

sg_status sg_sssp_set_tail(sg_sssp s, double fraction) {
  clear_error();
  SG_REQUIRE(s, SG_ERR_INVALID, "sssp is NULL");
  SG_REQUIRE(fraction >= 0.0 && fraction <= 1.0, SG_ERR_INVALID, "tail fraction must be in [0, 1]");
  s->tail = fraction;
  return SG_OK;
}

sg_status sg_sssp_set_delta(sg_sssp s, double delta) {
  clear_error();
  SG_REQUIRE(s, SG_ERR_INVALID, "sssp is NULL");
  SG_REQUIRE(delta >= 0.0 && delta < 1e30, SG_ERR_INVALID, "delta must be finite and non-negative");
  s->delta = delta;
  return SG_OK;
}

sg_status sg_sssp_init(sg_sssp s, uint32_t source) {
  clear_error();
  SG_REQUIRE(s, SG_ERR_INVALID, "sssp is NULL");
  SG_REQUIRE(source < s->g->n, SG_ERR_INVALID, "source out of range");
  s->source = source;
  s->initialised = true;
  s->fresh = true;
  return SG_OK;
}

sg_status sg_sssp_run_async(sg_sssp s) {
  clear_error();
  SG_REQUIRE(s, SG_ERR_INVALID, "sssp is NULL");
  SG_REQUIRE(s->initialised, SG_ERR_NOT_INITIALIZED, "SSSP instance not initialized");
  s->fresh = false;
  return sssp_launch(s);
}

sg_status sg_sssp_run(sg_sssp s, uint64_t* iterations) {
  SG_TRY(sg_sssp_run_async(s));
  return s->ws.finish(s->stream, iterations);
}

sg_status sg_sssp_get_distances(sg_sssp s, void* host_dist) {
  SG_REQUIRE(s && host_dist, SG_ERR_INVALID, "NULL argument");
  SG_REQUIRE(s->initialised, SG_ERR_NOT_INITIALIZED, "SSSP instance not initialized");
  SG_TRY(sssp_materialise(s));
  SG_CUDA(cudaMemcpyAsync(host_dist, s->dist, sizeof(uint32_t) * s->g->n, cudaMemcpyDeviceToHost, s->stream));
  SG_CUDA(cudaStreamSynchronize(s->stream));
  return SG_OK;
}

sg_status sg_sssp_distances_device(sg_sssp s, const void** dev_dist) {
  SG_REQUIRE(s && dev_dist, SG_ERR_INVALID, "NULL argument");
  if (s->initialised) SG_TRY(sssp_materialise(s));
  *dev_dist = s->dist;
  return SG_OK;
}

sg_status sg_run_sssp(sg_graph g, uint32_t source, void* host_dist, uint64_t* iterations) {
  sg_sssp s = nullptr;
  SG_TRY(sg_sssp_create(g, &s));
  sg_status st = sg_sssp_init(s, source);
  if (st == SG_OK) st = sg_sssp_run(s, iterations);
  if (st == SG_OK && host_dist) st = sg_sssp_get_distances(s, host_dist);
  sg_sssp_destroy(s);
  return st;
}

sg_status sg_cc_destroy(sg_cc_handle c) {
  if (c) {
    cudaStreamSynchronize(c->stream);
    c->ws.release();
    dev_free(c->labels);
    delete c;
  }
  return SG_OK;
}

sg_status sg_cc_create(sg_graph g, sg_cc_handle* out) {
  clear_error();
  SG_REQUIRE(g && out, SG_ERR_INVALID, "NULL argument");
  SG_REQUIRE(g->n > 0, SG_ERR_INVALID, "graph has no vertices");
  *out = nullptr;
  sg_cc_handle c = new sg_cc_s();
  c->g = g;
  c->stream = g->stream;
  sg_status st = c->ws.alloc(g->n);
  if (st == SG_OK) st = dev_alloc(&c->labels, g->n);
  if (st != SG_OK) {
    sg_cc_destroy(c);
    return st;
  }
  *out = c;
  return SG_OK;
}

sg_status sg_cc_set_method(sg_cc_handle c, int method) {
  clear_error();
  SG_REQUIRE(c, SG_ERR_INVALID, "cc is NULL");
  SG_REQUIRE(method == SG_CC_AUTO || method == SG_CC_PROPAGATION || method == SG_CC_UNION_FIND, SG_ERR_INVALID,
             "unknown CC method");
  SG_REQUIRE(method != SG_CC_UNION_FIND || !(c->g->flags & SG_GRAPH_DIRECTED), SG_ERR_UNSUPPORTED,
             "union-find components need an undirected graph");
  c->method = method;
  return SG_OK;
}

sg_status sg_cc_run_async(sg_cc_handle c) {
  clear_error();
  SG_REQUIRE(c, SG_ERR_INVALID, "cc is NULL");
  const sg_graph g = c->g;
  c->used_union_find = c->method == SG_CC_UNION_FIND || (c->method == SG_CC_AUTO && !(g->flags & SG_GRAPH_DIRECTED));
  if (c->used_union_find) {
    const unsigned vgrid = grid_for(g->n, 256, 8);
    // scratch from the push workspace, idle on this path: the giant root in
    // the first queue's first word, the per-root largest ids in the second
    uint32_t *giant = c->ws.q.small, *top = c->ws.q.big;
    uf_init_kernel<<<vgrid, 256, 0, c->stream>>>(c->labels, top, g->n);
    for (uint32_t r = 0; r < kSampled; r++)
      uf_sample_kernel<<<vgrid, 256, 0, c->stream>>>(g->fwd.ro, g->fwd.col, g->n, r, c->labels);
    uf_flatten_kernel<<<vgrid, 256, 0, c->stream>>>(c->labels, g->n);
    uf_giant_kernel<<<1, kGiantSamples, 0, c->stream>>>(c->labels, g->n, giant);
    uf_rest_kernel<<<vgrid, 256, 0, c->stream>>>(g->fwd.ro, g->fwd.col, g->n, giant, c->labels);
    uf_flatten_kernel<<<vgrid, 256, 0, c->stream>>>(c->labels, g->n);
    uf_top_kernel<<<vgrid, 256, 0, c->stream>>>(c->labels, top, g->n, giant);
    uf_label_kernel<<<vgrid, 256, 0, c->stream>>>(c->labels, top, g->n);
    SG_CUDA(cudaGetLastError());
    count_launch(6 + kSampled);
  } else {
    SG_CUDA(cudaMemsetAsync(c->ws.bar, 0, sizeof(GridBarrier), c->stream));
    CcParams P{c->ws.loop(g), c->labels, c->ws.result};
    SG_TRY(launch_persistent(cc_kernel, P, 2, c->stream));
  }
  c->ran = true;
  return SG_OK;
}

sg_status sg_cc_run(sg_cc_handle c, uint64_t* iterations) {
  SG_TRY(sg_cc_run_async(c));
  if (c->used_union_find) {
    SG_CUDA(cudaStreamSynchronize(c->stream));
    if (iterations) *iterations = 1;  // one pass over the edges (most skipped)
    return SG_OK;
  }
  return c->ws.finish(c->stream, iterations);
}

sg_status sg_cc_get_labels(sg_cc_handle c, uint32_t* host_labels) {
  clear_error();
  SG_REQUIRE(c && host_labels, SG_ERR_INVALID, "NULL argument");
  SG_REQUIRE(c->ran, SG_ERR_NOT_INITIALIZED, "CC not run");
  SG_CUDA(cudaMemcpyAsync(host_labels, c->labels, sizeof(uint32_t) * c->g->n, cudaMemcpyDeviceToHost, c->stream));
  SG_CUDA(cudaStreamSynchronize(c->stream));
  return SG_OK;
}

sg_status sg_cc_labels_device(sg_cc_handle c, const uint32_t** dev_labels) {
  clear_error();
  SG_REQUIRE(c && dev_labels, SG_ERR_INVALID, "NULL argument");
  *dev_labels = c->labels;
  return SG_OK;
}

sg_status sg_cc(sg_graph g, uint32_t* host_labels, uint64_t* iterations) {
  sg_cc_handle c = nullptr;
  SG_TRY(sg_cc_create(g, &c));
  sg_status st = sg_cc_run(c, iterations);
  if (st == SG_OK && host_labels) st = sg_cc_get_labels(c, host_labels);
  sg_cc_destroy(c);
  return st;
}

}  // extern "C"
