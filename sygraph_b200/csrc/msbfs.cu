// Batched multi-source BFS: up to 64 traversals of the same graph in one
// persistent cooperative kernel, bit-parallel (one uint64 word per vertex:
// bit s = source s).  Each traversal computes exactly the depths of
// BFS::run from its source (algorithms/bfs.hpp:153-238; depths are unique, so
// the result per source equals the single-source engine's).
//
// State: seen[v] (sources that reached v), frontier masks F[v] in three
// rotating buffers with an activity bitmap + summary for enumeration, and a
// "done" bitmap of vertices every source has reached.  Per level:
//   push: for every active v and edge (v,u): new = F[v] & ~seen[u];
//         atomicOr on seen[u] claims the bits, atomicOr on F'[u] publishes them
//   pull: every u not done ORs the frontier masks of its in-neighbours:
//         light u by a warp per word, each lane first probing a few
//         in-neighbours serially (stopping once every missing source is
//         covered), then the rest of the still-open lists walked
//         edge-parallel into per-owner shared slots (u owns seen[u]); heavy u
//         by static in-list chunks, each applied like a push relaxation
// No depth is stored during the traversal.  When F_{L-1} is cleared, each
// active vertex folds its mask into the depth bit-planes: plane b holds, per
// source bit, bit b of the vertex's depth, so v's planes get F_{L-1}[v] OR-ed
// into every plane b with bit b of L-1 set (one writer per vertex and level).
// After the last level one pass turns planes + seen into the source-major
// k x n depth array with full coalesced row stores (n+1 where a source never
// reached the vertex).  Plane b is zeroed at level 2^b, one level before its
// first fold.  One grid barrier per level.
#include <algorithm>
#include <cstring>
#include <vector>

#include "engine_common.cuh"
#include "selector_features.cuh"
#include "sygraph/detail/selector_mlp.cuh"

namespace sgb {
namespace ms {

using namespace eng;

constexpr uint32_t kHeavy = 256;
constexpr uint32_t kHeavyBuf = 1024;
constexpr uint32_t kPullHeavyIn = 256;  // in-degree from which a pulled vertex goes by chunks
constexpr uint32_t kPullChunkIn = 256;  // in-edges per chunk
constexpr uint32_t kPullProbe = 8;      // serial early-exit probes before the edge-parallel scan
using u64 = unsigned long long;

// Words of a pull level beyond each warp's first are handed out by
// kGrabDomains counters (warp w draws from counter w % kGrabDomains); the
// warps of a launch are a multiple of it (16 per CTA).
constexpr uint32_t kGrabDomains = 4;

struct LevelCounters {
  u64 heavy_packed;
  u64 new_count;     // vertices that became active
  u64 new_deg;       // their degree sum
  u64 reached_edges; // sum over (source, newly reached vertex) of the vertex degree
  u64 done_deg;      // degree of vertices every source reached at this level
  uint32_t grab[kGrabDomains];  // words handed out by each domain's counter
  u64 done_count;    // vertices every source reached at this level
};

// Each warp's first word is its own (word = its warp index); the later ones
// come from its domain's counter (word = nwarps + d + kGrabDomains * c), the
// next one requested before the current word is processed, so that warps
// that drew heavy words do not hold up the level's barrier.
template <class Fn>
__device__ __forceinline__ void for_each_word_balanced(uint32_t* grab, uint32_t w0, uint32_t gwarp, uint32_t nwarps,
                                                       Fn&& fn) {
  const uint32_t lane = threadIdx.x & 31u, d = gwarp % kGrabDomains;
  uint32_t* counter = grab + d;
  uint32_t nxt = lane == 0 ? atomicAdd(counter, 1u) : 0u;
  for (uint32_t wi = gwarp; wi < w0;) {
    fn(wi);
    wi = nwarps + d + kGrabDomains * __shfl_sync(0xffffffffu, nxt, 0);
    if (lane == 0) nxt = atomicAdd(counter, 1u);
  }
}

struct Params {
  uint32_t n, w0, w1, k;
  uint64_t m;
  const uint32_t* ro;
  const uint32_t* col;
  const uint32_t* iro;
  const uint32_t* icol;
  const uint32_t* sources;
  int mode;
  float alpha, beta;
  u64 all;
  u64* seen;
  u64* F;            // 3 * n
  uint32_t* fa;      // 3 * w0 activity bitmaps
  uint32_t* sm;      // 3 * w1 summaries
  uint32_t* done;    // w0
  const uint32_t* no_in_edges;
  uint32_t* heavy_v; // 2 * heavy_cap
  uint32_t* heavy_s;
  uint32_t heavy_cap;
  LevelCounters* cnt;
  GridBarrier* bar;
  const uint32_t* pull_chunk_v;    // in-degree >= kPullHeavyIn: (vertex, first edge) of each
  const uint32_t* pull_chunk_beg;  //   kPullChunkIn-edge chunk of its in-list, built at set-up
  uint32_t pull_chunks;
  u64* planes;       // n_planes * n: bit b of each (source, vertex) depth
  uint32_t n_planes;
  uint32_t* depth;   // k * n, source-major, written after the last level
  sg_level_record* log;
  u64* result;       // [iterations, push, pull, reached_edges]
  const int* schedule;    // optional direction per level: 0 push, 2 pull, -1 the mode decides
  uint32_t schedule_len;
  const sygraph::detail::MlpStaged* mlp_image;  // learned mode: the selector, staged per launch
  float margin;           // log-time gain the MLP must predict to overrule the heuristic
  float min_frontier;     // frontier sizes (fraction of n) the MLP is asked about
  float max_frontier;
  float* features;        // optional log: 12 floats per level decision
};

struct Shared {
  uint32_t scan[32];
  u64 red[32];
  u64 acc[kThreads];  // pull: per-warp OR accumulators of the word's 32 vertices
  uint32_t hv[kHeavyBuf];
  uint32_t hd[kHeavyBuf];
  uint32_t hn;
  uint32_t base_e, base_c;
  int choice;
  sygraph::detail::MlpStaged mlp;  // learned mode: parameters staged once per launch
  float mlp_scratch[sygraph::detail::kMlpHidden];
  eng::FeatureConst fk;
};

struct Level {
  const Params* P;
  Shared* S;
  LevelCounters* C;
  u64* F_next;
  uint32_t* fa_next;
  uint32_t* sm_next;
  uint32_t* hv_next;
  uint32_t* hs_next;
  uint32_t next_depth;
  uint32_t n_new = 0;
  u64 deg_new = 0, reached = 0, done_deg = 0, done_count = 0;

  __device__ __forceinline__ void add_heavy(uint32_t u, uint32_t du) {
    const uint32_t i = atomicAdd(&S->hn, 1u);
    if (i < kHeavyBuf) {
      S->hv[i] = u;
      S->hd[i] = du;
    } else {
      const u64 old = atomicAdd(&C->heavy_packed, (1ull << 32) | chunks_of(du));
      hv_next[old >> 32] = u;
      hs_next[old >> 32] = (uint32_t)old;
    }
  }
  // push: relax edge (v -> u) carrying frontier mask fv
  __device__ __forceinline__ void visit_push(uint32_t u, u64 fv) {
    const u64 su = ld_cg(P->seen + u);
    const u64 nb = fv & ~su;
    if (!nb) return;
    const u64 old = atomicOr(P->seen + u, nb);
    const u64 nw = nb & ~old;
    if (!nw) return;
    const uint32_t du = P->ro[u + 1] - P->ro[u];
    reached += (u64)__popcll(nw) * du;
    if ((old | nw) == P->all) {
      done_deg += du;
      done_count++;
      atomicOr(P->done + (u >> 5), 1u << (u & 31));
    }
    if (atomicOr(F_next + u, nw) == 0) {
      const uint32_t b = 1u << (u & 31);
      if (atomicOr(fa_next + (u >> 5), b) == 0) atomicOr(sm_next + (u >> 10), 1u << ((u >> 5) & 31));
      n_new++;
      deg_new += du;
      if (du >= kHeavy) add_heavy(u, du);
    }
  }
  // K edges (u[k] carrying mask fv[k]; bit k of `act` marks valid ones) at
  // once: the seen probes, then the claiming atomics with the row offsets,
  // then the frontier atomics of all K go out together
  template <int K>
  __device__ __forceinline__ void visit_push_n(const uint32_t (&u)[K], const u64 (&fv)[K], uint32_t act) {
    u64 nb[K];
#pragma unroll
    for (int k = 0; k < K; k++) nb[k] = ((act >> k) & 1u) ? fv[k] & ~ld_cg(P->seen + u[k]) : 0ull;
    u64 nw[K], old[K];
    uint32_t r0[K], r1[K];
#pragma unroll
    for (int k = 0; k < K; k++) {
      old[k] = 0;
      r0[k] = r1[k] = 0;
      if (nb[k]) {
        old[k] = atomicOr(P->seen + u[k], nb[k]);
        r0[k] = P->ro[u[k]];
        r1[k] = P->ro[u[k] + 1];
      }
    }
    u64 fo[K];
#pragma unroll
    for (int k = 0; k < K; k++) {
      nw[k] = nb[k] & ~old[k];
      fo[k] = nw[k] ? atomicOr(F_next + u[k], nw[k]) : ~0ull;
    }
#pragma unroll
    for (int k = 0; k < K; k++) {
      if (!nw[k]) continue;
      const uint32_t du = r1[k] - r0[k];
      reached += (u64)__popcll(nw[k]) * du;
      if ((old[k] | nw[k]) == P->all) {
        done_deg += du;
        done_count++;
        atomicOr(P->done + (u[k] >> 5), 1u << (u[k] & 31));
      }
      if (fo[k] == 0) {  // first sources to reach u this level: u joins the frontier
        atomicOr(fa_next + (u[k] >> 5), 1u << (u[k] & 31));
        atomicOr(sm_next + (u[k] >> 10), 1u << ((u[k] >> 5) & 31));
        n_new++;
        deg_new += du;
        if (du >= kHeavy) add_heavy(u[k], du);
      }
    }
  }
};

__device__ __forceinline__ u64 shfl64(u64 x, uint32_t src) {
  const uint32_t lo = __shfl_sync(kFullMask, (uint32_t)x, src);
  const uint32_t hi = __shfl_sync(kFullMask, (uint32_t)(x >> 32), src);
  return ((u64)hi << 32) | lo;
}

__device__ __forceinline__ void expand_group(Level& L, uint32_t beg, uint32_t deg, u64 fv) {
  const uint32_t lane = threadIdx.x & 31;
  const uint32_t incl = warp_inclusive_scan(deg);
  const uint32_t total = __shfl_sync(kFullMask, incl, 31);
  const uint32_t excl = incl - deg;
  for (uint32_t r0 = 0; r0 < total; r0 += 64) {
    uint32_t u[2], act = 0;
    u64 f[2];
#pragma unroll
    for (int k = 0; k < 2; k++) {
      const uint32_t r = r0 + k * 32 + lane;
      const bool a = r < total;
      const uint32_t o = warp_owner_of_rank(incl, a ? r : total - 1);
      const uint32_t ob = __shfl_sync(kFullMask, beg, o);
      const uint32_t oe = __shfl_sync(kFullMask, excl, o);
      f[k] = shfl64(fv, o);
      u[k] = a ? L.P->col[ob + (r - oe)] : 0u;
      act |= (uint32_t)a << k;
    }
    L.visit_push_n<2>(u, f, act);
  }
}

// Source-major depths of a warp's 32 consecutive vertices: bit b of depth(s, u)
// is bit s of plane b (planes below pb; F_last carries depth `last`); n+1
// where source s never reached u.  Every row store is a full 128-byte line.
template <int PB>
__device__ __forceinline__ void materialise(const Params& P, const u64* F_last, uint32_t last, uint32_t pb) {
  const uint32_t lane = threadIdx.x & 31;
  const uint32_t gwarp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const uint32_t nwarps = (gridDim.x * blockDim.x) >> 5;
  const uint32_t n = P.n;
  for (uint32_t wi = gwarp; wi < P.w0; wi += nwarps) {
    const uint32_t u = wi * 32 + lane;
    const bool in = u < n;
    const u64 sn = in ? ld_cg(P.seen + u) : 0ull;
    const u64 fl = in ? ld_cg(F_last + u) : 0ull;
    u64 pl[PB];
#pragma unroll
    for (int b = 0; b < PB; b++) {
      u64 x = (in && (uint32_t)b < pb) ? ld_cg(P.planes + (size_t)b * n + u) : 0ull;
      if ((last >> b) & 1u) x |= fl;
      pl[b] = x;
    }
    if (!in) continue;
    for (uint32_t s = 0; s < P.k; s++) {
      uint32_t d = 0;
#pragma unroll
      for (int b = 0; b < PB; b++) d |= (uint32_t)((pl[b] >> s) & 1ull) << b;
      __stcs(P.depth + (size_t)s * n + u, ((sn >> s) & 1ull) ? d : n + 1);
    }
  }
}

constexpr int kLearnedMode = SG_BFS_LEARNED;
constexpr uint32_t kMsAllowed = (1u << 0) | (1u << 2);  // the model's push/warp and pull/warp outputs

// Direction of level `level` (1 = pull), identical in every CTA (same inputs,
// same arithmetic): a forced direction from the schedule, else in learned
// mode the MLP's choice between push and pull where the heuristic would
// switch direction on a frontier inside [min_frontier, max_frontier] * n
// (warp 0 of each CTA; the heuristic's choice `h_pull` stands unless the
// model predicts it `margin` slower in log-time, and outside the trusted
// feature range), else the heuristic's.  Logs the features when asked.
__device__ __forceinline__ int ms_decide(const Params& P, Shared& S, int h_pull, const eng::FeatureInputs& x,
                                         uint32_t level) {
  const int forced = (P.schedule && level < P.schedule_len) ? P.schedule[level] : -1;
  const bool log = P.features && blockIdx.x == 0 && level < kMaxLog;
  const bool infer = forced < 0 && P.mode == kLearnedMode && P.mlp_image && (h_pull != 0) != (x.cur_pull != 0) &&
                     (float)x.ns >= P.min_frontier * (float)P.n && (float)x.ns <= P.max_frontier * (float)P.n;
  if (infer || log) {
    if (threadIdx.x < 32) {
      const float f = eng::feature_of_lane(threadIdx.x, P.n, S.fk, x);
      if (log && threadIdx.x < 12) P.features[(size_t)level * 12 + threadIdx.x] = f;
      if (infer) {
        const int c = sygraph::detail::mlp_choose(&S.mlp, f, kMsAllowed, S.mlp_scratch, h_pull ? 2 : 0, P.margin);
        if (threadIdx.x == 0) S.choice = c;
      }
    }
    __syncthreads();  // S.choice is written again only after the next grid barrier
  }
  if (forced >= 0) return forced >= 2;
  if (infer && S.choice >= 0) return S.choice >= 2;
  return h_pull;
}

__global__ void __launch_bounds__(kThreads, 2) msbfs_kernel(Params P) {
  __shared__ Shared S;
  const uint32_t gtid = blockIdx.x * blockDim.x + threadIdx.x;
  const uint32_t nthreads = gridDim.x * blockDim.x;
  const uint32_t lane = threadIdx.x & 31;
  const uint32_t gwarp = gtid >> 5, nwarps = nthreads >> 5;
  const uint32_t n = P.n, w0 = P.w0, w1 = P.w1;

  // learned mode: the staged MLP parameters arrive by asynchronous copies
  // while the state is cleared; the first barrier publishes them
  const bool learned = P.mode == kLearnedMode && P.mlp_image;
  if (learned) sygraph::detail::mlp_stage_async(P.mlp_image, &S.mlp);
  if (threadIdx.x == 0) S.fk = eng::feature_const(n, P.m, w0, w1);

  // ---- clear state
  for (uint32_t i = gtid; i < n; i += nthreads) {
    st_cg(P.seen + i, 0ull);
    st_cg(P.F + i, 0ull);
    st_cg(P.F + n + i, 0ull);
    st_cg(P.F + 2 * (size_t)n + i, 0ull);
  }
  for (uint32_t i = gtid; i < w0; i += nthreads) {
    st_cg(P.fa + i, 0u);
    st_cg(P.fa + w0 + i, 0u);
    st_cg(P.fa + 2 * w0 + i, 0u);
    st_cg(P.done + i, P.no_in_edges[i]);
  }
  for (uint32_t i = gtid; i < 3 * w1; i += nthreads) st_cg(P.sm + i, 0u);
  if (gtid < 3) {
    LevelCounters z = {};
    P.cnt[gtid] = z;
  }
  if (threadIdx.x == 0) S.hn = 0;
  if (learned) sygraph::detail::mlp_stage_wait();
  if (!grid_sync(P.bar)) return;
  // ---- sources: F_0, seen, depth 0, and the level-0 heavy list
  if (gtid == 0) {
    u64 cnt = 0, deg = 0;
    uint32_t hn = 0, hc = 0;
    for (uint32_t i = 0; i < P.k; i++) {
      const uint32_t s = P.sources[i];
      const u64 bit = 1ull << i;
      const u64 before = P.F[s];
      P.seen[s] |= bit;
      P.F[s] = before | bit;
      if (before == 0) {
        const uint32_t d = P.ro[s + 1] - P.ro[s];
        cnt++;
        deg += d;
        P.fa[s >> 5] |= 1u << (s & 31);
        P.sm[s >> 10] |= 1u << ((s >> 5) & 31);
        if (d >= kHeavy) {
          P.heavy_v[hn] = s;
          P.heavy_s[hn] = hc;
          hn++;
          hc += chunks_of(d);
        }
      }
    }
    LevelCounters c0 = {};
    c0.heavy_packed = ((u64)hn << 32) | hc;
    c0.new_count = cnt;
    c0.new_deg = deg;
    P.cnt[2] = c0;
    __threadfence();
  }
  if (!grid_sync(P.bar)) return;

  u64 unexplored = P.m;
  u64 frontier_size = ld_cg(&P.cnt[2].new_count), frontier_deg = ld_cg(&P.cnt[2].new_deg);
  u64 reached_total = 0;
  for (uint32_t i = 0; i < P.k; i++) {
    const uint32_t s = P.sources[i];
    reached_total += P.ro[s + 1] - P.ro[s];
  }
  u64 n_push = 0, n_pull = 0;
  // vertices every source has reached (the sources themselves when k == 1)
  u64 done_total = P.k == 1 ? 1 : 0;
  int pull = P.mode == SG_BFS_PULL;
  {
    const eng::FeatureInputs x{(double)frontier_size, (double)frontier_deg, (double)unexplored, (double)done_total,
                               (double)frontier_size, 0};
    pull = ms_decide(P, S, pull, x, 0);
  }
  uint32_t level = 0;
  for (;; level++) {
    LevelCounters* C = P.cnt + (level % 3);
    const LevelCounters* Cprev = P.cnt + ((level + 2) % 3);
    const size_t cur = level % 3, nxt = (level + 1) % 3, zro = (level + 2) % 3;
    u64* F_cur = P.F + cur * n;
    u64* F_zero = P.F + zro * n;
    uint32_t* fa_cur = P.fa + cur * w0;
    uint32_t* fa_zero = P.fa + zro * w0;
    uint32_t* sm_cur = P.sm + cur * w1;
    uint32_t* sm_zero = P.sm + zro * w1;
    const uint32_t par = level & 1;
    if (gtid == 0) {
      LevelCounters z = {};
      P.cnt[nxt] = z;
    }
    const uint64_t t0 = gtid == 0 ? sygraph::detail::global_timer_ns() : 0;
    Level L{&P, &S, C, P.F + nxt * n, P.fa + nxt * w0, P.sm + nxt * w1,
            P.heavy_v + (size_t)(par ^ 1) * P.heavy_cap, P.heavy_s + (size_t)(par ^ 1) * P.heavy_cap, level + 1};
    if (!pull) {
      n_push++;
      const u64 hp = ld_cg(&Cprev->heavy_packed);
      const uint32_t n_heavy = (uint32_t)(hp >> 32), n_chunks = (uint32_t)hp;
      const uint32_t* hv_cur = P.heavy_v + (size_t)par * P.heavy_cap;
      const uint32_t* hs_cur = P.heavy_s + (size_t)par * P.heavy_cap;
      const uint32_t units = w1 + n_chunks;
      for (uint32_t unit = gwarp; unit < units; unit += nwarps) {
        if (unit < w1) {
          const uint32_t s = ld_cg(sm_cur + unit);
          if (!s) continue;
          const uint32_t bits = ((s >> lane) & 1u) ? ld_cg(fa_cur + unit * 32 + lane) : 0u;
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
            u64 fv = 0;
            if (act) {
              const uint32_t v = (unit * 32 + o) * 32 + select_bit(ob, r - oe);
              beg = P.ro[v];
              deg = P.ro[v + 1] - beg;
              fv = F_cur[v];  // read-only until the next barrier: L1-cached
              if (deg >= kHeavy) deg = 0;
            }
            expand_group(L, beg, deg, fv);
          }
        } else {
          const uint32_t c = unit - w1;
          const uint32_t ent = warp_find_owner(hs_cur, n_heavy, c);
          const uint32_t v = ld_cg(hv_cur + ent);
          const uint32_t first = ld_cg(hs_cur + ent);
          const uint32_t cb = P.ro[v] + (c - first) * kChunk;
          const uint32_t ce = min(P.ro[v + 1], cb + kChunk);
          const u64 fv = F_cur[v];  // read-only until the next barrier: L1-cached
          const u64 f2[2] = {fv, fv};
          for (uint32_t eb = cb; eb < ce; eb += 64) {
            uint32_t u[2], act = 0;
#pragma unroll
            for (int k = 0; k < 2; k++) {
              const uint32_t e = eb + k * 32 + lane;
              u[k] = e < ce ? P.col[e] : 0u;
              act |= (uint32_t)(e < ce) << k;
            }
            L.visit_push_n<2>(u, f2, act);
          }
        }
      }
    } else {
      // pull: candidates OR the frontier masks of their in-neighbours.  Light
      // candidates: a warp per word, the word's in-lists walked edge-parallel
      // (coalesced column loads), masks OR-ed into the owner's shared slot;
      // the owner alone writes seen / F' of its vertex.  Heavy candidates: the
      // static chunk list, each chunk's OR applied like a push relaxation.
      n_pull++;
      const bool same = P.iro == P.ro;
      u64* acc_slot = S.acc + (threadIdx.x & ~31u);
      for_each_word_balanced(C->grab, w0, gwarp, nwarps, [&](uint32_t wi) {
        const uint32_t dw = ld_cg(P.done + wi);
        const uint32_t cand = ~dw & valid_bits(wi, w0, n);
        if (!cand) return;
        const uint32_t u = wi * 32 + lane;
        const bool mine = (cand >> lane) & 1u;
        const uint32_t beg = mine ? P.iro[u] : 0u;
        const uint32_t end = mine ? P.iro[u + 1] : 0u;
        const bool light = mine && end - beg < kPullHeavyIn;
        if (!__any_sync(kFullMask, light)) return;
        const u64 su = light ? ld_cg(P.seen + u) : P.all;
        // phase 1: a few serial probes; a vertex that every missing source
        // reaches through its first in-neighbours stops here
        u64 acc = 0;
        uint32_t e = beg;
        const uint32_t lim = light ? min(end, beg + kPullProbe) : beg;
        while (e < lim && (acc | su) != P.all) acc |= F_cur[P.icol[e++]];
        // phase 2: the rest of the still-open lists, edge-parallel into shared slots
        const bool open = light && (acc | su) != P.all && e < end;
        const uint32_t dg = open ? end - e : 0u;
        const uint32_t incl = warp_inclusive_scan(dg);
        const uint32_t total = __shfl_sync(kFullMask, incl, 31);
        if (total) {
          // kPullWin windows of 32 edges in flight: column loads, then mask
          // loads; each window's masks are OR-reduced per owner (a window's
          // lanes of one owner are one match group) and the group's first
          // lane adds the result to the owner's shared slot
          const uint32_t excl = incl - dg;
          acc_slot[lane] = acc;
          __syncwarp();
          for (uint32_t r0 = 0; r0 < total; r0 += 32 * kPullWin) {
            uint32_t c[kPullWin], own[kPullWin];
#pragma unroll
            for (int k = 0; k < kPullWin; k++) {
              const uint32_t r = r0 + k * 32 + lane;
              const bool act = r < total;
              const uint32_t o = warp_owner_of_rank(incl, act ? r : total - 1);
              const uint32_t ob = __shfl_sync(kFullMask, e, o);
              const uint32_t oe = __shfl_sync(kFullMask, excl, o);
              own[k] = act ? o : 32u;  // 32: no owner, a group of its own
              c[k] = act ? P.icol[ob + (r - oe)] : 0u;
            }
            u64 f[kPullWin];
#pragma unroll
            for (int k = 0; k < kPullWin; k++) f[k] = own[k] < 32 ? F_cur[c[k]] : 0ull;
#pragma unroll
            for (int k = 0; k < kPullWin; k++) {
              const uint32_t g = __match_any_sync(kFullMask, own[k]);
              const uint32_t lo = __reduce_or_sync(g, (uint32_t)f[k]);
              const uint32_t hi = __reduce_or_sync(g, (uint32_t)(f[k] >> 32));
              if (own[k] < 32 && lane == __ffs(g) - 1 && (lo | hi)) atomicOr(acc_slot + own[k], ((u64)hi << 32) | lo);
            }
          }
          __syncwarp();
          acc = acc_slot[lane];
          __syncwarp();
        }
        const u64 nw = light ? (acc & ~su) : 0ull;
        const bool got = light && nw != 0;
        const uint32_t du = got ? (same ? end - beg : P.ro[u + 1] - P.ro[u]) : 0u;
        if (got) {
          st_cg(P.seen + u, su | nw);
          st_cg(L.F_next + u, nw);
          L.n_new++;
          L.deg_new += du;
          L.reached += (u64)__popcll(nw) * du;
          if ((su | nw) == P.all) {
            L.done_deg += du;
            L.done_count++;
          }
          if (du >= kHeavy) L.add_heavy(u, du);
        }
        // heavy vertices of the same word update these words by atomics too
        const uint32_t gmask = __ballot_sync(kFullMask, got);
        const uint32_t dmask = __ballot_sync(kFullMask, got && (su | nw) == P.all);
        if (lane == 0) {
          if (gmask && atomicOr(L.fa_next + wi, gmask) == 0) atomicOr(L.sm_next + (wi >> 5), 1u << (wi & 31));
          if (dmask) atomicOr(P.done + wi, dmask);
        }
      });
      for (uint32_t c = gwarp; c < P.pull_chunks; c += nwarps) {
        const uint32_t v = P.pull_chunk_v[c];
        if (ld_cg(P.done + (v >> 5)) & (1u << (v & 31))) continue;
        const uint32_t cb = P.pull_chunk_beg[c];
        const uint32_t ce = min(P.iro[v + 1], cb + kPullChunkIn);
        u64 part = 0;
        for (uint32_t e = cb + lane; e < ce; e += 32) part |= F_cur[P.icol[e]];
#pragma unroll
        for (int d = 16; d > 0; d >>= 1) part |= shfl64(part, lane ^ d);
        if (lane == 0 && part) L.visit_push(v, part);
      }
    }
    // plane b is first folded at level 2^b + 1: zero it now
    if (level && !(level & (level - 1))) {
      u64* pz = P.planes + (size_t)(__ffs(level) - 1) * n;
      for (uint32_t i = gtid; i < n; i += nthreads) st_cg(pz + i, 0ull);
    }
    // fold F_{L-1} (depth L-1) into the planes and clear it, one fa word per warp step
    if (level) {
      const uint32_t dprev = level - 1;
      for (uint32_t j = gwarp; j < w1; j += nwarps) {
        const uint32_t s = ld_cg(sm_zero + j);
        if (!s) continue;
        for (uint32_t x = s; x; x &= x - 1) {
          const uint32_t w = j * 32 + (__ffs(x) - 1);
          const uint32_t word = ld_cg(fa_zero + w);
          if ((word >> lane) & 1u) {
            const uint32_t v = w * 32 + lane;
            const u64 f = ld_cg(F_zero + v);
            uint32_t b = 0;
            for (uint32_t d = dprev; d; d >>= 1, b++)
              if (d & 1u) {
                u64* p = P.planes + (size_t)b * n + v;
                st_cg(p, ld_cg(p) | f);
              }
            st_cg(F_zero + v, 0ull);
          }
        }
        __syncwarp();
        if ((s >> lane) & 1u) st_cg(fa_zero + j * 32 + lane, 0u);
        if (lane == 0) st_cg(sm_zero + j, 0u);
      }
    }
    __syncthreads();
    if (const uint32_t nb = min(S.hn, kHeavyBuf)) {  // block-uniform; most levels stage none
      const uint32_t k0 = 2 * threadIdx.x;
      uint32_t my = 0;
      if (k0 < nb) my += chunks_of(S.hd[k0]);
      if (k0 + 1 < nb) my += chunks_of(S.hd[k0 + 1]);
      uint32_t total;
      const uint32_t ex = sygraph::detail::block_excl_scan(my, &total, S.scan);
      if (threadIdx.x == 0 && nb) {
        const u64 old = atomicAdd(&C->heavy_packed, ((u64)nb << 32) | total);
        S.base_e = (uint32_t)(old >> 32);
        S.base_c = (uint32_t)old;
      }
      __syncthreads();
      if (nb) {
        uint32_t pc = S.base_c + ex;
        for (uint32_t k = k0; k < k0 + 2 && k < nb; k++) {
          L.hv_next[S.base_e + k] = S.hv[k];
          L.hs_next[S.base_e + k] = pc;
          pc += chunks_of(S.hd[k]);
        }
      }
      if (threadIdx.x == 0) S.hn = 0;
    }
    {
      const u64 c = block_sum<u64>(L.n_new, S.red);
      const u64 d = block_sum<u64>(L.deg_new, S.red);
      const u64 r = block_sum<u64>(L.reached, S.red);
      const u64 dd = block_sum<u64>(L.done_deg, S.red);
      const u64 dc = block_sum<u64>(L.done_count, S.red);
      if (threadIdx.x == 0) {
        if (c) atomicAdd(&C->new_count, c);
        if (d) atomicAdd(&C->new_deg, d);
        if (r) atomicAdd(&C->reached_edges, r);
        if (dd) atomicAdd(&C->done_deg, dd);
        if (dc) atomicAdd(&C->done_count, dc);
      }
    }
    if (!grid_sync(P.bar)) return;
    const u64 next_size = ld_cg(&C->new_count);
    const u64 next_deg = ld_cg(&C->new_deg);
    reached_total += ld_cg(&C->reached_edges);
    unexplored -= ld_cg(&C->done_deg);
    done_total += ld_cg(&C->done_count);
    if (gtid == 0 && level < kMaxLog) {
      sg_level_record rr;
      rr.level = level;
      rr.strategy = pull ? 2u : 0u;
      rr.frontier_size = (uint32_t)frontier_size;
      rr.next_size = (uint32_t)next_size;
      rr.frontier_degree = frontier_deg;
      rr.next_degree = next_deg;
      rr.unexplored_degree = unexplored;
      rr.t_start_ns = t0;
      rr.t_end_ns = sygraph::detail::global_timer_ns();
      P.log[level] = rr;
    }
    if (next_size == 0) break;
    int h_pull = pull;
    if (P.mode == SG_BFS_HYBRID || P.mode == kLearnedMode) {
      if (!pull) {
        if ((float)next_deg > (float)unexplored / P.alpha) h_pull = 1;
      } else {
        if ((float)next_size < (float)n / P.beta) h_pull = 0;
      }
    }
    const eng::FeatureInputs x{(double)next_size, (double)next_deg, (double)unexplored, (double)done_total,
                               (double)frontier_size, pull};
    pull = ms_decide(P, S, h_pull, x, level + 1);
    frontier_size = next_size;
    frontier_deg = next_deg;
  }
  // depths from the planes; F of the last level (depth `level`) is folded in registers
  {
    const uint32_t pb = level ? 32 - __clz(level) : 0;
    const u64* F_last = P.F + (size_t)(level % 3) * n;
    if (pb <= 4)
      materialise<4>(P, F_last, level, pb);
    else if (pb <= 8)
      materialise<8>(P, F_last, level, pb);
    else if (pb <= 16)
      materialise<16>(P, F_last, level, pb);
    else
      materialise<32>(P, F_last, level, pb);
  }
  if (gtid == 0) {
    P.result[0] = level + 1;
    P.result[1] = n_push;
    P.result[2] = n_pull;
    P.result[3] = reached_total;
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

}  // namespace ms
}  // namespace sgb

using namespace sgb;

struct sg_msbfs_s {
  sg_graph g = nullptr;
  cudaStream_t stream = nullptr;
  uint32_t max_ctas = 0;
  uint32_t k = 0, w0 = 0, w1 = 0, heavy_cap = 0;
  unsigned long long* seen = nullptr;
  unsigned long long* F = nullptr;
  uint32_t *fa = nullptr, *sm = nullptr, *done = nullptr, *no_in = nullptr;
  uint32_t *heavy_v = nullptr, *heavy_s = nullptr;
  uint32_t* sources = nullptr;
  unsigned long long* planes = nullptr;
  uint32_t n_planes = 0;
  uint32_t *pull_chunk_v = nullptr, *pull_chunk_beg = nullptr;
  uint32_t pull_chunks = 0;
  uint32_t* depth = nullptr;
  ms::LevelCounters* cnt = nullptr;
  sygraph::detail::GridBarrier* bar = nullptr;
  sg_level_record* log = nullptr;
  unsigned long long* result = nullptr;
  uint32_t last_k = 0;
  int* schedule = nullptr;  // forced direction per level (device)
  uint32_t schedule_len = 0;
  const void* mlp_image = nullptr;  // the selector's staged image (owned by the sg_mlp)
  float margin = 0.05f, min_frontier = 0.f, max_frontier = 1.f;
  float* features = nullptr;  // feature log, 12 floats per level
};

static void msbfs_release(sg_msbfs h) {
  if (!h) return;
  dev_free(h->seen);
  dev_free(h->F);
  dev_free(h->fa);
  dev_free(h->sm);
  dev_free(h->done);
  dev_free(h->no_in);
  dev_free(h->heavy_v);
  dev_free(h->heavy_s);
  dev_free(h->sources);
  dev_free(h->planes);
  dev_free(h->pull_chunk_v);
  dev_free(h->pull_chunk_beg);
  dev_free(h->depth);
  dev_free(h->cnt);
  dev_free(h->bar);
  dev_free(h->log);
  dev_free(h->result);
  dev_free(h->schedule);
  dev_free(h->features);
  delete h;
}

extern "C" {

sg_status sg_msbfs_create(sg_graph g, uint32_t max_sources, sg_msbfs* out) {
  clear_error();
  SG_REQUIRE(g && out, SG_ERR_INVALID, "NULL argument");
  SG_REQUIRE(max_sources >= 1 && max_sources <= 64, SG_ERR_INVALID, "a batch holds 1 to 64 sources");
  SG_REQUIRE(g->n > 0, SG_ERR_INVALID, "graph has no vertices");
  *out = nullptr;
  sg_msbfs h = new sg_msbfs_s();
  h->g = g;
  h->stream = g->stream;
  h->k = max_sources;
  h->w0 = div_up(g->n, 32);
  h->w1 = div_up(h->w0, 32);
  h->heavy_cap = (uint32_t)std::min<uint64_t>(g->n, g->m / ms::kHeavy + 1);
  const uint64_t n = g->n;
  // depths are below n: planes for the bits of n - 1 (at least one)
  h->n_planes = 1;
  while (h->n_planes < 32 && (n - 1) >> h->n_planes) h->n_planes++;
  sg_status s;
  if ((s = dev_alloc(&h->planes, (uint64_t)h->n_planes * n)) || (s = dev_alloc(&h->seen, n)) || (s = dev_alloc(&h->F, 3 * n)) || (s = dev_alloc(&h->fa, 3ull * h->w0)) ||
      (s = dev_alloc(&h->sm, 3ull * h->w1)) || (s = dev_alloc(&h->done, h->w0)) || (s = dev_alloc(&h->no_in, h->w0)) ||
      (s = dev_alloc(&h->heavy_v, 2ull * h->heavy_cap)) || (s = dev_alloc(&h->heavy_s, 2ull * h->heavy_cap)) ||
      (s = dev_alloc(&h->sources, 64)) || (s = dev_alloc(&h->depth, (uint64_t)max_sources * n)) ||
      (s = dev_alloc(&h->cnt, 3)) || (s = dev_alloc(&h->bar, 1)) || (s = dev_alloc(&h->log, SG_MAX_LOGGED_LEVELS)) ||
      (s = dev_alloc(&h->result, 8))) {
    msbfs_release(h);
    return s;
  }
  {
    // static chunk list of the in-lists pulled by chunks (in-degree >= kPullHeavyIn)
    std::vector<uint32_t> iro((size_t)g->n + 1), cv, cb;
    if (cudaMemcpy(iro.data(), g->inv.ro, sizeof(uint32_t) * iro.size(), cudaMemcpyDeviceToHost) != cudaSuccess) {
      cudaGetLastError();
      msbfs_release(h);
      return fail(SG_ERR_CUDA, "multi-source BFS set-up: reading the in-edge offsets failed");
    }
    for (uint32_t v = 0; v < g->n; v++)
      if (iro[v + 1] - iro[v] >= ms::kPullHeavyIn)
        for (uint32_t e = iro[v]; e < iro[v + 1]; e += ms::kPullChunkIn) {
          cv.push_back(v);
          cb.push_back(e);
        }
    if (!cv.empty()) {
      if ((s = dev_alloc(&h->pull_chunk_v, cv.size())) || (s = dev_alloc(&h->pull_chunk_beg, cb.size()))) {
        msbfs_release(h);
        return s;
      }
      if (cudaMemcpy(h->pull_chunk_v, cv.data(), 4 * cv.size(), cudaMemcpyHostToDevice) != cudaSuccess ||
          cudaMemcpy(h->pull_chunk_beg, cb.data(), 4 * cb.size(), cudaMemcpyHostToDevice) != cudaSuccess) {
        cudaGetLastError();
        msbfs_release(h);
        return fail(SG_ERR_CUDA, "multi-source BFS set-up: uploading the chunk list failed");
      }
      h->pull_chunks = (uint32_t)cv.size();
    }
  }
  ms::no_in_edges_kernel<<<grid_for((uint64_t)h->w0 * 32, 256), 256, 0, g->stream>>>(g->inv.ro, g->n, h->w0, h->no_in);
  if (cudaGetLastError() != cudaSuccess) {
    msbfs_release(h);
    return fail(SG_ERR_CUDA, "multi-source BFS set-up kernel failed to launch");
  }
  count_launch();
  *out = h;
  return SG_OK;
}

sg_status sg_msbfs_destroy(sg_msbfs h) {
  if (h) {
    cudaStreamSynchronize(h->stream);
    msbfs_release(h);
  }
  return SG_OK;
}

sg_status sg_msbfs_run_async(sg_msbfs h, const uint32_t* host_sources, uint32_t k, int direction, float alpha,
                             float beta) {
  clear_error();
  SG_REQUIRE(h && host_sources, SG_ERR_INVALID, "NULL argument");
  SG_REQUIRE(k >= 1 && k <= h->k, SG_ERR_INVALID, "source count exceeds the batch capacity");
  SG_REQUIRE(direction >= SG_BFS_PUSH && direction <= SG_BFS_LEARNED, SG_ERR_INVALID, "unknown BFS direction");
  SG_REQUIRE(direction != SG_BFS_LEARNED || h->mlp_image, SG_ERR_INVALID,
             "learned mode needs a selector (sg_msbfs_set_selector)");
  for (uint32_t i = 0; i < k; i++) SG_REQUIRE(host_sources[i] < h->g->n, SG_ERR_INVALID, "source out of range");
  sg_graph g = h->g;
  SG_CUDA(cudaMemcpyAsync(h->sources, host_sources, sizeof(uint32_t) * k, cudaMemcpyHostToDevice, h->stream));
  SG_CUDA(cudaMemsetAsync(h->bar, 0, sizeof(*h->bar), h->stream));
  ms::Params P;
  P.n = g->n;
  P.w0 = h->w0;
  P.w1 = h->w1;
  P.k = k;
  P.m = g->m;
  P.ro = g->fwd.ro;
  P.col = g->fwd.col;
  P.iro = g->inv.ro;
  P.icol = g->inv.col;
  P.sources = h->sources;
  P.mode = direction;
  P.alpha = alpha;
  P.beta = beta;
  P.all = k == 64 ? ~0ull : ((1ull << k) - 1ull);
  P.seen = h->seen;
  P.F = h->F;
  P.fa = h->fa;
  P.sm = h->sm;
  P.done = h->done;
  P.no_in_edges = h->no_in;
  P.heavy_v = h->heavy_v;
  P.heavy_s = h->heavy_s;
  P.heavy_cap = h->heavy_cap;
  P.cnt = h->cnt;
  P.bar = h->bar;
  P.pull_chunk_v = h->pull_chunk_v;
  P.pull_chunk_beg = h->pull_chunk_beg;
  P.pull_chunks = h->pull_chunks;
  P.planes = h->planes;
  P.n_planes = h->n_planes;
  P.depth = h->depth;
  P.log = h->log;
  P.result = h->result;
  P.schedule = h->schedule;
  P.schedule_len = h->schedule_len;
  P.mlp_image = static_cast<const sygraph::detail::MlpStaged*>(h->mlp_image);
  P.margin = h->margin;
  P.min_frontier = h->min_frontier;
  P.max_frontier = h->max_frontier;
  P.features = h->features;
  h->last_k = k;
  return eng::launch_persistent(ms::msbfs_kernel, P, 2, h->stream, h->max_ctas);
}

sg_status sg_msbfs_run(sg_msbfs h, const uint32_t* host_sources, uint32_t k, int direction, float alpha, float beta,
                       sg_msbfs_details* details) {
  SG_TRY(sg_msbfs_run_async(h, host_sources, k, direction, alpha, beta));
  unsigned long long r[4];
  sygraph::detail::GridBarrier b;
  SG_CUDA(cudaMemcpyAsync(r, h->result, sizeof(r), cudaMemcpyDeviceToHost, h->stream));
  SG_CUDA(cudaMemcpyAsync(&b, h->bar, sizeof(b), cudaMemcpyDeviceToHost, h->stream));
  SG_CUDA(cudaStreamSynchronize(h->stream));
  if (b.error) return fail(SG_ERR_TIMEOUT, "multi-source BFS: a grid barrier wait ran out");
  if (details) {
    details->iterations = r[0];
    details->push_steps = r[1];
    details->pull_steps = r[2];
    details->reached_edges = r[3];
  }
  return SG_OK;
}

}  // extern "C"

sg_status sgb::msbfs_launch_status(sg_msbfs h) {
  uint32_t err = 0;
  SG_CUDA(cudaMemcpyAsync(&err, &h->bar->error, sizeof(err), cudaMemcpyDeviceToHost, h->stream));
  SG_CUDA(cudaStreamSynchronize(h->stream));
  return err ? fail(SG_ERR_TIMEOUT, "batched BFS: a grid barrier wait ran out") : SG_OK;
}

extern "C" {

sg_status sg_msbfs_set_launch(sg_msbfs h, void* stream, uint32_t max_ctas) {
  clear_error();
  SG_REQUIRE(h, SG_ERR_INVALID, "NULL argument");
  SG_CUDA(cudaStreamSynchronize(h->stream));
  h->stream = stream ? (cudaStream_t)stream : h->g->stream;
  h->max_ctas = max_ctas;
  return SG_OK;
}

sg_status sg_msbfs_get_depths(sg_msbfs h, uint32_t* host_depth) {
  SG_REQUIRE(h && host_depth, SG_ERR_INVALID, "NULL argument");
  SG_REQUIRE(h->last_k, SG_ERR_NOT_INITIALIZED, "no batch has run");
  SG_CUDA(cudaMemcpyAsync(host_depth, h->depth, sizeof(uint32_t) * (uint64_t)h->last_k * h->g->n,
                          cudaMemcpyDeviceToHost, h->stream));
  SG_CUDA(cudaStreamSynchronize(h->stream));
  return SG_OK;
}

sg_status sg_msbfs_level_records(sg_msbfs h, sg_level_record* host_records, uint32_t cap, uint32_t* count) {
  SG_REQUIRE(h && count, SG_ERR_INVALID, "NULL argument");
  SG_CUDA(cudaStreamSynchronize(h->stream));
  unsigned long long it = 0;
  if (h->last_k) SG_CUDA(cudaMemcpy(&it, h->result, sizeof(it), cudaMemcpyDeviceToHost));
  uint32_t k = (uint32_t)(it < SG_MAX_LOGGED_LEVELS ? it : SG_MAX_LOGGED_LEVELS);
  if (k > cap) k = cap;
  if (host_records && k) SG_CUDA(cudaMemcpy(host_records, h->log, sizeof(sg_level_record) * k, cudaMemcpyDeviceToHost));
  *count = k;
  return SG_OK;
}

sg_status sg_msbfs_depths_device(sg_msbfs h, const uint32_t** dev_depth) {
  SG_REQUIRE(h && dev_depth, SG_ERR_INVALID, "NULL argument");
  *dev_depth = h->depth;
  return SG_OK;
}

sg_status sg_msbfs_set_schedule(sg_msbfs h, const int* host_directions, uint32_t len) {
  clear_error();
  SG_REQUIRE(h, SG_ERR_INVALID, "NULL argument");
  SG_REQUIRE(len == 0 || host_directions, SG_ERR_INVALID, "directions is NULL");
  for (uint32_t i = 0; i < len; i++)
    SG_REQUIRE(host_directions[i] == -1 || host_directions[i] == 0 || host_directions[i] == 2, SG_ERR_INVALID,
               "batched directions are 0 (push), 2 (pull) or -1 (the mode decides)");
  SG_CUDA(cudaStreamSynchronize(h->stream));  // a queued launch may still read the old schedule
  dev_free(h->schedule);
  h->schedule_len = 0;
  if (len) {
    SG_TRY(dev_alloc(&h->schedule, len));
    SG_CUDA(cudaMemcpy(h->schedule, host_directions, sizeof(int) * len, cudaMemcpyHostToDevice));
    h->schedule_len = len;
  }
  return SG_OK;
}

sg_status sg_msbfs_set_selector(sg_msbfs h, sg_mlp mlp, float margin, float min_frontier, float max_frontier) {
  clear_error();
  SG_REQUIRE(h, SG_ERR_INVALID, "NULL argument");
  SG_REQUIRE(margin >= 0.f && min_frontier >= 0.f && min_frontier <= max_frontier, SG_ERR_INVALID,
             "margin >= 0 and 0 <= min_frontier <= max_frontier");
  h->mlp_image = mlp ? mlp_device_image(mlp) : nullptr;
  h->margin = margin;
  h->min_frontier = min_frontier;
  h->max_frontier = max_frontier;
  return SG_OK;
}

sg_status sg_msbfs_log_features(sg_msbfs h, int enable) {
  clear_error();
  SG_REQUIRE(h, SG_ERR_INVALID, "NULL argument");
  SG_CUDA(cudaStreamSynchronize(h->stream));
  if (enable && !h->features) SG_TRY(dev_alloc(&h->features, 12ull * SG_MAX_LOGGED_LEVELS));
  if (!enable) dev_free(h->features);
  return SG_OK;
}

sg_status sg_msbfs_level_features(sg_msbfs h, float* host_features, uint32_t cap_levels, uint32_t* count) {
  SG_REQUIRE(h && count, SG_ERR_INVALID, "NULL argument");
  SG_REQUIRE(h->features, SG_ERR_NOT_INITIALIZED, "feature logging is off (sg_msbfs_log_features)");
  SG_CUDA(cudaStreamSynchronize(h->stream));
  unsigned long long it = 0;
  if (h->last_k) SG_CUDA(cudaMemcpy(&it, h->result, sizeof(it), cudaMemcpyDeviceToHost));
  uint32_t k = (uint32_t)(it < SG_MAX_LOGGED_LEVELS ? it : SG_MAX_LOGGED_LEVELS);
  if (k > cap_levels) k = cap_levels;
  if (host_features && k)
    SG_CUDA(cudaMemcpy(host_features, h->features, sizeof(float) * 12 * k, cudaMemcpyDeviceToHost));
  *count = k;
  return SG_OK;
}

}  // extern "C"
