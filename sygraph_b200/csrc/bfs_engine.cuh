// State of the fused BFS engine (bfs.cu): parameters, per-level counters,
// shared memory, the per-thread level context, the twelve selector features
// and the per-level strategy decision.
//
// Strategies (one per level): 0 push/warp, 1 push/CTA, 2 pull/warp,
// 3 pull/CTA, 4 pull_all/warp, 5 pull_all/CTA.  Every strategy yields the
// same frontier sets (BFS levels are unique); only the schedule changes.
#pragma once

#include "engine_common.cuh"
#include "selector_features.cuh"
#include "sygraph/detail/selector_mlp.cuh"

namespace sgb {
namespace bfs {

using namespace eng;

constexpr uint32_t kHeavy = 256;      // degree from which a vertex is expanded in chunks by many warps
constexpr uint32_t kHeavyBuf = 1024;  // per-CTA staging of newly discovered heavy vertices
constexpr uint32_t kBfsChunk = 64;    // edges per heavy-vertex chunk (one warp, two steps)
constexpr int kLearned = 3;           // mode: the MLP picks each level's strategy
constexpr unsigned long long kDirectClaimDeg = 1u << 16;  // push frontier degree below which claims skip the pre-load
// Two 512-thread CTAs per SM, as the other engines: one 1024-thread CTA per SM
// halves the barrier arrivals but was within 1% on RMAT-22, and whole-SM CTAs
// cannot share SMs with the half-SM CTAs of concurrent launches (serving).
constexpr uint32_t kBfsThreads = 512;
// Short-circuit pull of the engine: 0 = candidates ranked across each warp
// (pull_ranked); 2 or 4 = the older form, that many bitmap words per warp step.
constexpr uint32_t kDefaultPullWords = 0;

__device__ __forceinline__ uint32_t bfs_chunks(uint32_t deg) { return (deg + kBfsChunk - 1) / kBfsChunk; }

struct LevelCounters {
  unsigned long long heavy_packed;  // (entries << 32) | chunks of the heavy list being built
  unsigned long long new_count;     // vertices that joined the next frontier
  unsigned long long new_deg;       // their forward degrees
  unsigned long long pad[5];
};

struct Params {
  uint32_t n, w0, w1;
  uint64_t m;
  const uint32_t* ro;  // forward CSR
  const uint32_t* col;
  const uint32_t* iro;  // inverse CSR (aliases forward when undirected)
  const uint32_t* icol;
  uint32_t source;
  int mode;  // SG_BFS_PUSH / PULL / HYBRID / kLearned
  float alpha, beta;
  uint32_t* depth;
  uint32_t* visited;
  const uint32_t* no_in_edges;  // bitmap of vertices no edge reaches: never candidates
  // first in-neighbour of every vertex with one (nullptr: read through the
  // in-edge offsets): the short-circuit pull's first probe without the
  // dependent offset load and the random column read
  const uint32_t* first_in;
  uint32_t* fb;                 // 3 * w0
  uint32_t* sm;                 // 3 * w1
  uint32_t* heavy_v;            // 2 * heavy_cap
  uint32_t* heavy_s;            // 2 * heavy_cap
  uint32_t heavy_cap;
  LevelCounters* cnt;  // 3
  GridBarrier* bar;
  sg_level_record* log;
  unsigned long long* result;  // [iterations, push, pull, visited_vertices, visited_edges]
  const int* schedule;         // optional strategy per level (0..5), -1 = the mode decides
  uint32_t schedule_len;
  const sygraph::detail::MlpParams* mlp;  // learned mode
  const sygraph::detail::MlpStaged* mlp_image;  // its staged image (copied to shared memory per launch)
  uint32_t allowed;                       // strategies the MLP may pick (bit mask)
  float margin;                           // log-time gain the MLP must predict to overrule the heuristic
  float min_frontier;                     // smallest frontier (fraction of n) the MLP is asked about
  float max_frontier;                     // largest frontier (fraction of n) the MLP is asked about
  unsigned long long pull_reverse;        // bit L: level L's pull probes in-neighbours from the back
  uint32_t pull_words;                    // short-circuit pull: 0 ranked candidates, or 2 / 4 words per warp step
  float* features;                        // optional log: 12 floats per level decision
};

struct Shared {
  uint32_t pull_found[kBfsThreads / 32][32];  // ranked pull: hits per owned word, per warp
  uint32_t scan[32];
  unsigned long long red[32][4];
  unsigned long long acc[2];  // per-level totals of the CTA (new vertices, their degree)
  uint32_t hv[kHeavyBuf];
  uint32_t hd[kHeavyBuf];
  uint32_t hn;
  uint32_t base_e, base_c;
  uint32_t beg[kBfsThreads];
  uint32_t incl[kBfsThreads];
  uint32_t flag[kBfsThreads];
  int choice;
  sygraph::detail::MlpStaged mlp;  // learned mode: parameters staged once per launch
  float mlp_scratch[sygraph::detail::kMlpHidden];
  FeatureConst fk;  // set once per launch
};

// Per-thread context of one level's expansion.
struct Level {
  const Params* P;
  Shared* S;
  LevelCounters* C;
  uint32_t* fb_next;
  uint32_t* sm_next;
  uint32_t* hv_next;
  uint32_t* hs_next;
  uint32_t next_depth;
  // claim without the plain pre-load (small frontiers: their neighbours are
  // mostly unvisited, and the load would add a round trip to each discovery)
  bool direct_claim;
  uint32_t n_new = 0;
  unsigned long long deg_new = 0;

  __device__ __forceinline__ void add_heavy(uint32_t u, uint32_t du) {
    const uint32_t i = atomicAdd(&S->hn, 1u);
    if (i < kHeavyBuf) {
      S->hv[i] = u;
      S->hd[i] = du;
    } else {
      const unsigned long long old = atomicAdd(&C->heavy_packed, (1ull << 32) | bfs_chunks(du));
      hv_next[old >> 32] = u;
      hs_next[old >> 32] = (uint32_t)old;
    }
  }
  // u was discovered at this level (forward degree du); its frontier bit is set by the caller.
  __device__ __forceinline__ void discovered(uint32_t u, uint32_t du) {
    st_cg(P->depth + u, next_depth);
    n_new++;
    deg_new += du;
    if (du >= kHeavy) add_heavy(u, du);
  }
  // push: claim u through the visited bitmap (on large frontiers a plain
  // load first skips the atomic when u is visibly visited); u's row offsets
  // are loaded together
  // with the claiming atomic, so a discovery waits one round trip, not two
  __device__ __forceinline__ void visit_push(uint32_t u) {
    const uint32_t bit = 1u << (u & 31);
    uint32_t* vword = P->visited + (u >> 5);
    if (!direct_claim && (ld_cg(vword) & bit)) return;
    const uint32_t old = atomicOr(vword, bit);
    const uint32_t r0 = P->ro[u], r1 = P->ro[u + 1];
    if (old & bit) return;
    const uint32_t du = r1 - r0;
    atomicOr(fb_next + (u >> 5), 1u << (u & 31));  // results unused: fire-and-forget reductions
    atomicOr(sm_next + (u >> 10), 1u << ((u >> 5) & 31));
    discovered(u, du);
  }
  // push of K candidate targets at once (bit k of `act`: u[k] is valid): the
  // pre-loads, then the claiming atomics with the row offsets, of all K go
  // out together, so K edges cost the round trips of one
  template <int K>
  __device__ __forceinline__ void visit_push_n(const uint32_t (&u)[K], uint32_t act) {
    if (!direct_claim) {
      uint32_t w[K];
#pragma unroll
      for (int k = 0; k < K; k++) w[k] = ((act >> k) & 1u) ? ld_cg(P->visited + (u[k] >> 5)) : 0u;
#pragma unroll
      for (int k = 0; k < K; k++)
        if ((w[k] >> (u[k] & 31)) & 1u) act &= ~(1u << k);
    }
    uint32_t old[K], r0[K], r1[K];
#pragma unroll
    for (int k = 0; k < K; k++) {
      old[k] = 0xffffffffu;
      r0[k] = r1[k] = 0;
      if ((act >> k) & 1u) {
        old[k] = atomicOr(P->visited + (u[k] >> 5), 1u << (u[k] & 31));
        r0[k] = P->ro[u[k]];
        r1[k] = P->ro[u[k] + 1];
      }
    }
#pragma unroll
    for (int k = 0; k < K; k++) {
      if ((old[k] >> (u[k] & 31)) & 1u) continue;
      atomicOr(fb_next + (u[k] >> 5), 1u << (u[k] & 31));
      atomicOr(sm_next + (u[k] >> 10), 1u << ((u[k] >> 5) & 31));
      discovered(u[k], r1[k] - r0[k]);
    }
  }
  // pull: a warp publishes the vertices of word wi it found (lane 0 calls)
  __device__ __forceinline__ void publish_word(uint32_t wi, uint32_t vw, uint32_t fmask) {
    st_cg(P->visited + wi, vw | fmask);
    st_cg(fb_next + wi, fmask);
    atomicOr(sm_next + (wi >> 5), 1u << (wi & 31));
  }
};

// Sums four per-thread values over the block; the totals are valid in thread 0.
__device__ __forceinline__ void block_sum4(unsigned long long v[4], Shared& S) {
  const uint32_t lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
#pragma unroll
  for (int k = 0; k < 4; k++) {
    v[k] = sygraph::detail::warp_sum(v[k]);
    if (lane == 0) S.red[warp][k] = v[k];
  }
  __syncthreads();
  if (warp == 0) {
#pragma unroll
    for (int k = 0; k < 4; k++) {
      unsigned long long t = lane < nw ? S.red[lane][k] : 0ull;
      v[k] = sygraph::detail::warp_sum(t);
    }
  }
  __syncthreads();
}

// Strategy of the next level, identical in every CTA (same inputs, same
// arithmetic).  Heuristic: BFS::evaluateHeuristic (bfs.hpp:325-350), with the
// reference's float arithmetic; the learned mode asks the MLP (warp 0) and
// falls back to the heuristic outside the trusted feature range.
__device__ __forceinline__ int decide(const Params& P, Shared& S, int cur, const FeatureInputs& x, uint32_t level,
                                      float next_deg_f, float unexplored_f, unsigned long long next_size) {
  const bool cur_pull = cur >= 2;
  bool pull = cur_pull;
  if (P.mode == SG_BFS_HYBRID || P.mode == kLearned) {
    if (!cur_pull) {
      if (next_deg_f > unexplored_f / P.alpha) pull = true;
    } else {
      if ((float)next_size < (float)P.n / P.beta) pull = false;
    }
  }
  int h = P.mode == SG_BFS_PUSH ? 0 : P.mode == SG_BFS_PULL ? 2 : (pull ? 2 : 0);
  const bool log = P.features && blockIdx.x == 0 && level < kMaxLog;
  // The model is asked where the heuristic would switch direction, on a
  // frontier inside [min_frontier, max_frontier] * n, and wherever the
  // heuristic's choice is not allowed.  An inference is a latency of about a
  // microsecond on the critical path between two levels; away from the
  // switch points the model rarely overrules the heuristic, and the
  // frontier range is the one where, on the training tables, its choices
  // saved more than its inferences cost.
  const bool infer = P.mode == kLearned && P.mlp &&
                     ((((h >= 2) != cur_pull) && (float)x.ns >= P.min_frontier * (float)P.n &&
                       (float)x.ns <= P.max_frontier * (float)P.n) ||
                      !((P.allowed >> h) & 1u));
  if (infer || log) {
    if (threadIdx.x < 32) {
      const float f = feature_of_lane(threadIdx.x, P.n, S.fk, x);
      if (log && threadIdx.x < 12) P.features[(size_t)level * 12 + threadIdx.x] = f;
      if (infer) {
        const int c = sygraph::detail::mlp_choose(&S.mlp, f, P.allowed, S.mlp_scratch, h, P.margin);
        if (threadIdx.x == 0) S.choice = c;
      }
    }
    __syncthreads();  // S.choice is written again only after the next grid barrier
    if (infer && S.choice >= 0) h = S.choice;
  }
  return h;
}

}  // namespace bfs
}  // namespace sgb
