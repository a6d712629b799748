// Push-only level loop shared by the SSSP, CC and BC-forward engines: per
// level, compact the frontier bitmap into degree-bucketed queues, barrier,
// expand with a visitor that relaxes each edge, barrier, stop when no vertex
// joined the next frontier.
#pragma once

#include "engine_common.cuh"

namespace sgb {
namespace eng {

struct PushLoop {
  uint32_t n, w0;
  const uint32_t* ro;
  const uint32_t* col;
  uint32_t* fb;  // 3 * w0 rotating frontier bitmaps; fb[0] holds F_0 on entry
  Queues q;
  Counters* cnt;  // 3, zeroed before entry
  GridBarrier* bar;
  sg_level_record* log = nullptr;  // optional per-level log, entry log_base + level
  uint32_t log_base = 0;
};

// Marks u in the next frontier bitmap; counts it when this call set the bit.
struct NextFrontier {
  uint32_t* fb_next;
  uint32_t n_new = 0;
  __device__ __forceinline__ void mark(uint32_t u) {
    const uint32_t b = 1u << (u & 31);
    if (!(atomicOr(fb_next + (u >> 5), b) & b)) n_new++;
  }
};

// make(level, fb_next) returns a visitor with src / visit / mark and an
// n_new counter.  Returns the number of levels, or 0 when a barrier timed out.
template <class MakeVisitor>
__device__ __forceinline__ uint32_t push_levels(const PushLoop& S, MakeVisitor make, uint32_t* s_scan,
                                                unsigned long long* s_red) {
  const uint32_t gtid = blockIdx.x * blockDim.x + threadIdx.x;
  const uint32_t nthreads = gridDim.x * blockDim.x;
  for (uint32_t level = 0;; level++) {
    Counters* C = S.cnt + (level % 3);
    uint32_t* fb_cur = S.fb + (size_t)(level % 3) * S.w0;
    uint32_t* fb_next = S.fb + (size_t)((level + 1) % 3) * S.w0;
    uint32_t* fb_zero = S.fb + (size_t)((level + 2) % 3) * S.w0;
    if (gtid == 0) {
      Counters z = {};
      S.cnt[(level + 1) % 3] = z;
    }
    const uint64_t t0 = (S.log && gtid == 0) ? sygraph::detail::global_timer_ns() : 0;
    compact_frontier(fb_cur, S.w0, S.ro, C, S.q, s_scan);
    if (!grid_sync(S.bar)) return 0;
    const uint32_t ns = ld_cg(&C->small_tail);
    const unsigned long long bp = ld_cg(&C->big_packed);
    auto vis = make(level, fb_next);
    push_expand(S.ro, S.col, S.q, ns, (uint32_t)(bp >> 32), (uint32_t)bp, vis);
    for (uint32_t i = gtid; i < S.w0; i += nthreads) st_cg(fb_zero + i, 0u);
    const unsigned long long c = block_sum<unsigned long long>(vis.n_new, s_red);
    if (threadIdx.x == 0 && c) atomicAdd(&C->new_count, c);
    if (!grid_sync(S.bar)) return 0;
    if (S.log && gtid == 0 && S.log_base + level < kMaxLog) {
      sg_level_record r = {};
      r.level = S.log_base + level;
      r.frontier_size = ns + (uint32_t)(bp >> 32);
      r.frontier_degree = ld_cg(&C->frontier_deg);
      r.next_size = (uint32_t)ld_cg(&C->new_count);
      r.t_start_ns = t0;
      r.t_end_ns = sygraph::detail::global_timer_ns();
      S.log[S.log_base + level] = r;
    }
    if (ld_cg(&C->new_count) == 0) return level + 1;
  }
}

}  // namespace eng
}  // namespace sgb
