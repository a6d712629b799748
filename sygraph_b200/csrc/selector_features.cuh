// The twelve features the learned strategy selector reads at the end of a
// level, computed on the device the same way for training (the engines log
// them) and for inference, by the single-source BFS engine (bfs.cu) and the
// batched one (msbfs.cu).
#pragma once

#include <cstdint>

namespace sgb {
namespace eng {

// Per-launch constants of the features (reciprocals and logarithms of the
// graph's sizes), computed once so a level's features need no division by
// them.
struct FeatureConst {
  float inv_log_n, inv_n, inv_log_m, inv_m, inv_w0, inv_sw1, f9;
};

// The frontier about to be expanded.
struct FeatureInputs {
  double ns;     // frontier size (vertices)
  double nd;     // frontier degree sum
  double ud;     // unexplored degree (of the vertices not yet visited)
  double vis;    // visited vertices
  double prev;   // previous frontier size
  int cur_pull;  // direction of the level that produced this frontier
};

__device__ __forceinline__ FeatureConst feature_const(uint32_t n32, uint64_t m64, uint32_t w0, uint32_t w1) {
  const float n = (float)n32, m = (float)(m64 ? m64 : 1);
  return FeatureConst{1.f / log2f(1.f + n), 1.f / n, 1.f / log2f(1.f + m), 1.f / m, 1.f / (float)w0,
                      1.f / (32.f * (float)w1), log2f(1.f + m / n) / 8.f};
}

// Feature `lane` of a frontier, computed by lane `lane` < 12 of a full warp
// (every lane must call; lanes 12-31 get 0): log and linear frontier size and
// degree, unexplored-degree and unvisited fractions, the level-0 and summary
// bitmap occupancy a frontier of that size would have if spread at random,
// mean frontier degree, graph mean degree, current direction, frontier growth.
// Every lane evaluates one logarithm and one exponential of its own argument,
// so the twelve cost the latency of one of each.
__device__ __forceinline__ float feature_of_lane(uint32_t lane, uint32_t n, const FeatureConst& k,
                                                 const FeatureInputs& x) {
  const float ns = (float)x.ns, nd = (float)x.nd, prev = (float)x.prev;
  // logarithms: lanes 0 (frontier size), 2 (degree), 8 (mean degree), 11 (previous size)
  const float la = lane == 0 ? ns : lane == 2 ? nd : lane == 8 ? nd / fmaxf(1.f, ns) : prev;
  const float lg = log2f(1.f + la);
  const float lns = __shfl_sync(0xffffffffu, lg, 0);
  // expected occupancy of the frontier bitmap (lane 6) and of its summary
  // (lane 7) for a frontier of this size spread at random (the words are not
  // counted: that would make every bitmap atomic wait for its old value)
  const float occ = 1.f - expf(-ns * (lane == 6 ? k.inv_w0 : k.inv_sw1));
  // the lane's own feature, by selects (a branch per lane would serialise)
  float f = 0.f;
  f = lane == 0 ? lg * k.inv_log_n : f;
  f = lane == 1 ? ns * k.inv_n : f;
  f = lane == 2 ? lg * k.inv_log_m : f;
  f = lane == 3 ? nd * k.inv_m : f;
  f = lane == 4 ? (float)x.ud * k.inv_m : f;
  f = lane == 5 ? ((float)n - (float)x.vis) * k.inv_n : f;
  f = (lane == 6 || lane == 7) ? occ : f;
  f = lane == 8 ? lg / 16.f : f;
  f = lane == 9 ? k.f9 : f;
  f = lane == 10 ? (x.cur_pull ? 1.f : 0.f) : f;
  f = lane == 11 ? fminf(16.f, fmaxf(-16.f, lns - lg)) / 16.f : f;
  return f;
}

}  // namespace eng
}  // namespace sgb
