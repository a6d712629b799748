// Built-in device functors for the C ABI's sg_advance / filter / compute.
// Each restates one functor of the reference (file:line in the comments).
#pragma once

#include "internal.cuh"
#include "sygraph/detail/advance_kernels.cuh"

namespace sgb {
namespace ops {

using sygraph::detail::ld_cg;
using sygraph::detail::st_cg;

// algorithms/bfs.hpp:185-191
struct BfsPush {
  uint32_t* depth;
  uint32_t sentinel, iter;
  template <typename W>
  __device__ bool operator()(uint32_t, uint32_t dst, uint32_t, W) const {
    if (ld_cg(depth + dst) == sentinel) {
      st_cg(depth + dst, iter + 1);
      return true;
    }
    return false;
  }
};

// algorithms/bfs.hpp:201-207 (src = candidate, dst = in-frontier neighbour)
struct BfsPull {
  uint32_t* depth;
  uint32_t sentinel, iter;
  template <typename W>
  __device__ bool operator()(uint32_t src, uint32_t dst, uint32_t, W) const {
    if (ld_cg(depth + src) == sentinel && ld_cg(depth + dst) == iter) {
      st_cg(depth + src, iter + 1);
      return true;
    }
    return false;
  }
};

// algorithms/sssp.hpp:180-189: nd = d[src] + w; old = fetch_min(d[dst], nd); return nd < old
template <typename W>
struct SsspRelax {
  W* dist;
  __device__ bool operator()(uint32_t src, uint32_t dst, uint32_t, W w) const {
    const W nd = ld_cg(dist + src) + w;
    const W old = sygraph::detail::atomic_min_nonneg(dist + dst, nd);
    return nd < old;
  }
};

// algorithms/cc.hpp:137-142 ("if dst_label < src_label store src_label"), as an atomic max
struct CcMax {
  uint32_t* labels;
  template <typename W>
  __device__ bool operator()(uint32_t src, uint32_t dst, uint32_t, W) const {
    const uint32_t sl = ld_cg(labels + src);
    if (ld_cg(labels + dst) >= sl) return false;
    return atomicMax(labels + dst, sl) < sl;
  }
};

// algorithms/bc.hpp:144-153
struct BcForward {
  uint32_t* labels;
  float* sigma;
  uint32_t invalid;
  template <typename W>
  __device__ bool operator()(uint32_t src, uint32_t dst, uint32_t, W) const {
    const uint32_t nl = ld_cg(labels + src) + 1;
    const uint32_t old = atomicCAS(labels + dst, invalid, nl);
    if (old != invalid && old != nl) return false;
    atomicAdd(sigma + dst, ld_cg(sigma + src));
    return old == invalid;
  }
};

// algorithms/bc.hpp:174-186
struct BcBackward {
  const uint32_t* labels;
  const float* sigma;
  float* delta;
  float* bc;
  uint32_t source;
  template <typename W>
  __device__ bool operator()(uint32_t src, uint32_t dst, uint32_t, W) const {
    if (src == source) return false;
    if (ld_cg(labels + src) + 1 != ld_cg(labels + dst)) return false;
    const float upd = ld_cg(sigma + src) / ld_cg(sigma + dst) * (1.0f + ld_cg(delta + dst));
    atomicAdd(delta + src, upd);
    atomicAdd(bc + src, upd);
    return false;
  }
};

// tests/operators/advance_pull.cpp:29-32
struct CountVisits {
  uint32_t* visits;
  template <typename W>
  __device__ bool operator()(uint32_t src, uint32_t, uint32_t, W) const {
    atomicAdd(visits + src, 1u);
    return true;
  }
};

// tests/operators/advance_graph.cpp:19: device_graph.getDegree(u) != 0
struct NonzeroDegree {
  const uint32_t* ro;
  template <typename W>
  __device__ bool operator()(uint32_t src, uint32_t, uint32_t, W) const {
    return ro[src + 1] != ro[src];
  }
};

// tests/operators/advance.cpp:29-36 (visited flags, 64-bit distances)
struct BfsVisitFlag {
  uint8_t* visited;
  unsigned long long* dist;
  template <typename W>
  __device__ bool operator()(uint32_t src, uint32_t dst, uint32_t, W) const {
    if (!ld_cg(visited + dst)) {
      st_cg(visited + dst, (uint8_t)1);
      st_cg(dist + dst, ld_cg(dist + src) + 1ull);
      return true;
    }
    return false;
  }
};

struct AlwaysTrue {
  template <typename W>
  __device__ bool operator()(uint32_t, uint32_t, uint32_t, W) const {
    return true;
  }
};

// ---- filter predicates
struct PredEven {  // tests/operators/filter_compute.cpp:15
  __device__ bool operator()(uint32_t v) const { return v % 2 == 0; }
};
struct PredLess {  // filter_compute.cpp:19
  uint32_t bound;
  __device__ bool operator()(uint32_t v) const { return v < bound; }
};
struct PredIterMark {  // algorithms/sssp.hpp:546-550
  int32_t* visited;
  int32_t iter;
  __device__ bool operator()(uint32_t v) const {
    if (ld_cg(visited + v) == iter) return false;
    st_cg(visited + v, iter);
    return true;
  }
};
struct PredFlag {
  const uint8_t* flags;
  __device__ bool operator()(uint32_t v) const { return flags[v] != 0; }
};

// ---- compute functions
struct FnMark {  // filter_compute.cpp:26
  uint32_t* seen;
  __device__ void operator()(uint32_t v) const { seen[v] = 1u; }
};
struct FnSetU8 {  // advance_pull.cpp:36
  uint8_t* flags;
  __device__ void operator()(uint32_t v) const { flags[v] = 1; }
};
struct RedVertexId {  // filter_compute.cpp:35-36
  __device__ unsigned long long operator()(uint32_t v) const { return v; }
};
struct RedDegree {  // bfs.hpp:290-291
  const uint32_t* ro;
  __device__ unsigned long long operator()(uint32_t v) const { return ro[v + 1] - ro[v]; }
};
struct RedCount {
  __device__ unsigned long long operator()(uint32_t) const { return 1ull; }
};

}  // namespace ops
}  // namespace sgb
