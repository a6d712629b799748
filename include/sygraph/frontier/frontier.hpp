// Frontier<T, frontier_type> (frontier/frontier.hpp:45-101) over the
// two-level bitmap of libsygraph_b200.so (FrontierMLB,
// frontier/impls/mlb_frontier.hpp:155-449).  frontier_type::bitmap (the
// reference's deprecated one-level type) maps to the same implementation.
#pragma once

#include <cstdint>
#include <memory>
#include <vector>

#include "sygraph/detail/advance_kernels.cuh"
#include "sygraph/operators/config.hpp"
#include "sygraph/utils/runtime.hpp"

namespace sygraph {
namespace frontier {

// BitmapState (mlb_frontier.hpp:29-34): both levels, saved on the host.
struct BitmapState {
  std::vector<uint32_t> level0, level1;
};

template <typename T, frontier_type Type = frontier_type::mlb>
class Frontier {
 public:
  using type_t = T;
  using frontier_state_type = BitmapState;

  Frontier() = default;
  Frontier(const Queue& q, size_t num_elems) : _queue(q) {
    sg_frontier f = nullptr;
    sygraph::detail::throw_if(sg_frontier_create((uint32_t)num_elems, q.stream(), &f));
    _h = std::shared_ptr<sg_frontier_s>(f, [](sg_frontier x) { sg_frontier_destroy(x); });
  }

  size_t getNumElems() const { return view().num_elems; }
  size_t getBitmapSize() const { return view().words0; }
  size_t getBitmapRange() const { return 32; }

  bool insert(size_t idx) {
    sygraph::detail::throw_if(sg_frontier_insert(_h.get(), (uint32_t)idx));
    return true;
  }
  bool remove(size_t idx) {
    sygraph::detail::throw_if(sg_frontier_remove(_h.get(), (uint32_t)idx));
    return true;
  }
  bool check(size_t idx) const {
    int p = 0;
    sygraph::detail::throw_if(sg_frontier_check(_h.get(), (uint32_t)idx, &p));
    return p != 0;
  }
  bool empty() const {
    int e = 0;
    sygraph::detail::throw_if(sg_frontier_empty(_h.get(), &e));
    return e != 0;
  }
  size_t size() const {
    uint64_t s = 0;
    sygraph::detail::throw_if(sg_frontier_size(_h.get(), &s));
    return s;
  }
  void clear() { sygraph::detail::throw_if(sg_frontier_clear(_h.get())); }
  void merge(const Frontier& o) { sygraph::detail::throw_if(sg_frontier_merge(_h.get(), o._h.get())); }
  void intersect(const Frontier& o) { sygraph::detail::throw_if(sg_frontier_intersect(_h.get(), o._h.get())); }
  BitmapState saveState() const {
    auto v = view();
    BitmapState s;
    s.level0.resize(v.words0);
    s.level1.resize(v.words1);
    sygraph::detail::throw_if(sg_frontier_save(_h.get(), s.level0.data(), s.level1.data()));
    return s;
  }
  void loadState(const BitmapState& s) {
    sygraph::detail::throw_if(sg_frontier_load(_h.get(), s.level0.data(), s.level1.data()));
  }
  // computeActiveFrontier(invert) (mlb:388-442); the count stays on the device.
  void computeActiveFrontier(bool invert = false) const {
    sygraph::detail::throw_if(sg_frontier_compact(_h.get(), invert ? 1 : 0, nullptr));
  }

  // Device view for kernels and lambdas (check / insert / remove).
  sygraph::detail::MLBDev getDeviceFrontier() const {
    auto v = view();
    return sygraph::detail::MLBDev{v.num_elems, v.words0, v.words1, v.level0, v.level1, v.offsets, v.offsets_size};
  }
  sg_frontier handle() const { return _h.get(); }
  const Queue& getQueue() const { return _queue; }

  static void swap(Frontier& a, Frontier& b) { sygraph::detail::throw_if(sg_frontier_swap(a._h.get(), b._h.get())); }

 private:
  sg_frontier_view view() const {
    sg_frontier_view v{};
    sygraph::detail::throw_if(sg_frontier_device_view(_h.get(), &v));
    return v;
  }
  Queue _queue;
  std::shared_ptr<sg_frontier_s> _h;
};

// makeFrontier<View, Type>(q, graph) (frontier/frontier.hpp:68-80)
template <frontier_view View, frontier_type Type, typename GraphType>
auto makeFrontier(const Queue& q, const GraphType& graph) {
  static_assert(View == frontier_view::vertex || View == frontier_view::edge, "Invalid frontier view");
  if constexpr (View == frontier_view::vertex) {
    return Frontier<typename GraphType::vertex_t, Type>(q, graph.getVertexCount());
  } else {
    return Frontier<typename GraphType::edge_t, Type>(q, graph.getEdgeCount());
  }
}

// frontier::swap (frontier/frontier.hpp:94-101)
template <typename T, frontier_type FT>
void swap(Frontier<T, FT>& a, Frontier<T, FT>& b) {
  Frontier<T, FT>::swap(a, b);
}

}  // namespace frontier
}  // namespace sygraph
