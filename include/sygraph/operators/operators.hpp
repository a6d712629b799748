// operators::advance / filter / compute / intersection with user device
// lambdas (operators/advance/advance.hpp:46-218, operators/filter/filter.hpp:41-69,
// operators/for/for.hpp:48-92, operators/intersection/intersection.hpp:44-55).
//
// A functor is a device lambda, e.g. (nvcc --extended-lambda)
//   advance::frontier<load_balancer::workgroup_mapped, frontier_view::vertex,
//                     frontier_view::vertex>(G, in, out,
//       SYGRAPH_LAMBDA(auto src, auto dst, auto edge, auto weight) -> bool {...});
// Every call enqueues on the graph's queue and returns an Event; no call
// waits on the host (the reference blocks on a size read before each launch,
// operators/advance/common.hpp:112-119).
#pragma once

#include <type_traits>

#include "sygraph/detail/advance_kernels.cuh"
#include "sygraph/frontier/frontier.hpp"
#include "sygraph/graph/graph.hpp"
#include "sygraph/operators/config.hpp"
#include "sygraph/utils/runtime.hpp"

#ifndef SYGRAPH_LAMBDA
#define SYGRAPH_LAMBDA [=] __device__
#endif

namespace sygraph {
namespace operators {
namespace detail {

// SM count of the current device, queried once per device and thread.
inline unsigned sm_count() {
  static thread_local int cached_dev = -1, cached_sms = 148;
  int dev = 0;
  cudaGetDevice(&dev);
  if (dev != cached_dev) {
    int sms = 0;
    if (cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) == cudaSuccess && sms > 0) cached_sms = sms;
    else cudaGetLastError();
    cached_dev = dev;
  }
  return (unsigned)cached_sms;
}

inline unsigned advance_grid(int expected_size) {
  const unsigned full = sm_count() * 8u;
  if (expected_size > 0) {
    const unsigned want = (unsigned)(((uint64_t)expected_size + 255) / 256);
    return want < 1 ? 1 : (want < full ? want : full);
  }
  return full;
}

template <direction D>
constexpr int dir_code() {
  return D == direction::push ? sygraph::detail::kPush : (D == direction::pull ? sygraph::detail::kPull : sygraph::detail::kPullAll);
}

constexpr int view_code(frontier::frontier_view v) {
  return v == frontier::frontier_view::graph    ? sygraph::detail::kViewGraph
         : v == frontier::frontier_view::vertex ? sygraph::detail::kViewVertex
         : v == frontier::frontier_view::edge   ? sygraph::detail::kViewEdge
                                                : sygraph::detail::kViewNone;
}

constexpr int lb_code(load_balancer lb) {
  return lb == load_balancer::workitem_mapped    ? 0
         : lb == load_balancer::subgroup_mapped  ? 1
         : lb == load_balancer::workgroup_mapped ? 2
                                                 : 3;
}

template <direction D, load_balancer Lb, frontier::frontier_view InView, frontier::frontier_view OutView,
          typename GraphT, typename LambdaT>
Event launch(GraphT& graph, const sygraph::detail::MLBDev* in, sg_frontier in_handle,
             const sygraph::detail::MLBDev* out, LambdaT&& functor, int expected_size) {
  static_assert(InView == frontier::frontier_view::vertex || InView == frontier::frontier_view::graph,
                "Invalid frontier view for the advance input");
  using W = typename GraphT::weight_t;
  cudaStream_t s = graph.getQueue().stream();
  cudaEvent_t start = Event::mark(s);
  if (InView == frontier::frontier_view::vertex)
    sygraph::detail::throw_if(sg_frontier_compact(in_handle, is_pull<D>() ? 1 : 0, nullptr));
  const sg_graph_view v = graph.view(is_pull<D>());
  sygraph::detail::GraphDev<W> g{v.n, v.m, v.row_offsets, v.column_indices, reinterpret_cast<const W*>(v.values)};
  sygraph::detail::AdvanceArgs a{};
  a.in_view = view_code(InView);
  a.out_view = view_code(OutView);
  a.limit = v.n;
  if (in) a.in = *in;
  if (out) a.out = *out;
  using F = std::decay_t<LambdaT>;
  sygraph::detail::throw_if_cuda(
      sygraph::detail::launch_advance<dir_code<D>(), W, F>(lb_code(Lb), g, a, functor, advance_grid(expected_size), s),
      "advance launch");
  return Event(s, start);
}

}  // namespace detail

namespace advance {

// advance::frontier<Direction, Lb, InView, OutView>(G, in, out, f, expected_size)
template <direction Direction, load_balancer Lb, frontier::frontier_view InView, frontier::frontier_view OutView,
          typename GraphT, typename LambdaT, typename T, frontier::frontier_type FrontierType>
Event frontier(GraphT& graph, frontier::Frontier<T, FrontierType>& in, frontier::Frontier<T, FrontierType>& out,
               LambdaT&& functor, frontier::size::frontier_size_t expected_size = frontier::size::fetch_from_memory) {
  const auto di = in.getDeviceFrontier();
  const auto dout = out.getDeviceFrontier();
  return detail::launch<Direction, Lb, InView, OutView>(graph, &di, in.handle(), &dout,
                                                         std::forward<LambdaT>(functor), expected_size);
}

// Direction-less overload = push (advance.hpp:142-165)
template <load_balancer Lb, frontier::frontier_view InView, frontier::frontier_view OutView, typename GraphT,
          typename LambdaT, typename T, frontier::frontier_type FrontierType>
Event frontier(GraphT& graph, frontier::Frontier<T, FrontierType>& in, frontier::Frontier<T, FrontierType>& out,
               LambdaT&& functor, frontier::size::frontier_size_t expected_size = frontier::size::fetch_from_memory) {
  return frontier<direction::push, Lb, InView, OutView>(graph, in, out, std::forward<LambdaT>(functor), expected_size);
}

// No-output overloads (advance.hpp:190-218)
template <direction Direction, load_balancer Lb, frontier::frontier_view InView, typename GraphT, typename LambdaT,
          typename T, frontier::frontier_type FrontierType>
Event frontier(GraphT& graph, frontier::Frontier<T, FrontierType>& in, LambdaT&& functor,
               frontier::size::frontier_size_t expected_size = frontier::size::fetch_from_memory) {
  const auto di = in.getDeviceFrontier();
  return detail::launch<Direction, Lb, InView, frontier::frontier_view::none>(graph, &di, in.handle(), nullptr,
                                                                              std::forward<LambdaT>(functor),
                                                                              expected_size);
}

template <load_balancer Lb, frontier::frontier_view InView, typename GraphT, typename LambdaT, typename T,
          frontier::frontier_type FrontierType>
Event frontier(GraphT& graph, frontier::Frontier<T, FrontierType>& in, LambdaT&& functor,
               frontier::size::frontier_size_t expected_size = frontier::size::fetch_from_memory) {
  return frontier<direction::push, Lb, InView>(graph, in, std::forward<LambdaT>(functor), expected_size);
}

// advance::vertices<Lb, OutView>(G, out, f): every vertex is a candidate (advance.hpp:46-65)
template <load_balancer Lb, frontier::frontier_view FW, typename GraphT, typename LambdaT, typename T,
          frontier::frontier_type FrontierType>
Event vertices(GraphT& graph, frontier::Frontier<T, FrontierType>& out, LambdaT&& functor) {
  const auto dout = out.getDeviceFrontier();
  return detail::launch<direction::push, Lb, frontier::frontier_view::graph, FW>(
      graph, nullptr, nullptr, &dout, std::forward<LambdaT>(functor), frontier::size::fetch_from_memory);
}

// advance::vertices<Lb>(G, f) (advance.hpp:83-87)
template <load_balancer Lb, typename GraphT, typename LambdaT>
Event vertices(GraphT& graph, LambdaT&& functor) {
  return detail::launch<direction::push, Lb, frontier::frontier_view::graph, frontier::frontier_view::none>(
      graph, nullptr, nullptr, nullptr, std::forward<LambdaT>(functor), frontier::size::fetch_from_memory);
}

}  // namespace advance

namespace filter {

// filter::inplace(G, f, pred): removes every active v with pred(v) (filter.hpp:41-45)
template <typename GraphT, typename T, frontier::frontier_type FT, typename LambdaT>
Event inplace(GraphT& graph, frontier::Frontier<T, FT>& f, LambdaT&& pred) {
  cudaStream_t s = graph.getQueue().stream();
  cudaEvent_t start = Event::mark(s);
  f.computeActiveFrontier(false);
  const auto d = f.getDeviceFrontier();
  sygraph::detail::filter_inplace_kernel<<<operators::detail::advance_grid(-1), 256, 0, s>>>(
      d, (uint32_t)graph.getVertexCount(), pred);
  sygraph::detail::throw_if_cuda(cudaGetLastError(), "filter launch");
  return Event(s, start);
}

// filter::external(G, in, out, pred): out = { v in in : pred(v) } (filter.hpp:47-69)
template <typename GraphT, typename T, frontier::frontier_type FT, typename LambdaT>
Event external(GraphT& graph, frontier::Frontier<T, FT>& in, frontier::Frontier<T, FT>& out, LambdaT&& pred) {
  cudaStream_t s = graph.getQueue().stream();
  cudaEvent_t start = Event::mark(s);
  in.computeActiveFrontier(false);
  out.clear();
  sygraph::detail::filter_external_kernel<<<operators::detail::advance_grid(-1), 256, 0, s>>>(
      in.getDeviceFrontier(), out.getDeviceFrontier(), (uint32_t)graph.getVertexCount(), pred);
  sygraph::detail::throw_if_cuda(cudaGetLastError(), "filter launch");
  return Event(s, start);
}

}  // namespace filter

namespace compute {

template <typename R>
struct plus {};

// compute::execute<vertex>(G, f, fn) (for.hpp:48-60)
template <frontier::frontier_view FW, typename GraphT, typename T, typename LambdaT, frontier::frontier_type FT>
Event execute(GraphT& graph, frontier::Frontier<T, FT>& f, LambdaT&& fn,
              frontier::size::frontier_size_t = frontier::size::fetch_from_memory) {
  static_assert(FW == frontier::frontier_view::vertex, "Invalid frontier view for compute operation.");
  cudaStream_t s = graph.getQueue().stream();
  cudaEvent_t start = Event::mark(s);
  f.computeActiveFrontier(false);
  sygraph::detail::compute_execute_kernel<<<operators::detail::advance_grid(-1), 256, 0, s>>>(
      f.getDeviceFrontier(), (uint32_t)graph.getVertexCount(), fn);
  sygraph::detail::throw_if_cuda(cudaGetLastError(), "compute launch");
  return Event(s, start);
}

namespace detail {
template <typename R, typename LambdaT>
struct ReduceAdapter {
  LambdaT fn;
  __device__ R operator()(uint32_t v) const {
    R acc = R(0);
    fn(v, acc);
    return acc;
  }
};

template <typename R, typename Fn>
__global__ void __launch_bounds__(256) reduce_kernel(sygraph::detail::MLBDev f, uint32_t limit, Fn fn, R* out) {
  R acc = R(0);
  const uint64_t total = (uint64_t)sygraph::detail::ld_cg(f.offsets_size) * 32;
  for (uint64_t t = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; t < total; t += (uint64_t)gridDim.x * blockDim.x) {
    const uint32_t v = (uint32_t)sygraph::detail::ld_cg(f.offsets + (t >> 5)) * 32 + (uint32_t)(t & 31);
    if (v < limit && f.check(v)) acc += fn(v);
  }
  __shared__ R s_red[32];
  acc = sygraph::detail::block_sum(acc, s_red);
  if (threadIdx.x == 0) atomicAdd(out, acc);
}
}  // namespace detail

// compute::reduce<vertex, plus<R>>(G, f, acc, fn(v, acc&)) (for.hpp:62-92):
// the sum is added to `accumulator` when the call returns.
template <frontier::frontier_view FW, typename ReductionOperator, typename GraphT, typename T, typename R,
          frontier::frontier_type FT, typename LambdaT>
Event reduce(GraphT& graph, frontier::Frontier<T, FT>& f, R& accumulator, LambdaT&& function,
             frontier::size::frontier_size_t = frontier::size::fetch_from_memory) {
  static_assert(FW == frontier::frontier_view::vertex, "Invalid frontier view for compute operation.");
  cudaStream_t s = graph.getQueue().stream();
  cudaEvent_t start = Event::mark(s);
  static_assert(sizeof(R) <= GraphT::kScratchBytes, "reduction type larger than the graph's accumulator");
  f.computeActiveFrontier(false);
  // the graph's preallocated accumulator: no allocation per call
  R* d = static_cast<R*>(graph.scratch());
  sygraph::detail::throw_if_cuda(cudaMemsetAsync(d, 0, sizeof(R), s), "cudaMemsetAsync");
  using A = detail::ReduceAdapter<R, std::decay_t<LambdaT>>;
  detail::reduce_kernel<R, A><<<operators::detail::advance_grid(-1), 256, 0, s>>>(
      f.getDeviceFrontier(), (uint32_t)graph.getVertexCount(), A{function}, d);
  sygraph::detail::throw_if_cuda(cudaGetLastError(), "reduce launch");
  R h{};
  // the sum goes to a host reference, so the call waits for it, as the
  // reference's reduction into a host buffer does
  sygraph::detail::throw_if_cuda(cudaMemcpyAsync(&h, d, sizeof(R), cudaMemcpyDeviceToHost, s), "cudaMemcpyAsync");
  sygraph::detail::throw_if_cuda(cudaStreamSynchronize(s), "cudaStreamSynchronize");
  accumulator += h;
  return Event(s, start);
}

}  // namespace compute

namespace intersection {
// intersection::execute(G, in1, in2, out, f): out = in1 AND in2; f unused (intersection.hpp:44-55)
template <typename GraphT, typename T, frontier::frontier_type FT, typename LambdaT>
Event execute(GraphT& graph, frontier::Frontier<T, FT>& in1, frontier::Frontier<T, FT>& in2,
              frontier::Frontier<T, FT>& out, LambdaT&&) {
  cudaStream_t s = graph.getQueue().stream();
  cudaEvent_t start = Event::mark(s);
  sygraph::detail::throw_if(sg_intersection_execute(graph.handle(), in1.handle(), in2.handle(), out.handle()));
  return Event(s, start);
}
}  // namespace intersection

}  // namespace operators
}  // namespace sygraph
