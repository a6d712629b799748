// GraphCSR / GraphCSRDevice (graph/impls/graph_csr.hpp:15-439) and
// graph::build::fromCSR (graph/build.hpp:31-41).  The device arrays are owned
// by an sg_graph handle of libsygraph_b200.so; GraphCSRDevice is a trivially
// copyable view that device lambdas capture by value.
#pragma once

#include <cstdint>
#include <memory>

#include "sygraph/formats/csr.hpp"
#include "sygraph/graph/properties.hpp"
#include "sygraph/utils/runtime.hpp"

namespace sygraph {
namespace graph {
namespace detail {

template <typename IndexT, typename OffsetT, typename ValueT>
class GraphCSRDevice {
 public:
  using vertex_t = IndexT;
  using edge_t = OffsetT;
  using weight_t = ValueT;

  struct NeighborIterator {
    __host__ __device__ NeighborIterator(const IndexT* start, const IndexT* p) : _start_ptr(start), _ptr(p) {}
    __host__ __device__ IndexT operator*() const { return *_ptr; }
    __host__ __device__ NeighborIterator& operator++() {
      ++_ptr;
      return *this;
    }
    __host__ __device__ NeighborIterator operator+(int k) const { return NeighborIterator(_start_ptr, _ptr + k); }
    __host__ __device__ bool operator==(const NeighborIterator& o) const { return _ptr == o._ptr; }
    __host__ __device__ bool operator!=(const NeighborIterator& o) const { return _ptr != o._ptr; }
    __host__ __device__ edge_t getIndex() const { return static_cast<edge_t>(_ptr - _start_ptr); }
    const IndexT* _start_ptr;
    const IndexT* _ptr;
  };

  GraphCSRDevice() = default;
  GraphCSRDevice(const sg_graph_view& v)
      : _n_rows(v.n), _n_nonzeros((OffsetT)v.m), _column_indices(reinterpret_cast<const IndexT*>(v.column_indices)),
        _row_offsets(reinterpret_cast<const OffsetT*>(v.row_offsets)),
        _nnz_values(reinterpret_cast<const ValueT*>(v.values)) {}

  __host__ __device__ size_t getVertexCount() const { return _n_rows; }
  __host__ __device__ size_t getEdgeCount() const { return _n_nonzeros; }
  __device__ size_t getDegree(vertex_t v) const { return _row_offsets[v + 1] - _row_offsets[v]; }
  __device__ vertex_t getFirstNeighbor(vertex_t v) const { return _row_offsets[v]; }
  __device__ vertex_t getDestinationVertex(edge_t e) const { return _column_indices[e]; }
  __device__ weight_t getEdgeWeight(edge_t e) const { return _nnz_values[e]; }
  __device__ NeighborIterator begin(vertex_t v) const {
    return NeighborIterator(_column_indices, _column_indices + _row_offsets[v]);
  }
  __device__ NeighborIterator end(vertex_t v) const {
    return NeighborIterator(_column_indices, _column_indices + _row_offsets[v + 1]);
  }
  __host__ __device__ const IndexT* getColumnIndices() const { return _column_indices; }
  __host__ __device__ const OffsetT* getRowOffsets() const { return _row_offsets; }
  __host__ __device__ const ValueT* getValues() const { return _nnz_values; }

  // getIntersectionCount (graph_csr.hpp:109-135): merge of two sorted lists,
  // func(common) per match.
  template <typename Func>
  __device__ size_t getIntersectionCount(const vertex_t& src, const vertex_t& dst, Func&& func) const {
    size_t count = 0;
    auto a = begin(src), ae = end(src), b = begin(dst), be = end(dst);
    while (a != ae && b != be) {
      if (*a == *b) {
        func(*a);
        ++a;
        ++b;
        ++count;
      } else if (*a < *b) {
        ++a;
      } else {
        ++b;
      }
    }
    return count;
  }

  IndexT _n_rows = 0;
  OffsetT _n_nonzeros = 0;
  const IndexT* _column_indices = nullptr;
  const OffsetT* _row_offsets = nullptr;
  const ValueT* _nnz_values = nullptr;
};

template <typename IndexT, typename OffsetT, typename ValueT>
class GraphCSR {
 public:
  using vertex_t = IndexT;
  using edge_t = OffsetT;
  using weight_t = ValueT;
  using device_graph_t = GraphCSRDevice<IndexT, OffsetT, ValueT>;

  GraphCSR(const Queue& q, const formats::CSR<ValueT, IndexT, OffsetT>& csr, const Properties& properties)
      : _queue(q), _csr(csr), _properties(properties) {
    sg_graph g = nullptr;
    sygraph::detail::throw_if(sg_graph_create_csr(
        reinterpret_cast<const uint32_t*>(csr.getRowOffsets().data()),
        reinterpret_cast<const uint32_t*>(csr.getColumnIndices().data()),
        csr.getValues().empty() ? nullptr : csr.getValues().data(), formats::CSR<ValueT, IndexT, OffsetT>::value_type(),
        csr.getRowOffsetsSize(), csr.getNumNonzeros(),
        (properties.directed ? SG_GRAPH_DIRECTED : 0u) | (properties.weighted ? SG_GRAPH_WEIGHTED : 0u), q.stream(),
        &g));
    _handle = std::shared_ptr<sg_graph_s>(g, [](sg_graph h) { sg_graph_destroy(h); });
  }
  GraphCSR(const GraphCSR&) = delete;
  GraphCSR& operator=(const GraphCSR&) = delete;
  GraphCSR(GraphCSR&&) = default;

  size_t getVertexCount() const { return _csr.getRowOffsetsSize(); }
  size_t getEdgeCount() const { return _csr.getNumNonzeros(); }
  size_t getDegree(vertex_t v) const { return _csr.getRowOffsets()[v + 1] - _csr.getRowOffsets()[v]; }
  const OffsetT* getRowOffsets() const { return _csr.getRowOffsets().data(); }
  const IndexT* getColumnIndices() const { return _csr.getColumnIndices().data(); }
  const ValueT* getValues() const { return _csr.getValues().data(); }
  const Properties& getProperties() const { return _properties; }

  device_graph_t getDeviceGraph() const { return device_graph_t(view(false)); }
  device_graph_t getInverseDeviceGraph() const { return device_graph_t(view(true)); }
  sg_graph_view view(bool inverse) const {
    sg_graph_view v{};
    sygraph::detail::throw_if(sg_graph_device_view(_handle.get(), inverse ? 1 : 0, &v));
    return v;
  }
  sg_graph handle() const { return _handle.get(); }
  const Queue& getQueue() const { return _queue; }

  // 64 bytes of device memory owned by the graph, allocated on first use and
  // released with the graph: the accumulator of compute::reduce, so repeated
  // reductions allocate nothing.  Calls on one graph share it (they are
  // ordered on the graph's queue).
  static constexpr size_t kScratchBytes = 64;
  void* scratch() const {
    if (!_scratch) {
      void* p = nullptr;
      sygraph::detail::throw_if_cuda(cudaMalloc(&p, kScratchBytes), "cudaMalloc");
      _scratch = std::shared_ptr<void>(p, [](void* q) { cudaFree(q); });
    }
    return _scratch.get();
  }

 private:
  Queue _queue;
  formats::CSR<ValueT, IndexT, OffsetT> _csr;
  Properties _properties;
  std::shared_ptr<sg_graph_s> _handle;
  mutable std::shared_ptr<void> _scratch;
};

}  // namespace detail

namespace build {
// graph::build::fromCSR<Space>(q, csr, properties) (graph/build.hpp:31-41).
// The memory space is kept for source compatibility; the graph always lives
// in device memory and keeps a host copy of the CSR.
template <memory::space Space = memory::space::device, typename IndexT, typename OffsetT, typename ValueT>
auto fromCSR(const Queue& q, const formats::CSR<ValueT, IndexT, OffsetT>& csr, Properties properties = Properties()) {
  return detail::GraphCSR<IndexT, OffsetT, ValueT>(q, csr, properties);
}
}  // namespace build

}  // namespace graph
}  // namespace sygraph
