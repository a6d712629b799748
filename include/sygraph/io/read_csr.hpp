// io::csr readers / writers (io/read_csr.hpp:40-411): dense adjacency text,
// Matrix Market, CSR text, COO, and the "SYGRCSR" binary layout.
#pragma once

#include <fstream>
#include <istream>
#include <sstream>
#include <string>

#include "sygraph/formats/csr.hpp"
#include "sygraph/graph/properties.hpp"

namespace sygraph {
namespace io {
namespace csr {

// io::csr::fromMatrix: n, then an n x n matrix; each non-zero becomes an edge.
template <typename ValueT, typename IndexT, typename OffsetT>
formats::CSR<ValueT, IndexT, OffsetT> fromMatrix(std::istream& iss) {
  size_t n = 0;
  iss >> n;
  std::vector<OffsetT> ro{0};
  std::vector<IndexT> col;
  std::vector<ValueT> val;
  for (size_t i = 0; i < n; ++i) {
    for (size_t j = 0; j < n; ++j) {
      ValueT v{};
      iss >> v;
      if (v != static_cast<ValueT>(0)) {
        val.push_back(v);
        col.push_back((IndexT)j);
      }
    }
    ro.push_back((OffsetT)val.size());
  }
  return formats::CSR<ValueT, IndexT, OffsetT>(ro, col, val);
}

template <typename ValueT, typename IndexT, typename OffsetT>
formats::CSR<ValueT, IndexT, OffsetT> fromMM(const std::string& filename, graph::Properties* properties = nullptr) {
  sg_host_csr h{};
  sygraph::detail::throw_if(
      sg_csr_read_mm(filename.c_str(), formats::CSR<ValueT, IndexT, OffsetT>::value_type(), &h));
  if (properties) {
    properties->directed = (h.flags & SG_GRAPH_DIRECTED) != 0;
    properties->weighted = (h.flags & SG_GRAPH_WEIGHTED) != 0;
  }
  return formats::CSR<ValueT, IndexT, OffsetT>::from_host(h);
}

template <typename ValueT, typename IndexT, typename OffsetT>
formats::CSR<ValueT, IndexT, OffsetT> fromBinary(const std::string& filename,
                                                 graph::Properties* properties = nullptr) {
  sg_host_csr h{};
  sygraph::detail::throw_if(
      sg_csr_read_binary(filename.c_str(), formats::CSR<ValueT, IndexT, OffsetT>::value_type(), &h));
  if (properties) {
    properties->directed = (h.flags & SG_GRAPH_DIRECTED) != 0;
    properties->weighted = (h.flags & SG_GRAPH_WEIGHTED) != 0;
  }
  return formats::CSR<ValueT, IndexT, OffsetT>::from_host(h);
}

template <typename ValueT, typename IndexT, typename OffsetT>
void toBinary(const formats::CSR<ValueT, IndexT, OffsetT>& csr, const std::string& filename,
              const graph::Properties& properties = graph::Properties()) {
  sg_host_csr h = csr.host_view((properties.directed ? SG_GRAPH_DIRECTED : 0u) |
                                (properties.weighted ? SG_GRAPH_WEIGHTED : 0u));
  sygraph::detail::throw_if(sg_csr_write_binary(&h, filename.c_str()));
}

// io::csr::fromCOO (io/read_csr.hpp:260-300)
template <typename ValueT, typename IndexT, typename OffsetT>
formats::CSR<ValueT, IndexT, OffsetT> fromCOO(const formats::COO<ValueT, IndexT, OffsetT>& coo) {
  uint32_t n = 0;
  for (size_t i = 0; i < coo.getSize(); i++) {
    n = std::max<uint32_t>(n, coo.getRowIndices()[i] + 1);
    n = std::max<uint32_t>(n, coo.getColumnIndices()[i] + 1);
  }
  sg_host_csr h{};
  sygraph::detail::throw_if(sg_csr_from_edges(
      n, reinterpret_cast<const uint32_t*>(coo.getRowIndices().data()),
      reinterpret_cast<const uint32_t*>(coo.getColumnIndices().data()), coo.getValues().data(),
      formats::CSR<ValueT, IndexT, OffsetT>::value_type(), coo.getSize(), 0, 0, 0, &h));
  return formats::CSR<ValueT, IndexT, OffsetT>::from_host(h);
}

}  // namespace csr
}  // namespace io
}  // namespace sygraph
