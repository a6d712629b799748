// formats::CSR (formats/csr.hpp:32-215) and formats::COO (formats/coo.hpp:40-157):
// host containers; invert() builds the transpose through the C ABI.
#pragma once

#include <cstdint>
#include <cstring>
#include <type_traits>
#include <vector>

#include "sygraph/utils/runtime.hpp"

namespace sygraph {
namespace formats {

template <typename ValueT, typename IndexT = uint32_t, typename OffsetT = uint32_t>
class CSR {
  static_assert(sizeof(IndexT) == 4 && sizeof(OffsetT) == 4 && sizeof(ValueT) == 4,
                "sygraph_b200 stores vertex ids, offsets and weights as 32-bit values");

 public:
  using value_t = ValueT;
  using index_t = IndexT;
  using offset_t = OffsetT;

  CSR() = default;
  CSR(std::vector<OffsetT> row_offsets, std::vector<IndexT> column_indices, std::vector<ValueT> nnz_values)
      : _row_offsets(std::move(row_offsets)), _column_indices(std::move(column_indices)),
        _nnz_values(std::move(nnz_values)) {}

  IndexT getRowOffsetsSize() const { return (IndexT)(_row_offsets.size() - 1); }
  OffsetT getNumNonzeros() const { return (OffsetT)_column_indices.size(); }
  const std::vector<OffsetT>& getRowOffsets() const { return _row_offsets; }
  const std::vector<IndexT>& getColumnIndices() const { return _column_indices; }
  const std::vector<ValueT>& getValues() const { return _nnz_values; }
  std::vector<OffsetT>& getRowOffsets() { return _row_offsets; }
  std::vector<IndexT>& getColumnIndices() { return _column_indices; }
  std::vector<ValueT>& getValues() { return _nnz_values; }

  static constexpr int value_type() { return std::is_floating_point<ValueT>::value ? SG_WEIGHT_F32 : SG_WEIGHT_U32; }

  sg_host_csr host_view(uint32_t flags = 0) const {
    sg_host_csr h{};
    h.n = getRowOffsetsSize();
    h.m = getNumNonzeros();
    h.row_offsets = const_cast<uint32_t*>(reinterpret_cast<const uint32_t*>(_row_offsets.data()));
    h.column_indices = const_cast<uint32_t*>(reinterpret_cast<const uint32_t*>(_column_indices.data()));
    h.values = _nnz_values.empty() ? nullptr : const_cast<ValueT*>(_nnz_values.data());
    h.value_type = value_type();
    h.flags = flags;
    return h;
  }

  static CSR from_host(sg_host_csr& h) {
    CSR out;
    out._row_offsets.assign(reinterpret_cast<OffsetT*>(h.row_offsets), reinterpret_cast<OffsetT*>(h.row_offsets) + h.n + 1);
    out._column_indices.assign(reinterpret_cast<IndexT*>(h.column_indices),
                               reinterpret_cast<IndexT*>(h.column_indices) + h.m);
    out._nnz_values.resize(h.m);
    if (h.values)
      std::memcpy(out._nnz_values.data(), h.values, sizeof(ValueT) * h.m);
    else
      for (auto& v : out._nnz_values) v = (ValueT)1;
    sg_host_csr_free(&h);
    return out;
  }

  // CSR::invert (formats/csr.hpp:179-209): the transpose (incoming edges).
  CSR invert() const {
    sg_host_csr in = host_view(), out{};
    sygraph::detail::throw_if(sg_csr_invert(&in, &out));
    return from_host(out);
  }

 private:
  std::vector<OffsetT> _row_offsets{0};
  std::vector<IndexT> _column_indices;
  std::vector<ValueT> _nnz_values;
};

template <typename ValueT, typename IndexT = uint32_t, typename OffsetT = uint32_t>
class COO {
 public:
  COO(std::vector<IndexT> row_indices, std::vector<IndexT> column_indices, std::vector<ValueT> nnz_values)
      : _row_indices(std::move(row_indices)), _column_indices(std::move(column_indices)),
        _nnz_values(std::move(nnz_values)) {}
  const std::vector<IndexT>& getRowIndices() const { return _row_indices; }
  const std::vector<IndexT>& getColumnIndices() const { return _column_indices; }
  const std::vector<ValueT>& getValues() const { return _nnz_values; }
  size_t getSize() const { return _row_indices.size(); }

 private:
  std::vector<IndexT> _row_indices, _column_indices;
  std::vector<ValueT> _nnz_values;
};

}  // namespace formats
}  // namespace sygraph
