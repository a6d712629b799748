// sync:: device atomics (sync/atomics.hpp:24-100): relaxed, device scope.
#pragma once

#include <cuda_runtime.h>

#include <type_traits>

namespace sygraph {
namespace sync {

template <typename T>
__device__ __forceinline__ T atomicFetchAdd(T* ptr, T val) {
  return ::atomicAdd(ptr, val);
}

template <typename T>
__device__ __forceinline__ T load(T* ptr) {
  return *reinterpret_cast<volatile T*>(ptr);
}

template <typename T>
__device__ __forceinline__ void store(T* ptr, T val) {
  *reinterpret_cast<volatile T*>(ptr) = val;
}

// fetch_min of *v1 with *v2; returns the previous value of *v1.
template <typename T>
__device__ __forceinline__ T min(T* v1, T* v2) {
  const T x = load(v2);
  if constexpr (std::is_same<T, float>::value) {
    // non-negative floats order like their bit patterns
    return __int_as_float(::atomicMin(reinterpret_cast<int*>(v1), __float_as_int(x)));
  } else {
    return ::atomicMin(v1, x);
  }
}

// compare_exchange_strong: on failure `expected` receives the current value.
template <typename T>
__device__ __forceinline__ bool cas(T* ptr, T& expected, T desired) {
  const T old = ::atomicCAS(ptr, expected, desired);
  const bool ok = old == expected;
  expected = old;
  return ok;
}

}  // namespace sync
}  // namespace sygraph
