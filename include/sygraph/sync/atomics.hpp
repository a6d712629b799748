// sync:: device atomics (sync/atomics.hpp:24-100): every operation is an
// atomic of relaxed order and device scope on the object, as the reference's
// sycl::atomic_ref<T, relaxed, device> is; here cuda::atomic_ref.
#pragma once

#include <cuda_runtime.h>

#include <cuda/atomic>
#include <type_traits>

namespace sygraph {
namespace sync {

namespace detail {
template <typename T>
using device_ref = cuda::atomic_ref<T, cuda::thread_scope_device>;
}  // namespace detail

// fetch_add; returns the value before the addition (atomics.hpp:24-28).
template <typename T>
__device__ __forceinline__ T atomicFetchAdd(T* ptr, T val) {
  return detail::device_ref<T>(*ptr).fetch_add(val, cuda::memory_order_relaxed);
}

// Relaxed atomic load (atomics.hpp:41-45): never torn, and not cached across
// other threads' stores the way a plain load may be.
template <typename T>
__device__ __forceinline__ T load(T* ptr) {
  return detail::device_ref<T>(*ptr).load(cuda::memory_order_relaxed);
}

// Relaxed atomic store (atomics.hpp:58-62).
template <typename T>
__device__ __forceinline__ void store(T* ptr, T val) {
  detail::device_ref<T>(*ptr).store(val, cuda::memory_order_relaxed);
}

// fetch_min of *v1 with the value loaded from *v2 (atomics.hpp:76-81);
// returns the previous value of *v1.  Integers use the hardware minimum.
// Floating-point values (float, double) take a compare-exchange loop that
// stores only while the new value compares less than the current one, so
// every value orders as operator< does: negative numbers, -0.0 against +0.0
// (equal: nothing is stored) and NaN (never less: nothing is stored).
template <typename T>
__device__ __forceinline__ T min(T* v1, T* v2) {
  const T x = load(v2);
  detail::device_ref<T> ref(*v1);
  if constexpr (std::is_floating_point<T>::value) {
    T old = ref.load(cuda::memory_order_relaxed);
    while (x < old) {
      if (ref.compare_exchange_weak(old, x, cuda::memory_order_relaxed, cuda::memory_order_relaxed)) break;
    }
    return old;
  } else {
    return ref.fetch_min(x, cuda::memory_order_relaxed);
  }
}

// compare_exchange_strong (atomics.hpp:95-99): on failure `expected`
// receives the current value.
template <typename T>
__device__ __forceinline__ bool cas(T* ptr, T& expected, T desired) {
  return detail::device_ref<T>(*ptr).compare_exchange_strong(expected, desired, cuda::memory_order_relaxed,
                                                            cuda::memory_order_relaxed);
}

}  // namespace sync
}  // namespace sygraph
