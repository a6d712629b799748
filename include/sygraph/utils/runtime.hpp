// Queue, Event and memory spaces of the C++ API.
//
// The reference binds every object to a sycl::queue and returns a
// sygraph::Event (a sycl::event with waitAndThrow / getRuntime,
// sycl/event.hpp:19-44).  Here a Queue wraps a CUDA stream and an Event is a
// pair of CUDA events recorded around the submitted work.  memory::space and
// memoryAlloc / releaseUSM keep utils/memory.hpp:12-48 (shared = managed
// memory, readable from the host like USM shared allocations).
#pragma once

#include <cuda_runtime.h>

#include <memory>
#include <stdexcept>
#include <string>

#include "sygraph_b200.h"

namespace sygraph {

namespace detail {
inline void throw_if(sg_status s) {
  if (s != SG_OK) throw std::runtime_error(std::string(sg_status_string(s)) + ": " + sg_last_error());
}
inline void throw_if_cuda(cudaError_t e, const char* what) {
  if (e != cudaSuccess) throw std::runtime_error(std::string(what) + ": " + cudaGetErrorString(e));
}
}  // namespace detail

// A CUDA stream; the default Queue uses the legacy default stream.
class Queue {
 public:
  Queue() = default;
  explicit Queue(cudaStream_t s) : _stream(s) {}
  static Queue create() {
    cudaStream_t s;
    detail::throw_if_cuda(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking), "cudaStreamCreate");
    Queue q(s);
    q._owned = std::shared_ptr<void>(s, [](void* p) { cudaStreamDestroy((cudaStream_t)p); });
    return q;
  }
  cudaStream_t stream() const { return _stream; }
  void wait() const { detail::throw_if_cuda(cudaStreamSynchronize(_stream), "cudaStreamSynchronize"); }

 private:
  cudaStream_t _stream = nullptr;
  std::shared_ptr<void> _owned;
};

// Completion handle of submitted work.
class Event {
 public:
  Event() = default;
  explicit Event(cudaStream_t s, cudaEvent_t start = nullptr) : _stream(s) {
    cudaEvent_t e;
    detail::throw_if_cuda(cudaEventCreate(&e), "cudaEventCreate");
    detail::throw_if_cuda(cudaEventRecord(e, s), "cudaEventRecord");
    _end = std::shared_ptr<CUevent_st>(e, [](cudaEvent_t x) { cudaEventDestroy(x); });
    if (start) _start = std::shared_ptr<CUevent_st>(start, [](cudaEvent_t x) { cudaEventDestroy(x); });
  }
  static cudaEvent_t mark(cudaStream_t s) {
    cudaEvent_t e;
    detail::throw_if_cuda(cudaEventCreate(&e), "cudaEventCreate");
    detail::throw_if_cuda(cudaEventRecord(e, s), "cudaEventRecord");
    return e;
  }
  void wait() {
    if (_end) cudaEventSynchronize(_end.get());
  }
  void waitAndThrow() {
    if (_end) detail::throw_if_cuda(cudaEventSynchronize(_end.get()), "device work failed");
    detail::throw_if_cuda(cudaPeekAtLastError(), "device work failed");
  }
  // Milliseconds between the start mark and the end of the work.
  float getRuntime() const {
    if (!_start || !_end) return 0.0f;
    float ms = 0.0f;
    cudaEventSynchronize(_end.get());
    cudaEventElapsedTime(&ms, _start.get(), _end.get());
    return ms;
  }

 private:
  cudaStream_t _stream = nullptr;
  std::shared_ptr<CUevent_st> _start, _end;
};

namespace memory {
enum class space { host, device, shared };
namespace detail {
template <typename T, space V>
inline T* memoryAlloc(size_t n, const Queue&) {
  void* p = nullptr;
  cudaError_t e = V == space::host     ? cudaMallocHost(&p, sizeof(T) * (n ? n : 1))
                  : V == space::device ? cudaMalloc(&p, sizeof(T) * (n ? n : 1))
                                       : cudaMallocManaged(&p, sizeof(T) * (n ? n : 1));
  sygraph::detail::throw_if_cuda(e, "memoryAlloc");
  return static_cast<T*>(p);
}
template <typename T>
inline void releaseUSM(T*& ptr, const Queue& q) {
  if (!ptr) return;
  cudaStreamSynchronize(q.stream());
  cudaPointerAttributes a{};
  if (cudaPointerGetAttributes(&a, ptr) == cudaSuccess && a.type == cudaMemoryTypeHost)
    cudaFreeHost(ptr);
  else
    cudaFree(ptr);
  ptr = nullptr;
}
}  // namespace detail
}  // namespace memory

}  // namespace sygraph
