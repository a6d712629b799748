// Device primitives shared by the C ABI kernels (libsygraph_b200.so) and the
// templated C++ layer: warp collectives, bitmap helpers, cache-hinted loads and
// a bounded grid barrier.  sm_100a only.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

namespace sygraph {
namespace detail {

constexpr uint32_t kFullMask = 0xffffffffu;
constexpr int kWarp = 32;

__device__ __forceinline__ uint32_t lane_id() { return threadIdx.x & 31u; }
__device__ __forceinline__ uint32_t lanemask_lt() {
  uint32_t m;
  asm("mov.u32 %0, %%lanemask_lt;" : "=r"(m));
  return m;
}

// Loads of data that other CTAs of the same kernel write (bitmaps, queues,
// depths) bypass L1, which is not coherent across SMs.
template <typename T>
__device__ __forceinline__ T ld_cg(const T* p) { return __ldcg(p); }
template <typename T>
__device__ __forceinline__ void st_cg(T* p, T v) { __stcg(p, v); }

__device__ __forceinline__ uint32_t ld_acquire(const uint32_t* p) {
  uint32_t v;
  asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
  return v;
}
__device__ __forceinline__ void st_release(uint32_t* p, uint32_t v) {
  asm volatile("st.release.gpu.global.u32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}
__device__ __forceinline__ uint32_t ld_volatile(const uint32_t* p) {
  return *reinterpret_cast<const volatile uint32_t*>(p);
}

__device__ __forceinline__ uint64_t global_timer_ns() {
  uint64_t t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}

// Inclusive warp scan (Kogge-Stone over shuffles).
template <typename T>
__device__ __forceinline__ T warp_inclusive_scan(T v) {
#pragma unroll
  for (int d = 1; d < 32; d <<= 1) {
    T o = __shfl_up_sync(kFullMask, v, d);
    if ((int)lane_id() >= d) v += o;
  }
  return v;
}

template <typename T>
__device__ __forceinline__ T warp_sum(T v) {
#pragma unroll
  for (int d = 16; d > 0; d >>= 1) v += __shfl_xor_sync(kFullMask, v, d);
  return v;
}

// Lane that owns edge rank r given every lane's inclusive prefix `incl` of
// degrees: the number of lanes whose inclusive end is <= r.  All 32 lanes
// must call it (each with its own r).
__device__ __forceinline__ uint32_t warp_owner_of_rank(uint32_t incl, uint32_t r) {
  uint32_t j = 0;
#pragma unroll
  for (uint32_t s = 16; s >= 1; s >>= 1) {
    uint32_t c = __shfl_sync(kFullMask, incl, (j + s - 1) & 31);
    if (j + s - 1 < 32 && c <= r) j += s;
  }
  return j;
}

// Warp-aggregated append: every lane with `pred` gets a distinct slot in
// [base, base + popc(ballot)); one atomic per warp.  Must be called by the
// whole warp.
__device__ __forceinline__ uint32_t warp_append(bool pred, uint32_t* tail) {
  const uint32_t mask = __ballot_sync(kFullMask, pred);
  if (mask == 0) return 0;
  const uint32_t leader = __ffs(mask) - 1;
  uint32_t base = 0;
  if (lane_id() == leader) base = atomicAdd(tail, (uint32_t)__popc(mask));
  base = __shfl_sync(kFullMask, base, leader);
  return base + __popc(mask & lanemask_lt());
}

// Block-wide exclusive scan of one uint32 per thread; s_warp holds >= 32
// words.  Every thread of the block must call it.
__device__ __forceinline__ uint32_t block_excl_scan(uint32_t v, uint32_t* total, uint32_t* s_warp) {
  const uint32_t lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
  const uint32_t incl = warp_inclusive_scan(v);
  if (lane == 31) s_warp[warp] = incl;
  __syncthreads();
  if (warp == 0) {
    uint32_t x = lane < nw ? s_warp[lane] : 0;
    x = warp_inclusive_scan(x);
    s_warp[lane] = x;
  }
  __syncthreads();
  const uint32_t before = warp ? s_warp[warp - 1] : 0;
  *total = s_warp[nw - 1];
  __syncthreads();
  return before + incl - v;
}

// Block-wide sum; the result is valid in warp 0.  s_red holds >= 32 entries.
template <typename T>
__device__ __forceinline__ T block_sum(T v, T* s_red) {
  const uint32_t lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
  v = warp_sum(v);
  if (lane == 0) s_red[warp] = v;
  __syncthreads();
  T t = 0;
  if (warp == 0) {
    t = lane < nw ? s_red[lane] : (T)0;
    t = warp_sum(t);
  }
  __syncthreads();
  return t;
}

__device__ __forceinline__ uint32_t warp_min(uint32_t v) {
#pragma unroll
  for (int d = 16; d > 0; d >>= 1) v = min(v, __shfl_xor_sync(0xffffffffu, v, d));
  return v;
}

__device__ __forceinline__ bool bit_test(const uint32_t* bm, uint32_t i) {
  return (ld_cg(bm + (i >> 5)) >> (i & 31)) & 1u;
}
// L1-cached test, for a bitmap nobody writes until the next grid barrier (a
// frontier being expanded): the barrier's acquire fence orders these weak
// loads after every write of the previous level.
__device__ __forceinline__ bool bit_test_ro(const uint32_t* bm, uint32_t i) {
  return (bm[i >> 5] >> (i & 31)) & 1u;
}
// Sets bit i; returns true when this call changed it from 0 to 1.  The
// plain load skips the atomic when the bit is already visible as set.
__device__ __forceinline__ bool bit_set_once(uint32_t* bm, uint32_t i) {
  const uint32_t b = 1u << (i & 31);
  if (ld_cg(bm + (i >> 5)) & b) return false;
  return (atomicOr(bm + (i >> 5), b) & b) == 0;
}

// Non-negative IEEE floats order like their bit patterns.
__device__ __forceinline__ float atomic_min_nonneg(float* p, float v) {
  return __int_as_float(atomicMin(reinterpret_cast<int*>(p), __float_as_int(v)));
}
__device__ __forceinline__ uint32_t atomic_min_nonneg(uint32_t* p, uint32_t v) { return atomicMin(p, v); }

// ---------------------------------------------------------------------------
// Grid barrier for persistent cooperative kernels.  Every wait is bounded:
// after kBarrierSpinLimit polls a block records an error and every block
// leaves the kernel at its next barrier, so a lost block can never hang the
// GPU.  The grid must be co-resident (cooperative launch).
// ---------------------------------------------------------------------------
struct GridBarrier {
  unsigned long long count;  // arrivals since the launch began; top bit: a wait ran out
  uint32_t error;            // read by the host after the launch
  uint32_t exits;            // blocks past their last barrier (grid_exit)
};

constexpr uint64_t kBarrierSpinLimit = 1ull << 24;  // ~16M polls x >=64 ns sleep: over a second
constexpr unsigned long long kBarrierFailed = 1ull << 63;

__device__ __forceinline__ unsigned long long atom_add_acq_rel(unsigned long long* p, unsigned long long v) {
  unsigned long long old;
  asm volatile("atom.acq_rel.gpu.global.add.u64 %0, [%1], %2;" : "=l"(old) : "l"(p), "l"(v) : "memory");
  return old;
}
__device__ __forceinline__ unsigned long long ld_acquire(const unsigned long long* p) {
  unsigned long long v;
  asm volatile("ld.acquire.gpu.global.u64 %0, [%1];" : "=l"(v) : "l"(p) : "memory");
  return v;
}

// Returns false when the barrier timed out (here or in another block).
//
// The count starts at zero for each launch (the host clears it) and only
// grows: thread 0 of each block arrives with one acq_rel atomic (release for
// this block's writes, ordered before it by __syncthreads), and the value it
// returns names the phase, so the block waits until the count reaches the
// phase's end, (old / gridDim.x + 1) * gridDim.x, with acquire loads.  Every
// arrival is a read-modify-write of the same word, so the value a waiter
// reads carries the release of every earlier arrival.  The last arriver
// needs no wait and no second write: its own atomic completes the phase.  A
// block whose wait runs out sets the count's top bit (and the error word),
// which ends every other wait at once and fails every later barrier of the
// launch.
__device__ __forceinline__ bool grid_sync(GridBarrier* bar, uint64_t spin_limit = kBarrierSpinLimit) {
  __shared__ uint32_t s_ok;
  __syncthreads();
  if (threadIdx.x == 0) {
    uint32_t ok = 1;
    const unsigned long long old = atom_add_acq_rel(&bar->count, 1ull);
    if (old & kBarrierFailed) {
      ok = 0;
    } else {
      const unsigned long long target = (old / gridDim.x + 1) * gridDim.x;
      if (old + 1 != target) {
        uint64_t spins = 0;
        for (;;) {
          const unsigned long long c = ld_acquire(&bar->count);
          if (c & kBarrierFailed) {
            ok = 0;
            break;
          }
          if (c >= target) break;
          if (++spins > spin_limit) {
            atomicOr(&bar->count, kBarrierFailed);
            atomicExch(&bar->error, 1u);
            ok = 0;
            break;
          }
          // poll back-to-back first (a barrier normally completes within a few
          // microseconds), then back off
          if (spins > 512) __nanosleep(spins > 4096 ? 256 : 32);
        }
      }
    }
    s_ok = ok;
  }
  __syncthreads();
  return s_ok != 0;
}

// Called once by every block at the end of a launch that completed all its
// barriers: the last block out returns the barrier to its launch state
// (count and exits zero), so the next launch needs no host-side reset.
// Every other block has passed its last wait before it arrives here.  A
// launch that left through a failed barrier skips this, and its count keeps
// the failure bit until the host clears it.
__device__ __forceinline__ void grid_exit(GridBarrier* bar) {
  if (threadIdx.x == 0 && atomicAdd(&bar->exits, 1u) == gridDim.x - 1) {
    bar->count = 0;
    bar->exits = 0;
  }
}

}  // namespace detail
}  // namespace sygraph
