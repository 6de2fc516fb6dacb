// Device-side helpers shared by the engine's kernels.
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

namespace kc {

// Error word written by kernels that detect a violated invariant; the host
// reads it after the stage and turns a non-zero value into KC_ERR_INTERNAL or
// KC_ERR_DEVICE_TIMEOUT. Kernels never trap.
enum DevErr : uint32_t {
  DEV_OK = 0,
  DEV_ERR_STACK = 1,      // traversal deeper than the allocated stack
  DEV_ERR_CAPACITY = 2,   // a unit larger than its class capacity
  DEV_ERR_TIMEOUT = 3,    // a bounded wait ran out
  DEV_ERR_INPUT = 4,      // malformed input detected on the device
};

__device__ __forceinline__ void set_error(uint32_t* err, uint32_t code) {
  if (err) atomicCAS(err, 0u, code);
}

__device__ __forceinline__ uint32_t lane_id() { return threadIdx.x & 31u; }

__device__ __forceinline__ uint32_t lanemask_lt() {
  uint32_t m;
  asm volatile("mov.u32 %0, %%lanemask_lt;" : "=r"(m));
  return m;
}

// Exact 128-bit accumulation with two 64-bit atomics: the carry out of the low
// word is added to the high word, so concurrent additions commute exactly.
__device__ __forceinline__ void atomic_add_u128(unsigned long long* p, unsigned __int128 v) {
  unsigned long long lo = (unsigned long long)v;
  unsigned long long hi = (unsigned long long)(v >> 64);
  if (lo) {
    unsigned long long old = atomicAdd(p, lo);
    if (old + lo < old) hi += 1ull;
  }
  if (hi) atomicAdd(p + 1, hi);
}

__device__ __forceinline__ unsigned long long ld_u64(const unsigned long long* p) { return *p; }

// Partition mask: P consecutive lanes of the warp starting at the lane's group.
__device__ __forceinline__ uint32_t part_mask(uint32_t P) {
  if (P >= 32) return 0xffffffffu;
  uint32_t base = (lane_id() / P) * P;
  return ((1u << P) - 1u) << base;
}

template <class T>
__host__ __device__ __forceinline__ T ceil_div(T a, T b) { return (a + b - 1) / b; }

// Lower bound of x in the sorted array a[0, n).
__device__ __forceinline__ uint32_t lower_bound_u32(const uint32_t* a, uint32_t n, uint32_t x) {
  uint32_t lo = 0, hi = n;
  while (lo < hi) {
    uint32_t mid = (lo + hi) >> 1;
    if (a[mid] < x) lo = mid + 1; else hi = mid;
  }
  return lo;
}

}  // namespace kc
