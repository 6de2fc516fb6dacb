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
  DEV_ERR_BOUNDS = 5,     // a scratch index out of its array (KC_CHECKED builds only)
};

__device__ __forceinline__ void set_error(uint32_t* err, uint32_t code) {
  if (err) atomicCAS(err, 0u, code);
}

// KC_IN_BOUNDS(i, n, err): in a KC_CHECKED build, true when i < n and
// otherwise records DEV_ERR_BOUNDS and returns false, so the caller skips the
// access; in a normal build, true (no code). The checked library
// (libkc_checked.so) stands in for the closed compute-sanitizer.
#ifdef KC_CHECKED
#define KC_IN_BOUNDS(i, n, err) ((uint64_t)(i) < (uint64_t)(n) ? true : (::kc::set_error((err), ::kc::DEV_ERR_BOUNDS), false))
#else
#define KC_IN_BOUNDS(i, n, err) true
#endif

__device__ __forceinline__ uint32_t lane_id() { return threadIdx.x & 31u; }

// The GPU's global timer in nanoseconds (same epoch on every SM).
__device__ __forceinline__ unsigned long long global_ns() {
  unsigned long long t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}

// True when a counting pass with a device time limit has run past it; t0 is
// the pass's start, written by the queue set-up before any counting kernel.
__device__ __forceinline__ bool past_limit(unsigned long long limit_ns, const unsigned long long* t0) {
  return limit_ns != 0ull && global_ns() - *(volatile const unsigned long long*)t0 > limit_ns;
}

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
