// Device-allocation hook of the library, for fault-injection tests (host only).
//
// Every device allocation and free the engine makes goes through
// cudaMalloc / cudaMallocAsync / cudaFree / cudaFreeAsync, and the link step
// wraps those four (ld --wrap, kcgpu_b200/build.py), so this file sees them
// all. Two test facilities come out of it, both declared in include/kc.h:
//  * kc_test_fail_alloc_after(n): the (n+1)-th device allocation from now
//    fails with cudaErrorMemoryAllocation, which the engine reports as
//    KC_ERR_OOM; the real allocator is not called, so no CUDA state changes.
//    One failure, then the hook disarms itself; n < 0 disarms it.
//  * kc_test_live_allocations(): device allocations made and not yet freed,
//    so a test can check that a failing call leaks nothing.
// Without a test arming it the hook costs one atomic load per allocation plus
// the bookkeeping of the live set.
#include <atomic>
#include <cstdint>
#include <mutex>
#include <unordered_set>

#include <cuda_runtime.h>

namespace {

std::atomic<int64_t> g_fail_after{-1};
std::mutex g_mu;
std::unordered_set<void*>* g_live = nullptr;  // never destroyed: frees may come from static destructors

bool take_failure() {
  int64_t v = g_fail_after.load(std::memory_order_relaxed);
  while (v >= 0) {
    const int64_t next = v == 0 ? -1 : v - 1;
    if (g_fail_after.compare_exchange_weak(v, next, std::memory_order_relaxed)) return v == 0;
  }
  return false;
}

void track(void* p) {
  std::lock_guard<std::mutex> l(g_mu);
  if (!g_live) g_live = new std::unordered_set<void*>();
  g_live->insert(p);
}

void untrack(void* p) {
  if (!p) return;
  std::lock_guard<std::mutex> l(g_mu);
  if (g_live) g_live->erase(p);
}

}  // namespace

extern "C" {

cudaError_t __real_cudaMalloc(void** p, size_t n);
cudaError_t __real_cudaMallocAsync(void** p, size_t n, cudaStream_t s);
cudaError_t __real_cudaFree(void* p);
cudaError_t __real_cudaFreeAsync(void* p, cudaStream_t s);

cudaError_t __wrap_cudaMalloc(void** p, size_t n) {
  if (take_failure()) {
    if (p) *p = nullptr;
    return cudaErrorMemoryAllocation;
  }
  const cudaError_t e = __real_cudaMalloc(p, n);
  if (e == cudaSuccess) track(*p);
  return e;
}

cudaError_t __wrap_cudaMallocAsync(void** p, size_t n, cudaStream_t s) {
  if (take_failure()) {
    if (p) *p = nullptr;
    return cudaErrorMemoryAllocation;
  }
  const cudaError_t e = __real_cudaMallocAsync(p, n, s);
  if (e == cudaSuccess) track(*p);
  return e;
}

cudaError_t __wrap_cudaFree(void* p) {
  untrack(p);
  return __real_cudaFree(p);
}

cudaError_t __wrap_cudaFreeAsync(void* p, cudaStream_t s) {
  untrack(p);
  return __real_cudaFreeAsync(p, s);
}

void kc_test_fail_alloc_after(int64_t n) { g_fail_after.store(n < 0 ? -1 : n, std::memory_order_relaxed); }

uint64_t kc_test_live_allocations(void) {
  std::lock_guard<std::mutex> l(g_mu);
  return g_live ? (uint64_t)g_live->size() : 0u;
}

}  // extern "C"
