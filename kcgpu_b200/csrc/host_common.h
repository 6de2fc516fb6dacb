// Host-side helpers shared by the engine's C++ translation units: the
// thread-local error message behind kc_last_error(), CUDA call checking, and
// a small scope timer.
#pragma once
#include <chrono>
#include <cstdarg>
#include <cstdint>
#include <cstdio>
#include <map>
#include <mutex>
#include <string>
#include <unordered_map>
#include <vector>

#include <cuda_runtime.h>

#include "../../include/kc.h"

namespace kc {

// Records a message for kc_last_error() and returns the status unchanged.
kc_status fail(kc_status st, const char* fmt, ...)
#if defined(__GNUC__)
    __attribute__((format(printf, 2, 3)))
#endif
    ;

void clear_error();

// Converts a CUDA error into KC_ERR_CUDA / KC_ERR_OOM with the call site.
kc_status cuda_fail(cudaError_t e, const char* what, const char* file, int line);

inline double now_ms() {
  using namespace std::chrono;
  return duration<double, std::milli>(steady_clock::now().time_since_epoch()).count();
}

// Per-context cache of device blocks (devmem.cpp): blocks freed on the
// context's stream are reused by later allocations on that stream.
class BlockCache {
 public:
  cudaError_t get(void** p, size_t bytes, cudaStream_t s);
  void put(void* p, cudaStream_t s);
  void release(cudaStream_t s);  // returns every free block to the driver
  uint64_t cached_bytes();

 private:
  std::mutex mu_;
  std::multimap<size_t, void*> free_;
  std::unordered_map<void*, size_t> size_;  // every block of this cache, free or in use
  uint64_t free_bytes_ = 0;
};

// The cache serving allocations on stream s (a context's stream).
void register_stream_cache(cudaStream_t s, BlockCache* c);
void unregister_stream_cache(cudaStream_t s);

// Every device allocation of the engine: from the cache registered for s,
// else straight from the stream-ordered allocator; dfree returns the block
// the same way (stream-ordered on s).
cudaError_t dmalloc_raw(void** p, size_t bytes, cudaStream_t s);
template <class T>
cudaError_t dmalloc(T** p, size_t bytes, cudaStream_t s) {
  void* q = nullptr;
  const cudaError_t e = dmalloc_raw(&q, bytes, s);
  *p = static_cast<T*>(q);
  return e;
}
void dfree(void* p, cudaStream_t s);

// Device temporaries of one call: allocated on s and freed, stream-ordered,
// when the guard goes out of scope, so a call that fails half way leaks
// nothing. free_now() hands one back early to lower the peak.
class DevTemps {
 public:
  explicit DevTemps(cudaStream_t s) : s_(s) {}
  ~DevTemps() {
    for (void* p : ps_) dfree(p, s_);
  }
  DevTemps(const DevTemps&) = delete;
  DevTemps& operator=(const DevTemps&) = delete;

  template <class T>
  cudaError_t alloc(T** p, size_t bytes) {
    void* q = nullptr;
    const cudaError_t e = dmalloc_raw(&q, bytes, s_);
    *p = static_cast<T*>(q);
    if (e == cudaSuccess) ps_.push_back(q);
    return e;
  }

  void free_now(void* p) {
    for (size_t i = 0; i < ps_.size(); ++i)
      if (ps_[i] == p) {
        dfree(p, s_);
        ps_.erase(ps_.begin() + (long)i);
        return;
      }
  }

 private:
  cudaStream_t s_;
  std::vector<void*> ps_;
};

}  // namespace kc

// Returns from the enclosing function (which must return kc_status) on error.
#define KC_CUDA(call)                                                     \
  do {                                                                    \
    cudaError_t kc_e_ = (call);                                           \
    if (kc_e_ != cudaSuccess) return kc::cuda_fail(kc_e_, #call, __FILE__, __LINE__); \
  } while (0)

#define KC_TRY(expr)                        \
  do {                                      \
    kc_status kc_s_ = (expr);               \
    if (kc_s_ != KC_OK) return kc_s_;       \
  } while (0)
