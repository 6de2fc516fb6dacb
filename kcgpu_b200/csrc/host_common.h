// Host-side helpers shared by the engine's C++ translation units: the
// thread-local error message behind kc_last_error(), CUDA call checking, and
// a small scope timer.
#pragma once
#include <chrono>
#include <cstdarg>
#include <cstdint>
#include <cstdio>
#include <string>

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
