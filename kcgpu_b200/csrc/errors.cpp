// Status messages of the C ABI: the thread-local message behind
// kc_last_error(), the status names, and the CUDA-error conversion. Shared by
// the engine (libkc.so) and the host-only generator library (libkcgen.so).
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <string>

#include "host_common.h"

namespace kc {

namespace {
thread_local std::string g_last_error;
}

kc_status fail(kc_status st, const char* fmt, ...) {
  char buf[1024];
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(buf, sizeof(buf), fmt, ap);
  va_end(ap);
  g_last_error = buf;
  // a failing call leaves no pending (non-sticky) CUDA error for the next one
  cudaGetLastError();
  return st;
}

void clear_error() { g_last_error.clear(); }

kc_status cuda_fail(cudaError_t e, const char* what, const char* file, int line) {
  cudaGetLastError();
  const char* base = std::strrchr(file, '/');
  base = base ? base + 1 : file;
  kc_status st = (e == cudaErrorMemoryAllocation) ? KC_ERR_OOM : KC_ERR_CUDA;
  return fail(st, "%s failed: %s (%s:%d)", what, cudaGetErrorString(e), base, line);
}

}  // namespace kc

extern "C" {

const char* kc_last_error(void) { return kc::g_last_error.c_str(); }

const char* kc_status_string(kc_status s) {
  switch (s) {
    case KC_OK: return "ok";
    case KC_ERR_INVALID_ARG: return "invalid argument";
    case KC_ERR_OOM: return "out of memory";
    case KC_ERR_ADMISSION: return "admission rejected";
    case KC_ERR_DEVICE_TIMEOUT: return "device time limit exceeded";
    case KC_ERR_CUDA: return "CUDA error";
    case KC_ERR_INTERNAL: return "internal error";
    case KC_ERR_NOT_ORIENTED: return "graph not oriented";
    case KC_ERR_CANCELLED: return "cancelled";
    case KC_ERR_BUSY: return "busy";
  }
  return "unknown status";
}

}  // extern "C"
