// k-truss support without any allocation.
//
// Same result as kc_truss_support (sup(u,v) = |N(u) ∩ N(v)| for every
// undirected edge u < v, in the row-major order of the upper triangle), but
// for callers that cannot allocate device memory at call time:
//   * code running on a latency-critical stream, where cudaMalloc / cudaFree
//     (and the stream-ordered pool growing) can stall or synchronise work on
//     other streams;
//   * plugins hosted by another runtime (an inference server, a framework
//     operator) that owns all device memory through its own allocator and
//     forbids allocations behind its back;
//   * pipelines that reserve every byte up front so a call can never fail
//     with out-of-memory halfway through.
// The caller passes a device CSR and a device output buffer; the only extra
// memory is the fixed array below, compiled into the library.
//
// Limits and sharing rules:
//   * n_nodes <= KC_NOALLOC_MAX_ROWS (262,144); larger graphs are rejected
//     with KC_ERR_INVALID_ARG before anything is launched;
//   * every GPU that loads this library holds the array (1 MiB) until the
//     process exits;
//   * all calls on a device share the one array, and each call leaves its own
//     offsets in it; calls whose work overlaps on the GPU (different streams,
//     no ordering between them) race on it and must be serialised by the
//     caller;
//   * the first call on each device looks up the array's device address
//     (cudaGetSymbolAddress, with that device current) and caches it; make
//     that first call before any stream capture begins;
//   * the cached address belongs to the device's primary context: after
//     cudaDeviceReset (which destroys that context and the array in it) this
//     entry point must not be called again in the process.
#include <algorithm>
#include <mutex>

#include "dev_common.cuh"
#include "engine.h"

namespace {

constexpr uint32_t kMaxRows = 1u << 18;
constexpr uint32_t kScanThreads = 1024;

// Per-row offsets of the upper-triangle edges (kMaxRows + 1 entries).
static __device__ __align__(256) uint32_t g_noalloc_rows[kMaxRows + 1];

std::mutex g_setup_mu;
uint32_t* g_rows_addr[256] = {nullptr};  // device address of the array, per device ordinal

// Looks up the array's device address once per device (that device current).
kc_status scratch_for_current_device(uint32_t** out) {
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return kc::cuda_fail(e, "cudaGetDevice", __FILE__, __LINE__);
  if (dev < 0 || dev >= 256) return kc::fail(KC_ERR_INVALID_ARG, "device ordinal %d out of range", dev);
  std::lock_guard<std::mutex> l(g_setup_mu);
  if (!g_rows_addr[dev]) {
    void* p = nullptr;
    e = cudaGetSymbolAddress(&p, g_noalloc_rows);
    if (e != cudaSuccess) return kc::cuda_fail(e, "cudaGetSymbolAddress(g_noalloc_rows)", __FILE__, __LINE__);
    g_rows_addr[dev] = static_cast<uint32_t*>(p);
  }
  *out = g_rows_addr[dev];
  return KC_OK;
}

// rows[u] = number of neighbours of u larger than u (every entry rewritten).
__global__ void k_noalloc_upper(const uint32_t* __restrict__ rp, const uint32_t* __restrict__ col, uint32_t n,
                                uint32_t* rows) {
  for (uint32_t u = blockIdx.x * blockDim.x + threadIdx.x; u <= n; u += gridDim.x * blockDim.x) {
    if (u == n) {
      rows[n] = 0;
      continue;
    }
    const uint32_t b = rp[u], e = rp[u + 1];
    rows[u] = e - b - kc::lower_bound_u32(col + b, e - b, u + 1);
  }
}

// One block: exclusive scan of rows[0, n] in place (rows[n] becomes the edge count).
__global__ void __launch_bounds__(kScanThreads) k_noalloc_scan(uint32_t n, uint32_t* rows) {
  __shared__ uint32_t warp_tot[kScanThreads / 32];
  __shared__ uint32_t carry;
  const uint32_t lane = threadIdx.x & 31u, w = threadIdx.x >> 5;
  if (threadIdx.x == 0) carry = 0;
  __syncthreads();
  for (uint32_t base = 0; base <= n; base += kScanThreads) {
    const uint32_t i = base + threadIdx.x;
    const uint32_t v = i <= n ? rows[i] : 0u;
    uint32_t inc = v;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const uint32_t t = __shfl_up_sync(0xffffffffu, inc, o);
      if (lane >= (uint32_t)o) inc += t;
    }
    if (lane == 31) warp_tot[w] = inc;
    __syncthreads();
    if (w == 0) {
      const uint32_t x = warp_tot[lane];
      uint32_t xi = x;
#pragma unroll
      for (int o = 1; o < 32; o <<= 1) {
        const uint32_t t = __shfl_up_sync(0xffffffffu, xi, o);
        if (lane >= (uint32_t)o) xi += t;
      }
      warp_tot[lane] = xi - x;
    }
    __syncthreads();
    const uint32_t c = carry;
    if (i <= n) rows[i] = c + warp_tot[w] + inc - v;
    __syncthreads();
    if (threadIdx.x == kScanThreads - 1) carry = c + warp_tot[w] + inc;
    __syncthreads();
  }
}

// One warp per upper edge e (edge count read from rows[n] on the device).
__global__ void k_noalloc_support(const uint32_t* __restrict__ rp, const uint32_t* __restrict__ col, uint32_t n,
                                  const uint32_t* __restrict__ rows, uint32_t* sup) {
  const uint32_t lane = threadIdx.x & 31u;
  const uint32_t gw = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, nw = (gridDim.x * blockDim.x) >> 5;
  const uint32_t m = rows[n];
  for (uint32_t e = gw; e < m; e += nw) {
    uint32_t lo = 0, hi = n;
    while (hi - lo > 1) {
      const uint32_t mid = (lo + hi) >> 1;
      if (rows[mid] <= e) lo = mid; else hi = mid;
    }
    const uint32_t u = lo;
    const uint32_t ub = rp[u], ue = rp[u + 1];
    const uint32_t first_upper = ue - (rows[u + 1] - rows[u]);
    const uint32_t v = col[first_upper + (e - rows[u])];
    const uint32_t vb = rp[v], ve = rp[v + 1];
    const uint32_t *A, *L;
    uint32_t la, ll;
    if (ue - ub <= ve - vb) { A = col + ub; la = ue - ub; L = col + vb; ll = ve - vb; }
    else { A = col + vb; la = ve - vb; L = col + ub; ll = ue - ub; }
    uint32_t c = 0;
    for (uint32_t i0 = 0; i0 < la; i0 += 32) {
      const uint32_t i = i0 + lane;
      bool hit = false;
      if (i < la) {
        const uint32_t x = A[i];
        const uint32_t pos = kc::lower_bound_u32(L, ll, x);
        hit = pos < ll && L[pos] == x;
      }
      c += __popc(__ballot_sync(0xffffffffu, hit));
    }
    if (lane == 0) sup[e] = c;
  }
}

}  // namespace

extern "C" {

kc_status kc_truss_support_noalloc(const uint32_t* d_row_ptr, const uint32_t* d_col_ind, uint32_t n_nodes,
                                   uint32_t* d_support, void* stream) {
  kc::clear_error();
  if (n_nodes > kMaxRows)
    return kc::fail(KC_ERR_INVALID_ARG,
                    "kc_truss_support_noalloc handles at most %u vertices (got %u); use kc_truss_support",
                    kMaxRows, n_nodes);
  if (!d_row_ptr || (n_nodes && (!d_col_ind || !d_support)))
    return kc::fail(KC_ERR_INVALID_ARG, "NULL argument");
  uint32_t* rows = nullptr;
  KC_TRY(scratch_for_current_device(&rows));
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  int dev = 0, sms = 148;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  const uint32_t g1 = std::max(1u, std::min((n_nodes + 1 + 255) / 256, (uint32_t)sms * 8));
  k_noalloc_upper<<<g1, 256, 0, s>>>(d_row_ptr, d_col_ind, n_nodes, rows);
  k_noalloc_scan<<<1, kScanThreads, 0, s>>>(n_nodes, rows);
  k_noalloc_support<<<(uint32_t)sms * 16, 256, 0, s>>>(d_row_ptr, d_col_ind, n_nodes, rows, d_support);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return kc::cuda_fail(e, "kc_truss_support_noalloc launch", __FILE__, __LINE__);
  return KC_OK;
}

}  // extern "C"
