// k-truss support: sup(u,v) = |N(u) ∩ N(v)| for every undirected edge.
//
// The reference parses `-m ktruss` (include/Config.h:66-67) but never
// dispatches it; its only truss code is peeling helpers (truss/kernels.cuh).
// This kernel defines the operation the engine exports: one support value
// per edge u < v, in the row-major order of the symmetric CSR's upper
// triangle.
//
// One warp per edge, grid-stride over the edges: the warp streams the shorter
// adjacency list with coalesced loads and locates each element in the longer
// one by binary search; the hits are counted with one ballot per 32 elements.
#include <algorithm>

#include "dev_common.cuh"
#include "engine.h"
#include "prims.cuh"

namespace kc {

namespace {

// Number of neighbours of u that are larger than u.
__global__ void k_upper_count(const uint32_t* __restrict__ rp, const uint32_t* __restrict__ col, uint32_t n,
                              uint32_t* cnt) {
  for (uint32_t u = blockIdx.x * blockDim.x + threadIdx.x; u < n; u += gridDim.x * blockDim.x) {
    const uint32_t b = rp[u], e = rp[u + 1];
    cnt[u] = e - b - lower_bound_u32(col + b, e - b, u + 1);
  }
}

__global__ void k_support(const uint32_t* __restrict__ rp, const uint32_t* __restrict__ col, uint32_t n,
                          const uint32_t* __restrict__ ubase, uint32_t m, uint32_t* sup) {
  const uint32_t lane = lane_id();
  const uint32_t gw = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, nw = (gridDim.x * blockDim.x) >> 5;
  for (uint32_t e = gw; e < m; e += nw) {
    // row of edge e: last u with ubase[u] <= e
    uint32_t lo = 0, hi = n;
    while (hi - lo > 1) {
      const uint32_t mid = (lo + hi) >> 1;
      if (ubase[mid] <= e) lo = mid; else hi = mid;
    }
    const uint32_t u = lo;
    const uint32_t ub = rp[u], ue = rp[u + 1];
    const uint32_t first_upper = ue - (ubase[u + 1] - ubase[u]);
    const uint32_t v = col[first_upper + (e - ubase[u])];
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
        const uint32_t pos = lower_bound_u32(L, ll, x);
        hit = pos < ll && L[pos] == x;
      }
      c += __popc(__ballot_sync(0xffffffffu, hit));
    }
    if (lane == 0) sup[e] = c;
  }
}

}  // namespace

kc_status truss_support(kc_graph* g, uint32_t* d_support) {
  kc_ctx* ctx = g->ctx;
  cudaStream_t s = ctx->stream;
  const uint32_t n = g->n;
  if (g->m == 0) return KC_OK;
  DevTemps t(s);
  uint32_t *cnt = nullptr, *ubase = nullptr;
  KC_CUDA(t.alloc(&cnt, sizeof(uint32_t) * ((size_t)n + 1)));
  KC_CUDA(t.alloc(&ubase, sizeof(uint32_t) * ((size_t)n + 1)));
  const uint32_t g1 = (uint32_t)std::max<uint64_t>(1, std::min<uint64_t>((n + 255) / 256, (uint64_t)ctx->sms * 16));
  k_upper_count<<<g1, 256, 0, s>>>(g->rp, g->col, n, cnt);
  KC_CUDA(prim::scan_exclusive_u32(cnt, ubase, n, s));
  const uint32_t g2 = (uint32_t)std::max<uint64_t>(1, std::min<uint64_t>((g->m * 32 + 255) / 256, (uint64_t)ctx->sms * 32));
  k_support<<<g2, 256, 0, s>>>(g->rp, g->col, n, ubase, (uint32_t)g->m, d_support);
  KC_CUDA(cudaGetLastError());
  return KC_OK;
}

}  // namespace kc
