// CSR build on the GPU: edge list -> symmetric CSR with sorted rows, no
// self-loops and no duplicate edges.
//
// Replaces the host path of the reference: EdgeListFile::get_edges reading 100
// edges per call, std::sort and CSRCOO::from_edgelist (include/FIleReader.cuh:
// 383-411, include/CSRCOO.cuh:37-80), which drops self-loops but neither
// symmetrises nor deduplicates and needs input sorted by source.
//
// Passes (all HBM-bound):
//   1. max id + per-vertex degree of the symmetrised multigraph (atomics),
//   2. exclusive scan -> row offsets,
//   3. scatter both directions of every edge (atomic row cursors),
//   4. per-row sort + dedup in registers / shared memory,
//   5. scan of the distinct counts and an ordered row compaction.
#include <algorithm>

#include "dev_common.cuh"
#include "engine.h"
#include "prims.cuh"

namespace kc {

namespace {

__global__ void k_max_id(const uint32_t* __restrict__ src, const uint32_t* __restrict__ dst, uint64_t E,
                         uint32_t* out) {
  uint32_t mx = 0;
  for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < E; i += (uint64_t)gridDim.x * blockDim.x)
    mx = max(mx, max(src[i], dst[i]));
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) mx = max(mx, __shfl_xor_sync(0xffffffffu, mx, o));
  if (lane_id() == 0 && mx) atomicMax(out, mx);
}

// Edge lists usually arrive grouped by source (generators, sorted files), so
// the lanes of a warp often share a source row: its counter is bumped once per
// group of equal sources (__match_any_sync), not once per lane. Whole warps
// walk the grid-stride loop together; lanes past the end or on a self-loop
// carry the key 0xffffffff and do nothing.
__device__ __forceinline__ uint32_t grouped_add(uint32_t* ctr, uint32_t key, uint32_t lane) {
  const uint32_t peers = __match_any_sync(0xffffffffu, key);
  const uint32_t leader = (uint32_t)__ffs(peers) - 1u;
  uint32_t base = 0;
  if (lane == leader && key != 0xffffffffu) base = atomicAdd(&ctr[key], (uint32_t)__popc(peers));
  base = __shfl_sync(0xffffffffu, base, leader);
  return base + (uint32_t)__popc(peers & lanemask_lt());
}

// Also checks every endpoint against n (a known vertex count): an edge with
// an endpoint >= n sets *bad to 1 and is not counted (the build then fails).
__global__ void k_degree(const uint32_t* __restrict__ src, const uint32_t* __restrict__ dst, uint64_t E,
                         uint32_t n, uint32_t* deg, uint32_t* bad) {
  const uint32_t lane = lane_id();
  const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
  for (uint64_t b = (uint64_t)blockIdx.x * blockDim.x + (threadIdx.x & ~31u); b < E; b += stride) {
    const uint64_t i = b + lane;
    uint32_t u = 0xffffffffu, v = 0xffffffffu;
    if (i < E) {
      u = src[i];
      v = dst[i];
      if (u >= n || v >= n) {
        atomicOr(bad, 1u);
        u = v = 0xffffffffu;
      }
      if (u == v) u = v = 0xffffffffu;
    }
    grouped_add(deg, u, lane);
    if (v != 0xffffffffu) atomicAdd(&deg[v], 1u);
  }
}

__global__ void k_scatter(const uint32_t* __restrict__ src, const uint32_t* __restrict__ dst, uint64_t E,
                          uint32_t* cursor, uint32_t* adj) {
  const uint32_t lane = lane_id();
  const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
  for (uint64_t b = (uint64_t)blockIdx.x * blockDim.x + (threadIdx.x & ~31u); b < E; b += stride) {
    const uint64_t i = b + lane;
    uint32_t u = 0xffffffffu, v = 0xffffffffu;
    if (i < E) {
      u = src[i];
      v = dst[i];
      if (u == v) u = v = 0xffffffffu;
    }
    const uint32_t pu = grouped_add(cursor, u, lane);
    if (u != 0xffffffffu) {
      adj[pu] = v;
      adj[atomicAdd(&cursor[v], 1u)] = u;
    }
  }
}

__global__ void k_max_row(const uint32_t* __restrict__ off, uint32_t n, uint32_t* out) {
  uint32_t mx = 0;
  for (uint32_t v = blockIdx.x * blockDim.x + threadIdx.x; v < n; v += gridDim.x * blockDim.x)
    mx = max(mx, off[v + 1] - off[v]);
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) mx = max(mx, __shfl_xor_sync(0xffffffffu, mx, o));
  if (lane_id() == 0 && mx) atomicMax(out, mx);
}

}  // namespace

kc_status build_csr(kc_graph* g, const uint32_t* d_src, const uint32_t* d_dst, uint64_t E, uint32_t n_nodes) {
  cudaStream_t s = g->ctx->stream;
  const int sms = g->ctx->sms;
  const uint32_t grid_e = (uint32_t)std::max<uint64_t>(1, std::min<uint64_t>((E + 255) / 256, (uint64_t)sms * 16));

  DevTemps tmp(s);
  uint32_t* scal = nullptr;  // [0] max id, [1] max row length (with duplicates), [2] max degree
  KC_CUDA(tmp.alloc(&scal, 4 * sizeof(uint32_t)));
  KC_CUDA(cudaMemsetAsync(scal, 0, 4 * sizeof(uint32_t), s));
  uint32_t h[4] = {0, 0, 0, 0};
  // scal[3]: an endpoint >= n was seen (checked by k_degree)
  uint32_t n = n_nodes;
  if (n == 0 && E) {  // n from the largest id; a known n needs no extra pass
    k_max_id<<<grid_e, 256, 0, s>>>(d_src, d_dst, E, scal);
    KC_CUDA(cudaGetLastError());
    KC_CUDA(cudaMemcpyAsync(h, scal, sizeof(uint32_t), cudaMemcpyDeviceToHost, s));
    KC_CUDA(cudaStreamSynchronize(s));
    if (h[0] == 0xffffffffu) return fail(KC_ERR_INVALID_ARG, "vertex id 0xffffffff is reserved");
    n = h[0] + 1;
  }
  if (2 * E >= 0xffffffffull)
    return fail(KC_ERR_INVALID_ARG, "%llu input edges exceed the 32-bit offset range", (unsigned long long)E);
  g->n = n;

  uint32_t *deg = nullptr, *off = nullptr, *adj = nullptr, *ucnt = nullptr;
  KC_CUDA(tmp.alloc(&deg, sizeof(uint32_t) * ((size_t)n + 1)));
  KC_CUDA(tmp.alloc(&off, sizeof(uint32_t) * ((size_t)n + 1)));
  KC_CUDA(cudaMemsetAsync(deg, 0, sizeof(uint32_t) * ((size_t)n + 1), s));
  if (E) k_degree<<<grid_e, 256, 0, s>>>(d_src, d_dst, E, n, deg, scal + 3);
  KC_CUDA(prim::scan_exclusive_u32(deg, off, n, s));
  uint32_t total = 0;
  KC_CUDA(cudaMemcpyAsync(&total, off + n, sizeof(uint32_t), cudaMemcpyDeviceToHost, s));
  if (n) k_max_row<<<std::max(1u, std::min((n + 255) / 256, (uint32_t)sms * 8)), 256, 0, s>>>(off, n, scal + 1);
  KC_CUDA(cudaMemcpyAsync(h + 1, scal + 1, 3 * sizeof(uint32_t), cudaMemcpyDeviceToHost, s));
  KC_CUDA(cudaStreamSynchronize(s));
  if (h[3]) return fail(KC_ERR_INVALID_ARG, "an edge endpoint is not below n_nodes = %u", n);

  KC_CUDA(tmp.alloc(&adj, sizeof(uint32_t) * std::max<size_t>(1, total)));
  // deg is reused as the scatter cursor (a copy of the offsets)
  KC_CUDA(cudaMemcpyAsync(deg, off, sizeof(uint32_t) * ((size_t)n + 1), cudaMemcpyDeviceToDevice, s));
  if (E) k_scatter<<<grid_e, 256, 0, s>>>(d_src, d_dst, E, deg, adj);
  KC_CUDA(cudaGetLastError());

  KC_CUDA(tmp.alloc(&ucnt, sizeof(uint32_t) * ((size_t)n + 1)));
  KC_CUDA(prim::segmented_sort_unique(off, adj, ucnt, n, h[1], s));

  // final offsets and compaction into the graph's own arrays
  KC_TRY(dev_alloc(g, (void**)&g->rp, sizeof(uint32_t) * ((size_t)n + 1)));
  KC_CUDA(prim::scan_exclusive_u32(ucnt, g->rp, n, s));
  uint32_t m2 = 0;
  KC_CUDA(cudaMemcpyAsync(&m2, g->rp + n, sizeof(uint32_t), cudaMemcpyDeviceToHost, s));
  if (n) k_max_row<<<std::max(1u, std::min((n + 255) / 256, (uint32_t)sms * 8)), 256, 0, s>>>(g->rp, n, scal + 2);
  KC_CUDA(cudaMemcpyAsync(h + 2, scal + 2, sizeof(uint32_t), cudaMemcpyDeviceToHost, s));
  KC_CUDA(cudaStreamSynchronize(s));
  KC_TRY(dev_alloc(g, (void**)&g->col, sizeof(uint32_t) * std::max<size_t>(1, m2)));
  KC_CUDA(prim::compact_rows(off, adj, g->rp, g->col, n, s));
  g->m = m2 / 2;
  g->max_deg = h[2];
  KC_CUDA(cudaGetLastError());
  return KC_OK;
}

}  // namespace kc
