// Orientation: degree order or degeneracy (k-core peeling) order, then the
// DAG CSR relabelled by rank.
//
// Reference behaviour kept:
//   * degree orientation keeps u->v iff deg u < deg v, or equal and u < v
//     (include/main_support.cuh:54-87 with node degrees, src/main.cu:181);
//   * degeneracy orientation keeps u->v iff prio u < prio v, or equal and
//     u < v (include/main_support.cuh:89-128), where prio is the peel
//     sub-round of SingleGPU_Kcore::findKcoreIncremental_async
//     (kcore/kcore.cuh:442-584): level L peels every vertex of current degree
//     L in sub-rounds, each sub-round's vertices get the running sub-round
//     counter (kcore.cuh:192 and :564) and the batch that empties the graph
//     keeps the initial value 2m (kcore.cuh:471-472, break at :496-498).
//
// B200 design: the whole peel runs in ONE cooperative persistent kernel with
// grid-wide barriers between phases (the reference launches kernels and
// synchronises the host per sub-round). The bucket of candidate vertices is
// compacted every level so a level scans only live low-degree vertices.
//
// The DAG is stored in rank labels: a vertex's label is its position in the
// orientation's total order, so every out-list holds larger labels only and
// the induced-subgraph bitmaps of the counting stage are upper-triangular.
#include <algorithm>
#include <cooperative_groups.h>

#include "dev_common.cuh"
#include "engine.h"
#include "prims.cuh"

namespace cg = cooperative_groups;

namespace kc {

namespace {

int bits_for(uint64_t x) {  // bits needed to hold values in [0, x]
  int b = 0;
  while (b < 64 && (x >> b) != 0) ++b;
  return b;
}

uint32_t grid_for(uint64_t work, int sms, int per_sm = 16) {
  return (uint32_t)std::max<uint64_t>(1, std::min<uint64_t>((work + 255) / 256, (uint64_t)sms * per_sm));
}

// Sort keys (graph, major, v): the graph field (batches only) is the most
// significant so each graph's vertices get a contiguous range of ranks; it
// never changes the order of two vertices of the same graph.
__global__ void k_degree_keys(const uint32_t* __restrict__ rp, uint32_t n, int vbits, const uint32_t* __restrict__ vg,
                              int gshift, unsigned long long* keys) {
  for (uint32_t v = blockIdx.x * blockDim.x + threadIdx.x; v < n; v += gridDim.x * blockDim.x) {
    unsigned long long k = ((unsigned long long)(rp[v + 1] - rp[v]) << vbits) | v;
    if (vg) k |= (unsigned long long)vg[v] << gshift;
    keys[v] = k;
  }
}

__global__ void k_prio_keys(const uint32_t* __restrict__ prio, uint32_t n, int vbits, uint32_t cap,
                            const uint32_t* __restrict__ vg, int gshift, unsigned long long* keys) {
  for (uint32_t v = blockIdx.x * blockDim.x + threadIdx.x; v < n; v += gridDim.x * blockDim.x) {
    unsigned long long k = ((unsigned long long)min(prio[v], cap) << vbits) | v;
    if (vg) k |= (unsigned long long)vg[v] << gshift;
    keys[v] = k;
  }
}

__global__ void k_rank_from_sorted(const unsigned long long* __restrict__ keys, uint32_t n,
                                   unsigned long long vmask, uint32_t* rank, uint32_t* inv) {
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    uint32_t v = (uint32_t)(keys[i] & vmask);
    inv[i] = v;
    rank[v] = i;
  }
}

// Warp per vertex: out-degree in rank order (neighbours of larger rank).
__global__ void k_out_degree(const uint32_t* __restrict__ rp, const uint32_t* __restrict__ col, uint32_t n,
                             const uint32_t* __restrict__ rank, uint32_t* odeg) {
  const uint32_t lane = lane_id();
  const uint32_t gw = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, nw = (gridDim.x * blockDim.x) >> 5;
  for (uint32_t v = gw; v < n; v += nw) {
    const uint32_t rv = rank[v], b = rp[v], e = rp[v + 1];
    uint32_t c = 0;
    for (uint32_t i = b + lane; i < e; i += 32) c += rank[col[i]] > rv;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) c += __shfl_xor_sync(0xffffffffu, c, o);
    if (lane == 0) odeg[rv] = c;
  }
}

__global__ void k_fill_dag(const uint32_t* __restrict__ rp, const uint32_t* __restrict__ col, uint32_t n,
                           const uint32_t* __restrict__ rank, const uint32_t* __restrict__ drp, uint32_t* dcol) {
  const uint32_t lane = lane_id();
  const uint32_t gw = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, nw = (gridDim.x * blockDim.x) >> 5;
  for (uint32_t v = gw; v < n; v += nw) {
    const uint32_t rv = rank[v], b = rp[v], e = rp[v + 1];
    uint32_t pos = drp[rv];
    for (uint32_t i0 = b; i0 < e; i0 += 32) {
      uint32_t i = i0 + lane;
      uint32_t rw = i < e ? rank[col[i]] : 0;
      bool keep = i < e && rw > rv;
      uint32_t bal = __ballot_sync(0xffffffffu, keep);
      if (keep) dcol[pos + __popc(bal & lanemask_lt())] = rw;
      pos += __popc(bal);
    }
  }
}

__global__ void k_edge_rows(const uint32_t* __restrict__ drp, uint32_t n, uint32_t* erow) {
  const uint32_t lane = lane_id();
  const uint32_t gw = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, nw = (gridDim.x * blockDim.x) >> 5;
  for (uint32_t r = gw; r < n; r += nw)
    for (uint32_t i = drp[r] + lane; i < drp[r + 1]; i += 32) erow[i] = r;
}

__global__ void k_max_row_len(const uint32_t* __restrict__ off, uint32_t n, uint32_t* out) {
  uint32_t mx = 0;
  for (uint32_t v = blockIdx.x * blockDim.x + threadIdx.x; v < n; v += gridDim.x * blockDim.x)
    mx = max(mx, off[v + 1] - off[v]);
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) mx = max(mx, __shfl_xor_sync(0xffffffffu, mx, o));
  if (lane_id() == 0 && mx) atomicMax(out, mx);
}

// Original-id export of the DAG (the reference's layout): row of original u =
// original ids of the out-neighbours of rank[u].
__global__ void k_export_deg(const uint32_t* __restrict__ drp, const uint32_t* __restrict__ rank, uint32_t n,
                             uint32_t* deg) {
  for (uint32_t u = blockIdx.x * blockDim.x + threadIdx.x; u < n; u += gridDim.x * blockDim.x)
    deg[u] = drp[rank[u] + 1] - drp[rank[u]];
}

__global__ void k_export_fill(const uint32_t* __restrict__ drp, const uint32_t* __restrict__ dcol,
                              const uint32_t* __restrict__ rank, const uint32_t* __restrict__ inv, uint32_t n,
                              const uint32_t* __restrict__ orp, uint32_t* ocol) {
  const uint32_t lane = lane_id();
  const uint32_t gw = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, nw = (gridDim.x * blockDim.x) >> 5;
  for (uint32_t u = gw; u < n; u += nw) {
    const uint32_t r = rank[u], b = drp[r], e = drp[r + 1], o = orp[u];
    for (uint32_t i = b + lane; i < e; i += 32) ocol[o + (i - b)] = inv[dcol[i]];
  }
}

// ---- degeneracy peel: one cooperative persistent kernel -----------------------

constexpr uint32_t PEEL_WINDOW = 64;  // degree window of the candidate bucket

struct PeelArgs {
  const uint32_t* rp;
  const uint32_t* col;
  uint32_t n;
  uint32_t init_prio;   // 2m: the priority the final batch keeps
  int* deg;             // current degree among live vertices
  uint32_t* prio;
  uint32_t* level;
  uint32_t* removed;    // 1 once peeled
  uint32_t* inbucket;   // 1 while in the candidate bucket
  uint32_t* bucket_a;   // candidate bucket (ping-pong, capacity n)
  uint32_t* bucket_b;
  uint32_t* front_a;    // frontier (ping-pong, capacity n)
  uint32_t* front_b;
  uint32_t* ctr;        // 4 phase slots x 4 counters, zeroed
  uint32_t* out;        // [0] last level, [1] sub-rounds, [2] error
};

__global__ void k_peel_init(const uint32_t* __restrict__ rp, uint32_t n, uint32_t init_prio, int* deg,
                            uint32_t* prio, uint32_t* level, uint32_t* removed, uint32_t* inbucket) {
  for (uint32_t v = blockIdx.x * blockDim.x + threadIdx.x; v < n; v += gridDim.x * blockDim.x) {
    deg[v] = (int)(rp[v + 1] - rp[v]);
    prio[v] = init_prio;
    level[v] = 0;
    removed[v] = 0;
    inbucket[v] = 0;
  }
}

// Appends x to list (for the lanes with pred) with one atomic per warp.
__device__ __forceinline__ void warp_append(bool pred, uint32_t x, uint32_t* list, uint32_t* cnt) {
  uint32_t m = __ballot_sync(0xffffffffu, pred);
  if (!m) return;
  uint32_t leader = __ffs(m) - 1, base = 0;
  if (lane_id() == leader) base = atomicAdd(cnt, (uint32_t)__popc(m));
  base = __shfl_sync(0xffffffffu, base, leader);
  if (pred) list[base + __popc(m & lanemask_lt())] = x;
}

// Every thread keeps an identical copy of the control state (level, sizes,
// priority, phase), derived from counters read after a grid barrier, so all
// threads take the same branches and reach the same barriers. Counters live in
// four phase slots; a phase zeroes the slot two phases ahead, which every
// thread has finished reading by then.
__global__ void __launch_bounds__(256) k_peel(PeelArgs a) {
  cg::grid_group grid = cg::this_grid();
  const uint32_t tid = blockIdx.x * blockDim.x + threadIdx.x;
  const uint32_t nthreads = gridDim.x * blockDim.x;
  const uint32_t lane = lane_id();
  const uint32_t gw = tid >> 5, nw = nthreads >> 5;
  uint32_t* bucket = a.bucket_a;
  uint32_t* bucket2 = a.bucket_b;
  uint32_t* front = a.front_a;
  uint32_t* next = a.front_b;
  uint64_t todo = a.n;
  uint32_t L = 0, bucket_end = 0, bsize = 0, priority = 0, phase = 0, subrounds = 0;
  auto slot = [&](uint32_t ph) { return a.ctr + (ph & 3u) * 4u; };
  auto begin_phase = [&]() {
    if (tid == 0) {
      uint32_t* z = slot(phase + 2);
      z[0] = z[1] = z[2] = z[3] = 0;
    }
  };
  while (todo > 0) {
    if (L > a.n) {  // cannot happen for a valid CSR; never spin
      if (tid == 0) a.out[2] = DEV_ERR_INPUT;
      break;
    }
    if (L == bucket_end) {
      begin_phase();
      uint32_t* c = slot(phase);
      for (uint32_t v0 = gw * 32; v0 < a.n; v0 += nw * 32) {
        uint32_t v = v0 + lane;
        bool in = false;
        if (v < a.n && !a.removed[v]) {
          int d = a.deg[v];
          in = d >= (int)L && d < (int)(L + PEEL_WINDOW);
          a.inbucket[v] = in ? 1u : 0u;
        }
        warp_append(in, v, bucket, &c[0]);
      }
      grid.sync();
      bsize = min(c[0], a.n);
      bucket_end = L + PEEL_WINDOW;
      ++phase;
    }
    // frontier of level L, and compaction of the bucket
    begin_phase();
    uint32_t* c = slot(phase);
    for (uint32_t i0 = gw * 32; i0 < bsize; i0 += nw * 32) {
      uint32_t i = i0 + lane;
      uint32_t v = i < bsize ? bucket[i] : 0;
      bool live = i < bsize && !a.removed[v];
      int d = live ? a.deg[v] : 0;
      warp_append(live && d == (int)L, v, front, &c[0]);
      warp_append(live && d != (int)L, v, bucket2, &c[1]);
    }
    grid.sync();
    uint32_t fsize = min(c[0], a.n);
    bsize = min(c[1], a.n);
    { uint32_t* t = bucket; bucket = bucket2; bucket2 = t; }
    ++phase;
    while (fsize > 0) {
      todo -= fsize;
      for (uint32_t i = tid; i < fsize; i += nthreads) a.level[front[i]] = L;
      if (todo == 0) break;  // the final batch keeps its initial priority
      for (uint32_t i = tid; i < fsize; i += nthreads) {
        a.prio[front[i]] = priority;
        a.removed[front[i]] = 1u;
      }
      begin_phase();
      grid.sync();
      uint32_t* c2 = slot(phase);
      for (uint32_t i = gw; i < fsize; i += nw) {
        const uint32_t v = front[i];
        const uint32_t b = a.rp[v], e = a.rp[v + 1];
        for (uint32_t j0 = b; j0 < e; j0 += 32) {
          uint32_t j = j0 + lane;
          bool to_next = false, to_bucket = false;
          uint32_t u = 0;
          if (j < e) {
            u = a.col[j];
            if (!a.removed[u]) {
              int cur = atomicSub(&a.deg[u], 1);
              if (cur == (int)L + 1) {
                to_next = true;
              } else {
                int now = cur - 1;
                if (now > (int)L && now < (int)bucket_end) to_bucket = atomicExch(&a.inbucket[u], 1u) == 0u;
              }
            }
          }
          warp_append(to_next, u, next, &c2[0]);
          warp_append(to_bucket, u, bucket + bsize, &c2[1]);
        }
      }
      grid.sync();
      fsize = min(c2[0], a.n);
      bsize = min(bsize + c2[1], a.n);
      { uint32_t* t = front; front = next; next = t; }
      ++priority;
      ++subrounds;
      ++phase;
    }
    if (todo == 0) break;
    ++L;
  }
  if (tid == 0) {
    a.out[0] = L;
    a.out[1] = subrounds;
  }
}

}  // namespace

namespace {

// The peel into prio / level (n >= 1); temporaries freed on every path.
kc_status run_peel(kc_graph* g, uint32_t* prio, uint32_t* level) {
  kc_ctx* ctx = g->ctx;
  cudaStream_t s = ctx->stream;
  const uint32_t n = g->n;
  DevTemps t(s);
  int* deg = nullptr;
  uint32_t *removed = nullptr, *inb = nullptr, *ba = nullptr, *bb = nullptr, *fa = nullptr, *fb = nullptr,
           *ctr = nullptr;
  KC_CUDA(t.alloc(&deg, sizeof(int) * n));
  KC_CUDA(t.alloc(&removed, sizeof(uint32_t) * n));
  KC_CUDA(t.alloc(&inb, sizeof(uint32_t) * n));
  KC_CUDA(t.alloc(&ba, sizeof(uint32_t) * n));
  KC_CUDA(t.alloc(&bb, sizeof(uint32_t) * n));
  KC_CUDA(t.alloc(&fa, sizeof(uint32_t) * n));
  KC_CUDA(t.alloc(&fb, sizeof(uint32_t) * n));
  KC_CUDA(t.alloc(&ctr, sizeof(uint32_t) * 32));
  KC_CUDA(cudaMemsetAsync(ctr, 0, sizeof(uint32_t) * 32, s));
  const uint32_t init_prio = (uint32_t)std::min<uint64_t>(2 * g->m, 0xffffffffull);
  k_peel_init<<<grid_for(n, ctx->sms), 256, 0, s>>>(g->rp, n, init_prio, deg, prio, level, removed, inb);
  KC_CUDA(cudaGetLastError());

  PeelArgs a;
  a.rp = g->rp; a.col = g->col; a.n = n; a.init_prio = init_prio;
  a.deg = deg; a.prio = prio; a.level = level; a.removed = removed; a.inbucket = inb;
  a.bucket_a = ba; a.bucket_b = bb; a.front_a = fa; a.front_b = fb; a.ctr = ctr; a.out = ctr + 16;
  int per_sm = 0;
  KC_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_peel, 256, 0));
  per_sm = std::max(1, std::min(per_sm, 4));
  dim3 grid(ctx->sms * per_sm), block(256);
  void* args[] = {&a};
  KC_CUDA(cudaLaunchCooperativeKernel((void*)k_peel, grid, block, args, 0, s));
  uint32_t out[3] = {0, 0, 0};
  KC_CUDA(cudaMemcpyAsync(out, ctr + 16, sizeof(out), cudaMemcpyDeviceToHost, s));
  KC_CUDA(cudaStreamSynchronize(s));
  if (out[2]) return fail(KC_ERR_INTERNAL, "peel did not converge (device error %u)", out[2]);
  g->max_core = out[0];
  g->peel_rounds = out[1];
  return KC_OK;
}

}  // namespace

// Peel priorities and core numbers of the graph; the graph keeps them only
// when the whole peel succeeded.
kc_status peel_graph(kc_graph* g) {
  if (g->prio) return KC_OK;
  const uint32_t n = g->n;
  uint32_t *prio = nullptr, *level = nullptr;
  KC_TRY(dev_alloc(g, (void**)&prio, sizeof(uint32_t) * std::max<size_t>(1, n)));
  kc_status st = dev_alloc(g, (void**)&level, sizeof(uint32_t) * std::max<size_t>(1, n));
  if (st == KC_OK && n == 0) g->max_core = 0;
  else if (st == KC_OK) st = run_peel(g, prio, level);
  if (st != KC_OK) {
    dev_free(g, prio);
    dev_free(g, level);
    return st;
  }
  g->prio = prio;
  g->level = level;
  return KC_OK;
}

kc_status orient_graph(kc_graph* g, uint32_t orientation) {
  if (orientation > KC_ORIENT_DEGEN) return fail(KC_ERR_INVALID_ARG, "unknown orientation %u", orientation);
  kc_ctx* ctx = g->ctx;
  cudaStream_t s = ctx->stream;
  const uint32_t n = g->n;
  if (g->oriented == (int)orientation) return KC_OK;
  // drop a previous orientation
  dev_free(g, g->rank); dev_free(g, g->inv); dev_free(g, g->drp); dev_free(g, g->dcol); dev_free(g, g->erow);
  g->rank = g->inv = g->drp = g->dcol = g->erow = nullptr;
  g->oriented = -1;
  if (orientation == KC_ORIENT_DEGEN) KC_TRY(peel_graph(g));

  KC_TRY(dev_alloc(g, (void**)&g->rank, sizeof(uint32_t) * std::max<size_t>(1, n)));
  KC_TRY(dev_alloc(g, (void**)&g->inv, sizeof(uint32_t) * std::max<size_t>(1, n)));
  KC_TRY(dev_alloc(g, (void**)&g->drp, sizeof(uint32_t) * ((size_t)n + 1)));
  KC_TRY(dev_alloc(g, (void**)&g->dcol, sizeof(uint32_t) * std::max<uint64_t>(1, g->m)));
  const int vbits = bits_for(n ? n - 1 : 0);
  DevTemps t(s);
  unsigned long long *keys = nullptr, *tmp = nullptr;
  uint32_t *odeg = nullptr, *ucnt = nullptr, *mx = nullptr;
  KC_CUDA(t.alloc(&keys, sizeof(unsigned long long) * std::max<size_t>(1, n)));
  KC_CUDA(t.alloc(&tmp, sizeof(unsigned long long) * std::max<size_t>(1, n)));
  KC_CUDA(t.alloc(&odeg, sizeof(uint32_t) * ((size_t)n + 1)));
  KC_CUDA(t.alloc(&ucnt, sizeof(uint32_t) * ((size_t)n + 1)));
  KC_CUDA(t.alloc(&mx, sizeof(uint32_t)));
  KC_CUDA(cudaMemsetAsync(mx, 0, sizeof(uint32_t), s));
  int major_bits;
  const int graph_bits = g->vgraph_orig ? bits_for(g->n_graphs ? g->n_graphs - 1 : 0) : 0;
  if (orientation == KC_ORIENT_DEGREE) {
    major_bits = bits_for(g->max_deg);
    k_degree_keys<<<grid_for(n, ctx->sms), 256, 0, s>>>(g->rp, n, vbits, g->vgraph_orig, vbits + major_bits, keys);
  } else {
    // Peel priorities are sub-round indices below peel_rounds, except the
    // final batch's 2m; capping that one at peel_rounds keeps every order and
    // keeps the key narrow.
    const uint32_t cap = (uint32_t)std::min<uint64_t>(std::min<uint64_t>(2 * g->m, 0xffffffffull), g->peel_rounds);
    major_bits = bits_for(cap);
    k_prio_keys<<<grid_for(n, ctx->sms), 256, 0, s>>>(g->prio, n, vbits, cap, g->vgraph_orig, vbits + major_bits,
                                                    keys);
  }
  KC_CUDA(cudaGetLastError());
  if (vbits + major_bits + graph_bits > 64) return fail(KC_ERR_INTERNAL, "orientation key exceeds 64 bits");
  KC_CUDA(prim::radix_sort_u64(keys, tmp, n, vbits + major_bits + graph_bits, s));
  k_rank_from_sorted<<<grid_for(n, ctx->sms), 256, 0, s>>>(keys, n, (vbits >= 64) ? ~0ull : ((1ull << vbits) - 1),
                                                          g->rank, g->inv);
  const uint32_t gw = grid_for((uint64_t)n * 32, ctx->sms, 32);
  k_out_degree<<<gw, 256, 0, s>>>(g->rp, g->col, n, g->rank, odeg);
  KC_CUDA(prim::scan_exclusive_u32(odeg, g->drp, n, s));
  k_fill_dag<<<gw, 256, 0, s>>>(g->rp, g->col, n, g->rank, g->drp, g->dcol);
  if (n) k_max_row_len<<<grid_for(n, ctx->sms), 256, 0, s>>>(g->drp, n, mx);
  uint32_t max_out = 0;
  KC_CUDA(cudaMemcpyAsync(&max_out, mx, sizeof(uint32_t), cudaMemcpyDeviceToHost, s));
  KC_CUDA(cudaStreamSynchronize(s));
  // out-lists in rank order (values are distinct, so dedup keeps them all)
  KC_CUDA(prim::segmented_sort_unique(g->drp, g->dcol, ucnt, n, max_out, s));
  KC_CUDA(cudaGetLastError());
  KC_CUDA(cudaStreamSynchronize(s));
  g->max_out = max_out;
  g->oriented = (int)orientation;
  return KC_OK;
}

kc_status ensure_edge_rows(kc_graph* g) {
  if (g->erow) return KC_OK;
  KC_TRY(dev_alloc(g, (void**)&g->erow, sizeof(uint32_t) * std::max<uint64_t>(1, g->m)));
  k_edge_rows<<<grid_for((uint64_t)g->n * 32, g->ctx->sms, 32), 256, 0, g->ctx->stream>>>(g->drp, g->n, g->erow);
  KC_CUDA(cudaGetLastError());
  return KC_OK;
}

// Exports the DAG in original ids with rows sorted by id (host buffers).
kc_status export_dag(kc_graph* g, uint32_t* h_rp, uint32_t* h_col) {
  kc_ctx* ctx = g->ctx;
  cudaStream_t s = ctx->stream;
  const uint32_t n = g->n;
  DevTemps t(s);
  uint32_t *deg = nullptr, *orp = nullptr, *ocol = nullptr, *ucnt = nullptr;
  KC_CUDA(t.alloc(&deg, sizeof(uint32_t) * ((size_t)n + 1)));
  KC_CUDA(t.alloc(&orp, sizeof(uint32_t) * ((size_t)n + 1)));
  KC_CUDA(t.alloc(&ocol, sizeof(uint32_t) * std::max<uint64_t>(1, g->m)));
  KC_CUDA(t.alloc(&ucnt, sizeof(uint32_t) * ((size_t)n + 1)));
  k_export_deg<<<grid_for(n, ctx->sms), 256, 0, s>>>(g->drp, g->rank, n, deg);
  KC_CUDA(prim::scan_exclusive_u32(deg, orp, n, s));
  k_export_fill<<<grid_for((uint64_t)n * 32, ctx->sms, 32), 256, 0, s>>>(g->drp, g->dcol, g->rank, g->inv, n, orp, ocol);
  KC_CUDA(prim::segmented_sort_unique(orp, ocol, ucnt, n, g->max_out, s));
  KC_CUDA(cudaMemcpyAsync(h_rp, orp, sizeof(uint32_t) * ((size_t)n + 1), cudaMemcpyDeviceToHost, s));
  if (g->m) KC_CUDA(cudaMemcpyAsync(h_col, ocol, sizeof(uint32_t) * g->m, cudaMemcpyDeviceToHost, s));
  KC_CUDA(cudaStreamSynchronize(s));
  return KC_OK;
}

}  // namespace kc
