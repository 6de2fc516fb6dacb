// k-clique counting: the unit queue and the per-class persistent launches.
//
// Reference kernels replaced (kclique/):
//   node / orientation / bitmap  kckernel_node_block_warp_binary_count       kckernels_orientation.cuh:319-475
//   edge / orientation / bitmap  kckernel_edge_block_warp_binary_count_o2    kckernels_orientation.cuh:479-650
//   node / pivot / bitmap        kckernel_node_block_warp_binary_pivot_count kckernels_pivoting.cuh:2-346
//   edge / pivot / bitmap        kckernel_edge_block_warp_binary_pivot_count kckernels.cuh:2263-2630
//   and the list-encoded variants (count_list.cu).
//
// Unit semantics (as the reference): a node unit u counts the k-cliques whose
// lowest-ranked vertex is u, i.e. the (k-1)-cliques of the DAG induced on
// S = N+(u); an edge unit u->v counts those whose two lowest are u and v, the
// (k-2)-cliques on S = N+(u) ∩ N+(v). Units that cannot hold a k-clique
// (|N+(u)| < k-1, or min(|N+(u)|, |N+(v)|) < k-2) are dropped up front, as
// the reference's first bucket_scan does (kclique.cuh:1610-1614, 2041).
//
// The persistent work queue replaces GraphQueue + bucket_scan
// (include/GraphQueue.cuh, kclique.cuh:1318-1406): units are partitioned by
// size class with a stable two-pass partition (index order, i.e. graph order,
// inside a class), class bounds are computed on the device, and each class
// runs one persistent grid that takes units from a global ticket; units that
// outrun a warp's work budget go to a CTA-wide heavy pass. No per-window
// launch or host synchronisation (kclique.cuh:1645-1675 launches per
// 1024-wide degree window and syncs the host after each).
#include <algorithm>
#include <cstring>
#include <vector>

#include "count_kernels.cuh"
#include "dev_common.cuh"
#include "engine.h"
#include "prims.cuh"

namespace kc {

namespace {

struct ClassSpec {
  int64_t lo, hi;   // unit sizes (lo, hi]
  uint32_t G;       // threads per unit group
  uint32_t block;   // threads per CTA
};

// Size classes, largest first.
const ClassSpec kClasses[kNumClasses] = {
    {1024, 0xffffffffll, 256, 256},  // CTA per unit, bitmap in global memory
    {128, 1024, 256, 256},           // CTA per unit, bitmap in shared memory
    {32, 128, 32, 128},              // warp per unit
    {-1, 32, 32, 128},               // warp per unit, one word per row
};
__constant__ uint32_t kClassLo[kNumClasses - 1] = {1024, 128, 32};  // lower bounds of classes 0..2

// Size class of every unit (kNumClasses = dropped: it cannot hold a k-clique).
__global__ void k_unit_class(const uint32_t* __restrict__ drp, const uint32_t* __restrict__ dcol,
                             const uint32_t* __restrict__ erow, uint32_t n_units, int edge,
                             const uint32_t* __restrict__ vgraph, const uint32_t* __restrict__ gk, uint32_t k0,
                             uint8_t* cls) {
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n_units; i += gridDim.x * blockDim.x) {
    uint32_t s, src;
    if (!edge) {
      src = i;
      s = drp[i + 1] - drp[i];
    } else {
      src = erow[i];
      const uint32_t v = dcol[i];
      s = min(drp[src + 1] - drp[src], drp[v + 1] - drp[v]);
    }
    const uint32_t k = gk ? gk[vgraph ? vgraph[src] : 0u] : k0;
    bool keep;
    if (k == 0xffffffffu || k == 0u) keep = false;  // graph not in this pass
    else if (edge) keep = k >= 2u && s >= k - 2u;
    else keep = s >= k - 1u;
    uint8_t c = (uint8_t)kNumClasses;
    if (keep) c = s > kClassLo[0] ? 0 : (s > kClassLo[1] ? 1 : (s > kClassLo[2] ? 2 : 3));
    cls[i] = c;
  }
}

// Stable partition of the units by class, in two passes over chunks of
// kPartChunk units: per-chunk class counts (class-major, so one exclusive
// scan gives every chunk's start in every class), then an ordered scatter.
// Units keep their index order inside a class: the units of one graph (one
// contiguous range of rank labels) run close together and share the L2
// lines of their out-lists.
constexpr uint32_t kPartThreads = 256, kPartRounds = 8, kPartChunk = kPartThreads * kPartRounds;

__global__ void __launch_bounds__(kPartThreads) k_class_count(const uint8_t* __restrict__ cls, uint32_t n_units,
                                                              uint32_t n_chunks, uint32_t* cnt) {
  __shared__ uint32_t c4[kNumClasses];
  if (threadIdx.x < kNumClasses) c4[threadIdx.x] = 0;
  __syncthreads();
  const uint32_t base = blockIdx.x * kPartChunk;
  uint32_t mine[kNumClasses] = {};
  for (uint32_t r = 0; r < kPartRounds; ++r) {
    const uint32_t i = base + r * kPartThreads + threadIdx.x;
    const uint32_t c = i < n_units ? cls[i] : (uint32_t)kNumClasses;
#pragma unroll
    for (int q = 0; q < kNumClasses; ++q) mine[q] += c == (uint32_t)q;
  }
#pragma unroll
  for (int q = 0; q < kNumClasses; ++q) {
    uint32_t v = mine[q];
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    if ((threadIdx.x & 31u) == 0 && v) atomicAdd(&c4[q], v);
  }
  __syncthreads();
  if (threadIdx.x < kNumClasses) cnt[(size_t)threadIdx.x * n_chunks + blockIdx.x] = c4[threadIdx.x];
}

__global__ void __launch_bounds__(kPartThreads) k_class_scatter(const uint8_t* __restrict__ cls, uint32_t n_units,
                                                                uint32_t n_chunks, const uint32_t* __restrict__ off,
                                                                uint32_t* queue) {
  constexpr uint32_t kWarps = kPartThreads / 32;
  __shared__ uint32_t wc[kWarps][kNumClasses];
  __shared__ uint32_t run[kNumClasses];
  const uint32_t lane = threadIdx.x & 31u, warp = threadIdx.x >> 5;
  if (threadIdx.x < kNumClasses) run[threadIdx.x] = off[(size_t)threadIdx.x * n_chunks + blockIdx.x];
  const uint32_t base = blockIdx.x * kPartChunk;
  for (uint32_t r = 0; r < kPartRounds; ++r) {
    const uint32_t i = base + r * kPartThreads + threadIdx.x;
    const uint32_t c = i < n_units ? cls[i] : (uint32_t)kNumClasses;
    uint32_t rank = 0;
#pragma unroll
    for (int q = 0; q < kNumClasses; ++q) {
      const uint32_t m = __ballot_sync(0xffffffffu, c == (uint32_t)q);
      if (c == (uint32_t)q) rank = __popc(m & lanemask_lt());
      if (lane == 0) wc[warp][q] = __popc(m);
    }
    __syncthreads();
    if (c < (uint32_t)kNumClasses) {
      uint32_t pos = run[c] + rank;
      for (uint32_t w = 0; w < warp; ++w) pos += wc[w][c];
      queue[pos] = i;
    }
    __syncthreads();
    if (threadIdx.x < kNumClasses) {
      uint32_t add = 0;
      for (uint32_t w = 0; w < kWarps; ++w) add += wc[w][threadIdx.x];
      run[threadIdx.x] += add;
    }
    __syncthreads();
  }
}

// [begin, count] of every class from the scanned chunk counts; also stamps the
// pass's start on the global timer (the counting kernels' time limit). Unit
// shard `shard` of S takes a class's positions shard, shard + S, ...: its
// begin is the class start + shard, its count the positions left, and the
// launches step through the queue by S (CountParams::qstride). Inside a class
// units are in index order, so the stride deals out neighbouring units (and
// the few largest ones) evenly between the shards.
__global__ void k_class_bounds(const uint32_t* __restrict__ off, uint32_t n_chunks, uint32_t* bounds,
                               unsigned long long* t0, uint32_t shard, uint32_t n_shards) {
  if (threadIdx.x != 0 || blockIdx.x != 0) return;
  *t0 = global_ns();
  for (int c = 0; c < kNumClasses; ++c) {
    const uint32_t b = off[(size_t)c * n_chunks], e = off[(size_t)(c + 1) * n_chunks];
    const uint32_t cnt = e - b;
    bounds[2 * c] = cnt > shard ? b + shard : b;
    bounds[2 * c + 1] = cnt > shard ? (cnt - shard + n_shards - 1) / n_shards : 0u;
  }
}

uint32_t auto_part(uint32_t mode, uint32_t W) {
  if (mode == KC_MODE_ORIENT) return W <= 1 ? 1u : (W <= 2 ? 2u : (W <= 4 ? 4u : (W <= 8 ? 8u : (W <= 16 ? 16u : 32u))));
  // pivoting: a whole warp per clique-tree node. Partitions of one warp walk
  // different nodes and so run one after another; a full warp scores the
  // node's candidates one per lane instead.
  (void)W;
  return 32u;
}

}  // namespace

kc_status ensure_binom(kc_ctx* ctx, uint32_t rows, uint32_t cols) {
  if (ctx->d_binom && ctx->brows >= rows && ctx->bcols >= cols) return KC_OK;
  // Grown in large steps (rows to a power of two, at least 128; at least 34
  // columns, k up to 33), so a context regrows it a few times at most.
  uint32_t r2 = 128;
  while (r2 < std::max(rows, ctx->brows)) r2 <<= 1;
  rows = r2;
  cols = std::max<uint32_t>(std::max(cols, ctx->bcols), 34u);
  std::vector<unsigned __int128> t((size_t)(rows + 1) * (cols + 1), 0);
  for (uint32_t r = 0; r <= rows; ++r) {
    t[(size_t)r * (cols + 1)] = 1;
    for (uint32_t c = 1; c <= cols && c <= r; ++c)
      t[(size_t)r * (cols + 1) + c] = t[(size_t)(r - 1) * (cols + 1) + c - 1] + t[(size_t)(r - 1) * (cols + 1) + c];
  }
  std::vector<unsigned long long> h(t.size() * 2);
  for (size_t i = 0; i < t.size(); ++i) {
    h[2 * i] = (unsigned long long)t[i];
    h[2 * i + 1] = (unsigned long long)(t[i] >> 64);
  }
  // The new table replaces the old one once it is complete. Everything is
  // ordered on the context's own stream: no call here waits for the whole
  // device (a cudaFree would, stalling every other context's work). The old
  // table stays allocated until the context is destroyed: a plan prepared
  // before the growth may still point at it.
  unsigned long long* nb = nullptr;
  KC_CUDA(dmalloc(&nb, h.size() * sizeof(unsigned long long), ctx->stream));
  cudaError_t e = cudaMemcpyAsync(nb, h.data(), h.size() * sizeof(unsigned long long), cudaMemcpyHostToDevice,
                                  ctx->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(ctx->stream);  // (h is freed on return)
  if (e != cudaSuccess) {
    dfree(nb, ctx->stream);
    return cuda_fail(e, "binomial table upload", __FILE__, __LINE__);
  }
  if (ctx->d_binom) ctx->binom_retired.push_back(ctx->d_binom);
  ctx->d_binom = nb;
  ctx->brows = rows;
  ctx->bcols = cols;
  return KC_OK;
}

void count_release(CountPlan* pl) {
  if (!pl->ctx) return;  // never prepared
  cudaStream_t s = pl->ctx->stream;
  for (int c = 0; c <= kNumClasses; ++c) release_launch(pl->launches[c], s);
  void* ps[] = {pl->cls, pl->ccnt, pl->queue, pl->scratch, pl->heavy, pl->help};
  for (void* p : ps)
    if (p) dfree(p, s);
  pl->cls = nullptr;
  pl->ccnt = pl->queue = pl->scratch = pl->heavy = pl->help = nullptr;
}

// The context's side streams and events, created on first use.
static kc_status ensure_side(kc_ctx* ctx) {
  static_assert(kc_ctx::kSide == kNumClasses, "one side stream per size class");
  if (ctx->fork) return KC_OK;
  for (int c = 0; c < kNumClasses; ++c) {
    KC_CUDA(cudaStreamCreateWithFlags(&ctx->side[c], cudaStreamNonBlocking));
    KC_CUDA(cudaEventCreateWithFlags(&ctx->join[c], cudaEventDisableTiming));
  }
  for (int c = 0; c <= kNumClasses; ++c) {
    KC_CUDA(cudaEventCreate(&ctx->tbeg[c]));
    KC_CUDA(cudaEventCreate(&ctx->tend[c]));
  }
  KC_CUDA(cudaEventCreateWithFlags(&ctx->fork, cudaEventDisableTiming));
  return KC_OK;
}

kc_status warm_context(kc_ctx* ctx) {
  KC_TRY(ensure_side(ctx));
  return ensure_binom(ctx, 128, 34);
}

kc_status ensure_pass_streams(kc_ctx* ctx, size_t passes) {
  if (!ctx->pool_fork) KC_CUDA(cudaEventCreateWithFlags(&ctx->pool_fork, cudaEventDisableTiming));
  while (ctx->pool_done.size() < passes) {
    for (int c = 0; c <= kNumClasses; ++c) {
      cudaStream_t st = nullptr;
      KC_CUDA(cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking));
      ctx->pool.push_back(st);
    }
    cudaEvent_t e = nullptr;
    KC_CUDA(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
    ctx->pool_done.push_back(e);
  }
  return KC_OK;
}

// Allocates the queue and the class launches. No kernel runs; the plan can be
// enqueued (and captured) any number of times.
kc_status count_prepare(kc_graph* g, const CountRequest& req, unsigned long long* d_out, uint32_t depth_boost,
                        CountPlan* pl) {
  kc_ctx* ctx = req.ctx ? req.ctx : g->ctx;
  cudaStream_t s = ctx->stream;
  pl->g = g;
  pl->ctx = ctx;
  pl->req = req;
  // Edge units are grouped by source when the sources' out-neighbourhoods
  // fit a shared-memory bitmap: the unit u builds G[N+(u)] once and its
  // edges (u, v) are the root branches, each with the subproblem
  // N+(u) ∩ N+(v), the row of v. Orientation listing walks exactly those
  // branches for a node unit, so there the grouped form is the node form.
  const bool grouped = req.unit == KC_UNIT_EDGE && req.encoding == KC_ENC_BITMAP && g->max_out <= 1024;
  pl->edge = req.unit == KC_UNIT_EDGE && !grouped;
  pl->edge_roots = grouped;
  pl->d_out = d_out;
  const uint32_t k_max = std::max(req.k, req.k_max);
  if (pl->edge) KC_TRY(ensure_edge_rows(g));
  pl->n_units = pl->edge ? (uint32_t)g->m : g->n;
  pl->max_size = g->max_out;
  if (pl->max_size >= 65535u)
    return fail(KC_ERR_INVALID_ARG, "largest out-degree %u exceeds the 65534 supported per unit", pl->max_size);
  if (req.mode != KC_MODE_ORIENT) KC_TRY(ensure_binom(ctx, pl->max_size + 2, k_max + 1));
  const uint32_t nu = std::max<uint32_t>(1, pl->n_units);
  pl->n_chunks = (nu + kPartChunk - 1) / kPartChunk;
  KC_CUDA(dmalloc(&pl->cls, nu, s));
  KC_CUDA(dmalloc(&pl->ccnt, sizeof(uint32_t) * ((size_t)kNumClasses * pl->n_chunks + 1), s));
  KC_CUDA(dmalloc(&pl->queue, sizeof(uint32_t) * nu, s));
  KC_CUDA(dmalloc(&pl->heavy, sizeof(uint32_t) * nu, s));
  KC_CUDA(dmalloc(&pl->scratch, sizeof(uint32_t) * kScratchWords, s));
  // Tail helping for the pivoting launches with a CTA per unit (classes 0
  // and 1, the heavy pass): a cut-node ticket per queue position (the class
  // queue, then the heavy list), an active-unit word per CTA per launch, and
  // the exited CTAs of each class launch.
  const bool helping = ctx->tail_help && req.help && req.mode != KC_MODE_ORIENT &&
                       req.encoding == KC_ENC_BITMAP && req.d_local == nullptr;
  const size_t exit_at = 2 * (size_t)nu + (size_t)(kNumClasses + 1) * kHelpMaxGrid;
  if (helping) {
    pl->help_words = exit_at + kNumClasses;
    KC_CUDA(dmalloc(&pl->help, sizeof(uint32_t) * pl->help_words, s));
  }
  // Per-launch algorithm: orientation or pivot as requested; KC_MODE_AUTO
  // lists small units by orientation (cheap when their neighbourhood holds few
  // cliques) and counts large units and over-budget units with the pivot.
  const bool budget_ok = req.encoding == KC_ENC_BITMAP;
  auto launch_mode = [&](bool warp_group, bool heavy_pass) -> uint32_t {
    if (req.mode != KC_MODE_AUTO) return req.mode;
    // orientation listing only where a budget can hand a clique-heavy unit
    // on to the pivot; without one (list encoding) AUTO pivots everywhere
    return (warp_group && !heavy_pass && budget_ok) ? (uint32_t)KC_MODE_ORIENT : (uint32_t)KC_MODE_PIVOT;
  };
  bool any_budget = false;
  for (int c = 0; c <= kNumClasses; ++c) {
    const bool heavy_pass = c == kNumClasses;
    if (heavy_pass && !any_budget) continue;
    if (!heavy_pass && (int64_t)pl->max_size <= kClasses[c].lo) continue;
    const bool warp_group = !heavy_pass && kClasses[c].G == 32;
    LaunchPlan lp;
    lp.mode = launch_mode(warp_group, heavy_pass);
    lp.encoding = req.encoding;
    lp.edge = pl->edge;
    lp.dcap = heavy_pass ? std::max<uint32_t>(1, std::min<uint32_t>(kWarpClassMax, pl->max_size))
                         : (uint32_t)std::max<int64_t>(1, std::min<int64_t>(kClasses[c].hi, pl->max_size));
    // The heavy pass takes the units that outran a warp's budget: a CTA per
    // unit, its partitions sharing the unit's clique tree.
    lp.G = heavy_pass ? 256u : kClasses[c].G;
    lp.block = heavy_pass ? 256u : kClasses[c].block;
    lp.force_global_bitmap = (c == 0);
    lp.k_max = k_max;
    lp.part = req.part ? req.part : auto_part(lp.mode, (lp.dcap + 31) / 32);
    lp.q = lp.mode == KC_MODE_ORIENT ? 0u : req.part;
    if (req.nk) {  // several k: a full warp per walker, one lane per k
      lp.part = 32u;
      lp.q = 0u;
    }
    lp.local = req.d_local != nullptr;
    lp.depth_boost = depth_boost;
    CountParams p;
    std::memset(&p, 0, sizeof(p));
    p.rp = g->drp;
    p.col = g->dcol;
    p.erow = g->erow;
    p.queue = heavy_pass ? pl->heavy : pl->queue;
    p.qstride = heavy_pass ? 1u : std::max(1u, req.n_shards);
    p.bounds = pl->scratch + (heavy_pass ? kHeavyBounds : kClassBounds);
    p.cls = heavy_pass ? 0u : (uint32_t)c;
    p.n_units_max = pl->n_units;
    p.edge_units = pl->edge ? 1 : 0;
    p.edge_roots = pl->edge_roots ? 1 : 0;
    p.local = req.d_local;
    p.vgraph = g->vgraph;
    p.gk = req.d_graph_k;
    p.k0 = req.nk ? k_max : req.k;
    p.nk = req.nk;
    for (uint32_t i = 0; i < req.nk && i < 32u; ++i) p.kset[i] = req.kset[i];
    p.out = d_out;
    p.binom = ctx->d_binom;
    p.binom_cols = ctx->bcols;
    p.ticket = pl->scratch + c;
    p.err = pl->scratch + kErrWord;
    p.stats = (req.flags & KC_FLAG_STATS) ? reinterpret_cast<unsigned long long*>(pl->scratch + kStatsWords)
                                          : nullptr;
    p.time_limit_ns = ctx->time_limit_ns;
    p.t0 = reinterpret_cast<const unsigned long long*>(pl->scratch + kStartWord);
    if (warp_group && budget_ok) {
      p.budget = lp.mode == KC_MODE_PIVOT ? kPivotUnitBudget : kUnitBudget;
      p.heavy = pl->heavy;
      p.heavy_count = pl->scratch + kHeavyBounds + 1;
      any_budget = true;
    }
    if (helping && lp.mode == KC_MODE_PIVOT && lp.G > 32u) {
      p.help_ticket = pl->help + (heavy_pass ? nu : 0u);
      p.help_active = pl->help + 2 * (size_t)nu + (size_t)c * kHelpMaxGrid;
    }
    if (helping && !heavy_pass) p.class_exit = pl->help + exit_at;  // grids filled in below
    KC_TRY(prepare_launch(ctx, lp, p, s, &pl->launches[c]));
    if (pl->launches[c].grid > kHelpMaxGrid) {  // (never on one B200: 148 SMs x 3 CTAs)
      pl->launches[c].p.help_ticket = nullptr;
      pl->launches[c].p.help_active = nullptr;
    }
    pl->active[c] = true;
  }
  if (helping)
    for (int c = 0; c < kNumClasses; ++c)
      if (pl->active[c])
        for (int o = 0; o < kNumClasses; ++o)
          pl->launches[c].p.class_grid[o] = pl->active[o] ? pl->launches[o].grid : 0u;
  KC_TRY(ensure_side(ctx));
  for (int c = 0; c < kNumClasses; ++c) {
    pl->side[c] = ctx->side[c];
    pl->join[c] = ctx->join[c];
  }
  pl->fork = ctx->fork;
  for (int c = 0; c <= kNumClasses; ++c) {
    pl->tbeg[c] = ctx->tbeg[c];
    pl->tend[c] = ctx->tend[c];
  }
  return KC_OK;
}

// Enqueues queue construction and the class launches: no allocation, no
// synchronisation, so the whole sequence can be captured in a CUDA graph.
kc_status count_enqueue(const CountPlan& pl, cudaStream_t s) {
  kc_graph* g = pl.g;
  const int sms = pl.ctx->sms;
  KC_CUDA(cudaMemsetAsync(pl.scratch, 0, sizeof(uint32_t) * kScratchWords, s));
  if (pl.help) KC_CUDA(cudaMemsetAsync(pl.help, 0, sizeof(uint32_t) * pl.help_words, s));
  const uint32_t gq = (uint32_t)std::max<uint64_t>(1, std::min<uint64_t>((pl.n_units + 255) / 256, (uint64_t)sms * 16));
  if (pl.n_units)
    k_unit_class<<<gq, 256, 0, s>>>(g->drp, g->dcol, g->erow, pl.n_units, pl.edge ? 1 : 0, g->vgraph,
                                    pl.req.d_graph_k, pl.req.k, pl.cls);
  const uint32_t nc = pl.n_chunks;
  if (pl.n_units) k_class_count<<<nc, kPartThreads, 0, s>>>(pl.cls, pl.n_units, nc, pl.ccnt);
  else KC_CUDA(cudaMemsetAsync(pl.ccnt, 0, sizeof(uint32_t) * kNumClasses * (size_t)nc, s));
  KC_CUDA(prim::scan_exclusive_u32(pl.ccnt, pl.ccnt, (size_t)kNumClasses * nc, s));
  k_class_bounds<<<1, 32, 0, s>>>(pl.ccnt, nc, pl.scratch + kClassBounds,
                                  reinterpret_cast<unsigned long long*>(pl.scratch + kStartWord), pl.req.shard,
                                  std::max(1u, pl.req.n_shards));
  if (pl.n_units) k_class_scatter<<<nc, kPartThreads, 0, s>>>(pl.cls, pl.n_units, nc, pl.ccnt, pl.queue);
  KC_CUDA(cudaGetLastError());
  // class launches side by side, then the heavy pass over the units they handed on
  KC_CUDA(cudaEventRecord(pl.fork, s));
  for (int c = 0; c < kNumClasses; ++c) {
    if (!pl.active[c]) continue;
    KC_CUDA(cudaStreamWaitEvent(pl.side[c], pl.fork, 0));
    if (pl.timed) KC_CUDA(cudaEventRecord(pl.tbeg[c], pl.side[c]));
    KC_TRY(enqueue_launch(pl.launches[c], pl.side[c]));
    if (pl.timed) KC_CUDA(cudaEventRecord(pl.tend[c], pl.side[c]));
    KC_CUDA(cudaEventRecord(pl.join[c], pl.side[c]));
    KC_CUDA(cudaStreamWaitEvent(s, pl.join[c], 0));
  }
  if (pl.active[kNumClasses]) {
    if (pl.timed) KC_CUDA(cudaEventRecord(pl.tbeg[kNumClasses], s));
    KC_TRY(enqueue_launch(pl.launches[kNumClasses], s));
    if (pl.timed) KC_CUDA(cudaEventRecord(pl.tend[kNumClasses], s));
  }
  return KC_OK;
}

kc_status device_error_status(uint32_t err) {
  if (err == DEV_ERR_TIMEOUT)
    return fail(KC_ERR_DEVICE_TIMEOUT, "the counting pass ran past the context's device time limit");
  return fail(KC_ERR_INTERNAL, "counting kernel reported device error %u", err);
}

uint32_t count_error(const CountPlan& pl, cudaStream_t s, unsigned long long* stats) {
  static_assert(kStatsWords + 2 * kStatsCount <= kClassBounds, "stats overlap the class bounds");
  uint32_t h[kScratchWords];
  cudaMemcpyAsync(h, pl.scratch, sizeof(h), cudaMemcpyDeviceToHost, s);
  cudaStreamSynchronize(s);
  if (stats) std::memcpy(stats, h + kStatsWords, kStatsCount * sizeof(unsigned long long));
  return h[kErrWord];
}

uint32_t count_heavy(const CountPlan& pl, cudaStream_t s) {
  uint32_t h = 0;
  cudaMemcpyAsync(&h, pl.scratch + kHeavyBounds + 1, sizeof(h), cudaMemcpyDeviceToHost, s);
  cudaStreamSynchronize(s);
  return h;
}

uint64_t count_units(const CountPlan& pl, cudaStream_t s) {
  uint32_t b[2 * kNumClasses];
  cudaMemcpyAsync(b, pl.scratch + kClassBounds, sizeof(b), cudaMemcpyDeviceToHost, s);
  cudaStreamSynchronize(s);
  uint64_t t = 0;
  for (int c = 0; c < kNumClasses; ++c) t += b[2 * c + 1];
  return t;
}

kc_status count_graph(kc_graph* g, const CountRequest& req, unsigned long long* d_out, kc_count_stats* stats) {
  kc_ctx* ctx = req.ctx ? req.ctx : g->ctx;
  cudaStream_t s = ctx->stream;
  cudaEvent_t ev0, ev1;
  cudaEventCreate(&ev0);
  cudaEventCreate(&ev1);
  kc_status st = KC_OK;
  uint32_t kernels = 0;
  uint64_t units = 0, heavy = 0;
  unsigned long long sv[kStatsCount] = {};
  double ms_launch[kNumClasses + 1] = {};
  uint32_t deep = 0;
  for (uint32_t boost = 0; boost < 2; ++boost) {
    CountPlan pl;
    pl.timed = stats != nullptr;
    deep = boost;
    st = count_prepare(g, req, d_out, boost, &pl);
    if (st == KC_OK) {
      if (boost == 0) cudaEventRecord(ev0, s);
      st = count_enqueue(pl, s);
      cudaEventRecord(ev1, s);
    }
    uint32_t err = 0;
    if (st == KC_OK) {
      err = count_error(pl, s, sv);
      units = count_units(pl, s);
      heavy = count_heavy(pl, s);
      for (int c = 0; c <= kNumClasses; ++c) {
        float t = 0;
        if (pl.timed && pl.active[c] && cudaEventElapsedTime(&t, pl.tbeg[c], pl.tend[c]) == cudaSuccess)
          ms_launch[c] = t;
        else
          ms_launch[c] = 0;
      }
      kernels = 5;
      for (int c = 0; c <= kNumClasses; ++c) kernels += pl.active[c] ? 1 : 0;
    }
    count_release(&pl);
    if (st != KC_OK) break;
    if (err == DEV_ERR_STACK && boost == 0 && req.mode != KC_MODE_ORIENT) {
      // a clique tree deeper than the fast stack: rerun with the full depth
      KC_CUDA(cudaMemsetAsync(d_out, 0, sizeof(unsigned long long) * 2 * req.n_graphs * std::max(1u, req.nk), s));
      continue;
    }
    if (err) st = device_error_status(err);
    break;
  }
  if (stats && st == KC_OK) {
    float ms = 0;
    cudaEventElapsedTime(&ms, ev0, ev1);
    stats->units = units;
    stats->tree_nodes = sv[0];
    stats->word_ops = sv[1];
    stats->gather_bytes = sv[2];
    for (int q = 0; q < 3; ++q) stats->cycles[q] = sv[3 + q];
    stats->ms_total = ms;
    stats->ms_traversal = ms;
    stats->max_unit_size = g->max_out;
    stats->kernels = kernels;
    for (int c = 0; c <= kNumClasses; ++c) stats->ms_launch[c] = ms_launch[c];
    stats->heavy_units = heavy;
    stats->deep_retry = deep;
    stats->reserved = 0;
  }
  cudaEventDestroy(ev0);
  cudaEventDestroy(ev1);
  return st;
}

}  // namespace kc
