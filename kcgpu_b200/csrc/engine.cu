// The C ABI of the engine (include/kc.h): contexts, graphs, orientation,
// counting, k-core and k-truss support. Batched counting is in batch.cu and
// the request server in server.cpp.
//
// Every entry point returns a kc_status, records a message for kc_last_error()
// and never exits the process (the reference prints and continues on CUDA
// errors, include/utils.cuh:44-51, and exits on bad flags, include/Config.h:88-89).
#include <algorithm>
#include <atomic>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <mutex>
#include <new>
#include <string>
#include <vector>

#include "autotune_table.h"
#include "count_kernels.cuh"
#include "dev_common.cuh"
#include "engine.h"
#include "prims.cuh"

namespace kc {

kc_status dev_alloc(kc_graph* g, void** p, size_t bytes) {
  bytes = std::max<size_t>(bytes, 4);
  cudaError_t e = dmalloc_raw(p, bytes, g->ctx->stream);
  if (e != cudaSuccess) return cuda_fail(e, "device allocation", __FILE__, __LINE__);
  g->bytes += bytes;
  return KC_OK;
}

void dev_free(kc_graph* g, void* p) {
  if (p) dfree(p, g->ctx->stream);
}

namespace {

__global__ void k_expand_rows(const uint32_t* __restrict__ rp, uint32_t n, uint32_t* src) {
  const uint32_t lane = lane_id();
  const uint32_t gw = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, nw = (gridDim.x * blockDim.x) >> 5;
  for (uint32_t u = gw; u < n; u += nw)
    for (uint32_t i = rp[u] + lane; i < rp[u + 1]; i += 32) src[i] = u;
}

struct CtxLock {
  kc_ctx* c;
  explicit CtxLock(kc_ctx* ctx) : c(ctx) {
    c->mu.lock();
    cudaSetDevice(c->device);
    clear_error();
  }
  ~CtxLock() { c->mu.unlock(); }
};

void free_graph_arrays(kc_graph* g) {
  void* ps[] = {g->rp, g->col, g->rank, g->inv, g->drp, g->dcol, g->erow, g->prio, g->level, g->vgraph};
  for (void* p : ps)
    if (p) dfree(p, g->ctx->stream);
  g->rp = g->col = g->rank = g->inv = g->drp = g->dcol = g->erow = g->prio = g->level = g->vgraph = nullptr;
}

kc_status new_graph(kc_ctx* ctx, kc_graph** out) {
  if (!out) return fail(KC_ERR_INVALID_ARG, "output pointer is NULL");
  *out = nullptr;
  kc_graph* g = new (std::nothrow) kc_graph();
  if (!g) return fail(KC_ERR_OOM, "host allocation failed");
  g->ctx = ctx;
  *out = g;
  return KC_OK;
}

kc_status build_from_device(kc_graph* g, const uint32_t* d_src, const uint32_t* d_dst, uint64_t E, uint32_t n) {
  kc_status st = build_csr(g, d_src, d_dst, E, n);
  if (st != KC_OK) return st;
  return KC_OK;
}

}  // namespace

namespace {

uint32_t tune_band_u(uint32_t v, const uint32_t* lo, int n) {
  int b = 0;
  for (int i = 0; i < n; ++i)
    if (v >= lo[i]) b = i;
  return (uint32_t)b;
}

uint32_t tune_band_d(double v, const double* lo, int n) {
  int b = 0;
  for (int i = 0; i < n; ++i)
    if (v >= lo[i]) b = i;
  return (uint32_t)b;
}

}  // namespace

kc_params autotune(uint32_t n, uint64_t m, uint32_t max_out, uint32_t k, uint32_t max_core, uint32_t orientation) {
  // The measured table first: the fastest fixed method of the sweep for the
  // graph's (k, largest out-degree, density) bucket, for degree-oriented
  // graphs (the orientation the sweep measured).
  const double dens0 = n > 1 ? (2.0 * (double)m) / ((double)n * (n - 1)) : 0.0;
  if (orientation == KC_ORIENT_DEGREE && k >= 3) {
    constexpr int nk = sizeof(tune::kKBands) / sizeof(tune::kKBands[0]);
    constexpr int no = sizeof(tune::kOutBands) / sizeof(tune::kOutBands[0]);
    constexpr int nd = sizeof(tune::kDensBands) / sizeof(tune::kDensBands[0]);
    const tune::Entry& e = tune::kTable[tune_band_u(k, tune::kKBands, nk)][tune_band_u(max_out, tune::kOutBands, no)]
                                       [tune_band_d(dens0, tune::kDensBands, nd)];
    if (e.valid) {
      kc_params p;
      std::memset(&p, 0, sizeof(p));
      p.k = k;
      p.mode = e.mode;
      p.unit = e.unit;
      p.part = e.part;
      p.encoding = e.encoding;
      return p;
    }
  }
  // Otherwise a choice from shape features.
  //  * mode: pivoting wins when the graph holds large cliques (its cost follows
  //    the clique tree, not the clique count); orientation listing wins on
  //    sparse neighbourhoods. A unit inside a c-core lists about C(c, k - 1)
  //    cliques, so a graph whose core would make that a sizeable part of a
  //    warp unit's work budget (kUnitBudget / 4) pivots outright; the others
  //    run KC_MODE_AUTO, which lists small units and moves any unit that
  //    outgrows its budget (a hidden clique) to the pivot.
  //  * part: 0 lets each size class size its partitions to its word width.
  //  * unit: edge units spread the work of graphs with few vertices but wide
  //    out-neighbourhoods over more groups.
  //  * encoding: sorted lists only for very wide, very sparse neighbourhoods.
  kc_params p;
  std::memset(&p, 0, sizeof(p));
  p.k = k;
  const double dens = n > 1 ? (2.0 * (double)m) / ((double)n * (n - 1)) : 0.0;
  double listed = 1.0;  // C(max_core, k - 1)
  for (uint32_t i = 0; k >= 1 && i < k - 1 && i < max_core; ++i) listed = listed * (max_core - i) / (i + 1);
  if (k >= 1 && k - 1 > max_core) listed = 0.0;
  const bool dense_core = max_core >= 24 || listed > kUnitBudget / 4.0;
  p.mode = dense_core ? KC_MODE_PIVOT : KC_MODE_AUTO;
  p.unit = (n < 256 && max_out > 64) ? KC_UNIT_EDGE : KC_UNIT_NODE;
  p.part = 0;
  p.encoding = (max_out > 4096 && dens < 0.001) ? KC_ENC_LIST : KC_ENC_BITMAP;
  return p;
}

kc_status export_dag(kc_graph* g, uint32_t* h_rp, uint32_t* h_col);  // orient.cu

}  // namespace kc

using kc::fail;

namespace {
std::atomic<uint64_t> g_launches{0};
}

extern "C" {

// Every kernel launch of this library goes through cudaLaunchKernel (the
// <<<>>> stubs) or cudaLaunchCooperativeKernel; the link step wraps both
// (-Wl,--wrap) so the launches can be counted.
cudaError_t __real_cudaLaunchKernel(const void* f, dim3 g, dim3 b, void** a, size_t sm, cudaStream_t s);
cudaError_t __wrap_cudaLaunchKernel(const void* f, dim3 g, dim3 b, void** a, size_t sm, cudaStream_t s) {
  g_launches.fetch_add(1, std::memory_order_relaxed);
  return __real_cudaLaunchKernel(f, g, b, a, sm, s);
}
cudaError_t __real_cudaLaunchCooperativeKernel(const void* f, dim3 g, dim3 b, void** a, size_t sm, cudaStream_t s);
cudaError_t __wrap_cudaLaunchCooperativeKernel(const void* f, dim3 g, dim3 b, void** a, size_t sm,
                                               cudaStream_t s) {
  g_launches.fetch_add(1, std::memory_order_relaxed);
  return __real_cudaLaunchCooperativeKernel(f, g, b, a, sm, s);
}

uint64_t kc_kernel_launches(void) { return g_launches.load(std::memory_order_relaxed); }


kc_status kc_ctx_create(int device, kc_ctx** out) {
  kc::clear_error();
  if (!out) return fail(KC_ERR_INVALID_ARG, "output pointer is NULL");
  *out = nullptr;
  int ndev = 0;
  cudaError_t e = cudaGetDeviceCount(&ndev);
  if (e != cudaSuccess || ndev == 0) {
    cudaGetLastError();
    return fail(KC_ERR_CUDA, "no CUDA device available (%s)", cudaGetErrorString(e));
  }
  if (device < 0 || device >= ndev) return fail(KC_ERR_INVALID_ARG, "device %d out of range [0,%d)", device, ndev);
  kc_ctx* c = new (std::nothrow) kc_ctx();
  if (!c) return fail(KC_ERR_OOM, "host allocation failed");
  c->device = device;
  KC_CUDA(cudaSetDevice(device));
  cudaDeviceProp prop;
  KC_CUDA(cudaGetDeviceProperties(&prop, device));
  c->sms = prop.multiProcessorCount;
  c->max_smem_optin = (int)prop.sharedMemPerBlockOptin;
  c->total_mem = prop.totalGlobalMem;
  KC_CUDA(cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking));
  // keep freed stream-ordered memory in the pool between calls, and reuse the
  // context's own blocks before asking the pool (devmem.cpp)
  cudaMemPool_t pool;
  if (cudaDeviceGetDefaultMemPool(&pool, device) == cudaSuccess) {
    uint64_t thr = UINT64_MAX;
    cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &thr);
  }
  kc::register_stream_cache(c->stream, &c->cache);
  *out = c;
  return KC_OK;
}

kc_status kc_ctx_release_cached_memory(kc_ctx* ctx) {
  if (!ctx) return fail(KC_ERR_INVALID_ARG, "context is NULL");
  kc::CtxLock lock(ctx);
  ctx->cache.release(ctx->stream);
  KC_CUDA(cudaStreamSynchronize(ctx->stream));
  return KC_OK;
}

kc_status kc_ctx_destroy(kc_ctx* ctx) {
  if (!ctx) return KC_OK;
  {
    std::lock_guard<std::mutex> l(ctx->mu);
    cudaSetDevice(ctx->device);
    cudaStreamSynchronize(ctx->stream);
    if (ctx->d_binom) kc::dfree(ctx->d_binom, ctx->stream);
    for (unsigned long long* b : ctx->binom_retired) kc::dfree(b, ctx->stream);
    for (int c = 0; c < kc_ctx::kSide; ++c) {
      if (ctx->side[c]) cudaStreamSynchronize(ctx->side[c]);
      if (ctx->side[c]) cudaStreamDestroy(ctx->side[c]);
      if (ctx->join[c]) cudaEventDestroy(ctx->join[c]);
    }
    for (int c = 0; c <= kc_ctx::kSide; ++c) {
      if (ctx->tbeg[c]) cudaEventDestroy(ctx->tbeg[c]);
      if (ctx->tend[c]) cudaEventDestroy(ctx->tend[c]);
    }
    if (ctx->fork) cudaEventDestroy(ctx->fork);
    if (ctx->copy) {
      cudaStreamSynchronize(ctx->copy);
      cudaStreamDestroy(ctx->copy);
    }
    for (cudaStream_t st : ctx->pool) {
      cudaStreamSynchronize(st);
      cudaStreamDestroy(st);
    }
    for (cudaEvent_t e : ctx->pool_done) cudaEventDestroy(e);
    if (ctx->pool_fork) cudaEventDestroy(ctx->pool_fork);
    ctx->cache.release(ctx->stream);
    cudaStreamSynchronize(ctx->stream);
    kc::unregister_stream_cache(ctx->stream);
    cudaStreamDestroy(ctx->stream);
  }
  delete ctx;
  return KC_OK;
}

kc_status kc_ctx_set_time_limit(kc_ctx* ctx, uint64_t ns) {
  if (!ctx) return fail(KC_ERR_INVALID_ARG, "context is NULL");
  std::lock_guard<std::mutex> l(ctx->mu);
  ctx->time_limit_ns = ns;
  return KC_OK;
}

kc_status kc_ctx_set_batch_chunk_edges(kc_ctx* ctx, uint64_t edges) {
  if (!ctx) return fail(KC_ERR_INVALID_ARG, "context is NULL");
  std::lock_guard<std::mutex> l(ctx->mu);
  ctx->batch_chunk_edges = edges;
  return KC_OK;
}

kc_status kc_ctx_get_stream(kc_ctx* ctx, void** stream) {
  if (!ctx || !stream) return fail(KC_ERR_INVALID_ARG, "NULL argument");
  *stream = (void*)ctx->stream;
  return KC_OK;
}

kc_status kc_graph_from_edges(kc_ctx* ctx, const uint32_t* src, const uint32_t* dst, uint64_t n_edges,
                              uint32_t n_nodes, kc_graph** out) {
  if (!ctx) return fail(KC_ERR_INVALID_ARG, "context is NULL");
  if (n_edges && (!src || !dst)) return fail(KC_ERR_INVALID_ARG, "edge arrays are NULL");
  kc::CtxLock lock(ctx);
  kc_graph* g;
  KC_TRY(kc::new_graph(ctx, &g));
  cudaStream_t s = ctx->stream;
  kc_status st = KC_OK;
  {
    kc::DevTemps t(s);
    uint32_t *ds = nullptr, *dd = nullptr;
    const size_t bytes = std::max<uint64_t>(1, n_edges) * sizeof(uint32_t);
    cudaError_t e = t.alloc(&ds, bytes);
    if (e == cudaSuccess) e = t.alloc(&dd, bytes);
    if (e == cudaSuccess && n_edges) e = cudaMemcpyAsync(ds, src, n_edges * sizeof(uint32_t), cudaMemcpyHostToDevice, s);
    if (e == cudaSuccess && n_edges) e = cudaMemcpyAsync(dd, dst, n_edges * sizeof(uint32_t), cudaMemcpyHostToDevice, s);
    st = e == cudaSuccess ? kc::build_from_device(g, ds, dd, n_edges, n_nodes)
                          : kc::cuda_fail(e, "edge staging", __FILE__, __LINE__);
  }
  if (st != KC_OK) {
    kc::free_graph_arrays(g);
    delete g;
    return st;
  }
  *out = g;
  return KC_OK;
}

kc_status kc_graph_from_edges_device(kc_ctx* ctx, const uint32_t* d_src, const uint32_t* d_dst, uint64_t n_edges,
                                     uint32_t n_nodes, kc_graph** out) {
  if (!ctx) return fail(KC_ERR_INVALID_ARG, "context is NULL");
  if (n_edges && (!d_src || !d_dst)) return fail(KC_ERR_INVALID_ARG, "edge arrays are NULL");
  kc::CtxLock lock(ctx);
  kc_graph* g;
  KC_TRY(kc::new_graph(ctx, &g));
  kc_status st = kc::build_from_device(g, d_src, d_dst, n_edges, n_nodes);
  if (st != KC_OK) {
    kc::free_graph_arrays(g);
    delete g;
    return st;
  }
  *out = g;
  return KC_OK;
}

kc_status kc_graph_from_csr(kc_ctx* ctx, const uint32_t* row_ptr, const uint32_t* col_ind, uint32_t n_nodes,
                            kc_graph** out) {
  if (!ctx) return fail(KC_ERR_INVALID_ARG, "context is NULL");
  if (!row_ptr) return fail(KC_ERR_INVALID_ARG, "row_ptr is NULL");
  const uint64_t nnz = row_ptr[n_nodes];
  if (nnz && !col_ind) return fail(KC_ERR_INVALID_ARG, "col_ind is NULL");
  for (uint32_t v = 0; v < n_nodes; ++v)
    if (row_ptr[v + 1] < row_ptr[v]) return fail(KC_ERR_INVALID_ARG, "row_ptr decreases at row %u", v);
  kc::CtxLock lock(ctx);
  kc_graph* g;
  KC_TRY(kc::new_graph(ctx, &g));
  cudaStream_t s = ctx->stream;
  kc_status st = KC_OK;
  {
    kc::DevTemps t(s);
    uint32_t *drp = nullptr, *ds = nullptr, *dd = nullptr;
    cudaError_t e = t.alloc(&drp, sizeof(uint32_t) * ((size_t)n_nodes + 1));
    if (e == cudaSuccess) e = t.alloc(&ds, sizeof(uint32_t) * std::max<uint64_t>(1, nnz));
    if (e == cudaSuccess) e = t.alloc(&dd, sizeof(uint32_t) * std::max<uint64_t>(1, nnz));
    if (e == cudaSuccess)
      e = cudaMemcpyAsync(drp, row_ptr, sizeof(uint32_t) * ((size_t)n_nodes + 1), cudaMemcpyHostToDevice, s);
    if (e == cudaSuccess && nnz) e = cudaMemcpyAsync(dd, col_ind, sizeof(uint32_t) * nnz, cudaMemcpyHostToDevice, s);
    if (e == cudaSuccess && n_nodes)
      kc::k_expand_rows<<<std::max(1u, std::min((n_nodes * 32u + 255u) / 256u, (uint32_t)ctx->sms * 32)), 256, 0,
                          s>>>(drp, n_nodes, ds);
    st = e == cudaSuccess ? kc::build_from_device(g, ds, dd, nnz, n_nodes)
                          : kc::cuda_fail(e, "CSR staging", __FILE__, __LINE__);
  }
  if (st != KC_OK) {
    kc::free_graph_arrays(g);
    delete g;
    return st;
  }
  *out = g;
  return KC_OK;
}

kc_status kc_graph_destroy(kc_graph* g) {
  if (!g) return KC_OK;
  kc::CtxLock lock(g->ctx);
  kc::free_graph_arrays(g);
  cudaStreamSynchronize(g->ctx->stream);
  delete g;
  return KC_OK;
}

kc_status kc_graph_get_info(const kc_graph* g, kc_graph_info* out) {
  if (!g || !out) return fail(KC_ERR_INVALID_ARG, "NULL argument");
  out->n = g->n;
  out->m = g->m;
  out->max_degree = g->max_deg;
  out->oriented = g->oriented < 0 ? 0u : (uint32_t)g->oriented + 1u;
  out->max_out_degree = g->max_out;
  out->max_core = g->max_core;
  out->device_bytes = g->bytes;
  return KC_OK;
}

kc_status kc_graph_get_csr(const kc_graph* g, uint32_t* row_ptr, uint32_t* col_ind) {
  if (!g || !row_ptr || (g->m && !col_ind)) return fail(KC_ERR_INVALID_ARG, "NULL argument");
  kc::CtxLock lock(g->ctx);
  cudaStream_t s = g->ctx->stream;
  KC_CUDA(cudaMemcpyAsync(row_ptr, g->rp, sizeof(uint32_t) * ((size_t)g->n + 1), cudaMemcpyDeviceToHost, s));
  if (g->m) KC_CUDA(cudaMemcpyAsync(col_ind, g->col, sizeof(uint32_t) * 2 * g->m, cudaMemcpyDeviceToHost, s));
  KC_CUDA(cudaStreamSynchronize(s));
  return KC_OK;
}

kc_status kc_orient(kc_graph* g, uint32_t orientation) {
  if (!g) return fail(KC_ERR_INVALID_ARG, "graph is NULL");
  kc::CtxLock lock(g->ctx);
  return kc::orient_graph(g, orientation);
}

kc_status kc_graph_get_dag(const kc_graph* g, uint32_t* row_ptr, uint32_t* col_ind) {
  if (!g || !row_ptr || (g->m && !col_ind)) return fail(KC_ERR_INVALID_ARG, "NULL argument");
  if (g->oriented < 0) return fail(KC_ERR_NOT_ORIENTED, "call kc_orient first");
  kc::CtxLock lock(g->ctx);
  return kc::export_dag(const_cast<kc_graph*>(g), row_ptr, col_ind);
}

kc_status kc_graph_get_peel(const kc_graph* g, uint32_t* priority, uint32_t* level) {
  if (!g) return fail(KC_ERR_INVALID_ARG, "graph is NULL");
  if (!g->prio) return fail(KC_ERR_NOT_ORIENTED, "no degeneracy peel has run on this graph");
  kc::CtxLock lock(g->ctx);
  cudaStream_t s = g->ctx->stream;
  if (priority && g->n) KC_CUDA(cudaMemcpyAsync(priority, g->prio, sizeof(uint32_t) * g->n, cudaMemcpyDeviceToHost, s));
  if (level && g->n) KC_CUDA(cudaMemcpyAsync(level, g->level, sizeof(uint32_t) * g->n, cudaMemcpyDeviceToHost, s));
  KC_CUDA(cudaStreamSynchronize(s));
  return KC_OK;
}

kc_status kc_parse_spec(const char* spec, kc_params* io) {
  // include/Config.h:235-271: [o|p]<digits>[b|n|h]; strings of length <= 2
  // keep the defaults (orientation, partition 8, bitmap).
  if (!io) return fail(KC_ERR_INVALID_ARG, "params pointer is NULL");
  io->mode = KC_MODE_ORIENT;
  io->part = 8;
  io->encoding = KC_ENC_BITMAP;
  if (!spec) return KC_OK;
  const size_t len = std::strlen(spec);
  if (len <= 2) return KC_OK;
  if (spec[0] == 'p') io->mode = KC_MODE_PIVOT;
  size_t i = 1;
  uint32_t part = 0;
  if (spec[i] < '0' || spec[i] > '9') return fail(KC_ERR_INVALID_ARG, "spec '%s': partition size expected", spec);
  while (i < len && spec[i] >= '0' && spec[i] <= '9') part = part * 10 + (uint32_t)(spec[i++] - '0');
  if (part == 0 || part > 32 || (part & (part - 1)))
    return fail(KC_ERR_INVALID_ARG, "spec '%s': partition size %u is not one of 1,2,4,8,16,32", spec, part);
  io->part = part;
  if (i < len && spec[i] == 'n') io->encoding = KC_ENC_LIST;
  return KC_OK;
}

kc_status kc_count(kc_graph* g, const kc_params* p, kc_u128* out, kc_count_stats* stats) {
  if (!g) return fail(KC_ERR_INVALID_ARG, "NULL argument");
  return kc::count_on(g->ctx, g, p, out, stats);
}

kc_status kc_count_multi(kc_graph* g, const kc_params* p, const uint32_t* ks, uint32_t n_k, kc_u128* out) {
  if (!g) return fail(KC_ERR_INVALID_ARG, "NULL argument");
  return kc::count_multi_on(g->ctx, g, p, ks, n_k, out);
}

kc_status kc_count_shard(kc_graph* g, const kc_params* p, uint32_t shard, uint32_t n_shards, kc_u128* out,
                         kc_count_stats* stats) {
  if (!g) return fail(KC_ERR_INVALID_ARG, "NULL argument");
  if (n_shards == 0 || shard >= n_shards)
    return fail(KC_ERR_INVALID_ARG, "shard %u of %u: need shard < n_shards", shard, n_shards);
  return kc::count_on(g->ctx, g, p, out, stats, shard, n_shards);
}

}  // extern "C"

namespace kc {

kc_status count_on(kc_ctx* run, kc_graph* g, const kc_params* p, kc_u128* out, kc_count_stats* stats,
                   uint32_t shard, uint32_t n_shards) {
  if (!run || !g || !p || !out) return fail(KC_ERR_INVALID_ARG, "NULL argument");
  if (p->k < 1) return fail(KC_ERR_INVALID_ARG, "k must be >= 1");
  if (p->mode > KC_MODE_AUTO || p->unit > KC_UNIT_EDGE || p->encoding > KC_ENC_LIST)
    return fail(KC_ERR_INVALID_ARG, "unknown mode, unit or encoding");
  if (p->part != 0 && (p->part > 32 || (p->part & (p->part - 1))))
    return fail(KC_ERR_INVALID_ARG, "partition size %u is not one of 1,2,4,8,16,32", p->part);
  if (g->oriented < 0) return fail(KC_ERR_NOT_ORIENTED, "call kc_orient before kc_count");
  if (run != g->ctx && run->device != g->ctx->device)
    return fail(KC_ERR_INVALID_ARG, "a graph can only be counted by a context of its own device");
  kc::CtxLock lock(run);
  if (stats) std::memset(stats, 0, sizeof(*stats));
  out->lo = out->hi = 0;
  // k <= 2 needs no units: the whole count belongs to shard 0
  if (p->k == 1) { out->lo = shard == 0 ? g->n : 0; return KC_OK; }
  if (p->k == 2) { out->lo = shard == 0 ? g->m : 0; return KC_OK; }
  cudaStream_t s = run->stream;
  kc::DevTemps t(s);
  unsigned long long* d_out = nullptr;
  KC_CUDA(t.alloc(&d_out, 2 * sizeof(unsigned long long)));
  KC_CUDA(cudaMemsetAsync(d_out, 0, 2 * sizeof(unsigned long long), s));
  kc::CountRequest req;
  req.k = p->k;
  req.mode = p->mode;
  req.unit = p->unit;
  req.part = p->part;
  req.encoding = p->encoding;
  req.flags = p->flags;
  req.k_max = p->k;
  req.ctx = run;
  req.shard = shard;
  req.n_shards = n_shards;
  kc_status st = kc::count_graph(g, req, d_out, (p->flags & KC_FLAG_STATS) ? stats : nullptr);
  unsigned long long h[2] = {0, 0};
  if (st == KC_OK) {
    cudaError_t e = cudaMemcpyAsync(h, d_out, sizeof(h), cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    if (e != cudaSuccess) st = kc::cuda_fail(e, "count readback", __FILE__, __LINE__);
  }
  out->lo = h[0];
  out->hi = h[1];
  return st;
}

kc_status count_multi_on(kc_ctx* run, kc_graph* g, const kc_params* p, const uint32_t* ks, uint32_t n_k,
                         kc_u128* out) {
  if (!run || !g || !p || !ks || !out) return fail(KC_ERR_INVALID_ARG, "NULL argument");
  if (n_k == 0 || n_k > 32) return fail(KC_ERR_INVALID_ARG, "%u values of k: between 1 and 32 per call", n_k);
  if (p->unit > KC_UNIT_EDGE) return fail(KC_ERR_INVALID_ARG, "unknown unit");
  if (p->encoding != KC_ENC_BITMAP)
    return fail(KC_ERR_INVALID_ARG, "several k in one walk need the binary encoding");
  for (uint32_t i = 0; i < n_k; ++i)
    if (ks[i] < 1) return fail(KC_ERR_INVALID_ARG, "k must be >= 1");
  if (g->oriented < 0) return fail(KC_ERR_NOT_ORIENTED, "call kc_orient before kc_count_multi");
  if (run != g->ctx && run->device != g->ctx->device)
    return fail(KC_ERR_INVALID_ARG, "a graph can only be counted by a context of its own device");
  kc::CtxLock lock(run);
  // k <= 2 need no walk; the others, ascending and without repeats, share one
  std::vector<uint32_t> big;
  for (uint32_t i = 0; i < n_k; ++i) {
    out[i] = {0, 0};
    if (ks[i] == 1) out[i].lo = g->n;
    else if (ks[i] == 2) out[i].lo = g->m;
    else big.push_back(ks[i]);
  }
  std::sort(big.begin(), big.end());
  big.erase(std::unique(big.begin(), big.end()), big.end());
  if (big.empty()) return KC_OK;
  const uint32_t nb = (uint32_t)big.size();
  cudaStream_t s = run->stream;
  kc::DevTemps t(s);
  unsigned long long* d_out = nullptr;
  KC_CUDA(t.alloc(&d_out, 2 * sizeof(unsigned long long) * nb));
  KC_CUDA(cudaMemsetAsync(d_out, 0, 2 * sizeof(unsigned long long) * nb, s));
  kc::CountRequest req;
  req.k = big.front();
  req.k_max = big.back();
  req.mode = KC_MODE_PIVOT;
  req.unit = p->unit;
  req.part = 0;
  req.encoding = KC_ENC_BITMAP;
  req.flags = 0;
  req.ctx = run;
  req.nk = nb;
  for (uint32_t i = 0; i < nb; ++i) req.kset[i] = big[i];
  kc_status st = kc::count_graph(g, req, d_out, nullptr);
  std::vector<unsigned long long> h(2 * (size_t)nb, 0);
  if (st == KC_OK) {
    cudaError_t e = cudaMemcpyAsync(h.data(), d_out, h.size() * sizeof(unsigned long long), cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    if (e != cudaSuccess) st = kc::cuda_fail(e, "count readback", __FILE__, __LINE__);
  }
  if (st != KC_OK) return st;
  for (uint32_t i = 0; i < n_k; ++i) {
    if (ks[i] <= 2) continue;
    const size_t j = (size_t)(std::lower_bound(big.begin(), big.end(), ks[i]) - big.begin());
    out[i].lo = h[2 * j];
    out[i].hi = h[2 * j + 1];
  }
  return KC_OK;
}

kc_status complete_for_sharing(kc_graph* g) {
  if (!g) return fail(KC_ERR_INVALID_ARG, "graph is NULL");
  if (g->oriented < 0) return fail(KC_ERR_NOT_ORIENTED, "orient the graph before sharing it");
  kc::CtxLock lock(g->ctx);
  KC_TRY(ensure_edge_rows(g));
  KC_CUDA(cudaStreamSynchronize(g->ctx->stream));
  return KC_OK;
}

}  // namespace kc

extern "C" {

kc_status kc_count_local(kc_graph* g, const kc_params* p, kc_u128* per_vertex, kc_u128* total) {
  if (!g || !p || !per_vertex) return fail(KC_ERR_INVALID_ARG, "NULL argument");
  if (p->k < 1) return fail(KC_ERR_INVALID_ARG, "k must be >= 1");
  if (p->mode > KC_MODE_AUTO || p->encoding != KC_ENC_BITMAP)
    return fail(KC_ERR_INVALID_ARG, "local counts need binary encoding (as the reference's) and a known mode");
  if (p->unit > KC_UNIT_EDGE) return fail(KC_ERR_INVALID_ARG, "unknown unit");
  if (p->part != 0 && (p->part > 32 || (p->part & (p->part - 1))))
    return fail(KC_ERR_INVALID_ARG, "partition size %u is not one of 1,2,4,8,16,32", p->part);
  if (g->oriented < 0) return fail(KC_ERR_NOT_ORIENTED, "call kc_orient before kc_count_local");
  kc::CtxLock lock(g->ctx);
  const uint32_t n = g->n;
  cudaStream_t s = g->ctx->stream;
  std::vector<unsigned long long> loc(2 * (size_t)n, 0);
  unsigned long long tot_lo = 0, tot_hi = 0;
  if (p->k <= 2) {
    // k = 1: every vertex once; k = 2: every vertex in deg(v) edges
    std::vector<uint32_t> rp((size_t)n + 1, 0);
    if (n) {
      KC_CUDA(cudaMemcpyAsync(rp.data(), g->rp, sizeof(uint32_t) * ((size_t)n + 1), cudaMemcpyDeviceToHost, s));
      KC_CUDA(cudaStreamSynchronize(s));
    }
    for (uint32_t v = 0; v < n; ++v) per_vertex[v] = {p->k == 1 ? 1ull : (unsigned long long)(rp[v + 1] - rp[v]), 0};
    if (total) *total = {p->k == 1 ? (unsigned long long)n : (unsigned long long)g->m, 0};
    return KC_OK;
  }
  kc::DevTemps t(s);
  unsigned long long *d_out = nullptr, *d_local = nullptr;
  KC_CUDA(t.alloc(&d_out, 2 * sizeof(unsigned long long)));
  KC_CUDA(t.alloc(&d_local, 2 * sizeof(unsigned long long) * std::max<uint32_t>(1, n)));
  KC_CUDA(cudaMemsetAsync(d_out, 0, 2 * sizeof(unsigned long long), s));
  KC_CUDA(cudaMemsetAsync(d_local, 0, 2 * sizeof(unsigned long long) * std::max<uint32_t>(1, n), s));
  kc::CountRequest req;
  req.k = p->k;
  req.mode = p->mode;
  req.unit = p->unit;
  req.part = p->part;
  req.encoding = KC_ENC_BITMAP;
  req.flags = 0;
  req.k_max = p->k;
  req.d_local = d_local;
  kc_status st = kc::count_graph(g, req, d_out, nullptr);
  std::vector<uint32_t> rank(n);
  unsigned long long h[2] = {0, 0};
  if (st == KC_OK) {
    cudaError_t e = cudaMemcpyAsync(h, d_out, sizeof(h), cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess && n) e = cudaMemcpyAsync(loc.data(), d_local, sizeof(unsigned long long) * 2 * n, cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess && n) e = cudaMemcpyAsync(rank.data(), g->rank, sizeof(uint32_t) * n, cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    if (e != cudaSuccess) st = kc::cuda_fail(e, "local count readback", __FILE__, __LINE__);
  }
  if (st != KC_OK) return st;
  // counters are indexed by rank label; the caller's array by vertex id
  for (uint32_t v = 0; v < n; ++v) per_vertex[v] = {loc[2 * (size_t)rank[v]], loc[2 * (size_t)rank[v] + 1]};
  tot_lo = h[0];
  tot_hi = h[1];
  if (total) *total = {tot_lo, tot_hi};
  return KC_OK;
}

kc_status kc_kcore(kc_graph* g, uint32_t* core, uint32_t* max_core) {
  if (!g) return fail(KC_ERR_INVALID_ARG, "graph is NULL");
  kc::CtxLock lock(g->ctx);
  KC_TRY(kc::peel_graph(g));
  if (core && g->n) {
    KC_CUDA(cudaMemcpyAsync(core, g->level, sizeof(uint32_t) * g->n, cudaMemcpyDeviceToHost, g->ctx->stream));
    KC_CUDA(cudaStreamSynchronize(g->ctx->stream));
  }
  if (max_core) *max_core = g->max_core;
  return KC_OK;
}

kc_status kc_truss_support(kc_graph* g, uint32_t* support) {
  if (!g || (g->m && !support)) return fail(KC_ERR_INVALID_ARG, "NULL argument");
  kc::CtxLock lock(g->ctx);
  cudaStream_t s = g->ctx->stream;
  kc::DevTemps t(s);
  uint32_t* d = nullptr;
  KC_CUDA(t.alloc(&d, sizeof(uint32_t) * std::max<uint64_t>(1, g->m)));
  kc_status st = kc::truss_support(g, d);
  if (st == KC_OK && g->m) {
    cudaError_t e = cudaMemcpyAsync(support, d, sizeof(uint32_t) * g->m, cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    if (e != cudaSuccess) st = kc::cuda_fail(e, "support readback", __FILE__, __LINE__);
  }
  return st;
}

uint64_t kc_footprint_bytes(uint32_t n, uint64_t E, uint32_t max_out) {
  // Resident graph: symmetric CSR (4(n+1) + 8m), rank maps (8n), DAG
  // (4(n+1) + 4m), edge rows (4m), peel arrays (8n); build temporaries peak
  // at about 16E + 16n; counting adds the unit queue (8 max(n, m)) and the
  // per-group scratch of the largest class (bounded by 24 GiB).
  const uint64_t m = E;
  uint64_t resident = 4ull * (n + 1) + 8ull * m + 8ull * n + 4ull * (n + 1) + 4ull * m + 4ull * m + 8ull * n;
  uint64_t build = 16ull * E + 16ull * n;
  const uint64_t W = (max_out + 31) / 32;
  uint64_t scratch = max_out > 1024 ? std::min<uint64_t>(24ull << 30, 148ull * 4 * max_out * W) : 64ull << 20;
  uint64_t queue = 8ull * std::max<uint64_t>(n, m);
  return resident + std::max(build, queue + scratch);
}

}  // extern "C"
