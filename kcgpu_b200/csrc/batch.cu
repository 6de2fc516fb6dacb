// Batched counting: thousands of small graphs in one pass.
//
// No counterpart in the reference (one graph per process there). The batch is
// treated as ONE disjoint-union graph: ids of graph i are shifted by the
// vertex count of the graphs before it, so CSR build, orientation and the
// counting queue run once over the whole batch instead of once per graph.
// This is exact for both orientations: degree order only compares vertices
// of the same graph, and the degeneracy peel of a disjoint union visits each
// graph's (level, sub-round) pairs in the same order as a peel of that graph
// alone, so every graph keeps its own relative priority order (the union's
// final batch and a lone graph's final batch both get the largest priority).
//
// Every vertex carries its graph id; every unit reads the k of its graph and
// adds its count to its graph's 128-bit slot. The autotuner picks mode, unit,
// partition size and encoding per graph from its shape; graphs that share a
// choice form one counting pass, and all passes of the batch are captured into
// one CUDA graph that is launched once.
#include <algorithm>
#include <cstring>
#include <map>
#include <tuple>
#include <vector>

#include "count_kernels.cuh"
#include "dev_common.cuh"
#include "engine.h"
#include "prims.cuh"

namespace kc {

namespace {

// Local ids of graph g -> ids of the union (shifted by the vertices of the
// graphs before g), from (in_s, in_d) into (out_s, out_d); in place when they
// are the same arrays.
__global__ void k_globalize(const uint32_t* in_s, const uint32_t* in_d, uint32_t* out_s, uint32_t* out_d,
                            const unsigned long long* __restrict__ eoff, const uint32_t* __restrict__ voff,
                            const uint32_t* __restrict__ nn, uint32_t G, uint32_t* err) {
  for (uint32_t g = blockIdx.x; g < G; g += gridDim.x) {
    const unsigned long long b = eoff[g], e = eoff[g + 1];
    const uint32_t off = voff[g], n = nn[g];
    for (unsigned long long i = b + threadIdx.x; i < e; i += blockDim.x) {
      uint32_t u = in_s[i], v = in_d[i];
      if (u >= n || v >= n) {
        atomicCAS(err, 0u, g + 1u);
        u = v = 0;
      }
      out_s[i] = u + off;
      out_d[i] = v + off;
    }
  }
}

__global__ void k_vertex_graph(const uint32_t* __restrict__ voff, uint32_t G, uint32_t* vg) {
  for (uint32_t g = blockIdx.x; g < G; g += gridDim.x)
    for (uint32_t v = voff[g] + threadIdx.x; v < voff[g + 1]; v += blockDim.x) vg[v] = g;
}

__global__ void k_rank_graph(const uint32_t* __restrict__ vg_orig, const uint32_t* __restrict__ rank, uint32_t n,
                             uint32_t* vgraph) {
  for (uint32_t v = blockIdx.x * blockDim.x + threadIdx.x; v < n; v += gridDim.x * blockDim.x)
    vgraph[rank[v]] = vg_orig[v];
}

// Per graph: largest out-degree, edge count and largest peel level.
__global__ void k_graph_features(const uint32_t* __restrict__ drp, const uint32_t* __restrict__ vgraph,
                                 const uint32_t* __restrict__ inv, const uint32_t* __restrict__ level, uint32_t n,
                                 uint32_t* fmax, unsigned long long* fm, uint32_t* fcore) {
  for (uint32_t r = blockIdx.x * blockDim.x + threadIdx.x; r < n; r += gridDim.x * blockDim.x) {
    const uint32_t g = vgraph[r];
    const uint32_t d = drp[r + 1] - drp[r];
    atomicMax(&fmax[g], d);
    if (d) atomicAdd(&fm[g], (unsigned long long)d);
    if (level) atomicMax(&fcore[g], level[inv[r]]);
  }
}

uint32_t grid_for(uint64_t work, int sms) {
  return (uint32_t)std::max<uint64_t>(1, std::min<uint64_t>((work + 255) / 256, (uint64_t)sms * 16));
}

void free_union(kc_graph* g) {
  uint32_t** ps[] = {&g->rp, &g->col, &g->rank, &g->inv, &g->drp, &g->dcol, &g->erow, &g->prio, &g->level, &g->vgraph};
  for (uint32_t** p : ps) {
    if (*p) dfree(*p, g->ctx->stream);
    *p = nullptr;
  }
}

struct Choice {
  uint32_t mode, unit, part, enc;
  bool operator<(const Choice& o) const {
    return std::tie(mode, unit, part, enc) < std::tie(o.mode, o.unit, o.part, o.enc);
  }
};

// Where the edge arrays of run_batch live.
enum class Input {
  kHost,         // host memory: copied to device temporaries
  kDevice,       // the caller's device memory: read in place, written global into temporaries
  kDeviceOwned,  // device memory the call may overwrite (the batch pipeline's
                 // staging buffers): used in place, edge_off[0] must be 0
};

kc_status run_batch(kc_ctx* ctx, const uint32_t* src, const uint32_t* dst, Input input,
                    const uint64_t* edge_off, const uint32_t* n_nodes, const uint32_t* ks, uint32_t G,
                    const kc_batch_opts* opts, kc_u128* counts, kc_params* choice, kc_batch_stats* stats) {
  const double t0 = now_ms();
  cudaStream_t s = ctx->stream;
  if (G == 0) return KC_OK;
  if (!src || !dst || !edge_off || !n_nodes || !ks || !counts)
    return fail(KC_ERR_INVALID_ARG, "NULL argument");
  if (opts && opts->orientation > KC_ORIENT_DEGEN) return fail(KC_ERR_INVALID_ARG, "unknown orientation");
  std::vector<uint32_t> voff((size_t)G + 1, 0);
  uint64_t N = 0;
  for (uint32_t g = 0; g < G; ++g) {
    if (ks[g] < 1) return fail(KC_ERR_INVALID_ARG, "graph %u: k must be >= 1", g);
    if (edge_off[g + 1] < edge_off[g]) return fail(KC_ERR_INVALID_ARG, "edge_off decreases at graph %u", g);
    voff[g] = (uint32_t)N;
    N += n_nodes[g];
    if (N >= 0xffffffffull) return fail(KC_ERR_INVALID_ARG, "the batch holds more than 2^32-2 vertices");
  }
  voff[G] = (uint32_t)N;
  const uint64_t E = edge_off[G] - edge_off[0];
  const uint32_t orientation = opts ? opts->orientation : KC_ORIENT_DEGREE;

  // Everything the call creates is released on every return path: device
  // temporaries by t, the union graph, plans, captured graph and events by
  // the guard below.
  cudaEvent_t e0, e1, e2, e3, e4, ec, eo;  // ec / eo: CSR built / orientation done
  cudaEventCreate(&e0); cudaEventCreate(&e1); cudaEventCreate(&e2); cudaEventCreate(&e3); cudaEventCreate(&e4);
  cudaEventCreate(&ec); cudaEventCreate(&eo);
  kc_graph U;
  U.ctx = ctx;
  std::vector<CountPlan> plans;
  cudaGraph_t cg = nullptr;
  cudaGraphExec_t cge = nullptr;
  DevTemps t(s);
  struct Release {
    kc_graph* U;
    std::vector<CountPlan>* plans;
    cudaGraph_t* cg;
    cudaGraphExec_t* cge;
    cudaEvent_t ev[7];
    ~Release() {
      if (*cge) cudaGraphExecDestroy(*cge);
      if (*cg) cudaGraphDestroy(*cg);
      for (auto& pl : *plans) count_release(&pl);
      free_union(U);
      for (cudaEvent_t e : ev) cudaEventDestroy(e);
    }
  } release{&U, &plans, &cg, &cge, {e0, e1, e2, e3, e4, ec, eo}};
  uint32_t *ds = nullptr, *dd = nullptr, *dvoff = nullptr, *dnn = nullptr, *derr = nullptr, *vg = nullptr;
  unsigned long long* deoff = nullptr;
  if (input == Input::kDeviceOwned) {
    if (edge_off[0] != 0) return fail(KC_ERR_INTERNAL, "in-place batch input must start at edge 0");
    ds = const_cast<uint32_t*>(src);
    dd = const_cast<uint32_t*>(dst);
  } else {
    KC_CUDA(t.alloc(&ds, sizeof(uint32_t) * std::max<uint64_t>(1, E)));
    KC_CUDA(t.alloc(&dd, sizeof(uint32_t) * std::max<uint64_t>(1, E)));
  }
  KC_CUDA(t.alloc(&deoff, sizeof(unsigned long long) * ((size_t)G + 1)));
  KC_CUDA(t.alloc(&dvoff, sizeof(uint32_t) * ((size_t)G + 1)));
  KC_CUDA(t.alloc(&dnn, sizeof(uint32_t) * G));
  KC_CUDA(t.alloc(&derr, sizeof(uint32_t) * 4));
  KC_CUDA(cudaMemsetAsync(derr, 0, sizeof(uint32_t) * 4, s));
  std::vector<unsigned long long> eoff_rel((size_t)G + 1);
  for (uint32_t g = 0; g <= G; ++g) eoff_rel[g] = edge_off[g] - edge_off[0];
  cudaEventRecord(e0, s);
  // host input is copied in and made global in place; device input is read
  // where it lies and written global into the temporaries
  const uint32_t* gin_s = ds;
  const uint32_t* gin_d = dd;
  if (E && input == Input::kHost) {
    KC_CUDA(cudaMemcpyAsync(ds, src + edge_off[0], sizeof(uint32_t) * E, cudaMemcpyHostToDevice, s));
    KC_CUDA(cudaMemcpyAsync(dd, dst + edge_off[0], sizeof(uint32_t) * E, cudaMemcpyHostToDevice, s));
  } else if (input == Input::kDevice) {
    gin_s = src + edge_off[0];
    gin_d = dst + edge_off[0];
  }
  KC_CUDA(cudaMemcpyAsync(deoff, eoff_rel.data(), sizeof(unsigned long long) * ((size_t)G + 1), cudaMemcpyHostToDevice, s));
  KC_CUDA(cudaMemcpyAsync(dvoff, voff.data(), sizeof(uint32_t) * ((size_t)G + 1), cudaMemcpyHostToDevice, s));
  KC_CUDA(cudaMemcpyAsync(dnn, n_nodes, sizeof(uint32_t) * G, cudaMemcpyHostToDevice, s));
  cudaEventRecord(e1, s);
  k_globalize<<<std::min<uint32_t>(G, 65535), 256, 0, s>>>(gin_s, gin_d, ds, dd, deoff, dvoff, dnn, G, derr);
  uint32_t herr = 0;
  KC_CUDA(cudaMemcpyAsync(&herr, derr, sizeof(uint32_t), cudaMemcpyDeviceToHost, s));
  KC_CUDA(cudaStreamSynchronize(s));
  if (herr) return fail(KC_ERR_INVALID_ARG, "graph %u has an endpoint not below its n_nodes", herr - 1);

  double th[6] = {t0, 0, 0, 0, 0, 0};  // host phase boundaries (stats->host_ms)
  th[1] = now_ms();
  kc_status st = build_csr(&U, ds, dd, E, (uint32_t)N);
  cudaEventRecord(ec, s);
  t.free_now(ds);
  t.free_now(dd);
  // graph of every original vertex: gives each graph a contiguous rank range
  if (st == KC_OK) {
    KC_CUDA(t.alloc(&vg, sizeof(uint32_t) * std::max<uint64_t>(1, N)));
    k_vertex_graph<<<std::min<uint32_t>(G, 65535), 256, 0, s>>>(dvoff, G, vg);
    U.vgraph_orig = vg;
    U.n_graphs = G;
    st = orient_graph(&U, orientation);
    cudaEventRecord(eo, s);
    U.vgraph_orig = nullptr;
  }
  if (st == KC_OK) st = dev_alloc(&U, (void**)&U.vgraph, sizeof(uint32_t) * std::max<uint64_t>(1, N));
  std::vector<uint32_t> fmax(G, 0), fcore(G, 0);
  std::vector<unsigned long long> fm(G, 0);
  if (st == KC_OK) {
    k_rank_graph<<<grid_for(N, ctx->sms), 256, 0, s>>>(vg, U.rank, (uint32_t)N, U.vgraph);
    uint32_t *dfmax = nullptr, *dfcore = nullptr;
    unsigned long long* dfm = nullptr;
    KC_CUDA(t.alloc(&dfmax, sizeof(uint32_t) * G));
    KC_CUDA(t.alloc(&dfcore, sizeof(uint32_t) * G));
    KC_CUDA(t.alloc(&dfm, sizeof(unsigned long long) * G));
    KC_CUDA(cudaMemsetAsync(dfmax, 0, sizeof(uint32_t) * G, s));
    KC_CUDA(cudaMemsetAsync(dfcore, 0, sizeof(uint32_t) * G, s));
    KC_CUDA(cudaMemsetAsync(dfm, 0, sizeof(unsigned long long) * G, s));
    k_graph_features<<<grid_for(N, ctx->sms), 256, 0, s>>>(U.drp, U.vgraph, U.inv, U.level, (uint32_t)N, dfmax, dfm,
                                                          dfcore);
    KC_CUDA(cudaMemcpyAsync(fmax.data(), dfmax, sizeof(uint32_t) * G, cudaMemcpyDeviceToHost, s));
    KC_CUDA(cudaMemcpyAsync(fcore.data(), dfcore, sizeof(uint32_t) * G, cudaMemcpyDeviceToHost, s));
    KC_CUDA(cudaMemcpyAsync(fm.data(), dfm, sizeof(unsigned long long) * G, cudaMemcpyDeviceToHost, s));
    cudaEventRecord(e2, s);
    KC_CUDA(cudaStreamSynchronize(s));
    t.free_now(dfmax);
    t.free_now(dfcore);
    t.free_now(dfm);
  }
  if (vg) t.free_now(vg);

  th[2] = now_ms();
  // per-graph choices, grouped into counting passes
  std::map<Choice, std::vector<uint32_t>> groups;
  std::vector<kc_params> picked(G);
  if (st == KC_OK) {
    for (uint32_t g = 0; g < G; ++g) {
      kc_params p;
      if (opts && opts->graph_params) {
        p = opts->graph_params[g];
      } else if (!opts || opts->autotune) {
        p = autotune(n_nodes[g], fm[g], fmax[g], ks[g], fcore[g], orientation);
      } else {
        p = opts->fixed;  // part 0: each size class sizes its own partitions
      }
      p.k = ks[g];
      if (ks[g] <= 2) p.unit = KC_UNIT_NODE;  // an edge unit cannot count 1-cliques
      p.flags = 0;
      if (p.mode > KC_MODE_AUTO || p.unit > 1 || p.encoding > 1 || p.part > 32 || (p.part & (p.part - 1))) {
        st = fail(KC_ERR_INVALID_ARG, "bad fixed parameters for the batch");
        break;
      }
      picked[g] = p;
      groups[Choice{p.mode, p.unit, p.part, p.encoding}].push_back(g);
    }
  }

  unsigned long long* dout = nullptr;
  uint32_t kernels = 0;
  uint64_t units = 0;
  if (st == KC_OK) {
    KC_CUDA(t.alloc(&dout, sizeof(unsigned long long) * 2 * G));
    plans.reserve(groups.size());
    for (auto& kv : groups) {
      std::vector<uint32_t> hk(G, 0xffffffffu);
      uint32_t kmax = 0;
      for (uint32_t g : kv.second) {
        hk[g] = ks[g];
        kmax = std::max(kmax, ks[g]);
      }
      uint32_t* dk = nullptr;
      KC_CUDA(t.alloc(&dk, sizeof(uint32_t) * G));
      KC_CUDA(cudaMemcpyAsync(dk, hk.data(), sizeof(uint32_t) * G, cudaMemcpyHostToDevice, s));
      CountRequest req;
      req.k = kmax;
      req.mode = kv.first.mode;
      req.unit = kv.first.unit;
      req.part = kv.first.part;
      req.encoding = kv.first.enc;
      req.flags = opts ? (opts->flags & KC_FLAG_STATS) : 0u;
      req.d_graph_k = dk;
      req.n_graphs = G;
      req.k_max = kmax;
      req.help = groups.size() == 1;  // passes side by side share the SMs
      plans.emplace_back();
      st = count_prepare(&U, req, dout, 0, &plans.back());
      if (st != KC_OK) break;
    }
  }
  // Passes of different methods are independent (each graph is in one pass):
  // with more than one, pass i runs on its own stream with its own class
  // streams, all forked from s and joined back to it, so the passes' long
  // tails (a pass ends with its slowest unit) overlap instead of adding up.
  if (st == KC_OK && plans.size() > 1) {
    st = ensure_pass_streams(ctx, plans.size());
    for (size_t i = 0; st == KC_OK && i < plans.size(); ++i)
      for (int c = 0; c < kNumClasses; ++c) plans[i].side[c] = ctx->pool[i * (kNumClasses + 1) + 1 + c];
  }
  auto enqueue_passes = [&]() -> kc_status {
    if (plans.size() == 1) return count_enqueue(plans[0], s);
    KC_CUDA(cudaEventRecord(ctx->pool_fork, s));
    kc_status r = KC_OK;
    size_t forked = 0;
    for (size_t i = 0; i < plans.size(); ++i) {
      cudaStream_t ps = ctx->pool[i * (kNumClasses + 1)];
      cudaError_t e = cudaStreamWaitEvent(ps, ctx->pool_fork, 0);
      if (e != cudaSuccess) {
        r = cuda_fail(e, "cudaStreamWaitEvent", __FILE__, __LINE__);
        break;
      }
      ++forked;
      r = count_enqueue(plans[i], ps);
      if (r != KC_OK) break;
    }
    // every forked pass stream joins s, also after an error (a capture
    // must end with every stream joined)
    for (size_t i = 0; i < forked; ++i) {
      cudaStream_t ps = ctx->pool[i * (kNumClasses + 1)];
      cudaEventRecord(ctx->pool_done[i], ps);
      cudaStreamWaitEvent(s, ctx->pool_done[i], 0);
    }
    return r;
  };
  if (st == KC_OK) {
    KC_CUDA(cudaMemsetAsync(dout, 0, sizeof(unsigned long long) * 2 * G, s));
    KC_CUDA(cudaStreamSynchronize(s));
    th[3] = now_ms();
    const bool use_graph = !opts || opts->use_graph;
    if (use_graph) {
      KC_CUDA(cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal));
      st = enqueue_passes();
      cudaError_t ce = cudaStreamEndCapture(s, &cg);
      if (st == KC_OK && ce != cudaSuccess) st = cuda_fail(ce, "cudaStreamEndCapture", __FILE__, __LINE__);
      if (st == KC_OK) {
        ce = cudaGraphInstantiate(&cge, cg, 0);
        if (ce != cudaSuccess) st = cuda_fail(ce, "cudaGraphInstantiate", __FILE__, __LINE__);
      }
      if (st == KC_OK) {
        cudaEventRecord(e3, s);
        ce = cudaGraphLaunch(cge, s);
        cudaEventRecord(e4, s);
        if (ce != cudaSuccess) st = cuda_fail(ce, "cudaGraphLaunch", __FILE__, __LINE__);
      }
    } else {
      cudaEventRecord(e3, s);
      st = enqueue_passes();
      cudaEventRecord(e4, s);
    }
  }
  unsigned long long trav[kStatsCount] = {};
  uint64_t heavy_units = 0;
  if (st == KC_OK) {
    bool deep = false;
    for (auto& pl : plans) {
      unsigned long long sv[kStatsCount] = {};
      uint32_t err = count_error(pl, s, sv);
      if (err == DEV_ERR_STACK) deep = true;
      else if (err && st == KC_OK) st = device_error_status(err);
      for (int q = 0; q < kStatsCount; ++q) trav[q] += sv[q];
      heavy_units += count_heavy(pl, s);
      units += count_units(pl, s);
      kernels += 5;
      for (int c = 0; c <= kNumClasses; ++c) kernels += pl.active[c] ? 1 : 0;
    }
    if (st == KC_OK && deep) {
      // a clique tree deeper than the fast stack: rerun every pass with full depth
      KC_CUDA(cudaMemsetAsync(dout, 0, sizeof(unsigned long long) * 2 * G, s));
      for (size_t i = 0; i < plans.size() && st == KC_OK; ++i) {
        CountRequest req = plans[i].req;
        count_release(&plans[i]);
        plans[i] = CountPlan();
        st = count_prepare(&U, req, dout, 1, &plans[i]);
        if (st == KC_OK) st = count_enqueue(plans[i], s);
        if (st == KC_OK) {
          uint32_t err = count_error(plans[i], s, nullptr);
          if (err) st = device_error_status(err);
        }
      }
    }
  }
  th[4] = now_ms();
  std::vector<unsigned long long> hout(2 * (size_t)G, 0);
  if (st == KC_OK) {
    KC_CUDA(cudaMemcpyAsync(hout.data(), dout, sizeof(unsigned long long) * 2 * G, cudaMemcpyDeviceToHost, s));
    KC_CUDA(cudaStreamSynchronize(s));
    for (uint32_t g = 0; g < G; ++g) {
      counts[g].lo = hout[2 * g];
      counts[g].hi = hout[2 * g + 1];
      if (choice) choice[g] = picked[g];
    }
  }
  if (stats) std::memset(stats, 0, sizeof(*stats));
  if (stats && st == KC_OK) {  // (a failed call may not have recorded the events)
    float a = 0, b = 0, c = 0;
    cudaEventElapsedTime(&a, e0, e1);
    cudaEventElapsedTime(&b, e1, e2);
    cudaEventElapsedTime(&c, e3, e4);
    stats->ms_h2d = a;
    stats->ms_build = b;
    stats->ms_count = c;
    cudaEventElapsedTime(&a, e1, ec);
    stats->ms_csr = a;
    cudaEventElapsedTime(&a, ec, eo);
    stats->ms_orient = a;
    stats->units = units;
    stats->kernels = kernels;
    stats->n_graphs = G;
    stats->tree_nodes = trav[0];
    stats->word_ops = trav[1];
    stats->gather_bytes = trav[2];
    stats->heavy_units = heavy_units;
    for (int q = 0; q < 3; ++q) stats->cycles[q] = trav[3 + q];
  }
  cudaStreamSynchronize(s);
  th[5] = now_ms();
  if (stats) {
    stats->ms_total = th[5] - t0;
    for (int q = 0; q < 5; ++q) stats->host_ms[q] = th[q + 1] > 0 && th[q] > 0 ? th[q + 1] - th[q] : 0.0;
    stats->n_vertices = N;
    stats->n_edges = U.m;
  }
  return st;
}

// Host-input batches larger than the context's chunk size: chunks of whole
// graphs of about that many edges are counted one after another, each as a
// batch of its own (the graphs are independent), while the next chunk's edges
// are copied to the device on the context's copy stream into the other of two
// staging buffers. Each chunk is counted in place from its staging buffer.
// Buffer b is refilled (for chunk c + 1) only after the chunk that used it
// last (c - 1) has returned, and run_batch returns only once its stream is
// idle.
kc_status run_batch_pipelined(kc_ctx* ctx, const uint32_t* src, const uint32_t* dst, const uint64_t* edge_off,
                              const uint32_t* n_nodes, const uint32_t* ks, uint32_t G, uint64_t chunk_edges,
                              const kc_batch_opts* opts, kc_u128* counts, kc_params* choice,
                              kc_batch_stats* stats) {
  const double t0 = now_ms();
  for (uint32_t g = 0; g < G; ++g)
    if (edge_off[g + 1] < edge_off[g]) return fail(KC_ERR_INVALID_ARG, "edge_off decreases at graph %u", g);
  // ceil(E / chunk_edges) chunks of about equal edges; chunk c holds graphs
  // [cut[c], cut[c + 1])
  const uint64_t E = edge_off[G] - edge_off[0];
  const uint64_t n_chunks = (E + chunk_edges - 1) / chunk_edges;
  const uint64_t target = (E + n_chunks - 1) / n_chunks;
  std::vector<uint32_t> cut{0};
  for (uint32_t g = 0; g + 1 < G; ++g)
    if (edge_off[g + 1] - edge_off[cut.back()] >= target) cut.push_back(g + 1);
  cut.push_back(G);
  const uint32_t C = (uint32_t)cut.size() - 1;
  uint64_t max_chunk = 1;
  for (uint32_t c = 0; c < C; ++c) max_chunk = std::max<uint64_t>(max_chunk, edge_off[cut[c + 1]] - edge_off[cut[c]]);

  cudaStream_t s = ctx->stream;
  if (!ctx->copy) KC_CUDA(cudaStreamCreateWithFlags(&ctx->copy, cudaStreamNonBlocking));
  DevTemps t(s);
  uint32_t* buf[2][2] = {};
  for (auto& b : buf)
    for (auto& a : b) KC_CUDA(t.alloc(&a, sizeof(uint32_t) * max_chunk));
  // events: the staging buffers allocated (stream-ordered on s), and the
  // start / end of every chunk's copy; the guard (destroyed before t frees
  // the buffers) waits for the copy stream on every return path
  struct Guard {
    cudaStream_t copy;
    std::vector<cudaEvent_t> ev;
    ~Guard() {
      cudaStreamSynchronize(copy);
      for (cudaEvent_t e : ev) cudaEventDestroy(e);
    }
  } guard{ctx->copy, {}};
  guard.ev.resize(1 + 2 * (size_t)C, nullptr);
  for (auto& e : guard.ev) KC_CUDA(cudaEventCreate(&e));
  cudaEvent_t ready = guard.ev[0];
  auto cb = [&](uint32_t c) { return guard.ev[1 + 2 * (size_t)c]; };
  auto ce = [&](uint32_t c) { return guard.ev[2 + 2 * (size_t)c]; };
  KC_CUDA(cudaEventRecord(ready, s));
  KC_CUDA(cudaStreamWaitEvent(ctx->copy, ready, 0));
  auto issue_copy = [&](uint32_t c) -> kc_status {
    const uint64_t e0 = edge_off[cut[c]], n = edge_off[cut[c + 1]] - e0;
    KC_CUDA(cudaEventRecord(cb(c), ctx->copy));
    if (n) {
      KC_CUDA(cudaMemcpyAsync(buf[c & 1][0], src + e0, sizeof(uint32_t) * n, cudaMemcpyHostToDevice, ctx->copy));
      KC_CUDA(cudaMemcpyAsync(buf[c & 1][1], dst + e0, sizeof(uint32_t) * n, cudaMemcpyHostToDevice, ctx->copy));
    }
    KC_CUDA(cudaEventRecord(ce(c), ctx->copy));
    return KC_OK;
  };
  KC_TRY(issue_copy(0));
  if (stats) std::memset(stats, 0, sizeof(*stats));
  kc_batch_stats sum;
  std::memset(&sum, 0, sizeof(sum));
  std::vector<uint64_t> rel;
  for (uint32_t c = 0; c < C; ++c) {
    if (c + 1 < C) KC_TRY(issue_copy(c + 1));
    KC_CUDA(cudaStreamWaitEvent(s, ce(c), 0));
    const uint32_t g0 = cut[c], gn = cut[c + 1] - cut[c];
    rel.resize((size_t)gn + 1);
    for (uint32_t i = 0; i <= gn; ++i) rel[i] = edge_off[g0 + i] - edge_off[g0];
    kc_batch_stats cs;
    kc_batch_opts co;
    if (opts) {
      co = *opts;
      if (co.graph_params) co.graph_params += g0;
    }
    KC_TRY(run_batch(ctx, buf[c & 1][0], buf[c & 1][1], Input::kDeviceOwned, rel.data(), n_nodes + g0, ks + g0, gn,
                     opts ? &co : nullptr, counts + g0, choice ? choice + g0 : nullptr, stats ? &cs : nullptr));
    if (!stats) continue;
    sum.ms_build += cs.ms_build;
    sum.ms_count += cs.ms_count;
    sum.ms_csr += cs.ms_csr;
    sum.ms_orient += cs.ms_orient;
    sum.units += cs.units;
    sum.kernels += cs.kernels;
    sum.tree_nodes += cs.tree_nodes;
    sum.word_ops += cs.word_ops;
    sum.gather_bytes += cs.gather_bytes;
    sum.heavy_units += cs.heavy_units;
    for (int q = 0; q < 3; ++q) sum.cycles[q] += cs.cycles[q];
    for (int q = 0; q < 5; ++q) sum.host_ms[q] += cs.host_ms[q];
    sum.n_vertices += cs.n_vertices;
    sum.n_edges += cs.n_edges;
  }
  KC_CUDA(cudaStreamSynchronize(ctx->copy));
  if (stats) {
    for (uint32_t c = 0; c < C; ++c) {
      float ms = 0;
      if (cudaEventElapsedTime(&ms, cb(c), ce(c)) == cudaSuccess) sum.ms_h2d += ms;
    }
    sum.n_graphs = G;
    sum.ms_total = now_ms() - t0;
    *stats = sum;
  }
  return KC_OK;
}

}  // namespace
}  // namespace kc

extern "C" {

kc_status kc_batch_count_packed(kc_ctx* ctx, const uint32_t* src, const uint32_t* dst, const uint64_t* edge_off,
                                const uint32_t* n_nodes, const uint32_t* k, uint32_t n_graphs,
                                const kc_batch_opts* opts, kc_u128* counts, kc_params* choice,
                                kc_batch_stats* stats) {
  if (!ctx) return kc::fail(KC_ERR_INVALID_ARG, "context is NULL");
  std::lock_guard<std::mutex> l(ctx->mu);
  cudaSetDevice(ctx->device);
  kc::clear_error();
  const uint64_t chunk = ctx->batch_chunk_edges ? ctx->batch_chunk_edges : kc::kDefaultBatchChunkEdges;
  if (src && dst && edge_off && n_nodes && k && counts && n_graphs > 1 && edge_off[n_graphs] >= edge_off[0] &&
      edge_off[n_graphs] - edge_off[0] > chunk)
    return kc::run_batch_pipelined(ctx, src, dst, edge_off, n_nodes, k, n_graphs, chunk, opts, counts, choice, stats);
  return kc::run_batch(ctx, src, dst, kc::Input::kHost, edge_off, n_nodes, k, n_graphs, opts, counts, choice, stats);
}

kc_status kc_batch_count_packed_device(kc_ctx* ctx, const uint32_t* d_src, const uint32_t* d_dst,
                                       const uint64_t* edge_off, const uint32_t* n_nodes, const uint32_t* k,
                                       uint32_t n_graphs, const kc_batch_opts* opts, kc_u128* counts,
                                       kc_params* choice, kc_batch_stats* stats) {
  if (!ctx) return kc::fail(KC_ERR_INVALID_ARG, "context is NULL");
  std::lock_guard<std::mutex> l(ctx->mu);
  cudaSetDevice(ctx->device);
  kc::clear_error();
  return kc::run_batch(ctx, d_src, d_dst, kc::Input::kDevice, edge_off, n_nodes, k, n_graphs, opts, counts, choice,
                       stats);
}

kc_status kc_batch_count(kc_ctx* ctx, const kc_batch_graph* graphs, uint32_t n_graphs, const kc_batch_opts* opts,
                         kc_u128* counts, kc_params* choice, kc_batch_stats* stats) {
  if (!ctx || (n_graphs && !graphs)) return kc::fail(KC_ERR_INVALID_ARG, "NULL argument");
  std::vector<uint64_t> off((size_t)n_graphs + 1, 0);
  for (uint32_t g = 0; g < n_graphs; ++g) {
    if (graphs[g].n_edges && (!graphs[g].src || !graphs[g].dst))
      return kc::fail(KC_ERR_INVALID_ARG, "graph %u: edge arrays are NULL", g);
    off[g + 1] = off[g] + graphs[g].n_edges;
  }
  std::vector<uint32_t> s(off[n_graphs]), d(off[n_graphs]), nn(n_graphs), kk(n_graphs);
  for (uint32_t g = 0; g < n_graphs; ++g) {
    if (graphs[g].n_edges) {
      std::memcpy(s.data() + off[g], graphs[g].src, sizeof(uint32_t) * graphs[g].n_edges);
      std::memcpy(d.data() + off[g], graphs[g].dst, sizeof(uint32_t) * graphs[g].n_edges);
    }
    nn[g] = graphs[g].n_nodes;
    kk[g] = graphs[g].k;
  }
  return kc_batch_count_packed(ctx, s.data(), d.data(), off.data(), nn.data(), kk.data(), n_graphs, opts, counts,
                               choice, stats);
}

}  // extern "C"
