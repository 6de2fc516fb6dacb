// Internal structures of the engine: the context, the device-resident graph
// and the stage entry points that the C ABI (engine.cu) strings together.
#pragma once
#include <cstdint>
#include <mutex>
#include <vector>

#include <cuda_runtime.h>

#include "../../include/kc.h"
#include "host_common.h"

struct kc_ctx {
  int device = 0;
  cudaStream_t stream = nullptr;
  int sms = 148;
  int max_smem_optin = 227 * 1024;
  uint64_t time_limit_ns = 0;  // device time limit of a counting pass (0 = none)
  // host-input batches of more edges than this run as a pipeline of chunks of
  // about this many edges, the next chunk's copy overlapping this one's work
  // (0 = kc::kDefaultBatchChunkEdges, UINT64_MAX = never)
  uint64_t batch_chunk_edges = 0;
  cudaStream_t copy = nullptr;  // host->device copies of the batch pipeline (created on first use)
  // Idle CTAs of a pivoting launch join units still being walked (tail
  // helping). Off for a context that shares the GPU with other busy contexts
  // (the server's workers): a helping grid holds its SMs until its last unit
  // ends, which would stall the other contexts' launches.
  bool tail_help = true;
  kc::BlockCache cache;        // device blocks reused by allocations on `stream`
  uint64_t total_mem = 0;
  std::mutex mu;  // one call at a time per context
  // exact binomial table C(r, c) as (lo, hi) pairs, rows [0, brows], cols [0, bcols]
  unsigned long long* d_binom = nullptr;
  uint32_t brows = 0, bcols = 0;
  std::vector<unsigned long long*> binom_retired;  // earlier, smaller tables (freed with the context)
  // the counting pass's size classes run side by side on these streams
  // (created on first use; calls on one context are serialised by mu)
  static constexpr int kSide = 4;
  cudaStream_t side[kSide] = {};
  cudaEvent_t fork = nullptr, join[kSide] = {};
  cudaEvent_t tbeg[kSide + 1] = {}, tend[kSide + 1] = {};  // per-launch timing
  // a batch's counting passes (one per method) run side by side: pass i on
  // pool[i (1 + kSide)], its class launches on the next kSide streams; done[i]
  // joins pass i back to `stream` (created on first use, grown as needed)
  std::vector<cudaStream_t> pool;
  std::vector<cudaEvent_t> pool_done;
  cudaEvent_t pool_fork = nullptr;
};

struct kc_graph {
  kc_ctx* ctx = nullptr;
  uint32_t n = 0;
  uint64_t m = 0;            // undirected edges
  uint32_t max_deg = 0;
  uint32_t* rp = nullptr;    // symmetric CSR, sorted rows, no duplicates / self-loops
  uint32_t* col = nullptr;
  // orientation (rank labels: vertex v has label rank[v]; u -> w iff rank[u] < rank[w])
  int oriented = -1;         // -1 none, else kc_orientation
  uint32_t* rank = nullptr;  // original id -> rank
  uint32_t* inv = nullptr;   // rank -> original id
  uint32_t* drp = nullptr;   // DAG row pointer, rank labels [n+1]
  uint32_t* dcol = nullptr;  // DAG columns (ranks), sorted per row [m]
  uint32_t* erow = nullptr;  // source rank of every DAG edge [m] (edge units)
  uint32_t max_out = 0;
  // degeneracy peel
  uint32_t* prio = nullptr;  // reference-compatible peel priority (original ids)
  uint32_t* level = nullptr; // peel level = core number (original ids)
  uint32_t max_core = 0;
  uint32_t peel_rounds = 0;  // sub-rounds that received a priority
  uint32_t* vgraph = nullptr; // batch: graph of every rank label (null for single graphs)
  // batch: graph of every original vertex, set before kc_orient so each
  // graph's vertices get one contiguous range of rank labels (null otherwise)
  const uint32_t* vgraph_orig = nullptr;
  uint32_t n_graphs = 0;
  uint64_t bytes = 0;
};

namespace kc {

// At most 160M edges (1.28 GB of u32 pairs, about 22 ms of host->device copy
// at 57 GB/s) per chunk, in chunks of equal size: few chunks, so their fixed
// costs (a counting tail each) stay small. The 10,000-graph batch (387M
// edges) runs as 3 chunks: 55.4k graphs/s end to end, against 51.1k in one
// pass, 49.7k in 2 chunks and 54.2k in 4.
constexpr uint64_t kDefaultBatchChunkEdges = 160ull << 20;

// A device allocation tracked against the graph's byte count.
kc_status dev_alloc(kc_graph* g, void** p, size_t bytes);
void dev_free(kc_graph* g, void* p);

// ---- stages (csr.cu, orient.cu, count.cu) ----
// Builds the symmetric CSR from device edge arrays; n == 0 infers n.
kc_status build_csr(kc_graph* g, const uint32_t* d_src, const uint32_t* d_dst, uint64_t n_edges,
                    uint32_t n_nodes);
kc_status orient_graph(kc_graph* g, uint32_t orientation);
kc_status ensure_edge_rows(kc_graph* g);
// Creates a context's side streams and a first binomial table, so the first
// count on it pays for neither.
kc_status warm_context(kc_ctx* ctx);
// Grows the context's pass streams to hold `passes` counting passes side by side.
kc_status ensure_pass_streams(kc_ctx* ctx, size_t passes);
kc_status peel_graph(kc_graph* g);  // fills prio / level / max_core

struct CountRequest {
  uint32_t k;
  uint32_t mode, unit, part, encoding, flags;
  // batch: per-graph k (device, indexed by vgraph) and per-graph output
  const uint32_t* d_graph_k = nullptr;
  uint32_t n_graphs = 1;
  uint32_t k_max = 0;
  // local counts (orientation mode): (lo, hi) per rank label, zeroed; null otherwise
  unsigned long long* d_local = nullptr;
  // context whose stream, side streams and scratch run the count (null: the
  // graph's own); another context of the same device may count a graph that
  // is complete (oriented, edge rows built), which the count then only reads
  kc_ctx* ctx = nullptr;
  // unit shard: this count takes the units whose index inside their size
  // class is = shard (mod n_shards); the shards' counts add up to the whole
  uint32_t shard = 0, n_shards = 1;
  // several k in one walk (pivoting, one graph): nk ascending values >= 3,
  // d_out then holds nk (lo, hi) pairs; k is the smallest, k_max the largest
  uint32_t nk = 0;
  uint32_t kset[32] = {};
  // tail helping for this pass (also needs kc_ctx::tail_help); off for the
  // passes of a batch that run side by side, for the reason given there
  bool help = true;
};

// Runs the counting stage; d_out holds n_graphs (lo, hi) pairs and must be zeroed.
kc_status count_graph(kc_graph* g, const CountRequest& req, unsigned long long* d_out,
                      kc_count_stats* stats);
// kc_count run by the context `run` (its stream, scratch and lock) on a graph
// of the same device; the graph must be complete (see CountRequest::ctx).
kc_status count_on(kc_ctx* run, kc_graph* g, const kc_params* p, kc_u128* out, kc_count_stats* stats,
                   uint32_t shard = 0, uint32_t n_shards = 1);
// kc_count_multi run by the context `run` (see count_on).
kc_status count_multi_on(kc_ctx* run, kc_graph* g, const kc_params* p, const uint32_t* ks, uint32_t n_k,
                         kc_u128* out);
// Completes an oriented graph for counting by other contexts: builds every
// array a count could create lazily and waits for the graph's stream.
kc_status complete_for_sharing(kc_graph* g);

kc_status truss_support(kc_graph* g, uint32_t* d_support);

// Exact binomial table on the device, grown on demand.
kc_status ensure_binom(kc_ctx* ctx, uint32_t rows, uint32_t cols);

// Autotuner: the kc_params a graph of this shape runs best with.
// Per-graph method for the batched engine and the server: the measured table
// (autotune_table.h) for degree-oriented graphs where its bucket was sampled,
// the shape rule otherwise.
kc_params autotune(uint32_t n, uint64_t m, uint32_t max_out, uint32_t k, uint32_t max_core, uint32_t orientation);

}  // namespace kc
