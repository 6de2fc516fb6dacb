/*
 * kc.h — C ABI of the B200 k-clique counting engine.
 *
 * This header is the drop-in boundary for the `-m kc` path of KCGPU. Every
 * entry point takes plain pointers and sizes; nothing here depends on torch or
 * on CUDA headers. Every call returns a kc_status and never exits the process;
 * kc_last_error() gives a message for the last failing call on this thread.
 *
 * Reference interfaces replaced (paths are inside the KCGPU tree):
 *   kc_graph_from_edges / kc_graph_from_csr
 *       graph::EdgeListFile::get_edges + CSRCOO::from_edgelist
 *       (include/FIleReader.cuh:383-411, include/CSRCOO.cuh:37-80) and the
 *       host->device copies of src/main.cu:104-160. Unlike the reference, the
 *       engine symmetrises, drops self-loops and removes duplicate edges on the
 *       GPU, and does not require sorted input.
 *   kc_orient
 *       the orientation block of src/main.cu:164-229: degree orientation
 *       (include/main_support.cuh:54-87 with node degrees) and degeneracy
 *       orientation (kcore/kcore.cuh:442-584 + include/main_support.cuh:89-128).
 *   kc_count
 *       graph::SingleGPU_Kclique<uint>::findKclqueIncremental_{node,edge}_
 *       {async,binary_async,pivot_async,nobin_pivot_async}<PSIZE>
 *       (kclique/kclique.cuh:1448-2623) as dispatched by src/main.cu:263-588.
 *       The count is returned as an exact unsigned 128-bit integer instead of
 *       being printed as "Counter = N" (kclique/kclique.cuh:1671-1672).
 *   kc_parse_spec
 *       parseKcConfig, the `-q [o|p]<part>[b|n|h]` grammar (include/Config.h:235-271).
 *   kc_kcore
 *       the degeneracy peeling of kcore/kcore.cuh:442-584 exposed on its own
 *       (max core and the per-vertex peel level).
 *   kc_truss_support
 *       no counterpart in the reference: KTRUSS is parsed (include/Config.h:66-67)
 *       but never dispatched by src/main.cu.
 *   kc_batch_count, kc_server_*
 *       no counterpart in the reference (one graph per process there).
 */
#ifndef KC_H_
#define KC_H_

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define KC_ABI_VERSION 1

typedef enum kc_status {
  KC_OK = 0,
  KC_ERR_INVALID_ARG = 1,     /* bad pointer, size, k, partition size, ... */
  KC_ERR_OOM = 2,             /* device or pinned-host allocation failed */
  KC_ERR_ADMISSION = 3,       /* projected HBM footprint above the budget */
  KC_ERR_DEVICE_TIMEOUT = 4,  /* a bounded device wait gave up */
  KC_ERR_CUDA = 5,            /* a CUDA runtime call failed */
  KC_ERR_INTERNAL = 6,        /* engine invariant violated (device error word) */
  KC_ERR_NOT_ORIENTED = 7,    /* kc_count before kc_orient */
  KC_ERR_CANCELLED = 8,       /* request cancelled before it ran */
  KC_ERR_BUSY = 9             /* result not ready yet (non-blocking poll) */
} kc_status;

typedef enum kc_orientation { KC_ORIENT_DEGREE = 0, KC_ORIENT_DEGEN = 1 } kc_orientation;
/* KC_MODE_ORIENT and KC_MODE_PIVOT are the reference's two algorithms (-q o|p).
 * KC_MODE_AUTO (an engine extension) lists each small unit by orientation and
 * switches a unit to pivoting when its traversal outgrows a fixed budget, and
 * pivots every large unit; the count is the same in every mode. */
typedef enum kc_mode { KC_MODE_ORIENT = 0, KC_MODE_PIVOT = 1, KC_MODE_AUTO = 2 } kc_mode;
typedef enum kc_unit { KC_UNIT_NODE = 0, KC_UNIT_EDGE = 1 } kc_unit;
typedef enum kc_encoding { KC_ENC_BITMAP = 0, KC_ENC_LIST = 1 } kc_encoding;

/* kc_params.flags */
#define KC_FLAG_STATS 0x1u   /* fill kc_count_stats (tree nodes, word-ops) */

/* An exact unsigned 128-bit count: value = hi * 2^64 + lo. */
typedef struct kc_u128 { uint64_t lo; uint64_t hi; } kc_u128;

/* The reference's KcliqueConfig (include/Config.h:13-19) plus k and unit. */
typedef struct kc_params {
  uint32_t k;          /* clique size, >= 1 */
  uint32_t mode;       /* kc_mode */
  uint32_t unit;       /* kc_unit */
  uint32_t part;       /* partition size 1,2,4,8,16,32 (0 = auto): lanes that walk one
                          subtree together (orientation), or the most lanes that
                          score one pivot candidate while a warp walks the tree
                          (pivoting) */
  uint32_t encoding;   /* kc_encoding */
  uint32_t flags;      /* KC_FLAG_* */
} kc_params;

/* Optional per-call statistics (KC_FLAG_STATS). */
typedef struct kc_count_stats {
  uint64_t units;          /* node or edge units that entered the traversal */
  uint64_t tree_nodes;     /* traversal tree nodes expanded */
  uint64_t word_ops;       /* 32-bit AND+POPC word operations (bitmap encoding) */
  uint64_t gather_bytes;   /* adjacency bytes read to build induced subgraphs */
  double   ms_total;       /* device time of the whole count (CUDA events) */
  double   ms_traversal;   /* device time of the traversal kernels */
  uint32_t max_unit_size;  /* largest induced subgraph (vertices) */
  uint32_t kernels;        /* kernels launched by the call */
  double   ms_launch[5];   /* device time of each size-class launch (units > 1024,
                              (128,1024], (32,128], <= 32 vertices) and of the
                              heavy pass; 0 where nothing was launched */
  uint64_t heavy_units;    /* units handed on to the heavy pass */
  uint32_t deep_retry;     /* 1 when a clique tree outgrew the fast stack and the
                              count was rerun with the full depth */
  uint32_t reserved;
  uint64_t cycles[3];      /* SM clock cycles the unit groups spent, summed over
                              groups: [0] forming S and its hash, [1] building the
                              induced subgraph (gathering the out-lists),
                              [2] the traversal */
} kc_count_stats;

typedef struct kc_graph_info {
  uint32_t n;               /* vertices */
  uint64_t m;               /* undirected edges after symmetrise + dedup */
  uint32_t max_degree;
  uint32_t oriented;        /* 0 = not yet, else 1 + kc_orientation */
  uint32_t max_out_degree;  /* D: largest DAG out-degree (after kc_orient) */
  uint32_t max_core;        /* largest peel level (after KC_ORIENT_DEGEN) */
  uint64_t device_bytes;    /* device memory held by this graph */
} kc_graph_info;

typedef struct kc_ctx kc_ctx;
typedef struct kc_graph kc_graph;

/* ---- context --------------------------------------------------------- */
kc_status kc_ctx_create(int device, kc_ctx** out);
kc_status kc_ctx_destroy(kc_ctx* ctx);
/* Message for the last failing call on this host thread ("" if none). */
const char* kc_last_error(void);
const char* kc_status_string(kc_status s);
/* Device time limit of one counting pass, in nanoseconds of the GPU's global
 * timer (0 = none, the default). The counting kernels read the timer whenever
 * a unit group takes its next unit; once the pass has run longer than the
 * limit they stop taking units, and the call (kc_count, kc_count_local,
 * kc_batch_count*) returns KC_ERR_DEVICE_TIMEOUT with no count. Units already
 * started finish, so the pass ends within one unit's time of the limit; the
 * context stays usable. A batched call runs one pass per group of graphs that
 * share a method, each with this limit. The reference has no counterpart (its
 * count runs to completion, src/main.cu:303-580). */
kc_status kc_ctx_set_time_limit(kc_ctx* ctx, uint64_t ns);
/* Host-input batches (kc_batch_count, kc_batch_count_packed) holding more
 * than `edges` edges are counted as a pipeline of ceil(edges in the batch /
 * `edges`) chunks of whole graphs of about equal size: while one chunk is
 * built and counted, the next chunk's edges are copied to the device on a
 * second stream, so the
 * host->device copy of all but the first chunk is hidden behind device work.
 * Counts and choices are the same as in one pass; kc_batch_stats add up the
 * chunks (ms_h2d is the copy stream's time). 0 = the default (160M edges),
 * UINT64_MAX = never split. Device-input batches always run in one pass. */
kc_status kc_ctx_set_batch_chunk_edges(kc_ctx* ctx, uint64_t edges);
/* Device memory the context keeps for reuse: the engine's temporaries and the
 * arrays of destroyed graphs go back to a per-context cache of blocks, so
 * repeated calls of the same sizes make no driver allocations (up to 16 GiB of
 * free blocks are kept). This returns every cached block to the driver. No
 * counterpart in the reference (it allocates and frees per call,
 * kclique/kclique.cuh:1448-2623). */
kc_status kc_ctx_release_cached_memory(kc_ctx* ctx);
/* The CUDA stream (a cudaStream_t) every call of this context runs on, so a
 * caller can order its own work or record timing events on it. */
kc_status kc_ctx_get_stream(kc_ctx* ctx, void** stream);
/* Kernels this library has launched in this process (including those
 * recorded into CUDA graphs), for accounting; monotonically increasing. */
uint64_t kc_kernel_launches(void);
/* Fault injection for tests, host side only (no counterpart in the reference,
 * whose allocation failures print and continue, include/utils.cuh:44-51).
 * kc_test_fail_alloc_after(n): the (n+1)-th device allocation the library makes
 * from now fails as out of memory (the call returns KC_ERR_OOM); one failure,
 * then the hook disarms; n < 0 disarms it. kc_test_live_allocations(): device
 * allocations of the library not yet freed, to check that failing calls leak
 * nothing. Process-wide, not per context. */
void kc_test_fail_alloc_after(int64_t n);
uint64_t kc_test_live_allocations(void);

/* ---- graphs ---------------------------------------------------------- */
/* Edge list in host memory (pageable or pinned). Both directions, duplicates
 * and self-loops are allowed; n_nodes = 0 infers max id + 1. */
kc_status kc_graph_from_edges(kc_ctx* ctx, const uint32_t* src, const uint32_t* dst,
                              uint64_t n_edges, uint32_t n_nodes, kc_graph** out);
/* Same, with src/dst already in device memory of the context's GPU. */
kc_status kc_graph_from_edges_device(kc_ctx* ctx, const uint32_t* d_src, const uint32_t* d_dst,
                                     uint64_t n_edges, uint32_t n_nodes, kc_graph** out);
/* Host CSR (row_ptr has n_nodes+1 entries); need not be symmetric or sorted. */
kc_status kc_graph_from_csr(kc_ctx* ctx, const uint32_t* row_ptr, const uint32_t* col_ind,
                            uint32_t n_nodes, kc_graph** out);
kc_status kc_graph_destroy(kc_graph* g);
kc_status kc_graph_get_info(const kc_graph* g, kc_graph_info* out);
/* Symmetric, sorted, deduplicated CSR: row_ptr[n+1], col_ind[2m] (host). */
kc_status kc_graph_get_csr(const kc_graph* g, uint32_t* row_ptr, uint32_t* col_ind);

/* ---- orientation ----------------------------------------------------- */
kc_status kc_orient(kc_graph* g, uint32_t orientation);
/* Oriented graph in the reference's layout: original vertex ids, each
 * out-list sorted by id; row_ptr[n+1], col_ind[m] (host). */
kc_status kc_graph_get_dag(const kc_graph* g, uint32_t* row_ptr, uint32_t* col_ind);
/* Degeneracy orientation only: the peel priority of every vertex as the
 * reference computes nodePriority (kcore/kcore.cuh:471-564), and the peel
 * level (core number) of every vertex. Either pointer may be NULL. */
kc_status kc_graph_get_peel(const kc_graph* g, uint32_t* priority, uint32_t* level);

/* ---- counting -------------------------------------------------------- */
kc_status kc_count(kc_graph* g, const kc_params* p, kc_u128* out, kc_count_stats* stats);
/* The counts for several k of one graph in one walk: out[i] = the number of
 * ks[i]-cliques, for n_k <= 32 values of k in any order (repeats allowed).
 * Pivoting with the binary encoding and p->unit (p->mode and p->part are
 * not used): the succinct clique tree is walked once to the largest k, and
 * every smaller k is taken where it closes (k - held <= 2) or at the leaves,
 * so the call costs about as much as kc_count at the largest k. No reference
 * counterpart (the reference counts one k per run, src/main.cu:263-588). */
kc_status kc_count_multi(kc_graph* g, const kc_params* p, const uint32_t* ks, uint32_t n_k, kc_u128* out);
/* One unit shard of kc_count, for counting one graph on several GPUs (each
 * process holds the whole graph and counts its shard; the caller adds the
 * shards' counts, e.g. with an all-gather of the 16-byte results). Units are
 * the node or edge units of kc_count, dealt out by position inside their size
 * class: unit j of a class goes to shard j mod n_shards, so neighbouring units
 * and the few largest ones are spread evenly. The counts of shards
 * 0..n_shards-1 add up to kc_count's for the same graph and parameters
 * (k <= 2 counts belong to shard 0). stats describe this shard's units. No
 * reference counterpart (the reference counts on one GPU; its unit windows
 * are kclique/kclique.cuh:1645-1675). */
kc_status kc_count_shard(kc_graph* g, const kc_params* p, uint32_t shard, uint32_t n_shards, kc_u128* out,
                         kc_count_stats* stats);
/* Local (per-vertex) counts, the reference's -m lkc: per_vertex[v] = number of
 * k-cliques that contain vertex v (host array of n, indexed by vertex id);
 * total (may be NULL) = the k-clique count. Binary encoding (list encoding is
 * KC_ERR_INVALID_ARG, as in the reference), orientation, pivoting or auto,
 * node or edge units: SingleGPU_Kclique_Local::findKclqueIncremental_{node,edge}_
 * {binary,pivot}_async_local (kclique/kclique_local.cuh:162-610, dispatched at
 * src/main.cu:590-760), with exact 128-bit counters instead of u64. */
kc_status kc_count_local(kc_graph* g, const kc_params* p, kc_u128* per_vertex, kc_u128* total);
/* Parse the reference's -q spec ("o8b", "p16n", ...) into mode/part/encoding. */
kc_status kc_parse_spec(const char* spec, kc_params* inout);

/* ---- k-core and k-truss support -------------------------------------- */
/* Per-vertex core number (host array of n, may be NULL) and the max core. */
kc_status kc_kcore(kc_graph* g, uint32_t* core, uint32_t* max_core);
/* sup(u,v) = |N(u) ∩ N(v)| for every undirected edge u<v, in the row-major
 * order of the upper triangle of the symmetric CSR (m entries, host). */
kc_status kc_truss_support(kc_graph* g, uint32_t* support);
/* No counterpart in the reference. The same supports as kc_truss_support for
 * callers that may not allocate device memory during the call (a plugin whose
 * host runtime owns all device memory, a latency-critical stream that must not
 * be stalled by cudaMalloc/cudaFree, a pipeline that reserves memory up
 * front). Inputs and output are device pointers on the current device: a
 * symmetric CSR with sorted, duplicate-free rows (d_row_ptr[n_nodes+1],
 * d_col_ind) and d_support with room for one value per undirected edge. Work
 * is enqueued on `stream` (a cudaStream_t, NULL = default stream) and nothing
 * is allocated: the only scratch is a fixed 1 MiB array inside the library, so
 * n_nodes may be at most 262,144 (larger graphs return KC_ERR_INVALID_ARG).
 * Calls on one device share that array: calls that overlap on the GPU race and
 * must be ordered by the caller. The first call on each device looks up the
 * array's address; make it before any stream capture begins. That address
 * lives in the device's primary context: after cudaDeviceReset the entry point
 * must not be called again in the process. */
kc_status kc_truss_support_noalloc(const uint32_t* d_row_ptr, const uint32_t* d_col_ind,
                                   uint32_t n_nodes, uint32_t* d_support, void* stream);

/* ---- batched counting ------------------------------------------------ */
/* One graph of a batch: an edge list in host memory plus its own k. */
typedef struct kc_batch_graph {
  const uint32_t* src;
  const uint32_t* dst;
  uint64_t n_edges;
  uint32_t n_nodes;
  uint32_t k;
} kc_batch_graph;

typedef struct kc_batch_opts {
  uint32_t orientation;   /* kc_orientation for every graph */
  uint32_t autotune;      /* 1 = choose mode/unit/part/encoding per graph */
  kc_params fixed;        /* used when autotune == 0 (k ignored) */
  uint32_t use_graph;     /* 1 = replay the counting stage as a captured CUDA graph */
  uint32_t flags;         /* KC_FLAG_STATS: fill the traversal counters below */
  const kc_params* graph_params;  /* NULL, or the method of every graph (n_graphs
                                     entries, k ignored): used instead of the
                                     autotuner and `fixed` */
} kc_batch_opts;

typedef struct kc_batch_stats {
  double ms_total;        /* host wall time of the call */
  double ms_h2d;          /* device time of host->device copies */
  double ms_build;        /* device time of CSR build + orientation */
  double ms_count;        /* device time of the counting launch */
  uint64_t units;
  uint32_t kernels;
  uint32_t n_graphs;
  uint64_t tree_nodes;    /* with KC_FLAG_STATS: traversal nodes expanded */
  uint64_t word_ops;      /* with KC_FLAG_STATS: 32-bit AND+POPC word operations */
  uint64_t gather_bytes;  /* with KC_FLAG_STATS: adjacency bytes read for induced subgraphs */
  uint64_t heavy_units;   /* units handed from a warp to the CTA-wide heavy pass */
  uint64_t cycles[3];     /* with KC_FLAG_STATS: SM cycles of the unit groups in
                             forming S, gathering the induced subgraph, traversing */
  double ms_csr;          /* device time of the CSR build (part of ms_build) */
  double ms_orient;       /* device time of the orientation (part of ms_build) */
  double host_ms[5];      /* host wall time of the call's phases: input checks and
                             copies, build + per-graph features, method choice and
                             plan set-up, capture + counting launch until done,
                             read-back and release */
  uint64_t n_vertices;    /* vertices of the batch */
  uint64_t n_edges;       /* undirected edges after symmetrising and dedup */
} kc_batch_stats;

/* Counts every graph of the batch; counts[i] receives graph i's count and
 * choice[i] (may be NULL) the kc_params the autotuner picked. */
kc_status kc_batch_count(kc_ctx* ctx, const kc_batch_graph* graphs, uint32_t n_graphs,
                         const kc_batch_opts* opts, kc_u128* counts, kc_params* choice,
                         kc_batch_stats* stats);

/* Same, with the whole batch packed as one edge list: graph i owns edges
 * [edge_off[i], edge_off[i+1]) with ids local to the graph. */
kc_status kc_batch_count_packed(kc_ctx* ctx, const uint32_t* src, const uint32_t* dst,
                                const uint64_t* edge_off, const uint32_t* n_nodes,
                                const uint32_t* k, uint32_t n_graphs,
                                const kc_batch_opts* opts, kc_u128* counts, kc_params* choice,
                                kc_batch_stats* stats);

/* Same as kc_batch_count_packed with src/dst already in device memory of the
 * context's GPU (edge_off, n_nodes and k stay in host memory). The caller's
 * arrays are not modified. */
kc_status kc_batch_count_packed_device(kc_ctx* ctx, const uint32_t* d_src, const uint32_t* d_dst,
                                       const uint64_t* edge_off, const uint32_t* n_nodes,
                                       const uint32_t* k, uint32_t n_graphs,
                                       const kc_batch_opts* opts, kc_u128* counts, kc_params* choice,
                                       kc_batch_stats* stats);

/* ---- serving ----------------------------------------------------------- */
typedef struct kc_server kc_server;

typedef struct kc_server_opts {
  uint64_t hbm_budget_bytes;  /* admission budget (0 = 180 GB or device total) */
  uint32_t max_inflight;      /* request slots on the device (0 = 8) */
  uint32_t streams;           /* device streams work overlaps on (0 = 4) */
  uint32_t orientation;       /* kc_orientation used for new graphs */
  uint32_t autotune;          /* 1 = autotune each request */
  kc_params fixed;            /* used when autotune == 0 */
} kc_server_opts;

typedef struct kc_request_result {
  kc_u128 count;
  kc_status status;
  uint32_t k;
  double submit_ms;     /* host clock, ms since the server started */
  double start_ms;      /* admitted and launched */
  double done_ms;       /* result available */
  uint64_t graph_id;
  kc_params params;     /* what ran */
} kc_request_result;

kc_status kc_server_create(kc_ctx* ctx, const kc_server_opts* opts, kc_server** out);
kc_status kc_server_destroy(kc_server* s);
/* Make a graph resident (copied now); returns an id for later requests. */
kc_status kc_server_put_graph(kc_server* s, const uint32_t* src, const uint32_t* dst,
                              uint64_t n_edges, uint32_t n_nodes, uint64_t* graph_id);
kc_status kc_server_drop_graph(kc_server* s, uint64_t graph_id);
/* Queue a count of k-cliques of a resident graph. */
kc_status kc_server_submit(kc_server* s, uint64_t graph_id, uint32_t k, uint64_t* ticket);
/* Queue a one-shot request whose graph is copied in and freed afterwards. */
kc_status kc_server_submit_edges(kc_server* s, const uint32_t* src, const uint32_t* dst,
                                 uint64_t n_edges, uint32_t n_nodes, uint32_t k,
                                 uint64_t* ticket);
kc_status kc_server_cancel(kc_server* s, uint64_t ticket);
/* wait_ms < 0 blocks; 0 polls (KC_ERR_BUSY if not done). */
kc_status kc_server_wait(kc_server* s, uint64_t ticket, int64_t wait_ms, kc_request_result* out);
/* Projected device footprint of a graph of this size (admission model). */
uint64_t kc_footprint_bytes(uint32_t n_nodes, uint64_t n_edges, uint32_t max_out_degree);

/* ---- synthetic inputs (host) ------------------------------------------- */
/* A host edge list owned by the library; pinned = 1 uses page-locked memory. */
typedef struct kc_edgelist kc_edgelist;

/* Graph files (graph::EdgeListFile, include/FIleReader.cuh:33-937), parsed on
 * host threads: KC_FILE_TEXT = one edge per line "src dst [anything]" (space,
 * tab or comma separated; '#' / '%' comment and blank lines skipped);
 * KC_FILE_MTX = Matrix Market coordinate, 1-based; KC_FILE_BEL = 24-byte
 * records {dst u64, src u64, weight u64} (:84-90). KC_FILE_AUTO picks by
 * extension (.bel, .mtx, else text). Malformed lines and ids of 2^32-1 or more
 * are KC_ERR_INVALID_ARG (with the line number). */
typedef enum { KC_FILE_AUTO = 0, KC_FILE_TEXT = 1, KC_FILE_MTX = 2, KC_FILE_BEL = 3 } kc_file_format;
kc_status kc_edgelist_from_file(const char* path, uint32_t format, int pinned, kc_edgelist** out);
/* kc_edgelist_from_file + kc_graph_from_edges. */
kc_status kc_graph_from_file(kc_ctx* ctx, const char* path, uint32_t format, kc_graph** out);
kc_status kc_edgelist_data(const kc_edgelist* e, const uint32_t** src, const uint32_t** dst,
                           uint64_t* n_edges, uint32_t* n_nodes);
kc_status kc_edgelist_destroy(kc_edgelist* e);
kc_status kc_gen_er(uint32_t n, double p, uint64_t seed, int pinned, kc_edgelist** out);
kc_status kc_gen_rmat(uint32_t scale, double edge_factor, double a, double b, double c,
                      uint64_t seed, int pinned, kc_edgelist** out);
kc_status kc_gen_chung_lu(uint32_t n, double exponent, double mean_degree, double max_degree,
                          uint64_t seed, int pinned, kc_edgelist** out);
kc_status kc_gen_sbm(uint32_t n, uint32_t blocks, double p_in, double p_out, uint64_t seed,
                     int pinned, kc_edgelist** out);
/* Adds cliques on disjoint random vertex sets, sizes uniform in [smin, smax]. */
kc_status kc_gen_plant_cliques(kc_edgelist* e, uint32_t count, uint32_t smin, uint32_t smax,
                               uint64_t seed);
/* The mixed batch of small graphs: graph g uses seed base+g; writes packed
 * edges plus per-graph offsets, sizes and k into caller-visible arrays held
 * by the returned list (see kc_batchgen_meta). */
kc_status kc_gen_batch(uint32_t n_graphs, uint64_t base_seed, uint32_t n_min, uint32_t n_max,
                       uint32_t k_min, uint32_t k_max, int pinned, kc_edgelist** out);
kc_status kc_batchgen_meta(const kc_edgelist* e, const uint64_t** edge_off,
                           const uint32_t** n_nodes, const uint32_t** k, const uint32_t** family,
                           uint32_t* n_graphs);

#ifdef __cplusplus
}
#endif
#endif /* KC_H_ */
