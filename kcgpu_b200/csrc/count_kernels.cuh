// Launch plan and kernel parameters of the counting kernels.
#pragma once
#include <cstddef>
#include <cstdint>
#include <cuda_runtime.h>

#include "engine.h"

namespace kc {

// Everything a counting kernel reads; plain pointers, filled on the host.
struct CountParams {
  const uint32_t* rp;        // DAG row pointer (rank labels)
  const uint32_t* col;       // DAG columns, sorted per row
  const uint32_t* erow;      // source of every DAG edge (edge units)
  const uint32_t* queue;     // all units, largest first
  uint32_t qstride;          // queue positions between this launch's units (the unit shards' count)
  const uint32_t* bounds;    // device [begin, count] per size class
  uint32_t cls;              // this launch's class
  uint32_t n_units_max;      // host upper bound on the class size (grid sizing)
  uint32_t edge_units;       // 0 node units, 1 edge units
  uint32_t edge_roots;       // node units whose root branches are their out-edges (edge units grouped by source)
  const uint32_t* vgraph;    // graph of every rank label, or null
  const uint32_t* gk;        // k of every graph, or null
  uint32_t k0;               // k when gk is null (the largest k with several k)
  uint32_t nk;               // several k in one walk (pivoting, one graph): how many, 0 = one k
  uint32_t kset[32];         // the k values, ascending; out holds nk (lo, hi) pairs
  unsigned long long* out;   // (lo, hi) per graph
  const unsigned long long* binom;  // C(r, c) as (lo, hi), row stride binom_cols + 1
  uint32_t binom_cols;
  uint32_t dcap;             // largest |S| of this launch
  uint32_t W;                // words per bitmap row at dcap
  uint32_t P;                // lanes per partition
  uint32_t G;                // threads per unit group (32 or blockDim.x)
  uint32_t depth;            // traversal stack frames per partition
  uint32_t fw;               // words per frame
  uint32_t pstride;          // words per partition: depth frames, then (pivoting) a candidate list of dcap
  uint32_t Q;                // pivoting: most lanes that score one candidate (0 = no bound)
  unsigned long long* local; // local counts: (lo, hi) per rank label, or null
  uint32_t off_loc;          // shared-memory offset of the per-vertex local counters (u64 each)
  uint32_t group_words;      // shared-memory words per group
  uint32_t off_B, off_R0, off_fr;  // shared-memory offsets (words) inside a group
  uint32_t off_H;            // shared-memory offset of the hash of S (keys, then local indices)
  uint32_t hash_T;           // hash slots (power of two >= 2 dcap), 0 = binary search instead
  uint32_t lane_dfs;         // orientation with one lane per subtree (rows of W = 1, 2 or 4 words)
  uint32_t bitmap_global, frames_global;
  uint32_t* gbuf;            // global scratch, gbuf_words per group
  size_t gbuf_words;
  size_t goff_fr;            // frames offset inside a group's global scratch
  uint32_t* ticket;          // unit ticket (zeroed)
  uint32_t* err;             // device error word
  unsigned long long* stats; // [0] tree nodes [1] word-ops [2] gather bytes [3..5] phase cycles, or null
  unsigned long long time_limit_ns;  // device time limit of the pass (0 = none)
  const unsigned long long* t0;      // the pass's start on the global timer
  uint32_t budget;           // traversal nodes a unit may use before it is handed on (0 = no limit)
  uint32_t* heavy;           // units over budget, counted again by the heavy pass
  uint32_t* heavy_count;     // their number (atomic)
  // Tail helping (pivoting, a CTA per unit, no local counts; null = off):
  // the cut-node ticket of every queue position (bit 31 once every cut node
  // of the unit is claimed), and per CTA of the launch 1 + the queue
  // position of the unit it walks (0 = none).
  uint32_t* help_ticket;
  uint32_t* help_active;
  // Class launches that help: CTAs that have exited, per class launch of the
  // plan, and each launch's grid (0 = not launched); null for the heavy pass
  uint32_t* class_exit;
  uint32_t class_grid[4];
};

struct LaunchPlan {
  uint32_t mode = 0, encoding = 0, part = 0;
  uint32_t q = 0;  // pivoting: lanes per candidate score (the request's partition size, 0 = per node)
  bool local = false;  // per-vertex (local) counts
  bool edge = false;
  uint32_t dcap = 0, G = 32, block = 128;
  bool force_global_bitmap = false;
  uint32_t k_max = 0;
  uint32_t depth_boost = 0;
};

// A prepared launch: parameters, grid and the scratch it owns.
struct PreparedLaunch {
  CountParams p;
  uint32_t grid = 0, block = 0;
  size_t smem = 0;
  void* kernel = nullptr;     // __global__ function
  uint32_t* gbuf = nullptr;   // global scratch (freed by release_launch)
  bool list = false;
  size_t cap_edges = 0;       // list encoding: edge capacity per group
};

// Lays out shared/global scratch for the plan, sizes the persistent grid and
// allocates the global scratch (stream-ordered on s). No kernel is launched.
kc_status prepare_launch(kc_ctx* ctx, const LaunchPlan& lp, const CountParams& p, cudaStream_t s,
                         PreparedLaunch* out);
kc_status prepare_launch_list(kc_ctx* ctx, const LaunchPlan& lp, const CountParams& p, cudaStream_t s,
                              PreparedLaunch* out);
// Enqueues the kernel (capturable: no allocation, no synchronisation).
kc_status enqueue_launch(const PreparedLaunch& pl, cudaStream_t s);
void release_launch(PreparedLaunch& pl, cudaStream_t s);

// Unit-size classes of the persistent queue; launch kNumClasses is the heavy
// pass (CTA per unit) over the warp-class units that ran over budget.
constexpr int kNumClasses = 4;
constexpr uint32_t kWarpClassMax = 128;   // largest unit a warp group takes
// (the batched step took 139.8 / 139.6 / 139.3 ms with 8192 / 4096 / 2048:
// the budget hands on 35k / 39k / 42k units, and their wasted listing and the
// heavy pass's extra work balance out)
#ifndef KC_UNIT_BUDGET
#define KC_UNIT_BUDGET 8192
#endif
constexpr uint32_t kUnitBudget = KC_UNIT_BUDGET;  // traversal nodes before a warp unit is handed on
#ifndef KC_PIVOT_UNIT_BUDGET
#define KC_PIVOT_UNIT_BUDGET 2048
#endif
// the same for a warp unit walked by pivoting (a pivot node costs more: its
// candidates are scored). Measured on R-MAT scale 16 (edge units, p8): k = 5
// took 29.7 / 20.8 / 17.4 ms and k = 6 115 / 102 / 100 ms with 8192 / 2048 /
// 1024; the serving mix was fastest with 2048.
constexpr uint32_t kPivotUnitBudget = KC_PIVOT_UNIT_BUDGET;
constexpr size_t kStaticSmemBytes = 64;
constexpr uint32_t kHelpMaxGrid = 2048;   // most CTAs of a launch that takes part in tail helping   // static shared memory of the bitmap kernel (phase clocks), kept off the plan

// Layout of a plan's scratch words (zeroed by every enqueue).
constexpr uint32_t kScratchWords = 48;
constexpr uint32_t kErrWord = 8;          // device error word
constexpr uint32_t kStatsWords = 16;      // six u64 counters: tree nodes, word-ops, gather bytes, phase cycles
constexpr int kStatsCount = 6;
constexpr uint32_t kClassBounds = 32;     // [begin, count] per class
constexpr uint32_t kHeavyBounds = 40;     // [0, heavy count]
constexpr uint32_t kStartWord = 44;       // u64: the pass's start on the global timer

// Everything one counting pass needs, allocated once; enqueue may be
// repeated and captured in a CUDA graph.
struct CountPlan {
  kc_graph* g = nullptr;
  kc_ctx* ctx = nullptr;    // runs the plan (the request's context, else the graph's)
  CountRequest req;
  bool edge = false;        // one unit per DAG edge
  bool edge_roots = false;  // edge units grouped by source: node units, edges as root branches
  uint32_t n_units = 0, max_size = 0;
  uint8_t* cls = nullptr;       // size class of every unit
  uint32_t* ccnt = nullptr;     // per-chunk class counts, then their exclusive scan
  uint32_t n_chunks = 0;
  uint32_t *queue = nullptr, *scratch = nullptr;
  uint32_t* heavy = nullptr;
  uint32_t* help = nullptr;  // tail-helping words (zeroed by every enqueue), help_words of them
  size_t help_words = 0;
  unsigned long long* d_out = nullptr;
  PreparedLaunch launches[kNumClasses + 1];
  bool active[kNumClasses + 1] = {false, false, false, false, false};
  // the class launches run side by side, each on its own stream (the
  // context's), so one class's tail overlaps the others' work; the heavy pass
  // follows them all
  cudaStream_t side[kNumClasses] = {};
  cudaEvent_t fork = nullptr, join[kNumClasses] = {};
  // per-launch timing (single-graph calls that ask for statistics)
  bool timed = false;
  cudaEvent_t tbeg[kNumClasses + 1] = {}, tend[kNumClasses + 1] = {};
};

kc_status count_prepare(kc_graph* g, const CountRequest& req, unsigned long long* d_out, uint32_t depth_boost,
                        CountPlan* pl);
kc_status count_enqueue(const CountPlan& pl, cudaStream_t s);
void count_release(CountPlan* pl);
// Reads the device error word (and the kStatsCount stats counters when stats != null).
uint32_t count_error(const CountPlan& pl, cudaStream_t s, unsigned long long* stats);
// The call's status for a non-zero device error word.
kc_status device_error_status(uint32_t err);
uint64_t count_units(const CountPlan& pl, cudaStream_t s);
// Units the last enqueue handed to the heavy pass.
uint32_t count_heavy(const CountPlan& pl, cudaStream_t s);

}  // namespace kc
