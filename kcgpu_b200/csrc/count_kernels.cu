// Bitmap-encoded counting kernels (orientation and pivoting) and the launch
// planner shared with the list-encoded kernels.
//
// One kernel body serves node and edge units; the unit only changes how the
// vertex set S is formed:
//   node unit u:     S = N+(u)                 (kckernels_orientation.cuh:357-377)
//   edge unit u->v:  S = N+(u) ∩ N+(v)         (kckernels_orientation.cuh:518-555)
// Orientation traversal (kckernels_orientation.cuh:380-470): every t-clique
// (t = k-1 for node units, k-2 for edge units) of the DAG on S is counted
// once from its lowest vertex; the last level is counted by popcount.
// Pivot traversal (kckernels_pivoting.cuh:124-338): the succinct clique tree
// with the max-neighbourhood pivot, ties to the smallest index; a leaf adds
// C(drop, k - held) from an exact table (the reference parses doubles,
// kclique/kclique.cuh:1694-1717). Where this differs from the reference in
// how, not what:
//   * a whole warp walks one tree node (the reference walks one node per
//     block with __syncthreads between steps); the launch's partition size
//     bounds the lanes that score one pivot candidate, as the reference's
//     partitions split the candidates of the block's node (:250-308);
//   * nodes with r = k - held <= 2 are closed: 1, |C| + drop, or
//     edges(G[C]) + drop |C| + C(drop, 2), instead of expanding their leaves;
//   * the pivot's own branch is taken last and reuses its parent's frame, so
//     the stack holds at most k - held0 + 1 frames;
//   * a unit's tree is cut at depth 1, 2 or 3 and the nodes at the cut go to
//     the unit's warps by ticket (a dense unit's root has few branches);
//   * edge units are grouped by source when N+(u) fits a shared-memory bitmap:
//     the unit u builds G[N+(u)] once and its out-edges are the root branches.
#include <algorithm>

#include "count_kernels.cuh"
#include "dev_common.cuh"

namespace kc {

namespace {

struct Part {
  uint32_t P, plane, pmask, pbase;
};

// First set bit of set[w0, W) (all lanes of the partition agree); -1 if none.
__device__ __forceinline__ int part_next_bit(const uint32_t* set, uint32_t w0, uint32_t W, const Part& pt,
                                             uint32_t* wi) {
  for (uint32_t base = w0; base < W; base += pt.P) {
    const uint32_t w = base + pt.plane;
    const uint32_t x = w < W ? set[w] : 0u;
    const uint32_t bal = (__ballot_sync(pt.pmask, x != 0u) & pt.pmask) >> pt.pbase;
    if (bal) {
      const uint32_t f = __ffs(bal) - 1;
      const uint32_t xv = __shfl_sync(pt.pmask, x, pt.pbase + f);
      *wi = base + f;
      return (int)((base + f) * 32u + (uint32_t)__ffs(xv) - 1u);
    }
  }
  return -1;
}

__device__ __forceinline__ uint32_t low_mask(uint32_t v, uint32_t w) {  // bits < v inside word w
  const uint32_t vw = v >> 5;
  return w < vw ? 0xffffffffu : (w == vw ? ((1u << (v & 31u)) - 1u) : 0u);
}

__device__ __forceinline__ uint32_t valid_mask(uint32_t d, uint32_t w) {  // bits < d inside word w
  return low_mask(d, w);
}

constexpr int kLaneStack = 16;  // lane-DFS levels: t - 2 <= 16, i.e. k <= 19 (node units)
constexpr uint32_t kGatherRun = 8;    // warp gather: consecutive out-list words per lane per iteration
constexpr uint32_t kSpanWords = 256;  // warp gather: membership map of up to 8192 rank labels

// Offset (words) of a warp unit's gather row table inside the hash / map
// region, which holds the hash (2 hT words) or the membership map and its
// prefix (2 kSpanWords words).
__host__ __device__ constexpr uint32_t gather_rows_at(uint32_t hT) {
  return hT > kSpanWords ? 2u * hT : 2u * kSpanWords;
}

template <int NW>
__device__ __forceinline__ void load_row(const uint32_t* B, uint32_t v, uint32_t (&r)[NW]) {
  if constexpr (NW == 4) {
    const uint4 q = *reinterpret_cast<const uint4*>(B + v * 4u);
    r[0] = q.x; r[1] = q.y; r[2] = q.z; r[3] = q.w;
  } else if constexpr (NW == 2) {
    const uint2 q = *reinterpret_cast<const uint2*>(B + v * 2u);
    r[0] = q.x; r[1] = q.y;
  } else {
    r[0] = B[v];
  }
}

// Position of the r-th (0-based) set bit of x (x has more than r set bits).
__device__ __forceinline__ uint32_t select_bit(uint32_t x, uint32_t r) {
  uint32_t pos = 0;
#pragma unroll
  for (uint32_t w = 16; w; w >>= 1) {
    const uint32_t lowc = __popc(x & ((1u << w) - 1u));
    if (r >= lowc) {
      r -= lowc;
      x >>= w;
      pos += w;
    }
  }
  return pos;
}

// Orientation traversal with one lane per subtree: the candidate set (NW
// words) lives in registers, rows come from shared memory with one vector
// load, and a lane's stack holds only the sets of the levels above it.
// Counts the t-cliques of the unit whose bitmap B has rows of stride NW.
// Lanes take subtrees by ticket: second-level vertices j (row j), or, when
// pre holds the exclusive prefix of the row popcounts (pre[d] = edges of
// G[S]), the third-level pairs (j, i), i in row j, with candidates
// row j ∩ row i: a unit's first rows are its largest, and splitting them
// keeps one lane from holding a warp's whole tail.
// Returns false when the unit ran over its budget (its count is then void).
template <int NW>
__device__ bool lane_dfs(const uint32_t* B, uint32_t d, uint32_t t, const uint32_t* pre, uint32_t* hdr,
                         uint32_t budget, unsigned __int128& uacc, unsigned long long& st_nodes,
                         unsigned long long& st_words) {
  uint32_t stk[kLaneStack][NW];
  unsigned long long cnt = 0;
  uint32_t since = 0;
  bool ok = true;
  const bool pairs = pre != nullptr;
  const uint32_t total = pairs ? pre[d] : d;
  t = pairs ? t - 1u : t;  // a pair's candidates complete (t-1)-cliques the same way a row's complete t-cliques
  for (;;) {
    if (budget && *(volatile uint32_t*)&hdr[5]) { ok = false; break; }
    const uint32_t tk = atomicAdd(&hdr[1], 1u);
    if (tk >= total) break;
    uint32_t cur[NW];
    if (pairs) {
      uint32_t lo = 0, hi = d;  // pre[lo] <= tk < pre[hi]
      while (hi - lo > 1u) {
        const uint32_t mid = (lo + hi) >> 1;
        if (pre[mid] <= tk) lo = mid;
        else hi = mid;
      }
      uint32_t rj[NW], ri[NW];
      load_row<NW>(B, lo, rj);
      uint32_t r = tk - pre[lo], i = 0;
      bool found = false;
#pragma unroll
      for (int q = 0; q < NW; ++q) {
        const uint32_t pc = __popc(rj[q]);
        if (!found && r < pc) {
          i = (uint32_t)q * 32u + select_bit(rj[q], r);
          found = true;
        } else if (!found) {
          r -= pc;
        }
      }
      load_row<NW>(B, i, ri);
#pragma unroll
      for (int q = 0; q < NW; ++q) cur[q] = rj[q] & ri[q];
    } else {
      load_row<NW>(B, tk, cur);
    }
    uint32_t c = 0;
#pragma unroll
    for (int q = 0; q < NW; ++q) c += __popc(cur[q]);
    st_nodes++;
    st_words += NW;
    if (t == 2u) { cnt += c; continue; }
    if (c < t - 1u) continue;
    int lv = 0;
    for (;;) {
      int w = -1;
#pragma unroll
      for (int q = NW - 1; q >= 0; --q)
        if (cur[q]) w = q;
      if (w < 0) {
        if (lv == 0) break;
        --lv;
#pragma unroll
        for (int q = 0; q < NW; ++q) cur[q] = stk[lv][q];
        continue;
      }
      uint32_t word = 0;
#pragma unroll
      for (int q = 0; q < NW; ++q)
        if (q == w) { word = cur[q]; cur[q] = word & (word - 1u); }
      const uint32_t v = (uint32_t)w * 32u + (uint32_t)__ffs(word) - 1u;
      uint32_t row[NW], child[NW];
      load_row<NW>(B, v, row);
      uint32_t n = 0;
#pragma unroll
      for (int q = 0; q < NW; ++q) {
        child[q] = cur[q] & row[q];
        n += __popc(child[q]);
      }
      st_nodes++;
      st_words += NW;
      const uint32_t rem = t - (uint32_t)(lv + 2);
      if (rem == 1u) {
        cnt += n;
      } else if (n >= rem && KC_IN_BOUNDS(lv, kLaneStack, nullptr)) {
#pragma unroll
        for (int q = 0; q < NW; ++q) {
          stk[lv][q] = cur[q];
          cur[q] = child[q];
        }
        ++lv;
      }
      if (budget && ++since >= 64u) {
        since = 0;
        if (atomicAdd(&hdr[4], 64u) + 64u > budget) hdr[5] = 1u;
        if (*(volatile uint32_t*)&hdr[5]) { ok = false; break; }
      }
    }
    if (!ok) break;
  }
  uacc += cnt;
  return ok;
}

// Register budgets: orientation fits 56 registers without spills (four
// 256-thread CTAs per SM); pivoting needs 80 (three), spilling below that.
template <int MODE, bool LOCAL>
__global__ void __launch_bounds__(256, MODE == 0 ? 4 : 3) k_count_bitmap(CountParams p) {
  extern __shared__ __align__(16) uint32_t smem[];
  const uint32_t G = p.G;
  const uint32_t gpb = blockDim.x / G;
  const uint32_t gib = threadIdx.x / G;
  const uint32_t gt = threadIdx.x - gib * G;
  const uint32_t lane = lane_id();
  const uint32_t wig = gt >> 5, nwg = G >> 5;
  Part pt;
  pt.P = p.P;
  pt.plane = gt % p.P;
  pt.pbase = (lane / p.P) * p.P;
  pt.pmask = p.P >= 32 ? 0xffffffffu : (((1u << p.P) - 1u) << pt.pbase);
  const uint32_t part = gt / p.P;
  // Several k in one walk (pivoting, one graph, p.nk > 0): the walk goes to
  // the largest k, and lane `plane` of every partition keeps the count of
  // kset[plane]. A clique-tree node with `hold` held vertices, `drop` pivots
  // and candidate set C adds sum_j C(drop, j) cliques(G[C], k - hold - j);
  // for a given k that sum is closed once k - hold <= 2, so k is taken
  // (closed) at the first node on a path where k - hold <= 2, and the node
  // below a non-pivot step from a parent with k - hold = 3 is where k - hold
  // first reaches 2. A k that is still open at a leaf (no candidates) adds
  // C(drop, k - hold) there.
  const bool mk = MODE == 1 && !LOCAL && p.nk != 0u;
  const bool kon = mk && pt.plane < p.nk;
  const uint32_t kl = kon ? p.kset[pt.plane] : 0u;

  uint32_t* sb = smem + (size_t)gib * p.group_words;
  uint32_t* gb = p.gbuf ? p.gbuf + (size_t)(blockIdx.x * gpb + gib) * p.gbuf_words : nullptr;
  uint32_t* hdr = sb;
  uint32_t* S = sb + 16;
  uint32_t* B = p.bitmap_global ? gb : sb + p.off_B;
  uint32_t* R0 = sb + p.off_R0;
  uint32_t* frames = (p.frames_global ? gb + p.goff_fr : sb + p.off_fr) + (size_t)part * p.pstride;
  uint32_t* cand = frames + (size_t)p.depth * p.fw;  // pivoting: the candidates of the node being entered
  // open-addressing hash of S: vertex -> local index (linear probing, load <= 1/2)
  const uint32_t hT = p.hash_T;
  uint32_t* hkey = sb + p.off_H;
  uint32_t* hval = hkey + hT;

  // class bounds come from device memory: clamp them so no unit index can leave the queue
  const uint32_t ubeg = min(p.bounds[2 * p.cls], p.n_units_max);
  const uint32_t ucnt = min(p.bounds[2 * p.cls + 1], (p.n_units_max - ubeg + p.qstride - 1) / p.qstride);
  unsigned __int128 acc = 0;
  uint32_t acc_graph = 0xffffffffu;
  unsigned long long st_nodes = 0, st_words = 0, st_bytes = 0;
  // With statistics, each group leader times its units' phases with the SM
  // clock: [0] forming S and its hash, [1] gathering the induced subgraph,
  // [2] traversing. Sums go to a per-block shared array, then to global.
  __shared__ unsigned long long blk_cy[3];
  const bool timing = p.stats != nullptr && gt == 0;
  if (p.stats != nullptr) {
    if (threadIdx.x < 3) blk_cy[threadIdx.x] = 0ull;
    __syncthreads();
  }
  uint32_t tc = 0;
  auto clk32 = []() -> uint32_t {
    uint32_t t;
    asm volatile("mov.u32 %0, %%clock;" : "=r"(t));
    return t;
  };
  auto lap = [&](int phase) {
    if (timing) {
      const uint32_t t = clk32();
      atomicAdd(&blk_cy[phase], (unsigned long long)(t - tc));  // a phase over 2^32 cycles (~2 s) wraps
      tc = t;
    }
  };

  auto gsync = [&]() {
    if (G == 32) __syncwarp(); else __syncthreads();
  };
  auto flush = [&]() {
    if (mk) {
      if (kon && acc != 0 && acc_graph != 0xffffffffu)
        atomic_add_u128(p.out + 2ull * ((size_t)acc_graph * p.nk + pt.plane), acc);
    } else if (pt.plane == 0 && acc != 0 && acc_graph != 0xffffffffu) {
      atomic_add_u128(p.out + 2ull * acc_graph, acc);
    }
    acc = 0;
  };

  // Work budget: a unit whose traversal exceeds p.budget nodes stops, drops
  // its partial count and is appended to the heavy list, which a CTA-wide
  // pass counts afterwards. Nodes are charged to hdr[4] in steps of 64 and
  // hdr[5] flags the stop; each partition keeps the unit's count in uacc
  // until the unit is known to have finished.
  const bool budgeted = p.budget != 0;
  unsigned __int128 uacc = 0;
  uint32_t since_charge = 0;
  auto over_budget = [&]() -> bool {  // partition-uniform
    uint32_t stop = 0;
    if (pt.plane == 0) {
      stop = *(volatile uint32_t*)&hdr[5];
      if (!stop && ++since_charge >= 64) {
        since_charge = 0;
        if (atomicAdd(&hdr[4], 64u) + 64u > p.budget) {
          hdr[5] = 1u;
          stop = 1u;
        }
      }
    }
    return __shfl_sync(pt.pmask, stop, pt.pbase) != 0u;
  };

  // Local (per-vertex) counts, orientation mode: every vertex of S keeps a
  // u64 counter in shared memory for the unit, the unit's own vertices (u,
  // and v for an edge unit) get the unit's total; both are added to the
  // global (lo, hi) counters when the unit commits.
  unsigned long long* loc = reinterpret_cast<unsigned long long*>(smem + (size_t)gib * p.group_words + p.off_loc);
  auto local_add_bits = [&](uint32_t w, uint32_t x) {  // +1 for every vertex of word w of a set
    for (; x; x &= x - 1u) atomicAdd(&loc[w * 32u + (uint32_t)__ffs(x) - 1u], 1ull);
  };
  // pivoting keeps a (lo, hi) pair per vertex of S (counts of large cliques pass 2^64)
  auto loc2_add = [&](uint32_t i, unsigned __int128 v) { atomic_add_u128(loc + 2ull * i, v); };

  // Tail helping: once the queue is empty, a CTA joins a unit that another
  // CTA is still walking. Every walker of a unit (its owner's partitions and
  // the helpers') walks the clique tree above the cut the same way and takes
  // the nodes at the cut by a global ticket; only the owner's partition 0
  // adds what lies above the cut. A walker that has been through all of the
  // unit's cut nodes holds a ticket past the last one, so every cut node is
  // taken: it sets bit 31 of the ticket, and no helper joins after that.
  const bool help = MODE == 1 && !LOCAL && p.help_ticket != nullptr;
  for (;;) {
    if (gt == 0) {
      uint32_t tk = atomicAdd(p.ticket, 1u);
      if (tk < ucnt && past_limit(p.time_limit_ns, p.t0)) {  // out of time: take no more units
        set_error(p.err, DEV_ERR_TIMEOUT);
        tk = 0xffffffffu;
      }
      hdr[0] = tk;
      hdr[1] = 0;  // subtree ticket of this unit
      hdr[4] = 0;  // nodes charged to this unit
      hdr[5] = 0;  // unit over budget
      hdr[6] = 0;  // helping: 1 + the queue position of the unit joined
    }
    gsync();
    const uint32_t ui = hdr[0];
    size_t pos = ubeg + (size_t)ui * p.qstride;
    bool helper = false;
    if (ui >= ucnt) {
      if (!help || ui == 0xffffffffu) break;
      // A CTA of a class launch helps only once the plan's other class
      // launches have finished (all their CTAs exited): while they run, its
      // slot serves them better than a share of another CTA's unit. The
      // heavy pass runs alone and always helps.
      if (p.class_exit != nullptr) {
        uint32_t busy = 0;
        if (gt == 0)
          for (int c = 0; c < kNumClasses; ++c)
            if (c != (int)p.cls && p.class_grid[c] != 0u &&
                *(volatile const uint32_t*)&p.class_exit[c] < p.class_grid[c])
              busy = 1;
        if (gt == 0) hdr[7] = busy;
        gsync();
        if (hdr[7]) break;
      }
      if (wig == 0) {  // the first warp looks for a unit still being walked
        const uint32_t nb = gridDim.x;
        uint32_t pick = 0;
        for (uint32_t i0 = 0; i0 < nb && pick == 0u; i0 += 32u) {
          uint32_t c = 0;
          if (i0 + lane < nb) {
            const uint32_t b = (blockIdx.x + 1u + i0 + lane) % nb;
            const uint32_t a = *(volatile const uint32_t*)&p.help_active[b];
            if (a != 0u && !(*(volatile const uint32_t*)&p.help_ticket[a - 1u] & 0x80000000u)) c = a;
          }
          const uint32_t m = __ballot_sync(0xffffffffu, c != 0u);
          if (m) pick = __shfl_sync(0xffffffffu, c, __ffs(m) - 1);
        }
        if (lane == 0) hdr[6] = pick;
      }
      gsync();
      const uint32_t a = hdr[6];
      if (a == 0u) break;
      helper = true;
      pos = a - 1u;
    }
    if (timing) tc = clk32();
    const uint32_t unit = p.queue[pos];
    uacc = 0;
    since_charge = 0;
    uint32_t src, d;
    if (!p.edge_units) {
      src = unit;
      const uint32_t b = p.rp[src];
      d = p.rp[src + 1] - b;
      if (d <= p.dcap)
        for (uint32_t j = gt; j < d; j += G) S[j] = p.col[b + j];
    } else {
      src = p.erow[unit];
      const uint32_t v = p.col[unit];
      if (wig == 0) {
        // S = N+(u) ∩ N+(v): stream the shorter list, search the longer
        const uint32_t ub = p.rp[src], ue = p.rp[src + 1], vb = p.rp[v], ve = p.rp[v + 1];
        const uint32_t *A, *L;
        uint32_t la, ll;
        if (ue - ub <= ve - vb) { A = p.col + ub; la = ue - ub; L = p.col + vb; ll = ve - vb; }
        else { A = p.col + vb; la = ve - vb; L = p.col + ub; ll = ue - ub; }
        uint32_t cnt = 0;
        for (uint32_t i0 = 0; i0 < la; i0 += 32) {
          const uint32_t i = i0 + lane;
          bool found = false;
          uint32_t x = 0;
          if (i < la) {
            x = A[i];
            const uint32_t pos = lower_bound_u32(L, ll, x);
            found = pos < ll && L[pos] == x;
          }
          const uint32_t bal = __ballot_sync(0xffffffffu, found);
          if (found && cnt + __popc(bal & lanemask_lt()) < p.dcap) S[cnt + __popc(bal & lanemask_lt())] = x;
          cnt += __popc(bal);
        }
        if (lane == 0) hdr[2] = cnt;
        st_bytes += 4ull * (la + la * 8ull);
      }
      gsync();
      d = hdr[2];
    }
    const uint32_t gph = p.vgraph ? p.vgraph[src] : 0u;
    const uint32_t k = p.gk ? p.gk[gph] : p.k0;
    gsync();
    if (gph != acc_graph) {
      flush();
      acc_graph = gph;
    }
    if (d > p.dcap) {
      if (gt == 0) set_error(p.err, DEV_ERR_CAPACITY);
      gsync();
      continue;
    }
    // row stride in words: the unit's own width, or the launch's fixed 1/2/4
    // words when rows are read with one vector load by the lane traversal
    const uint32_t W = p.lane_dfs ? p.W : (d + 31u) >> 5;
    const bool sym = MODE == 1;
    // pivoting reads 32 rows at once (one candidate per lane): an odd row
    // stride puts them in distinct shared-memory banks
    const uint32_t Ws = sym ? (W | 1u) : W;

    if (MODE == 0) {
      const uint32_t t = p.edge_units ? k - 2u : k - 1u;
      if (t <= 1u || d < t) {
        if (part == 0 && d >= t) acc += (t == 0u) ? 1u : d;
        if (LOCAL && d >= t && d <= p.dcap) {
          if (t == 1u)
            for (uint32_t i = gt; i < d; i += G) atomic_add_u128(p.local + 2ull * S[i], 1u);
          if (gt == 0) {
            const unsigned long long tot = (t == 0u) ? 1ull : d;
            atomic_add_u128(p.local + 2ull * src, tot);
            if (p.edge_units) atomic_add_u128(p.local + 2ull * p.col[unit], tot);
          }
        }
        gsync();
        continue;
      }
    } else if (mk) {
      // several k: every k with k - hold0 <= 1 is closed at the unit (the
      // unit is the clique, or one more vertex of S); the others need G[S]
      const uint32_t hold0 = p.edge_units ? 2u : 1u;
      // (into uacc: a unit that outruns its budget drops it with its walk,
      // and the heavy pass counts the whole unit again)
      const uint32_t r0 = kl - hold0;  // (wraps for kl < hold0: no contribution)
      if (part == 0 && !helper && kon && r0 <= 1u) uacc += (r0 == 0u) ? 1u : d;
      if (d == 0u || k < hold0 + 2u || hold0 + d < max(p.kset[0], hold0 + 2u)) {
        acc += uacc;
        gsync();
        continue;
      }
    } else {
      // k - hold0 <= 1: the unit's count is 1 (the unit is the clique) or d
      const uint32_t hold0 = p.edge_units ? 2u : 1u;
      if (d == 0u || hold0 + d < k || k <= hold0 + 1u) {
        if (part == 0 && !helper && k >= hold0 && hold0 + d >= k) acc += (k == hold0) ? 1u : d;
        if (LOCAL && k >= hold0 && hold0 + d >= k && d <= p.dcap) {
          if (k == hold0 + 1u)
            for (uint32_t i = gt; i < d; i += G) atomic_add_u128(p.local + 2ull * S[i], 1u);
          if (gt == 0) {
            const unsigned long long tot = (k == hold0) ? 1ull : d;
            atomic_add_u128(p.local + 2ull * src, tot);
            if (p.edge_units) atomic_add_u128(p.local + 2ull * p.col[unit], tot);
          }
        }
        gsync();
        continue;
      }
    }

    // ---- induced subgraph on S as a bitmap (row j, bit i: S[i] in N+(S[j]))
    for (uint32_t i = gt; i < d * Ws; i += G) B[i] = 0u;
    if (LOCAL)
      for (uint32_t i = gt; i < (MODE == 0 ? d : 2u * d); i += G) loc[i] = 0ull;
    const uint32_t hshift = hT ? 33u - (uint32_t)__ffs(hT) : 0u;  // 32 - log2(hT)
    // A warp unit whose S spans at most kSpanWords * 32 rank labels finds
    // local indices in a membership map of that span instead of the hash:
    // bit x - S[0] is set for every x of S, and mpre[w] counts the members in
    // the words below w, so x's local index (or, for a non-member, the index
    // it would take) is mpre[w] + popc(map[w] & bits below x). Every row
    // word lies in [S[0], ...): DAG out-lists hold only higher ranks.
    const uint32_t s0 = S[0], last = S[d - 1];
    const bool wmap = G == 32 && hT != 0u && last - s0 < kSpanWords * 32u;
    uint32_t* map = hkey;
    uint32_t* mpre = hkey + kSpanWords;
    if (wmap) {
      const uint32_t nmw = ((last - s0) >> 5) + 1u;
      for (uint32_t w = lane; w < nmw; w += 32u) map[w] = 0u;
      __syncwarp();
      for (uint32_t i = lane; i < d; i += 32u) {
        const uint32_t o = S[i] - s0;
        if (KC_IN_BOUNDS(o >> 5, kSpanWords, p.err)) atomicOr(&map[o >> 5], 1u << (o & 31u));
      }
      __syncwarp();
      uint32_t carry = 0;
      for (uint32_t w0 = 0; w0 < nmw; w0 += 32u) {
        const uint32_t w = w0 + lane;
        const uint32_t c = w < nmw ? (uint32_t)__popc(map[w]) : 0u;
        uint32_t incl = c;
#pragma unroll
        for (uint32_t o = 1; o < 32u; o <<= 1) {
          const uint32_t y = __shfl_up_sync(0xffffffffu, incl, o);
          if (lane >= o) incl += y;
        }
        if (w < nmw) mpre[w] = carry + incl - c;
        carry += __shfl_sync(0xffffffffu, incl, 31);
      }
    } else if (hT) {
      for (uint32_t i = gt; i < hT; i += G) hkey[i] = 0xffffffffu;
      gsync();
      for (uint32_t i = gt; i < d; i += G) {
        const uint32_t x = S[i];
        uint32_t h = (x * 0x9e3779b1u) >> hshift;
        while (atomicCAS(&hkey[h], 0xffffffffu, x) != 0xffffffffu) h = (h + 1u) & (hT - 1u);
        hval[h] = i;
      }
    }
    gsync();
    lap(0);
    if (G == 32 && hT) {
      // Warp unit: the out-lists of S's rows are read as one flat array,
      // 32 kGatherRun words per iteration with every lane's loads in flight
      // together, so the unit's whole gather costs a few memory latencies
      // instead of one per word of its longest row. The row table (start of
      // each row in col, exclusive prefix of the row lengths, rpre[d] = total)
      // follows the hash / map region; word f belongs to the last row j with
      // rpre[j] <= f.
      uint32_t* rbase = hkey + gather_rows_at(hT);
      uint32_t* rpre = rbase + p.dcap;
      uint32_t carry = 0;
      for (uint32_t j0 = 0; j0 < d; j0 += 32u) {
        const uint32_t j = j0 + lane;
        uint32_t b = 0, len = 0;
        if (j < d) {
          const uint32_t x0 = S[j];
          b = p.rp[x0];
          len = p.rp[x0 + 1] - b;
        }
        uint32_t incl = len;
#pragma unroll
        for (uint32_t o = 1; o < 32u; o <<= 1) {
          const uint32_t y = __shfl_up_sync(0xffffffffu, incl, o);
          if (lane >= o) incl += y;
        }
        if (j < d) {
          rbase[j] = b;
          rpre[j] = carry + incl - len;
        }
        carry += __shfl_sync(0xffffffffu, incl, 31);
      }
      const uint32_t total = carry;
      if (lane == 0) rpre[d] = total;
      __syncwarp();
      st_bytes += 4ull * (total + d);
      // Each lane takes kGatherRun consecutive words of the flat array per
      // iteration (lane L: words f0 + L kGatherRun ...), so one row search
      // serves the run: its first word's row is jb (the row of the previous
      // iteration's last word) plus the number of the next 32 row starts at or
      // below it (a search over one start per lane), or, past 32 rows, a
      // binary search of the rest; the later words of the run move forward
      // over row starts one at a time. Almost every gathered word is not in S:
      // a non-member costs one map (or hash) read, and only members pay for
      // their local index and the bitmap atomic.
      uint32_t jb = 0;
      for (uint32_t f0 = 0; f0 < total; f0 += 32u * kGatherRun) {
        const uint32_t t = jb + 1u + lane;
        const uint32_t cand = t <= d ? rpre[t] : 0xffffffffu;
        const uint32_t cand_last = __shfl_sync(0xffffffffu, cand, 31);
        const uint32_t fl = f0 + lane * kGatherRun;
        uint32_t c = 0;
#pragma unroll
        for (uint32_t sft = 16; sft; sft >>= 1)
          if (__shfl_sync(0xffffffffu, cand, c + sft - 1u) <= fl) c += sft;
        uint32_t j = jb + c;
        if (c == 31u && cand_last <= fl) {
          uint32_t hi = d;
          j = jb + 32u;
          while (hi - j > 1u) {
            const uint32_t mid = (j + hi) >> 1;
            if (rpre[mid] <= fl) j = mid;
            else hi = mid;
          }
        }
        uint32_t xs[kGatherRun], js[kGatherRun];
#pragma unroll
        for (uint32_t q = 0; q < kGatherRun; ++q) {
          const uint32_t f = fl + q;
          xs[q] = 0xffffffffu;
          if (f < total) {
            while (rpre[j + 1u] <= f) ++j;  // rpre[d] = total > f
            if (KC_IN_BOUNDS(j, d, p.err)) xs[q] = __ldg(p.col + rbase[j] + (f - rpre[j]));
          }
          js[q] = j;
        }
        jb = __shfl_sync(0xffffffffu, j, 31);
#pragma unroll
        for (uint32_t q = 0; q < kGatherRun; ++q) {
          const uint32_t x = xs[q];
          if (x > last) continue;  // past every vertex of S (also the padding)
          uint32_t lo = 0xffffffffu;
          if (wmap) {
            const uint32_t o = x - s0, mw = map[o >> 5];
            if ((mw >> (o & 31u)) & 1u) lo = mpre[o >> 5] + (uint32_t)__popc(mw & ((1u << (o & 31u)) - 1u));
          } else {
            uint32_t h = (x * 0x9e3779b1u) >> hshift;
            for (uint32_t hk; (hk = hkey[h]) != 0xffffffffu; h = (h + 1u) & (hT - 1u))
              if (hk == x) {
                lo = hval[h];
                break;
              }
          }
          if (lo == 0xffffffffu) continue;
          const uint32_t jr = js[q];
          if (KC_IN_BOUNDS(jr * Ws + (lo >> 5), d * Ws, p.err)) atomicOr(&B[jr * Ws + (lo >> 5)], 1u << (lo & 31u));
          if (sym && KC_IN_BOUNDS(lo * Ws + (jr >> 5), d * Ws, p.err))
            atomicOr(&B[lo * Ws + (jr >> 5)], 1u << (jr & 31u));
        }
      }
    } else {
      for (uint32_t j = wig; j < d; j += nwg) {
        const uint32_t x0 = S[j];
        const uint32_t b = p.rp[x0], e = p.rp[x0 + 1];
        uint32_t i0 = b;
        for (; i0 < e; i0 += 32) {
          const uint32_t i = i0 + lane;
          const uint32_t x = i < e ? __ldg(p.col + i) : 0xffffffffu;
          const bool inr = x <= last;
          if (!__any_sync(0xffffffffu, inr)) break;
          if (inr) {
            uint32_t lo = 0xffffffffu;
            if (hT) {
              // the hash holds every vertex of S; x may be absent (a miss)
              uint32_t h = (x * 0x9e3779b1u) >> hshift;
              for (uint32_t key; (key = hkey[h]) != 0xffffffffu; h = (h + 1u) & (hT - 1u))
                if (key == x) { lo = hval[h]; break; }
            } else {
              uint32_t a = j + 1, c = d;
              while (a < c) {
                const uint32_t mid = (a + c) >> 1;
                if (S[mid] < x) a = mid + 1; else c = mid;
              }
              if (a < d && S[a] == x) lo = a;
            }
            if (lo != 0xffffffffu && KC_IN_BOUNDS(lo, d, p.err)) {
              atomicOr(&B[j * Ws + (lo >> 5)], 1u << (lo & 31u));
              if (sym) atomicOr(&B[lo * Ws + (j >> 5)], 1u << (j & 31u));
            }
          }
        }
        st_bytes += 4ull * (e - b + 1u);  // the row and its vertex of S (warp-uniform)
      }
    }
    gsync();
    lap(1);

    if (mk) {
      // several k: the k with k - hold0 = 2 is the number of edges of G[S]
      const uint32_t hold0 = p.edge_units ? 2u : 1u;
      if (part == 0 && !helper) {
        unsigned long long e2 = 0;  // twice the edges: the bitmap is symmetric
        for (uint32_t j = pt.plane; j < d; j += pt.P)
          for (uint32_t w = 0; w < W; ++w) e2 += __popc(B[j * Ws + w]);
        for (uint32_t o = 1; o < pt.P; o <<= 1) e2 += __shfl_xor_sync(pt.pmask, e2, o);
        if (kon && kl == hold0 + 2u) uacc += e2 / 2u;
      }
      if (k <= hold0 + 2u) {
        acc += uacc;
        gsync();
        continue;
      }
    } else if (MODE == 1 && k == (p.edge_units ? 4u : 3u)) {
      // k - hold0 = 2: the unit's count is the number of edges of G[S]; a
      // vertex of S is in as many of those cliques as it has neighbours in S
      if (part == 0 && !helper) {
        unsigned long long e2 = 0;  // twice the edges: the bitmap is symmetric
        for (uint32_t j = pt.plane; j < d; j += pt.P) {
          uint32_t dj = 0;
          for (uint32_t w = 0; w < W; ++w) dj += __popc(B[j * Ws + w]);
          e2 += dj;
          if (LOCAL && dj) atomic_add_u128(p.local + 2ull * S[j], dj);
        }
        for (uint32_t o = 1; o < pt.P; o <<= 1) e2 += __shfl_xor_sync(pt.pmask, e2, o);
        acc += e2 / 2u;
        if (LOCAL && pt.plane == 0 && e2) {
          atomic_add_u128(p.local + 2ull * src, e2 / 2u);
          if (p.edge_units) atomic_add_u128(p.local + 2ull * p.col[unit], e2 / 2u);
        }
      }
      gsync();
      continue;
    }

    if (MODE == 0 && p.lane_dfs) {
      // ---- orientation traversal, one lane per subtree
      const uint32_t t = p.edge_units ? k - 2u : k - 1u;
      const uint32_t bud = budgeted ? p.budget : 0u;
      // for t >= 4, the exclusive prefix of the row popcounts, in the hash
      // region (free once the bitmap is built; 2 hT >= 8 dcap words)
      const uint32_t* pre = nullptr;
      if (hT != 0u && t >= 4u) {
        uint32_t carry = 0;
        for (uint32_t j0 = 0; j0 < d; j0 += 32u) {
          const uint32_t j = j0 + lane;
          uint32_t c = 0;
          if (j < d)
            for (uint32_t q = 0; q < W; ++q) c += __popc(B[j * W + q]);
          uint32_t incl = c;
          for (uint32_t o = 1; o < 32u; o <<= 1) {
            const uint32_t y = __shfl_up_sync(0xffffffffu, incl, o);
            if (lane >= o) incl += y;
          }
          if (j < d) hkey[j] = carry + incl - c;
          carry += __shfl_sync(0xffffffffu, incl, 31);
        }
        if (lane == 0) hkey[d] = carry;
        __syncwarp();
        pre = hkey;
      }
      if (W == 1u) lane_dfs<1>(B, d, t, pre, hdr, bud, uacc, st_nodes, st_words);
      else if (W == 2u) lane_dfs<2>(B, d, t, pre, hdr, bud, uacc, st_nodes, st_words);
      else lane_dfs<4>(B, d, t, pre, hdr, bud, uacc, st_nodes, st_words);
    } else if (MODE == 0) {
      // ---- orientation traversal
      const uint32_t t = p.edge_units ? k - 2u : k - 1u;
      for (;;) {
        if (budgeted && over_budget()) break;
        uint32_t j = 0;
        if (pt.plane == 0) j = atomicAdd(&hdr[1], 1u);
        j = __shfl_sync(pt.pmask, j, pt.pbase);
        if (j >= d) break;
        uint32_t* F0 = frames;
        const uint32_t ws = j >> 5;
        uint32_t c = 0;
        for (uint32_t w = ws + pt.plane; w < W; w += pt.P) {
          const uint32_t x = B[j * W + w];
          F0[w] = x;
          c += __popc(x);
        }
        c = __reduce_add_sync(pt.pmask, c);
        st_nodes++;
        st_words += W - ws;
        if (t == 2u) {
          uacc += c;
          if (LOCAL) {  // the edges (j, x), x in row j
            if (pt.plane == 0 && c) atomicAdd(&loc[j], (unsigned long long)c);
            for (uint32_t w = ws + pt.plane; w < W; w += pt.P) local_add_bits(w, F0[w]);
          }
          continue;
        }
        if (c < t - 1u) continue;
        if (pt.plane == 0) {
          F0[W] = ws;
          if (LOCAL) { F0[W + 1] = j; F0[W + 2] = F0[W + 3] = 0u; }
        }
        __syncwarp(pt.pmask);
        int lv = 0;
        while (lv >= 0) {
          if (budgeted && over_budget()) break;
          uint32_t* F = frames + (size_t)lv * p.fw;
          uint32_t wi = 0;
          const int vb = part_next_bit(F, F[W], W, pt, &wi);
          if (vb < 0) {
            if (LOCAL && pt.plane == 0) {
              // the frame's subtree total belongs to its vertex and to every ancestor
              const unsigned long long tot = ((unsigned long long)F[W + 3] << 32) | F[W + 2];
              if (tot) {
                atomicAdd(&loc[F[W + 1]], tot);
                if (lv > 0) {
                  uint32_t* Fp = F - p.fw;
                  const unsigned long long pt2 = (((unsigned long long)Fp[W + 3] << 32) | Fp[W + 2]) + tot;
                  Fp[W + 2] = (uint32_t)pt2;
                  Fp[W + 3] = (uint32_t)(pt2 >> 32);
                }
              }
            }
            __syncwarp(pt.pmask);
            --lv;
            continue;
          }
          const uint32_t v = (uint32_t)vb;
          __syncwarp(pt.pmask);
          if (pt.plane == 0) { F[wi] &= ~(1u << (v & 31u)); F[W] = wi; }
          __syncwarp(pt.pmask);
          const uint32_t rem = t - (uint32_t)(lv + 2);
          uint32_t* Fc = F + p.fw;
          const bool store = rem > 1u && (uint32_t)(lv + 1) < p.depth;
          uint32_t cc = 0;
          for (uint32_t w = wi + pt.plane; w < W; w += pt.P) {
            const uint32_t x = F[w] & B[v * W + w];
            if (store) Fc[w] = x;
            cc += __popc(x);
          }
          cc = __reduce_add_sync(pt.pmask, cc);
          st_nodes++;
          st_words += W - wi;
          if (rem == 1u) {
            uacc += cc;
            if (LOCAL && cc) {
              // the cliques path + v + x: v gets cc now, the path's frames
              // their totals on the way up, each x of the child one
              for (uint32_t w = wi + pt.plane; w < W; w += pt.P) local_add_bits(w, F[w] & B[v * W + w]);
              if (pt.plane == 0) {
                atomicAdd(&loc[v], (unsigned long long)cc);
                const unsigned long long t2 = (((unsigned long long)F[W + 3] << 32) | F[W + 2]) + cc;
                F[W + 2] = (uint32_t)t2;
                F[W + 3] = (uint32_t)(t2 >> 32);
              }
              __syncwarp(pt.pmask);
            }
          } else if (cc >= rem) {
            if (!store) {
              if (pt.plane == 0) set_error(p.err, DEV_ERR_STACK);
            } else {
              if (pt.plane == 0) {
                Fc[W] = wi;
                if (LOCAL) { Fc[W + 1] = v; Fc[W + 2] = Fc[W + 3] = 0u; }
              }
              __syncwarp(pt.pmask);
              ++lv;
            }
          }
        }
      }
    } else {
      // ---- pivot traversal (succinct clique tree)
      // Root: a pivot p0 of G[S] and its branches R0 = S \ N(p0). With edge
      // roots the root has no pivot: every v in S is a branch, the edge
      // (u, S[v]) whose subproblem is N+(u) ∩ N+(S[v]), the bits above v of
      // row v.
      const uint32_t hold0 = p.edge_units ? 2u : 1u;
      if (p.edge_roots) {
        if (gt == 0) hdr[3] = 0xffffffffu;
        for (uint32_t w = gt; w < W; w += G) R0[w] = valid_mask(d, w);
      } else {
        uint32_t key = 0;
        for (uint32_t v = gt; v < d; v += G) {
          uint32_t c = 0;
          for (uint32_t w = 0; w < W; ++w) c += __popc(B[v * Ws + w]);
          key = max(key, (c << 16) | (0xffffu - v));
        }
        key = __reduce_max_sync(0xffffffffu, key);
        if (lane == 0) hdr[8 + wig] = key;
        gsync();
        if (gt == 0) {
          uint32_t m = 0;
          for (uint32_t q = 0; q < nwg; ++q) m = max(m, hdr[8 + q]);
          hdr[3] = 0xffffu - (m & 0xffffu);
        }
        gsync();
        const uint32_t q0 = hdr[3];
        for (uint32_t w = gt; w < W; w += G) R0[w] = ~B[q0 * Ws + w] & valid_mask(d, w);
      }
      gsync();
      const uint32_t p0 = hdr[3];

      auto binom = [&](uint32_t nn, uint32_t r) -> unsigned __int128 {
        if (r > nn) return 0;
        const unsigned long long* e = p.binom + 2ull * ((size_t)nn * (p.binom_cols + 1u) + r);
        return ((unsigned __int128)e[1] << 64) | e[0];
      };
      // A clique-tree node with `hold` held vertices, `drop` pivots and the
      // candidate set F[0, W) contributes sum_j C(drop, j) * cliques(G[F], r - j)
      // with r = k - hold. For r <= 2 that sum is closed (cliques of size 0,
      // 1, 2 are 1, |F| and the edges of G[F]), so the subtree is not walked.
      // Otherwise the node's pivot and branch set are stored and it is pushed.
      // Frame: F [0, W), branches R [W, 2W), then hold, drop, pivot, cursor.
      // The pivot's branch goes last and reuses its parent's slot (nothing of
      // the parent is needed after it), so only non-pivot branches, which
      // each hold one more vertex, deepen the stack: at most k - hold0 + 1
      // levels, whatever the length of the drop chains.
      // With a full-warp walker and rows of at most 32 words (every launch
      // but the one for units above 1024 vertices) lane w holds word w of a
      // candidate set, and a ballot gives the words that hold candidates:
      // the listing and the scoring below visit only those.
      const bool narrow = pt.P == 32u && W <= 32u;
      const bool lc = LOCAL;  // local (per-vertex) counts
      unsigned __int128 leaf_cnt = 0, leaf_pinc = 0;
      // pchild: the node is its parent's pivot branch (same held vertices);
      // otherwise it holds one vertex more than its parent
      auto enter = [&](uint32_t* F, uint32_t hold, uint32_t drop, bool own, bool pchild) -> bool {
        uint32_t nc = 0, nzm = 0;
        if (narrow) {
          const uint32_t x = pt.plane < W ? F[pt.plane] : 0u;
          nc = __reduce_add_sync(pt.pmask, (uint32_t)__popc(x));
          nzm = __ballot_sync(pt.pmask, x != 0u);
        } else {
          for (uint32_t w = pt.plane; w < W; w += pt.P) nc += __popc(F[w]);
          nc = __reduce_add_sync(pt.pmask, nc);
        }
        const uint32_t r = k - hold;  // callers keep hold <= k
        // a node that ends here leaves (for local counts) leaf_cnt, its
        // cliques (each holds the node's held vertices), and leaf_pinc, the
        // cliques that hold any one of its pivots
        leaf_cnt = 0;
        leaf_pinc = 0;
        // several k: this lane's k is still open here if its k - hold was
        // at least 3 at the parent
        const bool kopen = kon && kl + (pchild ? 0u : 1u) >= hold + 3u;
        if (nc == 0u) {
          leaf_cnt = binom(drop, r);
          if (r >= 1u && drop >= 1u) leaf_pinc = binom(drop - 1u, r - 1u);
          if (own) uacc += mk ? (kopen ? binom(drop, kl - hold) : (unsigned __int128)0u) : leaf_cnt;
          return false;
        }
        if (hold + drop + nc < (mk ? p.kset[0] : k)) return false;
        if (r <= 1u) {  // (never with several k: an open k has k - hold >= 2 here)
          leaf_cnt = (r == 0u) ? (unsigned __int128)1u : (unsigned __int128)(nc + drop);
          leaf_pinc = (r == 1u && drop >= 1u) ? 1u : 0u;
          if (own && !mk) uacc += leaf_cnt;
          if (lc && own && r == 1u)  // each candidate c completes one clique
            for (uint32_t w = pt.plane; w < W; w += pt.P)
              for (uint32_t x = F[w]; x; x &= x - 1u) loc2_add(w * 32u + (uint32_t)__ffs(x) - 1u, 1u);
          return false;
        }
        // score every candidate u by |F ∩ N(u)|: the candidates are listed
        // in order first (one pass over the words, a bit per lane), then the
        // lanes take them in turn, so each lane scores ceil(nc / P) of them
        uint32_t best = 0;
        unsigned long long esum = 0;
        if (narrow) {
          uint32_t base = 0;
          for (uint32_t m = nzm; m; m &= m - 1u) {
            const uint32_t q = (uint32_t)__ffs(m) - 1u;
            const uint32_t x = F[q];
            const uint32_t ci = base + __popc(x & ((1u << pt.plane) - 1u));
            if (((x >> pt.plane) & 1u) && KC_IN_BOUNDS(ci, p.dcap, p.err)) cand[ci] = q * 32u + pt.plane;
            base += __popc(x);
          }
        } else {
          uint32_t base = 0;
          for (uint32_t q = 0; q < W; ++q) {
            const uint32_t x = F[q];
            if (x == 0u) continue;
            for (uint32_t b = pt.plane; b < 32u; b += pt.P)
              if (((x >> b) & 1u) && KC_IN_BOUNDS(base + __popc(x & ((1u << b) - 1u)), p.dcap, p.err))
                cand[base + __popc(x & ((1u << b) - 1u))] = q * 32u + b;
            base += __popc(x);
          }
        }
        __syncwarp(pt.pmask);
        // Q lanes score one candidate, each over every Q-th word: as many as
        // leave no lane idle (one per candidate once there are 32 of them),
        // at most the launch's partition size
        const uint32_t nw = narrow ? (uint32_t)__popc(nzm) : W;
        uint32_t Q = 1u;
        while ((Q << 1) * nc <= pt.P && Q < nw) Q <<= 1;
        if (p.Q != 0u && Q > p.Q) Q = p.Q;
        const uint32_t qs = (uint32_t)__ffs(Q) - 1u;  // Q is a power of two
        const uint32_t ng = pt.P >> qs, gq = pt.plane >> qs, lq = pt.plane & (Q - 1u);
        for (uint32_t i0 = 0; i0 < nc; i0 += ng) {
          const uint32_t i = i0 + gq;
          uint32_t c = 0, u = 0;
          if (i < nc) {
            u = cand[i];
            const uint32_t* Bu = B + u * Ws;
            if (narrow) {
              uint32_t j = 0;
              for (uint32_t m = nzm; m; m &= m - 1u, ++j)
                if ((j & (Q - 1u)) == lq) {
                  const uint32_t q = (uint32_t)__ffs(m) - 1u;
                  c += __popc(F[q] & Bu[q]);
                }
            } else {
              for (uint32_t q = lq; q < W; q += Q) c += __popc(F[q] & Bu[q]);
            }
          }
          for (uint32_t o = 1; o < Q; o <<= 1) c += __shfl_xor_sync(pt.pmask, c, o);
          if (i < nc && lq == 0u) {
            esum += c;
            best = max(best, (c << 16) | (0xffffu - u));
            // r = 2: candidate u is in a clique with each neighbour in F and each pivot
            if (lc && own && r == 2u && c + drop) loc2_add(u, c + drop);
          }
        }
        if (own) st_words += (unsigned long long)nc * nw / pt.P;
        for (uint32_t o = 1; o < pt.P; o <<= 1) esum += __shfl_xor_sync(pt.pmask, esum, o);
        if (r == 2u) {  // edges of G[F] + drop * |F| + C(drop, 2)
          leaf_cnt = (unsigned __int128)(esum / 2u) + (unsigned __int128)drop * nc + binom(drop, 2u);
          leaf_pinc = drop >= 1u ? (unsigned __int128)(nc + drop - 1u) : 0u;
          if (own) uacc += mk ? ((kopen && kl == hold + 2u) ? leaf_cnt : (unsigned __int128)0u) : leaf_cnt;
          return false;
        }
        // several k: a smaller k that reaches k - hold = 2 here is closed here
        if (mk && own && kopen && kl == hold + 2u)
          uacc += (unsigned __int128)(esum / 2u) + (unsigned __int128)drop * nc + binom(drop, 2u);
        best = __reduce_max_sync(pt.pmask, best);
        const uint32_t piv = 0xffffu - (best & 0xffffu);
        // branch set: candidates outside N(piv), less the pivot itself, whose
        // branch is taken last in this frame's own slot
        for (uint32_t w = pt.plane; w < W; w += pt.P) {
          uint32_t rw = F[w] & ~B[piv * Ws + w];
          if (w == (piv >> 5)) rw &= ~(1u << (piv & 31u));
          F[W + w] = rw;
        }
        __syncwarp(pt.pmask);
        if (pt.plane == 0) {
          F[2 * W] = hold;
          F[2 * W + 1] = drop;
          F[2 * W + 2] = piv;
          F[2 * W + 3] = 0;
        }
        __syncwarp(pt.pmask);
        return true;
      };

      // Work split inside the unit: the clique tree (root at depth 0) is cut
      // at depth L and the nodes at depth L go out by ticket (hdr[1]) to the
      // group's partitions. Every partition walks the levels above the cut
      // itself, re-deriving the same pivots, so no frame crosses partitions;
      // partition 0 alone adds what the nodes above the cut contribute.
      // L grows when the root has few branches (dense units, whose pivot
      // neighbours nearly everything).
      // The cut is sized for the CTA's own partitions (helpers take what is
      // left of it): a deeper cut would make every walker, helpers included,
      // walk more levels above it, and on bushy trees that costs more than
      // the finer split gains.
      const uint32_t nparts = G / pt.P;
      uint32_t nr0 = 0;
      for (uint32_t w = pt.plane; w < W; w += pt.P) nr0 += __popc(R0[w]);
      nr0 = __reduce_add_sync(pt.pmask, nr0);
      const uint32_t L = (nparts == 1u || nr0 >= 4u * nparts) ? 1u : (nr0 <= 2u ? 3u : 2u);
      const bool top_owner = part == 0u && !helper;
      uint32_t* cut_ticket = help ? p.help_ticket + pos : &hdr[1];
      if (help && !helper && gt == 0) {  // the unit can take helpers from now on
        __threadfence();
        *(volatile uint32_t*)&p.help_active[blockIdx.x] = (uint32_t)pos + 1u;
      }
      auto ticket = [&]() -> uint32_t {
        uint32_t t = 0;
        if (pt.plane == 0) t = atomicAdd(cut_ticket, 1u);
        return __shfl_sync(pt.pmask, t, pt.pbase);
      };
      uint32_t seen = 0, mine = ticket();
      auto claim = [&]() -> bool {  // at a depth-L node: does this partition take it?
        const bool take = seen == mine;
        ++seen;
        if (take) mine = ticket();
        return take;
      };

      // Local counts: a frame also keeps its held vertex (the branch that
      // pushed it; none for the root pivot's branch), where its pivots start
      // in the walker's drop list, and the totals of the cliques ended below
      // it: T_H (each holds the frame's held vertices) and T_P (cliques that
      // hold any one of the frame's pivots). A pivot joins the list with
      // minus the T_P reached so far and gets the final T_P when its frame
      // pops; totals then move up to the parent frame.
      uint32_t* dl = cand + ((p.dcap + 3u) & ~3u);
      uint32_t ndl = 0;
      auto fr_get = [&](const uint32_t* F, uint32_t off) -> unsigned __int128 {
        const uint32_t* q = F + 2u * W + off;
        return ((unsigned __int128)q[3] << 96) | ((unsigned __int128)q[2] << 64) |
               ((unsigned __int128)q[1] << 32) | q[0];
      };
      auto fr_set = [&](uint32_t* F, uint32_t off, unsigned __int128 v) {
        uint32_t* q = F + 2u * W + off;
        q[0] = (uint32_t)v;
        q[1] = (uint32_t)(v >> 32);
        q[2] = (uint32_t)(v >> 64);
        q[3] = (uint32_t)(v >> 96);
      };
      auto fr_open = [&](uint32_t* F, uint32_t held) {  // plane 0
        F[2 * W + 4] = held;
        F[2 * W + 5] = ndl;
        fr_set(F, 6, 0);
        fr_set(F, 10, 0);
      };
      auto fr_take = [&](uint32_t* F) {  // a node that ended in this frame's slot (plane 0)
        fr_set(F, 6, fr_get(F, 6) + leaf_cnt);
        fr_set(F, 10, fr_get(F, 10) + leaf_pinc);
      };
      auto fr_close = [&](uint32_t* F, int level) {  // the frame pops (plane 0)
        const unsigned __int128 th = fr_get(F, 6), tp = fr_get(F, 10);
        const uint32_t hv = F[2 * W + 4], st = F[2 * W + 5];
        if (hv != 0xffffffffu && th) loc2_add(hv, th);
        if (tp)
          for (uint32_t i = st; i < ndl; ++i) loc2_add(dl[i], tp);
        if (level > 0) {
          uint32_t* Fp = F - p.fw;
          fr_set(Fp, 6, fr_get(Fp, 6) + th);
          fr_set(Fp, 10, fr_get(Fp, 10) + tp);
        }
      };

      for (uint32_t v = 0; v < d; ++v) {
        if (budgeted && over_budget()) break;
        if (!((R0[v >> 5] >> (v & 31u)) & 1u)) continue;
        if (L == 1u && !claim()) continue;
        const bool own1 = L == 1u || top_owner;
        const uint32_t hold = hold0 + (v != p0 ? 1u : 0u), drop = (v == p0) ? 1u : 0u;
        if (own1) st_nodes++;
        if (hold > k) continue;
        uint32_t* F0 = frames;
        for (uint32_t w = pt.plane; w < W; w += pt.P) F0[w] = B[v * Ws + w] & ~(R0[w] & low_mask(v, w));
        __syncwarp(pt.pmask);
        if (!enter(F0, hold, drop, own1, v == p0)) {
          if (lc && own1 && pt.plane == 0) {
            const unsigned __int128 x = (v != p0) ? leaf_cnt : leaf_pinc;
            if (x) loc2_add(v, x);
          }
          __syncwarp(pt.pmask);
          continue;
        }
        if (lc) {
          ndl = 0;
          if (pt.plane == 0) {
            fr_open(F0, v != p0 ? v : 0xffffffffu);
            if (v == p0) dl[0] = p0;  // the root pivot is a pivot of this whole subtree
          }
          ndl = (v == p0) ? 1u : 0u;
          __syncwarp(pt.pmask);
        }
        int lv = 0;
        while (lv >= 0) {
          if (budgeted && over_budget()) break;
          uint32_t* F = frames + (size_t)lv * p.fw;
          uint32_t wi = 0;
          const int vb = part_next_bit(F + W, F[2 * W + 3], W, pt, &wi);
          const uint32_t fh = F[2 * W], fd = F[2 * W + 1], fp = F[2 * W + 2];
          if (vb < 0) {
            // every other branch is done: the pivot's branch replaces the frame
            const bool own = (uint32_t)lv + 1u >= L || top_owner;
            if (own) st_nodes++;
            __syncwarp(pt.pmask);
            if (lc) {  // fp joins this frame's pivots
              if (pt.plane == 0) {
                dl[ndl] = fp;
                const unsigned __int128 tp = fr_get(F, 10);
                if (tp) loc2_add(fp, (unsigned __int128)0 - tp);
              }
              ++ndl;
            }
            for (uint32_t w = pt.plane; w < W; w += pt.P) F[w] &= B[fp * Ws + w];
            __syncwarp(pt.pmask);
            if (!enter(F, fh, fd + 1u, own, true)) {
              if (lc) {
                if (pt.plane == 0) {
                  if (own) fr_take(F);
                  fr_close(F, lv);
                }
                __syncwarp(pt.pmask);
                ndl = F[2 * W + 5];
                __syncwarp(pt.pmask);
              }
              --lv;
            }
            continue;
          }
          const uint32_t u = (uint32_t)vb;
          __syncwarp(pt.pmask);
          if (pt.plane == 0) {
            F[W + wi] &= ~(1u << (u & 31u));
            F[2 * W + 3] = wi;
          }
          const uint32_t h2 = fh + 1u;  // u is not the pivot
          bool descend = h2 <= k;
          if (descend && (uint32_t)(lv + 1) >= p.depth) {
            if (pt.plane == 0) set_error(p.err, DEV_ERR_STACK);
            descend = false;
          }
          bool own = (uint32_t)lv + 2u > L || top_owner;
          if (descend && (uint32_t)lv + 2u == L) own = descend = claim();
          if (own) st_nodes++;
          uint32_t* Fc = F + p.fw;
          if (descend)
            for (uint32_t w = pt.plane; w < W; w += pt.P) Fc[w] = F[w] & B[u * Ws + w];
          __syncwarp(pt.pmask);
          if (pt.plane == 0) F[u >> 5] &= ~(1u << (u & 31u));  // later siblings exclude u
          __syncwarp(pt.pmask);
          if (descend && enter(Fc, h2, fd, own, false)) {
            if (lc) {
              if (pt.plane == 0) fr_open(Fc, u);
              __syncwarp(pt.pmask);
            }
            ++lv;
          } else if (descend && lc && own) {
            // the child ended at once: u holds its cliques, this frame takes them too
            if (pt.plane == 0) {
              if (leaf_cnt) loc2_add(u, leaf_cnt);
              fr_take(F);
            }
            __syncwarp(pt.pmask);
          }
        }
      }
      // this walker has been through every cut node: all of them are taken
      if (help && pt.plane == 0) atomicOr(cut_ticket, 0x80000000u);
    }
    gsync();
    lap(2);
    if (help && !helper && gt == 0) *(volatile uint32_t*)&p.help_active[blockIdx.x] = 0u;
    // commit the unit, or hand it to the heavy pass when it ran over budget
    if (budgeted && hdr[5]) {
      if (gt == 0) p.heavy[atomicAdd(p.heavy_count, 1u)] = unit;
    } else {
      acc += uacc;
      if (LOCAL) {
        // the unit's total (its own vertices are in every one of its cliques)
        // in hdr[8..11], free once the root pivot is known
        unsigned long long* ut = reinterpret_cast<unsigned long long*>(&hdr[8]);
        if (gt == 0) ut[0] = ut[1] = 0ull;
        gsync();
        if (pt.plane == 0 && uacc != 0) atomic_add_u128(ut, uacc);
        gsync();
        for (uint32_t i = gt; i < d; i += G) {
          const unsigned __int128 v = MODE == 0 ? (unsigned __int128)loc[i]
                                                : (((unsigned __int128)loc[2 * i + 1] << 64) | loc[2 * i]);
          if (v) atomic_add_u128(p.local + 2ull * S[i], v);
        }
        if (gt == 0) {
          const unsigned __int128 tot = ((unsigned __int128)ut[1] << 64) | ut[0];
          if (tot) {
            atomic_add_u128(p.local + 2ull * src, tot);
            if (p.edge_units) atomic_add_u128(p.local + 2ull * p.col[unit], tot);
          }
        }
      }
    }
    gsync();
  }
  flush();
  if (p.class_exit != nullptr) {  // this CTA is done: count it out of its class launch
    __syncthreads();
    if (threadIdx.x == 0) {
      __threadfence();
      atomicAdd(&p.class_exit[p.cls], 1u);
    }
  }
  if (p.stats && pt.plane == 0) {
    atomicAdd(p.stats + 0, st_nodes);
    atomicAdd(p.stats + 1, st_words);
  }
  // gather bytes are counted warp-uniformly, once per warp
  if (p.stats && lane == 0 && st_bytes) atomicAdd(p.stats + 2, st_bytes);
  if (p.stats != nullptr) {
    __syncthreads();
    if (threadIdx.x < 3) atomicAdd(p.stats + 3 + threadIdx.x, blk_cy[threadIdx.x]);
  }
}

}  // namespace

kc_status prepare_launch(kc_ctx* ctx, const LaunchPlan& lp, const CountParams& p0, cudaStream_t s,
                         PreparedLaunch* out) {
  if (lp.encoding == KC_ENC_LIST) return prepare_launch_list(ctx, lp, p0, s, out);
  CountParams p = p0;
  uint32_t P = lp.part;
  if (P == 0 || P > 32 || (P & (P - 1)) != 0)
    return fail(KC_ERR_INVALID_ARG, "partition size %u is not one of 1,2,4,8,16,32", P);
  const uint32_t G = lp.G, block = lp.block;
  const uint32_t dcap = std::max<uint32_t>(1, lp.dcap);
  uint32_t W = (dcap + 31) / 32;
  const uint32_t t_max = lp.edge ? (lp.k_max >= 2 ? lp.k_max - 2 : 0) : lp.k_max - 1;
  // Warp units in orientation mode run the lane-per-subtree traversal: one
  // lane is one partition, rows have 1, 2 or 4 words, no frames in shared memory.
  const bool lane = lp.mode == KC_MODE_ORIENT && G == 32 && dcap <= 128 && t_max <= (uint32_t)kLaneStack + 2 &&
                    !lp.local;
  if (lane) {
    P = 1;
    W = W <= 1 ? 1 : (W <= 2 ? 2 : 4);
  }
  // Pivoting walks each clique-tree node with a whole warp (partitions of one
  // warp would walk different nodes one after another); the partition size
  // bounds the number of lanes that score one pivot candidate.
  if (lp.mode != KC_MODE_ORIENT) {
    p.Q = lp.q;
    P = 32;
  }
  const uint32_t nparts = G / P;
  const uint32_t gpb = block / G;
  uint32_t depth, fw;
  if (lp.mode == KC_MODE_ORIENT) {
    depth = std::max<uint32_t>(1, t_max >= 2 ? t_max - 2 : 1);
    fw = lp.local ? W + 4 : W + 1;  // local counts: + the frame's vertex and its subtree total
  } else {
    // a pushed frame holds one more vertex than its parent (pivot branches
    // reuse the parent's slot), so k - hold0 + 1 levels always suffice
    const uint32_t hold0 = lp.edge ? 2u : 1u;
    depth = std::min<uint32_t>(dcap + 2, std::max<uint32_t>(2, lp.k_max + 2 - std::min(lp.k_max, hold0)));
    fw = 2 * W + (lp.local ? 14 : 4);  // local counts: held vertex, drop-list start, two u128 totals
  }
  auto al4 = [](size_t x) { return (x + 3) & ~(size_t)3; };
  const size_t hdr = 16, sS = al4(dcap), sR0 = al4(W);
  const bool pivot = lp.mode != KC_MODE_ORIENT;
  const size_t sB = (size_t)dcap * (pivot ? (W | 1u) : W);  // pivot rows use an odd stride
  // per walker: the frames, then (pivoting) the candidate list and, for local
  // counts, the drop list
  const size_t pstride = (size_t)depth * fw + (pivot ? al4(dcap) * (lp.local ? 2 : 1) : 0);
  const size_t sFr = lane ? 0 : al4((size_t)nparts * pstride);
  const size_t limit_words = ((size_t)ctx->max_smem_optin - kStaticSmemBytes) / 4;
  // hash of S for the bitmap build: 2*hT words, hT the power of two >= 2 dcap
  // (load at most 1/2)
  uint32_t hT = 0;
  if (dcap <= 2048) {
    hT = 64;
    while (hT < 2u * dcap) hT <<= 1;
  }
  // warp units keep their gather's row table (start and prefix of each row,
  // 2 dcap + 1 words) behind the hash or the membership map
  const size_t sRow = G == 32 ? al4(2 * (size_t)dcap + 1) : 0;
  bool bitmap_global = lp.force_global_bitmap;
  bool frames_global = false;
  // The hash is needed only while the bitmap is built and the frames only
  // after it, so in shared memory they share one region.
  // local counts: a u64 (orientation) or a (lo, hi) pair (pivoting) per vertex of S
  const size_t sLoc = lp.local ? al4((pivot ? 4 : 2) * (size_t)dcap) : 0;
  auto group_words = [&]() {
    return hdr + sS + sR0 + (bitmap_global ? 0 : al4(sB)) + sLoc +
           std::max<size_t>(frames_global ? 0 : sFr,
                            !hT ? 0 : (G == 32 ? gather_rows_at(hT) + sRow : 2 * (size_t)hT));
  };
  if ((size_t)gpb * group_words() > limit_words) frames_global = true;
  if ((size_t)gpb * group_words() > limit_words) bitmap_global = true;
  if ((size_t)gpb * group_words() > limit_words) hT = 0;
  if ((size_t)gpb * group_words() > limit_words)
    return fail(KC_ERR_INVALID_ARG, "unit size %u does not fit the shared-memory plan", dcap);
  p.dcap = dcap;
  p.W = W;
  p.P = P;
  p.G = G;
  p.depth = depth;
  p.fw = fw;
  p.pstride = (uint32_t)pstride;
  p.group_words = (uint32_t)group_words();
  p.off_R0 = (uint32_t)(hdr + sS);
  p.hash_T = hT;
  p.lane_dfs = lane ? 1u : 0u;
  p.off_B = (uint32_t)(hdr + sS + sR0);
  p.off_loc = (uint32_t)(p.off_B + (bitmap_global ? 0 : al4(sB)));
  p.off_fr = (uint32_t)(p.off_loc + sLoc);
  p.off_H = p.off_fr;
  p.bitmap_global = bitmap_global;
  p.frames_global = frames_global;
  p.gbuf_words = (bitmap_global ? al4(sB) : 0) + (frames_global ? sFr : 0);
  p.goff_fr = bitmap_global ? al4(sB) : 0;
  p.gbuf = nullptr;

  const size_t smem_bytes = (size_t)gpb * p.group_words * 4;
  auto kern = lp.mode == KC_MODE_ORIENT ? (lp.local ? k_count_bitmap<0, true> : k_count_bitmap<0, false>)
                                         : (lp.local ? k_count_bitmap<1, true> : k_count_bitmap<1, false>);
  // Several classes launch the same kernel with different shared-memory sizes;
  // the attribute is per function, so it is set to the device maximum.
  // (the kernel's static shared memory counts against the same per-block limit)
  cudaFuncAttributes fa;
  KC_CUDA(cudaFuncGetAttributes(&fa, kern));
  if (fa.sharedSizeBytes > kStaticSmemBytes)
    return fail(KC_ERR_INTERNAL, "counting kernel uses %zu bytes of static shared memory, planned for %zu",
                fa.sharedSizeBytes, kStaticSmemBytes);
  KC_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize,
                               ctx->max_smem_optin - (int)fa.sharedSizeBytes));
  int per_sm = 0;
  KC_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, block, smem_bytes));
  per_sm = std::max(1, per_sm);
  uint64_t grid = std::min<uint64_t>((uint64_t)ctx->sms * per_sm, ((uint64_t)p.n_units_max + gpb - 1) / gpb);
  grid = std::max<uint64_t>(1, grid);
  if (p.gbuf_words) {
    // keep the global scratch of the whole grid within 24 GiB
    const uint64_t per_block = (uint64_t)gpb * p.gbuf_words * 4;
    const uint64_t cap = std::max<uint64_t>(1, (24ull << 30) / std::max<uint64_t>(1, per_block));
    grid = std::min(grid, cap);
    KC_CUDA(dmalloc(&out->gbuf, grid * per_block, s));
    p.gbuf = out->gbuf;
  }
  out->p = p;
  out->grid = (uint32_t)grid;
  out->block = block;
  out->smem = smem_bytes;
  out->kernel = (void*)kern;
  out->list = false;
  return KC_OK;
}

kc_status enqueue_launch(const PreparedLaunch& pl, cudaStream_t s) {
  CountParams p = pl.p;
  size_t cap = pl.cap_edges;
  void* args_bitmap[] = {&p};
  void* args_list[] = {&p, &cap};
  KC_CUDA(cudaLaunchKernel(pl.kernel, dim3(pl.grid), dim3(pl.block), pl.list ? args_list : args_bitmap, pl.smem, s));
  return KC_OK;
}

void release_launch(PreparedLaunch& pl, cudaStream_t s) {
  if (pl.gbuf) dfree(pl.gbuf, s);
  pl.gbuf = nullptr;
}

}  // namespace kc
