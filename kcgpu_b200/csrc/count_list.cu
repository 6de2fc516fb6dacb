// List-encoded counting kernels (the reference's `-q ..n` encoding).
//
// Reference kernels these replace:
//   node / orientation / list  kckernel_node_block_warp_subgraph_count  kclique/kckernels_orientation.cuh:48-315
//   edge / orientation / list  kckernel_edge_block_warp_subgraph_count  kclique/kckernels.cuh:790-1072
//   node / pivot / list        kckernel_node_block_warp_pivot_count     kclique/kclique.cuh:448-867
//   edge / pivot / list        kckernel_edge_block_warp_pivot_count     kclique/kclique.cuh:869-1298
//
// The induced subgraph on S is a local CSR of sorted local indices (memory
// grows with the edges of G[S] instead of |S|^2 bits), and every candidate set
// of the traversal is a sorted list. Intersections locate each candidate in
// the other sorted list by binary search, P lanes at a time, and compact the
// hits in order with one ballot. Pivot-mode rows hold both directions: the
// in-neighbours (smaller indices) are filled by a transpose of the forward
// rows taken in row order, so every row stays sorted without a sort.
//
// Unlike the reference's list kernels (|S| <= 512 or 1024 through fixed shared
// arrays, kclique.cuh:505-516, kckernels_orientation.cuh:72-79) the lists live in
// per-group global scratch sized from the launch's largest unit.
//
// The pivot traversal shares the bitmap kernel's structure: nodes with
// r = k - held <= 2 are closed (1, |C| + drop, edges(G[C]) + drop |C| +
// C(drop, 2)), the pivot's own branch is taken last in its parent's frame
// (stack depth bounded by k), and a unit's tree is cut at depth 1-3 with the
// nodes at the cut handed to the group's partitions by ticket.
#include <algorithm>

#include "count_kernels.cuh"
#include "dev_common.cuh"

namespace kc {

namespace {

struct LPart {
  uint32_t P, plane, pmask, pbase;
};

__device__ __forceinline__ bool bsearch_u32(const uint32_t* a, uint32_t n, uint32_t x) {
  uint32_t lo = 0, hi = n;
  while (lo < hi) {
    const uint32_t mid = (lo + hi) >> 1;
    if (a[mid] < x) lo = mid + 1; else hi = mid;
  }
  return lo < n && a[lo] == x;
}

// out = elements x of a[0,na) with keep(x), in order; returns the count
// (identical in all lanes of the partition). out may be null (count only).
template <class F>
__device__ __forceinline__ uint32_t part_filter(const uint32_t* a, uint32_t na, uint32_t* out, const LPart& pt,
                                                F keep) {
  uint32_t cnt = 0;
  for (uint32_t b = 0; b < na; b += pt.P) {
    const uint32_t i = b + pt.plane;
    bool k = false;
    uint32_t x = 0;
    if (i < na) {
      x = a[i];
      k = keep(x);
    }
    const uint32_t bal = (__ballot_sync(pt.pmask, k) & pt.pmask) >> pt.pbase;
    if (k && out) out[cnt + __popc(bal & ((1u << pt.plane) - 1u))] = x;
    cnt += __popc(bal);
  }
  return cnt;
}

// Layout of one group's global scratch (words).
struct ListLayout {
  size_t S, off, cnt, col, fr, total;
};

__host__ __device__ inline ListLayout list_layout(uint32_t dcap, size_t cap_edges, uint32_t nparts, uint32_t depth,
                                                  uint32_t fw) {
  ListLayout L;
  L.S = 0;
  L.off = L.S + ((dcap + 3u) & ~3u);
  L.cnt = L.off + ((dcap + 4u) & ~3u);
  L.col = L.cnt + ((dcap + 3u) & ~3u);
  L.fr = L.col + ((cap_edges + 3) & ~(size_t)3);
  L.total = L.fr + (size_t)nparts * depth * fw;
  return L;
}

template <int MODE>
__global__ void __launch_bounds__(256) k_count_list(CountParams p, size_t cap_edges) {
  __shared__ uint32_t shdr[8][16];  // per group header (up to 8 groups per block)
  const uint32_t G = p.G;
  const uint32_t gpb = blockDim.x / G;
  const uint32_t gib = threadIdx.x / G;
  const uint32_t gt = threadIdx.x - gib * G;
  const uint32_t lane = lane_id();
  const uint32_t wig = gt >> 5, nwg = G >> 5;
  LPart pt;
  pt.P = p.P;
  pt.plane = gt % p.P;
  pt.pbase = (lane / p.P) * p.P;
  pt.pmask = p.P >= 32 ? 0xffffffffu : (((1u << p.P) - 1u) << pt.pbase);
  const uint32_t part = gt / p.P;
  const uint32_t nparts = G / p.P;
  const ListLayout LY = list_layout(p.dcap, cap_edges, nparts, p.depth, p.fw);
  uint32_t* gb = p.gbuf + (size_t)(blockIdx.x * gpb + gib) * p.gbuf_words;
  uint32_t* hdr = shdr[gib];
  uint32_t* S = gb + LY.S;
  uint32_t* Loff = gb + LY.off;
  uint32_t* Lcnt = gb + LY.cnt;
  uint32_t* Lcol = gb + LY.col;
  uint32_t* frames = gb + LY.fr + (size_t)part * p.depth * p.fw;
  const uint32_t D = p.dcap;

  // class bounds come from device memory: clamp them so no unit index can leave the queue
  const uint32_t ubeg = min(p.bounds[2 * p.cls], p.n_units_max);
  const uint32_t ucnt = min(p.bounds[2 * p.cls + 1], (p.n_units_max - ubeg + p.qstride - 1) / p.qstride);
  unsigned __int128 acc = 0;
  uint32_t acc_graph = 0xffffffffu;
  unsigned long long st_nodes = 0, st_words = 0, st_bytes = 0;
  auto gsync = [&]() {
    if (G == 32) __syncwarp(); else __syncthreads();
  };
  auto flush = [&]() {
    if (pt.plane == 0 && acc != 0 && acc_graph != 0xffffffffu) atomic_add_u128(p.out + 2ull * acc_graph, acc);
    acc = 0;
  };

  for (;;) {
    if (gt == 0) {
      uint32_t tk = atomicAdd(p.ticket, 1u);
      if (tk < ucnt && past_limit(p.time_limit_ns, p.t0)) {  // out of time: take no more units
        set_error(p.err, DEV_ERR_TIMEOUT);
        tk = 0xffffffffu;
      }
      hdr[0] = tk;
      hdr[1] = 0;
    }
    gsync();
    const uint32_t ui = hdr[0];
    if (ui >= ucnt) break;
    const uint32_t unit = p.queue[ubeg + (size_t)ui * p.qstride];
    uint32_t src, d;
    if (!p.edge_units) {
      src = unit;
      const uint32_t b = p.rp[src];
      d = p.rp[src + 1] - b;
      if (d <= D)
        for (uint32_t j = gt; j < d; j += G) S[j] = p.col[b + j];
    } else {
      src = p.erow[unit];
      const uint32_t v = p.col[unit];
      if (wig == 0) {
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
          if (i < la) { x = A[i]; found = bsearch_u32(L, ll, x); }
          const uint32_t bal = __ballot_sync(0xffffffffu, found);
          if (found && cnt + __popc(bal & lanemask_lt()) < D) S[cnt + __popc(bal & lanemask_lt())] = x;
          cnt += __popc(bal);
        }
        if (lane == 0) hdr[2] = cnt;
      }
      gsync();
      d = hdr[2];
    }
    const uint32_t gph = p.vgraph ? p.vgraph[src] : 0u;
    const uint32_t k = p.gk ? p.gk[gph] : p.k0;
    __threadfence_block();
    gsync();
    if (gph != acc_graph) { flush(); acc_graph = gph; }
    if (d > D) {
      if (gt == 0) set_error(p.err, DEV_ERR_CAPACITY);
      gsync();
      continue;
    }
    if (MODE == 0) {
      const uint32_t t = p.edge_units ? k - 2u : k - 1u;
      if (t <= 1u || d < t) {
        if (part == 0 && d >= t) acc += (t == 0u) ? 1u : d;
        gsync();
        continue;
      }
    } else {
      const uint32_t hold0 = p.edge_units ? 2u : 1u;
      if (d == 0u || hold0 + d < k) {
        if (part == 0 && d == 0u && k == hold0) acc += 1u;
        gsync();
        continue;
      }
    }

    // ---- local CSR of G[S] ---------------------------------------------------
    for (uint32_t j = gt; j < d; j += G) Lcnt[j] = 0;
    gsync();
    const uint32_t last = S[d - 1];
    // pass 1: forward counts (and in-counts for the symmetric rows)
    for (uint32_t j = wig; j < d; j += nwg) {
      const uint32_t x0 = S[j];
      const uint32_t b = p.rp[x0], e = p.rp[x0 + 1];
      uint32_t c = 0;
      uint32_t i0 = b;
      for (; i0 < e; i0 += 32) {
        const uint32_t i = i0 + lane;
        const uint32_t x = i < e ? __ldg(p.col + i) : 0xffffffffu;
        const bool inr = x <= last;
        if (!__any_sync(0xffffffffu, inr)) break;
        bool hit = false;
        uint32_t pos = 0;
        if (inr) {
          pos = j + 1 + lower_bound_u32(S + j + 1, d - j - 1, x);
          hit = pos < d && S[pos] == x;
        }
        c += __popc(__ballot_sync(0xffffffffu, hit));
        if (MODE == 1 && hit) atomicAdd(&Lcnt[pos], 1u);
      }
      st_bytes += 4ull * (min(i0 + 32u, e) - b);
      if (lane == 0) atomicAdd(&Lcnt[j], c);
    }
    gsync();
    // offsets (one warp scans), and the forward counts again for pass 2
    if (wig == 0) {
      uint32_t run = 0;
      for (uint32_t b = 0; b < d; b += 32) {
        const uint32_t j = b + lane;
        const uint32_t v = j < d ? Lcnt[j] : 0u;
        uint32_t inc = v;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
          const uint32_t t = __shfl_up_sync(0xffffffffu, inc, o);
          if (lane >= (uint32_t)o) inc += t;
        }
        if (j < d) Loff[j] = run + inc - v;
        run += __shfl_sync(0xffffffffu, inc, 31);
      }
      if (lane == 0) Loff[d] = run;
    }
    gsync();
    const uint32_t E_S = Loff[d];
    if (E_S > cap_edges) {
      if (gt == 0) set_error(p.err, DEV_ERR_CAPACITY);
      gsync();
      continue;
    }
    for (uint32_t j = gt; j < d; j += G) Lcnt[j] = 0;  // becomes the in-neighbour cursor
    gsync();
    if (MODE == 1) {
      // in-neighbours first (smaller indices), taken in row order by one warp
      // so each row's prefix stays sorted; it needs the forward rows, which
      // are re-derived here from the stream.
      if (wig == 0) {
        for (uint32_t i = 0; i < d; ++i) {
          const uint32_t x0 = S[i];
          const uint32_t b = p.rp[x0], e = p.rp[x0 + 1];
          for (uint32_t i0 = b; i0 < e; i0 += 32) {
            const uint32_t q = i0 + lane;
            const uint32_t x = q < e ? __ldg(p.col + q) : 0xffffffffu;
            const bool inr = x <= last;
            if (!__any_sync(0xffffffffu, inr)) break;
            if (inr) {
              const uint32_t pos = i + 1 + lower_bound_u32(S + i + 1, d - i - 1, x);
              if (pos < d && S[pos] == x) Lcol[Loff[pos] + Lcnt[pos]++] = i;
            }
          }
          __syncwarp();
        }
      }
      gsync();
    }
    // forward entries (larger indices) after the in-neighbours
    for (uint32_t j = wig; j < d; j += nwg) {
      const uint32_t x0 = S[j];
      const uint32_t b = p.rp[x0], e = p.rp[x0 + 1];
      uint32_t w = Loff[j] + (MODE == 1 ? Lcnt[j] : 0u);
      for (uint32_t i0 = b; i0 < e; i0 += 32) {
        const uint32_t i = i0 + lane;
        const uint32_t x = i < e ? __ldg(p.col + i) : 0xffffffffu;
        const bool inr = x <= last;
        if (!__any_sync(0xffffffffu, inr)) break;
        bool hit = false;
        uint32_t pos = 0;
        if (inr) {
          pos = j + 1 + lower_bound_u32(S + j + 1, d - j - 1, x);
          hit = pos < d && S[pos] == x;
        }
        const uint32_t bal = __ballot_sync(0xffffffffu, hit);
        if (hit) Lcol[w + __popc(bal & lanemask_lt())] = pos;
        w += __popc(bal);
      }
    }
    __threadfence_block();
    gsync();

    auto row = [&](uint32_t v) { return Lcol + Loff[v]; };
    auto rowlen = [&](uint32_t v) { return Loff[v + 1] - Loff[v]; };

    if (MODE == 0) {
      // frame: list [0, D), [D] length, [D+1] cursor
      const uint32_t t = p.edge_units ? k - 2u : k - 1u;
      for (;;) {
        uint32_t j = 0;
        if (pt.plane == 0) j = atomicAdd(&hdr[1], 1u);
        j = __shfl_sync(pt.pmask, j, pt.pbase);
        if (j >= d) break;
        const uint32_t lj = rowlen(j);
        st_nodes++;
        if (t == 2u) { acc += lj; continue; }
        if (lj < t - 1u) continue;
        uint32_t* F0 = frames;
        for (uint32_t i = pt.plane; i < lj; i += pt.P) F0[i] = row(j)[i];
        if (pt.plane == 0) { F0[D] = lj; F0[D + 1] = 0; }
        __syncwarp(pt.pmask);
        int lv = 0;
        while (lv >= 0) {
          uint32_t* F = frames + (size_t)lv * p.fw;
          const uint32_t len = F[D], cur = F[D + 1];
          if (cur >= len) { --lv; continue; }
          const uint32_t v = F[cur];
          __syncwarp(pt.pmask);
          if (pt.plane == 0) F[D + 1] = cur + 1;
          const uint32_t rem = t - (uint32_t)(lv + 2);
          const uint32_t* Lv = row(v);
          const uint32_t lvn = rowlen(v);
          const bool store = rem > 1u && (uint32_t)(lv + 1) < p.depth;
          uint32_t* Fc = F + p.fw;
          const uint32_t c = part_filter(F + cur + 1, len - cur - 1, store ? Fc : nullptr, pt,
                                         [&](uint32_t x) { return bsearch_u32(Lv, lvn, x); });
          st_nodes++;
          st_words += len - cur - 1;
          if (rem == 1u) {
            acc += c;
          } else if (c >= rem) {
            if (!store) {
              if (pt.plane == 0) set_error(p.err, DEV_ERR_STACK);
            } else {
              __syncwarp(pt.pmask);
              if (pt.plane == 0) { Fc[D] = c; Fc[D + 1] = 0; }
              __syncwarp(pt.pmask);
              ++lv;
            }
          }
          __syncwarp(pt.pmask);
        }
      }
    } else {
      // frame: C [0,D), R [D,2D), meta at 2D: clen, rlen, rcur, hold, drop, pivot
      const uint32_t hold0 = p.edge_units ? 2u : 1u;
      // root pivot: largest degree in G[S], ties to the smallest index
      uint32_t key = 0;
      for (uint32_t v = gt; v < d; v += G) key = max(key, (rowlen(v) << 16) | (0xffffu - v));
      key = __reduce_max_sync(0xffffffffu, key);
      if (lane == 0) hdr[8 + wig] = key;
      gsync();
      if (gt == 0) {
        uint32_t m = 0;
        for (uint32_t q = 0; q < nwg; ++q) m = max(m, hdr[8 + q]);
        hdr[3] = 0xffffu - (m & 0xffffu);
      }
      gsync();
      const uint32_t p0 = hdr[3];
      const uint32_t* Lp0 = row(p0);
      const uint32_t lp0 = rowlen(p0);

      auto binom = [&](uint32_t nn, uint32_t r) -> unsigned __int128 {
        if (r > nn) return 0;
        const unsigned long long* e = p.binom + 2ull * ((size_t)nn * (p.binom_cols + 1u) + r);
        return ((unsigned __int128)e[1] << 64) | e[0];
      };
      // A node with `hold` held vertices, `drop` pivots and candidates F[0, nc)
      // contributes sum_j C(drop, j) * cliques(G[F], r - j), r = k - hold; for
      // r <= 2 the sum is closed (1, |F| and the edges of G[F]).
      auto enter = [&](uint32_t* F, uint32_t nc, uint32_t hold, uint32_t drop, bool own) -> bool {
        const uint32_t r = k - hold;  // callers keep hold <= k
        if (nc == 0u) {
          if (own) acc += binom(drop, r);
          return false;
        }
        if (hold + drop + nc < k) return false;
        if (r <= 1u) {
          if (own) acc += (r == 0u) ? (unsigned __int128)1u : (unsigned __int128)(nc + drop);
          return false;
        }
        // lanes take candidates in turn and score each by |F ∩ N(u)|
        uint32_t best = 0;
        unsigned long long esum = 0;
        for (uint32_t a = pt.plane; a < nc; a += pt.P) {
          const uint32_t u = F[a];
          const uint32_t* Lu = row(u);
          const uint32_t lu = rowlen(u);
          uint32_t c = 0;
          for (uint32_t q = 0; q < nc; ++q) c += bsearch_u32(Lu, lu, F[q]) ? 1u : 0u;
          esum += c;
          best = max(best, (c << 16) | (0xffffu - u));
        }
        for (uint32_t o = 1; o < pt.P; o <<= 1) esum += __shfl_xor_sync(pt.pmask, esum, o);
        if (r == 2u) {
          if (own) acc += (unsigned __int128)(esum / 2u) + (unsigned __int128)drop * nc + binom(drop, 2u);
          if (own) st_words += (unsigned long long)nc * nc;
          return false;
        }
        best = __reduce_max_sync(pt.pmask, best);
        if (own) st_words += (unsigned long long)nc * nc;
        const uint32_t piv = 0xffffu - (best & 0xffffu);
        const uint32_t* Lq = row(piv);
        const uint32_t lq = rowlen(piv);
        // branches: candidates outside N(piv) less the pivot, whose branch is
        // taken last in this frame's own slot
        const uint32_t rl = part_filter(F, nc, F + D, pt, [&](uint32_t x) { return x != piv && !bsearch_u32(Lq, lq, x); });
        __syncwarp(pt.pmask);
        if (pt.plane == 0) {
          F[2 * D] = nc; F[2 * D + 1] = rl; F[2 * D + 2] = 0;
          F[2 * D + 3] = hold; F[2 * D + 4] = drop; F[2 * D + 5] = piv;
        }
        __syncwarp(pt.pmask);
        return true;
      };

      // Work split inside the unit, as in the bitmap kernel: the tree is cut
      // at depth L, nodes at depth L go out by ticket (hdr[1]), every
      // partition walks the levels above the cut, partition 0 alone counts them.
      const uint32_t nparts = G / pt.P;
      uint32_t nr0 = 0;
      for (uint32_t v = pt.plane; v < d; v += pt.P) nr0 += (v == p0 || !bsearch_u32(Lp0, lp0, v)) ? 1u : 0u;
      nr0 = __reduce_add_sync(pt.pmask, nr0);
      const uint32_t L = (nparts == 1u || nr0 >= 4u * nparts) ? 1u : (nr0 <= 2u ? 3u : 2u);
      const bool top_owner = part == 0u;
      auto ticket = [&]() -> uint32_t {
        uint32_t t = 0;
        if (pt.plane == 0) t = atomicAdd(&hdr[1], 1u);
        return __shfl_sync(pt.pmask, t, pt.pbase);
      };
      uint32_t seen = 0, mine = ticket();
      auto claim = [&]() -> bool {
        const bool take = seen == mine;
        ++seen;
        if (take) mine = ticket();
        return take;
      };

      for (uint32_t v = 0; v < d; ++v) {
        // root branches: vertices not adjacent to the root pivot (p0 included)
        if (v != p0 && bsearch_u32(Lp0, lp0, v)) continue;
        if (L == 1u && !claim()) continue;
        const bool own1 = L == 1u || top_owner;
        const uint32_t hold = hold0 + (v != p0 ? 1u : 0u), drop = (v == p0) ? 1u : 0u;
        if (own1) st_nodes++;
        if (hold > k) continue;
        // child: N(v) minus the earlier root branches (indices < v not adjacent to p0)
        const uint32_t* Lv = row(v);
        const uint32_t lvn = rowlen(v);
        uint32_t* F0 = frames;
        const uint32_t nc = part_filter(Lv, lvn, F0, pt, [&](uint32_t x) {
          return !(x < v && (x == p0 || !bsearch_u32(Lp0, lp0, x)));
        });
        __syncwarp(pt.pmask);
        if (!enter(F0, nc, hold, drop, own1)) continue;
        int lv = 0;
        while (lv >= 0) {
          uint32_t* F = frames + (size_t)lv * p.fw;
          const uint32_t clen = F[2 * D], rlen = F[2 * D + 1], rcur = F[2 * D + 2];
          const uint32_t fh = F[2 * D + 3], fd = F[2 * D + 4], fp = F[2 * D + 5];
          __syncwarp(pt.pmask);
          if (rcur >= rlen) {
            // every other branch is done: the pivot's branch, C ∩ N(piv)
            // (disjoint from the branches), replaces the frame in place
            const bool own = (uint32_t)lv + 1u >= L || top_owner;
            if (own) st_nodes++;
            const uint32_t* Lq = row(fp);
            const uint32_t lq = rowlen(fp);
            const uint32_t nc = part_filter(F, clen, F, pt, [&](uint32_t x) { return bsearch_u32(Lq, lq, x); });
            __syncwarp(pt.pmask);
            if (!enter(F, nc, fh, fd + 1u, own)) --lv;
            continue;
          }
          const uint32_t u = F[D + rcur];
          __syncwarp(pt.pmask);
          if (pt.plane == 0) F[2 * D + 2] = rcur + 1;
          const uint32_t h2 = fh + 1u;  // u is not the pivot
          bool descend = h2 <= k;
          if (descend && (uint32_t)(lv + 1) >= p.depth) {
            if (pt.plane == 0) set_error(p.err, DEV_ERR_STACK);
            descend = false;
          }
          bool own = (uint32_t)lv + 2u > L || top_owner;
          if (descend && (uint32_t)lv + 2u == L) own = descend = claim();
          if (own) st_nodes++;
          if (descend) {
            // child = C ∩ N(u) minus the earlier branches R[0, rcur)
            const uint32_t* Lu = row(u);
            const uint32_t lu = rowlen(u);
            const uint32_t* Rl = F + D;
            uint32_t* Fc = F + p.fw;
            const uint32_t nc = part_filter(F, clen, Fc, pt, [&](uint32_t x) {
              return bsearch_u32(Lu, lu, x) && !(x < u && bsearch_u32(Rl, rcur, x));
            });
            __syncwarp(pt.pmask);
            if (enter(Fc, nc, h2, fd, own)) ++lv;
          }
          __syncwarp(pt.pmask);
        }
      }
    }
    gsync();
  }
  flush();
  if (p.stats && pt.plane == 0) {
    atomicAdd(p.stats + 0, st_nodes);
    atomicAdd(p.stats + 1, st_words);
    if (part == 0) atomicAdd(p.stats + 2, st_bytes);
  }
}

}  // namespace

kc_status prepare_launch_list(kc_ctx* ctx, const LaunchPlan& lp, const CountParams& p0, cudaStream_t s,
                              PreparedLaunch* out) {
  CountParams p = p0;
  const uint32_t P = lp.part;
  if (P == 0 || P > 32 || (P & (P - 1)) != 0)
    return fail(KC_ERR_INVALID_ARG, "partition size %u is not one of 1,2,4,8,16,32", P);
  const uint32_t G = lp.G, block = lp.block;
  if (block / G > 8) return fail(KC_ERR_INTERNAL, "list kernel supports at most 8 groups per block");
  const uint32_t D = std::max<uint32_t>(1, lp.dcap);
  const uint32_t nparts = G / P;
  uint32_t depth, fw;
  if (lp.mode == KC_MODE_ORIENT) {
    const uint32_t t = lp.edge ? (lp.k_max >= 2 ? lp.k_max - 2 : 0) : lp.k_max - 1;
    depth = std::max<uint32_t>(1, t >= 2 ? t - 2 : 1);
    fw = D + 2;
  } else {
    // pivot branches reuse their parent's slot: k - hold0 + 1 levels suffice
    const uint32_t hold0 = lp.edge ? 2u : 1u;
    depth = std::min<uint32_t>(D + 2, std::max<uint32_t>(2, lp.k_max + 2 - std::min(lp.k_max, hold0)));
    fw = 2 * D + 6;
  }
  const size_t full_edges = lp.mode == KC_MODE_ORIENT ? (size_t)D * (D - 1) / 2 : (size_t)D * (D - 1);
  const size_t cap_edges = std::max<size_t>(1, std::min<size_t>(full_edges, (size_t)1 << 26));
  const ListLayout LY = list_layout(D, cap_edges, nparts, depth, fw);
  p.dcap = D;
  p.W = (D + 31) / 32;
  p.P = P;
  p.G = G;
  p.depth = depth;
  p.fw = fw;
  p.gbuf_words = LY.total;
  const uint32_t gpb = block / G;
  auto kern = lp.mode == KC_MODE_ORIENT ? k_count_list<0> : k_count_list<1>;
  int per_sm = 0;
  KC_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, block, 0));
  per_sm = std::max(1, per_sm);
  uint64_t grid = std::min<uint64_t>((uint64_t)ctx->sms * per_sm, ((uint64_t)p.n_units_max + gpb - 1) / gpb);
  const uint64_t per_block = (uint64_t)gpb * LY.total * 4;
  grid = std::max<uint64_t>(1, std::min<uint64_t>(grid, std::max<uint64_t>(1, (16ull << 30) / per_block)));
  KC_CUDA(dmalloc(&out->gbuf, grid * per_block, s));
  p.gbuf = out->gbuf;
  out->p = p;
  out->grid = (uint32_t)grid;
  out->block = block;
  out->smem = 0;
  out->kernel = (void*)kern;
  out->list = true;
  out->cap_edges = cap_edges;
  return KC_OK;
}

}  // namespace kc
