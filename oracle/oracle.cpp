// oracle.cpp — CPU restatement of the KCGPU `-m kc` path. TEST INFRASTRUCTURE.
//
// This file is the checker, not the product: only tests/, the smoke check and
// bench.py's CPU-baseline leg load it. The engine never calls it.
//
// The reference has no CPU counting path (its CPU code is I/O and CSR only),
// so this is a restatement from the reference's rules and the mathematics:
//
//   CSR build        CSRCOO::from_edgelist (include/CSRCOO.cuh:37-80) drops
//                    self-loops; here the edge list is also symmetrised and
//                    deduplicated (the reference expects that of its input
//                    files, include/FIleReader.cuh:84-90).
//   degree orient    keep u->v iff deg u < deg v, or equal and u < v
//                    (include/main_support.cuh:54-87 called with node degrees
//                    at src/main.cu:181).
//   degen orient     keep u->v iff prio u < prio v, or equal and u < v
//                    (include/main_support.cuh:89-128), with prio the peel
//                    sub-round of kcore/kcore.cuh:442-584: levels L = 0,1,..;
//                    at each level the vertices of current degree L are peeled
//                    in sub-rounds, each sub-round's vertices get the running
//                    sub-round counter (kcore.cuh:192,564), and the batch that
//                    empties the graph keeps the initial value 2m
//                    (kcore.cuh:471-472, the break at :496-498).
//   node unit        k-cliques whose lowest vertex is u: (k-1)-cliques of the
//                    DAG induced on N+(u) (kclique/kckernels_orientation.cuh:319-475,
//                    start level 3).
//   edge unit        k-cliques whose lowest two vertices are u->v: (k-2)-cliques
//                    on N+(u) ∩ N+(v) (kclique/kckernels_orientation.cuh:479-650).
//   pivoting         the succinct clique tree of Pivoter (Jain & Seshadhri,
//                    WSDM 2020) as kclique/kckernels_pivoting.cuh:2-346 runs
//                    it: pivot = candidate with most neighbours among the
//                    candidates, ties to the smallest local index (:134-161,
//                    :250-308); branches = candidates not adjacent to the
//                    pivot, each excluding the earlier branches (:231-238);
//                    prune when held vertices exceed k (:214); a leaf adds
//                    C(drop, k - held) (:283-288), computed here with exact
//                    128-bit integers instead of the reference's double table.
//   truss support    sup(u,v) = |N(u) ∩ N(v)| (no counterpart in the reference).
//
// Counts are exact unsigned 128-bit integers (mod 2^128).
//
// Pinned against the reference itself: KCGPU ships no tests or fixtures, so
// its own -m kc program was rebuilt for sm_100a (oracle/build_ref.sh) and run
// on 8 graphs under every method (tests/golden/make_ref_golden.py ->
// tests/golden/ref_counts.json). This oracle equals every node-unit count and
// every edge-unit count outside four reference deviations, all undercounts
// (tests/ref_rules.py); one of them, edge-unit pivoting at k = 3, equals its
// own closed form. Also pinned by closed-form counts
// (tests/golden/closed_form.json), brute-force enumeration of small graphs,
// and agreement of its two algorithms (orientation listing and the Pivoter).
#include <algorithm>
#include <cstdint>
#include <cstring>
#include <vector>

#include <omp.h>

typedef unsigned __int128 u128;

struct or_graph {
  uint32_t n = 0;
  uint64_t m = 0;                      // undirected edges
  std::vector<uint32_t> rp, col;       // symmetric CSR, rows sorted, no dups
  int oriented = -1;
  std::vector<uint32_t> drp, dcol;     // DAG, original ids, rows sorted by id
  std::vector<uint32_t> prio, level;   // degeneracy peel results
};

namespace {

u128 binom_u128(uint32_t n, uint32_t r) {
  if (r > n) return 0;
  r = std::min(r, n - r);
  // Pascal's rule on one row: exact modulo 2^128 (no intermediate products).
  std::vector<u128> c((size_t)r + 1, 0);
  c[0] = 1;
  for (uint32_t i = 1; i <= n; ++i)
    for (uint32_t j = std::min(i, r); j >= 1; --j) c[j] += c[j - 1];
  return c[r];
}

struct Binom {
  // table[row][col] for row <= rows, col <= cols (Pascal recurrence, exact mod 2^128)
  uint32_t rows = 0, cols = 0;
  std::vector<u128> t;
  void build(uint32_t R, uint32_t C) {
    rows = R; cols = C;
    t.assign((size_t)(R + 1) * (C + 1), 0);
    for (uint32_t r = 0; r <= R; ++r) {
      t[(size_t)r * (C + 1)] = 1;
      for (uint32_t c = 1; c <= std::min(r, C); ++c)
        t[(size_t)r * (C + 1) + c] = t[(size_t)(r - 1) * (C + 1) + c - 1] +
                                     (c <= r - 1 ? t[(size_t)(r - 1) * (C + 1) + c] : 0);
    }
  }
  u128 get(uint32_t r, uint32_t c) const {
    if (c > r) return 0;
    if (r <= rows && c <= cols) return t[(size_t)r * (cols + 1) + c];
    return binom_u128(r, c);
  }
};

size_t intersect(const uint32_t* a, size_t na, const uint32_t* b, size_t nb, uint32_t* out) {
  size_t i = 0, j = 0, k = 0;
  while (i < na && j < nb) {
    if (a[i] < b[j]) ++i;
    else if (a[i] > b[j]) ++j;
    else { if (out) out[k] = a[i]; ++k; ++i; ++j; }
  }
  return k;
}

// ---- orientation counting (kClist-style listing on the DAG) --------------

struct OrientCounter {
  const or_graph& g;
  std::vector<std::vector<uint32_t>> buf;  // one candidate list per depth
  explicit OrientCounter(const or_graph& gr, uint32_t depth) : g(gr), buf(depth + 1) {}

  // t-cliques of the DAG induced on the sorted candidate list C.
  u128 rec(const uint32_t* C, size_t nc, uint32_t t, uint32_t depth) {
    if (t == 0) return 1;
    if (t == 1) return nc;
    u128 s = 0;
    auto& out = buf[depth];
    for (size_t i = 0; i < nc; ++i) {
      uint32_t v = C[i];
      const uint32_t* nv = g.dcol.data() + g.drp[v];
      size_t dv = g.drp[v + 1] - g.drp[v];
      out.resize(std::min(nc, dv));
      size_t c = intersect(C, nc, nv, dv, out.data());
      if (c >= t - 1) {
        std::vector<uint32_t> tmp(out.begin(), out.begin() + c);
        s += rec(tmp.data(), c, t - 1, depth + 1);
      }
    }
    return s;
  }
};

// Local counts: every k-clique adds 1 to each of its vertices
// (kclique/kclique_local.cuh, the reference's -m lkc). Listing from the lowest
// vertex u over the DAG, as the orientation counter; the path is kept so
// each found clique can credit its members.
struct LocalLister {
  const or_graph& g;
  std::vector<u128>& cnt;
  std::vector<uint32_t> path;
  LocalLister(const or_graph& gr, std::vector<u128>& c) : g(gr), cnt(c) {}

  void rec(const std::vector<uint32_t>& C, uint32_t t) {  // t more vertices from C
    if (t == 0) {
      for (uint32_t v : path) cnt[v] += 1;
      return;
    }
    if (C.size() < t) return;
    for (size_t i = 0; i < C.size(); ++i) {
      const uint32_t v = C[i];
      const uint32_t* nv = g.dcol.data() + g.drp[v];
      const size_t dv = g.drp[v + 1] - g.drp[v];
      std::vector<uint32_t> next(std::min(C.size(), dv));
      next.resize(intersect(C.data(), C.size(), nv, dv, next.data()));
      path.push_back(v);
      rec(next, t - 1);
      path.pop_back();
    }
  }
};

// ---- pivoting (succinct clique tree) on a local induced subgraph ---------

struct PivotCounter {
  uint32_t k;
  const Binom& B;
  uint32_t d = 0, W = 0;
  std::vector<uint64_t> adj;  // d rows of W 64-bit words, symmetric
  u128 total = 0;

  // closed: end nodes with r = k - hold <= 2 by the sum below instead of
  // expanding them (off by default; the plain expansion is the reference
  // behaviour, kclique/kckernels_pivoting.cuh:283-288).
  bool closed = false;

  PivotCounter(uint32_t kk, const Binom& b) : k(kk), B(b) {}

  // Builds the undirected induced subgraph on the sorted vertex list S using
  // the DAG out-lists (an edge of G[S] is an out-edge of its lower endpoint).
  void build(const or_graph& g, const std::vector<uint32_t>& S) {
    d = (uint32_t)S.size();
    W = (d + 63) / 64;
    adj.assign((size_t)d * W, 0);
    std::vector<uint32_t> tmp;
    for (uint32_t j = 0; j < d; ++j) {
      uint32_t v = S[j];
      const uint32_t* nv = g.dcol.data() + g.drp[v];
      size_t dv = g.drp[v + 1] - g.drp[v];
      // positions i with S[i] in N+(v)
      size_t a = 0, b = 0;
      while (a < d && b < dv) {
        if (S[a] < nv[b]) ++a;
        else if (S[a] > nv[b]) ++b;
        else {
          adj[(size_t)j * W + a / 64] |= 1ull << (a % 64);
          adj[(size_t)a * W + j / 64] |= 1ull << (j % 64);
          ++a; ++b;
        }
      }
    }
  }

  static uint32_t popc_and(const uint64_t* a, const uint64_t* b, uint32_t W) {
    uint32_t c = 0;
    for (uint32_t w = 0; w < W; ++w) c += (uint32_t)__builtin_popcountll(a[w] & b[w]);
    return c;
  }

  static uint32_t popc(const uint64_t* x, uint32_t W) {
    uint32_t c = 0;
    for (uint32_t w = 0; w < W; ++w) c += (uint32_t)__builtin_popcountll(x[w]);
    return c;
  }

  // scratch for depth l: candidate set, branch set, earlier branches, child (4 W words)
  std::vector<uint64_t> scratch;

  uint64_t* level(uint32_t l) {
    const size_t need = (size_t)(l + 2) * 4 * W;
    if (scratch.size() < need) scratch.resize(need * 2);
    return scratch.data() + (size_t)l * 4 * W;
  }

  // C is the candidate set stored in level(l)[0, W).
  void sct(uint32_t l, uint32_t hold, uint32_t drop) {
    if (hold > k) return;
    uint64_t* C = level(l);
    uint32_t nc = popc(C, W);
    if (nc == 0) {
      if (hold + drop >= k) total += B.get(drop, k - hold);
      return;
    }
    if (hold + drop + nc < k) return;  // not enough vertices left on this path
    if (closed && k - hold <= 2) {
      // Every clique Q of G[C] lies below this node once, and each can be
      // completed by any (r - |Q|) of the node's pivots (all adjacent to C and
      // to one another): the subtree adds sum_i kappa_i(G[C]) C(drop, r - i),
      // kappa_0 = 1, kappa_1 = |C|, kappa_2 = edges of G[C].
      const uint32_t r = k - hold;
      u128 add = B.get(drop, r);
      if (r >= 1) add += (u128)nc * B.get(drop, r - 1);
      if (r == 2) {
        uint64_t e2 = 0;
        for (uint32_t w = 0; w < W; ++w)
          for (uint64_t x = C[w]; x; x &= x - 1) {
            const uint32_t v = w * 64 + (uint32_t)__builtin_ctzll(x);
            e2 += popc_and(C, adj.data() + (size_t)v * W, W);
          }
        add += (u128)(e2 / 2);
      }
      total += add;
      return;
    }
    // pivot: most neighbours inside C, ties to the smallest index
    uint32_t best = UINT32_MAX, bestc = 0;
    for (uint32_t w = 0; w < W; ++w) {
      uint64_t x = C[w];
      while (x) {
        uint32_t v = w * 64 + (uint32_t)__builtin_ctzll(x);
        x &= x - 1;
        uint32_t c = 0;
        const uint64_t* av = adj.data() + (size_t)v * W;
        for (uint32_t q = 0; q < W; ++q) c += (uint32_t)__builtin_popcountll(C[q] & av[q]);
        if (best == UINT32_MAX || c > bestc) { best = v; bestc = c; }
      }
    }
    level(l + 1);  // grow the scratch before taking pointers into it
    C = level(l);
    uint64_t* branch = C + W;
    uint64_t* earlier = C + 2 * W;
    const uint64_t* ap = adj.data() + (size_t)best * W;
    for (uint32_t w = 0; w < W; ++w) {
      branch[w] = C[w] & ~ap[w];
      earlier[w] = 0;
    }
    for (uint32_t w = 0; w < W; ++w) {
      // the recursion below may grow (move) the scratch: index, never keep pointers
      uint64_t x = level(l)[W + w];
      while (x) {
        uint32_t v = w * 64 + (uint32_t)__builtin_ctzll(x);
        x &= x - 1;
        const uint64_t* av = adj.data() + (size_t)v * W;
        uint64_t* child = level(l + 1);
        C = level(l);
        earlier = C + 2 * W;
        for (uint32_t q = 0; q < W; ++q) child[q] = C[q] & av[q] & ~earlier[q];
        if (v == best) sct(l + 1, hold, drop + 1);
        else sct(l + 1, hold + 1, drop);
        C = level(l);  // the scratch may have grown during the recursion
        C[2 * W + v / 64] |= 1ull << (v % 64);
      }
    }
  }

  void run(uint32_t hold) {
    uint64_t* C = level(0);
    for (uint32_t w = 0; w < W; ++w) C[w] = 0;
    for (uint32_t i = 0; i < d; ++i) C[i / 64] |= 1ull << (i % 64);
    sct(0, hold, 0);
  }
};

// Vertices by decreasing out-degree (ties by id): the units a thread pool
// should take first, so the largest ones do not end up in the tail.
std::vector<uint32_t> heavy_first(const or_graph* g) {
  std::vector<uint32_t> order(g->n);
  for (uint32_t v = 0; v < g->n; ++v) order[v] = v;
  std::stable_sort(order.begin(), order.end(), [&](uint32_t a, uint32_t b) {
    return g->drp[a + 1] - g->drp[a] > g->drp[b + 1] - g->drp[b];
  });
  return order;
}

void peel(or_graph* g) {
  // Level-synchronous peeling with the reference's sub-round priorities.
  const uint32_t n = g->n;
  std::vector<int64_t> deg(n);
  for (uint32_t v = 0; v < n; ++v) deg[v] = g->rp[v + 1] - g->rp[v];
  g->prio.assign(n, (uint32_t)(2 * g->m));
  g->level.assign(n, 0);
  std::vector<char> removed(n, 0), infront(n, 0);
  uint64_t todo = n;
  uint32_t priority = 0;
  std::vector<uint32_t> front, next;
  for (int64_t L = 0; todo > 0; ++L) {
    front.clear();
    for (uint32_t v = 0; v < n; ++v)
      if (!removed[v] && deg[v] == L) front.push_back(v);
    while (!front.empty()) {
      todo -= front.size();
      for (uint32_t v : front) g->level[v] = (uint32_t)L;
      if (todo == 0) break;  // the final batch keeps priority 2m
      for (uint32_t v : front) { g->prio[v] = priority; infront[v] = 1; }
      next.clear();
      for (uint32_t v : front)
        for (uint32_t e = g->rp[v]; e < g->rp[v + 1]; ++e) {
          uint32_t u = g->col[e];
          if (removed[u] || infront[u]) continue;
          int64_t cur = deg[u]--;
          if (cur == L + 1) next.push_back(u);
        }
      for (uint32_t v : front) { removed[v] = 1; infront[v] = 0; }
      front.swap(next);
      ++priority;
    }
    if (todo == 0) {
      for (uint32_t v : front) removed[v] = 1;
    }
  }
}

int set_threads(int threads) {
  int nt = threads > 0 ? threads : omp_get_max_threads();
  return nt;
}

}  // namespace

extern "C" {

or_graph* or_from_edges(const uint32_t* src, const uint32_t* dst, uint64_t E, uint32_t n) {
  or_graph* g = new or_graph();
  uint32_t mx = 0;
  for (uint64_t i = 0; i < E; ++i) mx = std::max(mx, std::max(src[i], dst[i]));
  if (n == 0) n = E ? mx + 1 : 0;
  g->n = n;
  std::vector<uint64_t> keys;
  keys.reserve(2 * E);
  for (uint64_t i = 0; i < E; ++i) {
    uint32_t u = src[i], v = dst[i];
    if (u == v || u >= n || v >= n) continue;
    keys.push_back(((uint64_t)u << 32) | v);
    keys.push_back(((uint64_t)v << 32) | u);
  }
  std::sort(keys.begin(), keys.end());
  keys.erase(std::unique(keys.begin(), keys.end()), keys.end());
  g->rp.assign((size_t)n + 1, 0);
  g->col.resize(keys.size());
  for (size_t i = 0; i < keys.size(); ++i) {
    g->rp[(keys[i] >> 32) + 1]++;
    g->col[i] = (uint32_t)keys[i];
  }
  for (uint32_t v = 0; v < n; ++v) g->rp[v + 1] += g->rp[v];
  g->m = keys.size() / 2;
  return g;
}

or_graph* or_from_csr(const uint32_t* rp, const uint32_t* ci, uint32_t n) {
  std::vector<uint32_t> s, d;
  for (uint32_t v = 0; v < n; ++v)
    for (uint32_t e = rp[v]; e < rp[v + 1]; ++e) { s.push_back(v); d.push_back(ci[e]); }
  return or_from_edges(s.data(), d.data(), s.size(), n);
}

void or_free(or_graph* g) { delete g; }
uint32_t or_n(const or_graph* g) { return g->n; }
uint64_t or_m(const or_graph* g) { return g->m; }

void or_get_csr(const or_graph* g, uint32_t* rp, uint32_t* col) {
  std::copy(g->rp.begin(), g->rp.end(), rp);
  std::copy(g->col.begin(), g->col.end(), col);
}

uint32_t or_max_degree(const or_graph* g) {
  uint32_t mx = 0;
  for (uint32_t v = 0; v < g->n; ++v) mx = std::max(mx, g->rp[v + 1] - g->rp[v]);
  return mx;
}

// mode 0 = degree, 1 = degeneracy. Returns the largest out-degree.
uint32_t or_orient(or_graph* g, int mode) {
  const uint32_t n = g->n;
  std::vector<uint64_t> key(n);
  if (mode == 1) {
    peel(g);
    for (uint32_t v = 0; v < n; ++v) key[v] = ((uint64_t)g->prio[v] << 32) | v;
  } else {
    for (uint32_t v = 0; v < n; ++v) key[v] = ((uint64_t)(g->rp[v + 1] - g->rp[v]) << 32) | v;
  }
  g->drp.assign((size_t)n + 1, 0);
  g->dcol.clear();
  g->dcol.reserve(g->m);
  uint32_t mx = 0;
  for (uint32_t v = 0; v < n; ++v) {
    for (uint32_t e = g->rp[v]; e < g->rp[v + 1]; ++e) {
      uint32_t u = g->col[e];
      if (key[v] < key[u]) g->dcol.push_back(u);
    }
    g->drp[v + 1] = (uint32_t)g->dcol.size();
    mx = std::max(mx, g->drp[v + 1] - g->drp[v]);
  }
  g->oriented = mode;
  return mx;
}

void or_get_dag(const or_graph* g, uint32_t* rp, uint32_t* col) {
  std::copy(g->drp.begin(), g->drp.end(), rp);
  std::copy(g->dcol.begin(), g->dcol.end(), col);
}

void or_get_peel(const or_graph* g, uint32_t* prio, uint32_t* level) {
  if (prio) std::copy(g->prio.begin(), g->prio.end(), prio);
  if (level) std::copy(g->level.begin(), g->level.end(), level);
}

// Per-vertex core number (peel level) and the max core.
uint32_t or_kcore(or_graph* g, uint32_t* core) {
  if (g->level.size() != g->n) peel(g);
  uint32_t mx = 0;
  for (uint32_t v = 0; v < g->n; ++v) mx = std::max(mx, g->level[v]);
  if (core) std::copy(g->level.begin(), g->level.end(), core);
  return mx;
}

// mode 0 = orientation listing, 1 = pivoting; unit 0 = node, 1 = edge.
// flags bit 0 (pivoting): end clique-tree nodes with k - held <= 2 in closed
// form instead of expanding them (same count, far fewer nodes).
// Returns 0 on success, -1 if the graph is not oriented or k == 0.
int or_count_ex(const or_graph* g, uint32_t k, int mode, int unit, int threads, int flags, uint64_t* lo,
                uint64_t* hi) {
  if (g->oriented < 0 || k == 0) return -1;
  u128 total = 0;
  const uint32_t n = g->n;
  const int nt = set_threads(threads);
  if (k == 1) {
    total = n;
  } else if (k == 2) {
    total = g->m;
  } else if (unit == 0) {
    const uint32_t t = k - 1;
    uint32_t maxd = 0;
    for (uint32_t v = 0; v < n; ++v) maxd = std::max(maxd, g->drp[v + 1] - g->drp[v]);
    Binom B;
    B.build(maxd + 1, k);
    const std::vector<uint32_t> order = heavy_first(g);
#pragma omp parallel num_threads(nt)
    {
      u128 local = 0;
      OrientCounter oc(*g, k + 1);
      PivotCounter pc(k, B);
      pc.closed = (flags & 1) != 0;
#pragma omp for schedule(dynamic, 1)
      for (int64_t oi = 0; oi < (int64_t)n; ++oi) {
        const uint32_t v = order[oi];
        uint32_t d = g->drp[v + 1] - g->drp[v];
        if (d < t) continue;
        const uint32_t* nv = g->dcol.data() + g->drp[v];
        if (mode == 0) {
          local += oc.rec(nv, d, t, 0);
        } else {
          std::vector<uint32_t> S(nv, nv + d);
          pc.total = 0;
          pc.build(*g, S);
          pc.run(1);
          local += pc.total;
        }
      }
#pragma omp critical
      total += local;
    }
  } else {
    const uint32_t t = k - 2;
    uint32_t maxd = 0;
    for (uint32_t v = 0; v < n; ++v) maxd = std::max(maxd, g->drp[v + 1] - g->drp[v]);
    Binom B;
    B.build(maxd + 1, k);
    const std::vector<uint32_t> order = heavy_first(g);
#pragma omp parallel num_threads(nt)
    {
      u128 local = 0;
      OrientCounter oc(*g, k + 1);
      PivotCounter pc(k, B);
      pc.closed = (flags & 1) != 0;
      std::vector<uint32_t> tri;
#pragma omp for schedule(dynamic, 1)
      for (int64_t oi = 0; oi < (int64_t)n; ++oi) {
        const uint32_t u = order[oi];
        const uint32_t* nu = g->dcol.data() + g->drp[u];
        uint32_t du = g->drp[u + 1] - g->drp[u];
        for (uint32_t i = 0; i < du; ++i) {
          uint32_t v = nu[i];
          const uint32_t* nv = g->dcol.data() + g->drp[v];
          uint32_t dv = g->drp[v + 1] - g->drp[v];
          tri.resize(std::min(du, dv));
          size_t c = intersect(nu, du, nv, dv, tri.data());
          if (c < t) continue;
          if (mode == 0) {
            local += oc.rec(tri.data(), c, t, 0);
          } else {
            std::vector<uint32_t> S(tri.begin(), tri.begin() + c);
            pc.total = 0;
            pc.build(*g, S);
            pc.run(2);
            local += pc.total;
          }
        }
      }
#pragma omp critical
      total += local;
    }
  }
  *lo = (uint64_t)total;
  *hi = (uint64_t)(total >> 64);
  return 0;
}

int or_count(const or_graph* g, uint32_t k, int mode, int unit, int threads, uint64_t* lo, uint64_t* hi) {
  return or_count_ex(g, k, mode, unit, threads, 0, lo, hi);
}

// sup(u,v) = |N(u) ∩ N(v)| for every undirected edge u<v, in the row-major
// order of the upper triangle of the symmetric CSR.
void or_truss_support(const or_graph* g, uint32_t* sup) {
  const uint32_t n = g->n;
  std::vector<uint64_t> base((size_t)n + 1, 0);
  for (uint32_t u = 0; u < n; ++u) {
    uint64_t c = 0;
    for (uint32_t e = g->rp[u]; e < g->rp[u + 1]; ++e) c += g->col[e] > u;
    base[u + 1] = base[u] + c;
  }
#pragma omp parallel for schedule(dynamic, 64)
  for (int64_t u = 0; u < (int64_t)n; ++u) {
    uint64_t idx = base[u];
    const uint32_t* nu = g->col.data() + g->rp[u];
    uint32_t du = g->rp[u + 1] - g->rp[u];
    for (uint32_t i = 0; i < du; ++i) {
      uint32_t v = nu[i];
      if (v <= (uint32_t)u) continue;
      sup[idx++] = (uint32_t)intersect(nu, du, g->col.data() + g->rp[v], g->rp[v + 1] - g->rp[v], nullptr);
    }
  }
}

// Exact C(n, r) mod 2^128, for the tests of the engine's binomial table.
void or_binom(uint32_t n, uint32_t r, uint64_t* lo, uint64_t* hi) {
  u128 v = binom_u128(n, r);
  *lo = (uint64_t)v;
  *hi = (uint64_t)(v >> 64);
}

// Local counts (single-threaded; test sizes): out_lo/out_hi[v] for every vertex.
int or_count_local(const or_graph* g, uint32_t k, uint64_t* out_lo, uint64_t* out_hi) {
  if (g->oriented < 0 || k == 0) return -1;
  std::vector<u128> cnt(g->n, 0);
  LocalLister L(*g, cnt);
  for (uint32_t u = 0; u < g->n; ++u) {
    std::vector<uint32_t> C(g->dcol.begin() + g->drp[u], g->dcol.begin() + g->drp[u + 1]);
    L.path.assign(1, u);
    L.rec(C, k - 1);
  }
  for (uint32_t v = 0; v < g->n; ++v) {
    out_lo[v] = (uint64_t)cnt[v];
    out_hi[v] = (uint64_t)(cnt[v] >> 64);
  }
  return 0;
}

int or_max_threads(void) { return omp_get_max_threads(); }

}  // extern "C"
