// Seeded synthetic graph generators (host side).
//
// The reference ships no graphs and no generator (its inputs are SNAP files
// read by include/FIleReader.cuh). These generators produce raw edge lists of
// the shapes the benchmark configurations name; the engine then symmetrises,
// deduplicates and drops self-loops on the GPU, exactly as it does for any
// caller-supplied edge list.
//
// Randomness: splitmix64 seeds a xoshiro256** stream per independent chunk, so
// every generator is deterministic for a given seed regardless of the number of
// host threads.
#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstdint>
#include <cstdlib>
#include <cstring>
#include <new>
#include <thread>
#include <unordered_map>
#include <vector>

#include <cuda_runtime.h>

#include "../../include/kc.h"
#include "edgelist.h"
#include "host_common.h"

namespace kc {

struct Rng {
  uint64_t s[4];
  static uint64_t splitmix(uint64_t& x) {
    uint64_t z = (x += 0x9e3779b97f4a7c15ULL);
    z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ULL;
    z = (z ^ (z >> 27)) * 0x94d049bb133111ebULL;
    return z ^ (z >> 31);
  }
  explicit Rng(uint64_t seed) {
    uint64_t x = seed;
    for (int i = 0; i < 4; ++i) s[i] = splitmix(x);
  }
  static uint64_t rotl(uint64_t x, int k) { return (x << k) | (x >> (64 - k)); }
  uint64_t next() {
    const uint64_t r = rotl(s[1] * 5, 7) * 9;
    const uint64_t t = s[1] << 17;
    s[2] ^= s[0]; s[3] ^= s[1]; s[1] ^= s[2]; s[0] ^= s[3];
    s[2] ^= t; s[3] = rotl(s[3], 45);
    return r;
  }
  // Uniform in [0,1) with 53 random bits.
  double uniform() { return (double)(next() >> 11) * (1.0 / 9007199254740992.0); }
  // Uniform in (0,1].
  double uniform_pos() { return 1.0 - uniform(); }
  uint64_t below(uint64_t n) { return n ? next() % n : 0; }
};

static uint64_t mix_seed(uint64_t seed, uint64_t stream) {
  uint64_t x = seed ^ (stream * 0xd1342543de82ef95ULL + 0x2545f4914f6cdd1dULL);
  return Rng::splitmix(x);
}

}  // namespace kc

namespace {

using kc::Rng;
using kc::mix_seed;

int host_threads() {
  unsigned t = std::thread::hardware_concurrency();
  return t ? (int)std::min(t, 64u) : 1;
}

// Runs fn(chunk, out_src, out_dst) for chunks [0,nchunks) on host threads and
// appends the per-chunk outputs in chunk order (deterministic).
template <class F>
void parallel_chunks(uint64_t nchunks, std::vector<uint32_t>& S, std::vector<uint32_t>& D, F fn) {
  std::vector<std::vector<uint32_t>> cs(nchunks), cd(nchunks);
  int nt = (int)std::min<uint64_t>((uint64_t)host_threads(), std::max<uint64_t>(1, nchunks));
  std::vector<std::thread> th;
  std::atomic<uint64_t> next{0};
  for (int t = 0; t < nt; ++t)
    th.emplace_back([&]() {
      for (;;) {
        uint64_t c = next.fetch_add(1);
        if (c >= nchunks) break;
        fn(c, cs[c], cd[c]);
      }
    });
  for (auto& x : th) x.join();
  uint64_t tot = 0;
  for (auto& v : cs) tot += v.size();
  S.reserve(S.size() + tot);
  D.reserve(D.size() + tot);
  for (uint64_t c = 0; c < nchunks; ++c) {
    S.insert(S.end(), cs[c].begin(), cs[c].end());
    D.insert(D.end(), cd[c].begin(), cd[c].end());
  }
}

// G(n,p) on vertices [off, off+n): each pair i<j present with probability p,
// by geometric skipping over the pairs in row order (Batagelj-Brandes 2005).
void er_into(uint32_t n, double p, Rng& rng, uint32_t off, std::vector<uint32_t>& S,
             std::vector<uint32_t>& D) {
  if (n < 2 || p <= 0) return;
  if (p >= 1) {
    for (uint32_t v = 1; v < n; ++v)
      for (uint32_t w = 0; w < v; ++w) { S.push_back(off + v); D.push_back(off + w); }
    return;
  }
  const double lp = std::log(1.0 - p);
  int64_t v = 1, w = -1;
  while (v < (int64_t)n) {
    double r = rng.uniform_pos();
    w = w + 1 + (int64_t)std::floor(std::log(r) / lp);
    while (w >= v && v < (int64_t)n) { w -= v; ++v; }
    if (v < (int64_t)n) { S.push_back(off + (uint32_t)v); D.push_back(off + (uint32_t)w); }
  }
}

// Bipartite G(a,b,p) between [oa,oa+a) and [ob,ob+b) by geometric skipping.
void bip_into(uint32_t a, uint32_t b, double p, Rng& rng, uint32_t oa, uint32_t ob,
              std::vector<uint32_t>& S, std::vector<uint32_t>& D) {
  if (!a || !b || p <= 0) return;
  const uint64_t total = (uint64_t)a * b;
  if (p >= 1) {
    for (uint64_t i = 0; i < total; ++i) { S.push_back(oa + (uint32_t)(i / b)); D.push_back(ob + (uint32_t)(i % b)); }
    return;
  }
  const double lp = std::log(1.0 - p);
  int64_t idx = -1;
  for (;;) {
    double r = rng.uniform_pos();
    idx += 1 + (int64_t)std::floor(std::log(r) / lp);
    if (idx < 0 || (uint64_t)idx >= total) break;
    S.push_back(oa + (uint32_t)((uint64_t)idx / b));
    D.push_back(ob + (uint32_t)((uint64_t)idx % b));
  }
}

void clique_into(const std::vector<uint32_t>& vs, std::vector<uint32_t>& S, std::vector<uint32_t>& D) {
  for (size_t i = 0; i < vs.size(); ++i)
    for (size_t j = i + 1; j < vs.size(); ++j) { S.push_back(vs[i]); D.push_back(vs[j]); }
}

// Up to `count` disjoint random vertex sets of [0,n) with sizes uniform in
// [smin,smax], drawn by a sparse partial Fisher-Yates shuffle.
std::vector<std::vector<uint32_t>> disjoint_sets(uint32_t n, uint32_t count, uint32_t smin,
                                                 uint32_t smax, Rng& rng) {
  std::vector<uint32_t> sizes;
  uint64_t total = 0;
  for (uint32_t i = 0; i < count; ++i) {
    uint32_t s = smin + (uint32_t)rng.below((uint64_t)smax - smin + 1);
    if (total + s > n) break;
    sizes.push_back(s);
    total += s;
  }
  std::unordered_map<uint32_t, uint32_t> moved;  // sparse view of a permuted [0,n)
  auto at = [&](uint32_t i) { auto it = moved.find(i); return it == moved.end() ? i : it->second; };
  std::vector<uint32_t> picked(total);
  for (uint64_t i = 0; i < total; ++i) {
    uint32_t j = (uint32_t)(i + rng.below(n - i));
    uint32_t vi = at((uint32_t)i), vj = at(j);
    moved[(uint32_t)i] = vj;
    moved[j] = vi;
    picked[i] = vj;
  }
  std::vector<std::vector<uint32_t>> out;
  uint64_t pos = 0;
  for (uint32_t s : sizes) {
    out.emplace_back(picked.begin() + pos, picked.begin() + pos + s);
    pos += s;
  }
  return out;
}

kc_status make(kc_edgelist** out, kc_edgelist** e) {
  if (!out) return kc::fail(KC_ERR_INVALID_ARG, "output pointer is NULL");
  *e = new (std::nothrow) kc_edgelist();
  if (!*e) return kc::fail(KC_ERR_OOM, "host allocation failed");
  return KC_OK;
}

kc_status done(kc_edgelist* e, int pinned, kc_edgelist** out) {
  kc_status st = kc::edgelist_finish(e, pinned);
  if (st != KC_OK) { delete e; return st; }
  *out = e;
  return KC_OK;
}

}  // namespace

extern "C" {

kc_status kc_edgelist_data(const kc_edgelist* e, const uint32_t** src, const uint32_t** dst,
                           uint64_t* n_edges, uint32_t* n_nodes) {
  if (!e) return kc::fail(KC_ERR_INVALID_ARG, "edge list is NULL");
  if (src) *src = e->src();
  if (dst) *dst = e->dst();
  if (n_edges) *n_edges = e->n_edges;
  if (n_nodes) *n_nodes = e->n_nodes;
  return KC_OK;
}

kc_status kc_edgelist_destroy(kc_edgelist* e) {
  delete e;
  return KC_OK;
}

kc_status kc_gen_er(uint32_t n, double p, uint64_t seed, int pinned, kc_edgelist** out) {
  kc_edgelist* e;
  if (kc_status st = make(out, &e)) return st;
  if (!(p >= 0 && p <= 1)) { delete e; return kc::fail(KC_ERR_INVALID_ARG, "p must be in [0,1]"); }
  Rng rng(mix_seed(seed, 0));
  er_into(n, p, rng, 0, e->vsrc, e->vdst);
  e->n_nodes = n;
  return done(e, pinned, out);
}

// R-MAT (Chakrabarti et al. 2004): each of edge_factor * 2^scale samples picks
// one quadrant per bit level with probabilities (a, b, c, 1-a-b-c); no noise,
// no id permutation.
kc_status kc_gen_rmat(uint32_t scale, double edge_factor, double a, double b, double c,
                      uint64_t seed, int pinned, kc_edgelist** out) {
  kc_edgelist* e;
  if (kc_status st = make(out, &e)) return st;
  if (scale == 0 || scale > 31 || edge_factor <= 0 || a < 0 || b < 0 || c < 0 || a + b + c > 1.0 + 1e-12) {
    delete e;
    return kc::fail(KC_ERR_INVALID_ARG, "bad R-MAT parameters");
  }
  const uint64_t samples = (uint64_t)std::llround(edge_factor * (double)(1ull << scale));
  const uint64_t chunk = 1u << 16;
  const uint64_t nch = (samples + chunk - 1) / chunk;
  const double ab = a + b, abc = a + b + c;
  parallel_chunks(nch, e->vsrc, e->vdst, [&](uint64_t ci, std::vector<uint32_t>& S, std::vector<uint32_t>& D) {
    Rng rng(mix_seed(seed, ci + 1));
    uint64_t lo = ci * chunk, hi = std::min(samples, lo + chunk);
    S.reserve(hi - lo);
    D.reserve(hi - lo);
    for (uint64_t i = lo; i < hi; ++i) {
      uint32_t u = 0, v = 0;
      for (uint32_t lvl = 0; lvl < scale; ++lvl) {
        double r = rng.uniform();
        uint32_t bu = 0, bv = 0;
        if (r < a) {
        } else if (r < ab) {
          bv = 1;
        } else if (r < abc) {
          bu = 1;
        } else {
          bu = 1; bv = 1;
        }
        u = (u << 1) | bu;
        v = (v << 1) | bv;
      }
      S.push_back(u);
      D.push_back(v);
    }
  });
  e->n_nodes = 1u << scale;
  return done(e, pinned, out);
}

// Chung-Lu with expected degrees w_i proportional to (i+1)^(-1/(exponent-1)),
// scaled to the requested mean and then capped at max_degree, sampled with the
// linear-time method of Miller and Hagberg (2011): vertices are in decreasing
// weight order, and for each u the candidates v > u are visited by geometric
// skips under the running edge probability bound.
kc_status kc_gen_chung_lu(uint32_t n, double exponent, double mean_degree, double max_degree,
                          uint64_t seed, int pinned, kc_edgelist** out) {
  kc_edgelist* e;
  if (kc_status st = make(out, &e)) return st;
  if (n < 2 || exponent <= 1 || mean_degree <= 0) {
    delete e;
    return kc::fail(KC_ERR_INVALID_ARG, "bad Chung-Lu parameters");
  }
  std::vector<double> w(n);
  const double alpha = 1.0 / (exponent - 1.0);
  double sum = 0;
  for (uint32_t i = 0; i < n; ++i) { w[i] = std::pow((double)i + 1.0, -alpha); sum += w[i]; }
  const double scale = mean_degree * n / sum;
  double S_tot = 0;
  for (uint32_t i = 0; i < n; ++i) {
    w[i] *= scale;
    if (max_degree > 0 && w[i] > max_degree) w[i] = max_degree;
    S_tot += w[i];
  }
  const uint64_t chunk = 256;
  const uint64_t nch = (n + chunk - 1) / chunk;
  parallel_chunks(nch, e->vsrc, e->vdst, [&](uint64_t ci, std::vector<uint32_t>& S, std::vector<uint32_t>& D) {
    uint64_t lo = ci * chunk, hi = std::min<uint64_t>(n, lo + chunk);
    for (uint64_t u = lo; u < hi; ++u) {
      Rng rng(mix_seed(seed, u + 1));
      uint64_t v = u + 1;
      double p = (v < n) ? std::min(w[u] * w[v] / S_tot, 1.0) : 0;
      while (v < n && p > 0) {
        if (p != 1.0) {
          double r = rng.uniform_pos();
          double skip = std::floor(std::log(r) / std::log(1.0 - p));
          if (skip >= (double)n) break;
          v += (uint64_t)skip;
        }
        if (v >= n) break;
        double q = std::min(w[u] * w[v] / S_tot, 1.0);
        double r = rng.uniform();
        if (r < q / p) { S.push_back((uint32_t)u); D.push_back((uint32_t)v); }
        p = q;
        ++v;
      }
    }
  });
  e->n_nodes = n;
  return done(e, pinned, out);
}

// Stochastic block model: `blocks` near-equal blocks, p_in inside a block,
// p_out across blocks.
kc_status kc_gen_sbm(uint32_t n, uint32_t blocks, double p_in, double p_out, uint64_t seed,
                     int pinned, kc_edgelist** out) {
  kc_edgelist* e;
  if (kc_status st = make(out, &e)) return st;
  if (blocks == 0 || blocks > n) { delete e; return kc::fail(KC_ERR_INVALID_ARG, "bad block count"); }
  std::vector<uint32_t> off(blocks + 1);
  for (uint32_t b = 0; b <= blocks; ++b) off[b] = (uint32_t)((uint64_t)n * b / blocks);
  uint64_t stream = 1;
  for (uint32_t x = 0; x < blocks; ++x) {
    Rng rng(mix_seed(seed, stream++));
    er_into(off[x + 1] - off[x], p_in, rng, off[x], e->vsrc, e->vdst);
    for (uint32_t y = x + 1; y < blocks; ++y) {
      Rng r2(mix_seed(seed, stream++));
      bip_into(off[x + 1] - off[x], off[y + 1] - off[y], p_out, r2, off[x], off[y], e->vsrc, e->vdst);
    }
  }
  e->n_nodes = n;
  return done(e, pinned, out);
}

kc_status kc_gen_plant_cliques(kc_edgelist* e, uint32_t count, uint32_t smin, uint32_t smax,
                               uint64_t seed) {
  if (!e) return kc::fail(KC_ERR_INVALID_ARG, "edge list is NULL");
  if (smin > smax || smin < 1) return kc::fail(KC_ERR_INVALID_ARG, "bad clique sizes");
  Rng rng(mix_seed(seed, 0x5eed));
  auto sets = disjoint_sets(e->n_nodes, count, smin, smax, rng);
  std::vector<uint32_t> S, D;
  for (auto& s : sets) clique_into(s, S, D);
  if (e->pinned) {
    // rebuild the pinned arrays with the clique edges appended
    std::vector<uint32_t> a(e->psrc, e->psrc + e->n_edges), b(e->pdst, e->pdst + e->n_edges);
    a.insert(a.end(), S.begin(), S.end());
    b.insert(b.end(), D.begin(), D.end());
    cudaFreeHost(e->psrc);
    cudaFreeHost(e->pdst);
    e->psrc = e->pdst = nullptr;
    e->pinned = 0;
    e->vsrc.swap(a);
    e->vdst.swap(b);
    return kc::edgelist_finish(e, 1);
  }
  e->vsrc.insert(e->vsrc.end(), S.begin(), S.end());
  e->vdst.insert(e->vdst.end(), D.begin(), D.end());
  e->n_edges = e->vsrc.size();
  return KC_OK;
}

// The mixed batch of small graphs. Graph g draws everything from seed base+g:
//   n log-uniform in [n_min, n_max];
//   family 0: G(n,p), p ~ U[0.005, 0.05];
//   family 1: 4-block SBM, p_in 0.1, p_out 0.005;
//   family 2: G(n,p), p ~ U[0.005, 0.05], plus one clique of size U{20..40};
//   k uniform in [k_min, k_max].
kc_status kc_gen_batch(uint32_t n_graphs, uint64_t base_seed, uint32_t n_min, uint32_t n_max,
                       uint32_t k_min, uint32_t k_max, int pinned, kc_edgelist** out) {
  kc_edgelist* e;
  if (kc_status st = make(out, &e)) return st;
  if (n_min < 2 || n_max < n_min || k_min < 1 || k_max < k_min) {
    delete e;
    return kc::fail(KC_ERR_INVALID_ARG, "bad batch parameters");
  }
  e->nn.resize(n_graphs);
  e->kk.resize(n_graphs);
  e->fam.resize(n_graphs);
  std::vector<std::vector<uint32_t>> gs(n_graphs), gd(n_graphs);
  std::atomic<uint32_t> next{0};
  std::vector<std::thread> th;
  for (int t = 0; t < host_threads(); ++t)
    th.emplace_back([&]() {
      for (;;) {
        uint32_t g = next.fetch_add(1);
        if (g >= n_graphs) break;
        Rng rng(mix_seed(base_seed + g, 0));
        double lr = std::log((double)n_min) + rng.uniform() * (std::log((double)n_max) - std::log((double)n_min));
        uint32_t n = (uint32_t)std::llround(std::exp(lr));
        n = std::min(std::max(n, n_min), n_max);
        uint32_t fam = (uint32_t)rng.below(3);
        uint32_t k = k_min + (uint32_t)rng.below((uint64_t)k_max - k_min + 1);
        auto& S = gs[g];
        auto& D = gd[g];
        if (fam == 0 || fam == 2) {
          double p = 0.005 + rng.uniform() * (0.05 - 0.005);
          er_into(n, p, rng, 0, S, D);
          if (fam == 2) {
            uint32_t s = 20 + (uint32_t)rng.below(21);
            s = std::min(s, n);
            auto sets = disjoint_sets(n, 1, s, s, rng);
            for (auto& c : sets) clique_into(c, S, D);
          }
        } else {
          uint32_t off[5];
          for (uint32_t b = 0; b <= 4; ++b) off[b] = (uint32_t)((uint64_t)n * b / 4);
          for (uint32_t x = 0; x < 4; ++x) {
            er_into(off[x + 1] - off[x], 0.1, rng, off[x], S, D);
            for (uint32_t y = x + 1; y < 4; ++y)
              bip_into(off[x + 1] - off[x], off[y + 1] - off[y], 0.005, rng, off[x], off[y], S, D);
          }
        }
        e->nn[g] = n;
        e->kk[g] = k;
        e->fam[g] = fam;
      }
    });
  for (auto& x : th) x.join();
  e->edge_off.resize((size_t)n_graphs + 1);
  uint64_t tot = 0;
  for (uint32_t g = 0; g < n_graphs; ++g) { e->edge_off[g] = tot; tot += gs[g].size(); }
  e->edge_off[n_graphs] = tot;
  e->vsrc.resize(tot);
  e->vdst.resize(tot);
  for (uint32_t g = 0; g < n_graphs; ++g) {
    std::copy(gs[g].begin(), gs[g].end(), e->vsrc.begin() + e->edge_off[g]);
    std::copy(gd[g].begin(), gd[g].end(), e->vdst.begin() + e->edge_off[g]);
  }
  e->n_nodes = 0;
  return done(e, pinned, out);
}

kc_status kc_batchgen_meta(const kc_edgelist* e, const uint64_t** edge_off, const uint32_t** n_nodes,
                           const uint32_t** k, const uint32_t** family, uint32_t* n_graphs) {
  if (!e) return kc::fail(KC_ERR_INVALID_ARG, "edge list is NULL");
  if (e->edge_off.empty()) return kc::fail(KC_ERR_INVALID_ARG, "not a batch edge list");
  if (edge_off) *edge_off = e->edge_off.data();
  if (n_nodes) *n_nodes = e->nn.data();
  if (k) *k = e->kk.data();
  if (family) *family = e->fam.data();
  if (n_graphs) *n_graphs = (uint32_t)e->nn.size();
  return KC_OK;
}

}  // extern "C"
