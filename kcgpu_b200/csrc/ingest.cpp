// Graph files: text edge lists, Matrix Market and the reference's binary
// edge list, parsed on host threads into a kc_edgelist.
//
// The reference reads its inputs with graph::EdgeListFile (include/
// FIleReader.cuh:33-937): 100 edges per fscanf call for text, 24-byte records
// {dst, src, weight} as u64 for .bel (:84-90), and a Matrix Market reader
// (:187-234). Here the whole file is read once and split into chunks at line
// boundaries; each host thread parses its chunk and the pieces are
// concatenated in file order, so the result does not depend on the thread
// count. The engine symmetrises, drops self-loops and removes duplicates on
// the GPU afterwards, so a file may list each edge once or in both
// directions, in any order.
#include <algorithm>
#include <cerrno>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <new>
#include <string>
#include <thread>
#include <vector>

#include "edgelist.h"

namespace {

int reader_threads() {
  const unsigned t = std::thread::hardware_concurrency();
  return t ? (int)std::min(t, 32u) : 1;
}

kc_status read_file(const char* path, std::vector<char>* buf) {
  FILE* f = std::fopen(path, "rb");
  if (!f) return kc::fail(KC_ERR_INVALID_ARG, "cannot open %s: %s", path, std::strerror(errno));
  std::fseek(f, 0, SEEK_END);
  const long sz = std::ftell(f);
  std::fseek(f, 0, SEEK_SET);
  if (sz < 0) {
    std::fclose(f);
    return kc::fail(KC_ERR_INVALID_ARG, "cannot size %s", path);
  }
  try {
    buf->resize((size_t)sz);
  } catch (const std::bad_alloc&) {
    std::fclose(f);
    return kc::fail(KC_ERR_OOM, "host allocation of %ld bytes for %s failed", sz, path);
  }
  const size_t got = sz ? std::fread(buf->data(), 1, (size_t)sz, f) : 0;
  std::fclose(f);
  if (got != (size_t)sz) return kc::fail(KC_ERR_INVALID_ARG, "short read of %s", path);
  return KC_OK;
}

struct Piece {
  std::vector<uint32_t> src, dst;
  uint64_t bad = UINT64_MAX;  // byte offset of the first malformed line
  uint32_t max_id = 0;
  bool any = false;
};

inline bool is_space(char c) { return c == ' ' || c == '\t' || c == ',' || c == '\r'; }

// Parses "a b [anything]" lines of [beg, end). one_based: ids start at 1.
void parse_lines(const char* base, size_t beg, size_t end, bool one_based, Piece* out) {
  size_t i = beg;
  while (i < end) {
    const size_t line = i;
    while (i < end && is_space(base[i])) ++i;
    if (i >= end) break;
    if (base[i] == '\n' || base[i] == '#' || base[i] == '%') {  // blank or comment line
      while (i < end && base[i] != '\n') ++i;
      ++i;
      continue;
    }
    uint64_t v[2] = {0, 0};
    bool ok = true;
    for (int f = 0; f < 2 && ok; ++f) {
      while (i < end && is_space(base[i])) ++i;
      if (i >= end || base[i] < '0' || base[i] > '9') {
        ok = false;
        break;
      }
      uint64_t x = 0;
      while (i < end && base[i] >= '0' && base[i] <= '9') {
        x = x * 10 + (uint64_t)(base[i] - '0');
        if (x > 0xffffffffull) ok = false;
        ++i;
      }
      v[f] = x;
    }
    if (ok && one_based) {
      if (v[0] == 0 || v[1] == 0) ok = false;
      v[0] -= 1;
      v[1] -= 1;
    }
    if (ok && (v[0] >= 0xffffffffull || v[1] >= 0xffffffffull)) ok = false;
    if (!ok) {
      if (out->bad == UINT64_MAX) out->bad = line;
      while (i < end && base[i] != '\n') ++i;
      ++i;
      continue;
    }
    out->src.push_back((uint32_t)v[0]);
    out->dst.push_back((uint32_t)v[1]);
    out->max_id = std::max<uint32_t>(out->max_id, (uint32_t)std::max(v[0], v[1]));
    out->any = true;
    while (i < end && base[i] != '\n') ++i;  // rest of the line (weights, ...)
    ++i;
  }
}

kc_status parse_text(const std::vector<char>& buf, size_t start, bool one_based, kc_edgelist* e,
                     uint32_t* max_id, bool* any) {
  const size_t n = buf.size();
  const int T = (int)std::max<size_t>(1, std::min<size_t>(reader_threads(), (n - start) / (1u << 20) + 1));
  std::vector<size_t> cut((size_t)T + 1, n);
  cut[0] = start;
  for (int t = 1; t < T; ++t) {  // chunk boundaries on line starts
    size_t c = start + (n - start) * (size_t)t / (size_t)T;
    while (c < n && buf[c - 1] != '\n') ++c;
    cut[t] = std::max(c, cut[t - 1]);
  }
  std::vector<Piece> pieces((size_t)T);
  std::vector<std::thread> th;
  for (int t = 0; t < T; ++t)
    th.emplace_back([&, t]() { parse_lines(buf.data(), cut[t], cut[t + 1], one_based, &pieces[t]); });
  for (auto& x : th) x.join();
  size_t total = 0;
  for (auto& p : pieces) {
    if (p.bad != UINT64_MAX) {
      size_t lineno = 1 + (size_t)std::count(buf.begin(), buf.begin() + (long)p.bad, '\n');
      return kc::fail(KC_ERR_INVALID_ARG, "line %zu: expected two vertex ids%s below 2^32-1", lineno,
                      one_based ? " (1-based)" : "");
    }
    total += p.src.size();
  }
  e->vsrc.reserve(total);
  e->vdst.reserve(total);
  for (auto& p : pieces) {
    e->vsrc.insert(e->vsrc.end(), p.src.begin(), p.src.end());
    e->vdst.insert(e->vdst.end(), p.dst.begin(), p.dst.end());
    if (p.any) {
      *max_id = *any ? std::max(*max_id, p.max_id) : p.max_id;
      *any = true;
    }
  }
  return KC_OK;
}

kc_status parse_bel(const std::vector<char>& buf, kc_edgelist* e, uint32_t* max_id, bool* any) {
  if (buf.size() % 24 != 0)
    return kc::fail(KC_ERR_INVALID_ARG, "a .bel file holds 24-byte records; size %zu is not a multiple", buf.size());
  const size_t m = buf.size() / 24;
  e->vsrc.resize(m);
  e->vdst.resize(m);
  const int T = (int)std::max<size_t>(1, std::min<size_t>(reader_threads(), m / (1u << 18) + 1));
  std::vector<uint32_t> mx((size_t)T, 0);
  std::vector<int> bad((size_t)T, 0);
  std::vector<std::thread> th;
  for (int t = 0; t < T; ++t)
    th.emplace_back([&, t]() {
      const size_t b = m * (size_t)t / (size_t)T, en = m * (size_t)(t + 1) / (size_t)T;
      for (size_t i = b; i < en; ++i) {
        uint64_t rec[2];
        std::memcpy(rec, buf.data() + 24 * i, 16);  // {dst, src, weight}
        if (rec[0] >= 0xffffffffull || rec[1] >= 0xffffffffull) {
          bad[t] = 1;
          continue;
        }
        e->vdst[i] = (uint32_t)rec[0];
        e->vsrc[i] = (uint32_t)rec[1];
        mx[t] = std::max(mx[t], (uint32_t)std::max(rec[0], rec[1]));
      }
    });
  for (auto& x : th) x.join();
  for (int t = 0; t < T; ++t)
    if (bad[t]) return kc::fail(KC_ERR_INVALID_ARG, "a .bel record holds a vertex id of 2^32-1 or more");
  if (m) {
    *max_id = *std::max_element(mx.begin(), mx.end());
    *any = true;
  }
  return KC_OK;
}

bool ends_with(const std::string& s, const char* suf) {
  const size_t n = std::strlen(suf);
  return s.size() >= n && s.compare(s.size() - n, n, suf) == 0;
}

}  // namespace

extern "C" {

kc_status kc_edgelist_from_file(const char* path, uint32_t format, int pinned, kc_edgelist** out) {
  kc::clear_error();
  if (!path || !out) return kc::fail(KC_ERR_INVALID_ARG, "NULL argument");
  *out = nullptr;
  if (format > KC_FILE_BEL) return kc::fail(KC_ERR_INVALID_ARG, "unknown file format %u", format);
  const std::string p(path);
  if (format == KC_FILE_AUTO) format = ends_with(p, ".bel") ? KC_FILE_BEL : ends_with(p, ".mtx") ? KC_FILE_MTX : KC_FILE_TEXT;
  std::vector<char> buf;
  KC_TRY(read_file(path, &buf));
  kc_edgelist* e = new (std::nothrow) kc_edgelist();
  if (!e) return kc::fail(KC_ERR_OOM, "host allocation failed");
  uint32_t max_id = 0;
  bool any = false;
  uint64_t declared_n = 0;
  kc_status st = KC_OK;
  if (format == KC_FILE_BEL) {
    st = parse_bel(buf, e, &max_id, &any);
  } else if (format == KC_FILE_MTX) {
    // %%MatrixMarket banner, % comments, "rows cols entries", then 1-based entries
    size_t i = 0;
    if (buf.size() < 14 || std::memcmp(buf.data(), "%%MatrixMarket", 14) != 0) {
      st = kc::fail(KC_ERR_INVALID_ARG, "%s: no %%%%MatrixMarket banner", path);
    } else {
      bool sized = false;
      while (i < buf.size() && !sized) {
        const size_t line = i;
        while (i < buf.size() && buf[i] != '\n') ++i;
        ++i;
        if (buf[line] == '%' || buf[line] == '\n') continue;
        unsigned long long r = 0, c = 0, nz = 0;
        const std::string s(buf.data() + line, std::min(i, buf.size()) - line);
        if (std::sscanf(s.c_str(), "%llu %llu %llu", &r, &c, &nz) != 3) {
          st = kc::fail(KC_ERR_INVALID_ARG, "%s: bad size line", path);
          break;
        }
        declared_n = std::max(r, c);
        sized = true;
      }
      if (st == KC_OK) st = parse_text(buf, std::min(i, buf.size()), true, e, &max_id, &any);
    }
  } else {
    st = parse_text(buf, 0, false, e, &max_id, &any);
  }
  if (st == KC_OK) {
    const uint64_t n = std::max<uint64_t>(declared_n, any ? (uint64_t)max_id + 1 : 0);
    if (n >= 0xffffffffull) st = kc::fail(KC_ERR_INVALID_ARG, "more than 2^32-2 vertices");
    e->n_nodes = (uint32_t)n;
  }
  if (st == KC_OK) st = kc::edgelist_finish(e, pinned);
  if (st != KC_OK) {
    delete e;
    return st;
  }
  *out = e;
  return KC_OK;
}

kc_status kc_graph_from_file(kc_ctx* ctx, const char* path, uint32_t format, kc_graph** out) {
  kc_edgelist* e = nullptr;
  KC_TRY(kc_edgelist_from_file(path, format, 0, &e));
  const kc_status st = kc_graph_from_edges(ctx, e->src(), e->dst(), e->n_edges, e->n_nodes, out);
  delete e;
  return st;
}

}  // extern "C"
