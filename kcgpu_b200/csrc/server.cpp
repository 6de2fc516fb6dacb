// Continuous-batching request server for clique-count queries.
//
// No counterpart in the reference (one graph per process, results printed).
// Requests (a resident graph + k, or a one-shot edge list + k) enter a queue.
// W worker threads, each with its own context and CUDA stream, take the first
// queued request whose projected device footprint fits in the HBM budget next
// to the resident graphs and the requests already on the device, as soon as a
// worker is free (a blocked head can be passed only while it is young, see
// admissible()). Requests therefore start while others are still running,
// and their kernels overlap on the device through the workers' streams. A
// worker that takes a one-shot request also takes the other queued one-shot
// requests that fit (up to 512 requests / 8M edges) and counts them in one
// batched call; a worker that takes a request for a resident graph also takes
// the other queued requests for that graph (up to 32) and answers them with
// one walk for all their k. Results are exact integers, so a request's count
// is the same alone and in any mix.
#include <algorithm>
#include <atomic>
#include <chrono>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <memory>
#include <mutex>
#include <new>
#include <thread>
#include <unordered_map>
#include <vector>

#include <cuda_runtime.h>

#include "engine.h"
#include "host_common.h"

namespace {

// A resident graph is complete (oriented, edge rows built) before any request
// sees it, so requests only read it: any worker counts it on its own context
// and stream, several at a time.
struct Resident {
  kc_graph* g = nullptr;
  uint64_t bytes = 0;
  kc_graph_info info{};
  ~Resident() {
    if (g) kc_graph_destroy(g);
  }
};

struct Request {
  uint64_t ticket = 0;
  uint64_t graph_id = 0;  // 0: one-shot
  std::vector<uint32_t> src, dst;
  uint32_t n = 0;
  uint32_t k = 0;
  uint64_t footprint = 0;
  bool running = false, done = false;
  kc_request_result res{};
};

}  // namespace

struct kc_server {
  kc_ctx* base = nullptr;
  kc_server_opts opts{};
  uint64_t budget = 0;
  std::vector<kc_ctx*> wctx;
  std::vector<std::thread> workers;
  std::mutex mu;
  std::condition_variable cv_work, cv_done;
  std::deque<std::shared_ptr<Request>> queue;
  std::unordered_map<uint64_t, std::shared_ptr<Request>> reqs;
  std::unordered_map<uint64_t, std::shared_ptr<Resident>> graphs;
  uint64_t next_ticket = 1, next_graph = 1;
  uint64_t inflight_bytes = 0, resident_bytes = 0;
  uint32_t rr = 0;
  bool stop = false;
  std::chrono::steady_clock::time_point t0;

  double ms() const {
    return std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
  }
};

namespace {

kc_params choose(const kc_server* s, const kc_graph_info& inf, uint32_t k) {
  kc_params p;
  if (s->opts.autotune) {
    p = kc::autotune(inf.n, inf.m, inf.max_out_degree, k, inf.max_core, s->opts.orientation);
  } else {
    p = s->opts.fixed;
    if (p.part == 0) p.part = 8;
  }
  p.k = k;
  p.flags = 0;
  if (k <= 2) p.unit = KC_UNIT_NODE;
  return p;
}

void execute(kc_server* s, kc_ctx* ctx, Request& r) {
  kc_u128 out{0, 0};
  kc_status st = KC_OK;
  if (r.graph_id) {
    std::shared_ptr<Resident> res;
    {
      std::lock_guard<std::mutex> l(s->mu);
      auto it = s->graphs.find(r.graph_id);
      if (it != s->graphs.end()) res = it->second;
    }
    if (!res) {
      st = kc::fail(KC_ERR_INVALID_ARG, "graph %llu is not resident", (unsigned long long)r.graph_id);
    } else {
      kc_params p = choose(s, res->info, r.k);
      r.res.params = p;
      st = kc::count_on(ctx, res->g, &p, &out, nullptr);
    }
  } else {
    kc_graph* g = nullptr;
    st = kc_graph_from_edges(ctx, r.src.data(), r.dst.data(), r.src.size(), r.n, &g);
    if (st == KC_OK) st = kc_orient(g, s->opts.orientation);
    if (st == KC_OK) {
      kc_graph_info inf;
      kc_graph_get_info(g, &inf);
      kc_params p = choose(s, inf, r.k);
      r.res.params = p;
      st = kc_count(g, &p, &out, nullptr);
    }
    if (g) kc_graph_destroy(g);
    std::vector<uint32_t>().swap(r.src);
    std::vector<uint32_t>().swap(r.dst);
  }
  r.res.count = out;
  r.res.status = st;
}

// One-shot requests queued back to back are counted together: one batched
// call (disjoint union on the device, per-graph orientation and algorithm,
// one captured counting launch) instead of one call each.
constexpr size_t kBatchMaxRequests = 512;
constexpr uint64_t kBatchMaxEdges = 8u << 20;

void execute_batch(kc_server* s, kc_ctx* ctx, std::vector<std::shared_ptr<Request>>& rs) {
  std::vector<kc_batch_graph> gs(rs.size());
  for (size_t i = 0; i < rs.size(); ++i) {
    Request& r = *rs[i];
    gs[i].src = r.src.data();
    gs[i].dst = r.dst.data();
    gs[i].n_edges = r.src.size();
    gs[i].n_nodes = r.n;
    gs[i].k = r.k;
  }
  kc_batch_opts o;
  std::memset(&o, 0, sizeof(o));
  o.orientation = s->opts.orientation;
  o.autotune = s->opts.autotune;
  o.fixed = s->opts.fixed;
  if (o.fixed.part == 0) o.fixed.part = 8;
  o.use_graph = 1;
  std::vector<kc_u128> counts(rs.size());
  std::vector<kc_params> choice(rs.size());
  const kc_status st = kc_batch_count(ctx, gs.data(), (uint32_t)gs.size(), &o, counts.data(), choice.data(), nullptr);
  for (size_t i = 0; i < rs.size(); ++i) {
    Request& r = *rs[i];
    r.res.count = st == KC_OK ? counts[i] : kc_u128{0, 0};
    r.res.params = choice[i];
    r.res.status = st;
    std::vector<uint32_t>().swap(r.src);
    std::vector<uint32_t>().swap(r.dst);
  }
}

// Requests for one resident graph queued together are answered by one
// pivoting walk for all their k (kc_count_multi: the walk goes to the largest
// k and takes each smaller k where it closes), instead of one walk each.
void execute_resident_group(kc_server* s, kc_ctx* ctx, std::vector<std::shared_ptr<Request>>& rs) {
  std::shared_ptr<Resident> res;
  {
    std::lock_guard<std::mutex> l(s->mu);
    auto it = s->graphs.find(rs.front()->graph_id);
    if (it != s->graphs.end()) res = it->second;
  }
  kc_status st = KC_OK;
  std::vector<uint32_t> ks;
  std::vector<kc_u128> out(rs.size(), kc_u128{0, 0});
  kc_params p;
  std::memset(&p, 0, sizeof(p));
  if (!res) {
    st = kc::fail(KC_ERR_INVALID_ARG, "graph %llu is not resident", (unsigned long long)rs.front()->graph_id);
  } else {
    uint32_t kmax = 0;
    for (auto& r : rs) {
      ks.push_back(r->k);
      kmax = std::max(kmax, r->k);
    }
    p = choose(s, res->info, kmax);
    p.mode = KC_MODE_PIVOT;
    p.part = 32;
    p.encoding = KC_ENC_BITMAP;
    st = kc::count_multi_on(ctx, res->g, &p, ks.data(), (uint32_t)ks.size(), out.data());
  }
  for (size_t i = 0; i < rs.size(); ++i) {
    rs[i]->res.count = st == KC_OK ? out[i] : kc_u128{0, 0};
    rs[i]->res.params = p;
    rs[i]->res.params.k = rs[i]->k;
    rs[i]->res.status = st;
  }
}

// Admission: the first queued request whose projected footprint fits next to
// the resident graphs and the requests already running (any request when
// nothing runs, so a request as large as the whole budget still starts).
// Requests behind a blocked head may pass it, but only while the head is
// younger than kHeadAgeMs: after that nothing passes it, the device drains
// and the head starts, so a large request is not starved by a stream of
// small ones.
constexpr double kHeadAgeMs = 250.0;

std::deque<std::shared_ptr<Request>>::iterator admissible(kc_server* s) {
  auto fits = [&](const Request& r) {
    return s->inflight_bytes == 0 || s->resident_bytes + s->inflight_bytes + r.footprint <= s->budget;
  };
  if (s->queue.empty()) return s->queue.end();
  if (fits(*s->queue.front())) return s->queue.begin();
  if (s->ms() - s->queue.front()->res.submit_ms > kHeadAgeMs) return s->queue.end();
  for (auto it = s->queue.begin() + 1; it != s->queue.end(); ++it)
    if (fits(**it)) return it;
  return s->queue.end();
}

void worker_main(kc_server* s, size_t wi) {
  kc_ctx* ctx = s->wctx[wi];
  for (;;) {
    std::vector<std::shared_ptr<Request>> rs;
    {
      std::unique_lock<std::mutex> l(s->mu);
      auto pick = s->queue.end();
      // a blocked head that comes of age needs no event, so the wait wakes
      // up now and then to look again
      while (!s->stop && (pick = admissible(s)) == s->queue.end())
        s->cv_work.wait_for(l, std::chrono::milliseconds(20));
      if (s->stop) return;
      uint64_t edges = 0;
      auto take = [&](std::deque<std::shared_ptr<Request>>::iterator it) {
        std::shared_ptr<Request> r = *it;
        s->queue.erase(it);
        s->inflight_bytes += r->footprint;
        r->running = true;
        r->res.start_ms = s->ms();
        edges += r->src.size();
        rs.push_back(std::move(r));
      };
      take(pick);
      // requests for the same resident graph queued anywhere behind it join
      // it in one walk (at most 32 of them)
      if (rs.front()->graph_id != 0) {
        const uint64_t gid = rs.front()->graph_id;
        size_t i = 0;
        while (i < s->queue.size() && rs.size() < 32) {
          const Request& r = *s->queue[i];
          if (r.graph_id == gid && s->resident_bytes + s->inflight_bytes + r.footprint <= s->budget)
            take(s->queue.begin() + (long)i);
          else
            ++i;
        }
      }
      // one-shot requests (k >= 3) queued anywhere behind it join it in one
      // batched call while they fit
      if (rs.front()->graph_id == 0 && rs.front()->k >= 3) {
        size_t i = 0;  // (erase invalidates deque iterators: walk by index)
        while (i < s->queue.size() && rs.size() < kBatchMaxRequests) {
          const Request& r = *s->queue[i];
          if (r.graph_id == 0 && r.k >= 3 && edges + r.src.size() <= kBatchMaxEdges &&
              s->resident_bytes + s->inflight_bytes + r.footprint <= s->budget)
            take(s->queue.begin() + (long)i);  // the next request moves up to index i
          else
            ++i;
        }
      }
    }
    if (rs.size() == 1) execute(s, ctx, *rs[0]);
    else if (rs.front()->graph_id != 0) execute_resident_group(s, ctx, rs);
    else execute_batch(s, ctx, rs);
    {
      std::lock_guard<std::mutex> l(s->mu);
      const double t = s->ms();
      for (auto& r : rs) {
        s->inflight_bytes -= r->footprint;
        r->running = false;
        r->done = true;
        r->res.done_ms = t;
      }
    }
    s->cv_done.notify_all();
    s->cv_work.notify_all();
  }
}

kc_status enqueue(kc_server* s, std::shared_ptr<Request> r, uint64_t* ticket) {
  {
    std::lock_guard<std::mutex> l(s->mu);
    if (r->footprint + s->resident_bytes > s->budget)
      return kc::fail(KC_ERR_ADMISSION, "request needs %llu bytes; budget %llu with %llu resident",
                      (unsigned long long)r->footprint, (unsigned long long)s->budget,
                      (unsigned long long)s->resident_bytes);
    r->ticket = s->next_ticket++;
    r->res.submit_ms = s->ms();
    r->res.k = r->k;
    r->res.graph_id = r->graph_id;
    r->res.status = KC_ERR_BUSY;
    s->reqs[r->ticket] = r;
    s->queue.push_back(r);
    *ticket = r->ticket;
  }
  s->cv_work.notify_one();
  return KC_OK;
}

}  // namespace

extern "C" {

kc_status kc_server_create(kc_ctx* ctx, const kc_server_opts* opts, kc_server** out) {
  kc::clear_error();
  if (!ctx || !out) return kc::fail(KC_ERR_INVALID_ARG, "NULL argument");
  *out = nullptr;
  kc_server* s = new (std::nothrow) kc_server();
  if (!s) return kc::fail(KC_ERR_OOM, "host allocation failed");
  s->base = ctx;
  if (opts) s->opts = *opts;
  else {
    std::memset(&s->opts, 0, sizeof(s->opts));
    s->opts.autotune = 1;
  }
  if (s->opts.orientation > KC_ORIENT_DEGEN) {
    delete s;
    return kc::fail(KC_ERR_INVALID_ARG, "unknown orientation");
  }
  const uint64_t dev_total = ctx->total_mem ? ctx->total_mem : (180ull << 30);
  s->budget = s->opts.hbm_budget_bytes ? s->opts.hbm_budget_bytes : std::min<uint64_t>(180ull * 1000000000ull, dev_total);
  const uint32_t nw = std::max<uint32_t>(1, s->opts.streams ? s->opts.streams : (s->opts.max_inflight ? s->opts.max_inflight : 4));
  s->t0 = std::chrono::steady_clock::now();
  for (uint32_t i = 0; i < nw; ++i) {
    kc_ctx* w = nullptr;
    kc_status st = kc_ctx_create(ctx->device, &w);
    if (st == KC_OK) {
      w->tail_help = nw == 1;  // several workers share the SMs (see kc_ctx::tail_help)
      st = kc::warm_context(w);
      if (st != KC_OK) kc_ctx_destroy(w);
    }
    if (st != KC_OK) {
      for (auto* c : s->wctx) kc_ctx_destroy(c);
      delete s;
      return st;
    }
    s->wctx.push_back(w);
  }
  for (uint32_t i = 0; i < nw; ++i) s->workers.emplace_back(worker_main, s, (size_t)i);
  *out = s;
  return KC_OK;
}

kc_status kc_server_destroy(kc_server* s) {
  if (!s) return KC_OK;
  {
    std::lock_guard<std::mutex> l(s->mu);
    s->stop = true;
    for (auto& r : s->queue) {
      r->done = true;
      r->res.status = KC_ERR_CANCELLED;
    }
    s->queue.clear();
  }
  s->cv_work.notify_all();
  s->cv_done.notify_all();
  for (auto& t : s->workers) t.join();
  s->graphs.clear();
  s->reqs.clear();
  for (auto* c : s->wctx) kc_ctx_destroy(c);
  delete s;
  return KC_OK;
}

kc_status kc_server_put_graph(kc_server* s, const uint32_t* src, const uint32_t* dst, uint64_t n_edges,
                              uint32_t n_nodes, uint64_t* graph_id) {
  if (!s || !graph_id || (n_edges && (!src || !dst))) return kc::fail(KC_ERR_INVALID_ARG, "NULL argument");
  const uint64_t fp = kc_footprint_bytes(n_nodes, n_edges, 0);
  kc_ctx* owner;
  {
    std::lock_guard<std::mutex> l(s->mu);
    if (s->resident_bytes + fp > s->budget)
      return kc::fail(KC_ERR_ADMISSION, "graph needs %llu bytes; %llu of %llu already resident",
                      (unsigned long long)fp, (unsigned long long)s->resident_bytes, (unsigned long long)s->budget);
    owner = s->wctx[s->rr++ % s->wctx.size()];
  }
  auto res = std::make_shared<Resident>();
  KC_TRY(kc_graph_from_edges(owner, src, dst, n_edges, n_nodes, &res->g));
  KC_TRY(kc_orient(res->g, s->opts.orientation));
  KC_TRY(kc::complete_for_sharing(res->g));
  kc_graph_get_info(res->g, &res->info);
  res->bytes = res->info.device_bytes;
  std::lock_guard<std::mutex> l(s->mu);
  const uint64_t id = s->next_graph++;
  s->graphs[id] = res;
  s->resident_bytes += res->bytes;
  *graph_id = id;
  return KC_OK;
}

kc_status kc_server_drop_graph(kc_server* s, uint64_t graph_id) {
  if (!s) return kc::fail(KC_ERR_INVALID_ARG, "server is NULL");
  std::shared_ptr<Resident> res;
  {
    std::lock_guard<std::mutex> l(s->mu);
    auto it = s->graphs.find(graph_id);
    if (it == s->graphs.end()) return kc::fail(KC_ERR_INVALID_ARG, "graph %llu is not resident", (unsigned long long)graph_id);
    res = it->second;
    s->resident_bytes -= res->bytes;
    s->graphs.erase(it);
  }
  return KC_OK;  // freed when the last request using it finishes
}

kc_status kc_server_submit(kc_server* s, uint64_t graph_id, uint32_t k, uint64_t* ticket) {
  if (!s || !ticket) return kc::fail(KC_ERR_INVALID_ARG, "NULL argument");
  if (k < 1) return kc::fail(KC_ERR_INVALID_ARG, "k must be >= 1");
  auto r = std::make_shared<Request>();
  {
    std::lock_guard<std::mutex> l(s->mu);
    auto it = s->graphs.find(graph_id);
    if (it == s->graphs.end()) return kc::fail(KC_ERR_INVALID_ARG, "graph %llu is not resident", (unsigned long long)graph_id);
    const auto& inf = it->second->info;
    // counting scratch only: the graph itself is already resident
    r->footprint = kc_footprint_bytes(inf.n, inf.m, inf.max_out_degree) - inf.device_bytes / 2;
  }
  r->graph_id = graph_id;
  r->k = k;
  return enqueue(s, r, ticket);
}

kc_status kc_server_submit_edges(kc_server* s, const uint32_t* src, const uint32_t* dst, uint64_t n_edges,
                                 uint32_t n_nodes, uint32_t k, uint64_t* ticket) {
  if (!s || !ticket || (n_edges && (!src || !dst))) return kc::fail(KC_ERR_INVALID_ARG, "NULL argument");
  if (k < 1) return kc::fail(KC_ERR_INVALID_ARG, "k must be >= 1");
  auto r = std::make_shared<Request>();
  r->src.assign(src, src + n_edges);
  r->dst.assign(dst, dst + n_edges);
  r->n = n_nodes;
  r->k = k;
  r->footprint = kc_footprint_bytes(n_nodes, n_edges, 0);
  return enqueue(s, r, ticket);
}

kc_status kc_server_cancel(kc_server* s, uint64_t ticket) {
  if (!s) return kc::fail(KC_ERR_INVALID_ARG, "server is NULL");
  std::lock_guard<std::mutex> l(s->mu);
  auto it = s->reqs.find(ticket);
  if (it == s->reqs.end()) return kc::fail(KC_ERR_INVALID_ARG, "unknown ticket %llu", (unsigned long long)ticket);
  auto r = it->second;
  if (r->done) return KC_OK;
  if (r->running) return kc::fail(KC_ERR_BUSY, "request %llu is already running", (unsigned long long)ticket);
  s->queue.erase(std::remove(s->queue.begin(), s->queue.end(), r), s->queue.end());
  r->done = true;
  r->res.status = KC_ERR_CANCELLED;
  r->res.done_ms = s->ms();
  s->cv_done.notify_all();
  return KC_OK;
}

kc_status kc_server_wait(kc_server* s, uint64_t ticket, int64_t wait_ms, kc_request_result* out) {
  if (!s || !out) return kc::fail(KC_ERR_INVALID_ARG, "NULL argument");
  std::unique_lock<std::mutex> l(s->mu);
  auto it = s->reqs.find(ticket);
  if (it == s->reqs.end()) return kc::fail(KC_ERR_INVALID_ARG, "unknown ticket %llu", (unsigned long long)ticket);
  auto r = it->second;
  if (wait_ms < 0) s->cv_done.wait(l, [&]() { return r->done; });
  else if (wait_ms > 0) s->cv_done.wait_for(l, std::chrono::milliseconds(wait_ms), [&]() { return r->done; });
  if (!r->done) return kc::fail(KC_ERR_BUSY, "request %llu not finished", (unsigned long long)ticket);
  *out = r->res;
  s->reqs.erase(ticket);
  return r->res.status == KC_OK ? KC_OK
                                : kc::fail((kc_status)r->res.status, "request %llu failed: %s", (unsigned long long)ticket,
                                           kc_status_string((kc_status)r->res.status));
}

}  // extern "C"
