// Device memory of the engine: a per-context cache of blocks in front of the
// stream-ordered allocator.
//
// Every engine allocation and free names a stream, and every context
// registers its stream with its own cache. A block freed on a context's
// stream goes back to that context's free list (host bookkeeping only), and
// a later allocation on the same stream takes a free block of a fitting size.
// Reuse is safe without events: the block's last user and its next user are
// ordered by the one stream (work on the context's side streams is joined
// back to it before anything is freed). Steps that repeat the same
// allocations, as a benchmark or a server does, then make no driver
// allocations at all; on B200 the stream-ordered pool's growth and remapping
// of multi-gigabyte blocks cost up to hundreds of milliseconds per call,
// differently from one machine to the next.
//
// Sizes: up to 1 MiB, the next power of two (at least 512 B); above, the next
// multiple of 2 MiB, and a free block up to a quarter larger (plus 2 MiB)
// serves the request. Free blocks beyond kMaxCachedBytes per context are
// returned to the driver, largest first. kc_ctx_release_cached_memory()
// returns them all.
#include <algorithm>
#include <map>
#include <mutex>
#include <unordered_map>

#include "host_common.h"

namespace kc {

namespace {

constexpr size_t kMiB = 1u << 20;
constexpr size_t kMaxCachedBytes = 16ull << 30;

size_t round_size(size_t bytes) {
  if (bytes <= kMiB) {
    size_t r = 512;
    while (r < bytes) r <<= 1;
    return r;
  }
  return (bytes + 2 * kMiB - 1) / (2 * kMiB) * (2 * kMiB);
}

std::mutex g_reg_mu;
std::unordered_map<cudaStream_t, BlockCache*>* g_reg = nullptr;

BlockCache* cache_of(cudaStream_t s) {
  std::lock_guard<std::mutex> l(g_reg_mu);
  if (!g_reg) return nullptr;
  auto it = g_reg->find(s);
  return it == g_reg->end() ? nullptr : it->second;
}

}  // namespace

cudaError_t BlockCache::get(void** p, size_t bytes, cudaStream_t s) {
  const size_t want = round_size(bytes ? bytes : 4);
  {
    std::lock_guard<std::mutex> l(mu_);
    auto it = free_.lower_bound(want);
    const size_t limit = want <= kMiB ? want : want + want / 4 + 2 * kMiB;
    if (it != free_.end() && it->first <= limit) {
      *p = it->second;
      free_bytes_ -= it->first;
      free_.erase(it);
      return cudaSuccess;
    }
  }
  void* q = nullptr;
  const cudaError_t e = cudaMallocAsync(&q, want, s);
  if (e != cudaSuccess) {  // (kc_ctx_release_cached_memory gives the cached blocks back)
    *p = nullptr;
    return e;
  }
  std::lock_guard<std::mutex> l(mu_);
  size_[q] = want;
  *p = q;
  return cudaSuccess;
}

void BlockCache::put(void* p, cudaStream_t s) {
  if (!p) return;
  std::lock_guard<std::mutex> l(mu_);
  auto it = size_.find(p);
  if (it == size_.end()) {  // not from this cache
    cudaFreeAsync(p, s);
    return;
  }
  free_.emplace(it->second, p);
  free_bytes_ += it->second;
  while (free_bytes_ > kMaxCachedBytes && !free_.empty()) {
    auto big = std::prev(free_.end());
    free_bytes_ -= big->first;
    size_.erase(big->second);
    cudaFreeAsync(big->second, s);
    free_.erase(big);
  }
}

void BlockCache::release(cudaStream_t s) {
  std::lock_guard<std::mutex> l(mu_);
  for (auto& kv : free_) {
    size_.erase(kv.second);
    cudaFreeAsync(kv.second, s);
  }
  free_.clear();
  free_bytes_ = 0;
}

uint64_t BlockCache::cached_bytes() {
  std::lock_guard<std::mutex> l(mu_);
  return free_bytes_;
}

void register_stream_cache(cudaStream_t s, BlockCache* c) {
  std::lock_guard<std::mutex> l(g_reg_mu);
  if (!g_reg) g_reg = new std::unordered_map<cudaStream_t, BlockCache*>();
  (*g_reg)[s] = c;
}

void unregister_stream_cache(cudaStream_t s) {
  std::lock_guard<std::mutex> l(g_reg_mu);
  if (g_reg) g_reg->erase(s);
}

cudaError_t dmalloc_raw(void** p, size_t bytes, cudaStream_t s) {
  BlockCache* c = cache_of(s);
  if (c) return c->get(p, bytes, s);
  return cudaMallocAsync(p, bytes ? bytes : 4, s);
}

void dfree(void* p, cudaStream_t s) {
  if (!p) return;
  BlockCache* c = cache_of(s);
  if (c) c->put(p, s);
  else cudaFreeAsync(p, s);
}

}  // namespace kc
