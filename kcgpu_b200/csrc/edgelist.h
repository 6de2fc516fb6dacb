// The host edge list handed out by the generators and the file readers
// (kc_edgelist in include/kc.h).
#pragma once

#include <algorithm>
#include <cstdint>
#include <cstring>
#include <vector>

#include <cuda_runtime.h>

#include "../../include/kc.h"
#include "host_common.h"

struct kc_edgelist {
  std::vector<uint32_t> vsrc, vdst;  // used when not pinned
  uint32_t* psrc = nullptr;          // page-locked copies (when pinned)
  uint32_t* pdst = nullptr;
  uint64_t n_edges = 0;
  uint32_t n_nodes = 0;
  int pinned = 0;
  // batch metadata (kc_gen_batch)
  std::vector<uint64_t> edge_off;
  std::vector<uint32_t> nn, kk, fam;

  const uint32_t* src() const { return pinned ? psrc : vsrc.data(); }
  const uint32_t* dst() const { return pinned ? pdst : vdst.data(); }
  ~kc_edgelist() {
    if (psrc) cudaFreeHost(psrc);
    if (pdst) cudaFreeHost(pdst);
  }
};

namespace kc {

// Moves the vectors into page-locked memory when requested.
inline kc_status edgelist_finish(kc_edgelist* e, int pinned) {
  e->n_edges = e->vsrc.size();
  if (!pinned) return KC_OK;
  size_t bytes = std::max<size_t>(1, e->n_edges) * sizeof(uint32_t);
  if (cudaMallocHost(&e->psrc, bytes) != cudaSuccess || cudaMallocHost(&e->pdst, bytes) != cudaSuccess) {
    cudaGetLastError();
    return kc::fail(KC_ERR_OOM, "cudaMallocHost of %zu bytes for a pinned edge list failed", bytes);
  }
  std::memcpy(e->psrc, e->vsrc.data(), e->n_edges * sizeof(uint32_t));
  std::memcpy(e->pdst, e->vdst.data(), e->n_edges * sizeof(uint32_t));
  e->pinned = 1;
  std::vector<uint32_t>().swap(e->vsrc);
  std::vector<uint32_t>().swap(e->vdst);
  return KC_OK;
}

}  // namespace kc
