// Device-wide primitives: exclusive scan, LSD radix sort of 64-bit keys and
// segmented row sort + dedup. These replace the reference's CUB calls
// (CUBScanExclusive / CUBSelect, include/cub_wrappers.cuh:11-179, and the
// large-select path of include/ScanLarge.cuh:333-361) on the CSR-build and
// orientation passes. All passes are HBM-bound integer work.
#include <algorithm>
#include <cstdio>

#include "dev_common.cuh"
#include "host_common.h"
#include "prims.cuh"

namespace kc {
namespace prim {

namespace {

constexpr int NT = 256;             // threads per block for scan / radix
constexpr int ITEMS = 16;           // items per thread
constexpr int TILE = NT * ITEMS;    // 4096 elements per block

template <class T>
__device__ T warp_incl_scan(T v) {
  const uint32_t lane = lane_id();
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    T t = __shfl_up_sync(0xffffffffu, v, o);
    if (lane >= (uint32_t)o) v += t;
  }
  return v;
}

// Exclusive block scan of one value per thread (blockDim.x == NT); returns the
// exclusive prefix and writes the block total to *total.
template <class T>
__device__ T block_excl_scan(T v, T* total) {
  __shared__ T warp_sums[NT / 32];
  const uint32_t lane = lane_id(), w = threadIdx.x >> 5;
  T inc = warp_incl_scan(v);
  if (lane == 31) warp_sums[w] = inc;
  __syncthreads();
  if (w == 0) {
    T x = lane < NT / 32 ? warp_sums[lane] : T(0);
    T xi = warp_incl_scan(x);
    if (lane < NT / 32) warp_sums[lane] = xi - x;
    if (lane == NT / 32 - 1) *total = xi;
  }
  __syncthreads();
  T r = inc - v + warp_sums[w];
  __syncthreads();
  return r;
}

template <class TO>
__global__ void __launch_bounds__(NT) k_scan_reduce(const uint32_t* __restrict__ in, size_t n,
                                                    TO* __restrict__ sums) {
  size_t base = (size_t)blockIdx.x * TILE;
  TO acc = 0;
#pragma unroll
  for (int i = 0; i < ITEMS; ++i) {
    size_t idx = base + (size_t)i * NT + threadIdx.x;
    if (idx < n) acc += in[idx];
  }
  __shared__ TO tot;
  block_excl_scan<TO>(acc, &tot);
  if (threadIdx.x == 0) sums[blockIdx.x] = tot;
}

// Single block: exclusive scan of sums[0,nb) in place; writes the grand total.
template <class TO>
__global__ void __launch_bounds__(NT) k_scan_sums(TO* sums, uint32_t nb, TO* total_out) {
  __shared__ TO tot;
  TO carry = 0;
  for (uint32_t base = 0; base < nb; base += NT) {
    uint32_t i = base + threadIdx.x;
    TO v = i < nb ? sums[i] : TO(0);
    TO ex = block_excl_scan<TO>(v, &tot);
    if (i < nb) sums[i] = ex + carry;
    carry += tot;
    __syncthreads();
  }
  if (threadIdx.x == 0) *total_out = carry;
}

template <class TO>
__global__ void __launch_bounds__(NT) k_scan_apply(const uint32_t* in, TO* out, size_t n,
                                                   const TO* __restrict__ sums) {
  __shared__ TO tile[TILE + TILE / 32];
  __shared__ TO tot;
  const size_t base = (size_t)blockIdx.x * TILE;
  auto at = [](uint32_t i) { return i + (i >> 5); };  // padding against bank conflicts
#pragma unroll
  for (int i = 0; i < ITEMS; ++i) {
    uint32_t li = (uint32_t)i * NT + threadIdx.x;
    size_t idx = base + li;
    tile[at(li)] = idx < n ? (TO)in[idx] : TO(0);
  }
  __syncthreads();
  TO run = 0;
  const uint32_t t0 = threadIdx.x * ITEMS;
#pragma unroll
  for (int i = 0; i < ITEMS; ++i) {
    TO v = tile[at(t0 + i)];
    tile[at(t0 + i)] = run;
    run += v;
  }
  TO ex = block_excl_scan<TO>(run, &tot);
  ex += sums[blockIdx.x];
#pragma unroll
  for (int i = 0; i < ITEMS; ++i) tile[at(t0 + i)] += ex;
  __syncthreads();
#pragma unroll
  for (int i = 0; i < ITEMS; ++i) {
    uint32_t li = (uint32_t)i * NT + threadIdx.x;
    size_t idx = base + li;
    if (idx < n) out[idx] = tile[at(li)];
  }
}

template <class TO>
cudaError_t scan_impl(const uint32_t* in, TO* out, size_t n, cudaStream_t s) {
  const uint32_t nb = (uint32_t)std::max<size_t>(1, (n + TILE - 1) / TILE);
  TO* sums = nullptr;
  cudaError_t e = kc::dmalloc(&sums, sizeof(TO) * nb, s);
  if (e != cudaSuccess) return e;
  if (n) k_scan_reduce<TO><<<nb, NT, 0, s>>>(in, n, sums);
  else e = cudaMemsetAsync(sums, 0, sizeof(TO) * nb, s);
  if (e != cudaSuccess) { kc::dfree(sums, s); return e; }
  k_scan_sums<TO><<<1, NT, 0, s>>>(sums, nb, out + n);
  if (n) k_scan_apply<TO><<<nb, NT, 0, s>>>(in, out, n, sums);
  e = cudaGetLastError();
  kc::dfree(sums, s);
  return e;
}

// ---- radix sort -----------------------------------------------------------

__global__ void __launch_bounds__(NT) k_radix_hist(const unsigned long long* __restrict__ keys, size_t n,
                                                   int shift, uint32_t* __restrict__ hist, uint32_t nb) {
  __shared__ uint32_t h[256];
  for (uint32_t i = threadIdx.x; i < 256; i += NT) h[i] = 0;
  __syncthreads();
  const size_t base = (size_t)blockIdx.x * TILE;
#pragma unroll 4
  for (int i = 0; i < ITEMS; ++i) {
    size_t idx = base + (size_t)i * NT + threadIdx.x;
    if (idx < n) atomicAdd(&h[(uint32_t)(keys[idx] >> shift) & 255u], 1u);
  }
  __syncthreads();
  for (uint32_t d = threadIdx.x; d < 256; d += NT) hist[(size_t)d * nb + blockIdx.x] = h[d];
}

// Stable scatter: keys of the tile are ranked in their original order. Each
// round takes NT consecutive keys; lanes with equal digits find each other with
// __match_any_sync, and per-warp digit counts order the warps.
__global__ void __launch_bounds__(NT) k_radix_scatter(const unsigned long long* __restrict__ in,
                                                      unsigned long long* __restrict__ out, size_t n,
                                                      int shift, const uint32_t* __restrict__ offs,
                                                      uint32_t nb) {
  constexpr int NW = NT / 32;
  __shared__ uint32_t cnt[NW][256];
  __shared__ uint32_t run[256];
  __shared__ uint32_t boff[256];
  const uint32_t tid = threadIdx.x, w = tid >> 5, lane = lane_id();
  for (uint32_t d = tid; d < 256; d += NT) {
    run[d] = 0;
    boff[d] = offs[(size_t)d * nb + blockIdx.x];
#pragma unroll
    for (int q = 0; q < NW; ++q) cnt[q][d] = 0;
  }
  __syncthreads();
  const size_t base = (size_t)blockIdx.x * TILE;
  for (int r = 0; r < ITEMS; ++r) {
    size_t idx = base + (size_t)r * NT + tid;
    bool valid = idx < n;
    unsigned long long key = valid ? in[idx] : 0ull;
    uint32_t d = valid ? ((uint32_t)(key >> shift) & 255u) : 256u + lane;
    uint32_t peers = __match_any_sync(0xffffffffu, d);
    uint32_t rank = __popc(peers & lanemask_lt());
    if (valid && rank == 0) cnt[w][d] = __popc(peers);
    __syncthreads();
    if (valid) {
      uint32_t pos = boff[d] + run[d] + rank;
      for (uint32_t q = 0; q < w; ++q) pos += cnt[q][d];
      out[pos] = key;
    }
    __syncthreads();
    for (uint32_t dd = tid; dd < 256; dd += NT) {
      uint32_t s = 0;
#pragma unroll
      for (int q = 0; q < NW; ++q) { s += cnt[q][dd]; cnt[q][dd] = 0; }
      run[dd] += s;
    }
    __syncthreads();
  }
}

// ---- segmented sort + dedup --------------------------------------------------

enum RowClass { RC_TRIVIAL = 0, RC_WARP = 1, RC_B2K = 2, RC_B16K = 3, RC_B32K = 4, RC_HUGE = 5, RC_W256 = 6, RC_N = 7 };

__device__ __forceinline__ int row_class(uint32_t len) {
  if (len <= 1) return RC_TRIVIAL;
  if (len <= 32) return RC_WARP;
  if (len <= 256) return RC_W256;
  if (len <= 2048) return RC_B2K;
  if (len <= 16384) return RC_B16K;
  if (len <= 32768) return RC_B32K;
  return RC_HUGE;
}

// One pass over the rows: trivial rows get their count directly, the others
// are appended to the list of their size class (warp-aggregated atomics).
__global__ void k_classify_rows(const uint32_t* __restrict__ off, uint32_t n_rows, uint32_t* ucnt,
                                uint32_t* lists, uint32_t* counts, unsigned long long* huge_total) {
  const uint32_t lane = lane_id();
  for (uint32_t base = blockIdx.x * blockDim.x; base < n_rows; base += gridDim.x * blockDim.x) {
    uint32_t r = base + threadIdx.x;
    bool valid = r < n_rows;
    uint32_t len = valid ? off[r + 1] - off[r] : 0;
    int c = valid ? row_class(len) : -1;
    if (c == RC_TRIVIAL) ucnt[r] = len;
    for (int cls = RC_WARP; cls < RC_N; ++cls) {
      uint32_t m = __ballot_sync(0xffffffffu, c == cls);
      if (!m) continue;
      uint32_t leader = __ffs(m) - 1, pos0 = 0;
      if (lane == leader) pos0 = atomicAdd(&counts[cls], __popc(m));
      pos0 = __shfl_sync(0xffffffffu, pos0, leader);
      if (c == cls) lists[(size_t)cls * n_rows + pos0 + __popc(m & lanemask_lt())] = r;
      if (cls == RC_HUGE && c == cls) atomicAdd(huge_total, (unsigned long long)len);
    }
  }
}

__global__ void k_seg_warp(const uint32_t* __restrict__ off, uint32_t* data, uint32_t* ucnt,
                           const uint32_t* __restrict__ list, const uint32_t* count, uint32_t n_rows) {
  const uint32_t lane = lane_id();
  const uint32_t gw = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const uint32_t nw = (gridDim.x * blockDim.x) >> 5;
  const uint32_t cnt = min(*count, n_rows);
  for (uint32_t i = gw; i < cnt; i += nw) {
    const uint32_t r = list[i];
    const uint32_t b = off[r], len = off[r + 1] - b;
    uint32_t v = lane < len ? data[b + lane] : 0xffffffffu;
#pragma unroll
    for (int k = 2; k <= 32; k <<= 1) {
#pragma unroll
      for (int j = k >> 1; j > 0; j >>= 1) {
        uint32_t p = __shfl_xor_sync(0xffffffffu, v, j);
        bool asc = (lane & k) == 0;
        bool lower = (lane & j) == 0;
        v = (lower == asc) ? min(v, p) : max(v, p);
      }
    }
    uint32_t prev = __shfl_up_sync(0xffffffffu, v, 1);
    bool keep = lane < len && (lane == 0 || v != prev);
    uint32_t bal = __ballot_sync(0xffffffffu, keep);
    if (keep) data[b + __popc(bal & lanemask_lt())] = v;
    if (lane == 0) ucnt[r] = __popc(bal);
  }
}

// Warp per row for rows of 33..256 entries, sorted in registers: the row is
// padded to N = 32 E entries (E = 2, 4 or 8) and held striped, element
// i = e * 32 + lane in register e of that lane, so loads and stores are
// coalesced. Bitonic network: partners less than 32 apart are in other lanes
// (one shuffle), farther partners are in another register of the same lane.
// Dedup compares each element with its predecessor (lane - 1, or lane 31 of
// the previous register).
template <int E>
__device__ __forceinline__ void warp_sort_unique_row(uint32_t* data, uint32_t b, uint32_t len, uint32_t* ucnt_r,
                                                     uint32_t lane) {
  uint32_t v[E];
#pragma unroll
  for (int e = 0; e < E; ++e) {
    const uint32_t i = (uint32_t)e * 32u + lane;
    v[e] = i < len ? data[b + i] : 0xffffffffu;
  }
#pragma unroll
  for (uint32_t k = 2; k <= 32u * E; k <<= 1) {
#pragma unroll
    for (uint32_t j = k >> 1; j > 0; j >>= 1) {
      if (j >= 32u) {
        const uint32_t jj = j >> 5;
#pragma unroll
        for (int e = 0; e < E; ++e) {
          if ((uint32_t)e & jj) continue;
          const uint32_t i = (uint32_t)e * 32u + lane;
          const uint32_t a = v[e], c = v[e ^ jj];
          const bool asc = (i & k) == 0;
          v[e] = asc ? min(a, c) : max(a, c);
          v[e ^ jj] = asc ? max(a, c) : min(a, c);
        }
      } else {
        const bool lower = (lane & j) == 0;
#pragma unroll
        for (int e = 0; e < E; ++e) {
          const uint32_t i = (uint32_t)e * 32u + lane;
          const uint32_t p = __shfl_xor_sync(0xffffffffu, v[e], j);
          const bool asc = (i & k) == 0;
          v[e] = (lower == asc) ? min(v[e], p) : max(v[e], p);
        }
      }
    }
  }
  uint32_t outpos = 0;
#pragma unroll
  for (int e = 0; e < E; ++e) {
    const uint32_t i = (uint32_t)e * 32u + lane;
    const uint32_t up = __shfl_up_sync(0xffffffffu, v[e], 1);
    const uint32_t wrap = e > 0 ? __shfl_sync(0xffffffffu, v[e > 0 ? e - 1 : 0], 31) : 0u;
    const uint32_t prev = lane > 0 ? up : wrap;
    const bool keep = i < len && (i == 0 || v[e] != prev);
    const uint32_t bal = __ballot_sync(0xffffffffu, keep);
    if (keep) data[b + outpos + __popc(bal & lanemask_lt())] = v[e];
    outpos += __popc(bal);
  }
  if (lane == 0) *ucnt_r = outpos;
}

__global__ void __launch_bounds__(256) k_seg_warp_reg(const uint32_t* __restrict__ off, uint32_t* data,
                                                      uint32_t* ucnt, const uint32_t* __restrict__ list,
                                                      const uint32_t* count, uint32_t n_rows) {
  const uint32_t lane = lane_id();
  const uint32_t gw = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const uint32_t nw = (gridDim.x * blockDim.x) >> 5;
  const uint32_t cnt = min(*count, n_rows);
  for (uint32_t li = gw; li < cnt; li += nw) {
    const uint32_t r = list[li];
    const uint32_t b = off[r], len = off[r + 1] - b;
    if (len <= 64) warp_sort_unique_row<2>(data, b, len, ucnt + r, lane);
    else if (len <= 128) warp_sort_unique_row<4>(data, b, len, ucnt + r, lane);
    else if (len <= 256) warp_sort_unique_row<8>(data, b, len, ucnt + r, lane);
  }
}

// Block per row: bitonic sort in shared memory on the next power of two, then
// an ordered compaction of the distinct values.
template <int BT>
__global__ void __launch_bounds__(BT) k_seg_block(const uint32_t* __restrict__ off, uint32_t* data,
                                                  uint32_t* ucnt, const uint32_t* __restrict__ list,
                                                  const uint32_t* count, uint32_t n_rows, uint32_t cap) {
  extern __shared__ uint32_t sm[];
  __shared__ uint32_t wsum[BT / 32];
  const uint32_t tid = threadIdx.x, lane = lane_id(), w = tid >> 5;
  const uint32_t cnt = min(*count, n_rows);
  for (uint32_t li = blockIdx.x; li < cnt; li += gridDim.x) {
    const uint32_t r = list[li];
    const uint32_t b = off[r], len = off[r + 1] - b;
    if (len > cap) continue;  // never index past the shared buffer
    uint32_t p2 = 1;
    while (p2 < len) p2 <<= 1;
    for (uint32_t i = tid; i < p2; i += BT) sm[i] = i < len ? data[b + i] : 0xffffffffu;
    __syncthreads();
    for (uint32_t k = 2; k <= p2; k <<= 1) {
      for (uint32_t j = k >> 1; j > 0; j >>= 1) {
        for (uint32_t i = tid; i < p2; i += BT) {
          uint32_t ixj = i ^ j;
          if (ixj > i) {
            uint32_t a = sm[i], c = sm[ixj];
            bool asc = (i & k) == 0;
            if ((a > c) == asc) { sm[i] = c; sm[ixj] = a; }
          }
        }
        __syncthreads();
      }
    }
    uint32_t outpos = 0;
    for (uint32_t c0 = 0; c0 < len; c0 += BT) {
      uint32_t i = c0 + tid;
      bool keep = i < len && (i == 0 || sm[i] != sm[i - 1]);
      uint32_t bal = __ballot_sync(0xffffffffu, keep);
      if (lane == 0) wsum[w] = __popc(bal);
      __syncthreads();
      uint32_t before = 0, total = 0;
      for (uint32_t q = 0; q < BT / 32; ++q) {
        if (q < w) before += wsum[q];
        total += wsum[q];
      }
      if (keep) data[b + outpos + before + __popc(bal & lanemask_lt())] = sm[i];
      outpos += total;
      __syncthreads();
    }
    if (tid == 0) ucnt[r] = outpos;
    __syncthreads();
  }
}

// Huge rows: composite keys (list position << 32 | value), one radix sort.
__global__ void k_huge_keys(const uint32_t* __restrict__ off, const uint32_t* __restrict__ data,
                            const uint32_t* __restrict__ hlist, const uint32_t* __restrict__ hstart,
                            uint32_t H, unsigned long long* keys) {
  for (uint32_t h = blockIdx.x; h < H; h += gridDim.x) {
    const uint32_t r = hlist[h];
    const uint32_t b = off[r], len = off[r + 1] - b, s = hstart[h];
    for (uint32_t i = threadIdx.x; i < len; i += blockDim.x)
      keys[(size_t)s + i] = ((unsigned long long)h << 32) | data[b + i];
  }
}

__global__ void k_huge_lengths(const uint32_t* __restrict__ off, const uint32_t* __restrict__ hlist,
                               uint32_t H, uint32_t* len) {
  for (uint32_t h = blockIdx.x * blockDim.x + threadIdx.x; h < H; h += gridDim.x * blockDim.x)
    len[h] = off[hlist[h] + 1] - off[hlist[h]];
}

__global__ void k_huge_flags(const unsigned long long* __restrict__ keys, size_t T, uint32_t* flag) {
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < T; i += (size_t)gridDim.x * blockDim.x)
    flag[i] = (i == 0 || keys[i] != keys[i - 1]) ? 1u : 0u;
}

__global__ void k_huge_write(const unsigned long long* __restrict__ keys, size_t T,
                             const uint32_t* __restrict__ flag, const uint32_t* __restrict__ pos,
                             const uint32_t* __restrict__ hlist, const uint32_t* __restrict__ hstart,
                             const uint32_t* __restrict__ off, uint32_t* data) {
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < T; i += (size_t)gridDim.x * blockDim.x) {
    if (!flag[i]) continue;
    unsigned long long k = keys[i];
    uint32_t h = (uint32_t)(k >> 32);
    data[off[hlist[h]] + (pos[i] - pos[hstart[h]])] = (uint32_t)k;
  }
}

__global__ void k_huge_count(const uint32_t* __restrict__ hlist, const uint32_t* __restrict__ hstart,
                             uint32_t H, const uint32_t* __restrict__ pos, uint32_t* ucnt) {
  for (uint32_t h = blockIdx.x * blockDim.x + threadIdx.x; h < H; h += gridDim.x * blockDim.x)
    ucnt[hlist[h]] = pos[hstart[h + 1]] - pos[hstart[h]];
}

__global__ void k_compact_rows(const uint32_t* __restrict__ off, const uint32_t* __restrict__ src,
                               const uint32_t* __restrict__ new_off, uint32_t* __restrict__ dst,
                               uint32_t n_rows) {
  const uint32_t lane = lane_id();
  const uint32_t gw = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const uint32_t nw = (gridDim.x * blockDim.x) >> 5;
  for (uint32_t r = gw; r < n_rows; r += nw) {
    const uint32_t b = off[r], nb = new_off[r], c = new_off[r + 1] - nb;
    for (uint32_t i = lane; i < c; i += 32) dst[nb + i] = src[b + i];
  }
}

int g_sms = 0;

}  // namespace

int num_sms() {
  if (!g_sms) {
    int dev = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&g_sms, cudaDevAttrMultiProcessorCount, dev);
    if (g_sms <= 0) g_sms = 148;
  }
  return g_sms;
}

cudaError_t scan_exclusive_u32(const uint32_t* in, uint32_t* out, size_t n, cudaStream_t s) {
  return scan_impl<uint32_t>(in, out, n, s);
}

cudaError_t scan_exclusive_u32_to_u64(const uint32_t* in, unsigned long long* out, size_t n,
                                      cudaStream_t s) {
  return scan_impl<unsigned long long>(in, out, n, s);
}

cudaError_t radix_sort_u64(unsigned long long* keys, unsigned long long* tmp, size_t n, int bits,
                           cudaStream_t s) {
  if (n <= 1 || bits <= 0) return cudaSuccess;
  const uint32_t nb = (uint32_t)((n + TILE - 1) / TILE);
  uint32_t* hist = nullptr;
  cudaError_t e = kc::dmalloc(&hist, sizeof(uint32_t) * ((size_t)256 * nb + 1), s);
  if (e != cudaSuccess) return e;
  unsigned long long* a = keys;
  unsigned long long* b = tmp;
  int passes = 0;
  for (int shift = 0; shift < bits; shift += 8, ++passes) {
    k_radix_hist<<<nb, NT, 0, s>>>(a, n, shift, hist, nb);
    e = scan_exclusive_u32(hist, hist, (size_t)256 * nb, s);
    if (e != cudaSuccess) break;
    k_radix_scatter<<<nb, NT, 0, s>>>(a, b, n, shift, hist, nb);
    std::swap(a, b);
  }
  if (e == cudaSuccess && (passes & 1))
    e = cudaMemcpyAsync(keys, a, n * sizeof(unsigned long long), cudaMemcpyDeviceToDevice, s);
  kc::dfree(hist, s);
  if (e == cudaSuccess) e = cudaGetLastError();
  return e;
}

cudaError_t segmented_sort_unique(const uint32_t* off, uint32_t* data, uint32_t* ucount, uint32_t n_rows,
                                  uint32_t max_len, cudaStream_t s) {
  if (n_rows == 0) return cudaSuccess;
  uint32_t* lists = nullptr;
  uint32_t* counts = nullptr;
  unsigned long long* huge_total = nullptr;
  cudaError_t e = kc::dmalloc(&lists, sizeof(uint32_t) * (size_t)RC_N * n_rows, s);
  if (e != cudaSuccess) return e;
  // 8 class counters (RC_N used) followed by the 64-bit total of the huge rows
  constexpr size_t kCountBytes = sizeof(uint32_t) * 8 + sizeof(unsigned long long) * 2;
  e = kc::dmalloc(&counts, kCountBytes, s);
  if (e != cudaSuccess) { kc::dfree(lists, s); return e; }
  huge_total = reinterpret_cast<unsigned long long*>(counts + 8);
  e = cudaMemsetAsync(counts, 0, kCountBytes, s);
  if (e != cudaSuccess) { kc::dfree(lists, s); kc::dfree(counts, s); return e; }
  const int sms = num_sms();
  {
    uint32_t grid = (uint32_t)std::min<size_t>((n_rows + 255) / 256, (size_t)sms * 16);
    k_classify_rows<<<grid, 256, 0, s>>>(off, n_rows, ucount, lists, counts, huge_total);
  }
  if (max_len > 32)
    k_seg_warp_reg<<<sms * 8, 256, 0, s>>>(off, data, ucount, lists + (size_t)RC_W256 * n_rows, counts + RC_W256,
                                            n_rows);
  k_seg_warp<<<sms * 8, 256, 0, s>>>(off, data, ucount, lists + (size_t)RC_WARP * n_rows, counts + RC_WARP,
                                     n_rows);
  if (max_len > 32)
    k_seg_block<256><<<sms * 8, 256, 2048 * sizeof(uint32_t), s>>>(off, data, ucount,
                                                                  lists + (size_t)RC_B2K * n_rows, counts + RC_B2K,
                                                                  n_rows, 2048u);
  if (max_len > 2048) {
    cudaFuncSetAttribute(k_seg_block<1024>, cudaFuncAttributeMaxDynamicSharedMemorySize, 32768 * 4);
    k_seg_block<1024><<<sms, 1024, 16384 * sizeof(uint32_t), s>>>(off, data, ucount,
                                                                 lists + (size_t)RC_B16K * n_rows, counts + RC_B16K,
                                                                 n_rows, 16384u);
  }
  if (max_len > 16384)
    k_seg_block<1024><<<sms, 1024, 32768 * sizeof(uint32_t), s>>>(off, data, ucount,
                                                                 lists + (size_t)RC_B32K * n_rows, counts + RC_B32K,
                                                                 n_rows, 32768u);
  e = cudaGetLastError();
  if (e == cudaSuccess && max_len > 32768) {
    // Rows beyond shared memory: read back how many, sort them with one keyed radix sort.
    uint32_t H = 0;
    unsigned long long T = 0;
    cudaMemcpyAsync(&H, counts + RC_HUGE, sizeof(uint32_t), cudaMemcpyDeviceToHost, s);
    cudaMemcpyAsync(&T, huge_total, sizeof(T), cudaMemcpyDeviceToHost, s);
    e = cudaStreamSynchronize(s);
    if (e == cudaSuccess && H > 0) {
      const uint32_t* hlist = lists + (size_t)RC_HUGE * n_rows;
      uint32_t *hlen = nullptr, *hstart = nullptr, *flag = nullptr, *pos = nullptr;
      unsigned long long *keys = nullptr, *tmp = nullptr;
      // every allocation is checked: a failed one must stop the sort before a kernel sees its null pointer
      e = kc::dmalloc(&hlen, sizeof(uint32_t) * (H + 1), s);
      if (e == cudaSuccess) e = kc::dmalloc(&hstart, sizeof(uint32_t) * (H + 1), s);
      if (e == cudaSuccess) e = kc::dmalloc(&keys, sizeof(unsigned long long) * T, s);
      if (e == cudaSuccess) e = kc::dmalloc(&tmp, sizeof(unsigned long long) * T, s);
      if (e == cudaSuccess) e = kc::dmalloc(&flag, sizeof(uint32_t) * T, s);
      if (e == cudaSuccess) e = kc::dmalloc(&pos, sizeof(uint32_t) * (T + 1), s);
      if (e == cudaSuccess) {
        k_huge_lengths<<<(H + 255) / 256, 256, 0, s>>>(off, hlist, H, hlen);
        e = scan_exclusive_u32(hlen, hstart, H, s);
        k_huge_keys<<<std::min<uint32_t>(H, 4096), 1024, 0, s>>>(off, data, hlist, hstart, H, keys);
        int hb = 0;
        while ((1u << hb) < H) ++hb;
        if (e == cudaSuccess) e = radix_sort_u64(keys, tmp, T, 32 + hb, s);
        uint32_t g = (uint32_t)std::min<unsigned long long>((T + 255) / 256, (unsigned long long)sms * 32);
        k_huge_flags<<<g, 256, 0, s>>>(keys, T, flag);
        if (e == cudaSuccess) e = scan_exclusive_u32(flag, pos, T, s);
        k_huge_write<<<g, 256, 0, s>>>(keys, T, flag, pos, hlist, hstart, off, data);
        k_huge_count<<<(H + 255) / 256, 256, 0, s>>>(hlist, hstart, H, pos, ucount);
        if (e == cudaSuccess) e = cudaGetLastError();
      }
      void* hp[] = {hlen, hstart, keys, tmp, flag, pos};
      for (void* p : hp)
        if (p) kc::dfree(p, s);
    }
  }
  kc::dfree(lists, s);
  kc::dfree(counts, s);
  return e;
}

cudaError_t compact_rows(const uint32_t* off, const uint32_t* src, const uint32_t* new_off, uint32_t* dst,
                         uint32_t n_rows, cudaStream_t s) {
  if (!n_rows) return cudaSuccess;
  uint32_t grid = (uint32_t)std::min<size_t>(((size_t)n_rows * 32 + 255) / 256, (size_t)num_sms() * 32);
  k_compact_rows<<<grid, 256, 0, s>>>(off, src, new_off, dst, n_rows);
  return cudaGetLastError();
}

}  // namespace prim
}  // namespace kc
