// Device-wide primitives written for the engine (no CUB): exclusive scan,
// LSD radix sort of 64-bit keys, and segmented sort + dedup of CSR rows.
// Each takes the stream it runs on and allocates its temporaries with the
// stream-ordered allocator.
#pragma once
#include <cstddef>
#include <cstdint>
#include <cuda_runtime.h>

namespace kc {
namespace prim {

// out[i] = sum(in[0..i)), out[n] = total (out has n+1 entries). in may alias out.
cudaError_t scan_exclusive_u32(const uint32_t* in, uint32_t* out, size_t n, cudaStream_t s);
// 64-bit offsets variant (out has n+1 entries).
cudaError_t scan_exclusive_u32_to_u64(const uint32_t* in, unsigned long long* out, size_t n,
                                      cudaStream_t s);

// Sorts keys[0,n) ascending on bits [0, bits). tmp must hold n keys.
// The result ends in keys (the passes ping-pong through tmp).
cudaError_t radix_sort_u64(unsigned long long* keys, unsigned long long* tmp, size_t n, int bits,
                           cudaStream_t s);

// Sorts every row [off[r], off[r+1]) of data ascending and removes duplicates
// in place: the first ucount[r] entries of the row hold its distinct values.
// max_len must bound the longest row. Rows longer than 32768 go through a
// keyed radix sort; the others are sorted in registers or shared memory.
cudaError_t segmented_sort_unique(const uint32_t* off, uint32_t* data, uint32_t* ucount, uint32_t n_rows,
                                  uint32_t max_len, cudaStream_t s);

// Copies the first cnt[r] entries of row r of src (offsets off) into dst at
// new_off[r], for every row.
cudaError_t compact_rows(const uint32_t* off, const uint32_t* src, const uint32_t* new_off,
                         uint32_t* dst, uint32_t n_rows, cudaStream_t s);

// Number of SMs of the current device (cached).
int num_sms();

}  // namespace prim
}  // namespace kc
