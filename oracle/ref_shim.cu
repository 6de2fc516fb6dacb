// Link-time shim for the reference build (oracle/_ref/kcgpu_ref). TEST
// INFRASTRUCTURE: it is linked only into the reference's own main.cu, never
// into the engine, and it changes no counting arithmetic.
//
// Two wraps (ld --wrap), so the reference's sources stay as shipped:
//
//  * fopen: the reference's pivot drivers read the binomial table from a
//    hard-coded absolute path (kclique/kclique.cuh:1696,1858,2303,2472). A
//    path that ends in "/nCr.txt" is opened from $KC_REF_NCR instead (a table
//    written by tests/golden/make_ref_golden.py in the reference's format:
//    1001 rows of 401 comma-separated values, C(r, c), 0 for c > r).
//
//  * cudaGetDeviceProperties: the reference sizes its per-SM scratch slots as
//    multiProcessorCount x (maxThreadsPerMultiProcessor / 128) and indexes
//    them with the %smid register (kclique/common.cuh:73-84,
//    include/utils_cuda.cuh:160-176). PTX does not promise that %smid stays
//    below the SM count, only below %nsmid, so the wrap reports
//    max(multiProcessorCount, %nsmid): every slot index the kernels form is
//    then inside the arrays. Blocks of 128 threads fit at most
//    2048 / 128 = 16 per SM, the slots per SM, so the slot scan of one SM
//    never leaves that SM's range.
#include <cstdarg>
#include <cstdio>
#include <cstdlib>
#include <cstring>

#include <cuda_runtime.h>

extern "C" {

FILE* __real_fopen(const char* path, const char* mode);
cudaError_t __real_cudaGetDeviceProperties_v2(cudaDeviceProp* prop, int device);

FILE* __wrap_fopen(const char* path, const char* mode) {
  const char* tail = "/nCr.txt";
  const size_t n = path ? std::strlen(path) : 0, t = std::strlen(tail);
  if (n >= t && std::strcmp(path + n - t, tail) == 0) {
    const char* alt = std::getenv("KC_REF_NCR");
    if (alt && *alt) return __real_fopen(alt, mode);
  }
  return __real_fopen(path, mode);
}

}  // extern "C"

__global__ void k_read_nsmid(unsigned* out) {
  unsigned r;
  asm volatile("mov.u32 %0, %%nsmid;" : "=r"(r));
  *out = r;
}

extern "C" cudaError_t __wrap_cudaGetDeviceProperties_v2(cudaDeviceProp* prop, int device) {
  const cudaError_t e = __real_cudaGetDeviceProperties_v2(prop, device);
  if (e != cudaSuccess) return e;
  static int nsmid = -1;
  if (nsmid < 0) {
    int prev = 0;
    cudaGetDevice(&prev);
    cudaSetDevice(device);
    unsigned* d = nullptr;
    unsigned h = 0;
    if (cudaMalloc(&d, sizeof(unsigned)) == cudaSuccess) {
      k_read_nsmid<<<1, 1>>>(d);
      if (cudaMemcpy(&h, d, sizeof(unsigned), cudaMemcpyDeviceToHost) == cudaSuccess) nsmid = (int)h;
      cudaFree(d);
    }
    cudaSetDevice(prev);
    if (nsmid < 0) {
      std::fprintf(stderr, "kcgpu_ref: could not read %%nsmid; refusing to size the slot arrays\n");
      std::exit(3);
    }
    std::fprintf(stderr, "kcgpu_ref: multiProcessorCount %d, %%nsmid %d\n", prop->multiProcessorCount, nsmid);
  }
  if (nsmid > prop->multiProcessorCount) prop->multiProcessorCount = nsmid;
  return e;
}
