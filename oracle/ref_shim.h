/*
 * ref_shim.h -- TEST INFRASTRUCTURE ONLY (oracle side; never linked into the product).
 *
 * Force-included (g++ -include) in front of every reference source file when the
 * reference's own kernels are built as a host shared library under oracle/_ref/.
 * It turns the reference's CUDA C dialect into plain C++:
 *
 *   - __global__/__device__/__host__ become empty qualifiers, so every kernel is an
 *     ordinary host function;
 *   - blockIdx/threadIdx/blockDim/gridDim are per-OS-thread globals that the launch
 *     helper (ref_launch below) sets before calling the kernel body once per (block,
 *     thread) pair, exactly as the hardware would enumerate them;
 *   - cudaMalloc/cudaMemcpy map to calloc/memcpy ("device" memory is host memory).
 *     calloc models freshly cudaMalloc'd memory as zero, which fixes the values the
 *     reference reads before ever writing (zeta, the unused ss tail);
 *   - printf from kernels is routed through ref_printf, which is silent unless
 *     ref_verbose is set.
 *
 * Blocks are independent in every reference kernel (no shared memory, no atomics, no
 * __syncthreads), so ref_launch may run blocks on several OpenMP threads; the threads
 * of one block run serially in threadIdx order.
 */
#ifndef GPL_REF_SHIM_H
#define GPL_REF_SHIM_H

#include <cmath>
#include <math.h>
#include <cstdio>
#include <stdio.h>
#include <cstdlib>
#include <stdlib.h>
#include <cstring>
#include <string.h>
#include <cstdarg>
#include <cstddef>

#define __global__
#define __device__
#define __host__
#define __forceinline__ inline

struct dim3 {
  unsigned int x, y, z;
  constexpr dim3(unsigned int x_ = 1, unsigned int y_ = 1, unsigned int z_ = 1) : x(x_), y(y_), z(z_) {}
};
struct uint3_shim { unsigned int x, y, z; };

inline thread_local uint3_shim blockIdx = {0, 0, 0};
inline thread_local uint3_shim threadIdx = {0, 0, 0};
inline thread_local dim3 blockDim = dim3(1, 1, 1);
inline thread_local dim3 gridDim = dim3(1, 1, 1);

typedef int cudaError_t;
enum { cudaSuccess = 0, cudaErrorMemoryAllocation = 2 };
enum cudaMemcpyKind_shim {
  cudaMemcpyHostToHost = 0, cudaMemcpyHostToDevice = 1,
  cudaMemcpyDeviceToHost = 2, cudaMemcpyDeviceToDevice = 3
};

inline cudaError_t cudaMalloc(void** p, size_t n) {
  *p = calloc(n ? n : 1, 1);
  return *p ? cudaSuccess : cudaErrorMemoryAllocation;
}
inline cudaError_t cudaFree(void* p) { free(p); return cudaSuccess; }
inline cudaError_t cudaMemcpy(void* d, const void* s, size_t n, int) {
  if (n) memmove(d, s, n);
  return cudaSuccess;
}
inline cudaError_t cudaDeviceSynchronize() { return cudaSuccess; }

extern "C" int ref_verbose;
inline int ref_printf(const char* fmt, ...) {
  if (!ref_verbose) return 0;
  va_list ap; va_start(ap, fmt);
  int r = vprintf(fmt, ap);
  va_end(ap);
  return r;
}
#define printf(...) ref_printf(__VA_ARGS__)

/* Serial-per-block, OpenMP-across-blocks emulation of kernel<<<grid, block>>>(...). */
template <class F>
inline void ref_launch(dim3 g, dim3 b, F&& body) {
  const long nblk = (long)g.x * g.y * g.z;
#pragma omp parallel for schedule(dynamic, 8) if (nblk > 1)
  for (long bi = 0; bi < nblk; ++bi) {
    gridDim = g;
    blockDim = b;
    blockIdx.x = (unsigned)(bi % g.x);
    blockIdx.y = (unsigned)((bi / g.x) % g.y);
    blockIdx.z = (unsigned)(bi / ((long)g.x * g.y));
    for (unsigned tz = 0; tz < b.z; ++tz)
      for (unsigned ty = 0; ty < b.y; ++ty)
        for (unsigned tx = 0; tx < b.x; ++tx) {
          threadIdx.x = tx; threadIdx.y = ty; threadIdx.z = tz;
          body();
        }
  }
}

#endif
