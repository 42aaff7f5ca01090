/*
 * cuda_cpu_shim.h -- test infrastructure only.
 *
 * Force-included (g++ -include) when the unmodified CLAST reference sources
 * are compiled for the host CPU by oracle/build_ref.py.  Thrust is compiled
 * with its sequential CPP device system, so every thrust::device_vector lives
 * in host memory; this header supplies the few CUDA language pieces the
 * reference's kernels use (qualifiers, dim3, blockIdx/threadIdx, max, the
 * cudaEvent timer calls in main.cu) and a launcher that runs a __global__
 * function over its grid with OpenMP.  The build script rewrites each
 * `kernel<<<grid, block>>>(args)` into `clast_cpu_launch(grid, block, kernel, args)`.
 *
 * Nothing in the product links this file.
 */
#ifndef CLAST_CUDA_CPU_SHIM_H_
#define CLAST_CUDA_CPU_SHIM_H_

#include <algorithm>
#include <cmath>
#include <cstdlib>
#include <cstring>
#include <iostream>

/* Older Thrust releases pulled these in transitively; several reference
 * files use host_vector and std::cout without including them. */
#include <thrust/host_vector.h>
#include <thrust/device_vector.h>
#include <thrust/sequence.h>
#include <thrust/system_error.h>

#define __global__
#define __device__
#define __host__
#define __constant__
#define __forceinline__ inline

struct dim3 {
  unsigned int x, y, z;
  dim3(unsigned int x_ = 1, unsigned int y_ = 1, unsigned int z_ = 1) : x(x_), y(y_), z(z_) {}
};
struct clast_uint3 { unsigned int x, y, z; };

inline thread_local clast_uint3 threadIdx;
inline thread_local clast_uint3 blockIdx;
inline thread_local dim3 blockDim;
inline thread_local dim3 gridDim;

using std::max;
using std::min;

/* Runs kernel k over grid g x block b.  The reference's kernels are
 * embarrassingly parallel (each thread owns its outputs, no shared memory,
 * no barriers), so blocks are distributed over OpenMP threads.  Every
 * kernel guards its own work with `if (idx < limit)`, so the launcher runs
 * the full grid it is given, exactly as the GPU would. */
template <class Kernel, class... Args>
void clast_cpu_launch(dim3 g, dim3 b, Kernel k, Args... args) {
  const long long nblocks = (long long)g.x * g.y * g.z;
#pragma omp parallel for schedule(static)
  for (long long lin = 0; lin < nblocks; ++lin) {
    gridDim = g;
    blockDim = b;
    const unsigned int bx = (unsigned int)(lin % g.x);
    const unsigned int by = (unsigned int)((lin / g.x) % g.y);
    const unsigned int bz = (unsigned int)(lin / ((long long)g.x * g.y));
    blockIdx = clast_uint3{bx, by, bz};
    for (unsigned int tz = 0; tz < b.z; ++tz)
      for (unsigned int ty = 0; ty < b.y; ++ty)
        for (unsigned int tx = 0; tx < b.x; ++tx) {
          threadIdx = clast_uint3{tx, ty, tz};
          k(args...);
        }
  }
}

/* Timer calls made unconditionally by main.cu. */
typedef int cudaEvent_t;
typedef int cudaError_t;
inline cudaError_t cudaSetDevice(int) { return 0; }
inline cudaError_t cudaEventCreate(cudaEvent_t* e) { *e = 0; return 0; }
inline cudaError_t cudaEventRecord(cudaEvent_t, int) { return 0; }
inline cudaError_t cudaEventSynchronize(cudaEvent_t) { return 0; }
inline cudaError_t cudaEventElapsedTime(float* ms, cudaEvent_t, cudaEvent_t) { *ms = 0.f; return 0; }

#endif
