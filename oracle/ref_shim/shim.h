// Host-compilation shim for the reference's device header.
//
// Test infrastructure only: this lets g++ compile the reference's own
// `include/cudaKernel.cuh` (farceri/cudaRing) as ordinary host C++ so that its
// kernels can be run on CPU arrays as the parity oracle and as the timed CPU
// baseline.  Nothing in the shipped library includes this file.
//
// What it does:
//   * CUDA execution-space qualifiers become empty (`__shared__` becomes
//     `static`, so a "shared" array is one per host process);
//   * blockIdx/threadIdx/blockDim become thread-local variables that the driver
//     sets before calling a "kernel" as a plain function, one call per index;
//   * atomicAdd(double*) becomes an OpenMP atomic capture, so the reference's
//     atomic scatter kernels stay correct under `#pragma omp parallel for`.
#pragma once
#include <cmath>
#include <cstdlib>
#include <cstring>

#define __global__
#define __device__
#define __host__
#define __constant__
#define __shared__ static
#define __forceinline__ inline

struct crShimDim3 { unsigned long x, y, z; };
extern thread_local crShimDim3 blockIdx, threadIdx, blockDim;

static inline double atomicAdd(double* a, double v) {
  double old;
#pragma omp atomic capture
  { old = *a; *a += v; }
  return old;
}
static inline void __syncthreads() {}
