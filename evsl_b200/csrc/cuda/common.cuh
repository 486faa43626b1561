// Shared device helpers for the sm_100a back end.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>
#include <stdio.h>

#include "../evslcu.h"

namespace evslcu {

// Library stream and bookkeeping (context.cu).
cudaStream_t stream();
int fail(int code, const char *fmt, ...);
int check_launch(const char *what);
void count_launch(uint64_t k = 1);
int sm_count();
// The device the library was started on (its stream and memory live there).
int lib_device();

// Scratch for grid-wide reductions: partial sums (one slot per block) and
// "last block" counters.  Kernels on the single library stream run one after
// another, so one scratch area serves every reduction.
constexpr int kMaxPartials = 16384;
double *partials();
unsigned int *counters();  // kNumCounters counters, all zero between kernels
double *dev_scratch_scalars();  // 64 doubles of device scalar scratch
constexpr int kNumCounters = 16;
// Slots 8-10 hold the filter grid barrier (count, generation) and its error flag.
enum CounterId { CTR_DOT = 0, CTR_NRM = 1, CTR_CHEB = 2, CTR_CGS = 3, CTR_KPM = 4, CTR_COL = 5 };

// Grid-barrier state of the single-launch filter: generation word at [0],
// top-level arrival count at [32], group arrival counts at [64 + 32 g]
// (one 128-byte line each).
constexpr int kBarrierWords = 64 + 32 * 1024;
unsigned int *barrier_area();

constexpr int kThreads = 256;

inline int grid_for(long long n, int threads = kThreads, int cap = kMaxPartials) {
  long long g = (n + threads - 1) / threads;
  if (g < 1) g = 1;
  if (g > cap) g = cap;
  return (int)g;
}

__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
  return v;
}

// Deterministic block sum (fixed tree for a fixed block size); the result is
// valid in thread 0.  `sh` must hold blockDim.x/32 doubles.
__device__ __forceinline__ double block_sum(double v, double *sh) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
  v = warp_sum(v);
  __syncthreads();
  if (lane == 0) sh[warp] = v;
  __syncthreads();
  double r = 0.0;
  if (warp == 0) {
    r = (lane < nw) ? sh[lane] : 0.0;
    r = warp_sum(r);
  }
  return r;
}

// Marks this block finished; returns true in every thread of the block that
// finished last.  The caller then reduces the partials in index order.
__device__ __forceinline__ bool last_block(unsigned int *counter) {
  __shared__ bool am_last;
  __threadfence();
  __syncthreads();
  if (threadIdx.x == 0) {
    unsigned int prev = atomicAdd(counter, 1u);
    am_last = (prev == gridDim.x * gridDim.y * gridDim.z - 1);
  }
  __syncthreads();
  return am_last;
}

// Fixed-order sum of `count` partials by one block (the last one); resets
// the counter.  Result valid in thread 0.
__device__ __forceinline__ double reduce_partials(const double *part, int count,
                                                  unsigned int *counter, double *sh) {
  double s = 0.0;
  for (int i = threadIdx.x; i < count; i += blockDim.x) s += __ldcg(part + i);
  s = block_sum(s, sh);
  if (threadIdx.x == 0) *counter = 0u;
  return s;
}

}  // namespace evslcu

#define EVSLCU_LAUNCH_CHECK(what)                            \
  do {                                                       \
    evslcu::count_launch();                                  \
    int _rc = evslcu::check_launch(what);                    \
    if (_rc) return _rc;                                     \
  } while (0)

#define EVSLCU_CUDA(call)                                                          \
  do {                                                                             \
    cudaError_t _e = (call);                                                       \
    if (_e != cudaSuccess)                                                         \
      return evslcu::fail(EVSLCU_ERR_CUDA, "%s failed: %s", #call, cudaGetErrorString(_e)); \
  } while (0)
