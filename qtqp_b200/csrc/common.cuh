// Shared device helpers: block-wide fused reductions and error bookkeeping.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include <cstdio>
#include <string>

#include "qtqp_cuda.h"

namespace qtqp {

constexpr double kEps = 1e-15;  // src/qtqp/__init__.py:51

void set_last_error(const std::string& msg);
int fail(int code, const std::string& msg);
int cuda_check(cudaError_t err, const char* what);

// Propagates NaN like numpy's max (np.linalg.norm(.., inf) of a vector with
// a NaN is NaN); fmax would drop it.
__device__ __forceinline__ double nanmax(double a, double b) {
  return (a != a || b != b) ? __longlong_as_double(0x7ff8000000000000ll) : fmax(a, b);
}

// The IPM's heavy phases are compiled as separate device functions: each then
// gets its own register allocation, which keeps the long solve loop's live
// state from spilling into the phases' inner loops.
#define QTQP_PHASE __device__ __noinline__

// Largest number of values one fused reduction may carry.
constexpr int kRedMax = 16;

// Block-wide reduction of NS sums and NM maxima in one barrier.  Every thread
// receives the results.  `red` is shared scratch of 2 * (NT/32) * kRedMax
// doubles; `phase` alternates between its two halves so that consecutive
// reductions need a single __syncthreads each (a thread can only reach the
// reduction after next once every thread has finished reading this one,
// because the next reduction's barrier separates them).
template <int NT, int NS, int NM>
__device__ __forceinline__ void block_reduce(double (&sums)[NS > 0 ? NS : 1],
                                             double (&maxs)[NM > 0 ? NM : 1],
                                             double* red, int& phase) {
  static_assert(NS + NM <= kRedMax, "too many reduction slots");
  constexpr int NW = NT / 32;
#pragma unroll
  for (int off = 16; off > 0; off >>= 1) {
#pragma unroll
    for (int k = 0; k < NS; ++k) sums[k] += __shfl_xor_sync(0xffffffffu, sums[k], off);
#pragma unroll
    for (int k = 0; k < NM; ++k)
      maxs[k] = nanmax(maxs[k], __shfl_xor_sync(0xffffffffu, maxs[k], off));
  }
  if constexpr (NW == 1) {
    return;
  } else {
    double* buf = red + phase * (NW * kRedMax);
    phase ^= 1;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    if (lane == 0) {
#pragma unroll
      for (int k = 0; k < NS; ++k) buf[warp * kRedMax + k] = sums[k];
#pragma unroll
      for (int k = 0; k < NM; ++k) buf[warp * kRedMax + NS + k] = maxs[k];
    }
    __syncthreads();
#pragma unroll
    for (int k = 0; k < NS; ++k) {
      double acc = 0.0;
#pragma unroll
      for (int w = 0; w < NW; ++w) acc += buf[w * kRedMax + k];
      sums[k] = acc;
    }
#pragma unroll
    for (int k = 0; k < NM; ++k) {
      double acc = buf[NS + k];
#pragma unroll
      for (int w = 1; w < NW; ++w) acc = nanmax(acc, buf[w * kRedMax + NS + k]);
      maxs[k] = acc;
    }
  }
}

// A barrier for the whole group (one thread block).
template <int NT>
__device__ __forceinline__ void group_sync() {
  if constexpr (NT == 32) {
    __syncwarp();
  } else {
    __syncthreads();
  }
}

__device__ __forceinline__ uint64_t globaltimer_ns() {
  uint64_t t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}

// Optional per-phase cycle counters for profiling builds (-DQTQP_PHASE_TIMERS):
// thread 0 of each block adds the SM cycles spent in a phase to
// g_phase_cycles[phase].  Default builds compile these to nothing.
enum Phase : int {
  kPhLoad = 0, kPhNormalize, kPhGram, kPhChol, kPhSolve, kPhResidual, kPhTau, kPhStep,
  kPhTerm, kPhOther, kNumPhases
};
#ifdef QTQP_PHASE_TIMERS
extern __device__ unsigned long long g_phase_cycles[kNumPhases];
#define QTQP_TIC() long long qtqp_t0_ = clock64()
#define QTQP_RETIC() qtqp_t0_ = clock64()
#define QTQP_TOC(ph)                                                                   \
  do {                                                                                 \
    if (threadIdx.x == 0)                                                              \
      atomicAdd(&qtqp::g_phase_cycles[ph], (unsigned long long)(clock64() - qtqp_t0_)); \
  } while (0)
#else
#define QTQP_TIC() \
  do {             \
  } while (0)
#define QTQP_RETIC() \
  do {               \
  } while (0)
#define QTQP_TOC(ph) \
  do {               \
  } while (0)
#endif

}  // namespace qtqp
