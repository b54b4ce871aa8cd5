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
  // The loops over shuffle distances and warps stay rolled (the values of
  // one step unrolled): every reduction of the IPM is inlined at its call
  // site, and fully unrolled they made up much of the per-iteration code
  // that competes for the instruction cache.  The order of the operations
  // is the same either way.
#pragma unroll 1
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
    for (int k = 0; k < NS; ++k) sums[k] = 0.0;
#pragma unroll
    for (int k = 0; k < NM; ++k) maxs[k] = buf[NS + k];
#pragma unroll 1
    for (int w = 0; w < NW; ++w) {
#pragma unroll
      for (int k = 0; k < NS; ++k) sums[k] += buf[w * kRedMax + k];
      if (w > 0) {
#pragma unroll
        for (int k = 0; k < NM; ++k) maxs[k] = nanmax(maxs[k], buf[w * kRedMax + NS + k]);
      }
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

// ----------------------------------------------------------------------------
// Grid-wide barrier and reductions of a cooperative launch (every block
// resident), for one large QP solved by the whole GPU.  The barrier is a
// generation counter in global memory; a wait that exceeds kGridWaitLimit
// polls sets the sticky `err` flag, after which every barrier returns at once
// (the solve then finishes its bounded loops and reports the error).
// ----------------------------------------------------------------------------
constexpr int kGridMaxBlocks = 256;
constexpr int kGridBT = 256;  // threads per block of a grid-mode solve
// Supernodal factorisation: the widest supernode (its diagonal block stays in
// shared memory) and the rows of a top-level supernode per work item.  Both
// the host symbolic stage and the device phases use them.
constexpr int kSnMaxWidth = 64;
constexpr int kSnSlabRows = 64;
constexpr uint32_t kGridWaitLimit = 1u << 25;

struct GridCtl {
  unsigned int count;  // arrivals in the current generation
  unsigned int gen;    // completed barriers
  int err;             // 1: a barrier or flag wait gave up
  int pad;
  unsigned int flag[kGridMaxBlocks];        // per-block publication flags (flags_ready)
  double part[2][kGridMaxBlocks][kRedMax];  // per-block partials (double-buffered)
};

__device__ __forceinline__ void grid_sync(GridCtl* g, uint32_t limit = kGridWaitLimit) {
  __syncthreads();
  if (threadIdx.x == 0) {
    volatile GridCtl* vg = g;
    if (!vg->err) {
      const unsigned int gen = vg->gen;
      __threadfence();
      const unsigned int arrived = atomicAdd(&g->count, 1u) + 1u;
      if (arrived == gridDim.x) {
        atomicExch(&g->count, 0u);
        __threadfence();
        atomicAdd(&g->gen, 1u);
      } else {
        uint32_t it = 0;
        while (vg->gen == gen && !vg->err) {
          if (++it > limit) {
            atomicExch(&g->err, 1);
            break;
          }
          __nanosleep(64);
        }
      }
      __threadfence();
    }
  }
  __syncthreads();
}

// Point-to-point hand-off between the blocks of a cooperative grid.  Block c
// publishes a result by writing it, fencing, and storing a generation number
// to flag[c] with release semantics (flag_publish); a consumer's warp polls
// the flags with acquire loads (flags_ready).  Generations only grow within a
// launch and the flags start at zero with the rest of GridCtl, so a flag is
// never reset.  A wait that exceeds `limit` polls sets the sticky err flag;
// every later wait then returns at once, as grid_sync does.
__device__ __forceinline__ unsigned int ld_acquire_gpu(const unsigned int* p) {
  unsigned int v;
  asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
  return v;
}
__device__ __forceinline__ void st_release_gpu(unsigned int* p, unsigned int v) {
  asm volatile("st.release.gpu.global.u32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}

// Called by one whole warp.  Looks at flag[c], flag[c + dir], ... (up to 32
// of them, stopping before index `end`, dir = +1 or -1) and returns how many
// consecutive ones, starting at c, have reached `gen`; waits (bounded) until
// that is at least one.  Returns 0 only when the wait gave up or an earlier
// wait had (err set).  Every lane returns the same value.
__device__ __forceinline__ int flags_ready(GridCtl* g, int c, int dir, int end, unsigned int gen,
                                           uint32_t limit = kGridWaitLimit) {
  const int lane = threadIdx.x & 31;
  const int i = c + dir * lane;
  const bool in = dir > 0 ? i < end : i > end;
  for (uint32_t it = 0;; ++it) {
    const bool ok = in && ld_acquire_gpu(&g->flag[i]) >= gen;
    const unsigned int mask = __ballot_sync(0xffffffffu, ok);
    if (mask & 1u) return mask == 0xffffffffu ? 32 : __ffs(~mask) - 1;
    int err = lane == 0 ? *reinterpret_cast<volatile int*>(&g->err) : 0;
    err = __shfl_sync(0xffffffffu, err, 0);
    if (err) return 0;
    if (it >= limit) {
      if (lane == 0) atomicExch(&g->err, 1);
      return 0;
    }
    if (it >= 256) __nanosleep(64);  // each poll is an L2 round trip; back off later
  }
}

// Called by thread 0 after a __syncthreads that follows the block's writes
// (each writing thread fenced its own stores with __threadfence()).
__device__ __forceinline__ void flag_publish(GridCtl* g, int c, unsigned int gen) {
  st_release_gpu(&g->flag[c], gen);
}

// NS sums and NM maxima over every thread of the grid; all threads receive
// the same values (the partials are combined in one fixed order in every
// block, so control flow that depends on them agrees across blocks).  `red`
// is shared scratch of 2 * (blockDim.x / 32) * kRedMax doubles; `phase`
// alternates the global partial buffers (see block_reduce).
template <int BT, int NS, int NM>
__device__ __forceinline__ void grid_reduce(double (&sums)[NS > 0 ? NS : 1],
                                            double (&maxs)[NM > 0 ? NM : 1], double* red,
                                            GridCtl* g, int& phase) {
  static_assert(NS + NM <= kRedMax, "too many reduction slots");
  constexpr int NW = BT / 32;
#pragma unroll
  for (int off = 16; off > 0; off >>= 1) {
#pragma unroll
    for (int k = 0; k < NS; ++k) sums[k] += __shfl_xor_sync(0xffffffffu, sums[k], off);
#pragma unroll
    for (int k = 0; k < NM; ++k)
      maxs[k] = nanmax(maxs[k], __shfl_xor_sync(0xffffffffu, maxs[k], off));
  }
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  double* wbuf = red;                // NW x kRedMax warp partials
  double* res = red + NW * kRedMax;  // kRedMax results
  if (lane == 0) {
#pragma unroll
    for (int k = 0; k < NS; ++k) wbuf[warp * kRedMax + k] = sums[k];
#pragma unroll
    for (int k = 0; k < NM; ++k) wbuf[warp * kRedMax + NS + k] = maxs[k];
  }
  __syncthreads();
  double* part = &g->part[phase][0][0];
  phase ^= 1;
  if (threadIdx.x == 0) {
#pragma unroll
    for (int k = 0; k < NS; ++k) {
      double acc = 0.0;
      for (int w = 0; w < NW; ++w) acc += wbuf[w * kRedMax + k];
      part[blockIdx.x * kRedMax + k] = acc;
    }
#pragma unroll
    for (int k = 0; k < NM; ++k) {
      double acc = wbuf[NS + k];
      for (int w = 1; w < NW; ++w) acc = nanmax(acc, wbuf[w * kRedMax + NS + k]);
      part[blockIdx.x * kRedMax + NS + k] = acc;
    }
  }
  grid_sync(g);
  if (warp == 0) {
    const int nb = gridDim.x;
#pragma unroll
    for (int k = 0; k < NS; ++k) {
      double acc = 0.0;
      for (int b = lane; b < nb; b += 32) acc += part[b * kRedMax + k];
      for (int off = 16; off > 0; off >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, off);
      if (lane == 0) res[k] = acc;
    }
#pragma unroll
    for (int k = 0; k < NM; ++k) {
      double acc = part[NS + k];  // block 0's partial starts every lane
      for (int b = lane; b < nb; b += 32) acc = nanmax(acc, part[b * kRedMax + NS + k]);
      for (int off = 16; off > 0; off >>= 1)
        acc = nanmax(acc, __shfl_xor_sync(0xffffffffu, acc, off));
      if (lane == 0) res[NS + k] = acc;
    }
  }
  __syncthreads();
#pragma unroll
  for (int k = 0; k < NS; ++k) sums[k] = res[k];
#pragma unroll
  for (int k = 0; k < NM; ++k) maxs[k] = res[NS + k];
}

// Asynchronous global -> shared copies (cp.async): 8 bytes (zero-filled
// when !valid) or 4 bytes; commit a group; wait until at most N groups of
// this thread are in flight.
__device__ __forceinline__ void cp_async8(void* dst, const void* src, bool valid) {
  asm volatile("cp.async.ca.shared.global [%0], [%1], 8, %2;" ::"r"(static_cast<uint32_t>(__cvta_generic_to_shared(dst))),
               "l"(src), "r"(valid ? 8 : 0)
               : "memory");
}
__device__ __forceinline__ void cp_async_commit() {
  asm volatile("cp.async.commit_group;" ::: "memory");
}
__device__ __forceinline__ void cp_async4z(void* dst, const void* src, bool valid) {
  asm volatile("cp.async.ca.shared.global [%0], [%1], 4, %2;" ::"r"(
                   static_cast<uint32_t>(__cvta_generic_to_shared(dst))),
               "l"(src), "r"(valid ? 4 : 0)
               : "memory");
}
// Element copy of T (double or float), zero-filled when !valid.
template <typename T>
__device__ __forceinline__ void cp_async_elem(T* dst, const T* src, bool valid) {
  if constexpr (sizeof(T) == 8) {
    cp_async8(dst, src, valid);
  } else {
    cp_async4z(dst, src, valid);
  }
}
__device__ __forceinline__ void cp_async4(void* dst, const void* src) {
  asm volatile("cp.async.ca.shared.global [%0], [%1], 4;" ::"r"(static_cast<uint32_t>(__cvta_generic_to_shared(dst))), "l"(src)
               : "memory");
}
template <int N>
__device__ __forceinline__ void cp_async_wait() {
  asm volatile("cp.async.wait_group %0;" ::"n"(N) : "memory");
}


// One FP64 tensor-core step d += a b (mma.sync m8n8k4, row.col; tcgen05 has
// no FP64 kind): lane l holds a = A[l/4][l%4], b = B[l%4][l/4] and the
// accumulator entries (l/4, 2 (l%4)) and (l/4, 2 (l%4) + 1).
__device__ __forceinline__ void dmma_8x8x4(double (&d)[2], double a, double b) {
  asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0, %1}, {%2}, {%3}, {%0, %1};"
               : "+d"(d[0]), "+d"(d[1])
               : "d"(a), "d"(b));
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
  kPhTerm, kPhOther,
  // Sub-phases of the large (grid-mode) factorisation and solves.
  kPhLgDiag, kPhLgPanel, kPhLgTrail, kPhLgInv, kPhLgFwd, kPhLgBwd,
  // Sub-phases of the partitioned banded factorisation and solves.
  kPhBpInterior, kPhBpChain, kPhBpFwd, kPhBpChains, kPhBpBwd,
  // Steps of one reduction level (per participating block).
  kPhBpCrStage, kPhBpCrSweep, kPhBpCrGemm, kPhBpCrGather,
  // Sub-phases of the supernodal factorisation and solves (subtrees / top levels).
  kPhSnSub, kPhSnTop, kPhSnFwdSub, kPhSnFwdTop, kPhSnBwdTop, kPhSnBwdSub,
  kPhSnTopUpd, kPhSnTopDiag, kPhSnTopPanel,
  // Sub-phases of the dense KKT solve: the column sums A^T (r_y / Ry) and the
  // row products A x around the triangular solves.
  kPhSolveCols, kPhSolveRows,
  // Sub-phases of the per-block dense format: the inverse of the factor's
  // 32 x 32 diagonal blocks and the triangular solves of a KKT solve.
  kPhInv, kPhTri, kNumPhases
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
