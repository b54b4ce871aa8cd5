// The persistent batch kernel and its launcher, shared by the per-block-size
// translation units (batch_nt*.cu) so that they compile in parallel.
#pragma once

#include <algorithm>

#include "dense_ipm.cuh"

namespace qtqp {

constexpr size_t kWsHeader = 256;                 // one work counter per group
constexpr size_t kSmemPerSm = 228 * 1024;         // B200 shared memory per SM
constexpr size_t kSmemBlockMax = 227 * 1024 - 512;  // dynamic part of one block
constexpr size_t kSmemReserved = 1024;            // per-block system reservation

struct BatchParams {
  const qtqp_dense_instance* inst;
  const int32_t* order;
  int32_t count;
  const double* a_pool;
  const double* p_pool;
  const double* b_pool;
  const double* c_pool;
  double* x_pool;
  double* y_pool;
  double* s_pool;
  qtqp_result* results;
  qtqp_iter_stats* stats;
  char* ws;
  int* counter;
  qtqp_options opt;
  size_t smem_cap;
  const double* x0_pool;  // starting points laid out like x / y / s (or null)
  const double* y0_pool;
  const double* s0_pool;
};

template <int NT>
__host__ __device__ constexpr size_t red_bytes() {
  return round16(size_t(2) * (NT / 32) * kRedMax * sizeof(double));
}

inline size_t red_bytes_rt(int nt) {
  switch (nt) {
    case 32: return red_bytes<32>();
    case 64: return red_bytes<64>();
    case 128: return red_bytes<128>();
    default: return red_bytes<256>();
  }
}

// Each block size is compiled twice: MINB = 1 leaves the register count free
// (fewest spills, fewest resident blocks), the lean variant asks the
// compiler for kLeanBlocks<NT> resident blocks per SM (registers capped at
// 64K / (NT * MINB), more warps in flight).  The launch group's `lean` field
// picks one; the autotuner times both.
#ifdef QTQP_PHASE_TIMERS
// Profiling builds use relocatable device code, where a phase function is
// compiled once for every kernel that calls it: no register-capped variant.
template <int NT>
constexpr int kLeanBlocks = 1;
#else
template <int NT>
constexpr int kLeanBlocks = NT >= 256 ? 2 : (NT >= 128 ? 3 : (NT >= 64 ? 6 : 12));
#endif

template <int NT, int MINB>
__global__ void __launch_bounds__(NT, MINB) dense_batch_kernel(const BatchParams p) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  __shared__ qtqp_options sopt;
  __shared__ int next_idx;
  double* red = reinterpret_cast<double*>(smem_raw);
  char* inst_smem = reinterpret_cast<char*>(smem_raw) + red_bytes<NT>();
  if (threadIdx.x == 0) sopt = p.opt;
  __syncthreads();
  int idx = blockIdx.x;
  while (idx < p.count) {
    const int id = p.order[idx];
    const qtqp_dense_instance d = p.inst[id];
    DenseIpm<NT> s;
    s.bind(d.n, d.m, inst_smem, p.ws + d.ws_off, p.smem_cap);
    s.z = d.z;
    s.has_p = d.has_p != 0;
    s.A0 = p.a_pool + d.a_off;
    s.P0 = p.p_pool + d.p_off;
    s.colmajor = true;  // batch pools hold A and P column-major
    s.b0 = p.b_pool + d.m_off;
    s.c0 = p.c_pool + d.n_off;
    s.red = red;
    s.phase = 0;
    s.o = &sopt;
    double* st = p.stats ? reinterpret_cast<double*>(p.stats + d.st_off) : nullptr;
    if (p.x0_pool != nullptr) {
      s.solve(p.results + id, st, p.x_pool + d.n_off, p.y_pool + d.m_off, p.s_pool + d.m_off,
              nullptr, nullptr, nullptr, p.x0_pool + d.n_off, p.y0_pool + d.m_off,
              p.s0_pool + d.m_off);
    } else {
      s.solve(p.results + id, st, p.x_pool + d.n_off, p.y_pool + d.m_off, p.s_pool + d.m_off);
    }
    __syncthreads();
    if (threadIdx.x == 0) next_idx = atomicAdd(p.counter, 1) + int(gridDim.x);
    __syncthreads();
    idx = next_idx;
  }
}

// Cost model used for ordering: Gram SYRK + Cholesky flops.
inline double inst_cost(int n, int m) { return double(m) * n * n + double(n) * n * n / 3.0; }

template <int NT, int MINB>
inline int launch_group(const BatchParams& p, int smem_total, cudaStream_t stream) {
  auto kern = dense_batch_kernel<NT, MINB>;
  int rc = cuda_check(
      cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, smem_total),
      "cudaFuncSetAttribute");
  if (rc) return rc;
  int dev = 0, sms = 0, per_sm = 0;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  rc = cuda_check(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, NT, smem_total),
                  "cudaOccupancyMaxActiveBlocksPerMultiprocessor");
  if (rc) return rc;
  if (per_sm < 1) return fail(QTQP_ERR_BAD_ARG, "launch shape does not fit on an SM");
  const int grid = std::max(1, std::min(p.count, sms * per_sm));
  kern<<<grid, NT, smem_total, stream>>>(p);
  return cuda_check(cudaGetLastError(), "dense_batch_kernel launch");
}


// One per translation unit (batch_nt*.cu), so that they compile in parallel;
// lean != 0 selects the register-capped variant.
int launch_group_32(const BatchParams& p, int smem_total, cudaStream_t stream);
int launch_group_64(const BatchParams& p, int smem_total, cudaStream_t stream);
int launch_group_128(const BatchParams& p, int smem_total, cudaStream_t stream);
int launch_group_256(const BatchParams& p, int smem_total, cudaStream_t stream);
int launch_group_32_lean(const BatchParams& p, int smem_total, cudaStream_t stream);
int launch_group_64_lean(const BatchParams& p, int smem_total, cudaStream_t stream);
int launch_group_128_lean(const BatchParams& p, int smem_total, cudaStream_t stream);
int launch_group_256_lean(const BatchParams& p, int smem_total, cudaStream_t stream);

}  // namespace qtqp
