// One large dense QP on the whole GPU: the shared device IPM in grid mode
// (Ipm<kLargeNT, kFmtLarge>), one cooperative launch of kLargeBlocks CTAs.
#include <cudaTypedefs.h>

#include <mutex>

#include "large_ipm.cuh"

namespace qtqp {

int make_map_f32(CUtensorMap* map, const float* ptr, int rows, int cols, int ld);  // tc_gram.cu

struct LargeParams {
  int n, m, z, flags;
  const double* a;  // m x n row-major
  const double* p;  // n x n row-major (or null)
  const double* b;
  const double* c;
  double* x;
  double* y;
  double* s;
  qtqp_result* result;
  qtqp_iter_stats* stats;
  char* ws;
  qtqp_options opt;
};

__global__ void __launch_bounds__(kGridBT, 1)
    large_solve_kernel(const LargeParams p, const __grid_constant__ CUtensorMap map_hi,
                       const __grid_constant__ CUtensorMap map_lo) {
  __shared__ double red[2 * (kGridBT / 32) * kRedMax];
  __shared__ qtqp_options sopt;
  __shared__ uint32_t tmem_slot;
  extern __shared__ uint8_t dsmem[];
  uint8_t* arena = reinterpret_cast<uint8_t*>(
      (reinterpret_cast<uintptr_t>(dsmem) + 1023) & ~uintptr_t(1023));
  uint64_t* bars = reinterpret_cast<uint64_t*>(arena + kArenaBytes);
  const int warp = threadIdx.x >> 5;
  if (threadIdx.x == 0) {
    sopt = p.opt;
    for (int i = 0; i < 2 * kTcStages + 1; ++i) tc::mbar_init(&bars[i], 1);
    *reinterpret_cast<int*>(bars + 2 * kTcStages + 1) = 0;  // tensor-core failure flag
    tc::mbar_fence_init();
    tc::tma_prefetch_desc(&map_hi);
    tc::tma_prefetch_desc(&map_lo);
  }
  if (warp == 2) tc::tmem_alloc(&tmem_slot, kLB);
  tc::fence_before_sync();
  __syncthreads();
  tc::fence_after_sync();

  const LargeLayout L = plan_large_layout(p.n, p.m);
  Ipm<kLargeNT, kFmtLarge> s;
  s.tid = blockIdx.x * blockDim.x + threadIdx.x;
  s.n = p.n;
  s.m = p.m;
  s.N = p.n + p.m;
  s.z = p.z;
  s.has_p = (p.flags & QTQP_LARGE_HAS_P) != 0;
  s.colmajor = (p.flags & QTQP_LARGE_COLMAJOR) != 0;
  s.A0 = p.a;
  s.P0 = p.p;
  s.b0 = p.b;
  s.c0 = p.c;
  s.lda = p.n;
  s.ldp = p.n;
  s.ldg = L.npad;
  s.np = L.np;
  s.V = reinterpret_cast<double*>(p.ws + L.v_off);
  s.A = reinterpret_cast<double*>(p.ws + L.a_off);
  s.P = reinterpret_cast<double*>(p.ws + L.p_off);
  s.G = reinterpret_cast<double*>(p.ws + L.g64_off);
  s.gctl = reinterpret_cast<GridCtl*>(p.ws + L.ctl_off);
  s.linfo = reinterpret_cast<int*>(p.ws + L.info_off);
  s.npad = L.npad;
  s.mpad = L.mpad;
  s.g64 = reinterpret_cast<double*>(p.ws + L.g64_off);
  s.g32l = reinterpret_cast<float*>(p.ws + L.g32_off);
  s.linv = reinterpret_cast<double*>(p.ws + L.linv_off);
  s.sinv = reinterpret_cast<double*>(p.ws + L.sinv_off);
  s.xhi = reinterpret_cast<float*>(p.ws + L.xhi_off);
  s.xlo = reinterpret_cast<float*>(p.ws + L.xlo_off);
  s.colpart = reinterpret_cast<double*>(p.ws + L.cp_off);
  s.map_hi = &map_hi;
  s.map_lo = &map_lo;
  s.arena = arena;
  s.tmem = tmem_slot;
  s.tc_load = s.tc_mma = s.tc_tiles = 0;
  s.tri_gen = 0;
  s.red = red;
  s.phase = 0;
  s.o = &sopt;
  s.solve(p.result, p.stats ? reinterpret_cast<double*>(p.stats) : nullptr, p.x, p.y, p.s);

  tc::fence_before_sync();
  __syncthreads();
  if (warp == 2) {
    tc::fence_after_sync();
    tc::tmem_dealloc(tmem_slot, kLB);
  }
  if (blockIdx.x == 0 && threadIdx.x == 0 &&
      *reinterpret_cast<volatile int*>(&s.gctl->err) != 0) {
    p.result->status = QTQP_STATUS_FAILED;
    p.result->error = QTQP_ERR_TIMEOUT;
  }
}

}  // namespace qtqp

using namespace qtqp;

extern "C" int32_t qtqp_dense_large_blocks(void) { return kLargeBlocks; }

extern "C" size_t qtqp_dense_large_workspace_bytes(int32_t n, int32_t m) {
  if (n < 1 || m < 1) return 0;
  return plan_large_layout(n, m).total;
}

extern "C" int qtqp_dense_large_solve(int32_t n, int32_t m, int32_t z, int32_t flags,
                                      const double* d_a, const double* d_p, const double* d_b,
                                      const double* d_c, double* d_x, double* d_y, double* d_s,
                                      qtqp_result* d_result, qtqp_iter_stats* d_stats,
                                      void* d_workspace, size_t workspace_bytes,
                                      const qtqp_options* opt, void* stream) {
  if (n < 1 || m < 1 || z < 0 || z >= m)
    return fail(QTQP_ERR_BAD_ARG, "qtqp_dense_large_solve: needs n, m >= 1 and 0 <= z < m");
  if (flags & ~(QTQP_LARGE_HAS_P | QTQP_LARGE_COLMAJOR))
    return fail(QTQP_ERR_BAD_ARG, "qtqp_dense_large_solve: unknown flags");
  const bool has_p = (flags & QTQP_LARGE_HAS_P) != 0;
  if (n > kLB * kLargeBlocks)
    return fail(QTQP_ERR_BAD_ARG, "qtqp_dense_large_solve: n must be at most " +
                                      std::to_string(kLB * kLargeBlocks));
  if (size_t(m) * size_t(n) >= (size_t(1) << 31) || size_t(round_up(n, kLB)) * round_up(m, 32) >=
                                                        (size_t(1) << 31))
    return fail(QTQP_ERR_BAD_ARG, "qtqp_dense_large_solve: m * n must stay below 2^31");
  if (d_a == nullptr || (has_p && d_p == nullptr) || d_b == nullptr || d_c == nullptr ||
      d_x == nullptr || d_y == nullptr || d_s == nullptr || d_result == nullptr ||
      d_workspace == nullptr || opt == nullptr)
    return fail(QTQP_ERR_BAD_ARG, "qtqp_dense_large_solve: null argument");
  if (opt->max_iter < 1 || opt->max_iterative_refinement_steps < 1 ||
      !(opt->step_size_scale > 0.0 && opt->step_size_scale < 1.0))
    return fail(QTQP_ERR_BAD_ARG, "qtqp_dense_large_solve: invalid options");
  const LargeLayout L = plan_large_layout(n, m);
  if (workspace_bytes < L.total)
    return fail(QTQP_ERR_BAD_ARG, "qtqp_dense_large_solve: workspace smaller than "
                                  "qtqp_dense_large_workspace_bytes(n, m)");
  if (reinterpret_cast<uintptr_t>(d_workspace) & 1023)
    return fail(QTQP_ERR_BAD_ARG, "qtqp_dense_large_solve: workspace must be 1024-byte aligned");
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  char* ws = static_cast<char*>(d_workspace);
  int rc = cuda_check(cudaMemsetAsync(ws + L.ctl_off, 0, sizeof(GridCtl), st), "cudaMemsetAsync");
  if (rc) return rc;
  CUtensorMap mh, ml;
  rc = make_map_f32(&mh, reinterpret_cast<const float*>(ws + L.xhi_off), L.npad, L.mpad, L.mpad);
  if (rc) return rc;
  rc = make_map_f32(&ml, reinterpret_cast<const float*>(ws + L.xlo_off), L.npad, L.mpad, L.mpad);
  if (rc) return rc;
  // Set on every call: the attribute belongs to the current device.
  rc = cuda_check(cudaFuncSetAttribute(large_solve_kernel,
                                       cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       int(kLargeSmem)),
                  "cudaFuncSetAttribute(large_solve_kernel)");
  if (rc) return rc;
  int dev = 0, sms = 0, per_sm = 0, coop = 0;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  cudaDeviceGetAttribute(&coop, cudaDevAttrCooperativeLaunch, dev);
  rc = cuda_check(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, large_solve_kernel,
                                                                kGridBT, kLargeSmem),
                  "cudaOccupancyMaxActiveBlocksPerMultiprocessor");
  if (rc) return rc;
  if (!coop || per_sm * sms < kLargeBlocks)
    return fail(QTQP_ERR_CUDA, "qtqp_dense_large_solve: the device cannot hold " +
                                   std::to_string(kLargeBlocks) +
                                   " co-resident blocks of the cooperative solve");
  LargeParams p;
  p.n = n;
  p.m = m;
  p.z = z;
  p.flags = flags;
  p.a = d_a;
  p.p = has_p ? d_p : nullptr;
  p.b = d_b;
  p.c = d_c;
  p.x = d_x;
  p.y = d_y;
  p.s = d_s;
  p.result = d_result;
  p.stats = d_stats;
  p.ws = ws;
  p.opt = *opt;
  void* args[] = {&p, &mh, &ml};
  return cuda_check(cudaLaunchCooperativeKernel(reinterpret_cast<void*>(large_solve_kernel),
                                                dim3(kLargeBlocks), dim3(kGridBT), args,
                                                kLargeSmem, st),
                    "large_solve_kernel cooperative launch");
}
