// Self-test of the library's bounded device waits (no reference counterpart).
//
// Every spin-wait in the kernels gives up after a poll limit, records an
// error and returns instead of hanging: the grid barrier of the whole-GPU
// solves (grid_sync: a sticky error flag, QTQP_ERR_TIMEOUT) and the mbarrier
// waits of the tensor-core pipelines (mbar_wait returns false).  This entry
// point makes one of them run out on purpose, with a short limit, so a test
// can check that the error comes back and that the GPU stays usable:
//   mode 0: a cooperative grid where one host-chosen block never reaches the
//           barrier the others wait at;
//   mode 1: a wait on an mbarrier that nothing arrives on;
//   mode 2: the per-block flags of the whole-GPU triangular solves
//           (flags_ready / flag_publish): a cooperative grid where block b
//           waits for block b - 1's flag and then publishes its own, and a
//           host-chosen block never publishes.
// Nothing faults: the waits simply stop and the kernels return.
#include "common.cuh"
#include "tc_common.cuh"

namespace qtqp {

constexpr int kSelftestThreads = 64;

__global__ void __launch_bounds__(kSelftestThreads)
    grid_wait_selftest_kernel(GridCtl* g, int skip_block, int rounds, uint32_t limit) {
  if (int(blockIdx.x) == skip_block) return;  // never arrives
  for (int r = 0; r < rounds; ++r) grid_sync(g, limit);
}

__global__ void __launch_bounds__(kSelftestThreads)
    mbar_wait_selftest_kernel(uint32_t limit, int* status) {
  __shared__ __align__(8) uint64_t bar;
  if (threadIdx.x == 0) {
    tc::mbar_init(&bar, 1);
    tc::mbar_fence_init();
  }
  __syncthreads();
  if (threadIdx.x == 0 && !tc::mbar_wait(&bar, 0, limit)) *status = QTQP_ERR_TIMEOUT;
}

__global__ void __launch_bounds__(kSelftestThreads)
    flag_wait_selftest_kernel(GridCtl* g, int skip_block, uint32_t limit) {
  const int b = blockIdx.x;
  if (b == skip_block) return;  // never publishes
  if (b > 0 && threadIdx.x < 32) flags_ready(g, b - 1, 1, b, 1u, limit);
  __syncthreads();
  if (threadIdx.x == 0) flag_publish(g, b, 1u);
}

__global__ void grid_status_kernel(const GridCtl* g, int* status) {
  *status = g->err ? QTQP_ERR_TIMEOUT : QTQP_OK;
}

}  // namespace qtqp

using namespace qtqp;

extern "C" size_t qtqp_wait_selftest_workspace_bytes(void) { return sizeof(GridCtl); }

extern "C" int qtqp_wait_selftest(int32_t mode, int32_t blocks, int32_t skip_block,
                                  uint32_t limit, void* d_workspace, int32_t* d_status,
                                  void* stream) {
  if (d_status == nullptr || limit == 0 || limit > (1u << 24))
    return fail(QTQP_ERR_BAD_ARG, "qtqp_wait_selftest: need a status pointer and a limit in "
                                  "[1, 2^24] polls");
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  if (mode == 1) {
    int rc = cuda_check(cudaMemsetAsync(d_status, 0, sizeof(int32_t), st), "cudaMemsetAsync");
    if (rc) return rc;
    mbar_wait_selftest_kernel<<<1, kSelftestThreads, 0, st>>>(limit, d_status);
    return cuda_check(cudaGetLastError(), "mbar_wait_selftest_kernel launch");
  }
  if (mode != 0 && mode != 2)
    return fail(QTQP_ERR_BAD_ARG, "qtqp_wait_selftest: mode must be 0, 1 or 2");
  if (d_workspace == nullptr || blocks < 2 || blocks > 64 || skip_block < -1 ||
      skip_block >= blocks)
    return fail(QTQP_ERR_BAD_ARG, "qtqp_wait_selftest: need a workspace, 2..64 blocks and "
                                  "skip_block in [-1, blocks)");
  int dev = 0, coop = 0, per_sm = 0, sms = 0;
  int rc = cuda_check(cudaGetDevice(&dev), "cudaGetDevice");
  if (rc) return rc;
  cudaDeviceGetAttribute(&coop, cudaDevAttrCooperativeLaunch, dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  rc = cuda_check(cudaOccupancyMaxActiveBlocksPerMultiprocessor(
                      &per_sm, grid_wait_selftest_kernel, kSelftestThreads, 0),
                  "cudaOccupancyMaxActiveBlocksPerMultiprocessor");
  if (rc) return rc;
  if (!coop || per_sm * sms < blocks)
    return fail(QTQP_ERR_BAD_ARG, "qtqp_wait_selftest: the blocks cannot all be resident");
  GridCtl* g = static_cast<GridCtl*>(d_workspace);
  rc = cuda_check(cudaMemsetAsync(g, 0, sizeof(GridCtl), st), "cudaMemsetAsync");
  if (rc) return rc;
  int skip = skip_block, rounds = 4;
  if (mode == 0) {
    void* args[] = {&g, &skip, &rounds, &limit};
    rc = cuda_check(
        cudaLaunchCooperativeKernel(reinterpret_cast<void*>(grid_wait_selftest_kernel),
                                    dim3(blocks), dim3(kSelftestThreads), args, 0, st),
        "grid_wait_selftest_kernel launch");
  } else {
    void* args[] = {&g, &skip, &limit};
    rc = cuda_check(
        cudaLaunchCooperativeKernel(reinterpret_cast<void*>(flag_wait_selftest_kernel),
                                    dim3(blocks), dim3(kSelftestThreads), args, 0, st),
        "flag_wait_selftest_kernel launch");
  }
  if (rc) return rc;
  grid_status_kernel<<<1, 1, 0, st>>>(g, d_status);
  return cuda_check(cudaGetLastError(), "grid_status_kernel launch");
}
