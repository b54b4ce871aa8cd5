// Instantiation of the batch kernel for 128-thread blocks, register-capped
// for kLeanBlocks<128> resident blocks per SM.
#include "batch_kernel.cuh"

namespace qtqp {
int launch_group_128_lean(const BatchParams& p, int smem_total, cudaStream_t stream) {
  return launch_group<128, kLeanBlocks<128>>(p, smem_total, stream);
}
}  // namespace qtqp
