// Instantiation of the batch kernel for 32-thread blocks, register-capped
// for kLeanBlocks<32> resident blocks per SM.
#include "batch_kernel.cuh"

namespace qtqp {
int launch_group_32_lean(const BatchParams& p, int smem_total, cudaStream_t stream) {
  return launch_group<32, kLeanBlocks<32>>(p, smem_total, stream);
}
}  // namespace qtqp
