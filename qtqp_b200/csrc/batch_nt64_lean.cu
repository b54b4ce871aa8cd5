// Instantiation of the batch kernel for 64-thread blocks, register-capped
// for kLeanBlocks<64> resident blocks per SM.
#include "batch_kernel.cuh"

namespace qtqp {
int launch_group_64_lean(const BatchParams& p, int smem_total, cudaStream_t stream) {
  return launch_group<64, kLeanBlocks<64>>(p, smem_total, stream);
}
}  // namespace qtqp
