// Instantiation of the batch kernel for 256-thread blocks, register-capped
// for kLeanBlocks<256> resident blocks per SM.
#include "batch_kernel.cuh"

namespace qtqp {
int launch_group_256_lean(const BatchParams& p, int smem_total, cudaStream_t stream) {
  return launch_group<256, kLeanBlocks<256>>(p, smem_total, stream);
}
}  // namespace qtqp
