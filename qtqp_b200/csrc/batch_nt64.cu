// Instantiation of the batch kernel for 64-thread blocks.
#include "batch_kernel.cuh"

namespace qtqp {
int launch_group_64(const BatchParams& p, int smem_total, cudaStream_t stream) {
  return launch_group<64>(p, smem_total, stream);
}
}  // namespace qtqp
