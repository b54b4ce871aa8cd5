// Instantiation of the batch kernel for 32-thread blocks (free registers).
#include "batch_kernel.cuh"

namespace qtqp {
int launch_group_32(const BatchParams& p, int smem_total, cudaStream_t stream) {
  return launch_group<32, 1>(p, smem_total, stream);
}
}  // namespace qtqp
