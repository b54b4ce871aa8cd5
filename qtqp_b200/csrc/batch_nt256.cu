// Instantiation of the batch kernel for 256-thread blocks (free registers).
#include "batch_kernel.cuh"

namespace qtqp {
int launch_group_256(const BatchParams& p, int smem_total, cudaStream_t stream) {
  return launch_group<256, 1>(p, smem_total, stream);
}
}  // namespace qtqp
