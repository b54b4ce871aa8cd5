// Instantiation of the batch kernel for one-warp blocks (one QP per warp).
#include "batch_kernel.cuh"

namespace qtqp {
int launch_group_32(const BatchParams& p, int smem_total, cudaStream_t stream) {
  return launch_group<32>(p, smem_total, stream);
}
}  // namespace qtqp
