// Batched device-resident dense IPM: one persistent launch, one thread block
// per QP at a time, QPs taken from a cost-sorted work list.
#include <algorithm>
#include <numeric>
#include <vector>

#include "dense_ipm.cuh"

namespace qtqp {

constexpr size_t kWsHeader = 256;  // work counter lives here

struct BatchParams {
  const qtqp_dense_instance* inst;
  const int32_t* order;
  int32_t count;
  const double* a_pool;
  const double* p_pool;
  const double* b_pool;
  const double* c_pool;
  double* x_pool;
  double* y_pool;
  double* s_pool;
  qtqp_result* results;
  qtqp_iter_stats* stats;
  char* ws;
  int* counter;
  qtqp_options opt;
  size_t smem_cap;
};

template <int NT>
__host__ __device__ constexpr size_t red_bytes() {
  return round16(size_t(2) * (NT / 32) * kRedMax * sizeof(double));
}

template <int NT>
__global__ void __launch_bounds__(NT) dense_batch_kernel(const BatchParams p) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  __shared__ qtqp_options sopt;
  __shared__ int next_idx;
  double* red = reinterpret_cast<double*>(smem_raw);
  char* inst_smem = reinterpret_cast<char*>(smem_raw) + red_bytes<NT>();
  if (threadIdx.x == 0) sopt = p.opt;
  __syncthreads();
  int idx = blockIdx.x;
  while (idx < p.count) {
    const int id = p.order[idx];
    const qtqp_dense_instance d = p.inst[id];
    DenseIpm<NT> s;
    s.bind(d.n, d.m, inst_smem, p.ws + d.ws_off, p.smem_cap);
    s.z = d.z;
    s.has_p = d.has_p != 0;
    s.A0 = p.a_pool + d.a_off;
    s.P0 = p.p_pool + d.p_off;
    s.b0 = p.b_pool + d.m_off;
    s.c0 = p.c_pool + d.n_off;
    s.red = red;
    s.phase = 0;
    s.o = &sopt;
    double* st = p.stats ? reinterpret_cast<double*>(p.stats + d.st_off) : nullptr;
    s.solve(p.results + id, st, p.x_pool + d.n_off, p.y_pool + d.m_off, p.s_pool + d.m_off);
    __syncthreads();
    if (threadIdx.x == 0) next_idx = atomicAdd(p.counter, 1) + int(gridDim.x);
    __syncthreads();
    idx = next_idx;
  }
}

// Cost model used for ordering: Gram SYRK + Cholesky flops.
static double inst_cost(int n, int m) { return double(m) * n * n + double(n) * n * n / 3.0; }

template <int NT>
static int launch_batch(const BatchParams& p, int smem_total, cudaStream_t stream) {
  auto kern = dense_batch_kernel<NT>;
  if (smem_total > 48 * 1024) {
    int rc = cuda_check(
        cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, smem_total),
        "cudaFuncSetAttribute");
    if (rc) return rc;
  }
  int dev = 0, sms = 0, per_sm = 0;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  int rc = cuda_check(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, NT, smem_total),
                      "cudaOccupancyMaxActiveBlocksPerMultiprocessor");
  if (rc) return rc;
  if (per_sm < 1) return fail(QTQP_ERR_BAD_ARG, "launch shape does not fit on an SM");
  const int grid = std::max(1, std::min(p.count, sms * per_sm));
  kern<<<grid, NT, smem_total, stream>>>(p);
  return cuda_check(cudaGetLastError(), "dense_batch_kernel launch");
}

}  // namespace qtqp

using namespace qtqp;

extern "C" int qtqp_dense_batch_plan(qtqp_dense_instance* h_inst, int32_t count,
                                     const qtqp_options* opt, int32_t* h_order,
                                     int32_t* block_threads, int32_t* smem_bytes,
                                     size_t* workspace_bytes) {
  if (h_inst == nullptr || h_order == nullptr || opt == nullptr || block_threads == nullptr ||
      smem_bytes == nullptr || workspace_bytes == nullptr || count < 0)
    return fail(QTQP_ERR_BAD_ARG, "qtqp_dense_batch_plan: null argument or negative count");
  int max_n = 0, max_N = 0;
  size_t max_gv = 0, max_all = 0;
  for (int i = 0; i < count; ++i) {
    const qtqp_dense_instance& d = h_inst[i];
    if (d.n < 1 || d.m < 1 || d.z < 0 || d.z >= d.m)
      return fail(QTQP_ERR_BAD_ARG, "qtqp_dense_batch_plan: instance " + std::to_string(i) +
                                        " needs n >= 1, m >= 1 and 0 <= z < m");
    max_n = std::max(max_n, d.n);
    max_N = std::max(max_N, d.n + d.m);
    const InstLayout L = plan_layout(d.n, d.m, 0);
    max_gv = std::max(max_gv, L.g_bytes + L.v_bytes);
    max_all = std::max(max_all, L.g_bytes + L.v_bytes + L.a_bytes + L.p_bytes);
  }
  int nt = *block_threads;
  if (nt == 0) nt = max_N <= 64 ? 64 : (max_N <= 384 ? 128 : 256);
  if (nt != 32 && nt != 64 && nt != 128 && nt != 256)
    return fail(QTQP_ERR_BAD_ARG, "block_threads must be 32, 64, 128 or 256");
  size_t red = nt == 32    ? red_bytes<32>()
               : nt == 64  ? red_bytes<64>()
               : nt == 128 ? red_bytes<128>()
                           : red_bytes<256>();
  size_t cap;
  if (*smem_bytes > 0) {
    if (size_t(*smem_bytes) < red)
      return fail(QTQP_ERR_BAD_ARG, "smem_bytes smaller than the reduction scratch");
    cap = size_t(*smem_bytes) - red;
  } else if (max_all + red <= 64 * 1024) {
    cap = max_all;  // everything on chip, several blocks per SM
  } else if (max_gv + red <= 200 * 1024) {
    cap = max_gv;   // G + vectors on chip, A and P through L2
  } else {
    cap = 0;        // large instance: all in the global workspace
  }
  size_t off = kWsHeader;
  for (int i = 0; i < count; ++i) {
    const InstLayout L = plan_layout(h_inst[i].n, h_inst[i].m, cap);
    h_inst[i].ws_off = int64_t(off);
    off += (L.global_bytes + 255) & ~size_t(255);
  }
  std::vector<int32_t> ord(count);
  std::iota(ord.begin(), ord.end(), 0);
  std::stable_sort(ord.begin(), ord.end(), [&](int a, int b) {
    return inst_cost(h_inst[a].n, h_inst[a].m) > inst_cost(h_inst[b].n, h_inst[b].m);
  });
  std::copy(ord.begin(), ord.end(), h_order);
  *block_threads = nt;
  *smem_bytes = int32_t(cap + red);
  *workspace_bytes = off;
  return QTQP_OK;
}

extern "C" int qtqp_dense_batch_solve(const qtqp_dense_instance* d_inst, const int32_t* d_order,
                                      int32_t count, const double* d_a_pool,
                                      const double* d_p_pool, const double* d_b_pool,
                                      const double* d_c_pool, double* d_x_pool, double* d_y_pool,
                                      double* d_s_pool, qtqp_result* d_results,
                                      qtqp_iter_stats* d_stats, void* d_workspace,
                                      size_t workspace_bytes, const qtqp_options* opt,
                                      int32_t block_threads, int32_t smem_bytes, void* stream) {
  if (count == 0) return QTQP_OK;
  if (d_inst == nullptr || d_order == nullptr || d_a_pool == nullptr || d_b_pool == nullptr ||
      d_c_pool == nullptr || d_x_pool == nullptr || d_y_pool == nullptr || d_s_pool == nullptr ||
      d_results == nullptr || d_workspace == nullptr || opt == nullptr || count < 0)
    return fail(QTQP_ERR_BAD_ARG, "qtqp_dense_batch_solve: null argument");
  if (workspace_bytes < kWsHeader)
    return fail(QTQP_ERR_BAD_ARG, "qtqp_dense_batch_solve: workspace too small");
  if (opt->max_iter < 1 || opt->max_iterative_refinement_steps < 1 ||
      !(opt->step_size_scale > 0.0 && opt->step_size_scale < 1.0))
    return fail(QTQP_ERR_BAD_ARG, "qtqp_dense_batch_solve: invalid options");
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  BatchParams p;
  p.inst = d_inst;
  p.order = d_order;
  p.count = count;
  p.a_pool = d_a_pool;
  p.p_pool = d_p_pool != nullptr ? d_p_pool : d_a_pool;
  p.b_pool = d_b_pool;
  p.c_pool = d_c_pool;
  p.x_pool = d_x_pool;
  p.y_pool = d_y_pool;
  p.s_pool = d_s_pool;
  p.results = d_results;
  p.stats = d_stats;
  p.ws = static_cast<char*>(d_workspace);
  p.counter = static_cast<int*>(d_workspace);
  p.opt = *opt;
  int rc = cuda_check(cudaMemsetAsync(d_workspace, 0, kWsHeader, st), "cudaMemsetAsync");
  if (rc) return rc;
  switch (block_threads) {
    case 32:
      p.smem_cap = size_t(smem_bytes) - red_bytes<32>();
      return launch_batch<32>(p, smem_bytes, st);
    case 64:
      p.smem_cap = size_t(smem_bytes) - red_bytes<64>();
      return launch_batch<64>(p, smem_bytes, st);
    case 128:
      p.smem_cap = size_t(smem_bytes) - red_bytes<128>();
      return launch_batch<128>(p, smem_bytes, st);
    case 256:
      p.smem_cap = size_t(smem_bytes) - red_bytes<256>();
      return launch_batch<256>(p, smem_bytes, st);
    default:
      return fail(QTQP_ERR_BAD_ARG, "block_threads must be 32, 64, 128 or 256");
  }
}
