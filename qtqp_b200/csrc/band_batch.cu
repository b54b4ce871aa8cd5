// Batched banded / sparse device-resident IPM: a persistent launch in which
// each thread block solves one QP at a time in its own workspace slot.
#include <algorithm>
#include <numeric>
#include <vector>

#include "dense_ipm.cuh"

namespace qtqp {

constexpr int kBandThreads = 128;
constexpr size_t kBandHeader = 256;
constexpr int kBandMaxBlocksPerSm = 8;

struct BandParams {
  const qtqp_band_instance* inst;
  const int32_t* order;
  int32_t count;
  const int32_t* ipool;
  const double* vpool;
  const double* b_pool;
  const double* c_pool;
  double* x_pool;
  double* y_pool;
  double* s_pool;
  qtqp_result* results;
  qtqp_iter_stats* stats;
  char* slots;
  size_t slot_bytes;
  int32_t num_slots;
  int* counter;
  size_t win_bytes;      // dynamic shared memory (0: no window)
  const double* warm_x;  // learned warm start (null: plain method)
  const double* warm_y;
  const unsigned char* warm_act;
  qtqp_options opt;
};

__global__ void __launch_bounds__(kBandThreads) band_batch_kernel(const BandParams p) {
  __shared__ double red[2 * (kBandThreads / 32) * kRedMax];
  extern __shared__ double bwin[];  // window of the banded factorisation (win_bytes)
  __shared__ qtqp_options sopt;
  __shared__ int next_idx;
  if (threadIdx.x == 0) sopt = p.opt;
  __syncthreads();
  if (int(blockIdx.x) >= p.num_slots) return;  // never more blocks than slots
  char* slot = p.slots + size_t(blockIdx.x) * p.slot_bytes;
  int idx = blockIdx.x;
  while (idx < p.count) {
    const int id = p.order[idx];
    const qtqp_band_instance d = p.inst[id];
    Ipm<kBandThreads, kFmtBand> s;
    s.bind_band(d.n, d.m, d.bw, d.nnz_a, d.nnz_p, slot);
    s.z = d.z;
    s.has_p = d.has_p != 0;
    s.A0 = s.P0 = nullptr;
    s.b0 = p.b_pool + d.m_off;
    s.c0 = p.c_pool + d.n_off;
    s.ip = p.ipool + d.a_ptr;
    s.ix = p.ipool + d.a_idx;
    s.av0 = p.vpool + d.a_val;
    s.jp = p.ipool + d.at_ptr;
    s.jx = p.ipool + d.at_idx;
    s.at0 = p.vpool + d.at_val;
    s.pp = p.ipool + d.p_ptr;
    s.px = p.ipool + d.p_idx;
    s.pv0 = p.vpool + d.p_val;
    s.red = red;
    s.phase = 0;
    s.o = &sopt;
    s.bwin = (p.win_bytes > 0 && d.bw <= kBandWinMaxBw &&
              band_win_bytes(d.bw, kBandThreads) <= p.win_bytes)
                 ? bwin
                 : nullptr;
    double* st = p.stats ? reinterpret_cast<double*>(p.stats + d.st_off) : nullptr;
    if (p.warm_act != nullptr) {
      s.solve(p.results + id, st, p.x_pool + d.n_off, p.y_pool + d.m_off, p.s_pool + d.m_off,
              p.warm_x + d.n_off, p.warm_y + d.m_off, p.warm_act + d.m_off);
    } else {
      s.solve(p.results + id, st, p.x_pool + d.n_off, p.y_pool + d.m_off, p.s_pool + d.m_off);
    }
    __syncthreads();
    if (threadIdx.x == 0) next_idx = atomicAdd(p.counter, 1) + p.num_slots;
    __syncthreads();
    idx = next_idx;
  }
}

static double band_cost(const qtqp_band_instance& d) {
  return double(d.n) * (d.bw + 1) * (d.bw + 1) + 4.0 * d.nnz_a;
}

}  // namespace qtqp

using namespace qtqp;

extern "C" int qtqp_band_batch_plan(qtqp_band_instance* h_inst, int32_t count,
                                    const qtqp_options* opt, int32_t num_sms, int32_t* h_order,
                                    qtqp_batch_plan* plan) {
  if (h_inst == nullptr || h_order == nullptr || opt == nullptr || plan == nullptr || count < 0)
    return fail(QTQP_ERR_BAD_ARG, "qtqp_band_batch_plan: null argument or negative count");
  size_t slot = 0;
  for (int i = 0; i < count; ++i) {
    const qtqp_band_instance& d = h_inst[i];
    if (d.n < 1 || d.m < 1 || d.z < 0 || d.z >= d.m || d.bw < 0 || d.bw >= d.n ||
        d.nnz_a < 0 || d.nnz_p < 0)
      return fail(QTQP_ERR_BAD_ARG, "qtqp_band_batch_plan: instance " + std::to_string(i) +
                                        " needs n, m >= 1, 0 <= z < m, 0 <= bw < n");
    const BandLayout L = plan_band_layout(d.n, d.m, d.bw, d.nnz_a, d.nnz_p);
    slot = std::max(slot, (L.total + 255) & ~size_t(255));
  }
  std::vector<int32_t> ord(count);
  std::iota(ord.begin(), ord.end(), 0);
  std::stable_sort(ord.begin(), ord.end(),
                   [&](int a, int b) { return band_cost(h_inst[a]) > band_cost(h_inst[b]); });
  std::copy(ord.begin(), ord.end(), h_order);
  const int sms = num_sms > 0 ? num_sms : 148;
  const int slots = std::max(1, std::min(count, sms * kBandMaxBlocksPerSm));
  size_t win = 0;  // the widest band that still fits the shared-memory window
  for (int i = 0; i < count; ++i)
    if (h_inst[i].bw <= kBandWinMaxBw)
      win = std::max(win, band_win_bytes(std::min(h_inst[i].bw, h_inst[i].n - 1), kBandThreads));
  *plan = qtqp_batch_plan{};
  if (count == 0) return QTQP_OK;
  plan->num_groups = 1;
  qtqp_launch_group& g = plan->groups[0];
  g.begin = 0;
  g.count = count;
  g.block_threads = kBandThreads;
  g.smem_bytes = int32_t(win);
  g.slots = slots;
  g.slot_off = kBandHeader;
  g.slot_bytes = slot;
  plan->workspace_bytes = kBandHeader + size_t(slots) * slot;
  return QTQP_OK;
}

extern "C" int qtqp_band_batch_solve(const qtqp_band_instance* d_inst, const int32_t* d_order,
                                     const qtqp_batch_plan* plan, const int32_t* d_ipool,
                                     const double* d_vpool, const double* d_b_pool,
                                     const double* d_c_pool, double* d_x_pool, double* d_y_pool,
                                     double* d_s_pool, qtqp_result* d_results,
                                     qtqp_iter_stats* d_stats, void* d_workspace,
                                     size_t workspace_bytes, const qtqp_options* opt,
                                     const double* d_warm_x, const double* d_warm_y,
                                     const uint8_t* d_warm_active, void* stream) {
  if (plan == nullptr || opt == nullptr)
    return fail(QTQP_ERR_BAD_ARG, "qtqp_band_batch_solve: null plan/options");
  if (plan->num_groups == 0) return QTQP_OK;
  if (plan->num_groups != 1)
    return fail(QTQP_ERR_BAD_ARG, "qtqp_band_batch_solve: plan must have one group");
  if (d_inst == nullptr || d_order == nullptr || d_ipool == nullptr || d_vpool == nullptr ||
      d_b_pool == nullptr || d_c_pool == nullptr || d_x_pool == nullptr || d_y_pool == nullptr ||
      d_s_pool == nullptr || d_results == nullptr || d_workspace == nullptr)
    return fail(QTQP_ERR_BAD_ARG, "qtqp_band_batch_solve: null argument");
  const qtqp_launch_group& G = plan->groups[0];
  if (G.slots < 1 || workspace_bytes < plan->workspace_bytes ||
      plan->workspace_bytes < G.slot_off + size_t(G.slots) * G.slot_bytes)
    return fail(QTQP_ERR_BAD_ARG, "qtqp_band_batch_solve: workspace smaller than the plan's");
  if (opt->max_iter < 1 || opt->max_iterative_refinement_steps < 1 ||
      !(opt->step_size_scale > 0.0 && opt->step_size_scale < 1.0))
    return fail(QTQP_ERR_BAD_ARG, "qtqp_band_batch_solve: invalid options");
  if (d_warm_active != nullptr && (d_warm_x == nullptr || d_warm_y == nullptr))
    return fail(QTQP_ERR_BAD_ARG, "qtqp_band_batch_solve: warm start needs x, y and active");
  if (opt->warm_corrections < 0 || opt->warm_corrections > 64)
    return fail(QTQP_ERR_BAD_ARG, "qtqp_band_batch_solve: warm_corrections must be in [0, 64]");
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  int rc = cuda_check(cudaMemsetAsync(d_workspace, 0, kBandHeader, st), "cudaMemsetAsync");
  if (rc) return rc;
  int dev = 0, sms = 0, per_sm = 0;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  const size_t win = size_t(std::max(G.smem_bytes, 0));
  rc = cuda_check(cudaFuncSetAttribute(band_batch_kernel,
                                       cudaFuncAttributeMaxDynamicSharedMemorySize, int(win)),
                  "cudaFuncSetAttribute(band_batch_kernel)");
  if (rc) return rc;
  rc = cuda_check(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, band_batch_kernel,
                                                                kBandThreads, win),
                  "cudaOccupancyMaxActiveBlocksPerMultiprocessor");
  if (rc) return rc;
  BandParams p;
  p.inst = d_inst;
  p.order = d_order;
  p.count = G.count;
  p.ipool = d_ipool;
  p.vpool = d_vpool;
  p.b_pool = d_b_pool;
  p.c_pool = d_c_pool;
  p.x_pool = d_x_pool;
  p.y_pool = d_y_pool;
  p.s_pool = d_s_pool;
  p.results = d_results;
  p.stats = d_stats;
  p.slots = static_cast<char*>(d_workspace) + G.slot_off;
  p.slot_bytes = G.slot_bytes;
  p.counter = static_cast<int*>(d_workspace);
  p.win_bytes = win;
  p.warm_x = d_warm_x;
  p.warm_y = d_warm_y;
  p.warm_act = d_warm_active;
  p.opt = *opt;
  const int grid = std::max(1, std::min({G.count, G.slots, sms * std::max(per_sm, 1)}));
  p.num_slots = grid;
  band_batch_kernel<<<grid, kBandThreads, win, st>>>(p);
  return cuda_check(cudaGetLastError(), "band_batch_kernel launch");
}
