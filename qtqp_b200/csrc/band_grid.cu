// One large banded QP on the whole GPU: the shared device IPM in grid mode
// (Ipm<kBandGridNT, kFmtBand>) with the partitioned band factorisation of
// band_grid.cuh, one cooperative launch of kBandGridBlocks blocks.
#include <algorithm>

#include "band_grid.cuh"

namespace qtqp {

struct BandGridParams {
  qtqp_band_instance d;
  int parts;
  const int32_t* ipool;
  const double* vpool;
  const double* b_pool;
  const double* c_pool;
  double* x_pool;
  double* y_pool;
  double* s_pool;
  qtqp_result* result;
  qtqp_iter_stats* stats;
  char* ws;
  size_t smem;
  qtqp_options opt;
};

__global__ void __launch_bounds__(kGridBT, 1) band_grid_kernel(const BandGridParams p) {
  __shared__ double red[2 * (kGridBT / 32) * kRedMax];
  __shared__ qtqp_options sopt;
  extern __shared__ double bwin[];
  if (threadIdx.x == 0) sopt = p.opt;
  __syncthreads();
  const qtqp_band_instance& d = p.d;
  const BandGridLayout L = plan_band_grid_layout(d.n, d.m, d.bw, d.nnz_a, d.nnz_p, p.parts);
  Ipm<kBandGridNT, kFmtBand> s;
  s.bind_band(d.n, d.m, d.bw, d.nnz_a, d.nnz_p, p.ws + L.band_off);
  s.tid = blockIdx.x * blockDim.x + threadIdx.x;
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
  s.gctl = reinterpret_cast<GridCtl*>(p.ws + L.ctl_off);
  s.linfo = reinterpret_cast<int*>(p.ws + L.info_off);
  s.nparts = p.parts;
  s.bp_wl = reinterpret_cast<double*>(p.ws + L.wl_off);
  s.bp_sep = reinterpret_cast<double*>(p.ws + L.sep_off);
  s.bp_vec = reinterpret_cast<double*>(p.ws + L.vec_off);
  s.bwin = bwin;
  s.bwin_bytes = p.smem;
  s.red = red;
  s.phase = 0;
  s.o = &sopt;
  s.solve(p.result, p.stats ? reinterpret_cast<double*>(p.stats) : nullptr,
          p.x_pool + d.n_off, p.y_pool + d.m_off, p.s_pool + d.m_off);
  if (blockIdx.x == 0 && threadIdx.x == 0 &&
      *reinterpret_cast<volatile int*>(&s.gctl->err) != 0) {
    p.result->status = QTQP_STATUS_FAILED;
    p.result->error = QTQP_ERR_TIMEOUT;
  }
}

static int check_inst(const qtqp_band_instance* h, int parts, const char* who) {
  if (h == nullptr) return fail(QTQP_ERR_BAD_ARG, std::string(who) + ": null instance");
  const qtqp_band_instance& d = *h;
  if (d.n < 2 || d.m < 1 || d.z < 0 || d.z >= d.m || d.bw < 1 || d.bw >= d.n ||
      d.nnz_a < 0 || d.nnz_p < 0)
    return fail(QTQP_ERR_BAD_ARG, std::string(who) + ": needs n >= 2, m >= 1, 0 <= z < m, "
                                                     "1 <= bw < n");
  if (d.bw > kBandWinMaxBw || band_grid_smem_need(d.bw) > kBandGridSmemCap)
    return fail(QTQP_ERR_BAD_ARG, std::string(who) + ": half-bandwidth " + std::to_string(d.bw) +
                                      " is too wide for the partitioned factorisation");
  if (parts < 1 || parts > kBandGridBlocks || parts > band_grid_max_parts(d.n, d.bw))
    return fail(QTQP_ERR_BAD_ARG,
                std::string(who) + ": parts must be in [1, " +
                    std::to_string(std::min(kBandGridBlocks, band_grid_max_parts(d.n, d.bw))) +
                    "] (every interior at least bw columns, at most one per block)");
  return QTQP_OK;
}

}  // namespace qtqp

using namespace qtqp;

extern "C" int32_t qtqp_band_grid_default_parts(const qtqp_band_instance* h_inst) {
  if (h_inst == nullptr || h_inst->bw < 1 || h_inst->n < 2) return 1;
  // The separators are reduced in log2(parts) parallel levels, so the most
  // partitions (the shortest interiors) are the fastest: one per block, as
  // far as every interior stays at least bw long.
  return std::max(1, std::min(kBandGridBlocks, band_grid_max_parts(h_inst->n, h_inst->bw)));
}

extern "C" size_t qtqp_band_grid_workspace_bytes(const qtqp_band_instance* h_inst, int32_t parts) {
  if (check_inst(h_inst, parts, "qtqp_band_grid_workspace_bytes") != QTQP_OK) return 0;
  const qtqp_band_instance& d = *h_inst;
  return plan_band_grid_layout(d.n, d.m, d.bw, d.nnz_a, d.nnz_p, parts).total;
}

extern "C" int qtqp_band_grid_solve(const qtqp_band_instance* h_inst, int32_t parts,
                                    const int32_t* d_ipool, const double* d_vpool,
                                    const double* d_b_pool, const double* d_c_pool,
                                    double* d_x_pool, double* d_y_pool, double* d_s_pool,
                                    qtqp_result* d_result, qtqp_iter_stats* d_stats,
                                    void* d_workspace, size_t workspace_bytes,
                                    const qtqp_options* opt, void* stream) {
  int rc = check_inst(h_inst, parts, "qtqp_band_grid_solve");
  if (rc) return rc;
  if (d_ipool == nullptr || d_vpool == nullptr || d_b_pool == nullptr || d_c_pool == nullptr ||
      d_x_pool == nullptr || d_y_pool == nullptr || d_s_pool == nullptr || d_result == nullptr ||
      d_workspace == nullptr || opt == nullptr)
    return fail(QTQP_ERR_BAD_ARG, "qtqp_band_grid_solve: null argument");
  if (opt->max_iter < 1 || opt->max_iterative_refinement_steps < 1 ||
      !(opt->step_size_scale > 0.0 && opt->step_size_scale < 1.0))
    return fail(QTQP_ERR_BAD_ARG, "qtqp_band_grid_solve: invalid options");
  const qtqp_band_instance& d = *h_inst;
  const BandGridLayout L = plan_band_grid_layout(d.n, d.m, d.bw, d.nnz_a, d.nnz_p, parts);
  if (workspace_bytes < L.total)
    return fail(QTQP_ERR_BAD_ARG, "qtqp_band_grid_solve: workspace smaller than "
                                  "qtqp_band_grid_workspace_bytes(inst, parts)");
  if (reinterpret_cast<uintptr_t>(d_workspace) & 255)
    return fail(QTQP_ERR_BAD_ARG, "qtqp_band_grid_solve: workspace must be 256-byte aligned");
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  char* ws = static_cast<char*>(d_workspace);
  rc = cuda_check(cudaMemsetAsync(ws + L.ctl_off, 0, sizeof(GridCtl), st), "cudaMemsetAsync");
  if (rc) return rc;
  const size_t smem = band_grid_smem_bytes(d.bw);
  rc = cuda_check(cudaFuncSetAttribute(band_grid_kernel,
                                       cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem)),
                  "cudaFuncSetAttribute(band_grid_kernel)");
  if (rc) return rc;
  int dev = 0, sms = 0, per_sm = 0, coop = 0;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  cudaDeviceGetAttribute(&coop, cudaDevAttrCooperativeLaunch, dev);
  rc = cuda_check(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, band_grid_kernel,
                                                                kGridBT, smem),
                  "cudaOccupancyMaxActiveBlocksPerMultiprocessor");
  if (rc) return rc;
  if (!coop || per_sm * sms < kBandGridBlocks)
    return fail(QTQP_ERR_CUDA, "qtqp_band_grid_solve: the device cannot hold " +
                                   std::to_string(kBandGridBlocks) +
                                   " co-resident blocks of the cooperative solve");
  BandGridParams p;
  p.d = d;
  p.parts = parts;
  p.ipool = d_ipool;
  p.vpool = d_vpool;
  p.b_pool = d_b_pool;
  p.c_pool = d_c_pool;
  p.x_pool = d_x_pool;
  p.y_pool = d_y_pool;
  p.s_pool = d_s_pool;
  p.result = d_result;
  p.stats = d_stats;
  p.ws = ws;
  p.smem = smem;
  p.opt = *opt;
  void* args[] = {&p};
  return cuda_check(cudaLaunchCooperativeKernel(reinterpret_cast<void*>(band_grid_kernel),
                                                dim3(kBandGridBlocks), dim3(kGridBT), args, smem,
                                                st),
                    "band_grid_kernel cooperative launch");
}
