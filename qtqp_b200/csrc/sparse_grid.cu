// One sparse QP on the whole GPU: the shared device IPM in grid mode
// (Ipm<kSparseGridNT, kFmtSparse>) with the supernodal Cholesky of
// sparse_grid.cuh, one cooperative launch of kSparseGridBlocks blocks.  The
// QP arrives in the banded backend's pools (A as CSR + CSC, P as CSR), in the
// column order of the symbolic plan.
#include <algorithm>

#include "sparse_grid.cuh"

namespace qtqp {

struct SparseGridParams {
  qtqp_band_instance d;
  SnFactor f;
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
  qtqp_options opt;
};

__host__ __device__ inline size_t round256(size_t b) { return (b + 255) & ~size_t(255); }

struct SparseLayout {
  size_t band_off, vals_off, z_off, parts_off, upd_off, ctl_off, info_off, total;
};
// Workspace: the banded backend's vectors and working values, the factor
// (nvals), the forward products (one per stored row), the backward partial
// sums (kSnMaxW per top-level row slab), the partial updates of split row
// slabs, the grid's barrier state and the factorisation status.
__host__ __device__ inline SparseLayout plan_sparse_layout(int n, int m, int nnz_a, int nnz_p,
                                                           int64_t nvals, int64_t nrows,
                                                           int64_t nslabs) {
  SparseLayout L;
  const BandLayout B = plan_band_layout(n, m, 0, nnz_a, nnz_p);
  L.band_off = 0;
  L.vals_off = round256(B.total);
  L.z_off = round256(L.vals_off + size_t(nvals) * 8);
  L.parts_off = round256(L.z_off + size_t(nrows) * 8);
  L.upd_off = round256(L.parts_off + size_t(nslabs) * kSnMaxW * 8);
  L.ctl_off = round256(L.upd_off + size_t(kSparseGridBlocks) * kSnSlab * kSnMaxW * 8);
  L.info_off = round256(L.ctl_off + sizeof(GridCtl));
  L.total = L.info_off + 256;
  return L;
}

__global__ void __launch_bounds__(kGridBT, 1) sparse_grid_kernel(const SparseGridParams p) {
  __shared__ double red[2 * (kGridBT / 32) * kRedMax];
  __shared__ qtqp_options sopt;
  __shared__ SnFactor sf;
  extern __shared__ double snmem[];
  const qtqp_band_instance& d = p.d;
  const SparseLayout L =
      plan_sparse_layout(d.n, d.m, d.nnz_a, d.nnz_p, p.f.nvals, p.f.nrows, p.f.nslabs);
  if (threadIdx.x == 0) {
    sopt = p.opt;
    sf = p.f;
    sf.vals = reinterpret_cast<double*>(p.ws + L.vals_off);
    sf.zbuf = reinterpret_cast<double*>(p.ws + L.z_off);
    sf.pbuf = reinterpret_cast<double*>(p.ws + L.parts_off);
    sf.ubuf = reinterpret_cast<double*>(p.ws + L.upd_off);
  }
  __syncthreads();
  Ipm<kSparseGridNT, kFmtSparse> s;
  s.bind_band(d.n, d.m, 0, d.nnz_a, d.nnz_p, p.ws + L.band_off);
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
  s.sn = &sf;
  s.bwin = snmem;
  s.bwin_bytes = kSparseSmem;
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

// Row slabs of the top-level supernodes: the plan's top_slab[ntop] (also in
// the descriptor, so that the host needs no pool to size the workspace).
static int64_t top_slabs(const qtqp_sparse_desc& sd) { return sd.top_row_slabs; }

static int check_sparse(const qtqp_band_instance* h, const qtqp_sparse_desc* sd, const char* who) {
  if (h == nullptr || sd == nullptr)
    return fail(QTQP_ERR_BAD_ARG, std::string(who) + ": null instance or plan");
  const qtqp_band_instance& d = *h;
  if (d.n < 1 || d.m < 1 || d.z < 0 || d.z >= d.m || d.nnz_a < 0 || d.nnz_p < 0)
    return fail(QTQP_ERR_BAD_ARG, std::string(who) + ": needs n >= 1, m >= 1, 0 <= z < m");
  if (sd->n != d.n || sd->blocks != kSparseGridBlocks || sd->max_width > kSnMaxW ||
      sd->nsuper < 1 || sd->nvals < d.n)
    return fail(QTQP_ERR_BAD_ARG, std::string(who) + ": the plan does not match the instance "
                                                     "(n, " + std::to_string(kSparseGridBlocks) +
                                      " blocks, supernodes at most " + std::to_string(kSnMaxW) +
                                      " wide)");
  return QTQP_OK;
}

}  // namespace qtqp

using namespace qtqp;

extern "C" int32_t qtqp_sparse_grid_blocks(void) { return kSparseGridBlocks; }

extern "C" size_t qtqp_sparse_grid_workspace_bytes(const qtqp_band_instance* h_inst,
                                                   const qtqp_sparse_desc* h_desc) {
  if (check_sparse(h_inst, h_desc, "qtqp_sparse_grid_workspace_bytes") != QTQP_OK) return 0;
  const qtqp_band_instance& d = *h_inst;
  return plan_sparse_layout(d.n, d.m, d.nnz_a, d.nnz_p, h_desc->nvals, h_desc->nrows,
                            top_slabs(*h_desc))
      .total;
}

extern "C" int qtqp_sparse_grid_solve(const qtqp_band_instance* h_inst,
                                      const qtqp_sparse_desc* h_desc, const int32_t* d_sn32,
                                      const int64_t* d_sn64, const int32_t* d_ipool,
                                      const double* d_vpool, const double* d_b_pool,
                                      const double* d_c_pool, double* d_x_pool, double* d_y_pool,
                                      double* d_s_pool, qtqp_result* d_result,
                                      qtqp_iter_stats* d_stats, void* d_workspace,
                                      size_t workspace_bytes, const qtqp_options* opt,
                                      void* stream) {
  int rc = check_sparse(h_inst, h_desc, "qtqp_sparse_grid_solve");
  if (rc) return rc;
  if (d_sn32 == nullptr || d_sn64 == nullptr || d_ipool == nullptr || d_vpool == nullptr ||
      d_b_pool == nullptr || d_c_pool == nullptr || d_x_pool == nullptr || d_y_pool == nullptr ||
      d_s_pool == nullptr || d_result == nullptr || d_workspace == nullptr || opt == nullptr)
    return fail(QTQP_ERR_BAD_ARG, "qtqp_sparse_grid_solve: null argument");
  if (opt->max_iter < 1 || opt->max_iterative_refinement_steps < 1 ||
      !(opt->step_size_scale > 0.0 && opt->step_size_scale < 1.0))
    return fail(QTQP_ERR_BAD_ARG, "qtqp_sparse_grid_solve: invalid options");
  if (opt->warm_corrections != 0 || opt->warm_shift != 0.0)
    return fail(QTQP_ERR_BAD_ARG, "qtqp_sparse_grid_solve: warm starts are not supported");
  const qtqp_band_instance& d = *h_inst;
  const qtqp_sparse_desc& sd = *h_desc;
  const SparseLayout L = plan_sparse_layout(d.n, d.m, d.nnz_a, d.nnz_p, sd.nvals, sd.nrows,
                                            top_slabs(sd));
  if (workspace_bytes < L.total)
    return fail(QTQP_ERR_BAD_ARG, "qtqp_sparse_grid_solve: workspace smaller than "
                                  "qtqp_sparse_grid_workspace_bytes(inst, plan)");
  if ((reinterpret_cast<uintptr_t>(d_workspace) | reinterpret_cast<uintptr_t>(d_sn32) |
       reinterpret_cast<uintptr_t>(d_sn64)) & 15)
    return fail(QTQP_ERR_BAD_ARG, "qtqp_sparse_grid_solve: workspace and plan pools must be "
                                  "16-byte aligned");
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  char* ws = static_cast<char*>(d_workspace);
  rc = cuda_check(cudaMemsetAsync(ws + L.ctl_off, 0, sizeof(GridCtl), st), "cudaMemsetAsync");
  if (rc) return rc;
  rc = cuda_check(cudaFuncSetAttribute(sparse_grid_kernel,
                                       cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       int(kSparseSmem)),
                  "cudaFuncSetAttribute(sparse_grid_kernel)");
  if (rc) return rc;
  int dev = 0, sms = 0, per_sm = 0, coop = 0;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  cudaDeviceGetAttribute(&coop, cudaDevAttrCooperativeLaunch, dev);
  rc = cuda_check(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, sparse_grid_kernel,
                                                                kGridBT, kSparseSmem),
                  "cudaOccupancyMaxActiveBlocksPerMultiprocessor");
  if (rc) return rc;
  if (!coop || per_sm * sms < kSparseGridBlocks)
    return fail(QTQP_ERR_CUDA, "qtqp_sparse_grid_solve: the device cannot hold " +
                                   std::to_string(kSparseGridBlocks) +
                                   " co-resident blocks of the cooperative solve");
  SparseGridParams p;
  p.d = d;
  SnFactor& f = p.f;
  f.n = sd.n;
  f.nsuper = sd.nsuper;
  f.top_levels = sd.top_levels;
  f.nvals = sd.nvals;
  f.ngram = sd.ngram;
  f.nrows = sd.nrows;
  f.nslabs = top_slabs(sd);
  f.first = d_sn32 + sd.o_first;
  f.colsn = d_sn32 + sd.o_colsn;
  f.rows = d_sn32 + sd.o_rows;
  f.upd_ptr = d_sn32 + sd.o_upd_ptr;
  f.upd_src = d_sn32 + sd.o_upd_src;
  f.upd_off = d_sn32 + sd.o_upd_off;
  f.upd_cnt = d_sn32 + sd.o_upd_cnt;
  f.cta_ptr = d_sn32 + sd.o_cta_ptr;
  f.cta_range = d_sn32 + sd.o_cta_range;
  f.top_ptr = d_sn32 + sd.o_top_ptr;
  f.top_list = d_sn32 + sd.o_top_list;
  f.top_slab = d_sn32 + sd.o_top_slab;
  f.gcol = d_sn32 + sd.o_gcol;
  f.grow = d_sn32 + sd.o_grow;
  f.rowptr = d_sn64 + sd.o_rowptr;
  f.valptr = d_sn64 + sd.o_valptr;
  f.gpos = d_sn64 + sd.o_gpos;
  f.vals = nullptr;  // set on the device (inside the workspace)
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
  p.opt = *opt;
  void* args[] = {&p};
  return cuda_check(cudaLaunchCooperativeKernel(reinterpret_cast<void*>(sparse_grid_kernel),
                                                dim3(kSparseGridBlocks), dim3(kGridBT), args,
                                                kSparseSmem, st),
                    "sparse_grid_kernel cooperative launch");
}
