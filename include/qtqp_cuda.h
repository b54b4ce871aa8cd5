/* C-ABI of libqtqp_cuda.so: the B200 (sm_100a) interior-point hot path of QTQP.
 *
 * Conventions
 *   - Every entry point returns 0 (QTQP_OK) or a negative QTQP_ERR_* code; the
 *     message of the last failure on the calling thread is qtqp_last_error().
 *   - Pointers named d_* are device pointers (allocated by the caller, e.g. by
 *     PyTorch); h_* are host pointers.  No entry point allocates device memory
 *     unless its comment says so: scratch comes from the caller's workspace.
 *   - All kernels run on the caller's stream; entry points return without
 *     synchronising unless documented otherwise.
 *   - Arithmetic is FP64 except where an options field selects FP32 for the
 *     KKT factorisation (FP64 iterative refinement recovers the accuracy).
 *
 * Reference: google-deepmind/qtqp v0.0.5 (pure Python).  Each function names
 * the reference interface it replaces.
 */
#ifndef QTQP_CUDA_H_
#define QTQP_CUDA_H_

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define QTQP_OK 0
#define QTQP_ERR_BAD_ARG (-1)
#define QTQP_ERR_CUDA (-2)
#define QTQP_ERR_NOT_SPD (-3)
#define QTQP_ERR_TIMEOUT (-4)
#define QTQP_ERR_NAN (-5)

/* SolutionStatus codes (src/qtqp/__init__.py:129-137). */
#define QTQP_STATUS_SOLVED 0
#define QTQP_STATUS_INFEASIBLE 1
#define QTQP_STATUS_UNBOUNDED 2
#define QTQP_STATUS_HIT_MAX_ITER 3
#define QTQP_STATUS_FAILED 4
#define QTQP_STATUS_UNFINISHED 5

/* Precision of the KKT factorisation. */
#define QTQP_PREC_FP64 0  /* plain FP64 factor, FP64 refinement            */
#define QTQP_PREC_MIXED 1 /* FP32 factor + FP64 refinement; an instance whose
                             refinement stalls is refactorised in FP64 and
                             stays FP64 from then on                          */

/* Keyword arguments of QTQP.solve (src/qtqp/__init__.py:309-326). */
typedef struct {
  double atol, rtol, atol_infeas, rtol_infeas;
  double step_size_scale;
  double min_static_regularization;
  double linear_solver_atol, linear_solver_rtol;
  int32_t max_iter;
  int32_t max_iterative_refinement_steps;
  int32_t equilibrate;   /* 0 / 1 */
  int32_t precision;     /* QTQP_PREC_* */
  int32_t collect_stats; /* 1: write one qtqp_iter_stats record per iteration */
  int32_t tau_mode;      /* 0: quadratic with linearised fallback; 1: always
                            linearised (__init__.py:736-752)                 */
  int32_t warm_corrections; /* learned warm start only (no reference
                            counterpart): primal-dual active-set corrections
                            after the first reduced KKT solve; 0 = exactly
                            one reduced solve                                */
  double warm_shift;     /* learned warm start only: > 0 starts the IPM of an
                            instance whose prediction was not accepted from
                            that prediction, y and s on the inequality rows
                            shifted by warm_shift; 0 = the cold start         */
} qtqp_options;

/* One QP of a batch.  Offsets are element offsets into the caller's pools. */
typedef struct {
  int32_t n, m, z;  /* variables, constraints (after presolve), equalities */
  int32_t has_p;    /* nnz(P) > 0 (the reference's p.nnz > 0 tests)       */
  int64_t a_off;    /* A: m x n column-major FP64 in a_pool (the value
                       order of a CSC matrix that stores every entry)     */
  int64_t p_off;    /* P: n x n column-major FP64 (symmetric) in p_pool    */
  int64_t n_off;    /* c in c_pool, x in x_pool: n doubles each            */
  int64_t m_off;    /* b in b_pool, y / s in y_pool / s_pool: m doubles    */
  int64_t ws_off;   /* byte offset of this instance's global workspace     */
  int64_t st_off;   /* record offset in the stats pool (collect_stats)     */
} qtqp_dense_instance;

/* Per-instance outcome. */
typedef struct {
  int32_t status;           /* QTQP_STATUS_*                                  */
  int32_t iterations;       /* IPM steps taken (len(Solution.stats))           */
  int32_t error;            /* 0, QTQP_ERR_NOT_SPD or QTQP_ERR_NAN             */
  int32_t fp32_factorizations;
  int32_t fp64_factorizations;
  int32_t ir_solves;        /* backend solves summed over all KKT solves       */
  int32_t warm_started;     /* 1: the learned warm start was accepted          */
  int32_t reserved;
  double tau;               /* final tau                                       */
  double pcost, dcost, pres, dres, gap;
} qtqp_result;

/* Per-iteration record (the stats dict of __init__.py:967-1007 plus the three
 * lin_sys_stats dicts of direct.py:300-307).  Field order is fixed; the host
 * turns each record into the reference's dictionary. */
#define QTQP_STATS_DOUBLES 64
typedef struct {
  double v[QTQP_STATS_DOUBLES];
} qtqp_iter_stats;

/* A batch is solved by up to QTQP_MAX_GROUPS concurrent persistent launches,
 * one per size class of the instances (the shared-memory footprint of a QP
 * fixes how many thread blocks fit on an SM). */
#define QTQP_MAX_GROUPS 8
typedef struct {
  int32_t begin, count;  /* slice of the processing order                  */
  int32_t block_threads; /* threads per block                             */
  int32_t smem_bytes;    /* dynamic shared memory per block               */
  int32_t slots;         /* banded batches: workspace slots (max blocks)   */
  int32_t lean;          /* dense batches: 1 = the register-capped kernel
                            (more resident blocks), 0 = free registers     */
  uint64_t slot_off;     /* banded batches: byte offset of the first slot  */
  uint64_t slot_bytes;   /* banded batches: bytes per slot                 */
} qtqp_launch_group;

typedef struct {
  int32_t num_groups;
  int32_t reserved;
  qtqp_launch_group groups[QTQP_MAX_GROUPS];
  uint64_t workspace_bytes; /* global scratch the solve needs               */
} qtqp_batch_plan;

/* ---- library ------------------------------------------------------------ */
const char* qtqp_last_error(void);
int qtqp_version(void);
/* Number of SMs of the current device (0 when no device is visible). */
int qtqp_device_sm_count(void);

/* Host-only helper (no device work, no CUDA call): copies `count` host
 * blocks, h_src[i] (an address) of h_bytes[i] bytes, to h_dst + h_dst_off[i],
 * on `threads` host threads (0: up to 16).  Packs the batch pools below from
 * the thousands of per-QP arrays a batch arrives as (the reference packs
 * nothing: its solver handles one QP at a time, src/qtqp/__init__.py:183-246). */
int qtqp_host_gather(int32_t count, const uint64_t* h_src, const int64_t* h_bytes,
                     const int64_t* h_dst_off, void* h_dst, int32_t threads);

/* ---- batched dense device-resident IPM ---------------------------------- *
 * Replaces QTQP._solve_impl (src/qtqp/__init__.py:351-614) with its KKT layer
 * (src/qtqp/direct.py:112-311) and the dense Gram/Cholesky backend
 * (src/qtqp/solvers_dense.py:25-145), for a batch of independent QPs: one
 * thread block runs one QP's whole solve (Ruiz, normalise, KKT factor, IR,
 * predictor/corrector, ratio test, termination, unscaling).
 *
 * qtqp_dense_batch_plan: host-only.  Given the instances' (n, m, z) it fills
 * inst[i].ws_off, writes the processing order (descending cost) to h_order
 * and the launch groups and workspace size to *plan.  block_threads and
 * smem_bytes force one launch shape for every group when non-zero. */
int qtqp_dense_batch_plan(qtqp_dense_instance* h_inst, int32_t count,
                          const qtqp_options* opt, int32_t* h_order,
                          int32_t block_threads, int32_t smem_bytes,
                          qtqp_batch_plan* plan);

/* One entry of a launch-shape tuning table (no reference counterpart; the
 * library's autotuner writes them, qtqp_b200/autotune.py): a launch group
 * whose largest n lies in [n_lo, n_hi] runs with block_threads threads per
 * block (32, 64, 128 or 256), the register-capped kernel when lean != 0, and
 * A and P in shared memory when onchip != 0 and they fit (else only the Gram
 * matrix and the vectors).  qtqp_dense_batch_plan_tuned plans like
 * qtqp_dense_batch_plan and then applies the first matching entry to each
 * group; groups no entry matches keep the default shape. */
typedef struct {
  int32_t n_lo, n_hi;
  int32_t block_threads;
  int32_t lean;
  int32_t onchip;
  int32_t reserved;
} qtqp_batch_tuning;
int qtqp_dense_batch_plan_tuned(qtqp_dense_instance* h_inst, int32_t count,
                                const qtqp_options* opt, int32_t* h_order,
                                const qtqp_batch_tuning* table, int32_t entries,
                                qtqp_batch_plan* plan);

/* Device-resident solve of the whole batch.
 * d_inst / d_order: the planned descriptors and order, copied to the device by
 * the caller; plan: the host plan that produced them.  b/c pools are inputs;
 * x/y/s pools and d_results are outputs (x, y, s after the reference's
 * status-dependent scaling, __init__.py:580-614; presolve row restoration is
 * the host's job).  d_stats: qtqp_iter_stats[max_iter] per instance, or NULL.
 * The groups run on side streams forked from and joined back to `stream`. */
int qtqp_dense_batch_solve(const qtqp_dense_instance* d_inst,
                           const int32_t* d_order, const qtqp_batch_plan* plan,
                           const double* d_a_pool, const double* d_p_pool,
                           const double* d_b_pool, const double* d_c_pool,
                           double* d_x_pool, double* d_y_pool,
                           double* d_s_pool, qtqp_result* d_results,
                           qtqp_iter_stats* d_stats, void* d_workspace,
                           size_t workspace_bytes, const qtqp_options* opt,
                           void* stream);

/* Launch group `group` of the plan alone, on `stream` (the same arguments as
 * qtqp_dense_batch_solve; only that group's work counter is reset).  A caller
 * that packs and copies the batch group by group launches each group as soon
 * as its data is on the device, on a stream of its own, while it packs the
 * next one; the groups' instances do not overlap, so the launches may run
 * concurrently. */
int qtqp_dense_batch_solve_group(const qtqp_dense_instance* d_inst,
                                 const int32_t* d_order,
                                 const qtqp_batch_plan* plan, int32_t group,
                                 const double* d_a_pool, const double* d_p_pool,
                                 const double* d_b_pool, const double* d_c_pool,
                                 double* d_x_pool, double* d_y_pool,
                                 double* d_s_pool, qtqp_result* d_results,
                                 qtqp_iter_stats* d_stats, void* d_workspace,
                                 size_t workspace_bytes, const qtqp_options* opt,
                                 void* stream);

/* qtqp_dense_batch_solve started from given points instead of the cold
 * start of _init_variables (src/qtqp/__init__.py:299-307; the reference has
 * no warm start -- its re-solve, tests/test_qtqp.py:1578-1598, starts cold
 * every time): d_x0_pool / d_y0_pool / d_s0_pool hold one point per
 * instance laid out like the x / y / s pools, in the original scaling, with
 * y and s positive on the inequality rows (s zero on the equality rows).
 * An earlier solution of the same or a nearby QP, moved into the interior,
 * is the typical start. */
int qtqp_dense_batch_solve_from(const qtqp_dense_instance* d_inst,
                                const int32_t* d_order,
                                const qtqp_batch_plan* plan,
                                const double* d_a_pool, const double* d_p_pool,
                                const double* d_b_pool, const double* d_c_pool,
                                double* d_x_pool, double* d_y_pool,
                                double* d_s_pool, qtqp_result* d_results,
                                qtqp_iter_stats* d_stats, void* d_workspace,
                                size_t workspace_bytes, const qtqp_options* opt,
                                const double* d_x0_pool, const double* d_y0_pool,
                                const double* d_s0_pool, void* stream);

/* Allocation-free variant of qtqp_dense_batch_solve.  It has no counterpart
 * in the reference (whose solver is pure Python).  It exists for callers that
 * cannot allocate device memory at solve time -- code inside another
 * framework's memory pool, or a control loop that must not call the
 * allocator once running -- so it takes no workspace: its scratch is a fixed
 * 16 MiB array inside this library (reserved on every GPU that loads the
 * library until the process exits).  Plans needing more scratch than
 * qtqp_dense_batch_noalloc_max_workspace() are rejected with
 * QTQP_ERR_BAD_ARG.  The first call on a device looks up the array's device
 * address (cudaGetSymbolAddress), and so does the first call after the
 * device's context was replaced (cudaDeviceReset); make those calls before
 * any stream capture.  Every call uses the same array, so calls whose work overlaps on
 * the GPU (e.g. on two streams) race and must not be issued; groups run in
 * sequence on `stream`.  Arguments and results as qtqp_dense_batch_solve. */
size_t qtqp_dense_batch_noalloc_max_workspace(void);
int qtqp_dense_batch_solve_noalloc(const qtqp_dense_instance* d_inst,
                                   const int32_t* d_order,
                                   const qtqp_batch_plan* plan,
                                   const double* d_a_pool,
                                   const double* d_p_pool,
                                   const double* d_b_pool,
                                   const double* d_c_pool, double* d_x_pool,
                                   double* d_y_pool, double* d_s_pool,
                                   qtqp_result* d_results,
                                   qtqp_iter_stats* d_stats,
                                   const qtqp_options* opt, void* stream);

/* ---- batched banded / sparse device-resident IPM ------------------------ *
 * Same algorithm and outputs as qtqp_dense_batch_solve for QPs whose A and P
 * are sparse and whose Gram matrix G = P + A^T diag(1/Ry) A is banded with
 * half-bandwidth bw (e.g. stage-ordered MPC problems): A is given as CSR and
 * CSC, P as CSR with both triangles; the factor is a band Cholesky.  Replaces
 * QTQP._solve_impl (src/qtqp/__init__.py:351-614) with the KKT layer of
 * src/qtqp/direct.py:112-311 for this storage (the reference's sparse
 * backends factorise the full KKT; the Gram reduction follows
 * src/qtqp/solvers_dense.py:25-145 in band storage).
 * Offsets are element offsets: *_ptr/*_idx into the int32 pool, *_val into
 * the double pool. */
typedef struct {
  int32_t n, m, z, has_p;
  int32_t bw, nnz_a, nnz_p, reserved;
  int64_t a_ptr, a_idx, a_val;    /* A CSR: m+1 row pointers, columns, values */
  int64_t at_ptr, at_idx, at_val; /* A CSC: n+1 column pointers, rows, values */
  int64_t p_ptr, p_idx, p_val;    /* P CSR (symmetric, both triangles)       */
  int64_t n_off, m_off;           /* c/x and b/y/s pools                     */
  int64_t st_off;                 /* stats record offset (collect_stats)     */
} qtqp_band_instance;

/* Host-only planning.  Every block in flight owns one workspace slot sized
 * for the largest instance, so the workspace does not grow with the batch;
 * num_sms (0: 148) bounds the number of resident blocks. */
int qtqp_band_batch_plan(qtqp_band_instance* h_inst, int32_t count,
                         const qtqp_options* opt, int32_t num_sms,
                         int32_t* h_order, qtqp_batch_plan* plan);
int qtqp_band_batch_solve(const qtqp_band_instance* d_inst,
                          const int32_t* d_order, const qtqp_batch_plan* plan,
                          const int32_t* d_ipool, const double* d_vpool,
                          const double* d_b_pool, const double* d_c_pool,
                          double* d_x_pool, double* d_y_pool, double* d_s_pool,
                          qtqp_result* d_results, qtqp_iter_stats* d_stats,
                          void* d_workspace, size_t workspace_bytes,
                          const qtqp_options* opt, const double* d_warm_x,
                          const double* d_warm_y, const uint8_t* d_warm_active,
                          void* stream);
/* d_warm_x / d_warm_y / d_warm_active (no reference counterpart): null for
 * the plain method, or a learned warm start laid out like the x / y pools
 * (original scaling) plus one active flag per constraint row.  Each instance
 * then first solves the KKT system of the equality QP on its active rows
 * (opt->warm_corrections primal-dual corrections of the set at most) and
 * keeps that point only if the plain termination test reports SOLVED for it;
 * otherwise the plain method runs from its usual start.
 * qtqp_result.warm_started tells which. */

/* ---- one large banded QP on the whole GPU -------------------------------- *
 * The banded device IPM of qtqp_band_batch_solve (same algorithm, options
 * and outputs; QTQP._solve_impl, src/qtqp/__init__.py:351-614, with the KKT
 * layer of src/qtqp/direct.py:112-311) for a single large QP, run by one
 * cooperative launch of 128 blocks: Gram matrix, residuals and sparse
 * products over the whole grid, and a partitioned band Cholesky (`parts`
 * interiors factorised in parallel, a block-tridiagonal Cholesky over the
 * parts-1 separators of bw columns between them) with the matching
 * partitioned triangular solves.  h_inst: host pointer to the instance's
 * descriptor (offsets into the device pools as in the batch).  parts in
 * [1, min(128, (n + bw) / (2 bw))]; qtqp_band_grid_default_parts gives the
 * default.  bw <= 118 (the separator blocks are staged in shared memory);
 * wider bands return QTQP_ERR_BAD_ARG.  The workspace (>=
 * qtqp_band_grid_workspace_bytes, 256-byte aligned) is private.  A grid
 * barrier that waits too long ends the solve with status FAILED and error
 * QTQP_ERR_TIMEOUT. */
int32_t qtqp_band_grid_default_parts(const qtqp_band_instance* h_inst);
size_t qtqp_band_grid_workspace_bytes(const qtqp_band_instance* h_inst,
                                      int32_t parts);
int qtqp_band_grid_solve(const qtqp_band_instance* h_inst, int32_t parts,
                         const int32_t* d_ipool, const double* d_vpool,
                         const double* d_b_pool, const double* d_c_pool,
                         double* d_x_pool, double* d_y_pool, double* d_s_pool,
                         qtqp_result* d_result, qtqp_iter_stats* d_stats,
                         void* d_workspace, size_t workspace_bytes,
                         const qtqp_options* opt, void* stream);

/* ---- one sparse QP on the whole GPU: supernodal Cholesky ----------------- *
 * For QPs whose Gram matrix P + A^T D A is neither small and dense nor
 * narrow-banded: the role of the sparse direct backends behind the plugin
 * interface (src/qtqp/solvers_sparse.py:96-121 SuperLU,
 * src/qtqp/solvers_gpu.py:27-116 cuDSS), on the dense backend's Gram
 * reduction (src/qtqp/solvers_dense.py:99-116).
 *
 * Host symbolic stage: qtqp_sparse_analyze orders G's pattern (the union of
 * P's pattern and one clique per row of A; ordering 1 = minimum degree on the
 * quotient graph with approximate degrees, 0 = the given order), composes the
 * ordering with a postorder of the elimination tree, finds supernodes (at
 * most 64 columns wide), their row structures and left-looking update lists,
 * maps whole subtrees to the `blocks` blocks of the grid solve
 * (qtqp_sparse_grid_blocks()) and the supernodes above them to levels, and
 * maps G's lower entries to positions in the factor.  A and P are CSC
 * (int32 column pointers and row indices; P may be NULL).  The plan stays on
 * the host until qtqp_sparse_free; qtqp_sparse_export writes the column order
 * (perm[new] = old, n entries) and the plan's two pools (desc.n32 int32 and
 * desc.n64 int64 elements; the offsets in desc), which the caller copies to
 * the device unchanged. */
typedef struct qtqp_sparse_desc {
  int32_t n, nsuper, blocks, top_levels;
  int32_t max_rows, max_width, tree_levels, reserved;
  int64_t nvals;    /* factor values (column-major blocks of the supernodes) */
  int64_t ngram;    /* lower entries of G, diagonal included */
  int64_t nrows, nupd, nranges, ntop;
  int64_t nnz_l;    /* stored lower entries of L */
  int64_t top_row_slabs; /* 64-row work items of the supernodes above the subtrees */
  double flops;     /* multiply-adds x 2 of one numeric factorisation */
  int64_t o_first, o_colsn, o_rows, o_upd_ptr, o_upd_src, o_upd_off, o_upd_cnt,
      o_cta_ptr, o_cta_range, o_top_ptr, o_top_list, o_top_slab, o_gcol,
      o_grow;                                                     /* int32 pool */
  int64_t o_rowptr, o_valptr, o_gpos;                             /* int64 pool */
  int64_t n32, n64;
} qtqp_sparse_desc;
int qtqp_sparse_analyze(int32_t n, int32_t m, const int32_t* h_a_colptr,
                        const int32_t* h_a_rowind, const int32_t* h_p_colptr,
                        const int32_t* h_p_rowind, int32_t ordering, int32_t blocks,
                        void** h_plan, qtqp_sparse_desc* h_desc);
int qtqp_sparse_export(const void* h_plan, const qtqp_sparse_desc* h_desc,
                       int32_t* h_perm, int32_t* h_pool32, int64_t* h_pool64);
void qtqp_sparse_free(void* h_plan);
/* Grid solve: the banded backend's device IPM (same algorithm, options and
 * outputs as qtqp_band_grid_solve) with the supernodal factor.  h_inst
 * describes the QP in the pools exactly as for the banded backend, with its
 * columns in the plan's order (bw is ignored); d_sn32 / d_sn64 are the
 * exported pools on the device (16-byte aligned).  FP64 and mixed precision;
 * no learned warm start.  Every wait is bounded (status FAILED, error
 * QTQP_ERR_TIMEOUT). */
int32_t qtqp_sparse_grid_blocks(void);
size_t qtqp_sparse_grid_workspace_bytes(const qtqp_band_instance* h_inst,
                                        const qtqp_sparse_desc* h_desc);
int qtqp_sparse_grid_solve(const qtqp_band_instance* h_inst,
                           const qtqp_sparse_desc* h_desc, const int32_t* d_sn32,
                           const int64_t* d_sn64, const int32_t* d_ipool,
                           const double* d_vpool, const double* d_b_pool,
                           const double* d_c_pool, double* d_x_pool, double* d_y_pool,
                           double* d_s_pool, qtqp_result* d_result,
                           qtqp_iter_stats* d_stats, void* d_workspace,
                           size_t workspace_bytes, const qtqp_options* opt,
                           void* stream);

/* ---- learned warm start: MLP kernels (no reference counterpart) --------- *
 * theta -> 256 -> 256 -> (n + m) MLP, FP32, all matrices row-major.  Used to
 * train the network on plain-method solutions of a parametric family and to
 * produce warm starts for qtqp_band_batch_solve. */
/* C = alpha op(A) op(B) + beta C (+ bias per column) (ReLU if relu != 0);
 * op(A) is M x K (A stored K x M if trans_a), op(B) is K x N (B stored
 * N x K if trans_b).  C is not read when beta == 0. */
int qtqp_mlp_gemm(int32_t M, int32_t N, int32_t K, float alpha, const float* d_a,
                  int32_t lda, int32_t trans_a, const float* d_b, int32_t ldb,
                  int32_t trans_b, float beta, float* d_c, int32_t ldc,
                  const float* d_bias, int32_t relu, void* stream);
/* dh[i] = h[i] > 0 ? dh[i] : 0 (backward of the ReLU whose output is h). */
int qtqp_mlp_relu_grad(float* d_dh, const float* d_h, int64_t count, void* stream);
/* db[j] = sum_i d[i * cols + j]. */
int qtqp_mlp_colsum(const float* d_d, int32_t rows, int32_t cols, float* d_db,
                    void* stream);
/* dy = 2 (y - t) / count and *d_loss = sum (y - t)^2 (overwritten). */
int qtqp_mlp_mse_grad(const float* d_y, const float* d_t, int64_t count,
                      float* d_dy, double* d_loss, void* stream);
/* Hinge term on the sign of the inequality outputs, added to d_dy (after
 * qtqp_mlp_mse_grad on the same buffers): columns [col0, cols) of the
 * rows x cols output; d_zero[j - col0] is the column's decision point (the
 * standardised value of y_i - s_i = 0); the target's side of it gives the
 * sign s = +-1.  Adds weight * mean(relu(margin - s (y - zero))) to *d_loss
 * and its gradient to d_dy. */
int qtqp_mlp_hinge_grad(const float* d_y, const float* d_t, int32_t rows,
                        int32_t cols, int32_t col0, const float* d_zero,
                        float weight, float margin, float* d_dy, double* d_loss,
                        void* stream);
/* Forward-pass GEMM of the MLP on the tensor cores (tcgen05, BF16 inputs,
 * FP32 accumulation): C = A B^T (+ bias per column) (ReLU if relu != 0), A
 * M x K and B N x K BF16 row-major (K a multiple of 8, 16-byte aligned), C
 * M x N FP32 (leading dimension ldc) and, when d_c16 is not NULL, its BF16
 * copy (leading dimension ldc16) for the next layer.  *d_err (device int32)
 * is set to 1 if a bounded pipeline wait gave up (the tile is not written). */
int qtqp_mlp_gemm_bf16(int32_t M, int32_t N, int32_t K, const void* d_a,
                       const void* d_bt, float* d_c, int32_t ldc,
                       const float* d_bias, int32_t relu, void* d_c16,
                       int32_t ldc16, int32_t* d_err, void* stream);
/* FP32 rows x cols row-major -> BF16 (round to nearest even), transposed
 * (cols x rows) when transpose != 0. */
int qtqp_mlp_to_bf16(const float* d_src, int32_t rows, int32_t cols,
                     int32_t transpose, void* d_dst, void* stream);
/* One Adam step (bias-corrected, step >= 1). */
int qtqp_mlp_adam(float* d_p, const float* d_g, float* d_m, float* d_v,
                  int64_t count, float lr, float beta1, float beta2, float eps,
                  int32_t step, void* stream);
/* Network outputs (count x (n+m), standardised) -> warm-start x / y pools
 * and the active mask.  v = pred * scale + shift; v[0:n] is x, v[n:n+z] the
 * equality duals, and on inequality row i the signed v = y_i - s_i (at a
 * solution at most one of the two is non-zero), decoded as y_i = max(v, 0),
 * active[i] = (v > threshold); active is 1 on the z equality rows. */
int qtqp_mlp_decode(const float* d_pred, const double* d_scale,
                    const double* d_shift, int32_t n, int32_t m, int32_t z,
                    int32_t count, double threshold, double* d_x, double* d_y,
                    uint8_t* d_active, void* stream);

/* ---- one large dense QP on the whole GPU ---------------------------------- *
 * Replaces QTQP._solve_impl (src/qtqp/__init__.py:351-614) with the dense
 * KKT backend (src/qtqp/solvers_dense.py:25-145) for a single large QP: the
 * same device IPM as the batch, run by one cooperative launch of
 * qtqp_dense_large_blocks() blocks, one per SM of a B200 (grid barriers and
 * reductions; the triangular solves hand blocks over through per-block
 * flags), with a blocked Gram + Cholesky factor
 * (Gram on tcgen05 tensor cores, TF32 hi + lo split, when opt->precision is
 * QTQP_PREC_MIXED; FP64 otherwise) and blocked triangular solves.
 * flags: QTQP_LARGE_HAS_P (P is given) | QTQP_LARGE_COLMAJOR (A and P are
 * column-major -- the value order of a dense CSC matrix -- else row-major).
 * A: m x n FP64, P: n x n FP64 (null without QTQP_LARGE_HAS_P); b, c inputs; x, y, s, *d_result outputs (as the batch); d_stats:
 * qtqp_iter_stats[max_iter] or NULL.  The workspace (>=
 * qtqp_dense_large_workspace_bytes(n, m), 1024-byte aligned) is private.
 * n <= 128 * qtqp_dense_large_blocks(), m * n < 2^31.  A grid barrier or
 * flag wait that waits too long ends the solve with status FAILED and error
 * QTQP_ERR_TIMEOUT. */
size_t qtqp_dense_large_workspace_bytes(int32_t n, int32_t m);
int32_t qtqp_dense_large_blocks(void);
#define QTQP_LARGE_HAS_P 1
#define QTQP_LARGE_COLMAJOR 2
int qtqp_dense_large_solve(int32_t n, int32_t m, int32_t z, int32_t flags,
                           const double* d_a, const double* d_p,
                           const double* d_b, const double* d_c, double* d_x,
                           double* d_y, double* d_s, qtqp_result* d_result,
                           qtqp_iter_stats* d_stats, void* d_workspace,
                           size_t workspace_bytes, const qtqp_options* opt,
                           void* stream);

/* ---- tensor-core building blocks of the large dense KKT factorisation ---- *
 * (the Gram term A^T D A of src/qtqp/solvers_dense.py:99-116 on tcgen05).
 * qtqp_tc_split_tf32: hi = x rounded to TF32 (nearest), lo = x - hi.
 * qtqp_tc_gram_f32: the lower 128 x 128 tiles of C = X X^T (FP32, row-major,
 * leading dimension ldc; other tiles untouched) for X n x k row-major (ld),
 * on tcgen05 kind::tf32 with FP32 accumulation: X = hi when split == 0, and
 * hi hi^T + hi lo^T + lo hi^T (FP32-level accuracy) when split == 1.  n a
 * multiple of 128, k of 32, ld and ldc multiples of 4, 16-byte aligned
 * pointers.  *d_err (device int32) is set to 1 if a pipeline wait gave up. */
int qtqp_tc_split_tf32(const float* d_x, int64_t count, float* d_hi, float* d_lo,
                       void* stream);
int qtqp_tc_gram_f32(int32_t n, int32_t k, const float* d_hi, const float* d_lo,
                     int32_t ld, float* d_c, int32_t ldc, int32_t split,
                     int32_t* d_err, void* stream);

/* ---- dense KKT backend (the direct.LinearSolver plugin) ------------------ *
 * Replaces one backend of the plugin interface src/qtqp/direct.py:49-109
 * (set_dims / set_kkt / update_diag / factorize / solve / __matmul__) with the
 * Gram/Schur algorithm of src/qtqp/solvers_dense.py:99-142, on the device.
 * Workspace layout is private; size it with qtqp_kkt_dense_workspace_bytes.
 * All vectors are device FP64. */
size_t qtqp_kkt_dense_workspace_bytes(int32_t n, int32_t m);
/* set_kkt (solvers_dense.py:85-93): A is m x n row-major, P_off is n x n
 * row-major with a zero diagonal.  Copied into the workspace. */
int qtqp_kkt_dense_set(int32_t n, int32_t m, const double* d_a,
                       const double* d_p_off, void* d_ws, void* stream);
/* update_diag + factorize (solvers_dense.py:95-116): diag is the regularised
 * KKT diagonal of length n+m with the dual block negative.  d_info (device
 * int32) receives 0 or the 1-based failing pivot (LAPACK dpotrf convention). */
int qtqp_kkt_dense_factorize(int32_t n, int32_t m, const double* d_diag,
                             int32_t precision, void* d_ws, int32_t* d_info,
                             void* stream);
/* solve (solvers_dense.py:130-142): out = K_reg^{-1} rhs. */
int qtqp_kkt_dense_solve(int32_t n, int32_t m, const double* d_rhs,
                         double* d_out, void* d_ws, void* stream);
/* __matmul__ (solvers_dense.py:118-128): out = K_reg x. */
int qtqp_kkt_dense_matvec(int32_t n, int32_t m, const double* d_x,
                          double* d_out, void* d_ws, void* stream);

/* Ruiz equilibration of one dense QP on the device, the first phase of the
 * device IPM on its own: replaces QTQP._equilibrate
 * (src/qtqp/__init__.py:616-663; 10 sweeps, scales clipped to [1e-3, 1e3],
 * a_ij scaled by d_i * e_j).  Inputs: A (m x n) and P (n x n, or NULL for
 * P = 0), b (m), c (n), row-major.  Outputs: d (m), e (n), the equilibrated
 * A (m x n) and P (n x n).  d_ws: qtqp_kkt_dense_workspace_bytes(n, m)
 * bytes (overwritten). */
int qtqp_dense_equilibrate(int32_t n, int32_t m, const double* d_a,
                           const double* d_p, const double* d_b,
                           const double* d_c, void* d_ws, double* d_d,
                           double* d_e, double* d_a_eq, double* d_p_eq,
                           void* stream);

/* ---- self-test of the bounded device waits ------------------------------ *
 * No reference counterpart.  Every spin-wait of the kernels gives up after a
 * poll limit and reports an error instead of hanging (the grid barrier and
 * the per-block flags of the whole-GPU solves: QTQP_ERR_TIMEOUT from the
 * solve; the tensor-core pipelines' mbarrier waits).  This makes one run out on purpose with a short
 * limit (limit polls, at most 2^24) and writes the outcome to *d_status
 * (QTQP_OK or QTQP_ERR_TIMEOUT):
 *   mode 0: a cooperative grid of `blocks` blocks (2..64) where block
 *           skip_block never reaches the barrier the others wait at
 *           (skip_block = -1: every block arrives, a control run);
 *           d_workspace: qtqp_wait_selftest_workspace_bytes() bytes;
 *   mode 1: one block waits on an mbarrier that nothing arrives on;
 *   mode 2: a cooperative grid of `blocks` blocks (2..64) where block b
 *           waits for block b - 1's flag, then sets its own, and block
 *           skip_block never sets its flag (-1: a control run); the same
 *           workspace as mode 0.
 * Nothing faults: the waits stop and the kernels return. */
size_t qtqp_wait_selftest_workspace_bytes(void);
int qtqp_wait_selftest(int32_t mode, int32_t blocks, int32_t skip_block,
                       uint32_t limit, void* d_workspace, int32_t* d_status,
                       void* stream);

#ifdef __cplusplus
}
#endif

#endif /* QTQP_CUDA_H_ */
