// Device-resident interior-point solve of one dense QP by one thread block.
//
// Algorithm: the homogeneous-embedding Mehrotra predictor-corrector of
// google-deepmind/qtqp v0.0.5, src/qtqp/__init__.py:351-614, with the KKT layer
// of src/qtqp/direct.py:112-311 and the Gram/Cholesky backend of
// src/qtqp/solvers_dense.py:25-145.  Every scalar decision (IR convergence and
// stall, tau root selection and fallback, ratio test, termination precedence)
// follows the reference; only the summation order of reductions differs.
//
// Work distribution inside the block ("ownership"): every per-element vector
// lives in the N-space [0, n+m) with the x-part at [0, n) and the y/s-part at
// [n, n+m); element k is always handled by thread k % NT.  Elementwise phases
// therefore need no barrier between them; a barrier is only needed before a
// phase that reads other threads' elements (matrix-vector products, the
// triangular solves) and is folded into the block reductions where possible.
#pragma once

#include <math.h>

#include "common.cuh"

namespace qtqp {

// ----------------------------------------------------------------------------
// Per-instance memory layout (shared by host planning and device code).
// ----------------------------------------------------------------------------
enum VecId : int {
  kQ = 0,    // q = [c_eq; b_eq]
  kXY,       // iterate [x; y]
  kKQ,       // K^{-1} q (warm-started across iterations)
  kKQ0,      // warm start of K^{-1} q kept for an FP64 redo (mixed precision)
  kXYP,      // predictor K^{-1} r, then [x_p; y_p]
  kXYC,      // corrector K^{-1} r, then [x_c; y_c]
  kRHS,      // KKT right-hand side with the dual block negated
  kRES,      // IR residual
  kTMP,      // solve scratch (FP64 Gram right-hand side / solution)
  kREG,      // regularised KKT diagonal (dual block negative)
  kCORR,     // reg - true diagonal
  kDE,       // [e; d] accumulated Ruiz scalings
  kPI,       // [diag(P_eq); 1/Ry]
  kPW,       // [P_eq K^{-1}q_x; 1/sqrt(Ry)]
  kRS,       // [P_eq K^{-1}r_x; s]
  kXD,       // [P_eq x; d_s]
  kCT,       // [FP32 scratch (2n floats); Mehrotra correction / warm-start rows]
  kW,        // triangular-solve scratch (FP64)
  kNumVec
};

__host__ __device__ inline int odd_ld(int n) { return (n & 1) ? n : n + 1; }
__host__ __device__ inline size_t round16(size_t b) { return (b + 15) & ~size_t(15); }

// Panel buffer (PB): the tile Cholesky's two panels of (n+3)/4 tiles of
// 4 x 4, each tile padded to 17 elements so that lanes reading different
// tiles hit different banks; outside the factorisation, the staged column
// sums of fused_products (up to 8 warps x n) and a vector of n.
__host__ __device__ inline size_t panel_buf_elems(int n) {
  return size_t(34) * ((n + 3) >> 2) + size_t(2) * n;
}

struct InstLayout {
  int lda, ldp, ldg, np;  // leading dims (doubles) and padded vector length
  size_t a_bytes, p_bytes, g_bytes, v_bytes;  // v_bytes: vectors + panel buffer
  int ap_smem, gv_smem;   // 1 when that region lives in shared memory
  size_t smem_bytes, global_bytes;
};

// Places G + vectors (and A + P when they also fit) in `smem_cap` bytes of
// shared memory; everything else goes to the instance's global workspace.
__host__ __device__ inline InstLayout plan_layout(int n, int m, size_t smem_cap) {
  InstLayout L;
  L.lda = odd_ld(n);
  L.ldp = odd_ld(n);
  L.ldg = odd_ld(n);
  L.np = (max(n + m, n + 4) + 1) & ~1;  // >= n + 4: pivot broadcast scalars
  L.a_bytes = round16(size_t(m) * L.lda * 8);
  L.p_bytes = round16(size_t(n) * L.ldp * 8);
  L.g_bytes = round16(size_t(n) * L.ldg * 8);
  L.v_bytes = round16((size_t(kNumVec) * L.np + panel_buf_elems(n)) * 8);
  const size_t gv = L.g_bytes + L.v_bytes, ap = L.a_bytes + L.p_bytes;
  L.gv_smem = gv <= smem_cap;
  L.ap_smem = L.gv_smem && (gv + ap <= smem_cap);
  L.smem_bytes = (L.gv_smem ? gv : 0) + (L.ap_smem ? ap : 0);
  L.global_bytes = (L.gv_smem ? 0 : gv) + (L.ap_smem ? 0 : ap);
  return L;
}

// Global workspace of one banded instance: vectors, the band factor (n x
// (bw+1)) and working copies of the A (CSR and CSC) and P value arrays.
struct BandLayout {
  int np;
  size_t v_bytes, l_bytes, val_bytes, total;
};
__host__ __device__ inline BandLayout plan_band_layout(int n, int m, int bw, int nnz_a,
                                                       int nnz_p) {
  BandLayout L;
  L.np = (max(n + m, n + 4) + 1) & ~1;
  L.v_bytes = round16(size_t(kNumVec) * L.np * 8);
  L.l_bytes = round16(size_t(n) * (bw + 1) * 8);
  L.val_bytes = round16((2 * size_t(nnz_a) + size_t(nnz_p)) * 8);
  L.total = L.v_bytes + L.l_bytes + L.val_bytes;
  return L;
}

// Shared-memory window of the banded factorisation / solves: bands up to
// kBandWinMaxBw use it (the (bw+2)^2 window, the per-thread Gram columns and
// the 128-slot solve window must fit).
constexpr int kBandWinMaxBw = 126;
// Shared-memory elements reserved for the blocked band solves: 256 window
// slots, two staged blocks of factor entries (forward: 2 x 8 x (bw + 1);
// backward: 2 x (bw + 8) x 8, bw <= 126) and the block's 8 values.
constexpr int kBandSolveElems = 256 + 2 * (126 + 8) * 8 + 16;
constexpr int kBandPanel = 8;  // columns per panel of the blocked band Cholesky
// Shared memory of the blocked band Cholesky (band_chol_panel_range): the
// circular (bw + kBandPanel)^2 window, the panel rows, the publish slots
// and the 16-bit trailing-update offsets.
__host__ __device__ inline size_t band_panel_bytes(int bw) {
  const size_t B = size_t(bw) + kBandPanel;
  const size_t elems = B * B + (size_t(bw) + kBandPanel) * (kBandPanel + 1) + 2 * kBandPanel;
  return elems * sizeof(double) + size_t(bw) * (size_t(bw) + 1) / 2 * sizeof(uint16_t);
}
__host__ __device__ inline size_t band_win_bytes(int bw, int nt) {
  const size_t b2 = (size_t(bw) + 2) * (size_t(bw) + 2) * sizeof(double);
  const size_t pairs = size_t(bw) * (size_t(bw) + 1) / 2 * sizeof(uint32_t);
  const size_t cols = size_t(nt) * (size_t(bw) + 1) * sizeof(double);
  const size_t solve = size_t(kBandSolveElems) * sizeof(double);
  size_t e = b2 + pairs;
  if (bw + kBandPanel <= nt && band_panel_bytes(bw) > e) e = band_panel_bytes(bw);
  if (cols > e) e = cols;
  if (solve > e) e = solve;
  return (e + 15) & ~size_t(15);
}

// Fields of one qtqp_iter_stats record.
enum StatField : int {
  kStIter = 0, kStCtx, kStBty, kStPcost, kStDcost, kStPres, kStDres, kStGap,
  kStPinfeas, kStDinfeas, kStDinfeasA, kStDinfeasP, kStMu, kStSigma,
  kStAlpha, kStTau, kStNormX, kStNormY, kStStatus, kStTime, kStPrel, kStDrel,
  kStCompl, kStNormS, kStMaxSy, kStMinSy, kStStdSy, kStMaxSoy, kStMinSoy,
  kStMeanSoy, kStStdSoy,
  kStLin0 = 31,  // three blocks of kLinFields: q, predictor, corrector
};
enum LinField : int {
  kLinSolves = 0, kLinFinalRes, kLinRhsNorm, kLinTol, kLinStatus, kLinTau,
  kLinPrec, kLinFields
};
// kLinStatus: 0 non-converged, 1 converged, 2 stalled.  kLinTau: -1 none,
// 0 quadratic, 1 linearised.  kLinPrec: 32 or 64 (factor precision used).

struct IrOutcome {
  int solves;
  int status;  // 0 non-converged, 1 converged, 2 stalled
  double final_res, rhs_norm, tol;
  bool nan;
};

// Copies of the instance's fields as local constants.  Phase functions are
// not inlined, so `this` points at a stack object; reading fields through it
// inside loops would be a local-memory load after every store that might
// alias it.  Each phase therefore starts with QTQP_LOCALS.
#define QTQP_LOCALS                                                             \
  const int tid = this->tid, n = this->n, m = this->m, z = this->z, N = this->N; \
  const int lda = this->lda, ldp = this->ldp, ldg = this->ldg;                   \
  double* const A = this->A;                                                     \
  double* const P = this->P;                                                     \
  double* const G = this->G;                                                     \
  const bool has_p = this->has_p;                                                \
  (void)tid; (void)n; (void)m; (void)z; (void)N; (void)lda; (void)ldp; (void)ldg; \
  (void)A; (void)P; (void)G; (void)has_p

// Independent partial sums per lane of a block's row dots (rowdot) outside
// the per-block dense format, which sets its own by block size (rowdot).
#ifndef QTQP_ROWDOT_UNROLL
#define QTQP_ROWDOT_UNROLL 4
#endif

// Storage formats of A, P and the KKT factor.
enum MatFormat : int {
  kFmtDense = 0,  // dense A (m x n), dense P, dense Gram G / Cholesky factor
  kFmtBand = 1,   // sparse A (CSR + CSC), sparse P (CSR), banded Gram / factor
  kFmtLarge = 2,  // one large dense QP on the whole GPU (grid mode, NT > 1024):
                  // dense A / P in global memory, blocked Gram + Cholesky
  kFmtSparse = 3, // one sparse QP on the whole GPU (grid mode): A and P as in
                  // kFmtBand, a supernodal Cholesky of the Gram matrix
};

// ----------------------------------------------------------------------------
// The solver state of one instance, replicated in every thread of the block.
// FMT selects the matrix backend; the interior-point logic is shared.
// ----------------------------------------------------------------------------
// Large-format phases (large_ipm.cuh), called from the Ipm dispatch points.
template <typename T, class S>
__device__ int large_factorize(S& s);
template <typename T, class S>
__device__ void large_chol_solve(S& s, T* v, T* w);
template <class S, class RowEpi, class ColEpi>
__device__ void large_products(S& s, const double* vx, const double* vy, const double* vs,
                               const double* vp, RowEpi row_epi, ColEpi col_epi);
// Partitioned banded factorisation / solve of grid mode (band_grid.cuh).
template <typename T, class S>
__device__ int bandp_factorize(S& s);
template <typename T, class S>
__device__ void bandp_solve(S& s, T* v, T* w);
// Supernodal factorisation / solve of grid mode (sparse_grid.cuh).
struct SnFactor;
template <typename T, class S>
__device__ int sparse_factorize(S& s);
template <typename T, class S>
__device__ void sparse_solve(S& s, T* v, T* w);

template <int NT, int FMT = kFmtDense>
struct Ipm {
  // Sparse A and P (CSR / CSC) with a banded or supernodal Gram factor.
  static constexpr bool kSparseA = FMT == kFmtBand || FMT == kFmtSparse;
  int tid;
  int n, m, z, N;
  bool has_p;
  // Original (presolved, unequilibrated) data in global memory: row-major,
  // or column-major (the value order of a dense CSC matrix) when colmajor.
  const double* A0;
  const double* P0;
  bool colmajor = false;
  const double* b0;
  const double* c0;
  // Working data.
  double* A;  // m x lda equilibrated A
  double* P;  // n x ldp equilibrated P with a zero diagonal (P_off)
  double* G;  // n x ldg Gram matrix / Cholesky factor (FP64, or FP32 alias)
  double* V;  // kNumVec vectors of np doubles
  double* PB;  // panel buffer of tile_cholesky (panel_buf_elems(n) elements)
  int lda, ldp, ldg, np;
  double* red;
  int phase;
  // Options.
  const qtqp_options* o;
  // Banded backend (FMT == kFmtBand): A as CSR (ip, ix) and CSC (jp, jx),
  // P as CSR (pp, px) holding both triangles; the working (equilibrated)
  // values av / at / pv; the factor in lower band storage by columns,
  // Lb[j * (bw + 1) + (i - j)] = L_ij for j <= i <= j + bw.
  const int* ip;
  const int* ix;
  const int* jp;
  const int* jx;
  const int* pp;
  const int* px;
  const double* av0;
  const double* at0;
  const double* pv0;
  double* av;
  double* at;
  double* pv;
  double* Lb;
  int bw, nnz_a, nnz_p;
  // Shared-memory window of the banded factorisation and solves (null: the
  // band is too wide for it and the global-memory variants run).
  double* bwin;
  size_t bwin_bytes;
  // Banded backend in grid mode: the number of partitions of the columns,
  // the partitions' spikes, the separator blocks and the separator vectors.
  int nparts;
  double* bp_wl;
  double* bp_sep;
  double* bp_vec;
  // Supernodal factor of grid mode (FMT == kFmtSparse).
  const SnFactor* sn;

  // Grid mode (NT > 1024, FMT == kFmtLarge): the group is a cooperative grid
  // of NT / kGridBT blocks; barriers and reductions go through gctl.
  GridCtl* gctl;
  // Large format: padded sizes (multiples of 128 / 32), the factor in FP64
  // (g64) or FP32 (g32), both npad x npad row-major (lower triangle), the
  // inverses of its 128 x 128 diagonal blocks (linv, in the factor's
  // precision), the split TF32 operands X = (diag(1/sqrt(Ry)) A)^T
  // (xhi / xlo, npad x mpad), their tensor maps, the CTA's shared-memory
  // arena (tensor-core ring / staging tiles), its TMEM accumulator and the
  // per-thread pipeline counters of the tensor-core ring.
  int npad, mpad;
  int* linfo;  // factorisation status shared by the grid
  double* g64;
  float* g32l;
  double* linv;
  double* sinv;  // sub-block inverses of the current panel step
  double* colpart;  // per-block column sums of large_products (gridDim x npad)
  float* xhi;
  float* xlo;
  const void* map_hi;
  const void* map_lo;
  unsigned char* arena;
  uint32_t tmem;
  uint32_t tc_load, tc_mma, tc_tiles;
  uint32_t tri_gen;  // flag generations used by the whole-GPU triangular solves

  __device__ __forceinline__ void sync() const {
    if constexpr (NT > 1024) {
      grid_sync(gctl);
    } else {
      group_sync<NT>();
    }
  }
  template <int NS, int NM>
  __device__ __forceinline__ void reduce(double (&sums)[NS > 0 ? NS : 1],
                                         double (&maxs)[NM > 0 ? NM : 1]) {
    if constexpr (NT > 1024) {
      grid_reduce<kGridBT, NS, NM>(sums, maxs, red, gctl, phase);
    } else {
      block_reduce<NT, NS, NM>(sums, maxs, red, phase);
    }
  }

  __device__ __forceinline__ double* vec(int id) const { return V + size_t(id) * np; }
  // First index >= lo owned by this thread (k % NT == tid).  NT is a power of
  // two except for the large grid (one CTA per SM of a B200: 148 x 256).
  __device__ __forceinline__ int own(int lo) const {
    if constexpr ((NT & (NT - 1)) == 0) {
      return lo + ((tid - lo) & (NT - 1));
    } else {
      const int d = (tid - lo) % NT;
      return lo + (d < 0 ? d + NT : d);
    }
  }
  __device__ __forceinline__ float* g32() const { return reinterpret_cast<float*>(G); }

  // Lanes cooperating on one dot product when K outputs share the block.
  __device__ __forceinline__ int lanes_for(int K) const {
    int s = 1;
    while (s < 32 && K * s * 2 <= NT) s <<= 1;
    return s;
  }

  // out_k = sum_{i < len} body(k, i) for k < K, S = lanes_for(K) lanes per
  // output.  The S lanes of an output are strided across the warp (lane =
  // s * (32/S) + g) so that neighbouring lanes work on neighbouring outputs;
  // their partial sums are combined with xor shuffles, and lane s == 0 calls
  // epi(k, sum).  NACC independent sums per output.  No barrier inside.
  template <int NACC, bool MAXOP = false, int FORCE_S = 0, typename AccT = double,
            typename Body, typename Epi>
  __device__ __forceinline__ void rowdot(int K, int len, Body body, Epi epi) const {
    const int S = FORCE_S > 0 ? FORCE_S : lanes_for(K);
    const int per_warp = 32 / S;
    const int tid = this->tid;
    const int lane = tid & 31, warp = tid >> 5;
    const int s = lane / per_warp, g = lane - s * per_warp;
    const int per_pass = (NT / 32) * per_warp;
    for (int k0 = 0; k0 < K; k0 += per_pass) {
      const int k = k0 + warp * per_warp + g;
      AccT acc[NACC];
#pragma unroll
      for (int a = 0; a < NACC; ++a) acc[a] = AccT(0);
      if (k < K) {
        // U independent partial sums per lane keep U loads (and U FMA
        // chains) in flight: grid mode streams A and P from HBM; a block's
        // loads come from shared memory or L2.  The per-block dense format
        // keeps its loops short (one or two sums): its QPs are small, and
        // several blocks per SM run different phases of the IPM, whose code
        // then competes for the instruction cache (measured per block size:
        // 2-14 % faster at n = 16..64 than four sums).
        constexpr int U = NT > 1024                           ? 16
                          : (FMT == kFmtDense && NT <= 128)   ? 1
                          : FMT == kFmtDense                  ? 2
                                                              : QTQP_ROWDOT_UNROLL;
        AccT part[U][NACC];
#pragma unroll
        for (int u = 0; u < U; ++u)
#pragma unroll
          for (int a = 0; a < NACC; ++a) part[u][a] = AccT(0);
        int i = s;
        for (; i + (U - 1) * S < len; i += U * S) {
#pragma unroll
          for (int u = 0; u < U; ++u) body(k, i + u * S, part[u]);
        }
        for (; i < len; i += S) body(k, i, part[0]);
#pragma unroll
        for (int a = 0; a < NACC; ++a) {
          AccT t = part[0][a];
#pragma unroll
          for (int u = 1; u < U; ++u) t = MAXOP ? fmax(t, part[u][a]) : t + part[u][a];
          acc[a] = t;
        }
      }
#pragma unroll 1
      for (int off = 16; off >= per_warp; off >>= 1) {
#pragma unroll
        for (int a = 0; a < NACC; ++a) {
          const AccT o = __shfl_xor_sync(0xffffffffu, acc[a], off);
          acc[a] = MAXOP ? fmax(acc[a], o) : acc[a] + o;
        }
      }
      if (k < K && s == 0) epi(k, acc);
    }
  }
  // Lanes per output of a row dot (body reads element (k, j)): a whole warp
  // per output in grid mode (coalesced rows), the automatic split otherwise.
  static constexpr int kRowS = NT > 1024 ? 32 : 0;
  __device__ __forceinline__ float* t32() const { return reinterpret_cast<float*>(vec(kCT)); }

  // --------------------------------------------------------------------------
  // Binding of memory regions.
  // --------------------------------------------------------------------------
  __device__ void bind(int n_, int m_, char* smem, char* gmem, size_t smem_cap) {
    tid = threadIdx.x;
    n = n_;
    m = m_;
    N = n + m;
    const InstLayout L = plan_layout(n, m, smem_cap);
    lda = L.lda;
    ldp = L.ldp;
    ldg = L.ldg;
    np = L.np;
    char* gv = L.gv_smem ? smem : gmem;
    G = reinterpret_cast<double*>(gv);
    V = reinterpret_cast<double*>(gv + L.g_bytes);
    PB = V + size_t(kNumVec) * np;
    char* ap = L.ap_smem ? smem + L.g_bytes + L.v_bytes
                         : gmem + (L.gv_smem ? 0 : L.g_bytes + L.v_bytes);
    A = reinterpret_cast<double*>(ap);
    P = reinterpret_cast<double*>(ap + L.a_bytes);
  }

  // --------------------------------------------------------------------------
  // Ruiz equilibration (src/qtqp/__init__.py:616-663), done in place on the
  // working copies, bit-compatible with the reference: the nonzero a_ij is
  // multiplied by (d_i * e_j), the clip bounds are [1e-3, 1e3].
  // --------------------------------------------------------------------------
  QTQP_PHASE void load_and_equilibrate(bool equilibrate, double& nb, double& nc) {
    if constexpr (kSparseA) {
      band_load_and_equilibrate(equilibrate, nb, nc);
      return;
    }
    QTQP_LOCALS;
    double* de = vec(kDE);
    double* sc = vec(kTMP);  // per-sweep [e_i; d_i]
    const int warp = tid >> 5, lane = tid & 31;
    constexpr int NW = NT / 32;
    if (colmajor) {  // coalesced column reads; odd lda/ldp keep the stores conflict-free
      for (int j = warp; j < n; j += NW)
        for (int i = lane; i < m; i += 32) A[i * lda + j] = A0[size_t(j) * m + i];
      for (int j = warp; j < n; j += NW)
        for (int i = lane; i < n; i += 32) P[i * ldp + j] = has_p ? P0[size_t(j) * n + i] : 0.0;
    } else {
      for (int i = warp; i < m; i += NW)
        for (int j = lane; j < n; j += 32) A[i * lda + j] = A0[size_t(i) * n + j];
      for (int i = warp; i < n; i += NW)
        for (int j = lane; j < n; j += 32) P[i * ldp + j] = has_p ? P0[size_t(i) * n + j] : 0.0;
    }
    for (int k = tid; k < N; k += NT) de[k] = 1.0;
    sync();
    if (equilibrate) {
      const double* Ap = A;
      const double* Pp = P;
      const int la = lda, lp = ldp, mm = m, nn = n;
      const int plen = has_p ? n : 0;
      auto scale_of = [](double mx) {
        if (mx == 0.0) mx = 1.0;
        return fmin(fmax(1.0 / sqrt(mx), 1e-3), 1e3);
      };
      for (int sweep = 0; sweep < 10; ++sweep) {
        // Column maxima over A and P, row maxima over A.
        rowdot<1, true>(n, m + plen,
                        [&](int k, int i, double* acc) {
                          const double v = i < mm ? Ap[i * la + k] : Pp[(i - mm) * lp + k];
                          acc[0] = fmax(acc[0], fabs(v));
                        },
                        [&](int k, double* acc) { sc[k] = scale_of(acc[0]); });
        rowdot<1, true>(m, n,
                        [&](int k, int j, double* acc) {
                          acc[0] = fmax(acc[0], fabs(Ap[k * la + j]));
                        },
                        [&](int k, double* acc) { sc[nn + k] = scale_of(acc[0]); });
        sync();
        for (int i = warp; i < m; i += NW) {
          const double di = sc[n + i];
          for (int j = lane; j < n; j += 32) A[i * lda + j] *= di * sc[j];
        }
        if (has_p) {
          for (int i = warp; i < n; i += NW) {
            const double ei = sc[i];
            for (int j = lane; j < n; j += 32) P[i * ldp + j] *= ei * sc[j];
          }
        }
        for (int k = tid; k < N; k += NT) de[k] *= sc[k];
        sync();
      }
    }
    double* q = vec(kQ);
    double* pi = vec(kPI);
    double mx[2] = {0.0, 0.0};
    double dummy[1] = {0.0};
    for (int k = tid; k < N; k += NT) {
      if (k < n) {
        q[k] = c0[k] * de[k];
        pi[k] = P[k * ldp + k];  // diag(P_eq); P keeps only its off-diagonal
        P[k * ldp + k] = 0.0;
        mx[1] = nanmax(mx[1], fabs(c0[k]));
      } else {
        q[k] = b0[k - n] * de[k];
        mx[0] = nanmax(mx[0], fabs(b0[k - n]));
      }
    }
    reduce<0, 2>(dummy, mx);
    nb = mx[0];
    nc = mx[1];
    sync();
  }

  // --------------------------------------------------------------------------
  // DirectKktSolver.update (direct.py:183-216): true and regularised diagonal,
  // the backend's update_diag (solvers_dense.py:95-97) and the derived
  // 1/Ry and 1/sqrt(Ry) used by factorize/solve (solvers_dense.py:103, 132).
  // Owner-wise; the caller synchronises before factorising.
  // --------------------------------------------------------------------------
  __device__ void kkt_diag(double mu, double min_reg) {
    QTQP_LOCALS;
    const double* xy = vec(kXY);
    const double* s = vec(kRS);
    const double* pi = vec(kPI);
    double* reg = vec(kREG);
    double* corr = vec(kCORR);
    double* piw = vec(kPI);
    double* pw = vec(kPW);
    for (int k = tid; k < N; k += NT) {
      double t;
      if (k < n) {
        t = pi[k];
        t += mu;
      } else if (k < n + z) {
        t = mu;
      } else {
        t = s[k] / xy[k] + mu;
      }
      double r = fmax(t, min_reg);
      if (k >= n) {
        t = -t;
        r = -r;
        const double ry = -r;
        piw[k] = 1.0 / ry;
        pw[k] = 1.0 / sqrt(ry);
      }
      reg[k] = r;
      corr[k] = r - t;
    }
  }

  // Same for an externally supplied diagonal (the plugin's update_diag).
  __device__ void kkt_diag_given(const double* diag) {
    QTQP_LOCALS;
    double* reg = vec(kREG);
    double* piw = vec(kPI);
    double* pw = vec(kPW);
    for (int k = tid; k < N; k += NT) {
      const double r = diag[k];
      reg[k] = r;
      if (k >= n) {
        const double ry = -r;
        piw[k] = 1.0 / ry;
        pw[k] = 1.0 / sqrt(ry);
      }
    }
  }

  // --------------------------------------------------------------------------
  // factorize (solvers_dense.py:99-116): G = P_off + diag(Rx) + A_s^T A_s with
  // A_s = diag(1/sqrt(Ry)) A, a relative diagonal jitter, then Cholesky.
  // Returns 0 or the 1-based index of the first non-positive pivot.
  // Small n: the register-tiled path; otherwise Gram into memory + cholesky.
  // --------------------------------------------------------------------------
  template <typename T>
  QTQP_PHASE int factorize() {
    if constexpr (kSparseA) {
      return band_factorize<T>();
    } else if constexpr (FMT == kFmtLarge) {
      return large_factorize<T>(*this);
    } else {
      const int nb = (n + 3) >> 2;
      if (nb * (nb + 1) / 2 <= 2 * NT) return factorize_regs<T>();
      return factorize_mem<T>();
    }
  }

  // Register-tiled factorisation: each thread owns TPT (1 or 2) 4x4 tiles of
  // the lower triangle of G (tile t = tid + q NT, q < TPT); the Gram product
  // fills them (the FP64 one on the FP64 tensor cores through g, see
  // gram_dmma; the FP32 one on the registers), then tile_cholesky factors
  // them in place.  The finished L is written to G for the solves.
  template <typename T>
  __device__ int factorize_regs() {
    const int nb = (n + 3) >> 2;
    if (nb * (nb + 1) / 2 <= NT) return factorize_tiles<T, 1>();
    return factorize_tiles<T, 2>();
  }

  template <typename T, int TPT>
  __device__ int factorize_tiles() {
    QTQP_LOCALS;
    QTQP_TIC();
    T* g = reinterpret_cast<T*>(G);
    const double* reg = vec(kREG);
    const double* wsc = vec(kPW);
    const int nb = (n + 3) >> 2;
    const int tiles = nb * (nb + 1) / 2;
    bool mine[TPT];
    int bi[TPT], bj[TPT];
    T acc[TPT][4][4];
#pragma unroll
    for (int q = 0; q < TPT; ++q) {
      const int t = tid + q * NT;
      mine[q] = t < tiles;
      bi[q] = bj[q] = 0;
      if (mine[q]) {
        int b = int((sqrtf(8.0f * t + 1.0f) - 1.0f) * 0.5f);
        while (b * (b + 1) / 2 > t) --b;
        while ((b + 1) * (b + 2) / 2 <= t) ++b;
        bi[q] = b;
        bj[q] = t - b * (b + 1) / 2;
      }
#pragma unroll
      for (int a = 0; a < 4; ++a)
#pragma unroll
        for (int b = 0; b < 4; ++b) acc[q][a][b] = T(0);
    }
    if constexpr (sizeof(T) == 8) {
      // FP64 Gram on the FP64 tensor cores: each warp forms 8 x 8 lower
      // blocks of A^T diag(1/Ry) A with mma.sync m8n8k4 (DMMA) over 4-row
      // slices of A, writes them to g, and each thread then reads its tiles.
      gram_dmma(g);
#pragma unroll
      for (int q = 0; q < TPT; ++q) {
        if (!mine[q]) continue;
        const int i0 = bi[q] * 4, j0 = bj[q] * 4;
#pragma unroll
        for (int a = 0; a < 4; ++a)
#pragma unroll
          for (int b = 0; b < 4; ++b) {
            const int i = i0 + a, j = j0 + b;
            if (i < n && j <= i) acc[q][a][b] = g[i * ldg + j];
          }
      }
    } else {
#pragma unroll
      for (int q = 0; q < TPT; ++q) {
        if (!mine[q]) continue;
        const int i0 = bi[q] * 4, j0 = bj[q] * 4;
        for (int r = 0; r < m; ++r) {
          const double w = wsc[n + r];
          const double* row = A + r * lda;
          T ai[4], aj[4];
#pragma unroll
          for (int a = 0; a < 4; ++a) {
            ai[a] = (i0 + a < n) ? T(row[i0 + a] * w) : T(0);
            aj[a] = (j0 + a < n) ? T(row[j0 + a] * w) : T(0);
          }
#pragma unroll
          for (int a = 0; a < 4; ++a)
#pragma unroll
            for (int b = 0; b < 4; ++b) acc[q][a][b] = fma(ai[a], aj[b], acc[q][a][b]);
        }
      }
    }
    double dmax[1] = {0.0};
    double dummy[1] = {0.0};
#pragma unroll
    for (int q = 0; q < TPT; ++q) {
      if (!mine[q]) continue;
      const int i0 = bi[q] * 4, j0 = bj[q] * 4;
#pragma unroll
      for (int a = 0; a < 4; ++a) {
#pragma unroll
        for (int b = 0; b < 4; ++b) {
          const int i = i0 + a, j = j0 + b;
          if (i < n && j <= i) {
            double base = P[i * ldp + j];
            if (i == j) base += reg[i];
            acc[q][a][b] = T(base) + acc[q][a][b];
            if (i == j) dmax[0] = nanmax(dmax[0], double(acc[q][a][b]));
          }
        }
      }
    }
    reduce<0, 1>(dummy, dmax);
    const double jit = (sizeof(T) == 8 ? 1e-14 : 2.384185791015625e-07) * dmax[0];
#pragma unroll
    for (int q = 0; q < TPT; ++q)
#pragma unroll
      for (int a = 0; a < 4; ++a)
        if (mine[q] && bi[q] == bj[q] && bi[q] * 4 + a < n)
          acc[q][a][a] = T(double(acc[q][a][a]) + jit);
    QTQP_TOC(kPhGram);
    QTQP_RETIC();
    const int info = tile_cholesky<T, TPT>(acc, mine, bi, bj, g);
    QTQP_TOC(kPhChol);
    return info;
  }

  // Lower 8 x 8 blocks of the FP64 Gram A^T diag(1/Ry) A into g (entries
  // i >= j, i, j < n), one warp per block, on the FP64 tensor cores: for each
  // 4-row slice of A, lane l holds a = A[r + l%4][I + l/4] / Ry and
  // b = A[r + l%4][J + l/4] (dmma_8x8x4's fragment layout), rows past m and
  // columns past n are zero.  Ends with a barrier.
  __device__ __forceinline__ void gram_dmma(double* g) {
    QTQP_LOCALS;
    const double* iry = vec(kPI) + n;  // 1 / Ry
    const int lane = tid & 31, warp = tid >> 5;
    const int lr = lane & 3, lc = lane >> 2;
    const int n8 = (n + 7) >> 3;
    const int nblk = n8 * (n8 + 1) / 2;
    for (int t = warp; t < nblk; t += NT / 32) {
      int bi8 = int((sqrtf(8.0f * t + 1.0f) - 1.0f) * 0.5f);
      while (bi8 * (bi8 + 1) / 2 > t) --bi8;
      while ((bi8 + 1) * (bi8 + 2) / 2 <= t) ++bi8;
      const int bj8 = t - bi8 * (bi8 + 1) / 2;
      const int ci = bi8 * 8 + lc, cj = bj8 * 8 + lc;
      const bool ci_ok = ci < n, cj_ok = cj < n;
      double d[2] = {0.0, 0.0};
      int r = 0;
      // Four slices per step with their loads issued first (A may come from
      // L2 when it does not fit on chip); the products accumulate in the
      // same order as one slice at a time.
      for (; r + 16 <= m; r += 16) {
        double a[4], b[4];
#pragma unroll
        for (int u = 0; u < 4; ++u) {
          const int rr = r + 4 * u + lr;
          const double* row = A + rr * lda;
          a[u] = ci_ok ? row[ci] * iry[rr] : 0.0;
          b[u] = cj_ok ? row[cj] : 0.0;
        }
#pragma unroll
        for (int u = 0; u < 4; ++u) dmma_8x8x4(d, a[u], b[u]);
      }
      for (; r < m; r += 4) {
        const int rr = r + lr;
        double a = 0.0, b = 0.0;
        if (rr < m) {
          const double* row = A + rr * lda;
          if (ci_ok) a = row[ci] * iry[rr];
          if (cj_ok) b = row[cj];
        }
        dmma_8x8x4(d, a, b);
      }
      const int i = bi8 * 8 + lc, j = bj8 * 8 + 2 * lr;
      if (i < n) {
        if (j <= i) g[i * ldg + j] = d[0];
        if (j + 1 <= i) g[i * ldg + j + 1] = d[1];
      }
    }
    sync();
  }

  // Right-looking Cholesky of the register tiles of factorize_tiles in
  // 4-column panels, one barrier per panel.  Panel k's off-diagonal tiles
  // L_{i,k} = G_{i,k} L_kk^{-T} are published in the double-buffered panel
  // buffer PB; every tile right of panel k is then updated by the rank-4
  // product L_{i,k} L_{j,k}^T.  The 4 x 4 diagonal factor L_kk is formed by
  // each thread that owns a tile of panel k from the diagonal tile, which its
  // owner publishes in g (its own, not yet written, region of the factor) one
  // panel ahead, before its last update; each of them applies that update
  // itself in the owner's order, so all copies agree to the bit.  A
  // non-positive pivot is recorded in shared memory and stops every thread
  // after the panel's barrier.  The diagonal of the result keeps 1 / l_jj,
  // and every 32 x 32 diagonal block of L is inverted in place afterwards
  // (see chol_solve).  Returns 0 or the 1-based index of the first
  // non-positive pivot.
  template <typename T, int TPT>
  __device__ int tile_cholesky(T (&acc)[TPT][4][4], const bool (&mine)[TPT],
                               const int (&bi)[TPT], const int (&bj)[TPT], T* g) {
    QTQP_LOCALS;
    const int nb = (n + 3) >> 2;
    // Panel t's tiles (L values; exactly zero in rows and columns beyond n)
    // live in pb[t & 1] at 17 elements per tile.
    T* const pb0 = reinterpret_cast<T*>(PB);
    const int pstride = 17 * nb;
    // Lower entries of a diagonal tile into g (its own region).
    auto put_diag = [&](int t) {
#pragma unroll
      for (int q = 0; q < TPT; ++q) {
        if (!mine[q] || bi[q] != t || bj[q] != t) continue;
        const int i0 = bi[q] * 4, j0 = bj[q] * 4;
#pragma unroll
        for (int a = 0; a < 4; ++a)
#pragma unroll
          for (int b = 0; b < 4; ++b)
            if (b <= a && i0 + a < n) g[(i0 + a) * ldg + j0 + b] = acc[q][a][b];
      }
    };
    // The factor of diagonal tile t: D (as published, one update short when
    // t > 0) minus the rows of panel t-1, then the 4 x 4 Cholesky.  ld keeps
    // 1 / l on its diagonal.  Returns 0 or the failing 1-based column.
    auto diag_factor = [&](int t, T (&ld)[4][4]) -> int {
      T d[4][4];
      const int r0 = t * 4;
#pragma unroll
      for (int a = 0; a < 4; ++a)
#pragma unroll
        for (int b = 0; b < 4; ++b)
          d[a][b] = (b <= a && r0 + a < n) ? g[(r0 + a) * ldg + r0 + b] : T(0);
      if (t > 0) {  // the owner's last update, in the owner's order
        const T* pr = pb0 + ((t - 1) & 1) * pstride + t * 17;
#pragma unroll
        for (int c = 0; c < 4; ++c) {
          T l[4];
#pragma unroll
          for (int a = 0; a < 4; ++a) l[a] = pr[a * 4 + c];
#pragma unroll
          for (int a = 0; a < 4; ++a)
#pragma unroll
            for (int b = 0; b < 4; ++b) d[a][b] = fma(-l[a], l[b], d[a][b]);
        }
      }
#pragma unroll
      for (int c = 0; c < 4; ++c) {
#pragma unroll
        for (int a = 0; a < 4; ++a) ld[a][c] = T(0);
        if (r0 + c >= n) continue;
        const T piv = d[c][c];
        if (!(piv > T(0))) return r0 + c + 1;
        const T il = rsqrt(piv);
        ld[c][c] = il;
#pragma unroll
        for (int a = c + 1; a < 4; ++a) ld[a][c] = d[a][c] * il;
#pragma unroll
        for (int a = c + 1; a < 4; ++a)
#pragma unroll
          for (int b = c + 1; b <= a; ++b) d[a][b] = fma(-ld[a][c], ld[b][c], d[a][b]);
      }
      return 0;
    };
    // Tile q of panel t (already updated by panels < t) becomes
    // L_{i,t} = tile L_tt^{-T}, published in the panel buffer; the diagonal
    // tile becomes L_tt itself.
    auto finish_panel = [&](int q, int t, const T (&ld)[4][4]) {
      if (bi[q] == t) {
#pragma unroll
        for (int a = 0; a < 4; ++a)
#pragma unroll
          for (int c = 0; c < 4; ++c) acc[q][a][c] = ld[a][c];
        return;
      }
#pragma unroll
      for (int a = 0; a < 4; ++a) {
#pragma unroll
        for (int c = 0; c < 4; ++c) {
          T x = acc[q][a][c];
#pragma unroll
          for (int e = 0; e < c; ++e) x = fma(-acc[q][a][e], ld[c][e], x);
          acc[q][a][c] = x * ld[c][c];  // ld[c][c] = 1 / l_cc (0 beyond n)
        }
      }
      T* dst = pb0 + (t & 1) * pstride + bi[q] * 17;
#pragma unroll
      for (int a = 0; a < 4; ++a)
#pragma unroll
        for (int c = 0; c < 4; ++c) dst[a * 4 + c] = acc[q][a][c];
    };
    // Panel t for the tiles of this thread that belong to it.
    auto do_panel = [&](int t, int* s_info) {
      bool need = false;
#pragma unroll
      for (int q = 0; q < TPT; ++q) need = need || (mine[q] && bj[q] == t);
      if (!need) return;
      T ld[4][4];
      const int f = diag_factor(t, ld);
      if (f != 0) {
        *s_info = f;
        return;
      }
#pragma unroll
      for (int q = 0; q < TPT; ++q)
        if (mine[q] && bj[q] == t) finish_panel(q, t, ld);
    };
    __shared__ int s_info;
    if (tid == 0) s_info = 0;
    put_diag(0);
    put_diag(1);
    sync();
    do_panel(0, &s_info);
    sync();
    int info = s_info;
    for (int kb = 0; info == 0 && kb + 1 < nb; ++kb) {
#pragma unroll
      for (int q = 0; q < TPT; ++q) {
        if (!mine[q] || bj[q] <= kb) continue;
        // rank-4 update with panel kb, one column at a time
        const T* pi = pb0 + (kb & 1) * pstride + bi[q] * 17;
        const T* pj = pb0 + (kb & 1) * pstride + bj[q] * 17;
#pragma unroll
        for (int c = 0; c < 4; ++c) {
          T li[4], lj[4];
#pragma unroll
          for (int a = 0; a < 4; ++a) {
            li[a] = pi[a * 4 + c];
            lj[a] = pj[a * 4 + c];
          }
#pragma unroll
          for (int a = 0; a < 4; ++a)
#pragma unroll
            for (int b = 0; b < 4; ++b) acc[q][a][b] = fma(-li[a], lj[b], acc[q][a][b]);
        }
      }
      do_panel(kb + 1, &s_info);
      if (kb + 2 < nb) put_diag(kb + 2);
      sync();
      info = s_info;
    }
    if (info == 0) {
#pragma unroll
      for (int q = 0; q < TPT; ++q) {
        if (!mine[q]) continue;
        const int i0 = bi[q] * 4, j0 = bj[q] * 4;
#pragma unroll
        for (int a = 0; a < 4; ++a)
#pragma unroll
          for (int b = 0; b < 4; ++b) {
            const int i = i0 + a, j = j0 + b;
            if (i < n && j <= i) g[i * ldg + j] = acc[q][a][b];
          }
      }
    }
    sync();
    if (info == 0) invert_diag_blocks<T>(g);
    return info;
  }

  template <typename T>
  __device__ int factorize_mem() {
    QTQP_LOCALS;
    QTQP_TIC();
    T* g = reinterpret_cast<T*>(G);
    const double* reg = vec(kREG);
    const double* wsc = vec(kPW);
    const int nb = (n + 3) >> 2;
    const int tiles = nb * (nb + 1) / 2;
    double dmax[1] = {0.0};
    double dummy[1] = {0.0};
    for (int t = tid; t < tiles; t += NT) {
      int bi = int((sqrtf(8.0f * t + 1.0f) - 1.0f) * 0.5f);
      while (bi * (bi + 1) / 2 > t) --bi;
      while ((bi + 1) * (bi + 2) / 2 <= t) ++bi;
      const int bj = t - bi * (bi + 1) / 2;
      const int i0 = bi * 4, j0 = bj * 4;
      T acc[4][4];
#pragma unroll
      for (int a = 0; a < 4; ++a)
#pragma unroll
        for (int b = 0; b < 4; ++b) acc[a][b] = T(0);
      for (int r = 0; r < m; ++r) {
        const double w = wsc[n + r];
        const double* row = A + r * lda;
        T ai[4], aj[4];
#pragma unroll
        for (int a = 0; a < 4; ++a) {
          ai[a] = (i0 + a < n) ? T(row[i0 + a] * w) : T(0);
          aj[a] = (j0 + a < n) ? T(row[j0 + a] * w) : T(0);
        }
#pragma unroll
        for (int a = 0; a < 4; ++a)
#pragma unroll
          for (int b = 0; b < 4; ++b) acc[a][b] = fma(ai[a], aj[b], acc[a][b]);
      }
#pragma unroll
      for (int a = 0; a < 4; ++a) {
        const int i = i0 + a;
        if (i >= n) continue;
#pragma unroll
        for (int b = 0; b < 4; ++b) {
          const int j = j0 + b;
          if (j > i) continue;
          double base = P[i * ldp + j];
          if (i == j) base += reg[i];
          const T v = T(base) + acc[a][b];
          g[i * ldg + j] = v;
          if (i == j) dmax[0] = nanmax(dmax[0], double(v));
        }
      }
    }
    reduce<0, 1>(dummy, dmax);
    // FP64: the reference's 1e-14 relative jitter (solvers_dense.py:112).
    // FP32: the same idea at FP32 resolution (2^-22 relative).
    const double jit = (sizeof(T) == 8 ? 1e-14 : 2.384185791015625e-07) * dmax[0];
    for (int k = tid; k < n; k += NT) g[k * ldg + k] = T(double(g[k * ldg + k]) + jit);
    sync();
    QTQP_TOC(kPhGram);
    QTQP_RETIC();
    const int info = cholesky<T>(g);
    QTQP_TOC(kPhChol);
    return info;
  }

  // Right-looking Cholesky of the lower triangle, two barriers per column;
  // afterwards every 32x32 diagonal block of L is replaced by its inverse so
  // that the triangular solves are block-parallel (see chol_solve).
  //
  // One barrier per column: phase k updates the trailing matrix with the
  // still-unscaled column k (a_ij -= a_ik a_jk / d_k) and, independently,
  // finishes column k-1 (l_ik = a_ik / sqrt(d_{k-1}), l_kk = sqrt(d_{k-1})),
  // which phase k does not read.
  template <typename T>
  QTQP_PHASE int cholesky(T* g) {
    QTQP_LOCALS;
    const int warp = tid >> 5, lane = tid & 31;
    constexpr int NW = NT / 32;
    T il_prev = T(1);  // 1 / sqrt(d) of the previous pivot
    for (int k = 0; k <= n; ++k) {
      if (k > 0) {  // finish column k-1
        const T inv = il_prev;
        for (int i = k + tid; i < n; i += NT) g[i * ldg + k - 1] *= inv;
        if (tid == NT - 1) g[(k - 1) * ldg + k - 1] = inv;  // diagonal keeps 1/l_kk
      }
      if (k == n) break;
      const T d = g[k * ldg + k];
      if (!(d > T(0))) {
        sync();
        return k + 1;
      }
      // One reciprocal square root per pivot, no divisions on this chain:
      // 1 / l_kk = rsqrt(d), 1 / d = (1 / l_kk)^2.
      const T il = rsqrt(d);
      const T inv_d = il * il;
      for (int j = k + 1 + warp; j < n; j += NW) {
        const T t = g[j * ldg + k] * inv_d;
        for (int i = j + lane; i < n; i += 32) g[i * ldg + j] = fma(-g[i * ldg + k], t, g[i * ldg + j]);
      }
      il_prev = il;
      sync();
    }
    sync();
    invert_diag_blocks<T>(g);
    return 0;
  }

  // In-place inverse of each 32x32 lower-triangular diagonal block of L,
  // top-down: X_cc = 1 / L_cc, X_rc = -(sum_{c<=k<r} L_rk X_kc) / L_rr for
  // r > c.  Both Cholesky variants already store 1 / L_jj on the diagonal,
  // which is also the inverse's diagonal.  Column c of X keeps X_kc (k > c)
  // in the block's unused upper triangle at (c, k), so with the diagonal
  // U_ck = X_kc for every k >= c; L_rk is the same entry for every column (a
  // broadcast).  A block gets a team of P warps (P = 1, 2 or 4, as many as
  // the block's warps allow) and each column P neighbouring lanes of one
  // warp, which split the row's dot product (strided over k, combined by
  // xor shuffles), so the columns of a warp need no barrier but __syncwarp.
  // The loops stay rolled: the batch kernel runs several QPs per SM at
  // different phases of the IPM, and their code competes for the
  // instruction cache.  After a barrier the columns are copied from the
  // upper triangles into the lower ones.
  template <typename T>
  QTQP_PHASE void invert_diag_blocks(T* g) {
    QTQP_LOCALS;
    QTQP_TIC();
    const int warp = tid >> 5, lane = tid & 31;
    constexpr int NW = NT / 32;
    const int nblk = (n + 31) >> 5;
    int lanes = 1;  // P, the lanes per column
    while (lanes < 4 && 2 * lanes * nblk <= NW) lanes <<= 1;
    const int teams = NW / lanes, team = warp / lanes;
    const int c = (warp % lanes) * (32 / lanes) + lane / lanes, sub = lane % lanes;
    for (int blk = team; blk < nblk; blk += teams) {
      const int kb = blk * 32, bs = min(32, n - kb);
      T* L = g + kb * ldg + kb;
      T* U = L + c * ldg;  // row c: U[k] = X_kc for k >= c
#pragma unroll 1
      for (int r = 1; r < bs; ++r) {
        const T* Lr = L + r * ldg;
        T acc = T(0);
        // Four entries per lane and step, loads issued ahead of the FMAs.
#pragma unroll 1
        for (int k0 = c + sub; k0 < r; k0 += 4 * lanes) {
          T lv[4], uv[4];
#pragma unroll
          for (int u = 0; u < 4; ++u) {
            const int k = k0 + u * lanes;
            lv[u] = k < r ? Lr[k] : T(0);
            uv[u] = k < r ? U[k] : T(0);
          }
#pragma unroll
          for (int u = 0; u < 4; ++u) acc = fma(lv[u], uv[u], acc);
        }
        for (int o = 1; o < lanes; o <<= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
        if (sub == 0 && c < r) U[r] = -acc * Lr[r];
        __syncwarp();
      }
    }
    // Every column reads row r of L up to r - 1, including the columns of
    // the team's other warps, so the copy waits for all of them.
    sync();
    for (int blk = team; blk < nblk; blk += teams) {
      const int kb = blk * 32, bs = min(32, n - kb);
      T* L = g + kb * ldg + kb;
      const T* U = L + c * ldg;
#pragma unroll 1
      for (int r = c + 1 + sub; r < bs; r += lanes) L[r * ldg + c] = U[r];
    }
    sync();
    QTQP_TOC(kPhInv);
  }

  // Solves L L^T v = v in place with the block-inverted factor: forward
  // z_b = X_bb (v_b - sum_{c<b} L_bc z_c), backward x_b = X_bb^T (z_b -
  // sum_{c>b} L_cb^T x_c), two barriers per 32-block; w is n scratch entries.
  // Each phase is a set of row dots (rowdot: several lanes per row, partial
  // sums combined by shuffles), so no thread walks a 32-long chain alone.
  template <typename T>
  QTQP_PHASE void chol_solve(const T* g, T* v, T* w) {
    if constexpr (FMT == kFmtLarge) {
      large_chol_solve<T>(*this, v, w);
      return;
    }
    QTQP_LOCALS;
    const int nblk = (n + 31) >> 5;
    for (int blk = 0; blk < nblk; ++blk) {
      const int kb = blk * 32, bs = min(32, n - kb);
      const T* gb = g + kb * ldg + kb;
      rowdot<1, false, 0, T>(bs, bs,
                [&](int r, int k, T* acc) {
                  if (k <= r) acc[0] = fma(gb[r * ldg + k], v[kb + k], acc[0]);
                },
                [&](int r, T* acc) { w[kb + r] = acc[0]; });
      sync();
      if (kb + bs < n) {
        const T* gl = g + (kb + bs) * ldg + kb;
        rowdot<1, false, 0, T>(n - kb - bs, bs,
                  [&](int i, int k, T* acc) {
                    acc[0] = fma(gl[i * ldg + k], w[kb + k], acc[0]);
                  },
                  [&](int i, T* acc) { v[kb + bs + i] -= acc[0]; });
        sync();
      }
    }
    for (int blk = nblk - 1; blk >= 0; --blk) {
      const int kb = blk * 32, bs = min(32, n - kb);
      const T* gb = g + kb * ldg + kb;
      rowdot<1, false, 0, T>(bs, bs,
                [&](int r, int k, T* acc) {
                  if (k >= r) acc[0] = fma(gb[k * ldg + r], w[kb + k], acc[0]);
                },
                [&](int r, T* acc) { v[kb + r] = acc[0]; });
      sync();
      if (kb > 0) {
        const T* gc = g + kb * ldg;
        rowdot<1, false, 0, T>(kb, bs,
                  [&](int i, int k, T* acc) {
                    acc[0] = fma(gc[k * ldg + i], v[kb + k], acc[0]);
                  },
                  [&](int i, T* acc) { w[i] -= acc[0]; });
        sync();
      }
    }
  }

  // --------------------------------------------------------------------------
  // Backend solve (solvers_dense.py:130-142): out (+)= K_reg^{-1} r.
  // Entry: r complete (barrier passed).  Exit: out written (barrier needed
  // before other threads read it).
  // --------------------------------------------------------------------------
  QTQP_PHASE void kkt_solve(const double* r, double* out, bool accumulate, bool fp64) {
    if constexpr (kSparseA) {
      band_kkt_solve(r, out, accumulate, fp64);
      return;
    }
    QTQP_LOCALS;
    QTQP_TIC();
    const double* iry = vec(kPI);
    double* tmp = vec(kTMP);
    float* t32 = this->t32();
    const double* Ap = A;
    const int ld = lda, nn = n;
    // g = r_x + A^T (r_y / Ry)
    auto put_g = [&](int k, double g) {
      if (fp64) {
        tmp[k] = g;
      } else {
        t32[k] = float(g);
      }
    };
    // (In grid mode a lane group per column streams A with many loads in
    // flight; a row pass with per-block column sums measured slower here,
    // where no row dot rides along.)
    {
      QTQP_TIC();
      if constexpr (FMT == kFmtLarge) {
        large_products(*this, nullptr, r + n, iry + n, nullptr, [](int, double) {},
                       [&](int k, double cs) { put_g(k, r[k] + cs); });
      } else {
        rowdot<1>(n, m,
                  [&](int k, int i, double* acc) {
                    acc[0] = fma(Ap[i * ld + k], iry[nn + i] * r[nn + i], acc[0]);
                  },
                  [&](int k, double* acc) { put_g(k, r[k] + acc[0]); });
      }
      sync();
      QTQP_TOC(kPhSolveCols);
    }
    {
      QTQP_TIC();
      if (fp64) {
        chol_solve<double>(G, tmp, vec(kW));
      } else {
        chol_solve<float>(g32(), t32, t32 + n);
      }
      QTQP_TOC(kPhTri);
    }
    for (int k = tid; k < n; k += NT) {
      const double val = fp64 ? tmp[k] : double(t32[k]);
      out[k] = accumulate ? out[k] + val : val;
    }
    // y = (A x - r_y) / Ry
    {
      QTQP_TIC();
      rowdot<1, false, kRowS>(m, n,
                [&](int k, int j, double* acc) {
                  const double xj = fp64 ? tmp[j] : double(t32[j]);
                  acc[0] = fma(Ap[k * ld + j], xj, acc[0]);
                },
                [&](int k, double* acc) {
                  const double val = iry[nn + k] * (acc[0] - r[nn + k]);
                  out[nn + k] = accumulate ? out[nn + k] + val : val;
                });
      QTQP_TOC(kPhSolveRows);
    }
    QTQP_TOC(kPhSolve);
  }

  // One pass over A (and P) for the products a dense block needs together,
  // for n <= 64: the column sums c_k = sum_{i<m} A_ik wy_i + sum_{i<n} P_ik
  // wp_i (k < n; the P part only when has_p and wp is given), staged per warp
  // in the panel buffer PB
  // (PB[w * n + k]; the caller sums the warps' rows after a barrier), and
  // the row products (A vx)_i, passed to row_epi(i, value) by one lane each.
  // Each warp takes 16 rows of A at a time, lane l columns l and l + 32; the
  // 16 row sums are reduced across the warp in 16 shuffles (each step sends
  // half of the values to the partner lane and keeps the other half).
  static constexpr bool kFused = FMT == kFmtDense && NT <= 1024;
  __device__ __forceinline__ bool fused_ok() const { return kFused && n <= 64; }
  template <typename RowEpi>
  __device__ void fused_products(const double* vx, const double* wy, const double* wp,
                                 RowEpi row_epi) const {
    QTQP_LOCALS;
    constexpr int NW = NT / 32;
    const int lane = tid & 31, warp = tid >> 5;
    const int c0 = lane, c1 = lane + 32;
    const bool ok0 = c0 < n, ok1 = c1 < n;
    const double x0 = ok0 ? vx[c0] : 0.0, x1 = ok1 ? vx[c1] : 0.0;
    double cs0 = 0.0, cs1 = 0.0;
    const int rsel = ((lane >> 4) & 1) * 8 + ((lane >> 3) & 1) * 4 + ((lane >> 2) & 1) * 2 +
                     ((lane >> 1) & 1);  // the row of the 16 this lane ends with
    for (int base = warp * 16; base < m; base += NW * 16) {
      double t[16];
#pragma unroll
      for (int r = 0; r < 16; ++r) {
        const int i = base + r;
        double a0 = 0.0, a1 = 0.0, w = 0.0;
        if (i < m) {
          const double* row = A + i * lda;
          a0 = ok0 ? row[c0] : 0.0;
          a1 = ok1 ? row[c1] : 0.0;
          w = wy[i];
        }
        cs0 = fma(a0, w, cs0);
        cs1 = fma(a1, w, cs1);
        t[r] = fma(a0, x0, a1 * x1);
      }
#pragma unroll
      for (int half = 8, bit = 16; half >= 1; half >>= 1, bit >>= 1) {
        const bool hi = (lane & bit) != 0;
#pragma unroll
        for (int j = 0; j < half; ++j) {
          const double send = hi ? t[j] : t[j + half];
          const double keep = hi ? t[j + half] : t[j];
          t[j] = keep + __shfl_xor_sync(0xffffffffu, send, bit);
        }
      }
      t[0] += __shfl_xor_sync(0xffffffffu, t[0], 1);
      const int i = base + rsel;
      if ((lane & 1) == 0 && i < m) row_epi(i, t[0]);
    }
    if (has_p && wp != nullptr) {
      for (int i = warp; i < n; i += NW) {
        const double* row = P + i * ldp;
        const double w = wp[i];
        if (ok0) cs0 = fma(row[c0], w, cs0);
        if (ok1) cs1 = fma(row[c1], w, cs1);
      }
    }
    double* stage = PB + warp * n;
    if (ok0) stage[c0] = cs0;
    if (ok1) stage[c1] = cs1;
  }
  // Column sum k of fused_products (after a barrier).
  __device__ __forceinline__ double fused_colsum(int k) const {
    constexpr int NW = NT / 32;
    double t = 0.0;
#pragma unroll
    for (int w = 0; w < NW; ++w) t += PB[w * n + k];
    return t;
  }

  // res = krhs - K_reg v + corr o v (direct.py:256, 266 with the matvec of
  // solvers_dense.py:118-128).  Reads all of v; returns this thread's partial
  // max |res| and NaN flag of v (combined by the caller's reduction).
  QTQP_PHASE void kkt_residual(const double* v, const double* krhs, double* res, double& mres,
                               double& vnan) const {
    if constexpr (kSparseA) {
      band_kkt_residual(v, krhs, res, mres, vnan);
      return;
    }
    QTQP_LOCALS;
    if (fused_ok()) {
      const double* reg = vec(kREG);
      const double* corr = vec(kCORR);
      fused_products(v, v + n, v, [&](int i, double ax) {
        const int kk = n + i;
        const double kv = ax - (-reg[kk]) * v[kk];
        const double rk = krhs[kk] - kv + corr[kk] * v[kk];
        res[kk] = rk;
        mres = nanmax(mres, fabs(rk));
        vnan = fmax(vnan, (v[kk] != v[kk]) ? 1.0 : 0.0);
      });
      sync();
      for (int k = tid; k < n; k += NT) {
        const double kv = fused_colsum(k) + reg[k] * v[k];
        const double rk = krhs[k] - kv + corr[k] * v[k];
        res[k] = rk;
        mres = nanmax(mres, fabs(rk));
        vnan = fmax(vnan, (v[k] != v[k]) ? 1.0 : 0.0);
      }
      return;
    }
    const double* reg = vec(kREG);
    const double* corr = vec(kCORR);
    if constexpr (FMT == kFmtLarge) {
      // One pass over A (and P): row dots A v_x and column sums
      // A^T v_y + P v_x (large_ipm.cuh); the column epilogue runs after a
      // grid barrier, in the thread that owns column k.
      const int nn = n;
      large_products(*this, v, v + n, nullptr, has_p ? v : nullptr,
                     [&](int i, double ax) {
                       const int kk = nn + i;
                       const double kv = ax - (-reg[kk]) * v[kk];
                       const double rk = krhs[kk] - kv + corr[kk] * v[kk];
                       res[kk] = rk;
                       mres = nanmax(mres, fabs(rk));
                       vnan = fmax(vnan, (v[kk] != v[kk]) ? 1.0 : 0.0);
                     },
                     [&](int k, double cs) {
                       const double kv = cs + reg[k] * v[k];
                       const double rk = krhs[k] - kv + corr[k] * v[k];
                       res[k] = rk;
                       mres = nanmax(mres, fabs(rk));
                       vnan = fmax(vnan, (v[k] != v[k]) ? 1.0 : 0.0);
                     });
      return;
    }
    const double* Ap = A;
    const double* Pp = P;
    const int la = lda, lp = ldp, nn = n, mm = m;
    const int plen = has_p ? n : 0;
    rowdot<2>(n, m + plen,
              [&](int k, int i, double* acc) {
                if (i < mm) {
                  acc[1] = fma(Ap[i * la + k], v[nn + i], acc[1]);
                } else {
                  acc[0] = fma(Pp[(i - mm) * lp + k], v[i - mm], acc[0]);
                }
              },
              [&](int k, double* acc) {
                double t = acc[0];
                t += reg[k] * v[k];
                const double kv = t + acc[1];
                const double rk = krhs[k] - kv + corr[k] * v[k];
                res[k] = rk;
                mres = nanmax(mres, fabs(rk));
                vnan = fmax(vnan, (v[k] != v[k]) ? 1.0 : 0.0);
              });
    rowdot<1, false, kRowS>(m, n,
              [&](int k, int j, double* acc) { acc[0] = fma(Ap[k * la + j], v[j], acc[0]); },
              [&](int k, double* acc) {
                const int kk = nn + k;
                const double kv = acc[0] - (-reg[kk]) * v[kk];
                const double rk = krhs[kk] - kv + corr[kk] * v[kk];
                res[kk] = rk;
                mres = nanmax(mres, fabs(rk));
                vnan = fmax(vnan, (v[kk] != v[kk]) ? 1.0 : 0.0);
              });
  }

  // K_reg x (solvers_dense.py:118-128), written to out.
  __device__ void kkt_matvec(const double* v, double* out) const {
    QTQP_LOCALS;
    const double* reg = vec(kREG);
    const double* Ap = A;
    const double* Pp = P;
    const int la = lda, lp = ldp, nn = n, mm = m;
    rowdot<2>(n, m + n,
              [&](int k, int i, double* acc) {
                if (i < mm) {
                  acc[1] = fma(Ap[i * la + k], v[nn + i], acc[1]);
                } else {
                  acc[0] = fma(Pp[(i - mm) * lp + k], v[i - mm], acc[0]);
                }
              },
              [&](int k, double* acc) {
                double t = acc[0];
                t += reg[k] * v[k];
                out[k] = t + acc[1];
              });
    rowdot<1>(m, n,
              [&](int k, int j, double* acc) { acc[0] = fma(Ap[k * la + j], v[j], acc[0]); },
              [&](int k, double* acc) { out[nn + k] = acc[0] - (-reg[nn + k]) * v[nn + k]; });
  }

  // The KKT right-hand side of a solve into vec(kRHS): krhs[k] = rhs_k(k),
  // negated on the dual block (k >= n), owner-wise (k % NT == tid).
  template <typename RhsF>
  __device__ __forceinline__ void set_rhs(RhsF rhs_k) {
    double* krhs = vec(kRHS);
    for (int k = tid; k < N; k += NT) {
      const double r = rhs_k(k);
      krhs[k] = k >= n ? -r : r;
    }
  }

  // --------------------------------------------------------------------------
  // DirectKktSolver.solve (direct.py:218-307).  The right-hand side is in
  // vec(kRHS) (set_rhs, written owner-wise by this thread); `sol` holds the
  // warm start and receives the solution.  Entry: sol complete (barrier
  // passed).  One copy of this function serves every solve of an iteration,
  // which keeps the per-iteration code small for the instruction cache.
  // --------------------------------------------------------------------------
  QTQP_PHASE IrOutcome ir_solve(double* sol, bool fp64) {
    const qtqp_options& op = *o;
    const double* krhs = vec(kRHS);
    double* res = vec(kRES);
    double dummy[1] = {0.0};
    IrOutcome out;
    {
      double mx[3] = {0.0, 0.0, 0.0};  // |rhs|, |res|, nan(sol)
      for (int k = tid; k < N; k += NT) mx[0] = nanmax(mx[0], fabs(krhs[k]));
      sync();
      QTQP_TIC();
      kkt_residual(sol, krhs, res, mx[1], mx[2]);
      // The reduction's barrier also orders every thread's res writes before
      // the solve that reads them.
      reduce<0, 3>(dummy, mx);
      if constexpr (NT <= 1024) {
        if (NT / 32 == 1) sync();  // a one-warp reduction has no barrier
      } else {
        sync();
      }
      QTQP_TOC(kPhResidual);
      out.rhs_norm = mx[0];
      out.final_res = mx[1];
    }
    out.tol = op.linear_solver_atol + op.linear_solver_rtol * out.rhs_norm;
    out.status = 0;
    out.solves = 0;
    out.nan = false;
    double rn = out.final_res;
    for (int it = 1; it <= op.max_iterative_refinement_steps; ++it) {
      out.solves = it;
      const double prev = rn;
      kkt_solve(res, sol, true, fp64);
      sync();
      QTQP_TIC();
      double mx[2] = {0.0, 0.0};
      kkt_residual(sol, krhs, res, mx[0], mx[1]);
      reduce<0, 2>(dummy, mx);  // its barrier orders the res writes (as above)
      if constexpr (NT <= 1024) {
        if (NT / 32 == 1) sync();
      } else {
        sync();
      }
      QTQP_TOC(kPhResidual);
      rn = mx[0];
      out.nan = mx[1] > 0.0;
      if (rn < out.tol) {
        out.status = 1;
        break;
      }
      if (rn >= prev) {
        out.status = 2;
        break;
      }
    }
    out.final_res = rn;
    return out;
  }

  // IR with the mixed-precision policy: an FP32 factor whose refinement does
  // not converge is replaced by an FP64 factor (kept for the rest of the
  // solve) and the refinement is redone from the same warm start, so the
  // outcome is the one the plain FP64 path would produce.
  // `warm` is the warm start (a vector that the solve leaves unchanged); the
  // right-hand side is set once and kept in vec(kRHS) for the second try.
  template <typename RhsF>
  __device__ IrOutcome ir_solve_policy(RhsF rhs_k, const double* warm, double* sol, bool& fp64,
                                       int& n32, int& n64, int& err) {
    set_rhs(rhs_k);
    for (int k = tid; k < N; k += NT) sol[k] = warm[k];
    sync();
    IrOutcome r = ir_solve(sol, fp64);
    if (!fp64 && r.status != 1) {
      fp64 = true;
      ++n64;
      const int info = factorize<double>();
      if (info != 0) {
        err = QTQP_ERR_NOT_SPD;
        return r;
      }
      for (int k = tid; k < N; k += NT) sol[k] = warm[k];
      sync();
      r = ir_solve(sol, fp64);
    }
    return r;
  }

  // --------------------------------------------------------------------------
  // tau+ of the homogeneous embedding: the quadratic root
  // (__init__.py:759-817) or, when the KKT solve was not accurate or the
  // quadratic fails, the linearised update (__init__.py:819-857).
  // `kr` is K^{-1} r (complete).  Per-iteration constants come in `it`.
  // --------------------------------------------------------------------------
  struct IterConsts {
    double kqq;    // K^{-1}q . q
    double kqpkq;  // (K^{-1}q)_x . P (K^{-1}q)_x
    double qz;     // q_x . x + q_y . y
    double xpx;    // x . P x
    double pxkq;   // P x . (K^{-1}q)_x
  };

  QTQP_PHASE double tau_step(const double* kr, const IrOutcome& irr, double mu, double mu_t,
                             double r_tau, double tau, double tau_anchor, const IterConsts& ic,
                             int& method) {
    QTQP_LOCALS;
    const double* q = vec(kQ);
    const double* kq = vec(kKQ);
    const double* pkq = vec(kPW);
    const double* px = vec(kXD);
    const double* pi = vec(kPI);
    double* pkr = vec(kRS);
    double sm[5] = {0.0, 0.0, 0.0, 0.0, 0.0};  // kr.q, kr.Pkq, kq.Pkr, kr.Pkr, Px.kr
    double dummy[1] = {0.0};
    for (int k = tid; k < N; k += NT) sm[0] = fma(kr[k], q[k], sm[0]);
    if (has_p) {
      auto epi = [&](int k, double poff) {
        const double t = fma(pi[k], kr[k], poff);
        pkr[k] = t;
        sm[1] = fma(kr[k], pkq[k], sm[1]);
        sm[2] = fma(kq[k], t, sm[2]);
        sm[3] = fma(kr[k], t, sm[3]);
        sm[4] = fma(px[k], kr[k], sm[4]);
      };
      if constexpr (kSparseA) {
        for (int k = tid; k < n; k += NT) epi(k, band_poff_row(kr, k));
      } else {
        const double* Pp = P;
        const int lp = ldp;
        rowdot<1>(n, n,
                  [&](int k, int j, double* acc) { acc[0] = fma(Pp[j * lp + k], kr[j], acc[0]); },
                  [&](int k, double* acc) { epi(k, acc[0]); });
      }
    }
    reduce<5, 0>(sm, dummy);
    const bool accurate = irr.status == 1 || irr.final_res < 1e-7;
    if (o->tau_mode == 0 && accurate) {
      double ta = mu + ic.kqq;
      double tb = -r_tau - sm[0];
      double tc = -mu_t;
      if (has_p) {
        ta -= ic.kqpkq;
        tb += sm[1] + sm[2];
        tc -= sm[3];
      }
      double root = 0.0;
      bool ok = true;
      if (fabs(ta) < kEps) {
        if (fabs(tb) < kEps) {
          ok = false;
        } else {
          root = -tc / tb;
          ok = isfinite(root) && !(root < -1e-10);
        }
      } else {
        double disc = tb * tb - 4.0 * ta * tc;
        if (disc < -1e-9) {
          ok = false;
        } else {
          disc = fmax(0.0, disc);
          if (tb > 0.0) {
            root = tc / (-0.5 * (tb + sqrt(disc)));
          } else {
            root = (-0.5 * (tb - sqrt(disc))) / ta;
          }
          ok = isfinite(root) && !(root < -1e-10);
        }
      }
      if (ok) {
        method = 0;
        return fmax(0.0, root);
      }
    }
    method = 1;
    const double q_rz = sm[0] - tau * ic.kqq - ic.qz;
    const double px_rz = (has_p ? sm[4] : 0.0) - tau * ic.pxkq - ic.xpx;
    const double g = mu * tau * tau + (mu_t - mu) * tau_anchor * tau - tau * ic.qz - mu_t - ic.xpx;
    const double num = g - tau * q_rz - 2.0 * px_rz;
    const double den =
        2.0 * mu * tau + (mu_t - mu) * tau_anchor - ic.qz + tau * ic.kqq + 2.0 * ic.pxkq;
    const double root = tau + (fabs(den) < 1e-16 ? 0.0 : -num / den);
    if (!isfinite(root)) return tau;
    return fmin(fmax(root, 0.1 * tau), 10.0 * tau);
  }

  // Ratio test (__init__.py:671-680, 882-886) over the inequality block for
  // the step (dy, ds) given owner-wise by `dir(k, dy, ds)`.
  template <typename DirF>
  __device__ double step_to_boundary(DirF dir) {
    QTQP_LOCALS;
    const double* xy = vec(kXY);
    const double* s = vec(kRS);
    double mx[1] = {-1.0};  // max of -alpha candidates == -(min alpha)
    double dummy[1] = {0.0};
    for (int k = own(n + z); k < N; k += NT) {
      double dy, ds;
      dir(k, dy, ds);
      if (ds < -kEps) mx[0] = fmax(mx[0], -(-s[k] / ds));
      if (dy < -kEps) mx[0] = fmax(mx[0], -(-xy[k] / dy));
    }
    reduce<0, 1>(dummy, mx);
    return fmin(1.0, -mx[0]);
  }

  // --------------------------------------------------------------------------
  // _check_termination (__init__.py:888-1008) on the unequilibrated iterate,
  // computed from the equilibrated products: A_o x_o = (A_eq x)/d,
  // A_o^T y_o = (A_eq^T y)/e, P_o x_o = (P_eq x)/e.
  // --------------------------------------------------------------------------
  QTQP_PHASE int termination(double tau, double nb, double nc, double* st, bool collect) {
    QTQP_LOCALS;
    const qtqp_options& op = *o;
    const double* xy = vec(kXY);
    const double* s = vec(kRS);
    const double* de = vec(kDE);
    const double* pi = vec(kPI);
    const double inv_tau = 1.0 / fmax(tau, kEps);
    // sums: ctx, bty, xpx ; maxes: pres, dres, |aty|, |px|, |ax+s|, |ax|, |s|, |x|, |y|
    double sm[3] = {0.0, 0.0, 0.0};
    double mx[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
    const double* Ap = A;
    const double* Pp = P;
    const int la = lda, lp = ldp, nn = n, mm = m;
    const int plen = has_p ? n : 0;
    const bool hp = has_p;
    const double* b0p = b0;
    const double* c0p = c0;
    auto epi_x = [&](int k, double aty_raw, double poff) {
      const double aty = aty_raw / de[k];
      const double px = hp ? fma(pi[k], xy[k], poff) / de[k] : 0.0;
      const double xo = de[k] * xy[k];
      sm[0] = fma(c0p[k], xo, sm[0]);
      sm[2] = fma(xo, px, sm[2]);
      mx[1] = nanmax(mx[1], fabs((px + aty) * inv_tau + c0p[k]));
      mx[2] = nanmax(mx[2], fabs(aty));
      mx[3] = nanmax(mx[3], fabs(px));
      mx[7] = nanmax(mx[7], fabs(xo));
    };
    auto epi_y = [&](int k, double ax_raw) {
      const int kk = nn + k;
      const double ax = ax_raw / de[kk];
      const double yo = de[kk] * xy[kk];
      const double so = s[kk] / de[kk];
      const double bo = b0p[k];
      sm[1] = fma(bo, yo, sm[1]);
      mx[0] = nanmax(mx[0], fabs((ax + so) * inv_tau - bo));
      mx[4] = nanmax(mx[4], fabs(ax + so));
      mx[5] = nanmax(mx[5], fabs(ax));
      mx[6] = nanmax(mx[6], fabs(so));
      mx[8] = nanmax(mx[8], fabs(yo));
    };
    if constexpr (kSparseA) {
      for (int k = tid; k < n; k += NT) epi_x(k, band_at_col(xy, k), band_poff_row(xy, k));
      for (int k = tid; k < m; k += NT) epi_y(k, band_a_row(xy, k));
    } else if (fused_ok()) {
      // A^T y and A x in one pass over A; P x as row dots.  P x goes to the
      // panel buffer behind the warps' staged column sums.
      double* pxs = PB + (NT / 32) * n;
      if (hp) {
        rowdot<1>(n, n,
                  [&](int k, int i, double* acc) { acc[0] = fma(Pp[i * lp + k], xy[i], acc[0]); },
                  [&](int k, double* acc) { pxs[k] = acc[0]; });
      }
      fused_products(xy, xy + nn, nullptr, [&](int i, double ax) { epi_y(i, ax); });
      sync();
      for (int k = tid; k < n; k += NT) epi_x(k, fused_colsum(k), hp ? pxs[k] : 0.0);
    } else {
      rowdot<2>(n, m + plen,
                [&](int k, int i, double* acc) {
                  if (i < mm) {
                    acc[0] = fma(Ap[i * la + k], xy[nn + i], acc[0]);
                  } else {
                    acc[1] = fma(Pp[(i - mm) * lp + k], xy[i - mm], acc[1]);
                  }
                },
                [&](int k, double* acc) { epi_x(k, acc[0], acc[1]); });
      rowdot<1, false, kRowS>(m, n, [&](int k, int j, double* acc) { acc[0] = fma(Ap[k * la + j], xy[j], acc[0]); },
                [&](int k, double* acc) { epi_y(k, acc[0]); });
    }
    reduce<3, 9>(sm, mx);
    const double ctx = sm[0], bty = sm[1], xpx = has_p ? sm[2] : 0.0;
    const double pcost = (ctx + 0.5 * xpx * inv_tau) * inv_tau;
    const double dcost = (-bty - 0.5 * xpx * inv_tau) * inv_tau;
    const double pres = mx[0], dres = mx[1];
    const double gap = fabs((ctx + bty + xpx * inv_tau) * inv_tau);
    const double norm_aty = mx[2], norm_px = mx[3];
    const double dinf_a = mx[4] / (fabs(ctx) + kEps);
    const double dinf_p = norm_px / (fabs(ctx) + kEps);
    const double dinf = fmax(dinf_a, dinf_p);
    const double pinf = norm_aty / (fabs(bty) + kEps);
    const double prel = fmax(fmax(mx[5] * inv_tau, mx[6] * inv_tau), nb);
    const double drel = fmax(fmax(norm_px * inv_tau, norm_aty * inv_tau), nc);
    const double nx = mx[7], ny = mx[8];
    int status;
    if (gap < op.atol + op.rtol * fmin(fabs(pcost), fabs(dcost)) &&
        pres < op.atol + op.rtol * prel && dres < op.atol + op.rtol * drel) {
      status = QTQP_STATUS_SOLVED;
    } else if (ctx < -kEps && dinf < op.atol_infeas + op.rtol_infeas * nx / fabs(ctx)) {
      status = QTQP_STATUS_UNBOUNDED;
    } else if (bty < -kEps && pinf < op.atol_infeas + op.rtol_infeas * ny / fabs(bty)) {
      status = QTQP_STATUS_INFEASIBLE;
    } else {
      status = QTQP_STATUS_UNFINISHED;
    }
    if (st != nullptr && tid == 0) {
      st[kStCtx] = ctx;
      st[kStBty] = bty;
      st[kStPcost] = pcost;
      st[kStDcost] = dcost;
      st[kStPres] = pres;
      st[kStDres] = dres;
      st[kStGap] = gap;
      st[kStPinfeas] = pinf;
      st[kStDinfeas] = dinf;
      st[kStDinfeasA] = dinf_a;
      st[kStDinfeasP] = dinf_p;
      st[kStNormX] = nx;
      st[kStNormY] = ny;
      st[kStStatus] = status;
      st[kStPrel] = prel;
      st[kStDrel] = drel;
    }
    if (collect && st != nullptr) {
      // collect_stats extras (__init__.py:992-1007): complementarity, norm_s
      // and the per-inequality statistics of s*y and s/y.
      double a[5] = {0, 0, 0, 0, 0};  // y.s, sum sy, sum s/y
      double b[5] = {0, 0, -INFINITY, 0, 0};  // max sy, max -sy, max soy, max -soy
      b[0] = -INFINITY;
      b[1] = -INFINITY;
      b[3] = -INFINITY;
      for (int k = own(n); k < N; k += NT) {
        const double yo = de[k] * xy[k], so = s[k] / de[k];
        a[0] = fma(yo, so, a[0]);
        if (k >= n + z) {
          const double sy = so * yo, soy = so / fmax(kEps, yo);
          a[1] += sy;
          a[2] += soy;
          b[0] = fmax(b[0], sy);
          b[1] = fmax(b[1], -sy);
          b[2] = fmax(b[2], soy);
          b[3] = fmax(b[3], -soy);
        }
      }
      reduce<5, 5>(a, b);
      const int cnt = m - z;
      const double mean_sy = a[1] / cnt, mean_soy = a[2] / cnt;
      double v[2] = {0, 0};
      double dummy[1] = {0};
      for (int k = own(n + z); k < N; k += NT) {
        const double yo = de[k] * xy[k], so = s[k] / de[k];
        const double sy = so * yo, soy = so / fmax(kEps, yo);
        v[0] += (sy - mean_sy) * (sy - mean_sy);
        v[1] += (soy - mean_soy) * (soy - mean_soy);
      }
      reduce<2, 0>(v, dummy);
      if (tid == 0) {
        st[kStCompl] = fabs(a[0] * inv_tau * inv_tau);
        st[kStNormS] = mx[6];
        st[kStMaxSy] = b[0];
        st[kStMinSy] = -b[1];
        st[kStStdSy] = sqrt(v[0] / cnt);
        st[kStMaxSoy] = b[2];
        st[kStMinSoy] = -b[3];
        st[kStMeanSoy] = mean_soy;
        st[kStStdSoy] = sqrt(v[1] / cnt);
      }
    }
    last_pcost = pcost;
    last_dcost = dcost;
    last_pres = pres;
    last_dres = dres;
    last_gap = gap;
    return status;
  }
  double last_pcost = 0, last_dcost = 0, last_pres = 0, last_dres = 0, last_gap = 0;

  __device__ void write_lin_stats(double* st, int block, const IrOutcome& r, int tau_method,
                                  bool fp64) const {
    if (st == nullptr || tid != 0) return;
    double* b = st + kStLin0 + block * kLinFields;
    b[kLinSolves] = r.solves;
    b[kLinFinalRes] = r.final_res;
    b[kLinRhsNorm] = r.rhs_norm;
    b[kLinTol] = r.tol;
    b[kLinStatus] = r.status;
    b[kLinTau] = tau_method;
    b[kLinPrec] = fp64 ? 64 : 32;
  }

  // out[n + i] = (A v)_i (equilibrated A).  Exit: needs a barrier before
  // other threads read out.
  __device__ void a_times(const double* v, double* out) const {
    if constexpr (kSparseA) {
      for (int k = own(n); k < N; k += NT) out[k] = band_a_row(v, k - n);
    } else {
      const double* Ap = A;
      const int la = lda, nn = n;
      rowdot<1, false, kRowS>(m, n, [&](int k, int j, double* acc) { acc[0] = fma(Ap[k * la + j], v[j], acc[0]); },
                [&](int k, double* acc) { out[nn + k] = acc[0]; });
    }
  }

  // --------------------------------------------------------------------------
  // Learned warm start (no reference counterpart).  Given a predicted point
  // (wx, wy) in the original scaling and a predicted active set (act[i] for
  // the inequality rows), solve the KKT system of the equality QP
  //   min 1/2 x'Px + c'x  s.t.  a_i x = b_i for i < z or i active
  // (free rows carry a huge D, i.e. y_i = 0) by the IPM's own regularised
  // factorisation and FP64 refinement; then y_i = 0 on free rows and
  // s = b - A x.  Each solution is projected onto the cone (y[z:] >= 0,
  // s[z:] >= 0) and accepted only if the plain termination test reports
  // SOLVED for it at tau = 1.  Up to options.warm_corrections primal-dual
  // active-set corrections may follow a rejected solution (tight rows whose
  // dual came out negative leave, free rows whose slack came out negative
  // enter, and the reduced system is solved again) while the set changes;
  // 0 keeps exactly one reduced solve.  On false the caller runs the plain
  // method from its usual starting point.
  // --------------------------------------------------------------------------
  __device__ bool warm_try(const double* wx, const double* wy, const unsigned char* act,
                           double nb, double nc, bool& fp64, int& n32, int& n64, int& nsolves) {
    const qtqp_options& op = *o;
    double* xy = vec(kXY);
    double* s = vec(kRS);
    double* xyc = vec(kXYC);
    double* reg = vec(kREG);
    double* corr = vec(kCORR);
    double* pi = vec(kPI);
    double* pw = vec(kPW);
    double* tight = vec(kCT);  // at [n, N): 1.0 where the row is held tight
    const double* de = vec(kDE);
    const double* q = vec(kQ);
    const double dmin = fmax(op.min_static_regularization, 1e-10);
    const double big = 1e10;
    for (int k = tid; k < N; k += NT) {
      if (k < n) {
        xy[k] = wx[k] / de[k];
      } else {
        const int i = k - n;
        tight[k] = (i < z || act[i] != 0) ? 1.0 : 0.0;
        xy[k] = wy[i] / de[k];
      }
    }
    double dummy[1] = {0.0};
    const int rounds = 1 + max(0, min(op.warm_corrections, 64));
    for (int round = 0; round < rounds; ++round) {
      for (int k = tid; k < N; k += NT) {
        if (k < n) {
          const double t = pi[k];
          const double r = fmax(t, op.min_static_regularization);
          reg[k] = r;
          corr[k] = r - t;
        } else {
          const bool tk = tight[k] != 0.0;
          const double t = -(tk ? 0.0 : big), r = -(tk ? dmin : big);
          reg[k] = r;
          corr[k] = r - t;
          pi[k] = 1.0 / (-r);
          pw[k] = 1.0 / sqrt(-r);
        }
      }
      sync();
      int info;
      if (fp64) {
        ++n64;
        info = factorize<double>();
      } else {
        ++n32;
        info = factorize<float>();
        if (info != 0) {
          fp64 = true;
          ++n64;
          info = factorize<double>();
        }
      }
      if (info != 0) return false;  // not an error of the problem: fall back
      int err = 0;
      IrOutcome r = ir_solve_policy([&](int k) { return -q[k]; }, xy,
                                    xyc, fp64, n32, n64, err);
      nsolves += r.solves;
      if (err || r.nan) return false;
      a_times(xyc, s);  // s[n + i] = (A x)_i
      sync();
      double v[1] = {0.0};  // 1 when a row changes
      for (int k = tid; k < N; k += NT) {
        if (k < n) {
          xy[k] = xyc[k];
          continue;
        }
        const int i = k - n;
        const double sk = q[k] - s[k];
        if (i < z) {
          xy[k] = xyc[k];
          s[k] = 0.0;
        } else if (tight[k] != 0.0) {
          xy[k] = fmax(xyc[k], 0.0);
          if (xyc[k] < 0.0) {
            tight[k] = 0.0;
            v[0] = 1.0;
          }
          s[k] = fmax(sk, 0.0);
        } else {
          xy[k] = 0.0;
          if (sk < 0.0) {
            tight[k] = 1.0;
            v[0] = 1.0;
          }
          s[k] = fmax(sk, 0.0);
        }
      }
      reduce<0, 1>(dummy, v);
      // The plain test evaluates the projected point: clipped duals and slacks
      // show up in its residuals.
      if (termination(1.0, nb, nc, nullptr, false) == QTQP_STATUS_SOLVED) return true;
      if (!(v[0] > 0.0)) return false;  // the set is stable yet not acceptable
      sync();
    }
    return false;
  }

  // --------------------------------------------------------------------------
  // The whole solve (QTQP._solve_impl, __init__.py:429-614).  warm_*: the
  // learned warm start of this instance (x and y in the original scaling,
  // active-row mask), or null for the plain method.
  // --------------------------------------------------------------------------
  // start_*: a starting point in the original scaling (y, s positive on the
  // inequality rows) that replaces the cold start (no reference counterpart:
  // a re-solve started from an earlier solution), or null.
  __device__ void solve(qtqp_result* result, double* stats, double* x_out, double* y_out,
                        double* s_out, const double* warm_x = nullptr,
                        const double* warm_y = nullptr,
                        const unsigned char* warm_act = nullptr,
                        const double* start_x = nullptr, const double* start_y = nullptr,
                        const double* start_s = nullptr) {
    const qtqp_options& op = *o;
    const uint64_t t_start = globaltimer_ns();
    double nb, nc;
    {
      QTQP_TIC();
      load_and_equilibrate(op.equilibrate != 0, nb, nc);
      QTQP_TOC(kPhLoad);
    }
    int w32 = 0, w64 = 0, wsolves = 0;  // work of a rejected warm start counts too
    if (warm_act != nullptr) {
      // FP64 factor: the reduced system is as ill-conditioned as the last
      // interior-point iterations, where an FP32 factor is refused anyway.
      bool fp64w = true;
      const bool ok = warm_try(warm_x, warm_y, warm_act, nb, nc, fp64w, w32, w64, wsolves);
      sync();
      if (ok) {
        finish(QTQP_STATUS_SOLVED, 1.0, x_out, y_out, s_out);
        if (tid == 0) {
          result->status = QTQP_STATUS_SOLVED;
          result->iterations = 0;
          result->error = 0;
          result->fp32_factorizations = w32;
          result->fp64_factorizations = w64;
          result->ir_solves = wsolves;
          result->warm_started = 1;
          result->tau = 1.0;
          result->pcost = last_pcost;
          result->dcost = last_dcost;
          result->pres = last_pres;
          result->dres = last_dres;
          result->gap = last_gap;
        }
        return;
      }
    }
    double* xy = vec(kXY);
    double* s = vec(kRS);
    double* kq = vec(kKQ);
    double* kq0 = vec(kKQ0);
    double* xyp = vec(kXYP);
    double* xyc = vec(kXYC);
    double* ds = vec(kXD);  // d_s at [n, N)
    double* ct = vec(kCT);  // Mehrotra correction at [n, N)
    const double* q = vec(kQ);
    const double* de = vec(kDE);
    // Starting point.  A learned warm start that was not accepted starts the
    // method from its prediction when options.warm_shift > 0: x = x_hat,
    // y = y_hat on the equality rows, y = max(y_hat, 0) + shift and
    // s = max(b - A x_hat, 0) + shift on the inequality rows.  A given
    // start_* point is taken as it is.  Both are equilibrated like the cold
    // start (x/e, y/d, s*d).
    const bool from_pred = warm_act != nullptr && op.warm_shift > 0.0;
    const bool from_start = start_x != nullptr;
    if (from_pred || from_start) {
      const double sh = from_pred ? op.warm_shift : 0.0;
      const double* px0 = from_start ? start_x : warm_x;
      for (int k = tid; k < n; k += NT) xy[k] = px0[k] / de[k];
      sync();
      if (!from_start) {
        a_times(xy, s);  // s[n + i] = (A_eq x)_i = d_i (A x_hat)_i
        sync();
      }
      for (int k = own(n); k < N; k += NT) {
        const int i = k - n;
        const double yi = from_start ? start_y[i] : warm_y[i];
        if (i < z) {
          xy[k] = yi / de[k];
          s[k] = 0.0;
        } else if (from_start) {
          xy[k] = yi / de[k];
          s[k] = start_s[i] * de[k];
        } else {
          const double slack = fmax((q[k] - s[k]) / de[k], 0.0);  // b - A x_hat
          xy[k] = (fmax(yi, 0.0) + sh) / de[k];
          s[k] = (slack + sh) * de[k];
        }
      }
    }
    // _init_variables (__init__.py:299-307): x = 0, y[z:] = s[z:] = 1, then
    // equilibrated (x/e, y/d, s*d); K^{-1} q starts at zero.
    for (int k = tid; k < N; k += NT) {
      kq[k] = 0.0;
      if (from_pred || from_start) {
      } else if (k < n) {
        xy[k] = 0.0 / de[k];
      } else if (k < n + z) {
        xy[k] = 0.0;
        s[k] = 0.0;
      } else {
        xy[k] = 1.0 / de[k];
        s[k] = 1.0 * de[k];
      }
      ds[k] = 0.0;
      ct[k] = 0.0;
    }
    sync();
    double tau = 1.0, alpha = 0.0, sigma = 0.0, mu = 0.0;
    bool fp64 = op.precision == QTQP_PREC_FP64;
    int n32 = w32, n64 = w64, nsolves = wsolves, err = 0;
    int status = QTQP_STATUS_UNFINISHED;
    int it = 0, taken = 0;
    const double cnt = double(m - z);
    double dummy[1] = {0.0};
    for (it = 0; it < op.max_iter; ++it) {
      double* st = (stats != nullptr) ? stats + size_t(it) * QTQP_STATS_DOUBLES : nullptr;
      // _normalize (__init__.py:859-880) and mu (:477).
      {
        QTQP_TIC();
        double sm[2] = {0.0, 0.0};
        for (int k = tid; k < N; k += NT) {
          sm[0] = fma(xy[k], xy[k], sm[0]);
          if (k >= n) sm[1] = fma(xy[k], s[k], sm[1]);
        }
        reduce<2, 0>(sm, dummy);
        const double scale = sqrt(double(m - z + 1)) / fmax(kEps, sqrt(sm[0] + tau * tau));
        for (int k = tid; k < N; k += NT) {
          xy[k] *= scale;
          if (k >= n) s[k] *= scale;
        }
        tau *= scale;
        mu = (sm[1] * scale * scale) / cnt;
        QTQP_TOC(kPhNormalize);
      }
      // DirectKktSolver.update (direct.py:183-216).
      kkt_diag(mu, op.min_static_regularization);
      sync();
      {
        int info;
        if (fp64) {
          ++n64;
          info = factorize<double>();
        } else {
          ++n32;
          info = factorize<float>();
          if (info != 0) {  // FP32 pivot failure: refactor in FP64 for good
            fp64 = true;
            ++n64;
            info = factorize<double>();
          }
        }
        if (info != 0) {
          err = QTQP_ERR_NOT_SPD;
          break;
        }
      }
      // kinv_q = K^{-1} q, warm-started (__init__.py:484).
      for (int k = tid; k < N; k += NT) kq0[k] = kq[k];
      IrOutcome rq = ir_solve_policy([&](int k) { return q[k]; }, kq0,
                                     kq, fp64, n32, n64, err);
      nsolves += rq.solves;
      if (err) break;
      if (rq.nan) {
        err = QTQP_ERR_NAN;
        break;
      }
      write_lin_stats(st, 0, rq, -1, fp64);
      // Per-iteration constants of the tau equations: P K^{-1}q, P x and dots.
      IterConsts ic;
      {
        double* pkq = vec(kPW);
        double* px = vec(kXD);
        const double* pi = vec(kPI);
        double sm[5] = {0, 0, 0, 0, 0};
        for (int k = tid; k < N; k += NT) {
          sm[0] = fma(kq[k], q[k], sm[0]);
          sm[2] = fma(q[k], xy[k], sm[2]);
        }
        if (has_p) {
          auto epi = [&](int k, double pq, double pxk) {
            const double a = fma(pi[k], kq[k], pq);
            const double b = fma(pi[k], xy[k], pxk);
            pkq[k] = a;
            px[k] = b;
            sm[1] = fma(kq[k], a, sm[1]);
            sm[3] = fma(xy[k], b, sm[3]);
            sm[4] = fma(b, kq[k], sm[4]);
          };
          if constexpr (kSparseA) {
            for (int k = tid; k < n; k += NT) epi(k, band_poff_row(kq, k), band_poff_row(xy, k));
          } else {
            const double* Pp = P;
            const int lp = ldp;
            rowdot<2>(n, n,
                      [&](int k, int j, double* acc) {
                        const double pjk = Pp[j * lp + k];
                        acc[0] = fma(pjk, kq[j], acc[0]);
                        acc[1] = fma(pjk, xy[j], acc[1]);
                      },
                      [&](int k, double* acc) { epi(k, acc[0], acc[1]); });
          }
        }
        reduce<5, 0>(sm, dummy);
        ic.kqq = sm[0];
        ic.kqpkq = sm[1];
        ic.qz = sm[2];
        ic.xpx = has_p ? sm[3] : 0.0;
        ic.pxkq = has_p ? sm[4] : 0.0;
      }
      // ---- Predictor (__init__.py:489-516) -------------------------------
      const double mu_c = mu;
      auto rhs_pred = [&](int k) {
        double r = (mu_c - 0.0) * xy[k];
        if (k >= n + z) r += s[k];
        return r;
      };
      IrOutcome rp = ir_solve_policy(rhs_pred, xy, xyp, fp64, n32,
                                     n64, err);
      nsolves += rp.solves;
      if (err) break;
      if (rp.nan) {
        err = QTQP_ERR_NAN;
        break;
      }
      int tm_p = 0;
      double tau_p;
      {
        QTQP_TIC();
        tau_p = tau_step(xyp, rp, mu, 0.0, mu * tau, tau, tau, ic, tm_p);
        QTQP_TOC(kPhTau);
      }
      write_lin_stats(st, 1, rp, tm_p, fp64);
      for (int k = tid; k < N; k += NT) {
        xyp[k] -= kq[k] * tau_p;  // [x_p; y_p]
        if (k >= n + z) ds[k] = -xyp[k] * s[k] / xy[k];
      }
      const double alpha_p = step_to_boundary([&](int k, double& dy, double& dsk) {
        dy = xyp[k] - xy[k];
        dsk = ds[k];
      });
      // _compute_sigma (__init__.py:682-706).
      {
        double sm[3] = {0, 0, 0};
        const double dtp = tau_p - tau;
        for (int k = tid; k < N; k += NT) {
          const double va = xy[k] + alpha_p * (xyp[k] - xy[k]);
          if (k < n) {
            sm[0] = fma(va, va, sm[0]);
          } else {
            sm[1] = fma(va, va, sm[1]);
            const double sa = s[k] + alpha_p * ds[k];
            sm[2] = fma(va, sa, sm[2]);
          }
        }
        reduce<3, 0>(sm, dummy);
        const double ta = tau + alpha_p * dtp;
        const double nrm2 = sm[0] + sm[1] + ta * ta;
        const double scale_sq = double(m - z + 1) / fmax(kEps * kEps, nrm2);
        const double mu_aff = scale_sq * sm[2] / cnt;
        const double sb = mu_aff / fmax(kEps, mu);
        sigma = fmin(fmax(sb * sb * sb, 0.0), 1.0);
      }
      // Mehrotra correction (__init__.py:528).
      for (int k = own(n + z); k < N; k += NT) {
        const double dyp = xyp[k] - xy[k];
        ct[k] = -ds[k] * dyp / xy[k];
      }
      // ---- Corrector (__init__.py:529-543) -------------------------------
      const double mu_t = sigma * mu;
      auto rhs_corr = [&](int k) {
        double r = (mu_c - mu_t) * xyp[k];
        if (k >= n + z) {
          if (mu_t != 0.0) r += mu_t / xy[k];
          r += s[k];
          r += ct[k];
        }
        return r;
      };
      sync();  // x_p, y_p complete before the corrector reads them
      IrOutcome rc = ir_solve_policy(rhs_corr, xyp, xyc, fp64, n32,
                                     n64, err);
      nsolves += rc.solves;
      if (err) break;
      if (rc.nan) {
        err = QTQP_ERR_NAN;
        break;
      }
      int tm_c = 0;
      const double tau_c =
          tau_step(xyc, rc, mu, mu_t, (mu - mu_t) * tau_p, tau, tau_p, ic, tm_c);
      write_lin_stats(st, 2, rc, tm_c, fp64);
      for (int k = tid; k < N; k += NT) {
        xyc[k] -= kq[k] * tau_c;  // [x_c; y_c]
        if (k >= n + z) ds[k] = mu_t / xy[k] + ct[k] - xyc[k] * s[k] / xy[k];
      }
      alpha = step_to_boundary([&](int k, double& dy, double& dsk) {
        dy = xyc[k] - xy[k];
        dsk = ds[k];
      });
      // ---- Update (__init__.py:556-565) --------------------------------
      {
        const double stp = op.step_size_scale * alpha;
        for (int k = tid; k < N; k += NT) {
          xy[k] += stp * (xyc[k] - xy[k]);
          if (k >= n) s[k] += stp * ds[k];
          if (k >= n + z) {
            xy[k] = fmax(xy[k], 1e-30);
            s[k] = fmax(s[k], 1e-30);
          }
        }
        tau += stp * (tau_c - tau);
        tau = fmax(tau, 1e-30);
      }
      sync();
      {
        QTQP_TIC();
        status = termination(tau, nb, nc, st, op.collect_stats != 0);
        QTQP_TOC(kPhTerm);
      }
      taken = it + 1;
      if (st != nullptr && tid == 0) {
        st[kStIter] = it;
        st[kStMu] = mu;
        st[kStSigma] = sigma;
        st[kStAlpha] = alpha;
        st[kStTau] = tau;
        st[kStTime] = double(globaltimer_ns() - t_start) * 1e-9;
      }
      if (status != QTQP_STATUS_UNFINISHED) break;
    }
    if (err == 0 && status == QTQP_STATUS_UNFINISHED && taken == op.max_iter) {
      status = QTQP_STATUS_HIT_MAX_ITER;
      if (stats != nullptr && tid == 0)
        stats[size_t(taken - 1) * QTQP_STATS_DOUBLES + kStStatus] = status;
    }
    sync();
    finish(status, tau, x_out, y_out, s_out);
    if (tid == 0) {
      result->status = err ? QTQP_STATUS_FAILED : status;
      result->iterations = taken;
      result->error = err;
      result->fp32_factorizations = n32;
      result->fp64_factorizations = n64;
      result->ir_solves = nsolves;
      result->warm_started = 0;
      result->tau = tau;
      result->pcost = last_pcost;
      result->dcost = last_dcost;
      result->pres = last_pres;
      result->dres = last_dres;
      result->gap = last_gap;
    }
  }

  // Unequilibrate and scale by status (__init__.py:580-614).
  QTQP_PHASE void finish(int status, double tau, double* x_out, double* y_out, double* s_out) {
    QTQP_LOCALS;
    const double* xy = vec(kXY);
    const double* s = vec(kRS);
    const double* de = vec(kDE);
    const double nan = __longlong_as_double(0x7ff8000000000000ll);
    double sm[2] = {0.0, 0.0};  // b_o . y_o, c_o . x_o
    double dummy[1] = {0.0};
    if (status == QTQP_STATUS_INFEASIBLE || status == QTQP_STATUS_UNBOUNDED) {
      for (int k = tid; k < N; k += NT) {
        if (k < n) {
          sm[1] = fma(c0[k], de[k] * xy[k], sm[1]);
        } else {
          sm[0] = fma(b0[k - n], de[k] * xy[k], sm[0]);
        }
      }
      reduce<2, 0>(sm, dummy);
    }
    for (int k = tid; k < N; k += NT) {
      if (k < n) {
        const double xo = de[k] * xy[k];
        double v;
        if (status == QTQP_STATUS_INFEASIBLE) {
          v = nan;
        } else if (status == QTQP_STATUS_UNBOUNDED) {
          v = xo / fabs(sm[1]);
        } else {
          v = xo / tau;
        }
        x_out[k] = v;
      } else {
        const double yo = de[k] * xy[k], so = s[k] / de[k];
        double vy, vs;
        if (status == QTQP_STATUS_INFEASIBLE) {
          vy = yo / fabs(sm[0]);
          vs = nan;
        } else if (status == QTQP_STATUS_UNBOUNDED) {
          vy = nan;
          vs = so / fabs(sm[1]);
        } else {
          vy = yo / tau;
          vs = so / tau;
        }
        y_out[k - n] = vy;
        s_out[k - n] = vs;
      }
    }
  }
  // ==========================================================================
  // Banded backend (FMT == kFmtBand): sparse A and P, and the Gram matrix
  // G = P_off + diag(Rx) + A^T diag(1/Ry) A of half-bandwidth bw (e.g. the
  // block-tridiagonal Gram of a stage-ordered MPC problem).  Everything lives
  // in the instance's global workspace slot.
  // ==========================================================================
  __device__ void bind_band(int n_, int m_, int bw_, int nnz_a_, int nnz_p_, char* gmem) {
    tid = threadIdx.x;
    n = n_;
    m = m_;
    N = n + m;
    bw = bw_;
    nnz_a = nnz_a_;
    nnz_p = nnz_p_;
    const BandLayout L = plan_band_layout(n, m, bw, nnz_a, nnz_p);
    np = L.np;
    V = reinterpret_cast<double*>(gmem);
    Lb = reinterpret_cast<double*>(gmem + L.v_bytes);
    G = Lb;
    av = reinterpret_cast<double*>(gmem + L.v_bytes + L.l_bytes);
    at = av + nnz_a;
    pv = at + nnz_a;
    A = P = nullptr;
    lda = ldp = ldg = 0;
  }

#define QTQP_BAND_LOCALS                                                        \
  const int tid = this->tid, n = this->n, m = this->m, N = this->N;             \
  const int bw = this->bw, ldl = this->bw + 1;                                  \
  const int* const ip = this->ip;                                               \
  const int* const ix = this->ix;                                               \
  const int* const jp = this->jp;                                               \
  const int* const jx = this->jx;                                               \
  const int* const pp = this->pp;                                               \
  const int* const px = this->px;                                               \
  double* const av = this->av;                                                  \
  double* const at = this->at;                                                  \
  double* const pv = this->pv;                                                  \
  const bool has_p = this->has_p;                                               \
  (void)tid; (void)n; (void)m; (void)N; (void)bw; (void)ldl; (void)ip; (void)ix; \
  (void)jp; (void)jx; (void)pp; (void)px; (void)av; (void)at; (void)pv; (void)has_p

  // Ruiz equilibration on the CSR (A), CSC (A) and CSR (P) value arrays, with
  // the reference's arithmetic: a_ij *= (d_i * e_j), p_ij *= (e_i * e_j).
  __device__ void band_load_and_equilibrate(bool equilibrate, double& nb, double& nc) {
    QTQP_BAND_LOCALS;
    double* de = vec(kDE);
    double* sc = vec(kTMP);
    for (int q = tid; q < nnz_a; q += NT) {
      av[q] = av0[q];
      at[q] = at0[q];
    }
    for (int q = tid; q < nnz_p; q += NT) pv[q] = has_p ? pv0[q] : 0.0;
    for (int k = tid; k < N; k += NT) de[k] = 1.0;
    sync();
    auto scale_of = [](double mx) {
      if (mx == 0.0) mx = 1.0;
      return fmin(fmax(1.0 / sqrt(mx), 1e-3), 1e3);
    };
    if (equilibrate) {
      for (int sweep = 0; sweep < 10; ++sweep) {
        for (int k = tid; k < N; k += NT) {
          double mx = 0.0;
          if (k < n) {
            for (int q = jp[k]; q < jp[k + 1]; ++q) mx = fmax(mx, fabs(at[q]));
            if (has_p)
              for (int q = pp[k]; q < pp[k + 1]; ++q) mx = fmax(mx, fabs(pv[q]));
          } else {
            for (int q = ip[k - n]; q < ip[k - n + 1]; ++q) mx = fmax(mx, fabs(av[q]));
          }
          sc[k] = scale_of(mx);
        }
        sync();
        for (int r = tid; r < m; r += NT) {
          const double dr = sc[n + r];
          for (int q = ip[r]; q < ip[r + 1]; ++q) av[q] *= dr * sc[ix[q]];
        }
        for (int j = tid; j < n; j += NT) {
          const double ej = sc[j];
          for (int q = jp[j]; q < jp[j + 1]; ++q) at[q] *= sc[n + jx[q]] * ej;
        }
        if (has_p) {
          for (int i = tid; i < n; i += NT) {
            const double ei = sc[i];
            for (int q = pp[i]; q < pp[i + 1]; ++q) pv[q] *= ei * sc[px[q]];
          }
        }
        for (int k = tid; k < N; k += NT) de[k] *= sc[k];
        sync();
      }
    }
    double* q = vec(kQ);
    double* pi = vec(kPI);
    double mx[2] = {0.0, 0.0};
    double dummy[1] = {0.0};
    for (int k = tid; k < N; k += NT) {
      if (k < n) {
        q[k] = c0[k] * de[k];
        double d = 0.0;
        if (has_p) {
          for (int qq = pp[k]; qq < pp[k + 1]; ++qq) {
            if (px[qq] == k) {  // diag(P_eq); pv keeps only the off-diagonal
              d = pv[qq];
              pv[qq] = 0.0;
            }
          }
        }
        pi[k] = d;
        mx[1] = nanmax(mx[1], fabs(c0[k]));
      } else {
        q[k] = b0[k - n] * de[k];
        mx[0] = nanmax(mx[0], fabs(b0[k - n]));
      }
    }
    reduce<0, 2>(dummy, mx);
    nb = mx[0];
    nc = mx[1];
    sync();
  }

  // sum_{q0 <= q < q1} val[q] v[voff + idx[q]]: indices and values are
  // loaded 8 at a time, then the 8 gathers, so that several loads are in
  // flight per thread (these sparse dots are latency-bound).
  __device__ __forceinline__ static double sparse_dot(const int* idx, const double* val,
                                                      const double* v, int voff, int q0,
                                                      int q1) {
    double t0 = 0.0, t1 = 0.0;
    int q = q0;
    for (; q + 8 <= q1; q += 8) {
      int ii[8];
      double aa[8], xx[8];
#pragma unroll
      for (int e = 0; e < 8; ++e) {
        ii[e] = idx[q + e];
        aa[e] = val[q + e];
      }
#pragma unroll
      for (int e = 0; e < 8; ++e) xx[e] = v[voff + ii[e]];
#pragma unroll
      for (int e = 0; e < 8; e += 2) {
        t0 = fma(aa[e], xx[e], t0);
        t1 = fma(aa[e + 1], xx[e + 1], t1);
      }
    }
    for (; q < q1; ++q) t0 = fma(val[q], v[voff + idx[q]], t0);
    return t0 + t1;
  }
  // (P_off v)_k for the owner of row k (P symmetric, so row k = column k).
  __device__ __forceinline__ double band_poff_row(const double* v, int k) const {
    return has_p ? sparse_dot(px, pv, v, 0, pp[k], pp[k + 1]) : 0.0;
  }
  // (A^T y)_k with y at v[n + i].
  __device__ __forceinline__ double band_at_col(const double* v, int k) const {
    return sparse_dot(jx, at, v, n, jp[k], jp[k + 1]);
  }
  // (A x)_i.
  __device__ __forceinline__ double band_a_row(const double* v, int i) const {
    return sparse_dot(ix, av, v, 0, ip[i], ip[i + 1]);
  }

  // Column j of the Gram matrix G = P_off + diag(Rx) + A^T diag(1/Ry) A,
  // rows j .. j + bw, into acc[0 .. bw].  The loads of every level are issued
  // in batches of 8 before they are used (column j's rows and their
  // scalings, then each row's entries), so that this latency-bound gather
  // keeps several loads in flight.
  template <typename T>
  __device__ __forceinline__ void band_gram_column(int j, T* acc) const {
    QTQP_BAND_LOCALS;
    const double* reg = vec(kREG);
    const double* wsc = vec(kPW);
    for (int d = 0; d <= bw; ++d) acc[d] = T(0);
    const int qa = jp[j], qb = jp[j + 1];
    for (int q0 = qa; q0 < qb; q0 += 8) {
      int rr[8], r0[8], r1[8];
      double ww[8], aq[8];
#pragma unroll
      for (int u = 0; u < 8; ++u) {
        const bool ok = q0 + u < qb;
        rr[u] = ok ? jx[q0 + u] : 0;
        aq[u] = ok ? at[q0 + u] : 0.0;
      }
#pragma unroll
      for (int u = 0; u < 8; ++u) {
        const bool ok = q0 + u < qb;
        ww[u] = ok ? wsc[n + rr[u]] : 0.0;
        r0[u] = ok ? ip[rr[u]] : 0;
        r1[u] = ok ? ip[rr[u] + 1] : 0;
      }
#pragma unroll 1
      for (int u = 0; u < 8 && q0 + u < qb; ++u) {
        const double w = ww[u];
        const T arj = T(aq[u] * w);
        const int q1 = r1[u];
        int q2 = r0[u];
        for (; q2 + 8 <= q1; q2 += 8) {
          int ii[8];
          double aa[8];
#pragma unroll
          for (int e = 0; e < 8; ++e) {
            ii[e] = ix[q2 + e];
            aa[e] = av[q2 + e];
          }
#pragma unroll
          for (int e = 0; e < 8; ++e) {
            const int i = ii[e];
            if (i >= j && i - j <= bw) acc[i - j] = fma(arj, T(aa[e] * w), acc[i - j]);
          }
        }
        for (; q2 < q1; ++q2) {
          const int i = ix[q2];
          if (i >= j && i - j <= bw) acc[i - j] = fma(arj, T(av[q2] * w), acc[i - j]);
        }
      }
    }
    if (has_p) {
      for (int q = pp[j]; q < pp[j + 1]; ++q) {
        const int i = px[q];
        if (i > j && i - j <= bw) acc[i - j] = T(pv[q]) + acc[i - j];
      }
    }
    acc[0] = T(reg[j]) + acc[0];
  }

  // The Gram matrix in column band storage (Lb) plus the relative diagonal
  // jitter of the dense backend.  acc_smem: this thread's column scratch in
  // shared memory (bw + 1 entries), or null to accumulate in place.
  template <typename T>
  __device__ void band_gram(T* acc_smem) {
    const int ldl = bw + 1;
    T* L = reinterpret_cast<T*>(Lb);
    double dmax[1] = {0.0};
    double dummy[1] = {0.0};
    for (int j0 = 0; j0 < n; j0 += NT) {
      const int j = j0 + tid;
      if (j < n) {
        T* col = L + size_t(j) * ldl;
        T* acc = acc_smem != nullptr ? acc_smem : col;
        band_gram_column<T>(j, acc);
        dmax[0] = nanmax(dmax[0], double(acc[0]));
        if (acc_smem != nullptr)
          for (int d = 0; d <= bw; ++d) col[d] = acc[d];
      }
    }
    reduce<0, 1>(dummy, dmax);
    const double jit = (sizeof(T) == 8 ? 1e-14 : 2.384185791015625e-07) * dmax[0];
    for (int j = tid; j < n; j += NT) L[size_t(j) * ldl] = T(double(L[size_t(j) * ldl]) + jit);
    sync();
  }

  // Gram matrix in column band storage, then Cholesky.  With the shared-
  // memory window (bw <= kBandWinMaxBw): each thread accumulates its Gram
  // column in shared memory, and the factorisation keeps the active
  // (bw+2) x (bw+2) part of the band in shared memory (band_chol_window_range).
  // Otherwise the global-memory variant below runs.  In grid mode the
  // partitioned factorisation runs (band_grid.cuh).  The diagonal of the
  // factor keeps 1 / l_kk.
  template <typename T>
  __device__ int band_factorize() {
    if constexpr (FMT == kFmtSparse) {
      return sparse_factorize<T>(*this);
    } else if constexpr (NT > 1024) {
      return bandp_factorize<T>(*this);
    } else {
      if (bwin == nullptr) return band_factorize_global<T>();
      QTQP_TIC();
      band_gram<T>(reinterpret_cast<T*>(bwin) + size_t(tid) * (bw + 1));
      QTQP_TOC(kPhGram);
      QTQP_RETIC();
      const int info = bw + kBandPanel <= NT
                           ? band_chol_panel_range<T, NT>(tid, 0, n, n, nullptr, 0)
                           : band_chol_window_range<T, NT>(tid, 0, n, n, nullptr, 0);
      QTQP_TOC(kPhChol);
      return info;
    }
  }

  // Blocked form of band_chol_window_range (same arguments and results):
  // kBandPanel-column panels.  Each panel is factorised tall-skinny in
  // registers (thread r holds the panel's entries of row k + r, for the
  // kBandPanel + bw rows the panel touches; per column the diagonal block's
  // rows publish their entry, one barrier, then every row scales its entry
  // by one reciprocal square root and updates the rest of its panel row),
  // written to the factor, and applied to the active bw x bw window as one
  // rank-kBandPanel update.  The window is circular with period B = bw +
  // kBandPanel (lower triangle, shared memory); the kBandPanel rows that
  // enter it are loaded from the Gram matrix during the panel, and the
  // window columns left of an entering row's band are zeroed.  Needs
  // kBandPanel + bw <= BT.
  template <typename T, int BT>
  __device__ int band_chol_panel_range(int lt, int lo, int nsub, int ne, T* tail, int ldt) {
    constexpr int KP = kBandPanel, PP = KP + 1;
    const int bw = this->bw, ldl = bw + 1, B = bw + KP;
    T* L = reinterpret_cast<T*>(Lb) + size_t(lo) * ldl;
    T* W = reinterpret_cast<T*>(bwin);
    T* Pn = W + B * B;
    T* pub = Pn + (KP + bw) * PP;
    uint16_t* pairs = reinterpret_cast<uint16_t*>(pub + 2 * KP);
    const int npairs = bw * (bw + 1) / 2;
    for (int a = lt; a < bw; a += BT)
      for (int b = 0; b <= a; ++b) pairs[a * (a + 1) / 2 + b] = uint16_t(a | (b << 8));
    for (int e = lt; e < B * B; e += BT) {
      const int i = e / B, j = e - i * B;
      W[e] = (j <= i && i - j <= bw && i < nsub) ? L[size_t(j) * ldl + (i - j)] : T(0);
    }
    group_sync<BT>();
    int bad = 0;
    constexpr int MAXPRE = (KP * 128 + BT - 1) / BT;  // entering entries per thread (bw < 128)
    for (int k = 0; k < ne; k += KP) {
      const int pw = min(KP, ne - k);
      const int nr = min(pw + bw, nsub - k);
      const int sk = k % B;
      auto sl = [&](int x) {  // slot of index k + x, 0 <= x < 2 B
        int t = sk + x;
        t = t >= B ? t - B : t;
        return t >= B ? t - B : t;
      };
      // Rows k + B .. k + B + pw - 1 enter after this panel: prefetch their
      // band entries (row r, column r - bw + d).
      T pre[MAXPRE];
#pragma unroll
      for (int q = 0; q < MAXPRE; ++q) {
        const int f = lt + BT * q, e = f / (bw + 1), d = f - e * (bw + 1);
        const int r = k + B + e;
        pre[q] = (e < pw && r < nsub) ? L[size_t(r - bw + d) * ldl + (bw - d)] : T(0);
      }
      T v[KP];
#pragma unroll
      for (int c = 0; c < KP; ++c)
        v[c] = (lt < nr && c < pw && c <= lt) ? W[sl(lt) * B + sl(c)] : T(0);
#pragma unroll
      for (int c = 0; c < KP; ++c) {
        if (c < pw) {
          T* pc = pub + (c & 1) * KP;
          if (lt >= c && lt < pw) pc[lt] = v[c];
          group_sync<BT>();
          const T piv = pc[c];
          if (!(piv > T(0))) {
            bad = k + c + 1;
            break;
          }
          const T il = rsqrt(piv);
          if (lt < nr) {
            if (lt == c) {
              v[c] = il;  // the factor keeps 1 / l_cc
            } else if (lt > c) {
              const T lic = v[c] * il;
              v[c] = lic;
#pragma unroll
              for (int j = c + 1; j < KP; ++j)
                if (j < pw) v[j] = fma(-lic, pc[j] * il, v[j]);
            }
          }
        }
      }
      if (bad) break;
      if (lt < nr) {
#pragma unroll
        for (int c = 0; c < KP; ++c)
          if (c < pw && c <= lt && lt - c <= bw) L[size_t(k + c) * ldl + (lt - c)] = v[c];
        if (lt >= pw) {
#pragma unroll
          for (int c = 0; c < KP; ++c) Pn[lt * PP + c] = v[c];
        }
      }
      group_sync<BT>();
      // Trailing update of the window: rows / columns k + pw .. k + pw + bw - 1.
      for (int pi = lt; pi < npairs; pi += BT) {
        const int pr = pairs[pi];
        const int a = pr & 0xff, b = pr >> 8;
        const int i = pw + a, j = pw + b;
        if (k + i < nsub) {
          const T* ri = Pn + i * PP;
          const T* rj = Pn + j * PP;
          T acc = T(0);
#pragma unroll
          for (int c = 0; c < KP; ++c) acc = fma(ri[c], rj[c], acc);
          T* w = W + sl(i) * B + sl(j);
          *w -= acc;
        }
      }
      // Entering rows: band entries, and zeros left of the band.
#pragma unroll
      for (int q = 0; q < MAXPRE; ++q) {
        const int f = lt + BT * q, e = f / (bw + 1), d = f - e * (bw + 1);
        const int r = k + B + e;
        if (e < pw && r < nsub) W[sl(B + e) * B + sl(KP + e + d)] = pre[q];
      }
      for (int f = lt; f < pw * (KP - 1); f += BT) {
        const int e = f / (KP - 1), t = f - e * (KP - 1);
        const int r = k + B + e, j = k + pw + t;  // columns k+pw .. r-bw-1
        if (r < nsub && j < r - bw) W[sl(B + e) * B + sl(pw + t)] = T(0);
      }
      group_sync<BT>();
    }
    if (tail != nullptr && bad == 0) {
      const int t = nsub - ne;
      for (int e = lt; e < t * t; e += BT) {
        const int i = e / t, j = e - i * t;
        if (j <= i) tail[size_t(i) * ldt + j] = W[((ne + i) % B) * B + (ne + j) % B];
      }
    }
    group_sync<BT>();
    return bad == 0 ? 0 : lo + bad;
  }

  // Band Cholesky with the active part of the band in shared memory, over
  // the principal submatrix of rows / columns [lo, lo + nsub) of which the
  // first ne columns are eliminated (ne == nsub: the whole factorisation).
  // Local rows and columns k .. k+bw+1 live in a (bw+2) x (bw+2) window with
  // circular indices (slot = index mod (bw+2)); step k reads the still-
  // unscaled column k, writes the finished column k of L to global memory,
  // updates the window, and stores row k+bw+1 of the Gram matrix (prefetched
  // into registers during the previous step) into the slots that row k-1
  // and column k-1 have freed.  One barrier per column.  Columns before lo
  // are not part of the submatrix.  tail (when ne < nsub): the lower
  // triangle of the trailing (nsub-ne)^2 block after the elimination (the
  // Schur complement of the eliminated columns), row-major with leading
  // dimension ldt.  lt: this thread's index among the BT threads of the
  // group.  Returns 0 or the 1-based global column of the first
  // non-positive pivot.
  template <typename T, int BT>
  __device__ int band_chol_window_range(int lt, int lo, int nsub, int ne, T* tail, int ldt) {
    const int bw = this->bw, ldl = bw + 1;
    T* L = reinterpret_cast<T*>(Lb) + size_t(lo) * ldl;
    T* W = reinterpret_cast<T*>(bwin);
    const int B = bw + 2;
    // Offsets (oi, oj), 1 <= oj <= oi <= bw, of the trailing update relative
    // to k, the same every step; thread t handles pairs t, t + BT, ...
    uint32_t* pairs = reinterpret_cast<uint32_t*>(bwin + (size_t(B) * B * sizeof(T) + 7) / 8);
    const int npairs = bw * (bw + 1) / 2;
    for (int oi = 1 + lt; oi <= bw; oi += BT)
      for (int oj = 1; oj <= oi; ++oj) pairs[(oi - 1) * oi / 2 + oj - 1] = uint32_t(oi) | (uint32_t(oj) << 16);
    // Rows 0 .. min(bw, nsub-1): entries (i, j), j <= i.
    for (int e = lt; e < B * B; e += BT) {
      const int i = e / B, j = e - i * B;
      W[e] = (j <= i && i <= bw && i < nsub) ? L[size_t(j) * ldl + (i - j)] : T(0);
    }
    // Prefetch of the row that enters at step k: r = k + bw + 1, entries
    // (r, j) for j in [r - bw, r]; thread t takes j = r - bw + t.
    auto fetch = [&](int k) {
      const int r = k + bw + 1, j = r - bw + lt;
      return (r < nsub && lt <= bw) ? L[size_t(j) * ldl + (r - j)] : T(0);
    };
    T pre = fetch(0);
    group_sync<BT>();
    int info = 0;
    for (int k = 0; k < ne; ++k) {
      const int ks = k % B;
      const T d = W[ks * B + ks];
      if (!(d > T(0))) {
        info = k + 1;
        break;
      }
      const T il = rsqrt(d), inv_d = il * il;  // no division on this chain
      const int last = min(nsub - 1, k + bw);
      auto slot = [&](int i) {  // i % B for i in [k, k + B)
        const int t = ks + (i - k);
        return t >= B ? t - B : t;
      };
      // Finished column k of L (global); the window keeps it unscaled.
      for (int i = k + 1 + lt; i <= last; i += BT) L[size_t(k) * ldl + (i - k)] = W[slot(i) * B + ks] * il;
      if (lt == 0) L[size_t(k) * ldl] = il;
      // Trailing update: W_ij -= W_ik W_jk / d for k < j <= i <= last.
      const int span = last - k;
#pragma unroll 4
      for (int pi = lt; pi < npairs; pi += BT) {
        const uint32_t pr = pairs[pi];
        const int oi = int(pr & 0xffffu), oj = int(pr >> 16);
        if (oi <= span) {
          const int is = slot(k + oi), js = slot(k + oj);
          W[is * B + js] = fma(-W[is * B + ks] * inv_d, W[js * B + ks], W[is * B + js]);
        }
      }
      // Row r = k + bw + 1 enters: row slot (k-1) mod B, column slots of
      // j in [k+1, r] (never ks; the diagonal lands in column k-1's slot).
      {
        const int r = k + bw + 1;
        if (r < nsub && lt <= bw) {
          const int rs = ks == 0 ? B - 1 : ks - 1;  // (k - 1) mod B
          const int j = r - bw + lt;                // in [k + 1, r]
          W[rs * B + (j - k == B - 1 ? rs : slot(j))] = pre;
        }
        pre = fetch(k + 1);
      }
      group_sync<BT>();
    }
    group_sync<BT>();
    if (tail != nullptr && info == 0) {
      const int t = nsub - ne;
      for (int e = lt; e < t * t; e += BT) {
        const int i = e / t, j = e - i * t;
        if (j <= i) tail[size_t(i) * ldt + j] = W[((ne + i) % B) * B + (ne + j) % B];
      }
    }
    return info == 0 ? 0 : lo + info;
  }

  // Global-memory variant (wide bands): Gram in column band storage, then
  // Cholesky with one barrier per column (the unscaled column k updates the
  // trailing band and column k-1 is finished in the same phase).
  template <typename T>
  __device__ int band_factorize_global() {
    QTQP_BAND_LOCALS;
    QTQP_TIC();
    T* L = reinterpret_cast<T*>(Lb);
    const double* reg = vec(kREG);
    const double* wsc = vec(kPW);
    double dmax[1] = {0.0};
    double dummy[1] = {0.0};
    for (int j = tid; j < n; j += NT) {
      T* col = L + size_t(j) * ldl;
      for (int d = 0; d <= bw; ++d) col[d] = T(0);
      for (int q = jp[j]; q < jp[j + 1]; ++q) {
        const int r = jx[q];
        const double w = wsc[n + r];
        const T arj = T(at[q] * w);
        for (int q2 = ip[r]; q2 < ip[r + 1]; ++q2) {
          const int i = ix[q2];
          if (i >= j && i - j <= bw) col[i - j] = fma(arj, T(av[q2] * w), col[i - j]);
        }
      }
      if (has_p) {
        for (int q = pp[j]; q < pp[j + 1]; ++q) {
          const int i = px[q];
          if (i > j && i - j <= bw) col[i - j] = T(pv[q]) + col[i - j];
        }
      }
      col[0] = T(reg[j]) + col[0];
      dmax[0] = nanmax(dmax[0], double(col[0]));
    }
    reduce<0, 1>(dummy, dmax);
    const double jit = (sizeof(T) == 8 ? 1e-14 : 2.384185791015625e-07) * dmax[0];
    for (int j = tid; j < n; j += NT) L[size_t(j) * ldl] = T(double(L[size_t(j) * ldl]) + jit);
    sync();
    QTQP_TOC(kPhGram);
    QTQP_RETIC();
    const int warp = tid >> 5, lane = tid & 31;
    constexpr int NW = NT / 32;
    T il_prev = T(1);
    int info = 0;
    for (int k = 0; k <= n; ++k) {
      if (k > 0) {  // finish column k-1
        T* ck = L + size_t(k - 1) * ldl;
        const T il = il_prev;
        const int rows = min(bw, n - k);
        for (int d = 1 + tid; d <= rows; d += NT) ck[d] *= il;
        if (tid == NT - 1) ck[0] = il;
      }
      if (k == n) break;
      const T* ck = L + size_t(k) * ldl;
      const T d = ck[0];
      if (!(d > T(0))) {
        info = k + 1;
        break;
      }
      const T il = rsqrt(d), inv_d = il * il;
      const int last = min(n - 1, k + bw);
      for (int j = k + 1 + warp; j <= last; j += NW) {
        const T t = ck[j - k] * inv_d;
        T* cj = L + size_t(j) * ldl;
        for (int i = j + lane; i <= last; i += 32) cj[i - j] = fma(-ck[i - k], t, cj[i - j]);
      }
      il_prev = il;
      sync();
    }
    sync();
    QTQP_TOC(kPhChol);
    return info;
  }

  // Solves L L^T v = v (column band storage, reciprocal diagonal): forward
  // into w, backward into v.  With the shared-memory window the blocked
  // solves below run (the whole group); without it one warp walks the
  // columns in global memory.  In grid mode the partitioned solve runs
  // (band_grid.cuh).
  template <typename T>
  __device__ void band_chol_solve(T* v, T* w) {
    if constexpr (FMT == kFmtSparse) {
      sparse_solve<T>(*this, v, w);
    } else if constexpr (NT > 1024) {
      bandp_solve<T>(*this, v, w);
    } else {
      if (bwin == nullptr) {
        band_chol_solve_global<T>(v, w);
        return;
      }
      band_fwd_blocked<T, NT>(v, w, 0, n, n, tid);
      band_bwd_blocked<T, NT>(v, w, 0, n, n, tid);
    }
  }

  // Blocked band triangular solves, run by all BT threads of the group (lt:
  // this thread's index).  Forward: z_k = (v_k - sum_c l_kc z_c) / l_kk for
  // the columns [lo, lo + ne) into w[k], the rows [lo + ne, R) of v receiving
  // their updates.  Backward: x_k = (w_k - sum_d l_{k+d,k} x_{k+d}) / l_kk for
  // k in [lo, hi) into v[k], the rows [hi, R) holding known values of x in v
  // (the separator that follows a partition).
  // per block of 8 columns one thread solves the 8 x 8 diagonal block, then
  // one thread per row applies the block's 8 values to the next bw rows, with
  // the next block's factor entries copied in (cp.async) meanwhile.  The
  // active vector entries live in 256 circular slots of shared memory.
  static constexpr int kSolveBlk = 8;
  template <typename T, int BT>
  __device__ void band_fwd_blocked(T* v, T* w, int lo, int ne, int R, int lt) {
    constexpr int KB = kSolveBlk;
    const int bw = this->bw, ldl = bw + 1, hi = lo + ne;
    const T* L = reinterpret_cast<const T*>(Lb);
    T* win = reinterpret_cast<T*>(bwin);  // 256 slots: row r at r & 255
    T* pan = win + 256;                   // 2 x (KB ldl): factor columns of a block
    T* zz = pan + 2 * KB * ldl;           // the block's KB values
    auto issue = [&](int k0, int buf) {
      T* dst = pan + buf * KB * ldl;
      const int nel = min(KB, hi - k0) * ldl;
      for (int e = lt; e < KB * ldl; e += BT)
        cp_async_elem(dst + e, L + (e < nel ? size_t(k0) * ldl + e : 0), e < nel);
      cp_async_commit();
    };
    int loaded = min(R, lo + bw + KB);
    for (int r = lo + lt; r < loaded; r += BT) win[r & 255] = v[r];
    if (lo < hi) issue(lo, 0);
    int buf = 0;
    for (int k0 = lo; k0 < hi; k0 += KB, buf ^= 1) {
      const int pw = min(KB, hi - k0);
      // This block's columns have landed and every thread is done with the
      // previous block: the next block's copies may now fill the other buffer.
      cp_async_wait<0>();
      group_sync<BT>();
      if (k0 + KB < hi) issue(k0 + KB, buf ^ 1);
      const T* pc = pan + buf * KB * ldl;  // column k0 + c: pc[c * ldl + d], d = row - column
      if (lt == 0) {
        T zl[KB];
#pragma unroll
        for (int c = 0; c < KB; ++c) {
          if (c < pw) {
            T t = win[(k0 + c) & 255];
#pragma unroll
            for (int c2 = 0; c2 < c; ++c2)
              if (c - c2 <= bw) t = fma(-pc[c2 * ldl + (c - c2)], zl[c2], t);
            zl[c] = t * pc[c * ldl];
            zz[c] = zl[c];
            w[k0 + c] = zl[c];
          }
        }
      }
      group_sync<BT>();
      const int rend = min(R, k0 + pw + bw);
      for (int r = k0 + pw + lt; r < rend; r += BT) {
        T t = win[r & 255];
#pragma unroll
        for (int c = 0; c < KB; ++c) {
          const int d = r - k0 - c;
          if (c < pw && d <= bw) t = fma(-pc[c * ldl + d], zz[c], t);
        }
        win[r & 255] = t;
      }
      const int nload = min(R, k0 + 2 * KB + bw);
      for (int r = loaded + lt; r < nload; r += BT) win[r & 255] = v[r];
      loaded = max(loaded, nload);
    }
    cp_async_wait<0>();
    group_sync<BT>();
    for (int r = hi + lt; r < R; r += BT) v[r] = win[r & 255];
    group_sync<BT>();
  }

  template <typename T, int BT>
  __device__ void band_bwd_blocked(T* v, T* w, int lo, int hi, int R, int lt) {
    constexpr int KB = kSolveBlk;
    const int bw = this->bw, ldl = bw + 1;
    const T* L = reinterpret_cast<const T*>(Lb);
    T* win = reinterpret_cast<T*>(bwin);
    T* stg = win + 256;                   // 2 x ((bw + KB) x KB): entries L(kb + q, i)
    T* xx = stg + 2 * (bw + KB) * KB;     // the block's KB values
    const int SR = bw + KB;               // staged rows per block: i in [kb - bw, kb + KB)
    // Stage, for the block of rows [kb, k1], the entries L(kb + q, i) (band
    // column i, offset kb + q - i) for i in [kb - bw, k1].
    auto issue = [&](int kb, int k1, int buf) {
      T* dst = stg + buf * SR * KB;
      for (int e = lt; e < SR * KB; e += BT) {
        const int ii = e / KB, q = e - ii * KB, i = kb - bw + ii, d = kb + q - i;
        const bool ok = i >= lo && i <= k1 && kb + q <= k1 && d >= 0 && d <= bw;
        cp_async_elem(dst + e, L + (ok ? size_t(i) * ldl + d : 0), ok);
      }
      cp_async_commit();
    };
    // Window: w for rows [max(lo, hi - bw - KB), hi), the known x for [hi, R).
    const int wlo = max(lo, hi - bw - KB);
    for (int r = wlo + lt; r < R; r += BT) win[r & 255] = r >= hi ? v[r] : w[r];
    int kb = max(lo, hi - KB);
    if (lo < hi) issue(kb, hi - 1, 0);
    group_sync<BT>();
    // Known rows [hi, R): w_i -= sum_r L(r, i) x_r for i in [hi - bw, hi).
    if (R > hi) {
      for (int i = max(lo, hi - bw) + lt; i < hi; i += BT) {
        T t = win[i & 255];
        const int rmax = min(R - 1, i + bw);
        for (int r = hi; r <= rmax; ++r) t = fma(-L[size_t(i) * ldl + (r - i)], win[r & 255], t);
        win[i & 255] = t;
      }
    }
    int loaded = wlo;  // rows [loaded, hi) are in the window
    int buf = 0;
    for (int k1 = hi - 1; k1 >= lo; k1 = kb - 1, buf ^= 1) {
      kb = max(lo, k1 - KB + 1);
      const int pw = k1 - kb + 1;
      const int kbn = max(lo, kb - KB);
      // As in the forward: this block's entries have landed and the other
      // buffer is free once every thread has passed the barrier.
      cp_async_wait<0>();
      group_sync<BT>();
      if (kb > lo) issue(kbn, kb - 1, buf ^ 1);
      const T* sg = stg + buf * SR * KB;  // L(kb + q, i) at sg[(i - kb + bw) * KB + q]
      if (lt == 0) {
        T xl[KB];
#pragma unroll
        for (int c = KB - 1; c >= 0; --c) {
          if (c < pw) {
            const int r = kb + c;
            T t = win[r & 255];
#pragma unroll
            for (int c2 = c + 1; c2 < KB; ++c2)
              if (c2 < pw) t = fma(-sg[(c + bw) * KB + c2], xl[c2], t);
            xl[c] = t * sg[(c + bw) * KB + c];
            xx[c] = xl[c];
            v[r] = xl[c];
          }
        }
      }
      group_sync<BT>();
      for (int i = max(lo, kb - bw) + lt; i < kb; i += BT) {
        T t = win[i & 255];
        const T* si = sg + (i - kb + bw) * KB;
#pragma unroll
        for (int q = 0; q < KB; ++q)
          if (q < pw) t = fma(-si[q], xx[q], t);
        win[i & 255] = t;
      }
      const int nload = max(lo, kbn - bw);
      for (int r = nload + lt; r < loaded; r += BT) win[r & 255] = w[r];
      loaded = min(loaded, nload);
    }
    cp_async_wait<0>();
    group_sync<BT>();
  }

  template <typename T>
  __device__ void band_chol_solve_global(T* v, T* w) {
    QTQP_BAND_LOCALS;
    const T* L = reinterpret_cast<const T*>(Lb);
    if (tid < 32) {
      const int lane = tid;
      for (int k = 0; k < n; ++k) {
        const T* ck = L + size_t(k) * ldl;
        const T zk = v[k] * ck[0];
        const int rows = min(bw, n - 1 - k);
        for (int d = 1 + lane; d <= rows; d += 32) v[k + d] = fma(-ck[d], zk, v[k + d]);
        if (lane == 0) w[k] = zk;
        __syncwarp();
      }
      for (int k = n - 1; k >= 0; --k) {
        const T xk = w[k] * L[size_t(k) * ldl];
        const int rows = min(bw, k);
        for (int d = 1 + lane; d <= rows; d += 32) {
          const int i = k - d;
          w[i] = fma(-L[size_t(i) * ldl + d], xk, w[i]);
        }
        if (lane == 0) v[k] = xk;
        __syncwarp();
      }
    }
    sync();
  }

  __device__ void band_kkt_solve(const double* r, double* out, bool accumulate, bool fp64) {
    QTQP_BAND_LOCALS;
    QTQP_TIC();
    const double* iry = vec(kPI);
    double* tmp = vec(kTMP);
    float* t32 = this->t32();
    for (int j = tid; j < n; j += NT) {
      double acc = 0.0;
      for (int q = jp[j]; q < jp[j + 1]; ++q) {
        const int i = jx[q];
        acc = fma(at[q], iry[n + i] * r[n + i], acc);
      }
      const double g = r[j] + acc;
      if (fp64) {
        tmp[j] = g;
      } else {
        t32[j] = float(g);
      }
    }
    sync();
    if (fp64) {
      band_chol_solve<double>(tmp, vec(kW));
    } else {
      band_chol_solve<float>(t32, t32 + n);
    }
    for (int k = tid; k < N; k += NT) {
      double val;
      if (k < n) {
        val = fp64 ? tmp[k] : double(t32[k]);
      } else {
        const int i = k - n;
        double ax = 0.0;
        if (fp64) {
          for (int q = ip[i]; q < ip[i + 1]; ++q) ax = fma(av[q], tmp[ix[q]], ax);
        } else {
          for (int q = ip[i]; q < ip[i + 1]; ++q) ax = fma(av[q], double(t32[ix[q]]), ax);
        }
        val = iry[k] * (ax - r[k]);
      }
      out[k] = accumulate ? out[k] + val : val;
    }
    QTQP_TOC(kPhSolve);
  }

  __device__ void band_kkt_residual(const double* v, const double* krhs, double* res,
                                    double& mres, double& vnan) const {
    QTQP_BAND_LOCALS;
    const double* reg = vec(kREG);
    const double* corr = vec(kCORR);
    for (int k = tid; k < N; k += NT) {
      double kv;
      if (k < n) {
        double t = band_poff_row(v, k);
        t += reg[k] * v[k];
        kv = t + band_at_col(v, k);
      } else {
        kv = band_a_row(v, k - n) - (-reg[k]) * v[k];
      }
      const double rk = krhs[k] - kv + corr[k] * v[k];
      res[k] = rk;
      mres = nanmax(mres, fabs(rk));
      vnan = fmax(vnan, (v[k] != v[k]) ? 1.0 : 0.0);
    }
  }
};

template <int NT>
using DenseIpm = Ipm<NT, kFmtDense>;

}  // namespace qtqp
