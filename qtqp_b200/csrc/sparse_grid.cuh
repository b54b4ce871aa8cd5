// Supernodal Cholesky factorisation and solves of the Gram matrix
// G = P_off + diag(Rx) + A^T diag(1/Ry) A for one sparse QP on the whole GPU
// (grid mode of the shared device IPM, Ipm<NT, kFmtSparse>).  It takes the
// role of the reference's sparse direct backends behind the plugin interface
// (src/qtqp/solvers_sparse.py:96-121, src/qtqp/solvers_gpu.py:27-116), on the
// dense backend's Gram reduction (src/qtqp/solvers_dense.py:99-116).
//
// The symbolic stage (sparse_symbolic.cu) fixes the ordering, the supernodes
// (column ranges [first_s, first_{s+1}) of width <= kSnMaxW), each one's
// sorted row structure R_s (its own columns first) and its values, stored
// column-major |R_s| x w_s at valptr[s].  Numeric phases:
//  * assembly: every stored value is zeroed, then each lower entry (i, j) of
//    G is computed (a merge of columns i and j of A, plus P and the diagonal)
//    and written to its position; the dense backend's relative jitter
//    (1e-14 max diag) is added to the diagonal;
//  * factorisation, left-looking per supernode s: for every descendant d
//    with rows in s's column range (the update list: d, the first such row
//    `off` of R_d and their number `cnt`), L_s[rows, cols] -= L_d[off:, :]
//    L_d[off:off+cnt, :]^T, scattered by the position of each row of R_d in
//    R_s; then the Cholesky of the diagonal block in shared memory and the
//    triangular solve of the rows below it.  The diagonal keeps 1 / l_jj;
//  * forward solve: each supernode subtracts the stored products z_d =
//    L_d[r, :] y_d of its descendants' rows in its columns, solves with its
//    diagonal block, and stores its own products z_s for the rows below;
//  * backward solve: partial sums L_s[slab, :]^T x[rows] per row slab, then
//    per supernode their sum in slab order and the transposed block solve.
// No atomics: every result has a single writer and sums run in a fixed
// order, so the results are reproducible run to run.
// Order: each block first runs the subtrees the symbolic stage gave it (their
// supernodes in postorder, no grid barrier; a supernode is one block's work).
// Above the subtrees, each level is spread over the whole grid in 64-row
// slabs: the factorisation in three steps (updates of every slab, diagonal
// blocks, rows below), each solve direction in two (diagonal solves and the
// slabs' products / partial sums), with a grid barrier after each step.  The
// backward solve runs the schedule in reverse.
#pragma once

#include "dense_ipm.cuh"

namespace qtqp {

constexpr int kSparseGridBlocks = 128;
constexpr int kSparseGridNT = kSparseGridBlocks * kGridBT;
constexpr int kSnMaxW = kSnMaxWidth;    // widest supernode (the symbolic stage's cap)
constexpr int kSnLd = kSnMaxW + 1;      // leading dimension of the diagonal block in smem
constexpr int kSnStageK = 32;           // descendant columns staged per pass
constexpr int kSnCg = 8;                // target columns per thread in an update pass
constexpr int kSnSlab = kSnSlabRows;    // rows of a top-level supernode per work item
constexpr int kSnMaxSplit = 32;         // blocks sharing one slab's update list, at most
// Dynamic shared memory of a block: the diagonal block, its reciprocal
// diagonal, the staged descendant rows, and the partial sums of the solves.
constexpr size_t kSparseSmemElems =
    size_t(kSnMaxW) * kSnLd + kSnMaxW + size_t(kSnMaxW) * (kSnStageK + 1) + kGridBT + kSnMaxW;
constexpr size_t kSparseSmem = kSparseSmemElems * sizeof(double);

// Device view of the symbolic plan (qtqp_sparse_desc offsets into the pools)
// and the factor's value storage.
struct SnFactor {
  int n, nsuper, top_levels;
  int64_t nvals, ngram, nrows, nslabs;
  const int32_t* first;
  const int32_t* colsn;
  const int32_t* rows;
  const int32_t* upd_ptr;
  const int32_t* upd_src;
  const int32_t* upd_off;
  const int32_t* upd_cnt;
  const int32_t* cta_ptr;
  const int32_t* cta_range;
  const int32_t* top_ptr;
  const int32_t* top_list;
  const int32_t* top_slab;  // prefix counts of row slabs over top_list (ntop + 1)
  const int32_t* gcol;
  const int32_t* grow;
  const int64_t* rowptr;
  const int64_t* valptr;
  const int64_t* gpos;
  double* vals;
  double* zbuf;  // forward products per stored row (nrows)
  double* pbuf;  // backward partial sums per top-level row slab (kSnMaxW each)
  double* ubuf;  // partial updates of split row slabs (kSparseGridBlocks x kSnSlab x kSnMaxW)
};

// Position of `key` in the sorted rows[0 .. len) (present by construction).
__device__ __forceinline__ int sn_find(const int32_t* rows, int len, int key) {
  int lo = 0, hi = len;
  while (lo < hi) {
    const int mid = (lo + hi) >> 1;
    if (rows[mid] < key) {
      lo = mid + 1;
    } else {
      hi = mid;
    }
  }
  return lo;
}

// G[i, j] for i >= j: sum_r a_ri a_rj / Ry_r over the rows shared by columns
// i and j of A (a merge of the two sorted CSC columns), plus P_ij (i != j)
// or the regularised diagonal (i == j).
template <class S>
__device__ double sn_gram_entry(const S& s, int i, int j) {
  const double* wsc = s.vec(kPW);
  const int* jp = s.jp;
  const int* jx = s.jx;
  const double* at = s.at;
  const int n = s.n;
  double acc = 0.0;
  int qi = jp[i], qj = jp[j];
  const int ei = jp[i + 1], ej = jp[j + 1];
  if (i == j) {
    for (; qj < ej; ++qj) {
      const double v = at[qj] * wsc[n + jx[qj]];
      acc = fma(v, v, acc);
    }
    return acc + s.vec(kREG)[j];
  }
  while (qi < ei && qj < ej) {
    const int ri = jx[qi], rj = jx[qj];
    if (ri == rj) {
      const double w = wsc[n + ri];
      acc = fma(at[qi] * w, at[qj] * w, acc);
      ++qi;
      ++qj;
    } else if (ri < rj) {
      ++qi;
    } else {
      ++qj;
    }
  }
  if (s.has_p) {  // P_ij from row i of P (CSR, sorted columns)
    const int* px = s.px;
    const int lo = s.pp[i], hi = s.pp[i + 1];
    const int q = lo + sn_find(px + lo, hi - lo, j);
    if (q < hi && px[q] == j) acc += s.pv[q];
  }
  return acc;
}

// Updates of rows [r0, r1) (at most kSnSlab of them) of supernode sn's block
// from all its descendants (the calling block): L_s[r, j] -= the sum, over
// the descendants d holding both row R_s[r] and column f + j, of
// L_d[row, :] . L_d[col, :].  Each thread owns up to two (target row, kSnCg
// target columns) items and keeps their sums in registers while the block
// walks the update list in order: per descendant, the rows of R_d inside the
// slab (a range found by two binary searches, the same in every thread), then
// each item's row and columns in it.  No two threads write the same entry,
// every sum runs in a fixed order, and no barrier separates the descendants.
//
// [u0, u1) is the part of the update list to apply; out == nullptr subtracts
// the sums from the block, else they go to out (kSnSlab x kSnMaxW, row r - r0
// at out[(r - r0) * kSnMaxW + col]) for sn_add_partials.
template <typename T>
__device__ void sn_update_slab(const SnFactor& F, T* L, int sn, int r0, int r1, int u0, int u1,
                               double* out) {
  const int t = threadIdx.x;
  const int f = F.first[sn], w = F.first[sn + 1] - f;
  const int nr = int(F.rowptr[sn + 1] - F.rowptr[sn]);
  const int32_t* R = F.rows + F.rowptr[sn];
  T* Ls = L + F.valptr[sn];
  const int ngrp = (w + kSnCg - 1) / kSnCg;
  const int rows = r1 - r0;
  const int lo_key = R[r0], hi_key = R[r1 - 1];
  constexpr int kItems = kSnSlab * ((kSnMaxW + kSnCg - 1) / kSnCg) / kGridBT;
  static_assert(kItems * kGridBT >= kSnSlab * ((kSnMaxW + kSnCg - 1) / kSnCg), "items");
  int key[kItems], ck0[kItems], ck1[kItems];
  double acc[kItems][kSnCg];
#pragma unroll
  for (int it = 0; it < kItems; ++it) {
    const int item = t + it * kGridBT;
    key[it] = -1;
    if (item < rows * ngrp) {
      const int r = r0 + item % rows, cg = item / rows;
      ck0[it] = f + cg * kSnCg;
      ck1[it] = min(ck0[it] + kSnCg, f + w);
      if (R[r] >= ck0[it]) key[it] = R[r];  // else entirely in the upper triangle
    }
#pragma unroll
    for (int q = 0; q < kSnCg; ++q) acc[it][q] = 0.0;
  }
  for (int u = u0; u < u1; ++u) {
    const int off = F.upd_off[u], cnt = F.upd_cnt[u];
    const int d = F.upd_src[u];
    const int nrd = int(F.rowptr[d + 1] - F.rowptr[d]);
    const int32_t* Rd = F.rows + F.rowptr[d] + off;
    const int a = sn_find(Rd, nrd - off, lo_key);
    const int b = sn_find(Rd, nrd - off, hi_key + 1);
    if (a >= b) continue;  // none of d's rows in this slab
    const int wd = F.first[d + 1] - F.first[d];
    const T* Ld = L + F.valptr[d] + off;
#pragma unroll
    for (int it = 0; it < kItems; ++it) {
      if (key[it] < 0) continue;
      const int i = a + sn_find(Rd + a, b - a, key[it]);
      if (i >= b || Rd[i] != key[it]) continue;
      int c = sn_find(Rd, cnt, ck0[it]);
      const int c1 = sn_find(Rd, cnt, ck1[it]);
      const T* Li = Ld + i;
#pragma unroll
      for (int q = 0; q < kSnCg; ++q) {
        if (c < c1 && Rd[c] == ck0[it] + q) {
          const T* Lc = Ld + c;
          double sum = 0.0;
          for (int k = 0; k < wd; ++k)
            sum = fma(double(Li[size_t(k) * nrd]), double(Lc[size_t(k) * nrd]), sum);
          acc[it][q] += sum;
          ++c;
        }
      }
    }
  }
#pragma unroll
  for (int it = 0; it < kItems; ++it) {
    if (key[it] < 0) continue;
    const int item = t + it * kGridBT;
    const int r = r0 + item % rows, cg = item / rows;
#pragma unroll
    for (int q = 0; q < kSnCg; ++q) {
      if (ck0[it] + q < ck1[it] && ck0[it] + q <= key[it]) {
        const int col = cg * kSnCg + q;
        if (out != nullptr) {
          out[(r - r0) * kSnMaxW + col] = acc[it][q];
        } else {
          T* dst = Ls + size_t(r) + size_t(col) * nr;
          *dst = T(double(*dst) - acc[it][q]);
        }
      }
    }
  }
  __syncthreads();
}

// All rows [r0, r1) of supernode sn, slab by slab, from its whole update list.
template <typename T>
__device__ void sn_update_rows(const SnFactor& F, T* L, double* smem, int sn, int r0, int r1) {
  (void)smem;
  for (int lo = r0; lo < r1; lo += kSnSlab)
    sn_update_slab<T>(F, L, sn, lo, min(r1, lo + kSnSlab), F.upd_ptr[sn], F.upd_ptr[sn + 1],
                      nullptr);
}

// Subtracts from rows [r0, r1) of supernode sn the partial sums that `parts`
// blocks left in part[0 .. parts) (sn_update_slab with out), in that order.
template <typename T>
__device__ void sn_add_partials(const SnFactor& F, T* L, int sn, int r0, int r1,
                                const double* part, int parts) {
  const int f = F.first[sn], w = F.first[sn + 1] - f;
  const int nr = int(F.rowptr[sn + 1] - F.rowptr[sn]);
  const int32_t* R = F.rows + F.rowptr[sn];
  T* Ls = L + F.valptr[sn];
  const int rows = r1 - r0;
  for (int e = threadIdx.x; e < rows * w; e += blockDim.x) {
    const int rl = e % rows, col = e / rows;
    if (f + col > R[r0 + rl]) continue;  // the block's upper triangle
    double sum = 0.0;
    for (int c = 0; c < parts; ++c) sum += part[size_t(c) * kSnSlab * kSnMaxW + rl * kSnMaxW + col];
    T* dst = Ls + size_t(r0 + rl) + size_t(col) * nr;
    *dst = T(double(*dst) - sum);
  }
  __syncthreads();
}

// Cholesky of supernode sn's diagonal block (the calling block): the factor
// goes back to L with 1 / l_jj on the diagonal, and stays in shared memory
// (D, rdiag) for sn_panel_rows.
template <typename T>
__device__ void sn_diag(const SnFactor& F, T* L, double* smem, int* info, int sn) {
  const int t = threadIdx.x;
  const int f = F.first[sn], w = F.first[sn + 1] - f;
  const int nr = int(F.rowptr[sn + 1] - F.rowptr[sn]);
  T* Ls = L + F.valptr[sn];
  double* D = smem;                     // w x w (ld kSnLd)
  double* rdiag = D + kSnMaxW * kSnLd;  // 1 / l_jj
  for (int idx = t; idx < w * w; idx += blockDim.x) {
    const int c = idx / w, r = idx % w;
    if (r >= c) D[r * kSnLd + c] = double(Ls[size_t(r) + size_t(c) * nr]);
  }
  __syncthreads();
  // Right-looking in panels of 8 columns: warp 0 factors a panel in
  // registers (lane l holds rows p0 + l and p0 + l + 32 of the panel's
  // columns; pivots and multipliers by shuffles), then the whole block
  // applies its rank-8 update to the rest.  Two barriers per panel.
  const int lane = t & 31;
  for (int p0 = 0; p0 < w; p0 += 8) {
    const int pw = min(8, w - p0);
    if (t < 32) {
      const int ra = p0 + lane, rb = p0 + lane + 32;
      double va[8], vb[8];
#pragma unroll
      for (int c = 0; c < 8; ++c) {
        va[c] = (c < pw && ra < w) ? D[ra * kSnLd + p0 + c] : 0.0;
        vb[c] = (c < pw && rb < w) ? D[rb * kSnLd + p0 + c] : 0.0;
      }
#pragma unroll
      for (int c = 0; c < 8; ++c) {
        if (c < pw) {
          const double dk = __shfl_sync(0xffffffffu, va[c], c);  // pivot row p0 + c = lane c
          const double rk = dk > 0.0 ? 1.0 / sqrt(dk) : __longlong_as_double(0x7ff8000000000000ll);
          if (lane > c) va[c] *= rk;
          vb[c] *= rk;
          if (lane == c) va[c] = dk > 0.0 ? dk * rk : va[c];  // l_kk (kept in D, 1 / l_kk in rdiag)
          if (lane == 0) {
            rdiag[p0 + c] = rk;
            if (!(dk > 0.0)) atomicCAS(info, 0, f + p0 + c + 1);
          }
#pragma unroll
          for (int c2 = c + 1; c2 < 8; ++c2) {
            if (c2 < pw) {
              const double l2 = __shfl_sync(0xffffffffu, va[c], c2);  // L[p0 + c2][p0 + c]
              if (lane >= c2) va[c2] = fma(-va[c], l2, va[c2]);
              vb[c2] = fma(-vb[c], l2, vb[c2]);
            }
          }
        }
      }
#pragma unroll
      for (int c = 0; c < 8; ++c) {
        if (c < pw && ra < w && lane >= c) D[ra * kSnLd + p0 + c] = va[c];
        if (c < pw && rb < w) D[rb * kSnLd + p0 + c] = vb[c];
      }
    }
    __syncthreads();
    // Trailing update of rows and columns >= p0 + pw.
    const int t0 = p0 + pw, tn = w - t0;
    for (int idx = t; idx < tn * tn; idx += blockDim.x) {
      const int i = t0 + idx / tn, j = t0 + idx % tn;
      if (j > i) continue;
      double sum = 0.0;
#pragma unroll
      for (int c = 0; c < 8; ++c)
        if (c < pw) sum = fma(D[i * kSnLd + p0 + c], D[j * kSnLd + p0 + c], sum);
      D[i * kSnLd + j] -= sum;
    }
    __syncthreads();
  }
  for (int idx = t; idx < w * w; idx += blockDim.x) {
    const int c = idx / w, r = idx % w;
    if (r > c) Ls[size_t(r) + size_t(c) * nr] = T(D[r * kSnLd + c]);
    if (r == c) Ls[size_t(r) + size_t(c) * nr] = T(rdiag[c]);
  }
  __syncthreads();
}

// Rows [r0, r1) (all at or below the diagonal block) of supernode sn: the
// triangular solve x L_bb^T = a, forward substitution per row.  load: read
// the factored diagonal block back from L into shared memory first (another
// block factored it).
template <typename T>
__device__ void sn_panel_rows(const SnFactor& F, T* L, double* smem, int sn, int r0, int r1,
                              bool load) {
  const int t = threadIdx.x;
  const int w = F.first[sn + 1] - F.first[sn];
  const int nr = int(F.rowptr[sn + 1] - F.rowptr[sn]);
  T* Ls = L + F.valptr[sn];
  double* D = smem;
  double* rdiag = D + kSnMaxW * kSnLd;
  if (load) {
    for (int idx = t; idx < w * w; idx += blockDim.x) {
      const int c = idx / w, r = idx % w;
      if (r > c) D[r * kSnLd + c] = double(Ls[size_t(r) + size_t(c) * nr]);
      if (r == c) rdiag[c] = double(Ls[size_t(r) + size_t(c) * nr]);
    }
    __syncthreads();
  }
  for (int r = max(r0, w) + t; r < r1; r += blockDim.x) {
    for (int k = 0; k < w; ++k) {
      double acc = double(Ls[size_t(r) + size_t(k) * nr]);
      for (int p = 0; p < k; ++p)
        acc = fma(-double(Ls[size_t(r) + size_t(p) * nr]), D[k * kSnLd + p], acc);
      Ls[size_t(r) + size_t(k) * nr] = T(acc * rdiag[k]);
    }
  }
  __syncthreads();
}

// Left-looking factorisation of supernode `sn` by the calling block alone.
template <typename T>
__device__ void sn_factor_one(const SnFactor& F, T* L, double* smem, int* info, int sn) {
  const int nr = int(F.rowptr[sn + 1] - F.rowptr[sn]);
  sn_update_rows<T>(F, L, smem, sn, 0, nr);
  sn_diag<T>(F, L, smem, info, sn);
  sn_panel_rows<T>(F, L, smem, sn, 0, nr, false);
}

// The supernode and row range [r0, r1) of work item `item` of a top level
// whose supernodes are top_list[q0 .. q1) and whose row slabs (kSnSlab rows
// each) are numbered top_slab[q0] .. top_slab[q1] - 1.
__device__ __forceinline__ void sn_slab_item(const SnFactor& F, int q0, int q1, int item,
                                             int& sn, int& r0, int& r1) {
  int lo = q0, hi = q1 - 1;  // the last q with top_slab[q] <= item
  while (lo < hi) {
    const int mid = (lo + hi + 1) >> 1;
    if (F.top_slab[mid] <= item) {
      lo = mid;
    } else {
      hi = mid - 1;
    }
  }
  sn = F.top_list[lo];
  const int nr = int(F.rowptr[sn + 1] - F.rowptr[sn]);
  r0 = (item - F.top_slab[lo]) * kSnSlab;
  r1 = min(nr, r0 + kSnSlab);
}

// The forward contributions of the update list's entries [ua, ub) to the
// columns of supernode sn, per thread group (thread t: column t % W32, group
// t / W32 over every G-th entry; W32 = 32 or 64 by the width), into
// part[t]; ends with a barrier.
__device__ __forceinline__ void sn_fwd_gather_block(const SnFactor& F, const double* z, int sn,
                                                    int ua, int ub, double* part) {
  const int t = threadIdx.x;
  const int f = F.first[sn], w = F.first[sn + 1] - f;
  const int W32 = w <= 32 ? 32 : 64;
  const int G = blockDim.x / W32;
  const int j = t % W32, g = t / W32;
  double acc = 0.0;
  if (j < w) {
    for (int u = ua + g; u < ub; u += G) {
      const int d = F.upd_src[u], off = F.upd_off[u], cnt = F.upd_cnt[u];
      const int32_t* Rd = F.rows + F.rowptr[d] + off;
      const int c = sn_find(Rd, cnt, f + j);
      if (c < cnt && Rd[c] == f + j) acc += z[F.rowptr[d] + off + c];
    }
  }
  part[t] = acc;
  __syncthreads();
}

// sn_fwd_gather_block over [ua, ub), its groups summed in order into out[j]
// (j < the supernode's width), for sn_fwd_diag's `parts`.
__device__ __forceinline__ void sn_fwd_gather(const SnFactor& F, const double* z, double* smem,
                                              int sn, int ua, int ub, double* out) {
  const int t = threadIdx.x;
  const int w = F.first[sn + 1] - F.first[sn];
  const int W32 = w <= 32 ? 32 : 64;
  const int G = blockDim.x / W32;
  double* part = smem + kSnMaxW * kSnLd + kSnMaxW + kSnMaxW * (kSnStageK + 1);
  sn_fwd_gather_block(F, z, sn, ua, ub, part);
  if (t < w) {
    double sum = 0.0;
    for (int q = 0; q < G; ++q) sum += part[q * W32 + t];
    out[t] = sum;
  }
  __syncthreads();
}

// Forward solve, step 1 for supernode `sn` (the calling block): v[cols] -=
// the products z of its descendants with the rows in its columns (z_d[r] =
// L_d[r, :] y_d, stored per row of R_d by step 2), then y_cols = L_bb^{-1}
// v[cols] on one warp with the diagonal block in shared memory.  The
// contributions are summed in a fixed order (thread groups over the update
// list, then the groups in turn), so the result does not depend on timing.
//
// parts != nullptr: the contributions were gathered by sn_fwd_gather into
// parts[0 .. nparts) (kSnMaxW values each) and are subtracted in that order.
template <typename T>
__device__ void sn_fwd_diag(const SnFactor& F, const T* L, double* smem, const double* z, T* v,
                            int sn, const double* parts = nullptr, int nparts = 0) {
  const int t = threadIdx.x;
  const int f = F.first[sn], w = F.first[sn + 1] - f;
  const int nr = int(F.rowptr[sn + 1] - F.rowptr[sn]);
  const T* Ls = L + F.valptr[sn];
  double* D = smem;  // the diagonal block (factor, 1 / l_jj on the diagonal)
  double* part = smem + kSnMaxW * kSnLd + kSnMaxW + kSnMaxW * (kSnStageK + 1);
  double* yb = part + kGridBT;
  for (int idx = t; idx < w * w; idx += blockDim.x) {
    const int c = idx / w, r = idx % w;
    if (r >= c) D[r * kSnLd + c] = double(Ls[size_t(r) + size_t(c) * nr]);
  }
  const int W32 = w <= 32 ? 32 : 64;
  const int G = blockDim.x / W32;
  if (parts == nullptr) {
    sn_fwd_gather_block(F, z, sn, F.upd_ptr[sn], F.upd_ptr[sn + 1], part);
    if (t < w) {
      double bv = double(v[f + t]);
      for (int q = 0; q < G; ++q) bv -= part[q * W32 + t];
      yb[t] = bv;
    }
  } else if (t < w) {
    double bv = double(v[f + t]);
    for (int q = 0; q < nparts; ++q) bv -= parts[q * kSnMaxW + t];
    yb[t] = bv;
  }
  __syncthreads();
  if (t < 32) {  // one warp: lane l holds rows l and l + 32
    double r0 = t < w ? yb[t] : 0.0;
    double r1 = t + 32 < w ? yb[t + 32] : 0.0;
    for (int k = 0; k < w; ++k) {
      const double mine = k < 32 ? r0 : r1;
      const double yk = __shfl_sync(0xffffffffu, mine, k & 31) * D[k * kSnLd + k];
      if (t == (k & 31)) {
        if (k < 32) {
          r0 = yk;
        } else {
          r1 = yk;
        }
      }
      if (t > k && t < w) r0 = fma(-D[t * kSnLd + k], yk, r0);
      if (t + 32 > k && t + 32 < w) r1 = fma(-D[(t + 32) * kSnLd + k], yk, r1);
    }
    if (t < w) {
      v[f + t] = T(r0);
      yb[t] = r0;
    }
    if (t + 32 < w) {
      v[f + t + 32] = T(r1);
      yb[t + 32] = r1;
    }
  }
  __syncthreads();
}

// Forward solve, step 2: z[r] = L_s[r, :] y_s for the rows [r0, r1) of
// supernode sn below its diagonal block.  y_s is read from v (from_smem:
// from the yb slots that sn_fwd_diag of this block left in shared memory).
template <typename T>
__device__ void sn_fwd_rows(const SnFactor& F, const T* L, double* smem, double* z, const T* v,
                            int sn, int r0, int r1, bool from_smem) {
  const int t = threadIdx.x;
  const int f = F.first[sn], w = F.first[sn + 1] - f;
  const int nr = int(F.rowptr[sn + 1] - F.rowptr[sn]);
  const T* Ls = L + F.valptr[sn];
  double* yb = smem + kSnMaxW * kSnLd + kSnMaxW + kSnMaxW * (kSnStageK + 1) + kGridBT;
  if (!from_smem) {
    for (int k = t; k < w; k += blockDim.x) yb[k] = double(v[f + k]);
    __syncthreads();
  }
  double* zs = z + F.rowptr[sn];
  for (int r = max(r0, w) + t; r < r1; r += blockDim.x) {
    double acc = 0.0;
    for (int k = 0; k < w; ++k) acc = fma(double(Ls[size_t(r) + size_t(k) * nr]), yb[k], acc);
    zs[r] = acc;
  }
  __syncthreads();
}

// Backward solve, step 1: partial sums p[j] = sum_{r in [r0, r1), r >= w}
// L_s[r, j] x[R_s[r]] of supernode sn (the calling block), to `out` (w
// values).
template <typename T>
__device__ void sn_bwd_rows(const SnFactor& F, const T* L, const T* v, int sn, int r0, int r1,
                            double* out) {
  const int t = threadIdx.x, lane = t & 31, warp = t >> 5, nwarp = blockDim.x >> 5;
  const int w = F.first[sn + 1] - F.first[sn];
  const int nr = int(F.rowptr[sn + 1] - F.rowptr[sn]);
  const int32_t* R = F.rows + F.rowptr[sn];
  const T* Ls = L + F.valptr[sn];
  for (int j = warp; j < w; j += nwarp) {
    double acc = 0.0;
    for (int r = max(r0, w) + lane; r < r1; r += 32)
      acc = fma(double(Ls[size_t(r) + size_t(j) * nr]), double(v[R[r]]), acc);
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
    if (lane == 0) out[j] = acc;
  }
  __syncthreads();
}

// Backward solve, step 2: y_cols = v[cols] - (the partial sums of parts
// slabs, in order), then x_cols = L_bb^{-T} y_cols on one warp.
template <typename T>
__device__ void sn_bwd_diag(const SnFactor& F, const T* L, double* smem, const double* parts,
                            int nparts, T* v, int sn) {
  const int t = threadIdx.x;
  const int f = F.first[sn], w = F.first[sn + 1] - f;
  const int nr = int(F.rowptr[sn + 1] - F.rowptr[sn]);
  const T* Ls = L + F.valptr[sn];
  double* D = smem;
  double* yb = smem + kSnMaxW * kSnLd + kSnMaxW + kSnMaxW * (kSnStageK + 1) + kGridBT;
  for (int idx = t; idx < w * w; idx += blockDim.x) {
    const int c = idx / w, r = idx % w;
    if (r >= c) D[r * kSnLd + c] = double(Ls[size_t(r) + size_t(c) * nr]);
  }
  if (t < w) {
    double bv = double(v[f + t]);
    for (int q = 0; q < nparts; ++q) bv -= parts[q * kSnMaxW + t];
    yb[t] = bv;
  }
  __syncthreads();
  if (t < 32) {
    double r0 = t < w ? yb[t] : 0.0;
    double r1 = t + 32 < w ? yb[t + 32] : 0.0;
    for (int k = w - 1; k >= 0; --k) {
      const double mine = k < 32 ? r0 : r1;
      const double xk = __shfl_sync(0xffffffffu, mine, k & 31) * D[k * kSnLd + k];
      if (t == (k & 31)) {
        if (k < 32) {
          r0 = xk;
        } else {
          r1 = xk;
        }
      }
      // rows j < k: v_j -= L[k][j] x_k
      if (t < k) r0 = fma(-D[k * kSnLd + t], xk, r0);
      if (t + 32 < k) r1 = fma(-D[k * kSnLd + t + 32], xk, r1);
    }
    if (t < w) v[f + t] = T(r0);
    if (t + 32 < w) v[f + t + 32] = T(r1);
  }
  __syncthreads();
}

template <typename T, class S>
__device__ int sparse_factorize(S& s) {
  const SnFactor& F = *s.sn;
  T* L = reinterpret_cast<T*>(F.vals);
  const int tid = s.tid;
  constexpr int NT = kSparseGridNT;
  QTQP_TIC();
  if (tid == 0) *s.linfo = 0;
  for (int64_t e = tid; e < F.nvals; e += NT) L[e] = T(0);
  s.sync();
  double dmax[1] = {0.0};
  double dummy[1] = {0.0};
  for (int64_t e = tid; e < F.ngram; e += NT) {
    const int i = F.grow[e], j = F.gcol[e];
    const double g = sn_gram_entry(s, i, j);
    L[F.gpos[e]] = T(g);
    if (i == j) dmax[0] = nanmax(dmax[0], g);
  }
  s.template reduce<0, 1>(dummy, dmax);
  const double jit = (sizeof(T) == 8 ? 1e-14 : 2.384185791015625e-07) * dmax[0];
  for (int j = tid; j < F.n; j += NT) {
    const int sn = F.colsn[j];
    const int c = j - F.first[sn];
    const int64_t nr = F.rowptr[sn + 1] - F.rowptr[sn];
    T* p = L + F.valptr[sn] + c * nr + c;
    *p = T(double(*p) + jit);
  }
  s.sync();
  QTQP_TOC(kPhGram);
  QTQP_RETIC();
  double* smem = s.bwin;
  const int b = blockIdx.x;
  for (int q = F.cta_ptr[b]; q < F.cta_ptr[b + 1]; ++q)
    for (int sn = F.cta_range[2 * q]; sn <= F.cta_range[2 * q + 1]; ++sn)
      sn_factor_one<T>(F, L, smem, s.linfo, sn);
  s.sync();
  QTQP_TOC(kPhSnSub);
  QTQP_RETIC();
  // Above the subtrees, each level in three steps over the whole grid: the
  // updates of every row slab, the diagonal blocks, the rows below them.
  // A level with fewer row slabs than half the grid splits each slab's
  // update list over `split` blocks; their partial sums are added (in order)
  // by the diagonal step (slab 0 of each supernode) and the row step (the
  // other slabs), so the split costs no extra barrier.
  const int G = int(gridDim.x);
  for (int l = 0; l < F.top_levels; ++l) {
    const int q0 = F.top_ptr[l], q1 = F.top_ptr[l + 1];
    const int items = F.top_slab[q1] - F.top_slab[q0];
    int ulen = 0;  // update list entries of the level (the same in every block)
    for (int q = q0; q < q1; ++q) ulen += F.upd_ptr[F.top_list[q] + 1] - F.upd_ptr[F.top_list[q]];
    // At least 8 list entries per part on average: short lists stay whole.
    const int split = 2 * items > G ? 1
                                    : max(1, min(min(kSnMaxSplit, G / items), ulen / (8 * (q1 - q0))));
    QTQP_TIC();
    for (int it = b; it < items * split; it += G) {
      const int slab = it / split, part = it % split;
      int sn, r0, r1;
      sn_slab_item(F, q0, q1, F.top_slab[q0] + slab, sn, r0, r1);
      const int ua = F.upd_ptr[sn], len = F.upd_ptr[sn + 1] - ua;
      sn_update_slab<T>(F, L, sn, r0, r1, ua + len * part / split, ua + len * (part + 1) / split,
                        split > 1 ? F.ubuf + size_t(it) * kSnSlab * kSnMaxW : nullptr);
    }
    s.sync();
    QTQP_TOC(kPhSnTopUpd);
    QTQP_RETIC();
    for (int q = q0 + b; q < q1; q += G) {
      const int sn = F.top_list[q];
      if (split > 1) {
        const int slab = F.top_slab[q] - F.top_slab[q0];
        const int nr = int(F.rowptr[sn + 1] - F.rowptr[sn]);
        sn_add_partials<T>(F, L, sn, 0, min(nr, kSnSlab),
                           F.ubuf + size_t(slab) * split * kSnSlab * kSnMaxW, split);
      }
      sn_diag<T>(F, L, smem, s.linfo, sn);
    }
    s.sync();
    QTQP_TOC(kPhSnTopDiag);
    QTQP_RETIC();
    for (int it = b; it < items; it += G) {
      int sn, r0, r1;
      sn_slab_item(F, q0, q1, F.top_slab[q0] + it, sn, r0, r1);
      const int w = F.first[sn + 1] - F.first[sn];
      if (split > 1 && r0 > 0)
        sn_add_partials<T>(F, L, sn, r0, r1, F.ubuf + size_t(it) * split * kSnSlab * kSnMaxW,
                           split);
      if (r1 > w) sn_panel_rows<T>(F, L, smem, sn, r0, r1, true);
    }
    s.sync();
    QTQP_TOC(kPhSnTopPanel);
  }
  QTQP_TOC(kPhSnTop);
  return *reinterpret_cast<volatile int*>(s.linfo);
}

template <typename T, class S>
__device__ void sparse_solve(S& s, T* v, T* w) {
  (void)w;
  const SnFactor& F = *s.sn;
  const T* L = reinterpret_cast<const T*>(F.vals);
  double* smem = s.bwin;
  double* z = F.zbuf;
  double* parts = F.pbuf;
  const int b = blockIdx.x;
  QTQP_TIC();
  // Forward: the blocks' subtrees, then the top levels (the diagonal solves,
  // then every row slab's products).
  for (int q = F.cta_ptr[b]; q < F.cta_ptr[b + 1]; ++q)
    for (int sn = F.cta_range[2 * q]; sn <= F.cta_range[2 * q + 1]; ++sn) {
      sn_fwd_diag<T>(F, L, smem, z, v, sn);
      sn_fwd_rows<T>(F, L, smem, z, v, sn, 0, int(F.rowptr[sn + 1] - F.rowptr[sn]), true);
    }
  s.sync();
  QTQP_TOC(kPhSnFwdSub);
  QTQP_RETIC();
  const int G = int(gridDim.x);
  for (int l = 0; l < F.top_levels; ++l) {
    const int q0 = F.top_ptr[l], q1 = F.top_ptr[l + 1];
    // Long update lists are gathered by several blocks first (one more
    // barrier), each on a contiguous part, then summed in order.
    int ulen = 0;
    for (int q = q0; q < q1; ++q) ulen += F.upd_ptr[F.top_list[q] + 1] - F.upd_ptr[F.top_list[q]];
    const int nq = q1 - q0;
    const int split = ulen < 8 * kGridBT / 32 * nq || 2 * nq > G ? 1 : min(kSnMaxSplit, G / nq);
    if (split > 1) {
      for (int it = b; it < nq * split; it += G) {
        const int q = q0 + it / split, part = it % split;
        const int sn = F.top_list[q];
        const int ua = F.upd_ptr[sn], len = F.upd_ptr[sn + 1] - ua;
        sn_fwd_gather(F, z, smem, sn, ua + len * part / split, ua + len * (part + 1) / split,
                      F.ubuf + size_t(it) * kSnMaxW);
      }
      s.sync();
    }
    for (int q = q0 + b; q < q1; q += G)
      sn_fwd_diag<T>(F, L, smem, z, v, F.top_list[q],
                     split > 1 ? F.ubuf + size_t(q - q0) * split * kSnMaxW : nullptr, split);
    s.sync();
    if (l + 1 < F.top_levels) {  // the last level's products have no reader
      const int items = F.top_slab[q1] - F.top_slab[q0];
      for (int it = b; it < items; it += gridDim.x) {
        int sn, r0, r1;
        sn_slab_item(F, q0, q1, F.top_slab[q0] + it, sn, r0, r1);
        const int w = F.first[sn + 1] - F.first[sn];
        if (r1 > w) sn_fwd_rows<T>(F, L, smem, z, v, sn, r0, r1, false);
      }
      s.sync();
    }
  }
  QTQP_TOC(kPhSnFwdTop);
  QTQP_RETIC();
  // Backward: the top levels in reverse (every row slab's partial sums, then
  // the diagonal solves), then the subtrees in reverse.
  for (int l = F.top_levels - 1; l >= 0; --l) {
    const int q0 = F.top_ptr[l], q1 = F.top_ptr[l + 1];
    const int items = F.top_slab[q1] - F.top_slab[q0];
    for (int it = b; it < items; it += gridDim.x) {
      int sn, r0, r1;
      sn_slab_item(F, q0, q1, F.top_slab[q0] + it, sn, r0, r1);
      sn_bwd_rows<T>(F, L, v, sn, r0, r1, parts + size_t(F.top_slab[q0] + it) * kSnMaxW);
    }
    s.sync();
    for (int q = q0 + b; q < q1; q += gridDim.x)
      sn_bwd_diag<T>(F, L, smem, parts + size_t(F.top_slab[q]) * kSnMaxW,
                     F.top_slab[q + 1] - F.top_slab[q], v, F.top_list[q]);
    s.sync();
  }
  QTQP_TOC(kPhSnBwdTop);
  QTQP_RETIC();
  double* own = smem + kSnMaxW * kSnLd + kSnMaxW;  // one partial row (the staging area)
  for (int q = F.cta_ptr[b + 1] - 1; q >= F.cta_ptr[b]; --q)
    for (int sn = F.cta_range[2 * q + 1]; sn >= F.cta_range[2 * q]; --sn) {
      sn_bwd_rows<T>(F, L, v, sn, 0, int(F.rowptr[sn + 1] - F.rowptr[sn]), own);
      sn_bwd_diag<T>(F, L, smem, own, 1, v, sn);
    }
  s.sync();
  QTQP_TOC(kPhSnBwdSub);
}

}  // namespace qtqp
