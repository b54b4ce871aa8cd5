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
//  * factorisation, left-looking per supernode s (one block): for every
//    descendant d with rows in s's column range (the update list: d, the
//    first such row `off` of R_d and their number `cnt`), L_s[rows, cols] -=
//    L_d[off:, :] L_d[off:off+cnt, :]^T, scattered by the position of each
//    row of R_d in R_s; then the Cholesky of the diagonal block in shared
//    memory and the triangular solve of the rows below it.  The diagonal
//    keeps 1 / l_jj;
//  * solves: forward, per supernode, gathers the rows of L in its columns
//    from its update list, then solves with its diagonal block; backward
//    gathers x over R_s below the block, then solves with the transposed
//    block.  No atomics: every result has a single writer, so the results
//    are reproducible run to run.
// Order: each block first runs the subtrees the symbolic stage gave it (their
// supernodes in postorder, no grid barrier), then the supernodes above the
// subtrees run level by level with one grid barrier per level; the backward
// solve runs the same schedule in reverse.
#pragma once

#include "dense_ipm.cuh"

namespace qtqp {

constexpr int kSparseGridBlocks = 128;
constexpr int kSparseGridNT = kSparseGridBlocks * kGridBT;
constexpr int kSnMaxW = 64;             // widest supernode (the symbolic stage's cap)
constexpr int kSnLd = kSnMaxW + 1;      // leading dimension of the diagonal block in smem
constexpr int kSnStageK = 32;           // descendant columns staged per pass
constexpr int kSnCg = 8;                // target columns per thread in an update pass
// Dynamic shared memory of a block: the diagonal block, its reciprocal
// diagonal, the staged descendant rows, and the partial sums of the solves.
constexpr size_t kSparseSmemElems =
    size_t(kSnMaxW) * kSnLd + kSnMaxW + size_t(kSnMaxW) * (kSnStageK + 1) + kGridBT + kSnMaxW;
constexpr size_t kSparseSmem = kSparseSmemElems * sizeof(double);

// Device view of the symbolic plan (qtqp_sparse_desc offsets into the pools)
// and the factor's value storage.
struct SnFactor {
  int n, nsuper, top_levels;
  int64_t nvals, ngram;
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
  const int32_t* gcol;
  const int32_t* grow;
  const int64_t* rowptr;
  const int64_t* valptr;
  const int64_t* gpos;
  double* vals;
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

// Left-looking factorisation of supernode `sn` by the calling block.
template <typename T>
__device__ void sn_factor_one(const SnFactor& F, T* L, double* smem, int* info, int sn) {
  const int t = threadIdx.x;
  const int f = F.first[sn], w = F.first[sn + 1] - f;
  const int nr = int(F.rowptr[sn + 1] - F.rowptr[sn]);
  const int32_t* R = F.rows + F.rowptr[sn];
  T* Ls = L + F.valptr[sn];
  double* D = smem;                       // w x w (ld kSnLd)
  double* rdiag = D + kSnMaxW * kSnLd;    // 1 / l_jj
  double* C = rdiag + kSnMaxW;            // staged descendant rows (ld kSnStageK + 1)
  constexpr int ldc = kSnStageK + 1;
  // Updates from the descendants.
  for (int u = F.upd_ptr[sn]; u < F.upd_ptr[sn + 1]; ++u) {
    const int d = F.upd_src[u], off = F.upd_off[u], cnt = F.upd_cnt[u];
    const int wd = F.first[d + 1] - F.first[d];
    const int nrd = int(F.rowptr[d + 1] - F.rowptr[d]);
    const int32_t* Rd = F.rows + F.rowptr[d];
    const T* Ld = L + F.valptr[d];
    const int rem = nrd - off;
    const int ngrp = (cnt + kSnCg - 1) / kSnCg;
    for (int k0 = 0; k0 < wd; k0 += kSnStageK) {
      const int kc = min(kSnStageK, wd - k0);
      for (int idx = t; idx < cnt * kc; idx += blockDim.x) {
        const int c = idx % cnt, k = idx / cnt;
        C[c * ldc + k] = double(Ld[size_t(off + c) + size_t(k0 + k) * nrd]);
      }
      __syncthreads();
      for (int item = t; item < rem * ngrp; item += blockDim.x) {
        const int r = item % rem, cg = item / rem;
        const int row = off + r;
        double acc[kSnCg];
#pragma unroll
        for (int q = 0; q < kSnCg; ++q) acc[q] = 0.0;
        const int c0 = cg * kSnCg;
        for (int k = 0; k < kc; ++k) {
          const double a = double(Ld[size_t(row) + size_t(k0 + k) * nrd]);
#pragma unroll
          for (int q = 0; q < kSnCg; ++q)
            if (c0 + q < cnt) acc[q] = fma(a, C[(c0 + q) * ldc + k], acc[q]);
        }
        const int pos = sn_find(R, nr, Rd[row]);
#pragma unroll
        for (int q = 0; q < kSnCg; ++q) {
          const int c = c0 + q;
          if (c < cnt) {
            T* dst = Ls + size_t(pos) + size_t(Rd[off + c] - f) * nr;
            *dst = T(double(*dst) - acc[q]);
          }
        }
      }
      __syncthreads();
    }
  }
  // Cholesky of the diagonal block (left-looking by columns).
  for (int idx = t; idx < w * w; idx += blockDim.x) {
    const int c = idx / w, r = idx % w;
    if (r >= c) D[r * kSnLd + c] = double(Ls[size_t(r) + size_t(c) * nr]);
  }
  __syncthreads();
  for (int k = 0; k < w; ++k) {
    for (int i = k + t; i < w; i += blockDim.x) {
      double acc = D[i * kSnLd + k];
      for (int p = 0; p < k; ++p) acc = fma(-D[i * kSnLd + p], D[k * kSnLd + p], acc);
      D[i * kSnLd + k] = acc;
    }
    __syncthreads();
    const double dk = D[k * kSnLd + k];
    const double rk = dk > 0.0 ? 1.0 / sqrt(dk) : __longlong_as_double(0x7ff8000000000000ll);
    for (int i = k + 1 + t; i < w; i += blockDim.x) D[i * kSnLd + k] *= rk;
    if (t == 0) {
      rdiag[k] = rk;
      if (!(dk > 0.0)) atomicCAS(info, 0, f + k + 1);
    }
    __syncthreads();
  }
  for (int idx = t; idx < w * w; idx += blockDim.x) {
    const int c = idx / w, r = idx % w;
    if (r > c) Ls[size_t(r) + size_t(c) * nr] = T(D[r * kSnLd + c]);
    if (r == c) Ls[size_t(r) + size_t(c) * nr] = T(rdiag[c]);
  }
  // Rows below the block: x L_bb^T = a, forward substitution per row.
  for (int r = w + t; r < nr; r += blockDim.x) {
    for (int k = 0; k < w; ++k) {
      double acc = double(Ls[size_t(r) + size_t(k) * nr]);
      for (int p = 0; p < k; ++p)
        acc = fma(-double(Ls[size_t(r) + size_t(p) * nr]), D[k * kSnLd + p], acc);
      Ls[size_t(r) + size_t(k) * nr] = T(acc * rdiag[k]);
    }
  }
  __syncthreads();
}

// Forward solve of supernode `sn`: v[cols] -= L[cols, cols of descendants]
// y, then y_cols = L_bb^{-1} v[cols].
template <typename T>
__device__ void sn_fwd_one(const SnFactor& F, const T* L, double* smem, T* v, int sn) {
  const int t = threadIdx.x;
  const int f = F.first[sn], w = F.first[sn + 1] - f;
  const int nr = int(F.rowptr[sn + 1] - F.rowptr[sn]);
  const T* Ls = L + F.valptr[sn];
  double* part = smem + kSnMaxW * kSnLd + kSnMaxW + kSnMaxW * (kSnStageK + 1);
  double* yb = part + kGridBT;
  const int W32 = w <= 32 ? 32 : 64;
  const int G = blockDim.x / W32;
  const int j = t % W32, g = t / W32;
  double acc = 0.0;
  if (j < w) {
    for (int u = F.upd_ptr[sn] + g; u < F.upd_ptr[sn + 1]; u += G) {
      const int d = F.upd_src[u], off = F.upd_off[u], cnt = F.upd_cnt[u];
      const int fd = F.first[d], wd = F.first[d + 1] - fd;
      const int nrd = int(F.rowptr[d + 1] - F.rowptr[d]);
      const int32_t* Rd = F.rows + F.rowptr[d] + off;
      const int c = sn_find(Rd, cnt, f + j);
      if (c < cnt && Rd[c] == f + j) {
        const T* Ld = L + F.valptr[d] + off + c;
        for (int k = 0; k < wd; ++k)
          acc = fma(double(Ld[size_t(k) * nrd]), double(v[fd + k]), acc);
      }
    }
  }
  part[t] = acc;
  __syncthreads();
  if (t < w) {
    double b = double(v[f + t]);
    for (int q = 0; q < G; ++q) b -= part[q * W32 + t];
    yb[t] = b;
  }
  __syncthreads();
  if (t < 32) {  // one warp: lane l holds rows l and l + 32
    double r0 = t < w ? yb[t] : 0.0;
    double r1 = t + 32 < w ? yb[t + 32] : 0.0;
    for (int k = 0; k < w; ++k) {
      const double mine = k < 32 ? r0 : r1;
      const double yk = __shfl_sync(0xffffffffu, mine, k & 31) * double(Ls[size_t(k) * nr + k]);
      if (t == (k & 31)) {
        if (k < 32) {
          r0 = yk;
        } else {
          r1 = yk;
        }
      }
      if (t > k && t < w) r0 = fma(-double(Ls[size_t(t) + size_t(k) * nr]), yk, r0);
      if (t + 32 > k && t + 32 < w) r1 = fma(-double(Ls[size_t(t + 32) + size_t(k) * nr]), yk, r1);
    }
    if (t < w) v[f + t] = T(r0);
    if (t + 32 < w) v[f + t + 32] = T(r1);
  }
  __syncthreads();
}

// Backward solve of supernode `sn`: v[cols] -= L[below, cols]^T x[R below],
// then x_cols = L_bb^{-T} v[cols].
template <typename T>
__device__ void sn_bwd_one(const SnFactor& F, const T* L, double* smem, T* v, int sn) {
  const int t = threadIdx.x, lane = t & 31, warp = t >> 5, nwarp = blockDim.x >> 5;
  const int f = F.first[sn], w = F.first[sn + 1] - f;
  const int nr = int(F.rowptr[sn + 1] - F.rowptr[sn]);
  const int32_t* R = F.rows + F.rowptr[sn];
  const T* Ls = L + F.valptr[sn];
  double* yb = smem + kSnMaxW * kSnLd + kSnMaxW + kSnMaxW * (kSnStageK + 1) + kGridBT;
  for (int j = warp; j < w; j += nwarp) {
    double acc = 0.0;
    for (int r = w + lane; r < nr; r += 32)
      acc = fma(double(Ls[size_t(r) + size_t(j) * nr]), double(v[R[r]]), acc);
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
    if (lane == 0) yb[j] = double(v[f + j]) - acc;
  }
  __syncthreads();
  if (t < 32) {
    double r0 = t < w ? yb[t] : 0.0;
    double r1 = t + 32 < w ? yb[t + 32] : 0.0;
    for (int k = w - 1; k >= 0; --k) {
      const double mine = k < 32 ? r0 : r1;
      const double xk = __shfl_sync(0xffffffffu, mine, k & 31) * double(Ls[size_t(k) * nr + k]);
      if (t == (k & 31)) {
        if (k < 32) {
          r0 = xk;
        } else {
          r1 = xk;
        }
      }
      // rows j < k: v_j -= L[k][j] x_k
      if (t < k) r0 = fma(-double(Ls[size_t(k) + size_t(t) * nr]), xk, r0);
      if (t + 32 < k) r1 = fma(-double(Ls[size_t(k) + size_t(t + 32) * nr]), xk, r1);
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
  for (int l = 0; l < F.top_levels; ++l) {
    for (int q = F.top_ptr[l] + b; q < F.top_ptr[l + 1]; q += gridDim.x)
      sn_factor_one<T>(F, L, smem, s.linfo, F.top_list[q]);
    s.sync();
  }
  QTQP_TOC(kPhChol);
  return *reinterpret_cast<volatile int*>(s.linfo);
}

template <typename T, class S>
__device__ void sparse_solve(S& s, T* v, T* w) {
  (void)w;
  const SnFactor& F = *s.sn;
  const T* L = reinterpret_cast<const T*>(F.vals);
  double* smem = s.bwin;
  const int b = blockIdx.x;
  QTQP_TIC();
  for (int q = F.cta_ptr[b]; q < F.cta_ptr[b + 1]; ++q)
    for (int sn = F.cta_range[2 * q]; sn <= F.cta_range[2 * q + 1]; ++sn)
      sn_fwd_one<T>(F, L, smem, v, sn);
  s.sync();
  for (int l = 0; l < F.top_levels; ++l) {
    for (int q = F.top_ptr[l] + b; q < F.top_ptr[l + 1]; q += gridDim.x)
      sn_fwd_one<T>(F, L, smem, v, F.top_list[q]);
    s.sync();
  }
  for (int l = F.top_levels - 1; l >= 0; --l) {
    for (int q = F.top_ptr[l] + b; q < F.top_ptr[l + 1]; q += gridDim.x)
      sn_bwd_one<T>(F, L, smem, v, F.top_list[q]);
    s.sync();
  }
  for (int q = F.cta_ptr[b + 1] - 1; q >= F.cta_ptr[b]; --q)
    for (int sn = F.cta_range[2 * q + 1]; sn >= F.cta_range[2 * q]; --sn)
      sn_bwd_one<T>(F, L, smem, v, sn);
  s.sync();
  QTQP_TOC(kPhSolve);
}

}  // namespace qtqp
