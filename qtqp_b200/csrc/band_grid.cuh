// Banded backend in grid mode: one large banded QP (a long-horizon MPC
// problem, say) solved by the whole GPU.  The device IPM is the shared
// Ipm<NT, kFmtBand> run by a cooperative grid (NT > 1024: grid barriers and
// reductions); the Gram matrix, residuals and sparse products are spread
// over every thread of the grid, and the band Cholesky factorisation and its
// triangular solves are partitioned so that the grid's blocks work on them
// in parallel.
//
// Partitioned factorisation of the band matrix G (half-bandwidth bw), the
// Gram term of the regularised KKT system (src/qtqp/solvers_dense.py:99-116
// in band storage; the factorisation itself has no reference counterpart):
// the columns are split into P interiors I_k = [lo_k, lo_k + li_k), each but
// the last followed by a separator S_k of bw columns.  With li_k >= bw,
// interiors couple only to their neighbouring separators, so in the order
// (I_0 .. I_{P-1}, S_0 .. S_{P-2})
//   G = [G_II  G_IS; G_SI  G_SS],  G_II block diagonal,
//   L_II = chol(G_II) (one band Cholesky per interior, in parallel),
//   L_SI^T = L_II^{-1} G_IS: per interior the right spike W_R = the band
//     entries of L in the rows of S_k (the band factorisation writes them)
//     and the dense left spike W_L = L_{I_k}^{-1} G[I_k, S_{k-1}],
//   C = G_SS - L_SI L_SI^T: block tridiagonal over the separators,
//     D_k = G[S_k,S_k] - W_R^T W_R (of I_k) - W_L^T W_L (of I_{k+1}),
//     E_k = C[S_{k+1}, S_k] = -W_R^T W_L (both of I_{k+1}),
//   C^{-1} by block cyclic reduction over the separators (1-based j):
//     level l eliminates the j with lowest set bit 2^l, in parallel (one
//     block each): Di_j = D_j^{-1} by a symmetric sweep (in-place
//     Gauss-Jordan on the SPD block, one pivot per step), Yl_j = Di_j Cl_j
//     and Yr_j = Di_j Cr_j^T for the couplings Cl_j = C[j, j - 2^l], Cr_j =
//     C[j + 2^l, j]; then every surviving j' (multiple of 2^(l+1)) takes
//     D_j' -= Cr Yr (of its left neighbour) + Cl^T Yl (of its right
//     neighbour) and its new left coupling -Cr Yl of the left neighbour, in
//     parallel.
// Solve of G x = v: forward per interior (y = L_I^{-1} v_I, which also
// forms v_S - W_R^T y in the separator rows), t = v_S - W_L^T y, then the
// reduction levels forward (z_j = Di_j t_j, neighbours' t -= C z_j) and
// backward (x_j = z_j - Yl_j x_left - Yr_j x_right), then backward per
// interior with the separators' x known and the left spike's contribution
// removed first.
#pragma once

#include "dense_ipm.cuh"

namespace qtqp {

constexpr int kBandGridBlocks = 128;
constexpr int kBandGridNT = kBandGridBlocks * kGridBT;
// Dynamic shared memory available to one block of the grid solve.
constexpr size_t kBandGridSmemCap = 225 * 1024;

// bw x bw blocks kept per separator (row-major): D (Schur complement, lower),
// Q (W_L^T W_L of the next interior), E (coupling with the next separator
// from the interiors), C (left coupling created by the reduction), Di
// (inverse of D at elimination), Yl, Yr (reduced couplings) and R (the
// right coupling at elimination); and bw-vectors.
enum SepBlock : int { kSbD = 0, kSbQ, kSbE, kSbC, kSbI, kSbXl, kSbXr, kSbR, kSepBlocks };
enum SepVec : int { kSvCL = 0, kSvT, kSvZ, kSepVecs };

// The partition of the columns 0 .. n-1 into P interiors and P-1 separators.
struct BandParts {
  int P, bw, base, rem;
  __host__ __device__ BandParts(int n, int bw_, int P_) : P(P_), bw(bw_) {
    const int t = n - (P - 1) * bw;
    base = t / P;
    rem = t - base * P;
  }
  __host__ __device__ int lo(int k) const { return k * (base + bw) + (k < rem ? k : rem); }
  __host__ __device__ int li(int k) const { return base + (k < rem ? 1 : 0); }
  __host__ __device__ int lmax() const { return base + (rem > 0 ? 1 : 0); }
};

// The largest partition count that keeps every interior at least bw long.
__host__ __device__ inline int band_grid_max_parts(int n, int bw) {
  if (bw < 1) return 1;
  const int p = (n + bw) / (2 * bw);
  return p < 1 ? 1 : p;
}

// Pitch (elements) of a staged bw x bw separator block in shared memory
// (column-major, S(i, j) = buf[j * pitch + i]): odd, so that both rows and
// columns are read without bank conflicts.
__host__ __device__ inline int sep_pitch(int bw) { return bw | 1; }

// Dynamic shared memory of one block (sized for FP64): the largest of the
// band window (band_chol_window_range), the spike window, the products'
// staging, the separator reduction, and the solve rings; plus the
// per-thread Gram columns when they also fit.
__host__ __device__ inline size_t band_grid_smem_need(int bw) {
  const size_t e = sizeof(double);
  const size_t B = size_t(bw) + 2;
  size_t need = ((B * B * e + 7) & ~size_t(7)) + size_t(bw) * (bw + 1) / 2 * 4;
  if (band_panel_bytes(bw) > need) need = band_panel_bytes(bw);
  const size_t spike = (size_t(bw) + 1) * bw * e + 256 * e;
  const size_t prod = size_t(bw) * bw * e + 32 * 4 * ((size_t(bw) + 3) / 4) * e;
  const size_t chain = (2 * (size_t(bw) * sep_pitch(bw) + 4) + 3 * 128 + 256 + 2 * 16) * e;
  const size_t solve = (kBandSolveElems + 512) * e;
  if (spike > need) need = spike;
  if (prod > need) need = prod;
  if (chain > need) need = chain;
  if (solve > need) need = solve;
  return (need + 15) & ~size_t(15);
}
__host__ __device__ inline size_t band_grid_smem_bytes(int bw) {
  size_t need = band_grid_smem_need(bw);
  const size_t cols = size_t(kGridBT) * (size_t(bw) + 1) * sizeof(double);
  if (cols > need && cols <= kBandGridSmemCap) need = cols;
  return need;
}

// Global workspace of the grid solve: barrier / reduction state, the
// factorisation status, the banded instance's workspace, the left spikes
// (P x lmax x bw), the separator blocks ((P-1) x kSepBlocks x bw^2) and the
// separator vectors ((P-1) x kSepVecs x bw), all sized for FP64.
struct BandGridLayout {
  size_t ctl_off, info_off, band_off, wl_off, sep_off, vec_off, total;
};
__host__ __device__ inline size_t round256(size_t b) { return (b + 255) & ~size_t(255); }
__host__ __device__ inline BandGridLayout plan_band_grid_layout(int n, int m, int bw, int nnz_a,
                                                               int nnz_p, int P) {
  BandGridLayout L;
  const BandParts bp(n, bw, P);
  L.ctl_off = 0;
  L.info_off = round256(sizeof(GridCtl));
  L.band_off = L.info_off + 256;
  L.wl_off = round256(L.band_off + plan_band_layout(n, m, bw, nnz_a, nnz_p).total);
  L.sep_off = round256(L.wl_off + size_t(P) * bp.lmax() * bw * sizeof(double));
  L.vec_off = round256(L.sep_off + size_t(P - 1) * kSepBlocks * bw * bw * sizeof(double));
  L.total = round256(L.vec_off + size_t(P - 1) * kSepVecs * bw * sizeof(double));
  return L;
}

template <typename T, class S>
__device__ __forceinline__ T* part_wl(const S& s, const BandParts& bp, int k) {
  return reinterpret_cast<T*>(s.bp_wl) + size_t(k) * bp.lmax() * s.bw;
}
template <typename T, class S>
__device__ __forceinline__ T* sep_block(const S& s, int k, int which) {
  return reinterpret_cast<T*>(s.bp_sep) + (size_t(k) * kSepBlocks + which) * s.bw * s.bw;
}
template <typename T, class S>
__device__ __forceinline__ T* sep_vec(const S& s, int k, int which) {
  return reinterpret_cast<T*>(s.bp_vec) + (size_t(k) * kSepVecs + which) * s.bw;
}

template <typename T>
__device__ __forceinline__ T warp_sum(T v) {
#pragma unroll
  for (int off = 16; off > 0; off >>= 1) v += __shfl_xor_sync(0xffffffffu, v, off);
  return v;
}

// Row / column (a, b), a >= b, of lower-triangular tile u in row order.
__device__ __forceinline__ void tri_tile(int u, int& a, int& b) {
  int t = int((sqrtf(8.0f * u + 1.0f) - 1.0f) * 0.5f);
  while (t * (t + 1) / 2 > u) --t;
  while ((t + 1) * (t + 2) / 2 <= u) ++t;
  a = t;
  b = u - t * (t + 1) / 2;
}

// ---------------------------------------------------------------------------
// Left spike of interior k >= 1: W_L = L_I^{-1} G[I, S_{k-1}] (li x bw,
// row-major), by forward substitution through the interior's band factor.
// Rows p .. p+bw of the running spike live in a circular shared-memory
// window of bw+1 rows; G[I, S_{k-1}] is non-zero in the first bw rows only,
// so a row that enters the window (row p+bw at step p >= 1) starts at zero.
// One barrier per column; the factor column of the next step is staged
// while the current one is applied.
// ---------------------------------------------------------------------------
template <typename T, class S>
__device__ __noinline__ void bandp_spike(S& s, const BandParts& bp, int k) {
  const int bw = s.bw, ldl = bw + 1, B1 = bw + 1;
  const int lo = bp.lo(k), li = bp.li(k);
  const T* L = reinterpret_cast<const T*>(s.Lb);
  T* Ws = reinterpret_cast<T*>(s.bwin);
  T* lcol = Ws + size_t(B1) * bw;  // 2 x 128: factor columns p and p + 1
  T* WL = part_wl<T>(s, bp, k);
  const int lt = threadIdx.x;
  for (int e = lt; e < B1 * bw; e += kGridBT) {
    const int r = e / bw, c = e - r * bw;
    Ws[e] = (r <= c && r < li) ? L[size_t(lo - bw + c) * ldl + (r + bw - c)] : T(0);
  }
  if (lt <= bw) lcol[lt] = L[size_t(lo) * ldl + lt];
  __syncthreads();
  const int g = lt >> 7, c = lt & 127;
  for (int p = 0; p < li; ++p) {
    const T* lc = lcol + (p & 1) * 128;
    if (p + 1 < li && lt <= bw) lcol[((p + 1) & 1) * 128 + lt] = L[size_t(lo + p + 1) * ldl + lt];
    const int ps = p % B1;
    const int dmax = min(bw, li - 1 - p);
    if (c < bw) {
      const T x = Ws[ps * bw + c] * lc[0];
      if (g == 0) WL[size_t(p) * bw + c] = x;
      for (int d = 1 + g; d <= dmax; d += 2) {
        int rs = ps + d;
        if (rs >= B1) rs -= B1;
        T* cell = Ws + rs * bw + c;
        *cell = (d == bw && p >= 1) ? -lc[d] * x : fma(-lc[d], x, *cell);
      }
    }
    __syncthreads();
  }
}

// ---------------------------------------------------------------------------
// Products of interior k >= 1: Q = W_L^T W_L (the interior's share of the
// Schur complement of separator k-1, full bw x bw) and, when separator k
// exists, E_{k-1} = -W_R^T W_L with W_R^T[s][p] = L[hi + s][lo + p] (band
// entries, non-zero for p >= li + s - bw).  Q: 4 x 4 register tiles of the
// lower triangle over 32-row chunks of W_L staged in shared memory.
// ---------------------------------------------------------------------------
template <typename T, class S>
__device__ __noinline__ void bandp_products(S& s, const BandParts& bp, int k) {
  const int bw = s.bw, ldl = bw + 1;
  const int lo = bp.lo(k), li = bp.li(k);
  const T* WL = part_wl<T>(s, bp, k);
  const int lt = threadIdx.x;
  T* sm = reinterpret_cast<T*>(s.bwin);
  {
    const int nt4 = (bw + 3) / 4, ldc = 4 * nt4;
    const int ntiles = nt4 * (nt4 + 1) / 2;
    T* chunk = sm;
    T* Q = sep_block<T>(s, k - 1, kSbQ);
    for (int t0 = 0; t0 < ntiles; t0 += kGridBT) {
      const int u = t0 + lt;
      int ta = 0, tb = 0;
      if (u < ntiles) tri_tile(u, ta, tb);
      T acc[4][4];
#pragma unroll
      for (int i = 0; i < 4; ++i)
#pragma unroll
        for (int j = 0; j < 4; ++j) acc[i][j] = T(0);
      for (int p0 = 0; p0 < li; p0 += 32) {
        const int rows = min(32, li - p0);
        __syncthreads();
        for (int e = lt; e < 32 * ldc; e += kGridBT) {
          const int r = e / ldc, cc = e - r * ldc;
          chunk[e] = (r < rows && cc < bw) ? WL[size_t(p0 + r) * bw + cc] : T(0);
        }
        __syncthreads();
        if (u < ntiles) {
          for (int r = 0; r < rows; ++r) {
            const T* row = chunk + r * ldc;
            T a[4], b[4];
#pragma unroll
            for (int i = 0; i < 4; ++i) {
              a[i] = row[4 * ta + i];
              b[i] = row[4 * tb + i];
            }
#pragma unroll
            for (int i = 0; i < 4; ++i)
#pragma unroll
              for (int j = 0; j < 4; ++j) acc[i][j] = fma(a[i], b[j], acc[i][j]);
          }
        }
      }
      if (u < ntiles) {
#pragma unroll
        for (int i = 0; i < 4; ++i)
#pragma unroll
          for (int j = 0; j < 4; ++j) {
            const int a = 4 * ta + i, b = 4 * tb + j;
            if (a < bw && b < bw) {
              Q[size_t(a) * bw + b] = acc[i][j];
              Q[size_t(b) * bw + a] = acc[i][j];
            }
          }
      }
    }
  }
  if (k <= bp.P - 2) {
    __syncthreads();
    const T* L = reinterpret_cast<const T*>(s.Lb);
    T* wt = sm;  // the last bw rows of W_L
    const size_t r0 = size_t(li - bw) * bw;
    for (int e = lt; e < bw * bw; e += kGridBT) wt[e] = WL[r0 + e];
    __syncthreads();
    T* E = sep_block<T>(s, k - 1, kSbE);
    const int pb = lo + li - bw;  // first column of the interior's last bw
    for (int e = lt; e < bw * bw; e += kGridBT) {
      const int sr = e / bw, c = e - sr * bw;
      T acc = T(0);
      for (int q = sr; q < bw; ++q)
        acc = fma(L[size_t(pb + q) * ldl + (bw + sr - q)], wt[q * bw + c], acc);
      E[e] = -acc;
    }
  }
  __syncthreads();
}

// ---------------------------------------------------------------------------
// Staged separator blocks.  A row-major bw x bw block is staged in shared
// memory column-major with an odd pitch ldm: S(i, j) = buf[j * ldm + i]
// (trans: S(i, j) = src[j][i]), by asynchronous copies that are all in
// flight at once (one commit group); stage_wait ends the group for the
// whole block.
// ---------------------------------------------------------------------------
template <typename T>
__device__ void stage_async(T* buf, int ldm, const T* src, int bw, bool trans) {
  for (int e = threadIdx.x; e < bw * bw; e += kGridBT) {
    const int r = e / bw, c = e - r * bw;
    cp_async_elem(trans ? buf + r * ldm + c : buf + c * ldm + r, src + e, true);
  }
}
__device__ __forceinline__ void stage_wait() {
  cp_async_commit();
  cp_async_wait<0>();
  __syncthreads();
}
template <typename T>
__device__ void unstage(T* dst, const T* buf, int ldm, int bw) {
  for (int e = threadIdx.x; e < bw * bw; e += kGridBT) {
    const int r = e / bw, c = e - r * bw;
    dst[e] = buf[c * ldm + r];
  }
}

// The FP64 form of smem_gemm_nt on the FP64 tensor cores: each warp takes
// 16 x 16 blocks of the output (2 x 2 independent 8 x 8 accumulators),
// operands read straight from the staged blocks (zero beyond i1, j1, K).
template <class Fn>
__device__ __forceinline__ void smem_gemm_nt_dmma(const double* A, const double* B, int ldm, int K,
                                                  int i0, int i1, int j0, int j1, bool lower,
                                                  Fn fn) {
  if (i1 <= i0 || j1 <= j0) return;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int gi = lane >> 2, tg = lane & 3;
  const int ni = (i1 - i0 + 15) / 16, nj = (j1 - j0 + 15) / 16;
  for (int t = warp; t < ni * nj; t += kGridBT / 32) {
    const int ti = t % ni, tj = t / ni;
    const int ib = i0 + 16 * ti, jb = j0 + 16 * tj;
    if (lower && ib + 15 < jb) continue;  // above the diagonal
    double acc[2][2][2];
#pragma unroll
    for (int m = 0; m < 2; ++m)
#pragma unroll
      for (int n = 0; n < 2; ++n) acc[m][n][0] = acc[m][n][1] = 0.0;
    int ia[2], jc[2];
#pragma unroll
    for (int m = 0; m < 2; ++m) {
      ia[m] = ib + 8 * m + gi;
      jc[m] = jb + 8 * m + gi;
    }
#pragma unroll 2
    for (int c0 = 0; c0 < K; c0 += 4) {
      const int c = c0 + tg;
      double a[2], b[2];
#pragma unroll
      for (int m = 0; m < 2; ++m) {
        a[m] = (c < K && ia[m] < i1) ? A[c * ldm + ia[m]] : 0.0;
        b[m] = (c < K && jc[m] < j1) ? B[c * ldm + jc[m]] : 0.0;
      }
#pragma unroll
      for (int m = 0; m < 2; ++m)
#pragma unroll
        for (int n = 0; n < 2; ++n) dmma_8x8x4(acc[m][n], a[m], b[n]);
    }
#pragma unroll
    for (int m = 0; m < 2; ++m)
#pragma unroll
      for (int n = 0; n < 2; ++n)
#pragma unroll
        for (int e = 0; e < 2; ++e) {
          const int i = ia[m], j = jb + 8 * n + 2 * tg + e;
          if (i < i1 && j < j1 && (!lower || j <= i)) fn(i, j, acc[m][n][e]);
        }
  }
}

// acc(i, j) = sum_{c < K} A(i, c) B(j, c) for i in [i0, i1), j in [j0, j1)
// (lower: j <= i only), A and B staged column-major (pitch ldm); fn(i, j,
// acc) for each.  FP64: on the FP64 tensor cores (smem_gemm_nt_dmma).  4 x 4 register tiles: the tile's rows are strided across
// the lanes (consecutive lanes, consecutive rows: no bank conflicts with an
// odd pitch), its columns contiguous (the same for most of a warp).
template <typename T, class Fn>
__device__ __forceinline__ void smem_gemm_nt(const T* A, const T* B, int ldm, int K, int i0,
                                             int i1, int j0, int j1, bool lower, Fn fn) {
  if constexpr (sizeof(T) == 8) {
    smem_gemm_nt_dmma(A, B, ldm, K, i0, i1, j0, j1, lower, fn);
    return;
  }
  if (i1 <= i0 || j1 <= j0) return;
  const int ni = (i1 - i0 + 3) / 4, nj = (j1 - j0 + 3) / 4;
  for (int u = threadIdx.x; u < ni * nj; u += kGridBT) {
    const int tj = u / ni, ti = u - tj * ni;
    const int jb = j0 + 4 * tj;
    if (lower && min(i0 + ti + 3 * ni, i1 - 1) < jb) continue;  // above the diagonal
    int ia[4], jc[4];
#pragma unroll
    for (int q = 0; q < 4; ++q) {
      ia[q] = min(i0 + ti + ni * q, i1 - 1);
      jc[q] = min(jb + q, j1 - 1);
    }
    T acc[4][4];
#pragma unroll
    for (int p = 0; p < 4; ++p)
#pragma unroll
      for (int q = 0; q < 4; ++q) acc[p][q] = T(0);
#pragma unroll 2
    for (int c = 0; c < K; ++c) {
      const T* ac = A + c * ldm;
      const T* bc = B + c * ldm;
      T a[4], b[4];
#pragma unroll
      for (int q = 0; q < 4; ++q) {
        a[q] = ac[ia[q]];
        b[q] = bc[jc[q]];
      }
#pragma unroll
      for (int p = 0; p < 4; ++p)
#pragma unroll
        for (int q = 0; q < 4; ++q) acc[p][q] = fma(a[p], b[q], acc[p][q]);
    }
#pragma unroll
    for (int p = 0; p < 4; ++p) {
      const int i = i0 + ti + ni * p;
#pragma unroll
      for (int q = 0; q < 4; ++q) {
        const int j = jb + q;
        if (i < i1 && j < j1 && (!lower || j <= i)) fn(i, j, acc[p][q]);
      }
    }
  }
}

// Panel width of the blocked Cholesky of a separator block.
constexpr int kPanel = 16;

// Blocked Cholesky of the stacked [Mt; Mb] (Mt: bw x bw, lower; Mb: nb x bw
// rows below it), both staged column-major.  Each kPanel-column panel is
// factorised tall-skinny in registers: thread r holds the panel's entries of
// row r (top rows from the panel's diagonal down, then every bottom row); per
// column the diagonal block's rows publish their entries (double-buffered),
// one barrier, then every row scales its entry by one reciprocal square
// root of the pivot and updates the rest of its panel row.  The trailing
// columns then take a rank-kPanel update (tiled products).  Mt becomes L,
// Mb becomes Mb L^{-T}; needs bw - o + nb <= kGridBT rows per panel.
// pub: 2 x kPanel scratch.  Returns 0 or the 1-based column of a
// non-positive pivot (the same in every thread).
template <typename T>
__device__ __noinline__ int smem_chol_stacked(T* Mt, T* Mb, int nb, int bw, int ldm, T* pub) {
  const int lt = threadIdx.x;
  for (int o = 0; o < bw; o += kPanel) {
    const int pw = min(kPanel, bw - o);
    const int rows_top = bw - o;
    const bool own = lt < rows_top + nb;
    T* base = lt < rows_top ? Mt + o + lt : Mb + (lt - rows_top);
    T v[kPanel];
#pragma unroll
    for (int l = 0; l < kPanel; ++l) v[l] = (own && l < pw) ? base[(o + l) * ldm] : T(0);
    int bad = 0;
#pragma unroll
    for (int c = 0; c < kPanel; ++c) {
      if (c < pw) {
        T* pc = pub + (c & 1) * kPanel;
        if (lt >= c && lt < pw) pc[lt] = v[c];
        __syncthreads();
        const T piv = pc[c];
        if (!(piv > T(0))) {
          bad = c + 1;
          break;
        }
        const T il = rsqrt(piv);
        if (own) {
          if (lt == c) {
            v[c] = piv * il;
          } else if (lt > c) {
            const T lic = v[c] * il;
            v[c] = lic;
#pragma unroll
            for (int j = c + 1; j < kPanel; ++j)
              if (j < pw) v[j] = fma(-lic, pc[j] * il, v[j]);
          }
        }
      }
    }
    if (bad) return o + bad;
    if (own) {
#pragma unroll
      for (int l = 0; l < kPanel; ++l)
        if (l < pw) base[(o + l) * ldm] = v[l];
    }
    __syncthreads();
    const int t0 = o + pw;
    const T* Pt = Mt + o * ldm;
    smem_gemm_nt<T>(Pt, Pt, ldm, pw, t0, bw, t0, bw, true,
                    [&](int i, int j, T acc) { Mt[j * ldm + i] -= acc; });
    smem_gemm_nt<T>(Mb + o * ldm, Pt, ldm, pw, 0, nb, t0, bw, false,
                    [&](int i, int j, T acc) { Mb[j * ldm + i] -= acc; });
    __syncthreads();
  }
  return 0;
}

// Shared-memory layout of the reduction phases: two staged blocks, three
// vectors of 128, a 256-slot reduction scratch and the Cholesky panel's
// publish slots.
template <typename T>
struct CrSmem {
  T* Mt;
  T* Mb;
  T* vec;
  T* red;
  T* pub;
  __device__ CrSmem(double* base, int bw, int ldm) {
    Mt = reinterpret_cast<T*>(base);
    Mb = Mt + bw * ldm + 4;
    vec = Mb + bw * ldm + 4;
    red = vec + 3 * 128;
    pub = red + 256;
  }
};

// The start and end of separator k (k < P - 1): [hi_k, hi_k + bw).
__device__ __forceinline__ int sep_start(const BandParts& bp, int k) {
  return bp.lo(k) + bp.li(k);
}

// Reduction level l, eliminated separator j = 2^l (2 b + 1) (1-based;
// block b): the Cholesky of the stacked [D_j; I] gives L_j^{-T}, then Di_j =
// L_j^{-T} L_j^{-1}, Yl_j = Di_j Cl_j, Yr_j = Di_j Cr_j^T (tiled products),
// and a copy of Cr_j (its slot is rewritten at this level by j + 2^l).
template <typename T, class S>
__device__ __noinline__ int bandp_cr_eliminate(S& s, const BandParts& bp, int l, int j) {
  const int bw = s.bw, ldm = sep_pitch(bw), N = bp.P - 1, h = 1 << l, k = j - 1;
  CrSmem<T> sm(s.bwin, bw, ldm);
  QTQP_TIC();
  stage_async(sm.Mt, ldm, sep_block<T>(s, k, kSbD), bw, false);
  if (l == 0) stage_async(sm.Mb, ldm, sep_block<T>(s, k, kSbQ), bw, false);
  stage_wait();
  for (int e = threadIdx.x; e < bw * bw; e += kGridBT) {
    const int c = e / bw, i = e - c * bw;
    if (l == 0 && i >= c) sm.Mt[c * ldm + i] -= sm.Mb[c * ldm + i];
  }
  __syncthreads();
  for (int e = threadIdx.x; e < bw * bw; e += kGridBT) {
    const int c = e / bw, i = e - c * bw;
    sm.Mb[c * ldm + i] = i == c ? T(1) : T(0);
  }
  __syncthreads();
  QTQP_TOC(kPhBpCrStage);
  QTQP_RETIC();
  const int bad = smem_chol_stacked<T>(sm.Mt, sm.Mb, bw, bw, ldm, sm.pub);
  if (bad) return sep_start(bp, k) + bad;
  QTQP_TOC(kPhBpCrSweep);
  QTQP_RETIC();
  // Mb(i, c) = (L^{-T})(i, c); Di(i, jj) = sum_c Mb(i, c) Mb(jj, c) into Mt.
  T* Ig = sep_block<T>(s, k, kSbI);
  smem_gemm_nt<T>(sm.Mb, sm.Mb, ldm, bw, 0, bw, 0, bw, true, [&](int i, int jj, T acc) {
    sm.Mt[jj * ldm + i] = acc;
    sm.Mt[i * ldm + jj] = acc;
  });
  __syncthreads();
  unstage(Ig, sm.Mt, ldm, bw);
  for (int side = 0; side < 2; ++side) {
    const bool has = side == 0 ? j - h >= 1 : j + h <= N;
    if (!has) continue;
    // Staged so that Mb(jj, c) is column jj of Cl (side 0) or row jj of Cr.
    const T* src = side == 0 ? (l == 0 ? sep_block<T>(s, k - 1, kSbE) : sep_block<T>(s, k, kSbC))
                             : (l == 0 ? sep_block<T>(s, k, kSbE) : sep_block<T>(s, k + h, kSbC));
    __syncthreads();
    stage_async(sm.Mb, ldm, src, bw, side == 0);
    stage_wait();
    if (side == 1) unstage(sep_block<T>(s, k, kSbR), sm.Mb, ldm, bw);
    T* Y = sep_block<T>(s, k, side == 0 ? kSbXl : kSbXr);
    smem_gemm_nt<T>(sm.Mt, sm.Mb, ldm, bw, 0, bw, 0, bw, false,
                    [&](int i, int jj, T acc) { Y[size_t(i) * bw + jj] = acc; });
  }
  __syncthreads();
  QTQP_TOC(kPhBpCrGemm);
  return 0;
}

// Reduction level l, surviving separator j' = 2^(l+1) (b + 1) (block b):
// D_j' -= Cr Yr of the left neighbour jl = j' - 2^l (and Q at level 0),
// its new left coupling -Cr Yl of jl, and D_j' -= Cl^T Yl of the right
// neighbour jr = j' + 2^l.  D (lower, row-major) is updated in place.
template <typename T, class S>
__device__ __noinline__ void bandp_cr_gather(S& s, const BandParts& bp, int l, int jp) {
  const int bw = s.bw, ldm = sep_pitch(bw), N = bp.P - 1, h = 1 << l, k = jp - 1;
  CrSmem<T> sm(s.bwin, bw, ldm);
  QTQP_TIC();
  const int kl = jp - h - 1;
  T* D = sep_block<T>(s, k, kSbD);
  const T* Q = sep_block<T>(s, k, kSbQ);
  stage_async(sm.Mt, ldm, sep_block<T>(s, kl, kSbR), bw, false);
  stage_async(sm.Mb, ldm, sep_block<T>(s, kl, kSbXr), bw, true);
  stage_wait();
  smem_gemm_nt<T>(sm.Mt, sm.Mb, ldm, bw, 0, bw, 0, bw, true, [&](int i, int jj, T acc) {
    const size_t e = size_t(i) * bw + jj;
    D[e] -= l == 0 ? acc + Q[e] : acc;
  });
  __syncthreads();
  if (jp - 2 * h >= 1) {
    stage_async(sm.Mb, ldm, sep_block<T>(s, kl, kSbXl), bw, true);
    stage_wait();
    T* Cn = sep_block<T>(s, k, kSbC);
    smem_gemm_nt<T>(sm.Mt, sm.Mb, ldm, bw, 0, bw, 0, bw, false,
                    [&](int i, int jj, T acc) { Cn[size_t(i) * bw + jj] = -acc; });
    __syncthreads();
  }
  if (jp + h <= N) {
    const int kr = jp + h - 1;
    stage_async(sm.Mt, ldm, l == 0 ? sep_block<T>(s, k, kSbE) : sep_block<T>(s, kr, kSbC), bw,
                true);
    stage_async(sm.Mb, ldm, sep_block<T>(s, kr, kSbXl), bw, true);
    stage_wait();
    smem_gemm_nt<T>(sm.Mt, sm.Mb, ldm, bw, 0, bw, 0, bw, true,
                    [&](int i, int jj, T acc) { D[size_t(i) * bw + jj] -= acc; });
    __syncthreads();
  }
  QTQP_TOC(kPhBpCrGather);
}

// ---------------------------------------------------------------------------
// The partitioned factorisation (grid mode).  Every block of the grid takes
// part in the Gram matrix; block k < P eliminates interior k (and forms its
// spike products); the separators are reduced level by level.  Returns the
// same value in every thread: 0 or the 1-based column of a non-positive
// pivot.
// ---------------------------------------------------------------------------
template <typename T, class S>
__device__ int bandp_factorize(S& s) {
  QTQP_TIC();
  const int bw = s.bw;
  const BandParts bp(s.n, bw, s.nparts);
  volatile int* info = s.linfo;
  if (s.tid == 0) *info = 0;
  const bool smem_cols = size_t(kGridBT) * (size_t(bw) + 1) * sizeof(T) <= s.bwin_bytes;
  s.template band_gram<T>(smem_cols ? reinterpret_cast<T*>(s.bwin) + size_t(threadIdx.x) * (bw + 1)
                                    : nullptr);
  QTQP_TOC(kPhGram);
  QTQP_RETIC();
  const int k = blockIdx.x;
  if (k < bp.P) {
    const int lo = bp.lo(k), li = bp.li(k);
    const bool has_sep = k < bp.P - 1;
    const int bad = s.template band_chol_panel_range<T, kGridBT>(
        threadIdx.x, lo, li + (has_sep ? bw : 0), li,
        has_sep ? sep_block<T>(s, k, kSbD) : static_cast<T*>(nullptr), bw);
    if (bad != 0) {
      if (threadIdx.x == 0) atomicMax(const_cast<int*>(info), bad);
    } else if (k >= 1) {
      __syncthreads();
      bandp_spike<T>(s, bp, k);
      bandp_products<T>(s, bp, k);
    }
  }
  s.sync();
  QTQP_TOC(kPhBpInterior);
  QTQP_RETIC();
  const int N = bp.P - 1;
  for (int l = 0; (1 << l) <= N; ++l) {
    const int h = 1 << l;
    const int j = h * (2 * k + 1);
    // Another block may record a failure during this phase: the block
    // agrees on one reading of the status before it branches.
    const bool ok = __syncthreads_and(*info == 0) != 0;
    if (j <= N && ok) {
      const int bad = bandp_cr_eliminate<T>(s, bp, l, j);
      if (bad != 0 && threadIdx.x == 0) atomicMax(const_cast<int*>(info), bad);
    }
    s.sync();
    const int jp = 2 * h * (k + 1);
    if (jp <= N && *info == 0) bandp_cr_gather<T>(s, bp, l, jp);
    s.sync();
  }
  QTQP_TOC(kPhBpChain);
  return *info;
}

// Row / column matrix-vector products with a staged block, two halves of
// the block over the inner index, combined through red (256 slots):
// rows: y[i] = sum_c S(i, c) x[c]; cols: y[c] = sum_i S(i, c) x[i].
// Thread i (< bw) receives y[i].
template <typename T>
__device__ __forceinline__ T smem_matvec(const T* S, int ldm, int bw, const T* x, bool cols,
                                         T* red) {
  const int i = threadIdx.x & 127, half = threadIdx.x >> 7;
  T acc = T(0);
  if (i < bw) {
    if (cols) {
      for (int c = half; c < bw; c += 2) acc = fma(S[i * ldm + c], x[c], acc);
    } else {
      for (int c = half; c < bw; c += 2) acc = fma(S[c * ldm + i], x[c], acc);
    }
  }
  red[threadIdx.x] = acc;
  __syncthreads();
  const T y = threadIdx.x < 128 ? red[threadIdx.x] + red[threadIdx.x + 128] : T(0);
  __syncthreads();
  return y;
}

// ---------------------------------------------------------------------------
// The partitioned solve G x = v (grid mode), x into v; w is scratch of n
// entries.  Every thread of the grid calls it.
// ---------------------------------------------------------------------------
template <typename T, class S>
__device__ void bandp_solve(S& s, T* v, T* w) {
  const int bw = s.bw, ldm = sep_pitch(bw);
  const BandParts bp(s.n, bw, s.nparts);
  const int P = bp.P, N = P - 1, k = blockIdx.x, lt = threadIdx.x, lane = lt & 31,
            warp = lt >> 5;
  constexpr int kNW = kGridBT / 32;
  // Scratch after the blocked band solves' window and staging.
  T* scr = reinterpret_cast<T*>(s.bwin) + kBandSolveElems;
  QTQP_TIC();
  // Forward per interior; the spike term W_L^T y of interior k for
  // separator k - 1.
  if (k < P) {
    const int lo = bp.lo(k), li = bp.li(k), hi = lo + li, R = hi + (k < P - 1 ? bw : 0);
    s.template band_fwd_blocked<T, kGridBT>(v, w, lo, li, R, lt);
    if (k >= 1) {
      const T* WL = part_wl<T>(s, bp, k);
      const int c = lt & 127, g = lt >> 7;
      T acc = T(0);
      if (c < bw)
        for (int p = g; p < li; p += 2) acc = fma(WL[size_t(p) * bw + c], w[lo + p], acc);
      scr[lt] = acc;
      __syncthreads();
      if (lt < bw) sep_vec<T>(s, k - 1, kSvCL)[lt] = scr[lt] + scr[lt + 128];
    }
  }
  s.sync();
  QTQP_TOC(kPhBpFwd);
  QTQP_RETIC();
  CrSmem<T> sm(s.bwin, bw, ldm);
  T* t = sm.vec;
  T* xa = sm.vec + 128;
  T* xb = sm.vec + 256;
  T* red = sm.red;
  // t_j at level 0 is v[S] - W_L^T y; later levels keep it in kSvT.
  auto load_t = [&](int l, int kk) {
    if (lt < bw)
      t[lt] = l == 0 ? v[sep_start(bp, kk) + lt] - sep_vec<T>(s, kk, kSvCL)[lt]
                     : sep_vec<T>(s, kk, kSvT)[lt];
  };
  int levels = 0;
  while ((1 << levels) <= N) ++levels;
  // Level 0: z_j = Di_j t_j for the separators eliminated first.  Every
  // separator eliminated at level l + 1 is a survivor of level l, so its
  // block forms z right after updating t (one grid barrier per level).
  auto form_z = [&](int kk) {  // t (shared) -> z_kk
    stage_async(sm.Mt, ldm, sep_block<T>(s, kk, kSbI), bw, false);
    stage_wait();
    const T z = smem_matvec(sm.Mt, ldm, bw, t, false, red);
    if (lt < bw) sep_vec<T>(s, kk, kSvZ)[lt] = z;
  };
  if (N >= 1 && 2 * k + 1 <= N) {
    load_t(0, 2 * k);
    form_z(2 * k);
  }
  s.sync();
  for (int l = 0; l < levels; ++l) {
    const int h = 1 << l;
    const int jp = 2 * h * (k + 1);
    if (jp <= N) {  // t_j' -= Cr z (left neighbour) + Cl^T z (right neighbour)
      load_t(l, jp - 1);
      const int kl = jp - h - 1, kr = jp + h - 1;
      if (lt < bw) xa[lt] = sep_vec<T>(s, kl, kSvZ)[lt];
      stage_async(sm.Mt, ldm, sep_block<T>(s, kl, kSbR), bw, false);
      stage_wait();
      T acc = smem_matvec(sm.Mt, ldm, bw, xa, false, red);
      if (jp + h <= N) {
        if (lt < bw) xb[lt] = sep_vec<T>(s, kr, kSvZ)[lt];
        stage_async(sm.Mt, ldm, l == 0 ? sep_block<T>(s, jp - 1, kSbE) : sep_block<T>(s, kr, kSbC),
                    bw, false);
        stage_wait();
        acc += smem_matvec(sm.Mt, ldm, bw, xb, true, red);
      }
      const T tv = lt < bw ? t[lt] - acc : T(0);
      if ((jp & (4 * h - 1)) == 2 * h) {  // eliminated at level l + 1
        __syncthreads();                    // every thread has read t
        if (lt < bw) t[lt] = tv;
        form_z(jp - 1);                     // stage_wait orders t before the product
      } else if (lt < bw) {
        sep_vec<T>(s, jp - 1, kSvT)[lt] = tv;
      }
    }
    s.sync();
  }
  for (int l = levels - 1; l >= 0; --l) {
    const int h = 1 << l;
    const int j = h * (2 * k + 1);
    if (j <= N) {  // x_j = z_j - Yl_j x_left - Yr_j x_right
      const int kk = j - 1;
      T r = lt < bw ? sep_vec<T>(s, kk, kSvZ)[lt] : T(0);
      if (j - h >= 1) {
        if (lt < bw) xa[lt] = v[sep_start(bp, j - h - 1) + lt];
        stage_async(sm.Mt, ldm, sep_block<T>(s, kk, kSbXl), bw, false);
        stage_wait();
        r -= smem_matvec(sm.Mt, ldm, bw, xa, false, red);
      }
      if (j + h <= N) {
        if (lt < bw) xb[lt] = v[sep_start(bp, j + h - 1) + lt];
        stage_async(sm.Mt, ldm, sep_block<T>(s, kk, kSbXr), bw, false);
        stage_wait();
        r -= smem_matvec(sm.Mt, ldm, bw, xb, false, red);
      }
      if (lt < bw) v[sep_start(bp, kk) + lt] = r;
    }
    s.sync();
  }
  QTQP_TOC(kPhBpChains);
  QTQP_RETIC();
  // Backward per interior after removing W_L x_{S_{k-1}}.
  if (k < P) {
    const int lo = bp.lo(k), li = bp.li(k), hi = lo + li, R = hi + (k < P - 1 ? bw : 0);
    if (k >= 1) {
      const T* WL = part_wl<T>(s, bp, k);
      if (lt < bw) scr[lt] = v[lo - bw + lt];
      __syncthreads();
      for (int p = warp; p < li; p += kNW) {
        T acc = T(0);
        for (int c = lane; c < bw; c += 32) acc = fma(WL[size_t(p) * bw + c], scr[c], acc);
        acc = warp_sum(acc);
        if (lane == 0) w[lo + p] -= acc;
      }
      __syncthreads();
    }
    s.template band_bwd_blocked<T, kGridBT>(v, w, lo, hi, R, lt);
  }
  s.sync();
  QTQP_TOC(kPhBpBwd);
}

}  // namespace qtqp
