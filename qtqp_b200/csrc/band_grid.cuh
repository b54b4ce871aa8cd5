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
//   chol(C): one block's chain over the separators, Lc_k = chol(D_k -
//     F_{k-1} F_{k-1}^T), F_k = E_k Lc_k^{-T} (the panel below Lc_k in one
//     Cholesky of the stacked [D_k; E_k]),
//   then, in parallel per separator, Li_k = Lc_k^{-1}, G_k = Li_k F_{k-1}
//     and H_k = (F_k Li_k)^T, so that the two chains of a solve are one
//     bw x bw product per separator each.
// Solve of G x = v: forward per interior (y = L_I^{-1} v_I, which also
// forms v_S - W_R^T y in the separator rows), t_k = v_S - W_L^T y,
// u_k = Li_k t_k, z_k = u_k - G_k z_{k-1} (chain), v_k = Li_k^T z_k,
// x_k = v_k - H_k x_{k+1} (chain), then backward per interior with the
// separators' x known and the left spike's contribution removed first.
#pragma once

#include "dense_ipm.cuh"

namespace qtqp {

constexpr int kBandGridBlocks = 128;
constexpr int kBandGridNT = kBandGridBlocks * kGridBT;
// Dynamic shared memory available to one block of the grid solve.
constexpr size_t kBandGridSmemCap = 225 * 1024;

// bw x bw blocks kept per separator and bw-vectors per separator.
enum SepBlock : int { kSbD = 0, kSbQ, kSbE, kSbL, kSbF, kSbI, kSbG, kSbH, kSepBlocks };
enum SepVec : int { kSvCL = 0, kSvU, kSvZ, kSvV, kSepVecs };

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

// Pitch (elements) of a staged bw x bw separator block in shared memory.
__host__ __device__ inline int sep_pitch(int bw) { return bw + 1; }

// Dynamic shared memory of one block (sized for FP64): the largest of the
// band window (band_chol_window_range), the spike window, the products'
// staging, the separator chain and inverse, and the solve rings; plus the
// per-thread Gram columns when they also fit.
__host__ __device__ inline size_t band_grid_smem_need(int bw) {
  const size_t e = sizeof(double);
  const size_t B = size_t(bw) + 2;
  size_t need = ((B * B * e + 7) & ~size_t(7)) + size_t(bw) * (bw + 1) / 2 * 4;
  const size_t spike = (size_t(bw) + 1) * bw * e + 256 * e;
  const size_t prod = size_t(bw) * bw * e + 32 * 4 * ((size_t(bw) + 3) / 4) * e;
  const size_t chain = 2 * size_t(bw) * sep_pitch(bw) * e + 32 * 33 * e + 64;
  const size_t solve = (128 + kBandRing * 128 + kBandRing) * e + 512 * e;
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
__device__ void bandp_spike(S& s, const BandParts& bp, int k) {
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
__device__ void bandp_products(S& s, const BandParts& bp, int k) {
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
// One warp factors the pw x pw (pw <= 32) diagonal block at M[o][o] (pitch
// ldm) in place, rows and columns beyond pw taken as the identity, and
// writes the inverse of the factor to inv32 (32 x 33).  Crout order: lane
// r holds row r; one reciprocal square root per pivot.  Returns 0 or the
// 1-based column of a non-positive pivot.
// ---------------------------------------------------------------------------
template <typename T>
__device__ __noinline__ int warp_chol_panel(T* M, int ldm, int o, int pw, T* inv32, int lane) {
  const bool live = lane < pw;
  T* Lr = M + size_t(o + (live ? lane : 0)) * ldm + o;
  T idg[32];
  int bad = 0;
  {
    T a[32];
#pragma unroll
    for (int j = 0; j < 32; ++j) a[j] = (live && j <= lane) ? Lr[j] : (j == lane ? T(1) : T(0));
#pragma unroll
    for (int c = 0; c < 32; ++c) {
      T sr = a[c];
      if (c < pw) {
        const T* Lc = M + size_t(o + c) * ldm + o;
        T s0 = a[c], s1 = T(0);
#pragma unroll
        for (int q = 0; q < c; ++q) {
          if (q & 1) {
            s1 = fma(-a[q], Lc[q], s1);
          } else {
            s0 = fma(-a[q], Lc[q], s0);
          }
        }
        sr = s0 + s1;
      }
      const T piv = __shfl_sync(0xffffffffu, sr, c);
      if (c < pw && !(piv > T(0)) && bad == 0) bad = c + 1;
      const T il = c < pw ? rsqrt(piv) : T(1);
      idg[c] = il;
      if (lane == c) {
        a[c] = piv * il;
      } else if (lane > c) {
        a[c] = sr * il;
      }
      if (live && lane >= c && c < pw) Lr[c] = a[c];
      __syncwarp();
    }
  }
  if (bad) return bad;
  T x[32];
#pragma unroll
  for (int r = 0; r < 32; ++r) {
    if (r < pw) {
      const T* Lrow = M + size_t(o + r) * ldm + o;
      T a0 = T(0), a1 = T(0);
#pragma unroll
      for (int q = 0; q < r; ++q) {
        if (q >= lane) {
          if (q & 1) {
            a1 = fma(Lrow[q], x[q], a1);
          } else {
            a0 = fma(Lrow[q], x[q], a0);
          }
        }
      }
      x[r] = r < lane ? T(0) : (r == lane ? idg[r] : -(a0 + a1) * idg[r]);
    } else {
      x[r] = r == lane ? T(1) : T(0);
    }
  }
#pragma unroll
  for (int r = 0; r < 32; ++r) inv32[r * 33 + lane] = x[r];
  return 0;
}

// ---------------------------------------------------------------------------
// The separator chain (one block): for k = 0 .. P-2, D_k = Dp_k - Q_k -
// F_{k-1} F_{k-1}^T, then the blocked Cholesky of the stacked [D_k; E_k]
// (32-column panels: warp_chol_panel on the diagonal block, the rows below
// times its inverse, a rank-32 update of the trailing columns in 4 x 4
// register tiles) gives Lc_k (top, lower, l_cc on the diagonal) and F_k
// (bottom).  F_k stays in shared memory for the next separator.
// Returns 0 or the 1-based global column of a non-positive pivot.
// ---------------------------------------------------------------------------
template <typename T, class S>
__device__ int bandp_chain(S& s, const BandParts& bp) {
  const int bw = s.bw, ldm = sep_pitch(bw);
  const int lt = threadIdx.x, warp = lt >> 5, lane = lt & 31;
  T* Mt = reinterpret_cast<T*>(s.bwin);
  T* Mb = Mt + size_t(bw) * ldm;
  T* inv32 = Mb + size_t(bw) * ldm;
  int* flag = reinterpret_cast<int*>(inv32 + 32 * 33);
  const int nt4 = (bw + 3) / 4;
  for (int k = 0; k < bp.P - 1; ++k) {
    const T* Dg = sep_block<T>(s, k, kSbD);
    const T* Qg = sep_block<T>(s, k, kSbQ);
    // 1. Top block (lower triangle).
    if (k == 0) {
      for (int e = lt; e < bw * bw; e += kGridBT) {
        const int i = e / bw, j = e - i * bw;
        if (j <= i) Mt[i * ldm + j] = Dg[e] - Qg[e];
      }
    } else {
      const int ntiles = nt4 * (nt4 + 1) / 2;
      for (int u = lt; u < ntiles; u += kGridBT) {
        int ta, tb;
        tri_tile(u, ta, tb);
        T acc[4][4];
#pragma unroll
        for (int i = 0; i < 4; ++i)
#pragma unroll
          for (int j = 0; j < 4; ++j) acc[i][j] = T(0);
        int ra[4], rb[4];
#pragma unroll
        for (int i = 0; i < 4; ++i) {
          ra[i] = min(4 * ta + i, bw - 1) * ldm;
          rb[i] = min(4 * tb + i, bw - 1) * ldm;
        }
        for (int c = 0; c < bw; ++c) {
          T a[4], b[4];
#pragma unroll
          for (int i = 0; i < 4; ++i) {
            a[i] = Mb[ra[i] + c];
            b[i] = Mb[rb[i] + c];
          }
#pragma unroll
          for (int i = 0; i < 4; ++i)
#pragma unroll
            for (int j = 0; j < 4; ++j) acc[i][j] = fma(a[i], b[j], acc[i][j]);
        }
#pragma unroll
        for (int i = 0; i < 4; ++i)
#pragma unroll
          for (int j = 0; j < 4; ++j) {
            const int a = 4 * ta + i, b = 4 * tb + j;
            if (a < bw && b <= a)
              Mt[a * ldm + b] = Dg[size_t(a) * bw + b] - Qg[size_t(a) * bw + b] - acc[i][j];
          }
      }
    }
    __syncthreads();
    // 2. Bottom block E_k.
    const bool has_e = k < bp.P - 2;
    const int nb = has_e ? bw : 0;
    if (has_e) {
      const T* Eg = sep_block<T>(s, k, kSbE);
      for (int e = lt; e < bw * bw; e += kGridBT) {
        const int i = e / bw, j = e - i * bw;
        Mb[i * ldm + j] = Eg[e];
      }
    }
    __syncthreads();
    // 3. Blocked Cholesky of [Mt; Mb].
    for (int o = 0; o < bw; o += 32) {
      const int pw = min(32, bw - o);
      if (warp == 0) {
        const int bad = warp_chol_panel<T>(Mt, ldm, o, pw, inv32, lane);
        if (lane == 0) *flag = bad ? o + bad : 0;
      }
      __syncthreads();
      const int bad = *flag;
      if (bad) return bp.lo(k) + bp.li(k) + bad;
      // Rows below the diagonal block: row <- row inv^T (thread per row).
      const int rows_top = bw - o - pw;
      for (int r = lt; r < rows_top + nb; r += kGridBT) {
        T* row = r < rows_top ? Mt + (o + pw + r) * ldm + o : Mb + (r - rows_top) * ldm + o;
        T v[32];
#pragma unroll
        for (int l = 0; l < 32; ++l) v[l] = l < pw ? row[l] : T(0);
#pragma unroll
        for (int j = 0; j < 32; ++j) {
          if (j < pw) {
            T acc = T(0);
#pragma unroll
            for (int l = 0; l <= j; ++l) acc = fma(v[l], inv32[j * 33 + l], acc);
            row[j] = acc;
          }
        }
      }
      __syncthreads();
      // Trailing columns [t0, bw): top rows i >= j, all bottom rows.
      const int t0 = o + pw;
      if (t0 < bw) {
        const int nt = (bw - t0 + 3) / 4;
        const int ntop = nt * (nt + 1) / 2;
        const int nbot = ((nb + 3) / 4) * nt;
        for (int u = lt; u < ntop + nbot; u += kGridBT) {
          int i0, j0, lim;
          T* base;
          if (u < ntop) {
            int ta, tb;
            tri_tile(u, ta, tb);
            i0 = t0 + 4 * ta;
            j0 = t0 + 4 * tb;
            base = Mt;
            lim = bw;
          } else {
            const int v = u - ntop;
            const int ta = v / nt, tb = v - ta * nt;
            i0 = 4 * ta;
            j0 = t0 + 4 * tb;
            base = Mb;
            lim = nb;
          }
          T acc[4][4];
#pragma unroll
          for (int i = 0; i < 4; ++i)
#pragma unroll
            for (int j = 0; j < 4; ++j) acc[i][j] = T(0);
          int ra[4], rb[4];
#pragma unroll
          for (int i = 0; i < 4; ++i) {
            ra[i] = min(i0 + i, lim - 1) * ldm + o;
            rb[i] = min(j0 + i, bw - 1) * ldm + o;
          }
          for (int l = 0; l < pw; ++l) {
            T a[4], b[4];
#pragma unroll
            for (int i = 0; i < 4; ++i) {
              a[i] = base[ra[i] + l];
              b[i] = Mt[rb[i] + l];
            }
#pragma unroll
            for (int i = 0; i < 4; ++i)
#pragma unroll
              for (int j = 0; j < 4; ++j) acc[i][j] = fma(a[i], b[j], acc[i][j]);
          }
#pragma unroll
          for (int i = 0; i < 4; ++i)
#pragma unroll
            for (int j = 0; j < 4; ++j) {
              const int a = i0 + i, b = j0 + j;
              const bool ok = u < ntop ? (a < bw && b <= a) : (a < nb && b < bw);
              if (ok) base[a * ldm + b] -= acc[i][j];
            }
        }
      }
      __syncthreads();
    }
    // 4. Lc_k and F_k to global memory.
    T* Lg = sep_block<T>(s, k, kSbL);
    T* Fg = sep_block<T>(s, k, kSbF);
    for (int e = lt; e < bw * bw; e += kGridBT) {
      const int i = e / bw, j = e - i * bw;
      Lg[e] = j <= i ? Mt[i * ldm + j] : T(0);
      if (has_e) Fg[e] = Mb[i * ldm + j];
    }
    __syncthreads();
  }
  return 0;
}

// ---------------------------------------------------------------------------
// Per separator k (one block): Li_k = Lc_k^{-1} (thread per column), then
// G_k = Li_k F_{k-1} (k >= 1) and H_k = (F_k Li_k)^T (k <= P-3).
// ---------------------------------------------------------------------------
template <typename T, class S>
__device__ void bandp_sep_inverse(S& s, const BandParts& bp, int k) {
  const int bw = s.bw, ldm = sep_pitch(bw);
  const int lt = threadIdx.x;
  T* Ls = reinterpret_cast<T*>(s.bwin);
  T* X = Ls + size_t(bw) * ldm;
  T* idg = X + size_t(bw) * ldm;
  const T* Lg = sep_block<T>(s, k, kSbL);
  for (int e = lt; e < bw * bw; e += kGridBT) {
    const int i = e / bw, j = e - i * bw;
    Ls[i * ldm + j] = Lg[e];
  }
  __syncthreads();
  if (lt < bw) idg[lt] = T(1) / Ls[lt * ldm + lt];
  __syncthreads();
  if (lt < bw) {
    const int t = lt;
    for (int r = 0; r < t; ++r) X[r * ldm + t] = T(0);
    X[t * ldm + t] = idg[t];
    for (int r = t + 1; r < bw; ++r) {
      T a0 = T(0), a1 = T(0);
      int c = t;
      for (; c + 1 < r; c += 2) {
        a0 = fma(Ls[r * ldm + c], X[c * ldm + t], a0);
        a1 = fma(Ls[r * ldm + c + 1], X[(c + 1) * ldm + t], a1);
      }
      if (c < r) a0 = fma(Ls[r * ldm + c], X[c * ldm + t], a0);
      X[r * ldm + t] = -(a0 + a1) * idg[r];
    }
  }
  __syncthreads();
  T* Ig = sep_block<T>(s, k, kSbI);
  for (int e = lt; e < bw * bw; e += kGridBT) {
    const int i = e / bw, j = e - i * bw;
    Ig[e] = X[i * ldm + j];
  }
  if (k >= 1) {  // G_k = Li_k F_{k-1}: G[a][b] = sum_{c <= a} X[a][c] F[c][b]
    const T* Fg = sep_block<T>(s, k - 1, kSbF);
    __syncthreads();
    for (int e = lt; e < bw * bw; e += kGridBT) {
      const int i = e / bw, j = e - i * bw;
      Ls[i * ldm + j] = Fg[e];
    }
    __syncthreads();
    T* Gg = sep_block<T>(s, k, kSbG);
    for (int e = lt; e < bw * bw; e += kGridBT) {
      const int a = e / bw, b = e - a * bw;
      T acc = T(0);
      for (int c = 0; c <= a; ++c) acc = fma(X[a * ldm + c], Ls[c * ldm + b], acc);
      Gg[e] = acc;
    }
  }
  if (k <= bp.P - 3) {  // H_k = (F_k Li_k)^T: H[a][b] = sum_{c >= a} F[b][c] X[c][a]
    const T* Fg = sep_block<T>(s, k, kSbF);
    __syncthreads();
    for (int e = lt; e < bw * bw; e += kGridBT) {
      const int i = e / bw, j = e - i * bw;
      Ls[i * ldm + j] = Fg[e];
    }
    __syncthreads();
    T* Hg = sep_block<T>(s, k, kSbH);
    for (int e = lt; e < bw * bw; e += kGridBT) {
      const int a = e / bw, b = e - a * bw;
      T acc = T(0);
      for (int c = a; c < bw; ++c) acc = fma(Ls[b * ldm + c], X[c * ldm + a], acc);
      Hg[e] = acc;
    }
  }
  __syncthreads();
}

// ---------------------------------------------------------------------------
// The partitioned factorisation (grid mode).  Every block of the grid takes
// part in the Gram matrix; block k < P eliminates interior k (and forms its
// spike products), block 0 runs the separator chain, block k < P-1 inverts
// separator k.  Returns the same value in every thread: 0 or the 1-based
// column of a non-positive pivot.
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
    const int bad = s.template band_chol_window_range<T, kGridBT>(
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
  if (k == 0 && *info == 0) {
    const int bad = bandp_chain<T>(s, bp);
    if (bad != 0 && threadIdx.x == 0) atomicMax(const_cast<int*>(info), bad);
  }
  s.sync();
  QTQP_TOC(kPhBpChain);
  QTQP_RETIC();
  if (*info == 0 && k < bp.P - 1) bandp_sep_inverse<T>(s, bp, k);
  s.sync();
  QTQP_TOC(kPhBpSepInv);
  return *info;
}

// ---------------------------------------------------------------------------
// The partitioned solve G x = v (grid mode), x into v; w is scratch of n
// entries.  Every thread of the grid calls it.
// ---------------------------------------------------------------------------
template <typename T, class S>
__device__ void bandp_solve(S& s, T* v, T* w) {
  const int bw = s.bw;
  const BandParts bp(s.n, bw, s.nparts);
  const int P = bp.P, k = blockIdx.x, lt = threadIdx.x, lane = lt & 31, warp = lt >> 5;
  constexpr int kNW = kGridBT / 32;
  // Scratch after the solve rings (band_fwd_range / band_bwd_range).
  T* scr = reinterpret_cast<T*>(s.bwin) + (128 + kBandRing * 128 + kBandRing);
  QTQP_TIC();
  // Forward per interior; t_k's spike term W_L^T y of interior k+1.
  if (k < P) {
    const int lo = bp.lo(k), li = bp.li(k), hi = lo + li, R = hi + (k < P - 1 ? bw : 0);
    if (warp == 0) s.template band_fwd_range<T>(v, w, lo, li, R, lane);
    __syncthreads();
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
  // u_k = Li_k (v[S_k] - W_L^T y).
  if (k < P - 1) {
    const int hi = bp.lo(k) + bp.li(k);
    const T* cl = sep_vec<T>(s, k, kSvCL);
    if (lt < bw) scr[lt] = v[hi + lt] - cl[lt];
    __syncthreads();
    const T* Li = sep_block<T>(s, k, kSbI);
    T* u = sep_vec<T>(s, k, kSvU);
    for (int a = warp; a < bw; a += kNW) {
      T acc = T(0);
      for (int c = lane; c <= a; c += 32) acc = fma(Li[size_t(a) * bw + c], scr[c], acc);
      acc = warp_sum(acc);
      if (lane == 0) u[a] = acc;
    }
  }
  s.sync();
  // Chain z_k = u_k - G_k z_{k-1} (block 0).
  if (k == 0) {
    for (int j = 0; j < P - 1; ++j) {
      T* zs = scr + (j & 1) * 128;
      const T* zp = scr + ((j + 1) & 1) * 128;
      const T* u = sep_vec<T>(s, j, kSvU);
      const T* G = sep_block<T>(s, j, kSbG);
      T* z = sep_vec<T>(s, j, kSvZ);
      for (int a = warp; a < bw; a += kNW) {
        T acc = T(0);
        if (j > 0)
          for (int c = lane; c < bw; c += 32) acc = fma(G[size_t(a) * bw + c], zp[c], acc);
        acc = warp_sum(acc);
        if (lane == 0) {
          const T zv = u[a] - acc;
          zs[a] = zv;
          z[a] = zv;
        }
      }
      __syncthreads();
    }
  }
  s.sync();
  // v_k = Li_k^T z_k.
  if (k < P - 1) {
    const T* Li = sep_block<T>(s, k, kSbI);
    const T* z = sep_vec<T>(s, k, kSvZ);
    const int a = lt & 127, g = lt >> 7;
    T acc = T(0);
    if (a < bw)
      for (int c = a + g; c < bw; c += 2) acc = fma(Li[size_t(c) * bw + a], z[c], acc);
    scr[lt] = acc;
    __syncthreads();
    if (lt < bw) sep_vec<T>(s, k, kSvV)[lt] = scr[lt] + scr[lt + 128];
  }
  s.sync();
  // Chain x_k = v_k - H_k x_{k+1} (block 0), into the separator rows of v.
  if (k == 0) {
    for (int j = P - 2; j >= 0; --j) {
      T* xs = scr + (j & 1) * 128;
      const T* xn = scr + ((j + 1) & 1) * 128;
      const T* vv = sep_vec<T>(s, j, kSvV);
      const T* H = sep_block<T>(s, j, kSbH);
      const int hi = bp.lo(j) + bp.li(j);
      for (int a = warp; a < bw; a += kNW) {
        T acc = T(0);
        if (j < P - 2)
          for (int c = lane; c < bw; c += 32) acc = fma(H[size_t(a) * bw + c], xn[c], acc);
        acc = warp_sum(acc);
        if (lane == 0) {
          const T xv = vv[a] - acc;
          xs[a] = xv;
          v[hi + a] = xv;
        }
      }
      __syncthreads();
    }
  }
  s.sync();
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
    if (warp == 0) s.template band_bwd_range<T>(v, w, lo, hi, R, lane);
  }
  s.sync();
  QTQP_TOC(kPhBpBwd);
}

}  // namespace qtqp
