// Large-format phases of the device IPM (FMT == kFmtLarge): one large dense QP
// solved by a cooperative grid of kLargeBlocks blocks.  The interior-point
// logic is the shared Ipm code; here are the KKT factorisation and the
// triangular solves, blocked for the whole GPU:
//
//   Gram      G = P_off + diag(Rx) + A^T diag(1/Ry) A  (solvers_dense.py:99-116)
//             FP32 factor: X = (diag(1/sqrt(Ry)) A)^T split into TF32 hi + lo,
//             lower 128 x 128 tiles of X X^T on tcgen05 (three TF32 products,
//             FP32 accumulation in TMEM).  FP64 factor: lower 128 x 128 tiles
//             on the FP64 tensor cores (DMMA, mma.sync m8n8k4).
//   Cholesky  right-looking with 128-wide panels: the diagonal block by one
//             CTA in shared memory, the panel by row-wise substitution (one
//             warp per row), the trailing update in 128 x 128 tiles (DMMA in
//             FP64, 8 x 8 register tiles in FP32); then the inverse of every
//             diagonal block.
//   Solves    block forward / backward substitution with the inverted
//             diagonal blocks; CTA j owns block row j and waits on per-block
//             flags for the blocks it needs, one grid barrier per solve.
//
// Padding: the factor is npad x npad (npad = n rounded up to 128) with an
// identity on the padded diagonal; X is npad x mpad with zero padding.
#pragma once

#include "dense_ipm.cuh"
#include "tc_common.cuh"

namespace qtqp {

constexpr int kLB = 128;                          // panel / diagonal block size
constexpr int kLargeBlocks = 148;                 // CTAs of the cooperative grid: one per SM
constexpr int kLargeNT = kLargeBlocks * kGridBT;  // 37888 threads
constexpr int kTcStages = 3;
constexpr uint32_t kTcTileBytes = kLB * 32 * 4;        // 128 rows x 32 FP32
constexpr uint32_t kTcStageBytes = 4 * kTcTileBytes;   // A hi, B hi, A lo, B lo
constexpr size_t kArenaBytes = kTcStages * kTcStageBytes;  // 192 KB
constexpr size_t kLargeSmem = 1024 + kArenaBytes + 256;    // + alignment + barriers

__host__ __device__ inline int round_up(int v, int q) { return (v + q - 1) / q * q; }

// Global workspace of a large solve.
struct LargeLayout {
  int n, m, npad, mpad, nblk, np;
  size_t ctl_off, info_off, v_off, a_off, p_off, g64_off, g32_off, linv_off, sinv_off, xhi_off,
      xlo_off, cp_off, total;
};
__host__ __device__ inline LargeLayout plan_large_layout(int n, int m) {
  LargeLayout L;
  L.n = n;
  L.m = m;
  L.npad = round_up(n, kLB);
  L.mpad = round_up(m, 32);
  L.nblk = L.npad / kLB;
  L.np = (max(n + m, n + 4) + 1) & ~1;
  auto al = [](size_t b) { return (b + 1023) & ~size_t(1023); };
  size_t off = 0;
  L.ctl_off = off;
  off += al(sizeof(GridCtl));
  L.info_off = off;
  off += al(16);
  L.v_off = off;
  off += al(size_t(kNumVec) * L.np * 8);
  L.a_off = off;
  off += al(size_t(m) * n * 8);
  L.p_off = off;
  off += al(size_t(n) * n * 8);
  L.g64_off = off;
  off += al(size_t(L.npad) * L.npad * 8);
  L.g32_off = off;
  off += al(size_t(L.npad) * L.npad * 4);
  L.linv_off = off;
  off += al(2 * size_t(L.nblk) * kLB * kLB * 8);  // inverses and their transposes
  L.sinv_off = off;
  off += al(4 * 32 * 33 * 8);                      // sub-block inverses of one step
  L.xhi_off = off;
  off += al(size_t(L.npad) * L.mpad * 4);
  L.xlo_off = off;
  off += al(size_t(L.npad) * L.mpad * 4);
  L.cp_off = off;  // per-block column sums of large_products
  off += al(size_t(kLargeBlocks) * L.npad * 8);
  L.total = off;
  return L;
}

// ---------------------------------------------------------------------------
// One pass over the rows of A (and P) for the products a KKT residual needs
// together: the row dots (A vx)_i, passed to row_epi(i, value) by one thread
// each (none when vx is null), and the column sums c_k = sum_i A_ik vy_i
// vs_i (vs null: 1) + sum_i P_ik vp_i (when vp is given; P is symmetric, so
// that is (P vp)_k), passed to col_epi(k, c_k) by the thread k % NT after a
// grid barrier.  The rows of the stacked matrix
// [A; P] are cut into one contiguous band per block, and each band into
// chunks of kPrRows rows; within a tile of kPrTile columns each warp takes
// kPrCpl x 32 consecutive columns (lane l: columns l + 32 t), so every row is
// read once, coalesced, with kPrCpl loads in flight per lane, and each lane
// keeps its columns' sums in registers over the chunk.  The row dots of a
// chunk are combined over warps and tiles in shared memory; the blocks'
// column sums go to global memory and are added in block order.  Every sum
// runs in a fixed order, so the results are the same on every run.
// ---------------------------------------------------------------------------
constexpr int kPrCpl = 16;                         // columns per lane in a tile
constexpr int kPrTile = (kGridBT / 32) * 32 * kPrCpl;  // 4096 columns
constexpr int kPrRows = 256;                       // rows per chunk (rowpart in smem)
// The products' shared memory starts behind the diagonal-block inverse (128
// x 129 doubles) and the partial sums (128) that large_chol_solve keeps
// resident in the arena from the factorisation on.
constexpr size_t kPrSmemOff = (size_t(kLB) * (kLB + 1) + kLB) * sizeof(double);
static_assert(kPrSmemOff + (size_t(kPrRows) * (kGridBT / 32) + kPrTile) * sizeof(double) <=
                  kArenaBytes, "the products' shared memory exceeds the arena");

template <class S, class RowEpi, class ColEpi>
__device__ void large_products(S& s, const double* vx, const double* vy, const double* vs,
                               const double* vp, RowEpi row_epi, ColEpi col_epi) {
  constexpr int NW = kGridBT / 32;
  const int n = s.n, m = s.m, lda = s.lda, ldp = s.ldp;
  const double* A = s.A;
  const double* P = s.P;
  const int G = gridDim.x, b = blockIdx.x;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int rows = m + (vp != nullptr ? n : 0);
  const int band = (rows + G - 1) / G;
  const int r0 = min(rows, b * band), r1 = min(rows, r0 + band);
  double* rowpart = reinterpret_cast<double*>(s.arena + kPrSmemOff);  // kPrRows x NW
  double* xs = rowpart + kPrRows * NW;                    // vx of one tile
  double* part = s.colpart + size_t(b) * s.npad;
  for (int k = threadIdx.x; k < n; k += blockDim.x) part[k] = 0.0;
  __syncthreads();
  for (int c0 = r0; c0 < r1; c0 += kPrRows) {
    const int c1 = min(r1, c0 + kPrRows);
    for (int e = threadIdx.x; e < (c1 - c0) * NW; e += blockDim.x) rowpart[e] = 0.0;
    for (int t0 = 0; t0 < n; t0 += kPrTile) {
      if (vx != nullptr)
        for (int k = threadIdx.x; k < kPrTile; k += blockDim.x)
          xs[k] = t0 + k < n ? vx[t0 + k] : 0.0;
      __syncthreads();
      const int cb = t0 + warp * 32 * kPrCpl + lane;  // this lane's first column
      double acc[kPrCpl];
#pragma unroll
      for (int t = 0; t < kPrCpl; ++t) acc[t] = 0.0;
      auto row_of = [&](int i) {
        return i < m ? A + size_t(i) * lda : P + size_t(i - m) * ldp;
      };
      auto weight_of = [&](int i) {
        return i < m ? (vs != nullptr ? vy[i] * vs[i] : vy[i]) : vp[i - m];
      };
      // The row dot of row i from its loaded values (the same branch for the
      // whole warp).
      auto row_dot = [&](int i, const double (&a)[kPrCpl]) {
        if (i < m && vx != nullptr) {
          double d = 0.0;
#pragma unroll
          for (int t = 0; t < kPrCpl; ++t) d = fma(a[t], xs[cb - t0 + 32 * t], d);
#pragma unroll
          for (int o = 16; o > 0; o >>= 1) d += __shfl_xor_sync(0xffffffffu, d, o);
          if (lane == 0) rowpart[(i - c0) * NW + warp] += d;
        }
      };
      // Two rows per step, all of their loads issued before the first use
      // (2 x kPrCpl loads in flight per lane); the column sums still add row
      // i before row i + 1.
      int i = c0;
      for (; i + 1 < c1; i += 2) {
        const double* M0 = row_of(i);
        const double* M1 = row_of(i + 1);
        double a0[kPrCpl], a1[kPrCpl];
#pragma unroll
        for (int t = 0; t < kPrCpl; ++t) {
          const bool in = cb + 32 * t < n;
          a0[t] = in ? M0[cb + 32 * t] : 0.0;
          a1[t] = in ? M1[cb + 32 * t] : 0.0;
        }
        const double w0 = weight_of(i), w1 = weight_of(i + 1);
#pragma unroll
        for (int t = 0; t < kPrCpl; ++t) acc[t] = fma(a1[t], w1, fma(a0[t], w0, acc[t]));
        row_dot(i, a0);
        row_dot(i + 1, a1);
      }
      if (i < c1) {
        const double* M0 = row_of(i);
        double a0[kPrCpl];
#pragma unroll
        for (int t = 0; t < kPrCpl; ++t) a0[t] = cb + 32 * t < n ? M0[cb + 32 * t] : 0.0;
        const double w0 = weight_of(i);
#pragma unroll
        for (int t = 0; t < kPrCpl; ++t) acc[t] = fma(a0[t], w0, acc[t]);
        row_dot(i, a0);
      }
#pragma unroll
      for (int t = 0; t < kPrCpl; ++t)
        if (cb + 32 * t < n) part[cb + 32 * t] += acc[t];
      __syncthreads();
    }
    for (int i = c0 + threadIdx.x; i < c1 && vx != nullptr; i += blockDim.x) {
      if (i >= m) continue;
      double v = 0.0;
#pragma unroll
      for (int w = 0; w < NW; ++w) v += rowpart[(i - c0) * NW + w];
      row_epi(i, v);
    }
    __syncthreads();
  }
  s.sync();
  for (int k = s.tid; k < n; k += kLargeNT) {
    double v = 0.0;
    for (int bb = 0; bb < G; ++bb) v += s.colpart[size_t(bb) * s.npad + k];
    col_epi(k, v);
  }
}

// ---------------------------------------------------------------------------
// Gram of the FP32 factor on tcgen05.
// ---------------------------------------------------------------------------
// X = (diag(w) A)^T split into TF32 hi + lo (w = 1/sqrt(Ry) at vec(kPW)[n+i]),
// by 32 x 32 tiles transposed through shared memory.
template <class S>
__device__ void large_scale_split(S& s) {
  const int n = s.n, m = s.m, npad = s.npad, mpad = s.mpad;
  const double* A = s.A;
  const double* w = s.vec(kPW) + n;
  float* t = reinterpret_cast<float*>(s.arena);  // 32 x 33
  const int tr = threadIdx.x >> 5, tc = threadIdx.x & 31;  // 8 rows per pass
  const int tiles_i = mpad / 32, tiles_j = npad / 32;
  for (int t_id = blockIdx.x; t_id < tiles_i * tiles_j; t_id += gridDim.x) {
    const int i0 = (t_id % tiles_i) * 32, j0 = (t_id / tiles_i) * 32;
    for (int r = tr; r < 32; r += 8) {  // rows i of A, columns j coalesced
      const int i = i0 + r, j = j0 + tc;
      t[r * 33 + tc] = (i < m && j < n) ? float(A[size_t(i) * n + j] * w[i]) : 0.0f;
    }
    __syncthreads();
    for (int r = tr; r < 32; r += 8) {  // rows j of X, columns i coalesced
      const float v = t[tc * 33 + r];
      uint32_t h;
      asm("cvt.rna.tf32.f32 %0, %1;" : "=r"(h) : "f"(v));
      const size_t o = size_t(j0 + r) * mpad + i0 + tc;
      s.xhi[o] = __uint_as_float(h);
      s.xlo[o] = v - __uint_as_float(h);
    }
    __syncthreads();
  }
}

// Lower 128 x 128 tiles of X X^T (three TF32 products) into g32.  Warp 0
// lane 0 loads (TMA, 3-stage ring), warp 1 lane 0 issues the MMAs, all
// eight warps drain TMEM (warp w: lanes 32 (w % 4), columns 64 (w / 4)).
// The ring counters continue across tiles and calls (s.tc_load / s.tc_mma /
// s.tc_tiles are per-thread copies; each role advances its own).
template <class S>
__device__ void large_gram_tc(S& s) {
  const int npad = s.npad, k_tiles = s.mpad / 32, nt = npad / kLB;
  uint8_t* ring = s.arena;
  uint64_t* bars = reinterpret_cast<uint64_t*>(ring + kArenaBytes);
  uint64_t* full = bars;
  uint64_t* empty = bars + kTcStages;
  uint64_t* done = bars + 2 * kTcStages;
  int* failed = reinterpret_cast<int*>(done + 1);
  const CUtensorMap* mh = static_cast<const CUtensorMap*>(s.map_hi);
  const CUtensorMap* ml = static_cast<const CUtensorMap*>(s.map_lo);
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  constexpr uint32_t idesc = tc::idesc_f32acc(kLB, kLB, false);
  const int tiles = nt * (nt + 1) / 2;
  for (int t = blockIdx.x; t < tiles; t += gridDim.x) {
    int ti = 0;
    while ((ti + 1) * (ti + 2) / 2 <= t) ++ti;
    const int tj = t - ti * (ti + 1) / 2;
    if (warp == 0 && lane == 0) {
      for (int kt = 0; kt < k_tiles; ++kt) {
        const uint32_t g = s.tc_load++;
        const int st = int(g % kTcStages);
        const uint32_t use = g / kTcStages;
        if (use > 0 && !tc::mbar_wait(&empty[st], (use - 1) & 1)) {
          s.tc_load--;  // stage g was not issued
          atomicExch(failed, 1);
          break;
        }
        uint8_t* sb = ring + st * kTcStageBytes;
        tc::mbar_arrive_expect_tx(&full[st], kTcStageBytes);
        tc::tma_load_2d(sb, mh, kt * 32, ti * kLB, &full[st]);
        tc::tma_load_2d(sb + kTcTileBytes, mh, kt * 32, tj * kLB, &full[st]);
        tc::tma_load_2d(sb + 2 * kTcTileBytes, ml, kt * 32, ti * kLB, &full[st]);
        tc::tma_load_2d(sb + 3 * kTcTileBytes, ml, kt * 32, tj * kLB, &full[st]);
      }
    } else if (warp == 1 && lane == 0) {
      for (int kt = 0; kt < k_tiles; ++kt) {
        const uint32_t g = s.tc_mma++;
        const int st = int(g % kTcStages);
        const uint32_t use = g / kTcStages;
        if (!tc::mbar_wait(&full[st], use & 1)) {
          s.tc_mma--;  // stage g was not consumed
          atomicExch(failed, 1);
          break;
        }
        tc::fence_after_sync();
        const uint32_t a_hi = tc::smem_u32(ring + st * kTcStageBytes);
        const uint32_t b_hi = a_hi + kTcTileBytes, a_lo = a_hi + 2 * kTcTileBytes,
                       b_lo = a_hi + 3 * kTcTileBytes;
#pragma unroll
        for (int kk = 0; kk < 4; ++kk) {
          const uint32_t off = kk * 32;
          tc::mma_tf32(s.tmem, tc::desc_kmajor_sw128(a_hi + off), tc::desc_kmajor_sw128(b_hi + off),
                       idesc, (kt | kk) != 0);
          tc::mma_tf32(s.tmem, tc::desc_kmajor_sw128(a_hi + off), tc::desc_kmajor_sw128(b_lo + off),
                       idesc, 1);
          tc::mma_tf32(s.tmem, tc::desc_kmajor_sw128(a_lo + off), tc::desc_kmajor_sw128(b_hi + off),
                       idesc, 1);
        }
        tc::mma_commit(&empty[st]);
      }
      tc::mma_commit(done);
    }
    __syncwarp();
    if (!tc::mbar_wait(done, s.tc_tiles & 1)) atomicExch(failed, 1);
    s.tc_tiles++;
    tc::fence_after_sync();
    if (warp == 1 && lane == 0) failed[1] = int(s.tc_mma);  // stages consumed so far
    __syncthreads();
    if (*failed != 0) {
      // A bounded wait gave up: stop issuing tiles.  Before the CTA moves on,
      // the producer waits (again bounded) for the stages it issued that the
      // MMA issuer never consumed, so that no bulk copy still targets the
      // ring when the arena is reused.
      if (warp == 0 && lane == 0) {
        for (uint32_t g = uint32_t(failed[1]); g < s.tc_load; ++g)
          if (!tc::mbar_wait(&full[g % kTcStages], (g / kTcStages) & 1)) break;
      }
      __syncthreads();
      break;
    }
    {
      const int q = warp & 3, half = warp >> 2;
      const int row = ti * kLB + q * 32 + lane;
      float* grow = s.g32l + size_t(row) * npad + size_t(tj) * kLB + half * 64;
#pragma unroll 1
      for (int c0 = 0; c0 < 64; c0 += 32) {
        float v[32];
        tc::tmem_ld32(s.tmem + (uint32_t(q * 32) << 16) + uint32_t(half * 64 + c0), v);
#pragma unroll
        for (int e = 0; e < 32; e += 4)
          *reinterpret_cast<float4*>(grow + c0 + e) = make_float4(v[e], v[e + 1], v[e + 2], v[e + 3]);
      }
    }
    tc::fence_before_sync();
    __syncthreads();  // TMEM free for the next tile's MMAs
  }
  if (threadIdx.x == 0 && *failed) atomicExch(&s.gctl->err, 1);
}

// G_lower = A^T diag(1/Ry) A in FP64 on the FP64 tensor cores (DMMA,
// mma.sync m8n8k4): one CTA per 128 x 128 lower tile; K-slices of 16 rows of
// A (both column panels) and their weights staged by cp.async in a ring of
// four buffers (three slices in flight), with a row pitch of 132 so that each half-warp's fragment loads
// hit 16 different banks; warp w computes the 64 x 32 block (w / 4, w % 4)
// of the tile with 8 x 4 accumulators of 8 x 8.  Rows and columns beyond
// m, n are zero-filled.
template <class S>
__device__ __noinline__ void large_gram_dmma(S& s) {
  const int n = s.n, m = s.m, npad = s.npad;
  const double* A = s.A;
  const double* iry = s.vec(kPI) + n;  // 1 / Ry
  constexpr int KS = 16;               // rows per slice
  constexpr int LP = kLB + 4;          // staged row pitch
  constexpr int SL = 2 * KS * LP + KS; // doubles per buffer
  constexpr int NS = 4;                // slices in flight (ring of NS buffers)
  static_assert(NS * SL * sizeof(double) <= kArenaBytes, "Gram ring exceeds the arena");
  double* smem = reinterpret_cast<double*>(s.arena);
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int gi = lane >> 2, tg = lane & 3;
  const int wr = warp >> 2, wc = warp & 3;
  const int nt = npad / kLB, tiles = nt * (nt + 1) / 2;
  auto issue = [&](int r0, int i0, int j0, int buf) {
    double* sa = smem + buf * SL;
    double* sb = sa + KS * LP;
    double* sw = sb + KS * LP;
#pragma unroll
    for (int q = 0; q < 8; ++q) {
      const int e = threadIdx.x + q * kGridBT, r = e >> 7, c = e & 127, i = r0 + r;
      const bool ok = i < m;
      cp_async8(sa + r * LP + c, A + (ok && i0 + c < n ? size_t(i) * n + i0 + c : 0),
                ok && i0 + c < n);
      cp_async8(sb + r * LP + c, A + (ok && j0 + c < n ? size_t(i) * n + j0 + c : 0),
                ok && j0 + c < n);
    }
    if (threadIdx.x < KS) {
      const int i = r0 + threadIdx.x;
      cp_async8(sw + threadIdx.x, iry + (i < m ? i : 0), i < m);
    }
    cp_async_commit();
  };
  for (int t = blockIdx.x; t < tiles; t += gridDim.x) {
    int ti = 0;
    while ((ti + 1) * (ti + 2) / 2 <= t) ++ti;
    const int tj = t - ti * (ti + 1) / 2;
    const int i0 = ti * kLB, j0 = tj * kLB;
    double acc[8][4][2];
#pragma unroll
    for (int a = 0; a < 8; ++a)
#pragma unroll
      for (int b = 0; b < 4; ++b) acc[a][b][0] = acc[a][b][1] = 0.0;
    const int nsl = (m + KS - 1) / KS;
    // Slices 0 .. NS-2 in flight (empty groups past the end keep the count).
#pragma unroll
    for (int q = 0; q < NS - 1; ++q) {
      if (q < nsl) {
        issue(q * KS, i0, j0, q);
      } else {
        cp_async_commit();
      }
    }
    for (int q = 0; q < nsl; ++q) {
      // Slice q + NS - 1 goes into the buffer read at step q - 1 (released by
      // that step's closing barrier); then slice q has landed.
      const int nx = q + NS - 1;
      if (nx < nsl) {
        issue(nx * KS, i0, j0, nx % NS);
      } else {
        cp_async_commit();
      }
      cp_async_wait<NS - 1>();
      __syncthreads();
      const int buf = q % NS;
      const double* sa = smem + buf * SL + wr * 64 + gi;
      const double* sb = smem + buf * SL + KS * LP + wc * 32 + gi;
      const double* sw = smem + buf * SL + 2 * KS * LP;
#pragma unroll
      for (int k0 = 0; k0 < KS; k0 += 4) {
        const int r = k0 + tg;
        const double w = sw[r];
        double a[8], b[4];
#pragma unroll
        for (int mi = 0; mi < 8; ++mi) a[mi] = sa[r * LP + mi * 8] * w;
#pragma unroll
        for (int ni = 0; ni < 4; ++ni) b[ni] = sb[r * LP + ni * 8];
#pragma unroll
        for (int mi = 0; mi < 8; ++mi)
#pragma unroll
          for (int ni = 0; ni < 4; ++ni) dmma_8x8x4(acc[mi][ni], a[mi], b[ni]);
      }
      __syncthreads();  // everyone is done with `buf` before it is refilled
    }
#pragma unroll
    for (int mi = 0; mi < 8; ++mi)
#pragma unroll
      for (int ni = 0; ni < 4; ++ni) {
        const int i = i0 + wr * 64 + mi * 8 + gi, j = j0 + wc * 32 + ni * 8 + 2 * tg;
        s.g64[size_t(i) * npad + j] = acc[mi][ni][0];
        s.g64[size_t(i) * npad + j + 1] = acc[mi][ni][1];
      }
  }
}

// G += P_off + diag(Rx) on the lower triangle, identity padding, then the
// relative diagonal jitter (1e-14 in FP64 as solvers_dense.py:112; 2^-22 at
// FP32 resolution).
template <typename T, class S>
__device__ void large_finish_gram(S& s, T* g) {
  const int n = s.n, npad = s.npad, tid = s.tid;
  const double* P = s.P;
  const double* reg = s.vec(kREG);
  double dmax[1] = {0.0};
  double dummy[1] = {0.0};
  const size_t total = size_t(npad) * npad;
  for (size_t e = tid; e < total; e += kLargeNT) {
    const int i = int(e / npad), j = int(e % npad);
    if (j > i) continue;
    if (i >= n || j >= n) {
      g[e] = (i == j) ? T(1) : T(0);
      continue;
    }
    double base = P[size_t(i) * n + j];
    if (i == j) base += reg[i];
    const T v = T(base) + g[e];
    g[e] = v;
    if (i == j) dmax[0] = nanmax(dmax[0], double(v));
  }
  s.template reduce<0, 1>(dummy, dmax);
  const double jit = (sizeof(T) == 8 ? 1e-14 : 2.384185791015625e-07) * dmax[0];
  for (int k = tid; k < n; k += kLargeNT) g[size_t(k) * npad + k] = T(double(g[size_t(k) * npad + k]) + jit);
  s.sync();
}

// ---------------------------------------------------------------------------
// Blocked Cholesky of the lower triangle of g (npad x npad), then the
// inverses of the diagonal blocks into linv (and, resident in each CTA's
// shared memory, the inverse of the block the CTA owns in the solves).
// Returns 0 or the 1-based index of the first non-positive pivot (uniform
// over the grid).
//
// Step k (panel width 128):
//   (a) one CTA factors the diagonal block in shared memory, in four 32-wide
//       steps: one warp factors the 32 x 32 diagonal sub-block in registers
//       and inverts it, the rows below are solved with that inverse, and the
//       trailing part of the block is updated;
//   (b) every warp takes panel rows and solves x L_kk^T = g_i with the four
//       sub-block inverses (one lane per column, broadcasts by shuffle);
//   (c) the lower 128 x 128 tiles right of the panel get g_ij -= L_ik L_jk^T
//       with 8 x 8 outputs per thread and cp.async double-buffered slices.
// ---------------------------------------------------------------------------
constexpr int kPitch = kLB + 1;   // shared-memory pitch of a staged 128 x 128 block
constexpr int kSubPitch = 33;     // pitch of a staged 32 x 32 block

// 128 x 128 block of g at (r0, c0) into dst[r * kPitch + c], eight loads in
// flight per thread; the strict upper part is zero when lower_only.
template <typename T>
__device__ __forceinline__ void stage_block(T* dst, const T* g, size_t ld, int r0, int c0,
                                            bool lower_only) {
  for (int base = threadIdx.x; base < kLB * kLB; base += 8 * kGridBT) {
    T v[8];
#pragma unroll
    for (int q = 0; q < 8; ++q) {
      const int e = base + q * kGridBT, r = e >> 7, c = e & 127;
      v[q] = (!lower_only || c <= r) ? g[size_t(r0 + r) * ld + c0 + c] : T(0);
    }
#pragma unroll
    for (int q = 0; q < 8; ++q) {
      const int e = base + q * kGridBT;
      dst[(e >> 7) * kPitch + (e & 127)] = v[q];
    }
  }
}

// One warp factors the 32 x 32 lower block at sm[o][o] (pitch kPitch) and
// writes its inverse to inv32[r * kSubPitch + c].  Returns 0 or the 1-based
// failing pivot (the same in every lane).
//
// Factor: Crout order, lane r holds row r in registers; step c forms
// s_r = a_rc - sum_{k<c} l_rk l_ck (row c of L read back from shared memory,
// the same address in every lane), l_cc = sqrt(s_c), l_rc = s_r / l_cc.
// Inverse: lane c forms column c top-down, X_rc = -(sum_{c<=k<r} L_rk X_kc)
// / l_rr.  Every division and square root goes through one reciprocal
// square root per pivot (1 / l_cc = rsqrt(s_c)), kept for the inverse:
// these are the long-latency operations of this sequential chain.
template <typename T>
__device__ __noinline__ int warp_chol32(T* sm, int o, T* inv32, int lane) {
  T* Lr = sm + (o + lane) * kPitch + o;  // this lane's row
  T idg[32];                              // 1 / l_cc (the same in every lane)
  int bad = 0;
  {
    T a[32];
#pragma unroll
    for (int j = 0; j < 32; ++j) a[j] = (j <= lane) ? Lr[j] : T(0);
#pragma unroll
    for (int c = 0; c < 32; ++c) {
      const T* Lc = sm + (o + c) * kPitch + o;
      T s0 = a[c], s1 = T(0);
#pragma unroll
      for (int k = 0; k < c; ++k) {
        if (k & 1) {
          s1 = fma(-a[k], Lc[k], s1);
        } else {
          s0 = fma(-a[k], Lc[k], s0);
        }
      }
      const T sr = s0 + s1;
      const T piv = __shfl_sync(0xffffffffu, sr, c);
      if (!(piv > T(0)) && bad == 0) bad = c + 1;
      const T il = rsqrt(piv);
      idg[c] = il;
      if (lane == c) {
        a[c] = piv * il;
      } else if (lane > c) {
        a[c] = sr * il;
      }
      if (lane >= c) Lr[c] = a[c];
      __syncwarp();
    }
  }
  if (bad) return bad;
  T x[32];
  const T* L = sm + o * kPitch + o;
#pragma unroll
  for (int r = 0; r < 32; ++r) {
    T a0 = T(0), a1 = T(0);
#pragma unroll
    for (int k = 0; k < r; ++k) {
      if (k >= lane) {
        if (k & 1) {
          a1 = fma(L[r * kPitch + k], x[k], a1);
        } else {
          a0 = fma(L[r * kPitch + k], x[k], a0);
        }
      }
    }
    x[r] = r < lane ? T(0) : (r == lane ? idg[r] : -(a0 + a1) * idg[r]);
  }
#pragma unroll
  for (int r = 0; r < 32; ++r) inv32[r * kSubPitch + lane] = x[r];
  return 0;
}

template <typename T, class S>
__device__ int large_cholesky(S& s, T* g) {
  const int npad = s.npad, nblk = npad / kLB;
  int* info = s.linfo;
  T* sm = reinterpret_cast<T*>(s.arena);   // staged 128 x 128 block (pitch kPitch)
  T* sinv = sm + kLB * kPitch;              // 4 sub-block inverses (pitch kSubPitch)
  volatile int* sflag = reinterpret_cast<volatile int*>(sinv + 4 * 32 * kSubPitch);
  T* ginv = reinterpret_cast<T*>(s.sinv);   // the same inverses in global memory
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int gwarp = blockIdx.x * (kGridBT / 32) + warp, nwarps = gridDim.x * (kGridBT / 32);
  if (s.tid == 0) *info = 0;
  s.sync();
  QTQP_TIC();
  // (a) Factor the diagonal block starting at column k0 (the calling CTA):
  // in shared memory, 32 columns at a time, then back to g with the four
  // 32 x 32 sub-block inverses (also to global memory, for the panel step).
  auto factor_diag = [&](int k0) {
    QTQP_TIC();
    stage_block(sm, g, npad, k0, k0, true);
    __syncthreads();
    QTQP_TOC(kPhNormalize);
    int bad = 0;
    for (int q = 0; q < 4 && !bad; ++q) {
      const int o = 32 * q;
      QTQP_RETIC();
      if (warp == 0) {
        const int b = warp_chol32(sm, o, sinv + q * 32 * kSubPitch, lane);
        if (lane == 0) *sflag = b ? o + b : 0;
      }
      __syncthreads();
      QTQP_TOC(kPhStep);
      QTQP_RETIC();
      bad = *sflag;
      if (bad) break;
      // Rows below the sub-block: x = row inv(L_qq)^T (thread per row).
      const T* iq = sinv + q * 32 * kSubPitch;
      const int rows = kLB - o - 32;
      if (int(threadIdx.x) < rows) {
        T* row = sm + (o + 32 + threadIdx.x) * kPitch + o;
        T v[32];
#pragma unroll
        for (int l = 0; l < 32; ++l) v[l] = row[l];
#pragma unroll
        for (int j = 0; j < 32; ++j) {
          T acc = T(0);
#pragma unroll
          for (int l = 0; l <= j; ++l) acc = fma(v[l], iq[j * kSubPitch + l], acc);
          row[j] = acc;
        }
      }
      __syncthreads();
      // Trailing lower part of the block: a_ij -= sum_l a_il a_jl.
      const int t0 = o + 32, tn = kLB - t0, cnt = tn * (tn + 1) / 2;
      for (int e = threadIdx.x; e < cnt; e += blockDim.x) {
        int i = int((sqrtf(8.0f * e + 1.0f) - 1.0f) * 0.5f);
        while (i * (i + 1) / 2 > e) --i;
        while ((i + 1) * (i + 2) / 2 <= e) ++i;
        const int j = e - i * (i + 1) / 2;
        const T* ri = sm + (t0 + i) * kPitch + o;
        const T* rj = sm + (t0 + j) * kPitch + o;
        T acc0 = T(0), acc1 = T(0);
#pragma unroll
        for (int l = 0; l < 32; l += 2) {
          acc0 = fma(ri[l], rj[l], acc0);
          acc1 = fma(ri[l + 1], rj[l + 1], acc1);
        }
        sm[(t0 + i) * kPitch + t0 + j] -= acc0 + acc1;
      }
      __syncthreads();
      QTQP_TOC(kPhOther);
    }
    if (bad) {
      if (threadIdx.x == 0) atomicCAS(info, 0, k0 + bad);
    } else {
      for (int e = threadIdx.x; e < kLB * kLB; e += blockDim.x) {
        const int r = e >> 7, c = e & 127;
        if (c <= r) g[size_t(k0 + r) * npad + k0 + c] = sm[r * kPitch + c];
      }
      for (int e = threadIdx.x; e < 4 * 32 * kSubPitch; e += blockDim.x) ginv[e] = sinv[e];
    }
    __syncthreads();
  };
  for (int k = 0; k < nblk; ++k) {
    const int k0 = k * kLB;
    QTQP_RETIC();
    // (a) diagonal block: only for the first one; every later one is
    // factored during the previous step's trailing update (lookahead).
    if (k == 0 && blockIdx.x == 0) factor_diag(k0);
    if (k == 0) s.sync();
    QTQP_TOC(kPhLgDiag);
    QTQP_RETIC();
    if (*reinterpret_cast<volatile int*>(info) != 0) break;
    const int rest = npad - k0 - kLB;
    if (rest == 0) break;
    // (b) panel rows.
    if (k0 + kLB + int(blockIdx.x) * (kGridBT / 32) < npad) {  // this CTA has rows
      stage_block(sm, g, npad, k0, k0, true);
      for (int e = threadIdx.x; e < 4 * 32 * kSubPitch; e += blockDim.x) sinv[e] = ginv[e];
      __syncthreads();
      for (int row = k0 + kLB + gwarp; row < npad; row += nwarps) {
        T* gr = g + size_t(row) * npad + k0;
        T v[4];
#pragma unroll
        for (int q = 0; q < 4; ++q) v[q] = gr[32 * q + lane];
#pragma unroll
        for (int q = 0; q < 4; ++q) {
          const T* iq = sinv + q * 32 * kSubPitch;
          T x = T(0);
#pragma unroll
          for (int l = 0; l < 32; ++l)
            x = fma(__shfl_sync(0xffffffffu, v[q], l), iq[lane * kSubPitch + l], x);
          v[q] = x;
#pragma unroll
          for (int q2 = q + 1; q2 < 4; ++q2) {
            const T* lr = sm + (32 * q2 + lane) * kPitch + 32 * q;
#pragma unroll
            for (int l = 0; l < 32; ++l) v[q2] = fma(-__shfl_sync(0xffffffffu, x, l), lr[l], v[q2]);
          }
        }
#pragma unroll
        for (int q = 0; q < 4; ++q) gr[32 * q + lane] = v[q];
      }
    }
    s.sync();
    QTQP_TOC(kPhLgPanel);
    QTQP_RETIC();
    // (c) trailing update (FP64: on the FP64 tensor cores, DMMA m8n8k4, warp w
    // on the 64 x 32 block (w / 4, w % 4) of the tile; FP32: 8 x 8 SIMT tiles).
    {
      constexpr int KS = 16;
      constexpr int SP = sizeof(T) == 8 ? kLB + 4 : kLB + 1;  // slice pitch
      constexpr int SL = 2 * KS * SP;                 // elements per buffer
      const int tx = threadIdx.x & 15, ty = threadIdx.x >> 4;
      const int nt = rest / kLB, tiles = nt * (nt + 1) / 2;
      const int base = k0 + kLB;
      auto issue = [&](int kk0, int i0, int j0, int buf) {
        T* pa = sm + buf * SL;
        T* pb = pa + KS * SP;
#pragma unroll
        for (int q = 0; q < 8; ++q) {
          const int e = threadIdx.x + q * kGridBT, r = e >> 4, kk = e & 15;
          if constexpr (sizeof(T) == 8) {
            cp_async8(pa + kk * SP + r, g + size_t(i0 + r) * npad + k0 + kk0 + kk, true);
            cp_async8(pb + kk * SP + r, g + size_t(j0 + r) * npad + k0 + kk0 + kk, true);
          } else {
            cp_async4(pa + kk * SP + r, g + size_t(i0 + r) * npad + k0 + kk0 + kk);
            cp_async4(pb + kk * SP + r, g + size_t(j0 + r) * npad + k0 + kk0 + kk);
          }
        }
        cp_async_commit();
      };
      // Lookahead: the CTA that owns the next diagonal block updates tile 0
      // (that block) first and factors it at once; the other tiles go round
      // robin over the other CTAs.
      const int G = int(gridDim.x), owner = (k + 1) % G, me = int(blockIdx.x);
      const int first_t = me == owner ? 0 : 1 + (me - owner - 1 + G) % G;
      const int step_t = me == owner ? tiles : G - 1;
      for (int t = first_t; t < tiles; t += (t == 0 ? tiles : step_t)) {
        int ti = 0;
        while ((ti + 1) * (ti + 2) / 2 <= t) ++ti;
        const int tj = t - ti * (ti + 1) / 2;
        const int i0 = base + ti * kLB, j0 = base + tj * kLB;
        T acc[8][8];
#pragma unroll
        for (int a = 0; a < 8; ++a)
#pragma unroll
          for (int b = 0; b < 8; ++b) acc[a][b] = T(0);
        issue(0, i0, j0, 0);
        int buf = 0;
        for (int kk0 = 0; kk0 < kLB; kk0 += KS) {
          if (kk0 + KS < kLB) {
            issue(kk0 + KS, i0, j0, buf ^ 1);
            cp_async_wait<1>();
          } else {
            cp_async_wait<0>();
          }
          __syncthreads();
          const T* pa = sm + buf * SL;
          const T* pb = pa + KS * SP;
          if constexpr (sizeof(T) == 8) {
            // acc[mi][ni / 2][...]: the 8 x 4 DMMA accumulators of this warp.
            const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
            const int gi = lane >> 2, tg = lane & 3, wr = warp >> 2, wc = warp & 3;
#pragma unroll
            for (int k4 = 0; k4 < KS; k4 += 4) {
              const double* ra = reinterpret_cast<const double*>(pa) + (k4 + tg) * SP + wr * 64 + gi;
              const double* rb = reinterpret_cast<const double*>(pb) + (k4 + tg) * SP + wc * 32 + gi;
              double a[8], b[4];
#pragma unroll
              for (int mi = 0; mi < 8; ++mi) a[mi] = ra[mi * 8];
#pragma unroll
              for (int ni = 0; ni < 4; ++ni) b[ni] = rb[ni * 8];
#pragma unroll
              for (int mi = 0; mi < 8; ++mi)
#pragma unroll
                for (int ni = 0; ni < 4; ++ni)
                  dmma_8x8x4(reinterpret_cast<double(&)[2]>(acc[mi][2 * ni]), a[mi], b[ni]);
            }
          } else {
#pragma unroll 2
            for (int kk = 0; kk < KS; ++kk) {
              T av[8], bv[8];
#pragma unroll
              for (int a = 0; a < 8; ++a) {
                av[a] = pa[kk * SP + ty + 16 * a];
                bv[a] = pb[kk * SP + tx + 16 * a];
              }
#pragma unroll
              for (int a = 0; a < 8; ++a)
#pragma unroll
                for (int b = 0; b < 8; ++b) acc[a][b] = fma(av[a], bv[b], acc[a][b]);
            }
          }
          __syncthreads();
          buf ^= 1;
        }
        if constexpr (sizeof(T) == 8) {
          const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
          const int gi = lane >> 2, tg = lane & 3, wr = warp >> 2, wc = warp & 3;
#pragma unroll
          for (int mi = 0; mi < 8; ++mi) {
            const int i = i0 + wr * 64 + mi * 8 + gi;
#pragma unroll
            for (int ni = 0; ni < 4; ++ni)
#pragma unroll
              for (int e = 0; e < 2; ++e) {
                const int j = j0 + wc * 32 + ni * 8 + 2 * tg + e;
                if (j <= i) g[size_t(i) * npad + j] -= acc[mi][2 * ni + e];
              }
          }
        } else {
#pragma unroll
          for (int a = 0; a < 8; ++a) {
            const int i = i0 + ty + 16 * a;
#pragma unroll
            for (int b = 0; b < 8; ++b) {
              const int j = j0 + tx + 16 * b;
              if (j <= i) g[size_t(i) * npad + j] -= acc[a][b];
            }
          }
        }
        if (t == 0) {  // the next diagonal block is final: factor it now
          __syncthreads();
          factor_diag(base);
        }
      }
    }
    s.sync();
    QTQP_TOC(kPhLgTrail);
  }
  const int rc = *reinterpret_cast<volatile int*>(info);
  if (rc != 0) return rc;
  QTQP_RETIC();
  // Inverses of the diagonal blocks: column c of inv(L_bb) by thread c.
  T* lv = reinterpret_cast<T*>(s.linv);
  for (int b = blockIdx.x; b < nblk; b += gridDim.x) {
    const int b0 = b * kLB;
    stage_block(sm, g, npad, b0, b0, true);
    __syncthreads();
    T* inv = lv + size_t(b) * kLB * kLB;                 // inv(L_bb), row-major
    T* invt = lv + size_t(nblk + b) * kLB * kLB;         // its transpose
    T* rdiag = sm + kLB * kPitch;  // 1 / L_rr
    if (threadIdx.x < kLB) rdiag[threadIdx.x] = T(1) / sm[threadIdx.x * kPitch + threadIdx.x];
    __syncthreads();
    if (threadIdx.x < kLB) {
      const int c = threadIdx.x;
      // Column c of inv(L_bb) = row c of its transpose (contiguous for this
      // thread): x_c = 1 / L_cc; x_r = -(sum_{c <= l < r} L_rl x_l) / L_rr.
      T* xc = invt + size_t(c) * kLB;
      for (int r = 0; r < c; ++r) xc[r] = T(0);
      xc[c] = rdiag[c];
      for (int r = c + 1; r < kLB; ++r) {
        T acc0 = T(0), acc1 = T(0);
        int l = c;
        for (; l + 1 < r; l += 2) {
          acc0 = fma(sm[r * kPitch + l], xc[l], acc0);
          acc1 = fma(sm[r * kPitch + l + 1], xc[l + 1], acc1);
        }
        if (l < r) acc0 = fma(sm[r * kPitch + l], xc[l], acc0);
        xc[r] = -(acc0 + acc1) * rdiag[r];
      }
    }
    __syncthreads();
    for (int e = threadIdx.x; e < kLB * kLB; e += blockDim.x) {
      const int r = e >> 7, c = e & 127;
      inv[e] = invt[size_t(c) * kLB + r];
    }
    __syncthreads();
  }
  s.sync();
  // Each CTA keeps the inverse of the block it owns in the solves resident
  // in shared memory until the next factorisation.
  if (int(blockIdx.x) < nblk) {
    stage_block(sm, lv + size_t(blockIdx.x) * kLB * kLB, kLB, 0, 0, false);
    __syncthreads();
  }
  QTQP_TOC(kPhLgInv);
  return 0;
}

template <typename T, class S>
__device__ int large_factorize(S& s) {
  QTQP_TIC();
  int info;
  if constexpr (sizeof(T) == 4) {
    large_scale_split(s);
    s.sync();
    large_gram_tc(s);
    s.sync();
    large_finish_gram<float>(s, s.g32l);
    QTQP_TOC(kPhGram);
    QTQP_RETIC();
    info = large_cholesky<float>(s, s.g32l);
  } else {
    large_gram_dmma(s);
    s.sync();
    large_finish_gram<double>(s, s.g64);
    QTQP_TOC(kPhGram);
    QTQP_RETIC();
    info = large_cholesky<double>(s, s.g64);
  }
  QTQP_TOC(kPhChol);
  return info;
}

// ---------------------------------------------------------------------------
// L L^T v = v in place (v, w: n entries of T; w is scratch), block by block
// with flags instead of grid barriers.  CTA j (j < nb) owns block row j and
// keeps inv(L_jj) resident in shared memory since the factorisation.
//   Forward:  z_j = inv(L_jj) (v_j - sum_{c<j} L_jc z_c) into w.  CTA j adds
//             L_jc z_c as soon as flag c shows z_c published, in the order
//             c = 0, 1, ..., so only the last product L_{j,j-1} z_{j-1} and
//             the diagonal step lie on the chain from one block to the next.
//   Backward: x_j = inv(L_jj)^T (z_j - sum_{c>j} L_cj^T x_c) into v, the
//             same way from c = nb-1 down.
// Every sum runs in a fixed order (c ascending or descending, then the
// lanes' and warps' partials in a fixed tree), so results do not depend on
// timing.  Flag generations: 2t - 1 (forward) and 2t (backward) for the t-th
// solve of the launch.  One grid barrier at the end.
// ---------------------------------------------------------------------------
template <typename T, class S>
__device__ void large_chol_solve(S& s, T* v, T* w) {
  const int n = s.n, npad = s.npad;
  const int nb = (n + kLB - 1) / kLB;
  const T* g = sizeof(T) == 4 ? reinterpret_cast<const T*>(s.g32l)
                              : reinterpret_cast<const T*>(s.g64);
  constexpr int WPB = kGridBT / 32;
  static_assert(WPB * 16 == kLB, "one warp per 16 rows of a block");
  // Shared memory: inv(L_bb) (pitch kPitch), then the block's right-hand side
  // (kLB), the warps' column partials of the backward step (WPB x kLB), and
  // the hand-off of the polling warp's result.
  const T* rinv = reinterpret_cast<const T*>(s.arena);
  T* red = reinterpret_cast<T*>(s.arena) + kLB * kPitch;
  T* cpart = red + kLB;
  volatile int* sready = reinterpret_cast<volatile int*>(cpart + WPB * kLB);
  static_assert((size_t(kLB) * kPitch + kLB) * sizeof(double) <= kPrSmemOff,
                "large_products would overwrite the resident inverse");
  static_assert((size_t(kLB) * kPitch + kLB + WPB * kLB) * sizeof(double) + sizeof(int) <=
                    kArenaBytes, "the solve's shared memory exceeds the arena");
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int j = blockIdx.x;
  auto bsz = [&](int b) { return min(kLB, n - b * kLB); };
  s.tri_gen += 1;
  const unsigned int gen_fwd = 2 * s.tri_gen - 1, gen_bwd = 2 * s.tri_gen;
  GridCtl* gc = s.gctl;
  // The polling warp's count of consecutive published blocks from c (dir +1
  // or -1, stopping before `end`), passed to the whole CTA; `none` when the
  // wait gave up (the solve then runs to its end on whatever is there, and the
  // sticky error reports it).
  auto ready_until = [&](int c, int dir, int end) {
    if (warp == 0) {
      const int k = flags_ready(gc, c, dir, end, dir > 0 ? gen_fwd : gen_bwd);
      if (lane == 0) *sready = k > 0 ? c + dir * k : end;
    }
    __syncthreads();
    const int r = *sready;
    __syncthreads();
    return r;
  };
  // Brings the 128 x 128 block of g at (row block rb, column block cb) into
  // L2 ahead of the step that has it on the chain between blocks (L_{j,j-1}
  // forward, L_{j+1,j} backward), one 128-byte line per request.
  auto prefetch_block = [&](int rb, int cb) {
    constexpr int kLines = kLB * int(sizeof(T)) / 128;  // lines per block row
    const int rows = bsz(rb);
    for (int e = threadIdx.x; e < rows * kLines; e += blockDim.x) {
      const T* p = g + size_t(rb * kLB + e / kLines) * npad + cb * kLB +
                   (e % kLines) * (128 / int(sizeof(T)));
      asm volatile("prefetch.global.L2 [%0];" ::"l"(p));
    }
  };
  QTQP_TIC();
  if (j < nb) {
    const int b0 = j * kLB, bs = bsz(j);
    const int r0 = 16 * warp;  // this warp's 16 rows of the block
    if (j > 1) prefetch_block(j, j - 1);
    // Forward: lane partials of rows r0 + r over columns lane + 32 q.
    T acc[16];
#pragma unroll
    for (int r = 0; r < 16; ++r) acc[r] = T(0);
    for (int c = 0; c < j;) {
      const int hi = ready_until(c, 1, j);
      for (; c < hi; ++c) {
        T z[4];
#pragma unroll
        for (int q = 0; q < 4; ++q) z[q] = __ldcg(w + c * kLB + lane + 32 * q);
        const T* lr = g + size_t(b0 + r0) * npad + c * kLB + lane;
#pragma unroll
        for (int r = 0; r < 16; ++r) {
          if (r0 + r < bs) {
#pragma unroll
            for (int q = 0; q < 4; ++q) acc[r] = fma(lr[size_t(r) * npad + 32 * q], z[q], acc[r]);
          }
        }
      }
    }
    // Sum the 16 rows over the warp: each exchange step sends half of the
    // values to the partner lane and keeps the other half, so lane l ends with
    // row rsel(l) (lanes l and l ^ 1 hold the same row).
#pragma unroll
    for (int half = 8, bit = 16; half >= 1; half >>= 1, bit >>= 1) {
      const bool up = (lane & bit) != 0;
#pragma unroll
      for (int q = 0; q < half; ++q) {
        const T send = up ? acc[q] : acc[q + half];
        const T keep = up ? acc[q + half] : acc[q];
        acc[q] = keep + __shfl_xor_sync(0xffffffffu, send, bit);
      }
    }
    acc[0] += __shfl_xor_sync(0xffffffffu, acc[0], 1);
    const int rsel = ((lane >> 4) & 1) * 8 + ((lane >> 3) & 1) * 4 + ((lane >> 2) & 1) * 2 +
                     ((lane >> 1) & 1);
    if ((lane & 1) == 0 && r0 + rsel < bs) red[r0 + rsel] = v[b0 + r0 + rsel] - acc[0];
    __syncthreads();
    {
      // z_r = sum_{c <= r} inv(L_jj)_rc u_c by two threads per row: the
      // half-warp h of warp w takes rows 16 w .. 16 w + 15 and the columns
      // c = h (mod 2) (distinct banks across the half-warp, u_c broadcast).
      const int r = r0 + (lane & 15), h = lane >> 4;
      const T* ir = rinv + r * kPitch;
      T a0 = T(0), a1 = T(0), a2 = T(0), a3 = T(0);
      if (r < bs) {
        int c = h;
        for (; c + 6 <= r; c += 8) {
          a0 = fma(ir[c + 0], red[c + 0], a0);
          a1 = fma(ir[c + 2], red[c + 2], a1);
          a2 = fma(ir[c + 4], red[c + 4], a2);
          a3 = fma(ir[c + 6], red[c + 6], a3);
        }
        for (; c <= r; c += 2) a0 = fma(ir[c], red[c], a0);
      }
      T zr = (a0 + a1) + (a2 + a3);
      zr += __shfl_xor_sync(0xffffffffu, zr, 16);
      if (h == 0 && r < bs) {
        w[b0 + r] = zr;
        __threadfence();
      }
    }
    __syncthreads();
    if (threadIdx.x == 0) flag_publish(gc, j, gen_fwd);
  }
  QTQP_TOC(kPhLgFwd);
  QTQP_RETIC();
  if (j < nb) {
    const int b0 = j * kLB, bs = bsz(j);
    const int r0 = 16 * warp;
    if (j + 1 < nb) prefetch_block(j + 1, j);
    // Backward: lane partials of columns lane + 32 q of block j over this
    // warp's 16 rows of every later block.
    T acc[4];
#pragma unroll
    for (int q = 0; q < 4; ++q) acc[q] = T(0);
    for (int c = nb - 1; c > j;) {
      const int lo = ready_until(c, -1, j);
      for (; c > lo; --c) {
        const int cb0 = c * kLB, cbs = bsz(c);
#pragma unroll
        for (int r = 0; r < 16; ++r) {
          if (r0 + r < cbs) {
            const T xi = __ldcg(v + cb0 + r0 + r);
            const T* lr = g + size_t(cb0 + r0 + r) * npad + b0 + lane;
#pragma unroll
            for (int q = 0; q < 4; ++q) acc[q] = fma(lr[32 * q], xi, acc[q]);
          }
        }
      }
    }
#pragma unroll
    for (int q = 0; q < 4; ++q) cpart[warp * kLB + lane + 32 * q] = acc[q];
    __syncthreads();
    if (int(threadIdx.x) < bs) {
      const int k = threadIdx.x;
      T t = T(0);
#pragma unroll
      for (int q = 0; q < WPB; ++q) t += cpart[q * kLB + k];
      red[k] = w[b0 + k] - t;  // w_j: this CTA's forward result
    }
    __syncthreads();
    {
      // x_r = sum_{c >= r} inv(L_jj)_cr u_c, two threads per row as forward
      // (half-warp h: the columns c >= r with c = r + h (mod 2)).
      const int r = r0 + (lane & 15), h = lane >> 4;
      T a0 = T(0), a1 = T(0), a2 = T(0), a3 = T(0);
      if (r < bs) {
        int c = r + h;
        for (; c + 6 < bs; c += 8) {
          a0 = fma(rinv[(c + 0) * kPitch + r], red[c + 0], a0);
          a1 = fma(rinv[(c + 2) * kPitch + r], red[c + 2], a1);
          a2 = fma(rinv[(c + 4) * kPitch + r], red[c + 4], a2);
          a3 = fma(rinv[(c + 6) * kPitch + r], red[c + 6], a3);
        }
        for (; c < bs; c += 2) a0 = fma(rinv[c * kPitch + r], red[c], a0);
      }
      T xr = (a0 + a1) + (a2 + a3);
      xr += __shfl_xor_sync(0xffffffffu, xr, 16);
      if (h == 0 && r < bs) {
        v[b0 + r] = xr;
        __threadfence();
      }
    }
    __syncthreads();
    if (threadIdx.x == 0) flag_publish(gc, j, gen_bwd);
  }
  s.sync();
  QTQP_TOC(kPhLgBwd);
}

}  // namespace qtqp
