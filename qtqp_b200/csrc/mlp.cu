// Kernels of the warm-start MLP (no reference counterpart): a tiled FP32 GEMM
// with fused bias and ReLU, the ReLU backward mask, column sums (bias
// gradients), the MSE gradient with its loss, the hinge term on the sign of
// the inequality outputs, Adam, and the decoder that
// turns network outputs into per-instance warm starts for the banded solver.
#include <algorithm>
#include <cmath>

#include "common.cuh"

namespace qtqp {

constexpr int kTile = 64;         // C tile is kTile x kTile
constexpr int kTk = 16;           // K slice staged in shared memory
constexpr int kGemmThreads = 256; // 16 x 16 threads, 4 x 4 outputs each

// C = alpha op(A) op(B) + beta C (+ bias[col]) (ReLU).  op(A)(r, k) is
// A[r * lda + k], or A[k * lda + r] when trans_a; op(B)(k, c) is
// B[k * ldb + c], or B[c * ldb + k] when trans_b.  Both operand slices are
// staged k-major in shared memory, so the inner product reads two float4
// rows per k.
__global__ void __launch_bounds__(kGemmThreads)
gemm_kernel(int M, int N, int K, float alpha, const float* __restrict__ a, int lda, int ta,
            const float* __restrict__ b, int ldb, int tb, float beta, float* __restrict__ c,
            int ldc, const float* __restrict__ bias, int relu) {
  __shared__ __align__(16) float as[kTk][kTile];
  __shared__ __align__(16) float bs[kTk][kTile];
  const int tid = threadIdx.x;
  const int tx = tid & 15, ty = tid >> 4;
  const int row0 = blockIdx.y * kTile, col0 = blockIdx.x * kTile;
  float acc[4][4];
#pragma unroll
  for (int i = 0; i < 4; ++i)
#pragma unroll
    for (int j = 0; j < 4; ++j) acc[i][j] = 0.0f;
  for (int k0 = 0; k0 < K; k0 += kTk) {
    // 64 x 16 elements of each operand, 4 per thread.
#pragma unroll
    for (int t = 0; t < 4; ++t) {
      const int e = tid + t * kGemmThreads;  // 0 .. 1023
      int r, kk;
      if (ta) {  // consecutive threads walk r (contiguous in A)
        r = e & 63;
        kk = e >> 6;
      } else {   // consecutive threads walk k (contiguous in A)
        kk = e & 15;
        r = e >> 4;
      }
      const int gr = row0 + r, gk = k0 + kk;
      float v = 0.0f;
      if (gr < M && gk < K) v = ta ? a[size_t(gk) * lda + gr] : a[size_t(gr) * lda + gk];
      as[kk][r] = v;
      int cc, kb;
      if (tb) {
        kb = e & 15;
        cc = e >> 4;
      } else {
        cc = e & 63;
        kb = e >> 6;
      }
      const int gc = col0 + cc, gkb = k0 + kb;
      float w = 0.0f;
      if (gc < N && gkb < K) w = tb ? b[size_t(gc) * ldb + gkb] : b[size_t(gkb) * ldb + gc];
      bs[kb][cc] = w;
    }
    __syncthreads();
#pragma unroll
    for (int kk = 0; kk < kTk; ++kk) {
      const float4 av = *reinterpret_cast<const float4*>(&as[kk][ty * 4]);
      const float4 bv = *reinterpret_cast<const float4*>(&bs[kk][tx * 4]);
      const float ar[4] = {av.x, av.y, av.z, av.w};
      const float br[4] = {bv.x, bv.y, bv.z, bv.w};
#pragma unroll
      for (int i = 0; i < 4; ++i)
#pragma unroll
        for (int j = 0; j < 4; ++j) acc[i][j] = fmaf(ar[i], br[j], acc[i][j]);
    }
    __syncthreads();
  }
#pragma unroll
  for (int i = 0; i < 4; ++i) {
    const int r = row0 + ty * 4 + i;
    if (r >= M) continue;
#pragma unroll
    for (int j = 0; j < 4; ++j) {
      const int cc = col0 + tx * 4 + j;
      if (cc >= N) continue;
      float v = alpha * acc[i][j];
      if (beta != 0.0f) v = fmaf(beta, c[size_t(r) * ldc + cc], v);
      if (bias != nullptr) v += bias[cc];
      if (relu) v = fmaxf(v, 0.0f);
      c[size_t(r) * ldc + cc] = v;
    }
  }
}

__global__ void relu_grad_kernel(float* __restrict__ dh, const float* __restrict__ h,
                                 int64_t count) {
  for (int64_t i = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; i < count;
       i += int64_t(gridDim.x) * blockDim.x)
    if (!(h[i] > 0.0f)) dh[i] = 0.0f;
}

// One thread per column; consecutive threads read consecutive columns.
__global__ void colsum_kernel(const float* __restrict__ d, int rows, int cols,
                              float* __restrict__ db) {
  const int j = blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= cols) return;
  float t = 0.0f;
  for (int i = 0; i < rows; ++i) t += d[size_t(i) * cols + j];
  db[j] = t;
}

// dy = 2 (y - t) / count; the squared errors are summed per block in FP64
// and added to *loss (zeroed by the caller's memset on the same stream).
__global__ void mse_grad_kernel(const float* __restrict__ y, const float* __restrict__ t,
                                int64_t count, float* __restrict__ dy, double* loss) {
  __shared__ double part[32];
  double acc = 0.0;
  const float scale = 2.0f / float(count);
  for (int64_t i = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; i < count;
       i += int64_t(gridDim.x) * blockDim.x) {
    const float e = y[i] - t[i];
    dy[i] = scale * e;
    acc += double(e) * double(e);
  }
  for (int off = 16; off > 0; off >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, off);
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  if (lane == 0) part[warp] = acc;
  __syncthreads();
  if (warp == 0) {
    acc = lane < int(blockDim.x >> 5) ? part[lane] : 0.0;
    for (int off = 16; off > 0; off >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, off);
    if (lane == 0) atomicAdd(loss, acc);
  }
}

// Hinge on the sign of the inequality outputs, added to dy after the MSE
// gradient: for columns [col0, cols) of a rows x cols output, with the
// column's decision point zero[j] (the standardised value of y_i - s_i = 0)
// and the target's side sign = +1 (t > zero) or -1,
//   loss += weight * mean relu(margin - sign (y - zero))  (as a sum, see below),
//   dy   += -weight * sign * [margin - sign (y - zero) > 0] / (rows (cols - col0)).
__global__ void hinge_grad_kernel(const float* __restrict__ y, const float* __restrict__ t,
                                  int rows, int cols, int col0, const float* __restrict__ zero,
                                  float weight, float margin, float* __restrict__ dy,
                                  double* loss) {
  __shared__ double part[32];
  const int w = cols - col0;
  const int64_t total = int64_t(rows) * w;
  const float inv = 1.0f / float(total);
  double acc = 0.0;
  for (int64_t e = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; e < total;
       e += int64_t(gridDim.x) * blockDim.x) {
    const int r = int(e / w), j = col0 + int(e % w);
    const size_t i = size_t(r) * cols + j;
    const float z0 = zero[j - col0];
    const float sg = t[i] > z0 ? 1.0f : -1.0f;
    const float h = margin - sg * (y[i] - z0);
    if (h > 0.0f) {
      dy[i] -= weight * sg * inv;
      acc += double(h);
    }
  }
  for (int off = 16; off > 0; off >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, off);
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  if (lane == 0) part[warp] = acc;
  __syncthreads();
  if (warp == 0) {
    acc = lane < int(blockDim.x >> 5) ? part[lane] : 0.0;
    for (int off = 16; off > 0; off >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, off);
    // *loss holds a sum over all rows x cols outputs (the MSE kernel's sum of
    // squares); scaled so that loss / (rows cols) = mse + weight mean(h).
    if (lane == 0)
      atomicAdd(loss, double(weight) * acc * (double(rows) * cols / double(total)));
  }
}

__global__ void adam_kernel(float* __restrict__ p, const float* __restrict__ g,
                            float* __restrict__ m, float* __restrict__ v, int64_t count, float lr,
                            float b1, float b2, float eps, float c1, float c2) {
  for (int64_t i = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; i < count;
       i += int64_t(gridDim.x) * blockDim.x) {
    const float gi = g[i];
    const float mi = b1 * m[i] + (1.0f - b1) * gi;
    const float vi = b2 * v[i] + (1.0f - b2) * gi * gi;
    m[i] = mi;
    v[i] = vi;
    p[i] -= lr * (mi / c1) / (sqrtf(vi / c2) + eps);
  }
}

// v = pred * scale + shift per coordinate.  x = v[0:n], y_eq = v[n:n+z];
// inequality row i carries v_i = y_i - s_i, decoded as y_i = max(v_i, 0) and
// active[i] = (v_i > threshold).
__global__ void decode_kernel(const float* __restrict__ pred, const double* __restrict__ scale,
                              const double* __restrict__ shift, int n, int m, int z, int count,
                              double threshold, double* __restrict__ x_out,
                              double* __restrict__ y_out, unsigned char* __restrict__ active) {
  const int N = n + m;
  const size_t total = size_t(count) * N;
  for (size_t e = blockIdx.x * size_t(blockDim.x) + threadIdx.x; e < total;
       e += size_t(gridDim.x) * blockDim.x) {
    const int inst = int(e / N), k = int(e % N);
    const double v = double(pred[e]) * scale[k] + shift[k];
    if (k < n) {
      x_out[size_t(inst) * n + k] = v;
    } else {
      const int i = k - n;
      y_out[size_t(inst) * m + i] = (i < z) ? v : fmax(v, 0.0);
      active[size_t(inst) * m + i] = (i < z || v > threshold) ? 1 : 0;
    }
  }
}

static int grid_for(size_t count) {
  return int(std::max<size_t>(1, std::min<size_t>((count + 255) / 256, 148 * 16)));
}

}  // namespace qtqp

using namespace qtqp;

extern "C" int qtqp_mlp_gemm(int32_t M, int32_t N, int32_t K, float alpha, const float* d_a,
                             int32_t lda, int32_t trans_a, const float* d_b, int32_t ldb,
                             int32_t trans_b, float beta, float* d_c, int32_t ldc,
                             const float* d_bias, int32_t relu, void* stream) {
  if (M < 0 || N < 0 || K < 0 || d_a == nullptr || d_b == nullptr || d_c == nullptr ||
      ldc < N || lda < (trans_a ? M : K) || ldb < (trans_b ? K : N))
    return fail(QTQP_ERR_BAD_ARG, "qtqp_mlp_gemm: bad sizes, leading dimensions or pointers");
  if (M == 0 || N == 0) return QTQP_OK;
  dim3 grid((N + kTile - 1) / kTile, (M + kTile - 1) / kTile);
  gemm_kernel<<<grid, kGemmThreads, 0, static_cast<cudaStream_t>(stream)>>>(
      M, N, K, alpha, d_a, lda, trans_a, d_b, ldb, trans_b, beta, d_c, ldc, d_bias, relu);
  return cuda_check(cudaGetLastError(), "gemm_kernel launch");
}

extern "C" int qtqp_mlp_relu_grad(float* d_dh, const float* d_h, int64_t count, void* stream) {
  if (count < 0 || (count > 0 && (d_dh == nullptr || d_h == nullptr)))
    return fail(QTQP_ERR_BAD_ARG, "qtqp_mlp_relu_grad: bad arguments");
  if (count == 0) return QTQP_OK;
  relu_grad_kernel<<<grid_for(count), 256, 0, static_cast<cudaStream_t>(stream)>>>(d_dh, d_h,
                                                                                   count);
  return cuda_check(cudaGetLastError(), "relu_grad_kernel launch");
}

extern "C" int qtqp_mlp_colsum(const float* d_d, int32_t rows, int32_t cols, float* d_db,
                               void* stream) {
  if (rows < 0 || cols < 0 || (cols > 0 && (d_d == nullptr || d_db == nullptr)))
    return fail(QTQP_ERR_BAD_ARG, "qtqp_mlp_colsum: bad arguments");
  if (cols == 0) return QTQP_OK;
  colsum_kernel<<<(cols + 255) / 256, 256, 0, static_cast<cudaStream_t>(stream)>>>(d_d, rows,
                                                                                   cols, d_db);
  return cuda_check(cudaGetLastError(), "colsum_kernel launch");
}

extern "C" int qtqp_mlp_mse_grad(const float* d_y, const float* d_t, int64_t count, float* d_dy,
                                 double* d_loss, void* stream) {
  if (count < 1 || d_y == nullptr || d_t == nullptr || d_dy == nullptr || d_loss == nullptr)
    return fail(QTQP_ERR_BAD_ARG, "qtqp_mlp_mse_grad: bad arguments");
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  int rc = cuda_check(cudaMemsetAsync(d_loss, 0, sizeof(double), st), "cudaMemsetAsync");
  if (rc) return rc;
  mse_grad_kernel<<<grid_for(count), 256, 0, st>>>(d_y, d_t, count, d_dy, d_loss);
  return cuda_check(cudaGetLastError(), "mse_grad_kernel launch");
}

extern "C" int qtqp_mlp_adam(float* d_p, const float* d_g, float* d_m, float* d_v, int64_t count,
                             float lr, float beta1, float beta2, float eps, int32_t step,
                             void* stream) {
  if (count < 0 || step < 1 || d_p == nullptr || d_g == nullptr || d_m == nullptr ||
      d_v == nullptr)
    return fail(QTQP_ERR_BAD_ARG, "qtqp_mlp_adam: bad arguments");
  if (count == 0) return QTQP_OK;
  const float c1 = 1.0f - float(std::pow(double(beta1), double(step)));
  const float c2 = 1.0f - float(std::pow(double(beta2), double(step)));
  adam_kernel<<<grid_for(count), 256, 0, static_cast<cudaStream_t>(stream)>>>(
      d_p, d_g, d_m, d_v, count, lr, beta1, beta2, eps, c1, c2);
  return cuda_check(cudaGetLastError(), "adam_kernel launch");
}

extern "C" int qtqp_mlp_decode(const float* d_pred, const double* d_scale, const double* d_shift,
                               int32_t n, int32_t m, int32_t z, int32_t count, double threshold,
                               double* d_x, double* d_y, unsigned char* d_active, void* stream) {
  if (n < 1 || m < 1 || z < 0 || z > m || count < 0)
    return fail(QTQP_ERR_BAD_ARG, "qtqp_mlp_decode: bad sizes");
  if (count == 0) return QTQP_OK;
  if (d_pred == nullptr || d_scale == nullptr || d_shift == nullptr || d_x == nullptr ||
      d_y == nullptr || d_active == nullptr)
    return fail(QTQP_ERR_BAD_ARG, "qtqp_mlp_decode: null pointer");
  decode_kernel<<<grid_for(size_t(count) * (n + m)), 256, 0, static_cast<cudaStream_t>(stream)>>>(
      d_pred, d_scale, d_shift, n, m, z, count, threshold, d_x, d_y, d_active);
  return cuda_check(cudaGetLastError(), "decode_kernel launch");
}

extern "C" int qtqp_mlp_hinge_grad(const float* d_y, const float* d_t, int32_t rows,
                                   int32_t cols, int32_t col0, const float* d_zero, float weight,
                                   float margin, float* d_dy, double* d_loss, void* stream) {
  if (rows < 1 || cols < 1 || col0 < 0 || col0 >= cols || d_y == nullptr || d_t == nullptr ||
      d_zero == nullptr || d_dy == nullptr || d_loss == nullptr)
    return fail(QTQP_ERR_BAD_ARG, "qtqp_mlp_hinge_grad: bad arguments");
  hinge_grad_kernel<<<grid_for(size_t(rows) * (cols - col0)), 256, 0,
                      static_cast<cudaStream_t>(stream)>>>(d_y, d_t, rows, cols, col0, d_zero,
                                                            weight, margin, d_dy, d_loss);
  return cuda_check(cudaGetLastError(), "hinge_grad_kernel launch");
}
