// BF16 tensor-core GEMM of the warm-start MLP's forward pass (no reference
// counterpart): C = A B^T (+ bias per column) (ReLU), A (M x K) and B (N x K)
// BF16 row-major (both K-major), FP32 accumulation in TMEM, C in FP32 and,
// optionally, a BF16 copy that is the next layer's A.
//
// One CTA per 128 x 128 tile of C: warp 0 (one lane) loads 128 x 64 tiles of
// A and B with TMA (128-byte swizzle) into a 3-stage ring, warp 1 (one lane)
// issues tcgen05.mma kind::f16 (M = N = 128, K = 16 per instruction), and the
// four warps drain TMEM (warp w: rows 32w .. 32w + 31).  Rows of A / B past
// M / N and columns past K load as zeros (TMA out-of-bounds fill); stores
// are guarded.  Every wait is bounded: a wait that gives up sets *err, the
// producer waits (bounded) for the stages it issued, and the CTA frees its
// TMEM and returns.
#include <cuda_bf16.h>

#include <algorithm>

#include "common.cuh"
#include "tc_common.cuh"

namespace qtqp {

constexpr int kBfTile = 128;                               // BM = BN
constexpr int kBfBK = 64;                                  // BF16 per 128-byte row
constexpr int kBfStages = 3;
constexpr uint32_t kBfTileBytes = kBfTile * kBfBK * 2;     // 16 KB
constexpr uint32_t kBfStageBytes = 2 * kBfTileBytes;       // A, B
constexpr size_t kBfSmem = 1024 + kBfStages * kBfStageBytes + 256;

__global__ void __launch_bounds__(128, 1)
    mlp_gemm_bf16_kernel(const __grid_constant__ CUtensorMap map_a,
                         const __grid_constant__ CUtensorMap map_b, int M, int N, int k_tiles,
                         float* __restrict__ c, int ldc, const float* __restrict__ bias,
                         int relu, __nv_bfloat16* __restrict__ c16, int ldc16, int* err) {
  extern __shared__ uint8_t smem_raw[];
  uint8_t* base = reinterpret_cast<uint8_t*>(
      (reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~uintptr_t(1023));
  uint64_t* full = reinterpret_cast<uint64_t*>(base + kBfStages * kBfStageBytes);
  uint64_t* empty = full + kBfStages;
  uint64_t* done = empty + kBfStages;
  uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(done + 1);
  int* failed = reinterpret_cast<int*>(tmem_slot + 1);
  int* consumed = failed + 1;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int tm = blockIdx.y, tn = blockIdx.x;

  if (threadIdx.x == 0) {
    for (int s = 0; s < kBfStages; ++s) {
      tc::mbar_init(&full[s], 1);
      tc::mbar_init(&empty[s], 1);
    }
    tc::mbar_init(done, 1);
    *failed = 0;
    *consumed = 0;
    tc::mbar_fence_init();
    tc::tma_prefetch_desc(&map_a);
    tc::tma_prefetch_desc(&map_b);
  }
  if (warp == 2) tc::tmem_alloc(tmem_slot, kBfTile);
  tc::fence_before_sync();
  __syncthreads();
  tc::fence_after_sync();
  const uint32_t tmem = *tmem_slot;

  int issued = 0;  // producer: stages loaded
  if (warp == 0 && lane == 0) {
    for (int kt = 0; kt < k_tiles; ++kt) {
      const int s = kt % kBfStages;
      if (kt >= kBfStages && !tc::mbar_wait(&empty[s], ((kt / kBfStages) - 1) & 1)) {
        atomicExch(failed, 1);
        break;
      }
      uint8_t* st = base + s * kBfStageBytes;
      tc::mbar_arrive_expect_tx(&full[s], kBfStageBytes);
      tc::tma_load_2d(st, &map_a, kt * kBfBK, tm * kBfTile, &full[s]);
      tc::tma_load_2d(st + kBfTileBytes, &map_b, kt * kBfBK, tn * kBfTile, &full[s]);
      ++issued;
    }
  } else if (warp == 1 && lane == 0) {
    constexpr uint32_t idesc = tc::idesc_f32acc(kBfTile, kBfTile, true);
    int kt = 0;
    for (; kt < k_tiles; ++kt) {
      const int s = kt % kBfStages;
      if (!tc::mbar_wait(&full[s], (kt / kBfStages) & 1)) {
        atomicExch(failed, 1);
        break;
      }
      tc::fence_after_sync();
      const uint32_t a = tc::smem_u32(base + s * kBfStageBytes);
      const uint32_t b = a + kBfTileBytes;
#pragma unroll
      for (int kk = 0; kk < kBfBK / 16; ++kk) {
        const uint32_t off = kk * 32;  // 16 BF16 = 32 bytes along K
        tc::mma_f16(tmem, tc::desc_kmajor_sw128(a + off), tc::desc_kmajor_sw128(b + off), idesc,
                    (kt | kk) != 0);
      }
      tc::mma_commit(&empty[s]);
    }
    *consumed = kt;
    tc::mma_commit(done);
  }
  __syncwarp();
  if (!tc::mbar_wait(done, 0)) atomicExch(failed, 1);
  tc::fence_after_sync();
  __syncthreads();
  if (*failed != 0) {
    // Stages the producer issued that the MMA issuer never waited for:
    // wait (bounded) for their copies before the CTA leaves.
    if (warp == 0 && lane == 0) {
      for (int kt = *consumed; kt < issued; ++kt)
        if (!tc::mbar_wait(&full[kt % kBfStages], (kt / kBfStages) & 1)) break;
    }
    if (threadIdx.x == 0) atomicExch(err, 1);
  } else {
    const int row = tm * kBfTile + warp * 32 + lane;
#pragma unroll 1
    for (int c0 = 0; c0 < kBfTile; c0 += 32) {
      float v[32];
      tc::tmem_ld32(tmem + (uint32_t(warp * 32) << 16) + uint32_t(c0), v);
      if (row < M) {
        const int col0 = tn * kBfTile + c0;
#pragma unroll
        for (int q = 0; q < 32; ++q) {
          const int col = col0 + q;
          if (col < N) {
            float x = v[q];
            if (bias != nullptr) x += bias[col];
            if (relu) x = fmaxf(x, 0.0f);
            c[size_t(row) * ldc + col] = x;
            if (c16 != nullptr) c16[size_t(row) * ldc16 + col] = __float2bfloat16_rn(x);
          }
        }
      }
    }
  }
  tc::fence_before_sync();
  __syncthreads();
  if (warp == 2) {
    tc::fence_after_sync();
    tc::tmem_dealloc(tmem, kBfTile);
  }
}

// FP32 -> BF16 (round to nearest even), optionally transposed: dst is cols x
// rows when transpose != 0.
__global__ void to_bf16_kernel(const float* __restrict__ src, int rows, int cols, int transpose,
                               __nv_bfloat16* __restrict__ dst) {
  const size_t total = size_t(rows) * cols;
  for (size_t e = blockIdx.x * size_t(blockDim.x) + threadIdx.x; e < total;
       e += size_t(gridDim.x) * blockDim.x) {
    const int r = int(e / cols), cc = int(e % cols);
    const __nv_bfloat16 v = __float2bfloat16_rn(src[e]);
    if (transpose) {
      dst[size_t(cc) * rows + r] = v;
    } else {
      dst[e] = v;
    }
  }
}

int make_map_bf16(CUtensorMap* map, const void* ptr, int rows, int cols);

}  // namespace qtqp

using namespace qtqp;

extern "C" int qtqp_mlp_gemm_bf16(int32_t M, int32_t N, int32_t K, const void* d_a,
                                  const void* d_bt, float* d_c, int32_t ldc, const float* d_bias,
                                  int32_t relu, void* d_c16, int32_t ldc16, int32_t* d_err,
                                  void* stream) {
  if (M < 1 || N < 1 || K < 1 || K % 8 != 0 || d_a == nullptr || d_bt == nullptr ||
      d_c == nullptr || d_err == nullptr || ldc < N || (d_c16 != nullptr && ldc16 < N))
    return fail(QTQP_ERR_BAD_ARG, "qtqp_mlp_gemm_bf16: bad sizes (K a multiple of 8), leading "
                                  "dimensions or pointers");
  if ((reinterpret_cast<uintptr_t>(d_a) | reinterpret_cast<uintptr_t>(d_bt)) & 15)
    return fail(QTQP_ERR_BAD_ARG, "qtqp_mlp_gemm_bf16: operands must be 16-byte aligned");
  CUtensorMap ma, mb;
  int rc = make_map_bf16(&ma, d_a, M, K);
  if (rc) return rc;
  rc = make_map_bf16(&mb, d_bt, N, K);
  if (rc) return rc;
  rc = cuda_check(cudaFuncSetAttribute(mlp_gemm_bf16_kernel,
                                       cudaFuncAttributeMaxDynamicSharedMemorySize, int(kBfSmem)),
                  "cudaFuncSetAttribute(mlp_gemm_bf16_kernel)");
  if (rc) return rc;
  const dim3 grid((N + kBfTile - 1) / kBfTile, (M + kBfTile - 1) / kBfTile);
  mlp_gemm_bf16_kernel<<<grid, 128, kBfSmem, static_cast<cudaStream_t>(stream)>>>(
      ma, mb, M, N, (K + kBfBK - 1) / kBfBK, d_c, ldc, d_bias, relu,
      static_cast<__nv_bfloat16*>(d_c16), ldc16, d_err);
  return cuda_check(cudaGetLastError(), "mlp_gemm_bf16_kernel launch");
}

extern "C" int qtqp_mlp_to_bf16(const float* d_src, int32_t rows, int32_t cols,
                                int32_t transpose, void* d_dst, void* stream) {
  if (rows < 0 || cols < 0 || (size_t(rows) * cols > 0 && (d_src == nullptr || d_dst == nullptr)))
    return fail(QTQP_ERR_BAD_ARG, "qtqp_mlp_to_bf16: bad arguments");
  const size_t total = size_t(rows) * cols;
  if (total == 0) return QTQP_OK;
  const int grid = int(std::min<size_t>((total + 255) / 256, 148 * 16));
  to_bf16_kernel<<<grid, 256, 0, static_cast<cudaStream_t>(stream)>>>(
      d_src, rows, cols, transpose, static_cast<__nv_bfloat16*>(d_dst));
  return cuda_check(cudaGetLastError(), "to_bf16_kernel launch");
}
