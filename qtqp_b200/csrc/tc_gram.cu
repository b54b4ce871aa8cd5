// Tensor-core Gram product C = X X^T (lower 128 x 128 tiles) on tcgen05 with
// TF32 inputs and FP32 accumulation in TMEM, for the large dense KKT
// factorisation (the A^T D A term of solvers_dense.py:99-116 with
// X = (diag(1/sqrt(Ry)) A)^T).
//
// X is n x k FP32, row-major (K-major for both MMA operands).  With split = 1
// the caller passes X = hi + lo, hi = X rounded to TF32 and lo = X - hi, and
// the kernel accumulates hi hi^T + hi lo^T + lo hi^T: three TF32 products
// that together carry FP32-level accuracy (the lo lo^T term is below FP32
// rounding).  With split = 0 only hi hi^T is formed (plain TF32).
//
// One CTA per lower tile; 4 warps: warp 0 lane 0 issues the TMA loads of a
// 3-stage shared-memory ring (128-byte swizzle), warp 1 lane 0 issues the
// MMAs (M = N = 128, K = 8 per instruction, 4 per 32-wide K slice), warp 2
// owns the 128-column TMEM accumulator, and all four warps read TMEM back in
// the epilogue (warp w owns accumulator rows 32w .. 32w + 31).
#include <cudaTypedefs.h>

#include <algorithm>
#include <mutex>

#include "common.cuh"
#include "tc_common.cuh"

namespace qtqp {

constexpr int kGramTile = 128;                               // BM = BN
constexpr int kGramBK = 32;                                  // FP32 per 128-byte row
constexpr int kGramStages = 3;
constexpr uint32_t kGramTileBytes = kGramTile * kGramBK * 4;  // 16 KB
constexpr uint32_t kGramStageBytes = 4 * kGramTileBytes;      // A hi, B hi, A lo, B lo
constexpr size_t kGramSmem = 1024 + kGramStages * kGramStageBytes + 256;

__global__ void __launch_bounds__(128, 1)
    gram_tf32_kernel(const __grid_constant__ CUtensorMap map_hi,
                     const __grid_constant__ CUtensorMap map_lo, int k_tiles, int split,
                     float* __restrict__ c, int ldc, int* err) {
  extern __shared__ uint8_t smem_raw[];
  uint8_t* base = reinterpret_cast<uint8_t*>(
      (reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~uintptr_t(1023));
  uint64_t* full = reinterpret_cast<uint64_t*>(base + kGramStages * kGramStageBytes);
  uint64_t* empty = full + kGramStages;
  uint64_t* done = empty + kGramStages;
  uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(done + 1);
  int* failed = reinterpret_cast<int*>(tmem_slot + 1);
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;

  // Lower-triangular tile (ti >= tj) of this CTA.
  const int b = blockIdx.x;
  int ti = 0;
  while ((ti + 1) * (ti + 2) / 2 <= b) ++ti;
  const int tj = b - ti * (ti + 1) / 2;

  if (threadIdx.x == 0) {
    for (int s = 0; s < kGramStages; ++s) {
      tc::mbar_init(&full[s], 1);
      tc::mbar_init(&empty[s], 1);
    }
    tc::mbar_init(done, 1);
    *failed = 0;
    tc::mbar_fence_init();
    tc::tma_prefetch_desc(&map_hi);
    if (split) tc::tma_prefetch_desc(&map_lo);
  }
  if (warp == 2) tc::tmem_alloc(tmem_slot, kGramTile);
  tc::fence_before_sync();
  __syncthreads();
  tc::fence_after_sync();
  const uint32_t tmem = *tmem_slot;

  if (warp == 0 && lane == 0) {
    // Producer: stage s is reused once the MMAs that read it have completed.
    const uint32_t bytes = (split ? 4u : 2u) * kGramTileBytes;
    for (int kt = 0; kt < k_tiles; ++kt) {
      const int s = kt % kGramStages;
      if (kt >= kGramStages && !tc::mbar_wait(&empty[s], ((kt / kGramStages) - 1) & 1)) {
        atomicExch(failed, 1);
        break;
      }
      uint8_t* st = base + s * kGramStageBytes;
      tc::mbar_arrive_expect_tx(&full[s], bytes);
      tc::tma_load_2d(st, &map_hi, kt * kGramBK, ti * kGramTile, &full[s]);
      tc::tma_load_2d(st + kGramTileBytes, &map_hi, kt * kGramBK, tj * kGramTile, &full[s]);
      if (split) {
        tc::tma_load_2d(st + 2 * kGramTileBytes, &map_lo, kt * kGramBK, ti * kGramTile,
                        &full[s]);
        tc::tma_load_2d(st + 3 * kGramTileBytes, &map_lo, kt * kGramBK, tj * kGramTile,
                        &full[s]);
      }
    }
  } else if (warp == 1 && lane == 0) {
    // MMA issuer.
    constexpr uint32_t idesc = tc::idesc_f32acc(kGramTile, kGramTile, false);
    for (int kt = 0; kt < k_tiles; ++kt) {
      const int s = kt % kGramStages;
      if (!tc::mbar_wait(&full[s], (kt / kGramStages) & 1)) {
        atomicExch(failed, 1);
        break;
      }
      tc::fence_after_sync();
      const uint32_t a_hi = tc::smem_u32(base + s * kGramStageBytes);
      const uint32_t b_hi = a_hi + kGramTileBytes;
      const uint32_t a_lo = a_hi + 2 * kGramTileBytes;
      const uint32_t b_lo = a_hi + 3 * kGramTileBytes;
#pragma unroll
      for (int kk = 0; kk < kGramBK / 8; ++kk) {
        const uint32_t off = kk * 32;  // 8 TF32 = 32 bytes along K
        tc::mma_tf32(tmem, tc::desc_kmajor_sw128(a_hi + off), tc::desc_kmajor_sw128(b_hi + off),
                     idesc, (kt | kk) != 0);
        if (split) {
          tc::mma_tf32(tmem, tc::desc_kmajor_sw128(a_hi + off),
                       tc::desc_kmajor_sw128(b_lo + off), idesc, 1);
          tc::mma_tf32(tmem, tc::desc_kmajor_sw128(a_lo + off),
                       tc::desc_kmajor_sw128(b_hi + off), idesc, 1);
        }
      }
      tc::mma_commit(&empty[s]);
    }
    tc::mma_commit(done);
  }
  __syncwarp();

  // Epilogue: TMEM -> registers -> global (row = lane of the warp's quarter).
  if (!tc::mbar_wait(done, 0)) atomicExch(failed, 1);
  tc::fence_after_sync();
  __syncthreads();
  if (*failed == 0) {
    const int row = ti * kGramTile + warp * 32 + lane;
    float* crow = c + size_t(row) * ldc + size_t(tj) * kGramTile;
#pragma unroll 1
    for (int c0 = 0; c0 < kGramTile; c0 += 32) {
      float v[32];
      tc::tmem_ld32(tmem + (uint32_t(warp * 32) << 16) + uint32_t(c0), v);
#pragma unroll
      for (int q = 0; q < 32; q += 4)
        *reinterpret_cast<float4*>(crow + c0 + q) = make_float4(v[q], v[q + 1], v[q + 2], v[q + 3]);
    }
  } else if (threadIdx.x == 0) {
    atomicExch(err, 1);
  }
  tc::fence_before_sync();
  __syncthreads();
  if (warp == 2) {
    tc::fence_after_sync();
    tc::tmem_dealloc(tmem, kGramTile);
  }
}

// ---- host ------------------------------------------------------------------
static PFN_cuTensorMapEncodeTiled_v12000 encode_fn() {
  static PFN_cuTensorMapEncodeTiled_v12000 fn = nullptr;
  static std::once_flag once;
  std::call_once(once, [] {
    void* p = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) ==
            cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      fn = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(p);
  });
  return fn;
}

// Row-major FP32 rows x cols (leading dimension ld elements) as 128 x 32 boxes
// with the 128-byte swizzle.
int make_map_f32(CUtensorMap* map, const float* ptr, int rows, int cols, int ld) {
  auto fn = encode_fn();
  if (fn == nullptr) return fail(QTQP_ERR_CUDA, "cuTensorMapEncodeTiled is unavailable");
  const cuuint64_t dims[2] = {cuuint64_t(cols), cuuint64_t(rows)};
  const cuuint64_t strides[1] = {cuuint64_t(ld) * 4};
  const cuuint32_t box[2] = {kGramBK, kGramTile};
  const cuuint32_t estr[2] = {1, 1};
  const CUresult r = fn(map, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 2, const_cast<float*>(ptr), dims,
                        strides, box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE,
                        CU_TENSOR_MAP_SWIZZLE_128B, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                        CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  if (r != CUDA_SUCCESS)
    return fail(QTQP_ERR_CUDA, "cuTensorMapEncodeTiled failed (code " + std::to_string(r) + ")");
  return QTQP_OK;
}

// Row-major BF16 rows x cols (leading dimension cols) as 128 x 64 boxes
// (128 bytes per row) with the 128-byte swizzle; columns past `cols` and rows
// past `rows` load as zeros.
int make_map_bf16(CUtensorMap* map, const void* ptr, int rows, int cols) {
  auto fn = encode_fn();
  if (fn == nullptr) return fail(QTQP_ERR_CUDA, "cuTensorMapEncodeTiled is unavailable");
  const cuuint64_t dims[2] = {cuuint64_t(cols), cuuint64_t(rows)};
  const cuuint64_t strides[1] = {cuuint64_t(cols) * 2};
  const cuuint32_t box[2] = {64, 128};
  const cuuint32_t estr[2] = {1, 1};
  const CUresult r = fn(map, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 2, const_cast<void*>(ptr), dims,
                        strides, box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE,
                        CU_TENSOR_MAP_SWIZZLE_128B, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                        CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  if (r != CUDA_SUCCESS)
    return fail(QTQP_ERR_CUDA, "cuTensorMapEncodeTiled (bf16) failed (code " + std::to_string(r) +
                                   ")");
  return QTQP_OK;
}

int launch_gram_tf32(int n, int k, const float* hi, const float* lo, int ld, float* c, int ldc,
                     int split, int* d_err, cudaStream_t st) {
  CUtensorMap mh, ml;
  int rc = make_map_f32(&mh, hi, n, k, ld);
  if (rc) return rc;
  rc = make_map_f32(&ml, split ? lo : hi, n, k, ld);
  if (rc) return rc;
  // Set on every call: the attribute belongs to the current device.
  rc = cuda_check(cudaFuncSetAttribute(gram_tf32_kernel,
                                       cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       int(kGramSmem)),
                  "cudaFuncSetAttribute(gram_tf32_kernel)");
  if (rc) return rc;
  const int nt = n / kGramTile;
  gram_tf32_kernel<<<nt * (nt + 1) / 2, 128, kGramSmem, st>>>(mh, ml, k / kGramBK, split, c, ldc,
                                                               d_err);
  return cuda_check(cudaGetLastError(), "gram_tf32_kernel launch");
}

}  // namespace qtqp

using namespace qtqp;

extern "C" int qtqp_tc_gram_f32(int32_t n, int32_t k, const float* d_hi, const float* d_lo,
                                int32_t ld, float* d_c, int32_t ldc, int32_t split, int32_t* d_err,
                                void* stream) {
  if (n < kGramTile || n % kGramTile != 0 || k < kGramBK || k % kGramBK != 0 || ld < k ||
      ld % 4 != 0 || ldc < n || ldc % 4 != 0)
    return fail(QTQP_ERR_BAD_ARG,
                "qtqp_tc_gram_f32: n must be a multiple of 128, k of 32, ld >= k and ldc >= n "
                "multiples of 4");
  if (d_hi == nullptr || d_c == nullptr || d_err == nullptr || (split && d_lo == nullptr))
    return fail(QTQP_ERR_BAD_ARG, "qtqp_tc_gram_f32: null pointer");
  if ((reinterpret_cast<uintptr_t>(d_hi) | reinterpret_cast<uintptr_t>(d_c) |
       reinterpret_cast<uintptr_t>(split ? d_lo : d_hi)) & 15)
    return fail(QTQP_ERR_BAD_ARG, "qtqp_tc_gram_f32: pointers must be 16-byte aligned");
  return launch_gram_tf32(n, k, d_hi, d_lo, ld, d_c, ldc, split, d_err,
                          static_cast<cudaStream_t>(stream));
}

namespace qtqp {
// hi = x rounded to TF32 (nearest, ties away), lo = x - hi (exact in FP32).
__global__ void split_tf32_kernel(const float* __restrict__ x, int64_t count,
                                  float* __restrict__ hi, float* __restrict__ lo) {
  for (int64_t i = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; i < count;
       i += int64_t(gridDim.x) * blockDim.x) {
    const float v = x[i];
    uint32_t h;
    asm("cvt.rna.tf32.f32 %0, %1;" : "=r"(h) : "f"(v));
    const float hf = __uint_as_float(h);
    hi[i] = hf;
    lo[i] = v - hf;
  }
}
}  // namespace qtqp

extern "C" int qtqp_tc_split_tf32(const float* d_x, int64_t count, float* d_hi, float* d_lo,
                                  void* stream) {
  if (count < 0 || (count > 0 && (d_x == nullptr || d_hi == nullptr || d_lo == nullptr)))
    return fail(QTQP_ERR_BAD_ARG, "qtqp_tc_split_tf32: bad arguments");
  if (count == 0) return QTQP_OK;
  const int grid = int(std::min<int64_t>((count + 255) / 256, 148 * 16));
  split_tf32_kernel<<<grid, 256, 0, static_cast<cudaStream_t>(stream)>>>(d_x, count, d_hi, d_lo);
  return cuda_check(cudaGetLastError(), "split_tf32_kernel launch");
}
