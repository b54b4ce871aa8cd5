// Dense KKT backend behind the direct.LinearSolver plugin interface
// (src/qtqp/direct.py:49-109), algorithm of src/qtqp/solvers_dense.py:99-142.
// Each call is one single-block launch on the caller's stream; the workspace
// holds A, P_off, the factor and the vectors (layout of dense_ipm.cuh with
// every region in global memory) behind a small header.
#include "dense_ipm.cuh"

namespace qtqp {

constexpr int kPluginThreads = 256;
constexpr size_t kPluginHeader = 256;  // int32 factor precision (32 or 64)

__host__ __device__ inline size_t plugin_bytes(int n, int m) {
  const InstLayout L = plan_layout(n, m, 0);
  return kPluginHeader + L.global_bytes;
}

__device__ inline void plugin_bind(DenseIpm<kPluginThreads>& s, int n, int m, char* ws,
                                   double* red) {
  s.bind(n, m, nullptr, ws + kPluginHeader, 0);
  s.z = 0;
  s.has_p = true;
  s.red = red;
  s.phase = 0;
  s.o = nullptr;
}

__global__ void __launch_bounds__(kPluginThreads)
    plugin_set_kernel(int n, int m, const double* a, const double* p_off, char* ws) {
  DenseIpm<kPluginThreads> s;
  plugin_bind(s, n, m, ws, nullptr);
  for (int idx = threadIdx.x; idx < m * n; idx += kPluginThreads) {
    const int i = idx / n, j = idx - i * n;
    s.A[i * s.lda + j] = a[idx];
  }
  for (int idx = threadIdx.x; idx < n * n; idx += kPluginThreads) {
    const int i = idx / n, j = idx - i * n;
    s.P[i * s.ldp + j] = (i == j) ? 0.0 : p_off[idx];
  }
}

__global__ void __launch_bounds__(kPluginThreads)
    plugin_factorize_kernel(int n, int m, const double* diag, int prec, char* ws, int* info) {
  __shared__ double red[2 * (kPluginThreads / 32) * kRedMax];
  DenseIpm<kPluginThreads> s;
  plugin_bind(s, n, m, ws, red);
  s.kkt_diag_given(diag);
  __syncthreads();
  int rc = prec == QTQP_PREC_FP64 ? s.template factorize<double>() : s.template factorize<float>();
  if (threadIdx.x == 0) {
    *info = rc;
    *reinterpret_cast<int*>(ws) = prec == QTQP_PREC_FP64 ? 64 : 32;
  }
}

__global__ void __launch_bounds__(kPluginThreads)
    plugin_solve_kernel(int n, int m, const double* rhs, double* out, char* ws) {
  DenseIpm<kPluginThreads> s;
  plugin_bind(s, n, m, ws, nullptr);
  const bool fp64 = *reinterpret_cast<const int*>(ws) != 32;
  s.kkt_solve(rhs, out, false, fp64);
}

__global__ void __launch_bounds__(kPluginThreads)
    plugin_matvec_kernel(int n, int m, const double* x, double* out, char* ws) {
  DenseIpm<kPluginThreads> s;
  plugin_bind(s, n, m, ws, nullptr);
  s.kkt_matvec(x, out);
}

// Ruiz equilibration alone (the device IPM's load_and_equilibrate phase, the
// algorithm of src/qtqp/__init__.py:616-663) with its outputs written back:
// d (m), e (n), the equilibrated A (m x n) and P (n x n, diagonal included),
// all row-major.
__global__ void __launch_bounds__(kPluginThreads)
    plugin_equilibrate_kernel(int n, int m, const double* a, const double* p, const double* b,
                              const double* c, char* ws, double* d_out, double* e_out,
                              double* a_eq, double* p_eq) {
  __shared__ double red[2 * (kPluginThreads / 32) * kRedMax];
  DenseIpm<kPluginThreads> s;
  plugin_bind(s, n, m, ws, red);
  s.has_p = p != nullptr;
  s.A0 = a;
  s.P0 = p;
  s.b0 = b;
  s.c0 = c;
  double nb, nc;
  s.load_and_equilibrate(true, nb, nc);
  const double* de = s.vec(kDE);
  const double* pi = s.vec(kPI);
  for (int k = threadIdx.x; k < n + m; k += kPluginThreads) {
    if (k < n) {
      e_out[k] = de[k];
    } else {
      d_out[k - n] = de[k];
    }
  }
  for (int idx = threadIdx.x; idx < m * n; idx += kPluginThreads) {
    const int i = idx / n, j = idx - i * n;
    a_eq[idx] = s.A[i * s.lda + j];
  }
  for (int idx = threadIdx.x; idx < n * n; idx += kPluginThreads) {
    const int i = idx / n, j = idx - i * n;
    p_eq[idx] = (i == j) ? pi[i] : s.P[i * s.ldp + j];
  }
}

static int plugin_args(int n, int m, const void* ws) {
  if (n < 1 || m < 1) return fail(QTQP_ERR_BAD_ARG, "dense KKT: need n >= 1 and m >= 1");
  if (ws == nullptr) return fail(QTQP_ERR_BAD_ARG, "dense KKT: null workspace");
  return QTQP_OK;
}

}  // namespace qtqp

using namespace qtqp;

extern "C" size_t qtqp_kkt_dense_workspace_bytes(int32_t n, int32_t m) {
  if (n < 1 || m < 1) return 0;
  return plugin_bytes(n, m);
}

extern "C" int qtqp_kkt_dense_set(int32_t n, int32_t m, const double* d_a,
                                  const double* d_p_off, void* d_ws, void* stream) {
  int rc = plugin_args(n, m, d_ws);
  if (rc) return rc;
  if (d_a == nullptr || d_p_off == nullptr) return fail(QTQP_ERR_BAD_ARG, "dense KKT: null A/P");
  plugin_set_kernel<<<1, kPluginThreads, 0, static_cast<cudaStream_t>(stream)>>>(
      n, m, d_a, d_p_off, static_cast<char*>(d_ws));
  return cuda_check(cudaGetLastError(), "plugin_set_kernel launch");
}

extern "C" int qtqp_kkt_dense_factorize(int32_t n, int32_t m, const double* d_diag,
                                        int32_t precision, void* d_ws, int32_t* d_info,
                                        void* stream) {
  int rc = plugin_args(n, m, d_ws);
  if (rc) return rc;
  if (d_diag == nullptr || d_info == nullptr)
    return fail(QTQP_ERR_BAD_ARG, "dense KKT: null diag/info");
  if (precision != QTQP_PREC_FP64 && precision != QTQP_PREC_MIXED)
    return fail(QTQP_ERR_BAD_ARG, "dense KKT: unknown precision");
  plugin_factorize_kernel<<<1, kPluginThreads, 0, static_cast<cudaStream_t>(stream)>>>(
      n, m, d_diag, precision, static_cast<char*>(d_ws), d_info);
  return cuda_check(cudaGetLastError(), "plugin_factorize_kernel launch");
}

extern "C" int qtqp_kkt_dense_solve(int32_t n, int32_t m, const double* d_rhs, double* d_out,
                                    void* d_ws, void* stream) {
  int rc = plugin_args(n, m, d_ws);
  if (rc) return rc;
  if (d_rhs == nullptr || d_out == nullptr || d_rhs == d_out)
    return fail(QTQP_ERR_BAD_ARG, "dense KKT: rhs/out must be distinct device vectors");
  plugin_solve_kernel<<<1, kPluginThreads, 0, static_cast<cudaStream_t>(stream)>>>(
      n, m, d_rhs, d_out, static_cast<char*>(d_ws));
  return cuda_check(cudaGetLastError(), "plugin_solve_kernel launch");
}

extern "C" int qtqp_kkt_dense_matvec(int32_t n, int32_t m, const double* d_x, double* d_out,
                                     void* d_ws, void* stream) {
  int rc = plugin_args(n, m, d_ws);
  if (rc) return rc;
  if (d_x == nullptr || d_out == nullptr || d_x == d_out)
    return fail(QTQP_ERR_BAD_ARG, "dense KKT: x/out must be distinct device vectors");
  plugin_matvec_kernel<<<1, kPluginThreads, 0, static_cast<cudaStream_t>(stream)>>>(
      n, m, d_x, d_out, static_cast<char*>(d_ws));
  return cuda_check(cudaGetLastError(), "plugin_matvec_kernel launch");
}

extern "C" int qtqp_dense_equilibrate(int32_t n, int32_t m, const double* d_a, const double* d_p,
                                      const double* d_b, const double* d_c, void* d_ws,
                                      double* d_d, double* d_e, double* d_a_eq, double* d_p_eq,
                                      void* stream) {
  int rc = plugin_args(n, m, d_ws);
  if (rc) return rc;
  if (d_a == nullptr || d_b == nullptr || d_c == nullptr || d_d == nullptr || d_e == nullptr ||
      d_a_eq == nullptr || d_p_eq == nullptr)
    return fail(QTQP_ERR_BAD_ARG, "qtqp_dense_equilibrate: null argument");
  plugin_equilibrate_kernel<<<1, kPluginThreads, 0, static_cast<cudaStream_t>(stream)>>>(
      n, m, d_a, d_p, d_b, d_c, static_cast<char*>(d_ws), d_d, d_e, d_a_eq, d_p_eq);
  return cuda_check(cudaGetLastError(), "plugin_equilibrate_kernel launch");
}
