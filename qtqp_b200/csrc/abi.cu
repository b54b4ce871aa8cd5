// Library-level entry points: error reporting, version, device query.
#include <string>

#include "common.cuh"

namespace qtqp {

static thread_local std::string g_last_error;

void set_last_error(const std::string& msg) { g_last_error = msg; }

int fail(int code, const std::string& msg) {
  g_last_error = msg;
  return code;
}

int cuda_check(cudaError_t err, const char* what) {
  if (err == cudaSuccess) return QTQP_OK;
  g_last_error = std::string(what) + ": " + cudaGetErrorString(err);
  return QTQP_ERR_CUDA;
}

}  // namespace qtqp

#ifdef QTQP_PHASE_TIMERS
namespace qtqp {
__device__ unsigned long long g_phase_cycles[kNumPhases];
}
// Profiling builds only: copies (and clears) the per-phase cycle counters.
extern "C" int qtqp_phase_cycles(unsigned long long* h_out, int count) {
  if (count > qtqp::kNumPhases) count = qtqp::kNumPhases;
  int rc = qtqp::cuda_check(cudaMemcpyFromSymbol(h_out, qtqp::g_phase_cycles,
                                                 sizeof(unsigned long long) * count),
                            "cudaMemcpyFromSymbol");
  if (rc) return rc;
  unsigned long long zero[qtqp::kNumPhases] = {};
  return qtqp::cuda_check(cudaMemcpyToSymbol(qtqp::g_phase_cycles, zero, sizeof(zero)),
                          "cudaMemcpyToSymbol");
}
#endif

extern "C" const char* qtqp_last_error(void) { return qtqp::g_last_error.c_str(); }

extern "C" int qtqp_version(void) { return 1; }

extern "C" int qtqp_device_sm_count(void) {
  int dev = 0, sms = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) {
    cudaGetLastError();
    return 0;
  }
  if (cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess) {
    cudaGetLastError();
    return 0;
  }
  return sms;
}
