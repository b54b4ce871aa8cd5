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
