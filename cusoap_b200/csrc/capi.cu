// Error reporting and version of the C ABI (include/soapb200.h).
#include <stdarg.h>
#include <stdio.h>

#include <atomic>

#include "common.cuh"

namespace soapb {

static thread_local char g_err[512] = "";
static std::atomic<long long> g_launches{0};

void count_launches(int n) { g_launches.fetch_add(n, std::memory_order_relaxed); }

int set_error(int status, const char* fmt, ...) {
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(g_err, sizeof(g_err), fmt, ap);
  va_end(ap);
  return status;
}

int check_cuda(cudaError_t e, const char* what) {
  if (e == cudaSuccess) return SOAPB_OK;
  return set_error(SOAPB_ERR_CUDA, "%s: %s", what, cudaGetErrorString(e));
}

}  // namespace soapb

extern "C" const char* soapb_last_error(void) { return soapb::g_err; }

extern "C" const char* soapb_version(void) { return "soapb200 0.1.0 (sm_100a)"; }

extern "C" int64_t soapb_kernel_launches(void) { return soapb::g_launches.load(std::memory_order_relaxed); }
