// Status and error-message plumbing of the C-ABI.
#include <stdarg.h>
#include <stdio.h>

#include <vector>

#include "pk_common.cuh"

namespace {
thread_local char g_last_error[512] = "";
}

namespace pk {

void set_error(const char* fmt, ...) {
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(g_last_error, sizeof(g_last_error), fmt, ap);
  va_end(ap);
}

int cuda_status(cudaError_t e, const char* where) {
  if (e == cudaSuccess) return PK_OK;
  set_error("%s: %s", where, cudaGetErrorString(e));
  return PK_ERR_CUDA;
}

int set_smem_limit(const void* kernel, size_t bytes) {
  if (bytes <= 48 * 1024) return PK_OK;
  return cuda_status(cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes),
                     "cudaFuncSetAttribute");
}

// Readers of the per-file counters of bounded waits that gave up, one per
// source file that stages the world; filled at library load.
static std::vector<int (*)(unsigned long long*)>& timeout_readers() {
  static std::vector<int (*)(unsigned long long*)> v;
  return v;
}

int register_timeout_reader(int (*reader)(unsigned long long*)) {
  timeout_readers().push_back(reader);
  return (int)timeout_readers().size();
}

}  // namespace pk

extern "C" int pk_stage_wait_timeouts(uint64_t* count) {
  PK_CHECK_ARG(count != nullptr, "null count");
  unsigned long long acc = 0;
  for (auto reader : pk::timeout_readers())
    if (int s = reader(&acc)) return s;
  *count = acc;
  return PK_OK;
}

extern "C" {

const char* pk_version(void) { return "pyroffi_b200 0.1 (sm_100a)"; }

const char* pk_last_error(void) { return g_last_error; }

const char* pk_status_string(int status) {
  switch (status) {
    case PK_OK: return "ok";
    case PK_ERR_INVALID: return "invalid argument";
    case PK_ERR_CAPACITY: return "capacity exceeded";
    case PK_ERR_CUDA: return "CUDA error";
    case PK_ERR_TIMEOUT: return "device wait timed out";
    default: return "unknown status";
  }
}

}  // extern "C"
