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

// The bounded-wait hooks of every source file that stages the world; filled
// at library load.
static std::vector<StageWaitHooks>& stage_wait_hooks() {
  static std::vector<StageWaitHooks> v;
  return v;
}

int register_stage_wait_hooks(StageWaitHooks h) {
  stage_wait_hooks().push_back(h);
  return (int)stage_wait_hooks().size();
}

}  // namespace pk

extern "C" int pk_stage_wait_timeouts(uint64_t* count) {
  PK_CHECK_ARG(count != nullptr, "null count");
  unsigned long long gave_up = 0, abandoned = 0;
  for (const auto& h : pk::stage_wait_hooks())
    if (int s = h.read(&gave_up, &abandoned)) return s;
  *count = gave_up;
  if (gave_up == 0) return PK_OK;
  pk::set_error("%llu block(s) gave up waiting for the TMA copy of the obstacle arrays and loaded them plainly; "
                "%llu of them finished with the copy possibly in flight%s",
                gave_up, abandoned, abandoned ? ": outputs since then are untrusted" : "");
  return PK_ERR_TIMEOUT;
}

extern "C" int pk_stage_wait_reset(void) {
  for (const auto& h : pk::stage_wait_hooks())
    if (int s = h.reset()) return s;
  return PK_OK;
}

extern "C" int pk_stage_wait_configure(int32_t force_timeout, int64_t limit_ns) {
  PK_CHECK_ARG(force_timeout == 0 || force_timeout == 1, "force_timeout must be 0 or 1");
  const unsigned long long lim = limit_ns > 0 ? (unsigned long long)limit_ns : 1000000000ull;
  for (const auto& h : pk::stage_wait_hooks())
    if (int s = h.set((unsigned)force_timeout, lim)) return s;
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
