// capi.cu -- library identity and thread-local error messages.
#include <cstdarg>
#include <cstdio>

#include "wf_common.cuh"

namespace {
thread_local char g_err[512] = "";
}

namespace wf {

int set_error(int code, const char* fmt, ...) {
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(g_err, sizeof(g_err), fmt, ap);
  va_end(ap);
  return code;
}

int cuda_fail(cudaError_t e, const char* what) {
  return set_error(WF_E_CUDA, "%s: %s", what, cudaGetErrorString(e));
}

}  // namespace wf

extern "C" int32_t wf_abi_version(void) { return WF_ABI_VERSION; }

extern "C" const char* wf_last_error(void) { return g_err; }
