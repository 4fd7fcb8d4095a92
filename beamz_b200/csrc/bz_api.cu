// Library-wide entries: version string and thread-local error reporting.
#include <stdarg.h>
#include <string.h>

#include "bz_internal.cuh"

namespace bz {

static thread_local char g_err_msg[512] = {0};
static thread_local int g_err_code = BZ_OK;

int fail(int code, const char* fmt, ...) {
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(g_err_msg, sizeof(g_err_msg), fmt, ap);
  va_end(ap);
  g_err_code = code;
  return code;
}

void clear_error() {
  g_err_msg[0] = 0;
  g_err_code = BZ_OK;
}

int check_launch(const char* what) {
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return fail(BZ_ERR_CUDA, "%s: %s", what, cudaGetErrorString(e));
  return BZ_OK;
}

}  // namespace bz

extern "C" const char* bz_version(void) { return "beamz_b200 0.1.0 sm_100a"; }

extern "C" int bz_last_error(char* buf, size_t len) {
  if (buf && len > 0) {
    strncpy(buf, bz::g_err_msg, len - 1);
    buf[len - 1] = 0;
  }
  return bz::g_err_code;
}

namespace {
__global__ void advance_step_kernel(int64_t* d_step, int64_t n) { *d_step += n; }
}  // namespace

extern "C" int bz_advance_step(int64_t* d_step, int64_t n, void* stream) {
  BZ_REQUIRE(d_step != nullptr, "bz_advance_step: d_step is NULL");
  advance_step_kernel<<<1, 1, 0, bz::as_stream(stream)>>>(d_step, n);
  return bz::check_launch("bz_advance_step");
}
