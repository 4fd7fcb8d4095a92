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

// ---- divergence check ------------------------------------------------------------
// One pass over a field array: a value that is not finite or whose magnitude exceeds
// `limit` marks the run as diverged. The first detection of a launch writes
// BZ_ERR_DIVERGED into status[0] and the step into status[1]; later launches leave a
// recorded detection in place. The host reads the words when it next synchronizes.
namespace {
template <typename T>
__global__ void field_check_kernel(const T* __restrict__ f, long long n, double limit, long long step,
                                   long long* __restrict__ status) {
  bool bad = false;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
    const double v = (double)__ldg(f + i);
    bad |= !(fabs(v) <= limit);  // NaN compares false
  }
  if (__any_sync(0xffffffffu, bad) && (threadIdx.x & 31) == 0) {
    if (atomicCAS(reinterpret_cast<unsigned long long*>(status), 0ull, (unsigned long long)(long long)BZ_ERR_DIVERGED) == 0ull)
      status[1] = step;
  }
}
}  // namespace

extern "C" int bz_field_check(const void* field, int32_t dtype, int64_t n, double limit, int64_t step,
                              int64_t* status, void* stream) {
  BZ_REQUIRE(field && status, "bz_field_check: NULL field or status");
  BZ_REQUIRE(n >= 0 && limit > 0, "bz_field_check: need n >= 0 and limit > 0");
  if (n == 0) return BZ_OK;
  const int threads = 256;
  const unsigned blocks = (unsigned)(bz::ceil_div(n, threads * 8) < 148 * 8 ? bz::ceil_div(n, threads * 8) : 148 * 8);
  cudaStream_t st = bz::as_stream(stream);
  if (dtype == BZ_F32)
    field_check_kernel<float><<<blocks, threads, 0, st>>>((const float*)field, n, limit, step, (long long*)status);
  else if (dtype == BZ_F64)
    field_check_kernel<double><<<blocks, threads, 0, st>>>((const double*)field, n, limit, step, (long long*)status);
  else
    return bz::fail(BZ_ERR_INVALID, "bz_field_check: unknown dtype %d", dtype);
  return bz::check_launch("bz_field_check");
}
