// Update coefficients from the rasterised material, computed once per run
// instead of every step. The arithmetic is that of
// beamz/simulation/backends/numpy_backend.py:52-60,80-84 (2D) and
// beamz/simulation/fdtd.py:232-305 (3D), rewritten in terms of two stored values:
//   loss a = sigma*dt/(2*eps0)           H:  factor = (1-a)/(1+a), source = (dt/mu0)/(1+a)
//   ce     = dt/(eps0*dy*(eps_r + a))    E:  factor = 1 - 2a/(eps_r+a) = 1 - a*ce*(2*eps0*dy/dt)
//                                             source = (dt/(eps0*eps_r))/(1 + a/eps_r) = ce*dy
// Both are evaluated in float64 and rounded once to the field dtype.
#include "bz_internal.cuh"

namespace bz {
namespace {

template <typename T>
__global__ void prepare_coeffs_kernel(const double* __restrict__ eps, const double* __restrict__ sig, long long rows,
                                      int nx, int pitch, double dt, double eps0, double dy, T* __restrict__ ce,
                                      T* __restrict__ loss) {
  const long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (i >= rows * (long long)pitch) return;
  const long long row = i / pitch;
  const int x = (int)(i - row * pitch);
  if (x >= nx) {
    ce[i] = T(0);
    loss[i] = T(0);
    return;
  }
  const double e = eps[row * nx + x];
  const double s = sig[row * nx + x];
  const double a = (s * dt) / (2.0 * eps0);
  ce[i] = (T)(dt / (eps0 * dy * (e + a)));
  loss[i] = (T)a;
}

}  // namespace
}  // namespace bz

extern "C" int bz_prepare_coeffs(const double* eps_r, const double* sigma, int64_t rows, int32_t nx, int32_t pitch,
                                 int32_t dtype, double dt, double eps0, double dy, void* ce, void* loss,
                                 void* stream) {
  BZ_REQUIRE(eps_r && sigma && ce && loss, "bz_prepare_coeffs: NULL buffer");
  BZ_REQUIRE(rows >= 0 && nx >= 1 && pitch >= nx, "bz_prepare_coeffs: bad shape rows=%lld nx=%d pitch=%d",
             (long long)rows, nx, pitch);
  BZ_REQUIRE(dt > 0 && eps0 > 0 && dy > 0, "bz_prepare_coeffs: dt, eps0 and dy must be positive");
  const long long n = rows * (long long)pitch;
  if (n == 0) return BZ_OK;
  const int threads = 256;
  const unsigned blocks = (unsigned)bz::ceil_div(n, threads);
  cudaStream_t st = bz::as_stream(stream);
  if (dtype == BZ_F32)
    bz::prepare_coeffs_kernel<float><<<blocks, threads, 0, st>>>(eps_r, sigma, rows, nx, pitch, dt, eps0, dy,
                                                                  (float*)ce, (float*)loss);
  else if (dtype == BZ_F64)
    bz::prepare_coeffs_kernel<double><<<blocks, threads, 0, st>>>(eps_r, sigma, rows, nx, pitch, dt, eps0, dy,
                                                                   (double*)ce, (double*)loss);
  else
    return bz::fail(BZ_ERR_INVALID, "bz_prepare_coeffs: unknown dtype %d", dtype);
  return bz::check_launch("bz_prepare_coeffs");
}
