// Unfused 2D half-step updates behind the Backend interface
// (beamz/simulation/backends/base.py:33-43, numpy_backend.py:34-88).
//
// These serve callers that drive update_h_fields / update_e_field themselves on
// arrays with the reference's shapes: Ez (ny, nx), Hx (ny, nx-1), Hy (ny-1, nx),
// sigma and eps_r (ny, nx). Real fields use nc = 1; complex fields are passed as
// interleaved (re, im) pairs with nc = 2 (the update is real-linear, so each part
// evolves on its own). Coefficients are formed per cell in float64 from the
// reference's expressions. The fused stepping path is bz_step2d.
#include "bz_internal.cuh"

namespace bz {
namespace {

template <typename T>
__global__ void update_h2d_kernel(T* __restrict__ hx, T* __restrict__ hy, const T* __restrict__ ez,
                                  const T* __restrict__ sigma, int ny, int nx, int nc, double dx, double dy,
                                  double dt, double mu0, double eps0) {
  const int x = blockIdx.x * blockDim.x + threadIdx.x;
  const int y = blockIdx.y * blockDim.y + threadIdx.y;
  if (y >= ny || x >= nx) return;
  const double sm = (double)sigma[(long long)y * nx + x] * mu0 / eps0;
  const double den = 1.0 + sm * dt / (2.0 * mu0);
  const double f = (1.0 - sm * dt / (2.0 * mu0)) / den;
  const double s = (dt / mu0) / den;
  for (int c = 0; c < nc; ++c) {
    const double e0 = (double)ez[((long long)y * nx + x) * nc + c];
    if (x < nx - 1) {  // Hx -= s * (Ez[:, 1:] - Ez[:, :-1]) / dy
      const long long i = ((long long)y * (nx - 1) + x) * nc + c;
      const double e1 = (double)ez[((long long)y * nx + x + 1) * nc + c];
      hx[i] = (T)(f * (double)hx[i] - s * ((e1 - e0) / dy));
    }
    if (y < ny - 1) {  // Hy += s * (Ez[1:, :] - Ez[:-1, :]) / dx
      const long long i = ((long long)y * nx + x) * nc + c;
      const double e1 = (double)ez[((long long)(y + 1) * nx + x) * nc + c];
      hy[i] = (T)(f * (double)hy[i] + s * ((e1 - e0) / dx));
    }
  }
}

template <typename T>
__global__ void update_e2d_kernel(T* __restrict__ ez, const T* __restrict__ hx, const T* __restrict__ hy,
                                  const T* __restrict__ sigma, const T* __restrict__ eps_r, int ny, int nx, int nc,
                                  double dx, double dy, double dt, double eps0) {
  const int x = blockIdx.x * blockDim.x + threadIdx.x;
  const int y = blockIdx.y * blockDim.y + threadIdx.y;
  if (y < 1 || y >= ny - 1 || x < 1 || x >= nx - 1) return;
  const long long k = (long long)y * nx + x;
  const double sg = (double)sigma[k], er = (double)eps_r[k];
  const double den = 1.0 + sg * dt / (2.0 * eps0 * er);
  const double f1 = (1.0 - sg * dt / (2.0 * eps0 * er)) / den;
  const double f2 = (dt / (eps0 * er)) / den;
  for (int c = 0; c < nc; ++c) {
    const double cx = ((double)hx[((long long)y * (nx - 1) + x) * nc + c] -
                       (double)hx[((long long)y * (nx - 1) + x - 1) * nc + c]) / dy;
    const double cy = ((double)hy[((long long)y * nx + x) * nc + c] -
                       (double)hy[((long long)(y - 1) * nx + x) * nc + c]) / dx;
    ez[k * nc + c] = (T)(f1 * (double)ez[k * nc + c] + f2 * (-cx + cy));
  }
}

}  // namespace
}  // namespace bz

extern "C" int bz_update_h2d(int32_t dtype, int32_t ny, int32_t nx, int32_t nc, void* hx, void* hy, const void* ez,
                             const void* sigma, double dx, double dy, double dt, double mu0, double eps0,
                             void* stream) {
  BZ_REQUIRE(hx && hy && ez && sigma, "bz_update_h2d: NULL buffer");
  BZ_REQUIRE(ny >= 2 && nx >= 2 && (nc == 1 || nc == 2), "bz_update_h2d: bad shape %d x %d x %d", ny, nx, nc);
  dim3 b(32, 8), g((unsigned)bz::ceil_div(nx, 32), (unsigned)bz::ceil_div(ny, 8));
  cudaStream_t st = bz::as_stream(stream);
  if (dtype == BZ_F32)
    bz::update_h2d_kernel<float><<<g, b, 0, st>>>((float*)hx, (float*)hy, (const float*)ez, (const float*)sigma, ny,
                                                  nx, nc, dx, dy, dt, mu0, eps0);
  else if (dtype == BZ_F64)
    bz::update_h2d_kernel<double><<<g, b, 0, st>>>((double*)hx, (double*)hy, (const double*)ez,
                                                   (const double*)sigma, ny, nx, nc, dx, dy, dt, mu0, eps0);
  else
    return bz::fail(BZ_ERR_INVALID, "bz_update_h2d: unknown dtype %d", dtype);
  return bz::check_launch("bz_update_h2d");
}

extern "C" int bz_update_e2d(int32_t dtype, int32_t ny, int32_t nx, int32_t nc, void* ez, const void* hx,
                             const void* hy, const void* sigma, const void* eps_r, double dx, double dy, double dt,
                             double eps0, void* stream) {
  BZ_REQUIRE(hx && hy && ez && sigma && eps_r, "bz_update_e2d: NULL buffer");
  BZ_REQUIRE(ny >= 2 && nx >= 2 && (nc == 1 || nc == 2), "bz_update_e2d: bad shape %d x %d x %d", ny, nx, nc);
  dim3 b(32, 8), g((unsigned)bz::ceil_div(nx, 32), (unsigned)bz::ceil_div(ny, 8));
  cudaStream_t st = bz::as_stream(stream);
  if (dtype == BZ_F32)
    bz::update_e2d_kernel<float><<<g, b, 0, st>>>((float*)ez, (const float*)hx, (const float*)hy,
                                                  (const float*)sigma, (const float*)eps_r, ny, nx, nc, dx, dy, dt,
                                                  eps0);
  else if (dtype == BZ_F64)
    bz::update_e2d_kernel<double><<<g, b, 0, st>>>((double*)ez, (const double*)hx, (const double*)hy,
                                                   (const double*)sigma, (const double*)eps_r, ny, nx, nc, dx, dy,
                                                   dt, eps0);
  else
    return bz::fail(BZ_ERR_INVALID, "bz_update_e2d: unknown dtype %d", dtype);
  return bz::check_launch("bz_update_e2d");
}
