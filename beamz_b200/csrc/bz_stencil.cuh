// Device helpers shared by the 2D forward and adjoint step kernels.
#pragma once

#include "bz_internal.cuh"

namespace bz {

// H-update factors for a cell with conductivity term a (numpy_backend.py:52-60):
// factor = (1-a)/(1+a), source = c/(1+a). a == 0 (all non-PML cells) is exact.
template <typename T>
__device__ __forceinline__ void h_coeffs(T a, T chx, T chy, T& fh, T& cx, T& cy) {
  if (a == T(0)) {
    fh = T(1);
    cx = chx;
    cy = chy;
  } else {
    const T den = T(1) + a;
    fh = (T(1) - a) / den;
    cx = chx / den;
    cy = chy / den;
  }
}

// Explicitly rounded arithmetic, so that every kernel evaluating an update gets
// the same bits whatever the compiler would contract in its context.
__device__ __forceinline__ float fma_rn(float a, float b, float c) { return __fmaf_rn(a, b, c); }
__device__ __forceinline__ double fma_rn(double a, double b, double c) { return __fma_rn(a, b, c); }
__device__ __forceinline__ float mul_rn(float a, float b) { return __fmul_rn(a, b); }
__device__ __forceinline__ double mul_rn(double a, double b) { return __dmul_rn(a, b); }
__device__ __forceinline__ float sub_rn(float a, float b) { return __fsub_rn(a, b); }
__device__ __forceinline__ double sub_rn(double a, double b) { return __dsub_rn(a, b); }

// Hx' = fh*Hx - cx*(Ez(x+1) - Ez(x))   (numpy_backend.py:55-57)
template <typename T>
__device__ __forceinline__ T hx_update(T fh, T hx, T cx, T ez_right, T ez) {
  return fma_rn(fh, hx, -mul_rn(cx, sub_rn(ez_right, ez)));
}
// Hy' = fh*Hy + cy*(Ez(y+1) - Ez(y))   (numpy_backend.py:58-60)
template <typename T>
__device__ __forceinline__ T hy_update(T fh, T hy, T cy, T ez_down, T ez) {
  return fma_rn(fh, hy, mul_rn(cy, sub_rn(ez_down, ez)));
}
// Ez' = fe*Ez + ce*(-(Hx - Hx(x-1)) + qy*(Hy - Hy(y-1)))   (numpy_backend.py:80-88)
template <typename T>
__device__ __forceinline__ T ez_update(T fe, T ez, T ce, T qy, T hx, T hx_left, T hy, T hy_up) {
  return fma_rn(fe, ez, mul_rn(ce, fma_rn(qy, sub_rn(hy, hy_up), -sub_rn(hx, hx_left))));
}

__device__ __forceinline__ int lower_bound_i(const int* a, int lo, int hi, int key) {
  while (lo < hi) {
    const int mid = (lo + hi) >> 1;
    if (__ldg(a + mid) < key) lo = mid + 1; else hi = mid;
  }
  return lo;
}

// Operation ranges of a block's rows: thread t < nrows finds, in row y0+t, the
// sorted operations whose cell lies in [xlo, xhi); prefix sums let all threads
// share the flattened list. Returns the number of operations.
__device__ __forceinline__ int block_op_ranges(const int* row_ptr, const int* cells, int y0, int nrows, int nx,
                                               int xlo, int xhi, int* s_k0, int* s_pre) {
  if (threadIdx.x < nrows) {
    const int y = y0 + threadIdx.x;
    const int lo = __ldg(row_ptr + y), hi = __ldg(row_ptr + y + 1);
    int k0 = lo, k1 = lo;
    if (lo < hi) {
      k0 = lower_bound_i(cells, lo, hi, y * nx + xlo);
      k1 = lower_bound_i(cells, k0, hi, y * nx + xhi);
    }
    s_k0[threadIdx.x] = k0;
    s_pre[threadIdx.x + 1] = k1 - k0;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    s_pre[0] = 0;
    for (int t = 0; t < nrows; ++t) s_pre[t + 1] += s_pre[t];
  }
  __syncthreads();
  return s_pre[nrows];
}

// i-th operation of the flattened block list -> (row offset t, op index).
__device__ __forceinline__ int op_at(int i, int nrows, const int* s_k0, const int* s_pre, int& t) {
  t = 0;
  while (t + 1 < nrows && s_pre[t + 1] <= i) ++t;
  return s_k0[t] + (i - s_pre[t]);
}

}  // namespace bz
