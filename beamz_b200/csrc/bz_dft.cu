// Frequency-domain monitor accumulation: folds a ring of per-step monitor
// samples into float64 running DFT sums. The reference has no frequency-domain
// monitors; this is the readout behind Monitor(frequencies=...).flux().
//
// One warp per (item, frequency): lanes take interleaved steps, accumulate the
// five (re, im) products in float64 registers, and reduce across the warp with
// shuffles; lane 0 adds the result to the running sums. Phasors come from a
// host-built float64 table so no transcendental runs on the device.
#include "bz_internal.cuh"

namespace bz {
namespace {

constexpr int FOLD_WARPS = 4;

template <typename T, int NQ>
__global__ void __launch_bounds__(32 * FOLD_WARPS) dft_fold_kernel(const T* __restrict__ ring, int ring_len,
                                                                     long long n_items, int n_e, int n_freq,
                                                                     const double* __restrict__ phasor,
                                                                     long long n_phasor, long long step0, int count,
                                                                     double* __restrict__ dft) {
  const long long w = blockIdx.x * (long long)FOLD_WARPS + (threadIdx.x >> 5);
  const int lane = threadIdx.x & 31;
  if (w >= n_items * n_freq) return;
  const long long item = w / n_freq;
  const int f = (int)(w - item * n_freq);
  double acc[2 * NQ];
#pragma unroll
  for (int q = 0; q < 2 * NQ; ++q) acc[q] = 0.0;
  for (int j = lane; j < count; j += 32) {
    const long long s = step0 + j;
    if (s >= n_phasor) continue;
    const T* smp = ring + ((s % ring_len) * n_items + item) * NQ;
    const double* ph = phasor + (s * n_freq + f) * 4;
    const double ce = __ldg(ph), se = __ldg(ph + 1), ch = __ldg(ph + 2), sh = __ldg(ph + 3);
#pragma unroll
    for (int q = 0; q < NQ; ++q) {
      const double v = (double)smp[q];
      acc[2 * q] += v * (q < n_e ? ce : ch);
      acc[2 * q + 1] += v * (q < n_e ? se : sh);
    }
  }
#pragma unroll
  for (int q = 0; q < 2 * NQ; ++q) {
    double v = acc[q];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
    acc[q] = v;
  }
  if (lane == 0) {
    double* out = dft + (item * n_freq + f) * (2 * NQ);
#pragma unroll
    for (int q = 0; q < 2 * NQ; ++q) out[q] += acc[q];
  }
}

template <typename T, int NQ>
int fold_t(const void* ring, int ring_len, long long n_items, int n_e, int n_freq, const double* phasor,
           long long n_phasor, long long step0, int count, double* dft, cudaStream_t st) {
  const long long warps = n_items * (long long)n_freq;
  const unsigned blocks = (unsigned)ceil_div(warps, FOLD_WARPS);
  dft_fold_kernel<T, NQ><<<blocks, 32 * FOLD_WARPS, 0, st>>>((const T*)ring, ring_len, n_items, n_e, n_freq, phasor,
                                                             n_phasor, step0, count, dft);
  return check_launch("bz_dft_fold");
}

template <typename T>
int fold_q(const void* ring, int ring_len, long long n_items, int n_q, int n_e, int n_freq, const double* phasor,
           long long n_phasor, long long step0, int count, double* dft, cudaStream_t st) {
  switch (n_q) {
    case 1: return fold_t<T, 1>(ring, ring_len, n_items, n_e, n_freq, phasor, n_phasor, step0, count, dft, st);
    case 2: return fold_t<T, 2>(ring, ring_len, n_items, n_e, n_freq, phasor, n_phasor, step0, count, dft, st);
    case 3: return fold_t<T, 3>(ring, ring_len, n_items, n_e, n_freq, phasor, n_phasor, step0, count, dft, st);
    case 4: return fold_t<T, 4>(ring, ring_len, n_items, n_e, n_freq, phasor, n_phasor, step0, count, dft, st);
    case 5: return fold_t<T, 5>(ring, ring_len, n_items, n_e, n_freq, phasor, n_phasor, step0, count, dft, st);
    default: return fold_t<T, 6>(ring, ring_len, n_items, n_e, n_freq, phasor, n_phasor, step0, count, dft, st);
  }
}

}  // namespace
}  // namespace bz

extern "C" int bz_dft_fold_q(const void* ring, int32_t dtype, int32_t ring_len, int64_t n_items, int32_t n_q,
                             int32_t n_e, int32_t n_freq, const double* phasor, int64_t n_phasor, int64_t step0,
                             int32_t count, double* dft, void* stream) {
  BZ_REQUIRE(ring && phasor && dft, "bz_dft_fold: NULL buffer");
  BZ_REQUIRE(ring_len >= 1 && count >= 0 && count <= ring_len, "bz_dft_fold: count %d must be in [0, ring_len %d]",
             count, ring_len);
  BZ_REQUIRE(n_items >= 0 && n_freq >= 0 && step0 >= 0 && n_phasor >= 0, "bz_dft_fold: negative size");
  BZ_REQUIRE(n_q >= 1 && n_q <= 6 && n_e >= 0 && n_e <= n_q, "bz_dft_fold: need 1 <= n_q <= 6, 0 <= n_e <= n_q");
  if (n_items * (long long)n_freq == 0 || count == 0) return BZ_OK;
  cudaStream_t st = bz::as_stream(stream);
  if (dtype == BZ_F32)
    return bz::fold_q<float>(ring, ring_len, n_items, n_q, n_e, n_freq, phasor, n_phasor, step0, count, dft, st);
  if (dtype == BZ_F64)
    return bz::fold_q<double>(ring, ring_len, n_items, n_q, n_e, n_freq, phasor, n_phasor, step0, count, dft, st);
  return bz::fail(BZ_ERR_INVALID, "bz_dft_fold: unknown dtype %d", dtype);
}

extern "C" int bz_dft_fold(const void* ring, int32_t dtype, int32_t ring_len, int64_t n_items, int32_t n_freq,
                           const double* phasor, int64_t n_phasor, int64_t step0, int32_t count, double* dft,
                           void* stream) {
  // 2D monitor samples: (Ez, Hx(x), Hx(x-1), Hy(y), Hy(y-1)), Ez on the E phasor
  return bz_dft_fold_q(ring, dtype, ring_len, n_items, 5, 1, n_freq, phasor, n_phasor, step0, count, dft, stream);
}
