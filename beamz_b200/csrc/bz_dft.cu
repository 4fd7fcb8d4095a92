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

template <typename T>
__global__ void __launch_bounds__(32 * FOLD_WARPS) dft_fold_kernel(const T* __restrict__ ring, int ring_len,
                                                                     long long n_items, int n_freq,
                                                                     const double* __restrict__ phasor,
                                                                     long long n_phasor, long long step0, int count,
                                                                     double* __restrict__ dft) {
  const long long w = blockIdx.x * (long long)FOLD_WARPS + (threadIdx.x >> 5);
  const int lane = threadIdx.x & 31;
  if (w >= n_items * n_freq) return;
  const long long item = w / n_freq;
  const int f = (int)(w - item * n_freq);
  double acc[10];
#pragma unroll
  for (int q = 0; q < 10; ++q) acc[q] = 0.0;
  for (int j = lane; j < count; j += 32) {
    const long long s = step0 + j;
    if (s >= n_phasor) continue;
    const T* smp = ring + ((s % ring_len) * n_items + item) * 5;
    const double* ph = phasor + (s * n_freq + f) * 4;
    const double ce = __ldg(ph), se = __ldg(ph + 1), ch = __ldg(ph + 2), sh = __ldg(ph + 3);
    const double q0 = (double)smp[0];
    acc[0] += q0 * ce;
    acc[1] += q0 * se;
#pragma unroll
    for (int q = 1; q < 5; ++q) {
      const double v = (double)smp[q];
      acc[2 * q] += v * ch;
      acc[2 * q + 1] += v * sh;
    }
  }
#pragma unroll
  for (int q = 0; q < 10; ++q) {
    double v = acc[q];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
    acc[q] = v;
  }
  if (lane == 0) {
    double* out = dft + (item * n_freq + f) * 10;
#pragma unroll
    for (int q = 0; q < 10; ++q) out[q] += acc[q];
  }
}

}  // namespace
}  // namespace bz

extern "C" int bz_dft_fold(const void* ring, int32_t dtype, int32_t ring_len, int64_t n_items, int32_t n_freq,
                           const double* phasor, int64_t n_phasor, int64_t step0, int32_t count, double* dft,
                           void* stream) {
  BZ_REQUIRE(ring && phasor && dft, "bz_dft_fold: NULL buffer");
  BZ_REQUIRE(ring_len >= 1 && count >= 0 && count <= ring_len, "bz_dft_fold: count %d must be in [0, ring_len %d]",
             count, ring_len);
  BZ_REQUIRE(n_items >= 0 && n_freq >= 0 && step0 >= 0 && n_phasor >= 0, "bz_dft_fold: negative size");
  const long long warps = n_items * (long long)n_freq;
  if (warps == 0 || count == 0) return BZ_OK;
  const unsigned blocks = (unsigned)bz::ceil_div(warps, bz::FOLD_WARPS);
  cudaStream_t st = bz::as_stream(stream);
  if (dtype == BZ_F32)
    bz::dft_fold_kernel<float><<<blocks, 32 * bz::FOLD_WARPS, 0, st>>>((const float*)ring, ring_len, n_items, n_freq,
                                                                       phasor, n_phasor, step0, count, dft);
  else if (dtype == BZ_F64)
    bz::dft_fold_kernel<double><<<blocks, 32 * bz::FOLD_WARPS, 0, st>>>((const double*)ring, ring_len, n_items,
                                                                        n_freq, phasor, n_phasor, step0, count, dft);
  else
    return bz::fail(BZ_ERR_INVALID, "bz_dft_fold: unknown dtype %d", dtype);
  return bz::check_launch("bz_dft_fold");
}
