// Allocation-free variant of the 2D stepping path with frequency-domain monitors.
//
// Who needs it: callers that cannot call cudaMalloc. Examples are a binding driven
// from a runtime that owns every device allocation through its own pool and must not
// see allocations it does not track, and an embedded or real-time host whose
// device-memory budget is fixed when it starts. The regular path (bz_step2d +
// bz_dft_fold) needs a monitor-sample ring that the caller allocates and passes in
// bz_monitor_ops.ring. This entry keeps that ring in a fixed array that is compiled
// into the library, so the caller passes only its inputs and outputs.
//
// Limit: the ring holds at most BZ_STATIC_RING_BYTES (8 MiB). A step's samples take
// n_designs * n_comp * n_points * 5 * sizeof(dtype) bytes. The ring keeps
// min(64, 8 MiB / that) steps, and at least one step must fit. Every GPU that loads
// the library holds the 8 MiB until the process exits.
//
// Sharing: all calls share the array, and it keeps the last call's contents. Nothing
// in it needs to start at zero, because each slot is written by a step of the current
// call before the fold reads it. Calls that overlap on the GPU (on different streams,
// or from different host threads) race on the ring.
//
// Set-up: host code cannot use the array's name as a device address. So every call
// made outside a stream capture looks the address up with cudaGetSymbolAddress, with
// the device current, and keeps it per device ordinal; a call made while its stream is
// being captured uses the kept address (a lookup can load the module, which a capture
// does not allow). Make the first call on each device before any stream capture. A
// device reset between a capture and its replay leaves the captured address stale.
#include <mutex>

#include "bz_internal.cuh"

#define BZ_STATIC_RING_BYTES (8u << 20)

namespace {

__device__ __align__(256) unsigned char g_static_ring[BZ_STATIC_RING_BYTES];

constexpr int kMaxDevices = 64;
void* g_ring_addr[kMaxDevices] = {};
std::mutex g_ring_mu;

// Device address of g_static_ring on the current device: looked up on every call
// outside a capture (so a new context after a device reset gets its own address), the
// kept one during a capture.
int static_ring_address(cudaStream_t stream, void** out) {
  int dev = -1;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return bz::fail(BZ_ERR_CUDA, "bz_step2d_dft_static: cudaGetDevice: %s", cudaGetErrorString(e));
  if (dev < 0 || dev >= kMaxDevices)
    return bz::fail(BZ_ERR_UNSUPPORTED, "bz_step2d_dft_static: device ordinal %d is not below %d", dev, kMaxDevices);
  cudaStreamCaptureStatus cap = cudaStreamCaptureStatusNone;
  e = cudaStreamIsCapturing(stream, &cap);
  if (e != cudaSuccess)
    return bz::fail(BZ_ERR_CUDA, "bz_step2d_dft_static: cudaStreamIsCapturing: %s", cudaGetErrorString(e));
  std::lock_guard<std::mutex> lock(g_ring_mu);
  if (cap == cudaStreamCaptureStatusNone || g_ring_addr[dev] == nullptr) {
    if (cap != cudaStreamCaptureStatusNone)
      return bz::fail(BZ_ERR_INVALID, "bz_step2d_dft_static: the first call on device %d is inside a stream "
                      "capture; call it once before capturing", dev);
    void* p = nullptr;
    e = cudaGetSymbolAddress(&p, g_static_ring);
    if (e != cudaSuccess || p == nullptr)
      return bz::fail(BZ_ERR_CUDA, "bz_step2d_dft_static: cudaGetSymbolAddress: %s", cudaGetErrorString(e));
    g_ring_addr[dev] = p;
  }
  *out = g_ring_addr[dev];
  return BZ_OK;
}

}  // namespace

extern "C" int bz_step2d_dft_static(const bz_grid2d* g, const bz_fields2d* f, const bz_source_ops* src,
                                    const bz_monitor_ops* mon, int64_t step0, int32_t n_steps, int32_t n_freq,
                                    const double* phasor, int64_t n_phasor, double* dft, void* stream) {
  BZ_REQUIRE(g && f && mon, "bz_step2d_dft_static: grid, fields or monitors is NULL");
  BZ_REQUIRE(mon->n_points >= 1, "bz_step2d_dft_static: no monitor points");
  BZ_REQUIRE(mon->ring == nullptr, "bz_step2d_dft_static: monitors.ring must be NULL (this entry supplies the ring)");
  BZ_REQUIRE(n_freq >= 1 && phasor && dft, "bz_step2d_dft_static: needs n_freq >= 1, phasor and dft");
  BZ_REQUIRE(n_steps >= 0 && step0 >= 0, "bz_step2d_dft_static: negative step0 or n_steps");
  BZ_REQUIRE(g->dtype == BZ_F32 || g->dtype == BZ_F64, "bz_step2d_dft_static: unknown dtype %d", g->dtype);
  BZ_REQUIRE(g->n_designs >= 1 && (g->n_comp == 1 || g->n_comp == 2), "bz_step2d_dft_static: bad batch shape");
  const unsigned long long elem = g->dtype == BZ_F64 ? 8ull : 4ull;
  const long long items = (long long)g->n_designs * g->n_comp * mon->n_points;
  const unsigned long long step_bytes = (unsigned long long)items * 5ull * elem;
  if (step_bytes > BZ_STATIC_RING_BYTES)
    return bz::fail(BZ_ERR_INVALID,
                    "bz_step2d_dft_static: one step of monitor samples needs %llu bytes, more than the %u-byte "
                    "static ring; use bz_step2d with a caller-allocated ring",
                    step_bytes, (unsigned)BZ_STATIC_RING_BYTES);
  unsigned long long fit = BZ_STATIC_RING_BYTES / step_bytes;
  const int ring_len = (int)(fit < 64ull ? fit : 64ull);
  void* ring = nullptr;
  int st = static_ring_address(bz::as_stream(stream), &ring);
  if (st != BZ_OK) return st;
  bz_monitor_ops m = *mon;
  m.ring = ring;
  m.ring_len = ring_len;
  int64_t folded = step0;
  for (int32_t k = 0; k < n_steps; ++k) {
    st = bz_step2d(g, f, src, &m, step0 + k, nullptr, stream);
    if (st != BZ_OK) return st;
    const int64_t done = step0 + k + 1;
    if (done - folded >= ring_len) {
      st = bz_dft_fold(ring, g->dtype, ring_len, items, n_freq, phasor, n_phasor, folded, (int32_t)(done - folded),
                       dft, stream);
      if (st != BZ_OK) return st;
      folded = done;
    }
  }
  if (folded < step0 + n_steps)
    return bz_dft_fold(ring, g->dtype, ring_len, items, n_freq, phasor, n_phasor, folded,
                       (int32_t)(step0 + n_steps - folded), dft, stream);
  return BZ_OK;
}
