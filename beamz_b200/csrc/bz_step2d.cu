// 2D Ez-mode Yee time step, fused: H update, E update (PEC ring), source
// injection, optional |S|^2 accumulation, monitor sampling.
//
// Reference semantics (beamz project paths):
//   H update  beamz/simulation/backends/numpy_backend.py:34-61
//   E update  beamz/simulation/backends/numpy_backend.py:63-88
//   sources   beamz/simulation/helper.py:5-118 (applied after the E update)
//   power     beamz/simulation/helper.py:152-187
//   monitors  beamz/simulation/helper.py:245-256, beamz/devices/monitors.py:279-315
//
// Data layout: every field is [design][component][ny][pitch] with x contiguous.
// Ping-pong: the launch reads the *_in copies and writes the *_out copies, so
// blocks never see a neighbour's half-updated values. One thread owns one column
// x of a tile of RB rows and marches along y, carrying Ez(y) and the new Hy(y-1)
// in registers; Ez(y, x+1) and the new Hx(y, x-1) come from the neighbouring
// lanes by warp shuffles (warp-edge lanes read/recompute them from global
// memory). The row loop is fully unrolled so the loads of later rows issue
// before the arithmetic of earlier ones.
//
// After the tile is written, the block applies the source and monitor
// operations that fall inside it, spread over all its threads.
#include "bz_stencil.cuh"

namespace bz {
namespace {

constexpr int BX = 128;  // threads (columns) per block
constexpr unsigned FULL = 0xffffffffu;

template <typename T>
struct Geo2D {
  int nx, ny, pitch, n_designs, n_mat;
  long long plane;  // ny * pitch
  T chx, chy, qy, inv_kd2;
};

template <typename T>
struct Ops2D {
  int n_src, src_steps;
  const int* src_row;
  const int* src_cell;
  const T* src_mul;
  const T* src_w;
  long long w_stride;
  const int* src_sig;
  const T* signals;
  int n_mon, ring_len;
  const int* mon_row;
  const int* mon_cell;
  const int* mon_point;
  T* record;
  long long rec_step0;
  int n_rec;
  T* ring;
  T* region;
  int rx0, ry0, rw, rh, n_reg;
  long long reg_step0;
};

template <typename T>
__device__ __forceinline__ double sq_pow(const T* ez, const T* hx, const T* hy, int nc) {
  // |S|^2 with Sx = -sum_c Ez*Hy, Sy = sum_c Ez*Hx (helper.py:171-179)
  double sx = 0.0, sy = 0.0;
  for (int c = 0; c < nc; ++c) {
    sx -= (double)ez[c] * (double)hy[c];
    sy += (double)ez[c] * (double)hx[c];
  }
  return sx * sx + sy * sy;
}

template <typename T, int NC, bool PWR, int RB>
__global__ void __launch_bounds__(BX) step2d_kernel(
    const T* __restrict__ ez_in, const T* __restrict__ hx_in, const T* __restrict__ hy_in,
    T* __restrict__ ez_out, T* __restrict__ hx_out, T* __restrict__ hy_out,
    const T* __restrict__ ce, const T* __restrict__ loss, double* __restrict__ pwr,
    Geo2D<T> g, Ops2D<T> o, long long step_base, const long long* __restrict__ d_step) {
  const long long step = d_step ? (__ldg(d_step) + step_base) : step_base;
  const int nx = g.nx, ny = g.ny, pitch = g.pitch;
  const int x = blockIdx.x * BX + threadIdx.x;
  const int wl = threadIdx.x & 31;
  const int d = blockIdx.z;
  const int y0 = blockIdx.y * RB;
  const int nrows = min(RB, ny - y0);
  const bool xin = x < nx;
  const long long fb = (long long)d * NC * g.plane;
  const long long mb = (g.n_mat > 1 ? (long long)d : 0LL) * g.plane;
  const T* __restrict__ cep = ce + mb;
  const T* __restrict__ lsp = loss + mb;

  T ezc[NC], hyp[NC];
#pragma unroll
  for (int c = 0; c < NC; ++c) {
    ezc[c] = xin ? __ldg(ez_in + fb + c * g.plane + (long long)y0 * pitch + x) : T(0);
    hyp[c] = T(0);
  }
  if (y0 >= 1) {
    // New Hy(y0-1, x): needed by the E update of row y0, owned by the tile above.
    const long long r = (long long)(y0 - 1) * pitch + x;
    T fh, cx, cy;
    h_coeffs(xin ? __ldg(lsp + r) : T(0), g.chx, g.chy, fh, cx, cy);
#pragma unroll
    for (int c = 0; c < NC; ++c) {
      const long long off = fb + c * g.plane + r;
      const T ezm = xin ? __ldg(ez_in + off) : T(0);
      const T hy = xin ? __ldg(hy_in + off) : T(0);
      hyp[c] = fh * hy + cy * (ezc[c] - ezm);
    }
  }

#pragma unroll
  for (int i = 0; i < RB; ++i) {
    const int y = y0 + i;
    if (i < nrows) {  // uniform across the block
      const long long r = (long long)y * pitch + x;
      const T a = xin ? __ldg(lsp + r) : T(0);
      const T cec = xin ? __ldg(cep + r) : T(0);
      T fh, cx, cy;
      h_coeffs(a, g.chx, g.chy, fh, cx, cy);
      // Warp-edge lane 0 recomputes the new Hx(y, x-1) of the lane to its left.
      const bool left_fix = (wl == 0) && xin && x >= 1;
      T fhl = T(0), cxl = T(0), cyl;
      if (left_fix) h_coeffs(__ldg(lsp + r - 1), g.chx, g.chy, fhl, cxl, cyl);
      const bool interior = (x >= 1) && (x <= nx - 2) && (y >= 1) && (y <= ny - 2);
      const T fe = T(1) - a * cec * g.inv_kd2;
      T ezo[NC], hxo[NC], hyo[NC];
#pragma unroll
      for (int c = 0; c < NC; ++c) {
        const T* __restrict__ E = ez_in + fb + c * g.plane;
        const T ezn = (xin && y + 1 < ny) ? __ldg(E + r + pitch) : T(0);
        T ezr = __shfl_down_sync(FULL, ezc[c], 1);
        if (wl == 31) ezr = (x + 1 < nx) ? __ldg(E + r + 1) : T(0);
        const T hx0 = xin ? __ldg(hx_in + fb + c * g.plane + r) : T(0);
        const T hy0 = xin ? __ldg(hy_in + fb + c * g.plane + r) : T(0);
        const T hxn = fh * hx0 - cx * (ezr - ezc[c]);
        const T hyn = fh * hy0 + cy * (ezn - ezc[c]);
        T hxl = __shfl_up_sync(FULL, hxn, 1);
        if (left_fix) {
          const T hxl0 = __ldg(hx_in + fb + c * g.plane + r - 1);
          hxl = fhl * hxl0 - cxl * (ezc[c] - __ldg(E + r - 1));
        }
        T ez_new = ezc[c];
        if (interior) ez_new = fe * ezc[c] + cec * (-(hxn - hxl) + g.qy * (hyn - hyp[c]));
        ezo[c] = ez_new;
        hxo[c] = (x < nx - 1) ? hxn : T(0);
        hyo[c] = (y < ny - 1) ? hyn : T(0);
        if (xin) {
          const long long off = fb + c * g.plane + r;
          ez_out[off] = ez_new;
          if (x < nx - 1) hx_out[off] = hxn;
          if (y < ny - 1) hy_out[off] = hyn;
        }
        ezc[c] = ezn;
        hyp[c] = hyn;
      }
      if (PWR && xin) pwr[(long long)d * g.plane + r] += sq_pow<T>(ezo, hxo, hyo, NC);
      if (o.region != nullptr) {  // Ez after this step inside the capture box
        const long long slot = step + 1 - o.reg_step0;
        const int rx = x - o.rx0, ry = y - o.ry0;
        if (slot >= 1 && slot < o.n_reg && rx >= 0 && rx < o.rw && ry >= 0 && ry < o.rh) {
#pragma unroll
          for (int c = 0; c < NC; ++c)
            o.region[(((slot * g.n_designs + d) * NC + c) * o.rh + ry) * (long long)o.rw + rx] = ezo[c];
        }
      }
    }
  }

  if (o.n_src == 0 && o.n_mon == 0) return;  // uniform across the grid
  // ---- post phase: operations on cells of this block's tile -----------------
  __shared__ int s_k0[RB], s_pre[RB + 1];
  const int xlo = blockIdx.x * BX;
  const int xhi = min(xlo + BX, nx);
  __syncthreads();  // this block's field writes are now visible to all its threads
  if (o.n_src > 0) {
    const int total = block_op_ranges(o.src_row, o.src_cell, y0, nrows, nx, xlo, xhi, s_k0, s_pre);
    for (int i = threadIdx.x; i < total; i += BX) {
      int t;
      const int k = op_at(i, nrows, s_k0, s_pre, t);
      const int cell = __ldg(o.src_cell + k);
      if (i > s_pre[t] && __ldg(o.src_cell + k - 1) == cell) continue;  // not first of its cell's run
      const int y = y0 + t;
      const long long rr = (long long)y * pitch + (cell - y * nx);
      T e[NC], hx[NC], hy[NC];
#pragma unroll
      for (int c = 0; c < NC; ++c) {
        e[c] = ez_out[fb + c * g.plane + rr];
        hx[c] = hx_out[fb + c * g.plane + rr];
        hy[c] = hy_out[fb + c * g.plane + rr];
      }
      double p_old = 0.0;
      if (PWR) p_old = sq_pow<T>(e, hx, hy, NC);
      for (int kk = k; kk < o.n_src && __ldg(o.src_cell + kk) == cell; ++kk) {
        const T m = __ldg(o.src_mul + kk);
        const int sg = __ldg(o.src_sig + kk);
        const T s = (step < o.src_steps) ? __ldg(o.signals + (long long)sg * o.src_steps + step) : T(0);
#pragma unroll
        for (int c = 0; c < NC; ++c) e[c] = m * e[c] + __ldg(o.src_w + d * o.w_stride + (long long)kk * NC + c) * s;
      }
#pragma unroll
      for (int c = 0; c < NC; ++c) ez_out[fb + c * g.plane + rr] = e[c];
      if (PWR) {
        double* pp = pwr + (long long)d * g.plane + rr;
        *pp = (*pp - p_old) + sq_pow<T>(e, hx, hy, NC);
      }
    }
    __syncthreads();
  }
  if (o.n_mon > 0) {
    const int total = block_op_ranges(o.mon_row, o.mon_cell, y0, nrows, nx, xlo, xhi, s_k0, s_pre);
    const bool rec = o.record != nullptr && step >= o.rec_step0 && step < o.rec_step0 + o.n_rec;
    const long long slot = o.ring != nullptr ? step % o.ring_len : 0;
    for (int i = threadIdx.x; i < total; i += BX) {
      int t;
      const int k = op_at(i, nrows, s_k0, s_pre, t);
      const int cell = __ldg(o.mon_cell + k);
      const int p = __ldg(o.mon_point + k);
      const int y = y0 + t;
      const int xx = cell - y * nx;
      const long long rr = (long long)y * pitch + xx;
#pragma unroll
      for (int c = 0; c < NC; ++c) {
        const long long off = fb + c * g.plane + rr;
        const T ez = ez_out[off];
        const T hx = hx_out[off];
        const T hy = hy_out[off];
        if (rec) {
          T* dst = o.record + ((((step - o.rec_step0) * g.n_designs + d) * NC + c) * (long long)o.n_mon + p) * 3;
          dst[0] = ez;
          dst[1] = hx;
          dst[2] = hy;
        }
        if (o.ring) {
          T* q = o.ring + (((slot * g.n_designs + d) * NC + c) * (long long)o.n_mon + p) * 5;
          q[0] = ez;
          q[1] = hx;
          q[2] = xx >= 1 ? hx_out[off - 1] : T(0);
          q[3] = hy;
          q[4] = y >= 1 ? hy_out[off - pitch] : T(0);
        }
      }
    }
  }
}

template <typename T, int NC, bool PWR, int RB>
int launch(const bz_grid2d* gd, const bz_fields2d* f, const bz_source_ops* s, const bz_monitor_ops* m,
           int64_t step, const int64_t* d_step, cudaStream_t st) {
  Geo2D<T> g;
  g.nx = gd->nx;
  g.ny = gd->ny;
  g.pitch = gd->pitch;
  g.n_designs = gd->n_designs;
  g.n_mat = gd->n_mat;
  g.plane = (long long)gd->ny * gd->pitch;
  g.chx = (T)gd->chx;
  g.chy = (T)gd->chy;
  g.qy = (T)gd->qy;
  g.inv_kd2 = (T)gd->inv_kd2;
  Ops2D<T> o = {};
  if (s && s->n_ops > 0) {
    o.n_src = s->n_ops;
    o.src_steps = s->n_steps;
    o.src_row = s->row_ptr;
    o.src_cell = s->cell;
    o.src_mul = (const T*)s->mul;
    o.src_w = (const T*)s->weight;
    o.w_stride = s->weight_stride;
    o.src_sig = s->sig;
    o.signals = (const T*)s->signals;
  }
  if (m && m->n_points > 0 && (m->record || m->ring)) {
    o.n_mon = m->n_points;
    o.ring_len = m->ring_len;
    o.mon_row = m->row_ptr;
    o.mon_cell = m->cell;
    o.mon_point = m->point;
    o.record = (T*)m->record;
    o.rec_step0 = m->rec_step0;
    o.n_rec = m->n_rec;
    o.ring = (T*)m->ring;
  }
  if (m && m->region && m->n_reg > 1) {
    o.region = (T*)m->region;
    o.rx0 = m->rx0;
    o.ry0 = m->ry0;
    o.rw = m->rw;
    o.rh = m->rh;
    o.n_reg = m->n_reg;
    o.reg_step0 = m->reg_step0;
  }
  const int src = (int)(step & 1);  // copy read by this launch: parity of the host-side step argument
  dim3 grid((unsigned)ceil_div(gd->nx, BX), (unsigned)ceil_div(gd->ny, RB), (unsigned)gd->n_designs);
  step2d_kernel<T, NC, PWR, RB><<<grid, BX, 0, st>>>(
      (const T*)f->ez[src], (const T*)f->hx[src], (const T*)f->hy[src], (T*)f->ez[src ^ 1], (T*)f->hx[src ^ 1],
      (T*)f->hy[src ^ 1], (const T*)f->ce, (const T*)f->loss, f->power, g, o, (long long)step,
      (const long long*)d_step);
  return check_launch("bz_step2d");
}

template <typename T, int NC, bool PWR>
int by_rows(const bz_grid2d* g, const bz_fields2d* f, const bz_source_ops* s, const bz_monitor_ops* m,
            int64_t step, const int64_t* d_step, cudaStream_t st) {
  switch (g->tile_rows) {
    case 4: return launch<T, NC, PWR, 4>(g, f, s, m, step, d_step, st);
    case 8: return launch<T, NC, PWR, 8>(g, f, s, m, step, d_step, st);
    case 32: return launch<T, NC, PWR, 32>(g, f, s, m, step, d_step, st);
    default: return launch<T, NC, PWR, 16>(g, f, s, m, step, d_step, st);
  }
}

template <typename T>
int dispatch(const bz_grid2d* g, const bz_fields2d* f, const bz_source_ops* s, const bz_monitor_ops* m,
             int64_t step, const int64_t* d_step, cudaStream_t st) {
  const bool pw = f->power != nullptr;
  if (g->n_comp == 1) return pw ? by_rows<T, 1, true>(g, f, s, m, step, d_step, st) : by_rows<T, 1, false>(g, f, s, m, step, d_step, st);
  return pw ? by_rows<T, 2, true>(g, f, s, m, step, d_step, st) : by_rows<T, 2, false>(g, f, s, m, step, d_step, st);
}

}  // namespace
}  // namespace bz

extern "C" int bz_step2d(const bz_grid2d* g, const bz_fields2d* f, const bz_source_ops* s,
                         const bz_monitor_ops* m, int64_t step, const int64_t* d_step, void* stream) {
  BZ_REQUIRE(g && f, "bz_step2d: grid or fields is NULL");
  BZ_REQUIRE(g->nx >= 2 && g->ny >= 2, "bz_step2d: grid must be at least 2x2 (got %d x %d)", g->nx, g->ny);
  BZ_REQUIRE(g->pitch >= g->nx && g->pitch % 32 == 0, "bz_step2d: pitch %d must be >= nx and a multiple of 32",
             g->pitch);
  BZ_REQUIRE(g->n_designs >= 1 && g->n_designs <= 65535, "bz_step2d: n_designs %d out of range", g->n_designs);
  BZ_REQUIRE(g->n_comp == 1 || g->n_comp == 2, "bz_step2d: n_comp must be 1 or 2 (got %d)", g->n_comp);
  BZ_REQUIRE(g->n_mat == 1 || g->n_mat == g->n_designs, "bz_step2d: n_mat must be 1 or n_designs");
  BZ_REQUIRE(g->dtype == BZ_F32 || g->dtype == BZ_F64, "bz_step2d: unknown dtype %d", g->dtype);
  BZ_REQUIRE(g->tile_rows == 0 || g->tile_rows == 4 || g->tile_rows == 8 || g->tile_rows == 16 || g->tile_rows == 32,
             "bz_step2d: tile_rows must be 0, 4, 8, 16 or 32 (got %d)", g->tile_rows);
  for (int i = 0; i < 2; ++i)
    BZ_REQUIRE(f->ez[i] && f->hx[i] && f->hy[i], "bz_step2d: field buffer %d is NULL", i);
  BZ_REQUIRE(f->ce && f->loss, "bz_step2d: coefficient arrays are NULL");
  BZ_REQUIRE(step >= 0, "bz_step2d: negative step");
  if (s && s->n_ops > 0)
    BZ_REQUIRE(s->row_ptr && s->cell && s->mul && s->weight && s->sig && s->signals && s->n_steps >= 0,
               "bz_step2d: incomplete source ops");
  if (m && m->region) BZ_REQUIRE(m->rw >= 1 && m->rh >= 1 && m->n_reg >= 1, "bz_step2d: bad capture box");
  if (m && m->n_points > 0) {
    BZ_REQUIRE(m->row_ptr && m->cell && m->point, "bz_step2d: incomplete monitor ops");
    BZ_REQUIRE(m->ring == nullptr || m->ring_len >= 1, "bz_step2d: ring without length");
    BZ_REQUIRE(m->record == nullptr || m->n_rec >= 0, "bz_step2d: bad record length");
  }
  cudaStream_t st = bz::as_stream(stream);
  return g->dtype == BZ_F32 ? bz::dispatch<float>(g, f, s, m, step, d_step, st)
                            : bz::dispatch<double>(g, f, s, m, step, d_step, st);
}
