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
      hyp[c] = hy_update(fh, hy, cy, ezc[c], ezm);
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
      const T fe = sub_rn(T(1), mul_rn(mul_rn(a, cec), g.inv_kd2));
      T ezo[NC], hxo[NC], hyo[NC];
#pragma unroll
      for (int c = 0; c < NC; ++c) {
        const T* __restrict__ E = ez_in + fb + c * g.plane;
        const T ezn = (xin && y + 1 < ny) ? __ldg(E + r + pitch) : T(0);
        T ezr = __shfl_down_sync(FULL, ezc[c], 1);
        if (wl == 31) ezr = (x + 1 < nx) ? __ldg(E + r + 1) : T(0);
        const T hx0 = xin ? __ldg(hx_in + fb + c * g.plane + r) : T(0);
        const T hy0 = xin ? __ldg(hy_in + fb + c * g.plane + r) : T(0);
        const T hxn = hx_update(fh, hx0, cx, ezr, ezc[c]);
        const T hyn = hy_update(fh, hy0, cy, ezn, ezc[c]);
        T hxl = __shfl_up_sync(FULL, hxn, 1);
        if (left_fix) {
          const T hxl0 = __ldg(hx_in + fb + c * g.plane + r - 1);
          hxl = hx_update(fhl, hxl0, cxl, ezc[c], __ldg(E + r - 1));
        }
        T ez_new = ezc[c];
        if (interior) ez_new = ez_update(fe, ezc[c], cec, g.qy, hxn, hxl, hyn, hyp[c]);
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
        for (int c = 0; c < NC; ++c) e[c] = fma_rn(m, e[c], mul_rn(__ldg(o.src_w + d * o.w_stride + (long long)kk * NC + c), s));
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
          // The new Hx(x-1) and Hy(y-1) may belong to another block of this launch, so
          // they are recomputed from the step's inputs (same arithmetic as their owner).
          const T* __restrict__ E = ez_in + fb + c * g.plane;
          T hxl = T(0), hyu = T(0);
          if (xx >= 1) {
            T fh, cx, cy;
            h_coeffs(__ldg(lsp + rr - 1), g.chx, g.chy, fh, cx, cy);
            hxl = hx_update(fh, __ldg(hx_in + off - 1), cx, __ldg(E + rr), __ldg(E + rr - 1));
          }
          if (y >= 1) {
            T fh, cx, cy;
            h_coeffs(__ldg(lsp + rr - pitch), g.chx, g.chy, fh, cx, cy);
            hyu = hy_update(fh, __ldg(hy_in + off - pitch), cy, __ldg(E + rr), __ldg(E + rr - pitch));
          }
          T* q = o.ring + (((slot * g.n_designs + d) * NC + c) * (long long)o.n_mon + p) * 5;
          q[0] = ez;
          q[1] = hx;
          q[2] = hxl;
          q[3] = hy;
          q[4] = hyu;
        }
      }
    }
  }
}

// ---- temporal blocking ---------------------------------------------------------
// step2d_tb_kernel advances TS (odd) steps per launch. A block holds a tile of 64
// columns x NW*R rows in registers: lane l of warp w owns columns X0+l and X0+32+l
// (coalesced loads) of rows Y0+w*R .. Y0+w*R+R-1, together with their update
// factors. Each sub-step is the single-step update restricted to the tile; the
// values next to the tile's edges go stale by one cell per sub-step, so after TS
// sub-steps the tile minus TS cells on every side (the owned box, which tiles the
// grid) is exact, and only it is stored. x neighbours come from shuffles, the rows
// across warps from shared memory (two barriers per sub-step). Sources act on every
// tile cell (halo cells have to evolve like the real ones); monitors sample owned
// cells only. Reads copy (step & 1) and writes the other, like TS single steps.
template <typename T, int NC, int TS, int R, int NW>
__global__ void __launch_bounds__(32 * NW) step2d_tb_kernel(
    const T* __restrict__ ez_in, const T* __restrict__ hx_in, const T* __restrict__ hy_in,
    T* __restrict__ ez_out, T* __restrict__ hx_out, T* __restrict__ hy_out,
    const T* __restrict__ ce, const T* __restrict__ loss, Geo2D<T> g, Ops2D<T> o, long long step_base,
    const long long* __restrict__ d_step) {
  constexpr int TW = 64, TH = NW * R;
  constexpr int OW = TW - 2 * TS, OH = TH - 2 * TS;
  static_assert(TS % 2 == 1 && OH > 0 && R * 2 <= 32, "bad temporal tile");
  const long long step0 = d_step ? (__ldg(d_step) + step_base) : step_base;
  const int nx = g.nx, ny = g.ny, pitch = g.pitch;
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  const int d = blockIdx.z;
  const int X0 = (int)blockIdx.x * OW - TS, Y0 = (int)blockIdx.y * OH - TS;
  const int yb = Y0 + w * R;
  const long long fb = (long long)d * NC * g.plane;
  const long long mb = (g.n_mat > 1 ? (long long)d : 0LL) * g.plane;

  __shared__ T s_top[NW][NC][TW];  // first row's Ez of each warp, before the H update
  __shared__ T s_bot[NW][NC][TW];  // last row's new Hy of each warp
  __shared__ int s_src[TH][2], s_mon[TH][2];  // op ranges of each tile row

  // row pointers of the op lists first, so their latency overlaps the tile loads
  int rs_lo = 0, rs_hi = 0, rm_lo = 0, rm_hi = 0;
  if (lane < R) {
    const int y = yb + lane;
    if (y >= 0 && y < ny) {
      if (o.n_src > 0) {
        rs_lo = __ldg(o.src_row + y);
        rs_hi = __ldg(o.src_row + y + 1);
      }
      if (o.n_mon > 0) {
        rm_lo = __ldg(o.mon_row + y);
        rm_hi = __ldg(o.mon_row + y + 1);
      }
    }
  }

  int xs[2];
  xs[0] = X0 + lane;
  xs[1] = X0 + 32 + lane;
  T ez[R][2][NC], hx[R][2][NC], hy[R][2][NC];
  // Cells whose H or E the reference never changes (Hx in the last column, Hy in the
  // last row, E on the PEC ring, everything outside the grid) get factors that keep
  // the value: cx = 0 / cy = 0 for H (those values start and stay zero), fe = 1 and
  // ce = 0 for E. The sub-step loop then needs no per-cell masks.
  T fh[R][2], cx[R][2], cy[R][2], fe[R][2], cc[R][2];
#pragma unroll
  for (int i = 0; i < R; ++i) {
    const int y = yb + i;
#pragma unroll
    for (int j = 0; j < 2; ++j) {
      const int x = xs[j];
      const bool in = x >= 0 && x < nx && y >= 0 && y < ny;
      const long long r = in ? (long long)y * pitch + x : 0LL;
      const T a = in ? __ldg(loss + mb + r) : T(0);
      const T c = in ? __ldg(ce + mb + r) : T(0);
      h_coeffs(a, g.chx, g.chy, fh[i][j], cx[i][j], cy[i][j]);
      const bool interior = x >= 1 && x <= nx - 2 && y >= 1 && y <= ny - 2;
      fe[i][j] = interior ? sub_rn(T(1), mul_rn(mul_rn(a, c), g.inv_kd2)) : T(1);
      cc[i][j] = interior ? c : T(0);
      if (!(in && x < nx - 1)) cx[i][j] = T(0);
      if (!(in && y < ny - 1)) cy[i][j] = T(0);
#pragma unroll
      for (int k = 0; k < NC; ++k) {
        const long long off = fb + k * g.plane + r;
        ez[i][j][k] = in ? __ldg(ez_in + off) : T(0);
        hx[i][j][k] = (in && x < nx - 1) ? __ldg(hx_in + off) : T(0);
        hy[i][j][k] = (in && y < ny - 1) ? __ldg(hy_in + off) : T(0);
      }
    }
  }
  // Operation ranges: sources over the tile's columns, monitors over the owned ones.
  if (lane < R) {
    const int y = yb + lane, tr = w * R + lane;
    int s0 = 0, s1 = 0, m0 = 0, m1 = 0;
    if (y >= 0 && y < ny) {
      if (o.n_src > 0) {
        const int lo = rs_lo, hi = rs_hi;
        if (lo < hi) {
          s0 = lower_bound_i(o.src_cell, lo, hi, y * nx + max(X0, 0));
          s1 = lower_bound_i(o.src_cell, s0, hi, y * nx + min(X0 + TW, nx));
        }
      }
      if (o.n_mon > 0 && tr >= TS && tr < TH - TS) {
        const int lo = rm_lo, hi = rm_hi;
        if (lo < hi) {
          m0 = lower_bound_i(o.mon_cell, lo, hi, y * nx + X0 + TS);
          m1 = lower_bound_i(o.mon_cell, m0, hi, y * nx + min(X0 + TW - TS, nx));
        }
      }
    }
    s_src[tr][0] = s0;
    s_src[tr][1] = s1;
    s_mon[tr][0] = m0;
    s_mon[tr][1] = m1;
  }
  __syncwarp();
  unsigned src_rows = 0u, mon_rows = 0u;
#pragma unroll
  for (int i = 0; i < R; ++i) {
    if (s_src[w * R + i][0] < s_src[w * R + i][1]) src_rows |= 1u << i;
    if (s_mon[w * R + i][0] < s_mon[w * R + i][1]) mon_rows |= 1u << i;
  }
  bool own[2];
  own[0] = lane >= TS && xs[0] < nx;
  own[1] = lane < 32 - TS && xs[1] < nx;
  // owned cells inside the capture box (adjoint recompute): bit i*2+j
  unsigned cap = 0u;
  if (o.region != nullptr) {
#pragma unroll
    for (int i = 0; i < R; ++i) {
      const int tr = w * R + i, y = yb + i;
#pragma unroll
      for (int j = 0; j < 2; ++j) {
        const int rx = xs[j] - o.rx0, ry = y - o.ry0;
        if (own[j] && tr >= TS && tr < TH - TS && y < ny && rx >= 0 && rx < o.rw && ry >= 0 && ry < o.rh)
          cap |= 1u << (i * 2 + j);
      }
    }
  }

#pragma unroll 1
  for (int s = 0; s < TS; ++s) {
    const long long step = step0 + s;
#pragma unroll
    for (int j = 0; j < 2; ++j)
#pragma unroll
      for (int k = 0; k < NC; ++k) s_top[w][k][j * 32 + lane] = ez[0][j][k];
    __syncthreads();
    // H update: Ez(x+1) by shuffle, Ez(y+1) from the next row (or warp)
#pragma unroll
    for (int i = 0; i < R; ++i) {
#pragma unroll
      for (int k = 0; k < NC; ++k) {
        const T r0 = __shfl_sync(FULL, ez[i][0][k], (lane + 1) & 31);
        const T r1 = __shfl_sync(FULL, ez[i][1][k], (lane + 1) & 31);
        T er[2], ed[2];
        er[0] = lane == 31 ? r1 : r0;  // right of column 31 is column 32
        er[1] = r1;                    // lane 31: beyond the tile (stale halo)
        if (i + 1 < R) {
          ed[0] = ez[i + 1][0][k];
          ed[1] = ez[i + 1][1][k];
        } else if (w + 1 < NW) {
          ed[0] = s_top[w + 1][k][lane];
          ed[1] = s_top[w + 1][k][32 + lane];
        } else {
          ed[0] = ed[1] = T(0);
        }
#pragma unroll
        for (int j = 0; j < 2; ++j) {
          hx[i][j][k] = hx_update(fh[i][j], hx[i][j][k], cx[i][j], er[j], ez[i][j][k]);
          hy[i][j][k] = hy_update(fh[i][j], hy[i][j][k], cy[i][j], ed[j], ez[i][j][k]);
        }
      }
    }
#pragma unroll
    for (int j = 0; j < 2; ++j)
#pragma unroll
      for (int k = 0; k < NC; ++k) s_bot[w][k][j * 32 + lane] = hy[R - 1][j][k];
    __syncthreads();
    // E update (interior): Hx(x-1) by shuffle, Hy(y-1) from the previous row (or warp)
#pragma unroll
    for (int i = 0; i < R; ++i) {
#pragma unroll
      for (int k = 0; k < NC; ++k) {
        const T l0 = __shfl_sync(FULL, hx[i][0][k], (lane + 31) & 31);
        const T l1 = __shfl_sync(FULL, hx[i][1][k], (lane + 31) & 31);
        T hl[2], hu[2];
        hl[0] = l0;  // lane 0: beyond the tile (stale halo)
        hl[1] = lane == 0 ? l0 : l1;
        if (i > 0) {
          hu[0] = hy[i - 1][0][k];
          hu[1] = hy[i - 1][1][k];
        } else if (w > 0) {
          hu[0] = s_bot[w - 1][k][lane];
          hu[1] = s_bot[w - 1][k][32 + lane];
        } else {
          hu[0] = hu[1] = T(0);
        }
#pragma unroll
        for (int j = 0; j < 2; ++j)
          ez[i][j][k] = ez_update(fe[i][j], ez[i][j][k], cc[i][j], g.qy, hx[i][j][k], hl[j], hy[i][j][k], hu[j]);
      }
    }
    // Sources (helper.py:5-118), in operation order per cell
    if (src_rows) {
#pragma unroll
      for (int i = 0; i < R; ++i) {
        if (!(src_rows & (1u << i))) continue;  // uniform across the warp
        const int y = yb + i;
        const int k0 = s_src[w * R + i][0], k1 = s_src[w * R + i][1];
        for (int kk = k0; kk < k1; ++kk) {
          const int xo = __ldg(o.src_cell + kk) - y * nx;
          if (xo != xs[0] && xo != xs[1]) continue;
          const T m = __ldg(o.src_mul + kk);
          const int sg = __ldg(o.src_sig + kk);
          const T sv = (step < o.src_steps) ? __ldg(o.signals + (long long)sg * o.src_steps + step) : T(0);
#pragma unroll
          for (int k = 0; k < NC; ++k) {
            const T wv = __ldg(o.src_w + d * o.w_stride + (long long)kk * NC + k);
#pragma unroll
            for (int j = 0; j < 2; ++j)
              if (xo == xs[j]) ez[i][j][k] = fma_rn(m, ez[i][j][k], mul_rn(wv, sv));
          }
        }
      }
    }
    // Ez after this sub-step inside the capture box (the box holds no sources)
    if (cap) {
      const long long slot = step + 1 - o.reg_step0;
      if (slot >= 1 && slot < o.n_reg) {
#pragma unroll
        for (int i = 0; i < R; ++i)
#pragma unroll
          for (int j = 0; j < 2; ++j)
            if (cap & (1u << (i * 2 + j))) {
              const int rx = xs[j] - o.rx0, ry = yb + i - o.ry0;
#pragma unroll
              for (int k = 0; k < NC; ++k)
                o.region[(((slot * g.n_designs + d) * NC + k) * o.rh + ry) * (long long)o.rw + rx] = ez[i][j][k];
            }
      }
    }
    // Monitor samples of owned cells: record and DFT ring
    if (mon_rows) {
      const long long slot = o.ring != nullptr ? step % o.ring_len : 0;
      const bool rec = o.record != nullptr && step >= o.rec_step0 && step < o.rec_step0 + o.n_rec;
#pragma unroll
      for (int i = 0; i < R; ++i) {
        if (!(mon_rows & (1u << i))) continue;  // uniform across the warp
        const int y = yb + i;
        T hl[2][NC], hu[2][NC];
#pragma unroll
        for (int k = 0; k < NC; ++k) {
          const T l0 = __shfl_sync(FULL, hx[i][0][k], (lane + 31) & 31);
          const T l1 = __shfl_sync(FULL, hx[i][1][k], (lane + 31) & 31);
          hl[0][k] = l0;
          hl[1][k] = lane == 0 ? l0 : l1;
#pragma unroll
          for (int j = 0; j < 2; ++j) hu[j][k] = i > 0 ? hy[i - 1][j][k] : (w > 0 ? s_bot[w - 1][k][j * 32 + lane] : T(0));
        }
        const int k0 = s_mon[w * R + i][0], k1 = s_mon[w * R + i][1];
        for (int kk = k0; kk < k1; ++kk) {
          const int xo = __ldg(o.mon_cell + kk) - y * nx;
          const int p = __ldg(o.mon_point + kk);
#pragma unroll
          for (int j = 0; j < 2; ++j) {
            if (xo != xs[j] || !own[j]) continue;
#pragma unroll
            for (int k = 0; k < NC; ++k) {
              if (rec) {
                T* dst = o.record + ((((step - o.rec_step0) * g.n_designs + d) * NC + k) * (long long)o.n_mon + p) * 3;
                dst[0] = ez[i][j][k];
                dst[1] = hx[i][j][k];
                dst[2] = hy[i][j][k];
              }
              if (o.ring) {
                T* q = o.ring + (((slot * g.n_designs + d) * NC + k) * (long long)o.n_mon + p) * 5;
                q[0] = ez[i][j][k];
                q[1] = hx[i][j][k];
                q[2] = xo >= 1 ? hl[j][k] : T(0);
                q[3] = hy[i][j][k];
                q[4] = y >= 1 ? hu[j][k] : T(0);
              }
            }
          }
        }
      }
    }
  }
  // Store the owned box
#pragma unroll
  for (int i = 0; i < R; ++i) {
    const int tr = w * R + i, y = yb + i;
    if (tr < TS || tr >= TH - TS || y >= ny) continue;
#pragma unroll
    for (int j = 0; j < 2; ++j) {
      const int x = xs[j];
      if (!own[j]) continue;
      const long long r = (long long)y * pitch + x;
#pragma unroll
      for (int k = 0; k < NC; ++k) {
        const long long off = fb + k * g.plane + r;
        ez_out[off] = ez[i][j][k];
        if (x < nx - 1) hx_out[off] = hx[i][j][k];
        if (y < ny - 1) hy_out[off] = hy[i][j][k];
      }
    }
  }
}

template <typename T>
Geo2D<T> make_geo(const bz_grid2d* gd) {
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
  return g;
}

template <typename T>
Ops2D<T> make_ops(const bz_source_ops* s, const bz_monitor_ops* m) {
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
  return o;
}

template <typename T, int NC, int TS, int R, int NW>
int launch_tb(const bz_grid2d* gd, const bz_fields2d* f, const bz_source_ops* s, const bz_monitor_ops* m,
              int64_t step, const int64_t* d_step, cudaStream_t st) {
  constexpr int OW = 64 - 2 * TS, OH = NW * R - 2 * TS;
  const Geo2D<T> g = make_geo<T>(gd);
  Ops2D<T> o = make_ops<T>(s, m);
  if (m && m->region && m->n_reg > 1) {
    o.region = (T*)m->region;
    o.rx0 = m->rx0;
    o.ry0 = m->ry0;
    o.rw = m->rw;
    o.rh = m->rh;
    o.n_reg = m->n_reg;
    o.reg_step0 = m->reg_step0;
  }
  const int src = (int)(step & 1);
  dim3 grid((unsigned)ceil_div(gd->nx, OW), (unsigned)ceil_div(gd->ny, OH), (unsigned)gd->n_designs);
  step2d_tb_kernel<T, NC, TS, R, NW><<<grid, 32 * NW, 0, st>>>(
      (const T*)f->ez[src], (const T*)f->hx[src], (const T*)f->hy[src], (T*)f->ez[src ^ 1], (T*)f->hx[src ^ 1],
      (T*)f->hy[src ^ 1], (const T*)f->ce, (const T*)f->loss, g, o, (long long)step, (const long long*)d_step);
  return check_launch("bz_step2d_multi");
}

// Tile shapes: 1 = 4 rows x 8 warps, 2 = 4 rows x 16 warps, 3 = 8 rows x 8 warps,
// 4 = 5 rows x 16 warps, 5 = 6 rows x 12 warps (float, one component); wider types
// use 2 rows x 16 warps.
template <typename T, int NC, int TS>
int tb_by_tile(const bz_grid2d* g, const bz_fields2d* f, const bz_source_ops* s, const bz_monitor_ops* m,
               int64_t step, int32_t tile, const int64_t* d_step, cudaStream_t st) {
  if constexpr (sizeof(T) == 4 && NC == 1) {
    switch (tile) {
      case 1: return launch_tb<T, NC, TS, 4, 8>(g, f, s, m, step, d_step, st);
      case 3: return launch_tb<T, NC, TS, 8, 8>(g, f, s, m, step, d_step, st);
      case 4: return launch_tb<T, NC, TS, 5, 16>(g, f, s, m, step, d_step, st);
      case 5: return launch_tb<T, NC, TS, 6, 12>(g, f, s, m, step, d_step, st);
      default: return launch_tb<T, NC, TS, 4, 16>(g, f, s, m, step, d_step, st);
    }
  } else {
    return launch_tb<T, NC, TS, 2, 16>(g, f, s, m, step, d_step, st);
  }
}

template <typename T, int NC>
int tb_by_steps(const bz_grid2d* g, const bz_fields2d* f, const bz_source_ops* s, const bz_monitor_ops* m,
                int64_t step, int32_t n_sub, int32_t tile, const int64_t* d_step, cudaStream_t st) {
  switch (n_sub) {
    case 3: return tb_by_tile<T, NC, 3>(g, f, s, m, step, tile, d_step, st);
    case 7: return tb_by_tile<T, NC, 7>(g, f, s, m, step, tile, d_step, st);
    case 9: return tb_by_tile<T, NC, 9>(g, f, s, m, step, tile, d_step, st);
    default: return tb_by_tile<T, NC, 5>(g, f, s, m, step, tile, d_step, st);
  }
}

template <typename T, int NC, bool PWR, int RB>
int launch(const bz_grid2d* gd, const bz_fields2d* f, const bz_source_ops* s, const bz_monitor_ops* m,
           int64_t step, const int64_t* d_step, cudaStream_t st) {
  const Geo2D<T> g = make_geo<T>(gd);
  Ops2D<T> o = make_ops<T>(s, m);
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

namespace bz {
namespace {

int check_step_args(const char* who, const bz_grid2d* g, const bz_fields2d* f, const bz_source_ops* s,
                    const bz_monitor_ops* m, int64_t step) {
  BZ_REQUIRE(g && f, "%s: grid or fields is NULL", who);
  BZ_REQUIRE(g->nx >= 2 && g->ny >= 2, "%s: grid must be at least 2x2 (got %d x %d)", who, g->nx, g->ny);
  BZ_REQUIRE(g->pitch >= g->nx && g->pitch % 32 == 0, "%s: pitch %d must be >= nx and a multiple of 32", who,
             g->pitch);
  BZ_REQUIRE(g->n_designs >= 1 && g->n_designs <= 65535, "%s: n_designs %d out of range", who, g->n_designs);
  BZ_REQUIRE(g->n_comp == 1 || g->n_comp == 2, "%s: n_comp must be 1 or 2 (got %d)", who, g->n_comp);
  BZ_REQUIRE(g->n_mat == 1 || g->n_mat == g->n_designs, "%s: n_mat must be 1 or n_designs", who);
  BZ_REQUIRE(g->dtype == BZ_F32 || g->dtype == BZ_F64, "%s: unknown dtype %d", who, g->dtype);
  for (int i = 0; i < 2; ++i) BZ_REQUIRE(f->ez[i] && f->hx[i] && f->hy[i], "%s: field buffer %d is NULL", who, i);
  BZ_REQUIRE(f->ce && f->loss, "%s: coefficient arrays are NULL", who);
  BZ_REQUIRE(step >= 0, "%s: negative step", who);
  if (s && s->n_ops > 0)
    BZ_REQUIRE(s->row_ptr && s->cell && s->mul && s->weight && s->sig && s->signals && s->n_steps >= 0,
               "%s: incomplete source ops", who);
  if (m && m->region) BZ_REQUIRE(m->rw >= 1 && m->rh >= 1 && m->n_reg >= 1, "%s: bad capture box", who);
  if (m && m->n_points > 0) {
    BZ_REQUIRE(m->row_ptr && m->cell && m->point, "%s: incomplete monitor ops", who);
    BZ_REQUIRE(m->ring == nullptr || m->ring_len >= 1, "%s: ring without length", who);
    BZ_REQUIRE(m->record == nullptr || m->n_rec >= 0, "%s: bad record length", who);
  }
  return BZ_OK;
}

}  // namespace
}  // namespace bz

extern "C" int bz_step2d(const bz_grid2d* g, const bz_fields2d* f, const bz_source_ops* s,
                         const bz_monitor_ops* m, int64_t step, const int64_t* d_step, void* stream) {
  const int rc = bz::check_step_args("bz_step2d", g, f, s, m, step);
  if (rc != BZ_OK) return rc;
  BZ_REQUIRE(g->tile_rows == 0 || g->tile_rows == 4 || g->tile_rows == 8 || g->tile_rows == 16 || g->tile_rows == 32,
             "bz_step2d: tile_rows must be 0, 4, 8, 16 or 32 (got %d)", g->tile_rows);
  cudaStream_t st = bz::as_stream(stream);
  return g->dtype == BZ_F32 ? bz::dispatch<float>(g, f, s, m, step, d_step, st)
                            : bz::dispatch<double>(g, f, s, m, step, d_step, st);
}

extern "C" int bz_step2d_multi(const bz_grid2d* g, const bz_fields2d* f, const bz_source_ops* s,
                               const bz_monitor_ops* m, int64_t step, int32_t n_sub, int32_t tile,
                               const int64_t* d_step, void* stream) {
  const int rc = bz::check_step_args("bz_step2d_multi", g, f, s, m, step);
  if (rc != BZ_OK) return rc;
  BZ_REQUIRE(n_sub == 1 || n_sub == 3 || n_sub == 5 || n_sub == 7 || n_sub == 9,
             "bz_step2d_multi: n_sub must be 1, 3, 5, 7 or 9 (got %d)",
             n_sub);
  BZ_REQUIRE(tile >= 0 && tile <= 5, "bz_step2d_multi: tile must be 0..5 (got %d)", tile);
  if (n_sub == 1) return bz_step2d(g, f, s, m, step, d_step, stream);
  if (f->power != nullptr)
    return bz::fail(BZ_ERR_UNSUPPORTED, "bz_step2d_multi: power accumulation needs bz_step2d");
  cudaStream_t st = bz::as_stream(stream);
  if (g->dtype == BZ_F32)
    return g->n_comp == 1 ? bz::tb_by_steps<float, 1>(g, f, s, m, step, n_sub, tile, d_step, st)
                          : bz::tb_by_steps<float, 2>(g, f, s, m, step, n_sub, tile, d_step, st);
  return g->n_comp == 1 ? bz::tb_by_steps<double, 1>(g, f, s, m, step, n_sub, tile, d_step, st)
                        : bz::tb_by_steps<double, 2>(g, f, s, m, step, n_sub, tile, d_step, st);
}
