// Exact discrete adjoint of the 2D step (bz_step2d), one time step backwards.
//
// Forward step n (coefficients per cell from ce, loss; interior mask I):
//   Hx' = fh*Hx - cx*(E(x+1) - E(x))        Hy' = fh*Hy + cy*(E(y+1) - E(y))
//   Et  = Fe*E + Ce*((Hx'(x-1) - Hx'(x)) - qy*(Hy'(y-1) - Hy'(y)))    Fe = I?fe:1, Ce = I?ce:0
//   E_{n+1} = mul*Et + sources,   J reads E_{n+1} at monitor cells.
// Reverse mode with e = dJ/dEt (already multiplied by mul and fed the objective's
// dJ/dE_{n+1}), and carried adjoints hx, hy of H' from later steps:
//   U   = Ce*e
//   hx' = hx + U(x+1) - U(x)                hy' = hy - qy*(U(y+1) - U(y))
//   wx  = cx*hx',  wy = cy*hy'   (zero where Hx, Hy do not exist)
//   dJ/dE_n = Fe*e - (wx(x-1) - wx(x)) + (wy(y-1) - wy(y))
//   carried: hx <- fh*hx', hy <- fh*hy'
// The data flow mirrors the forward kernel (an H-like pass reading +1 neighbours,
// then an E-like pass reading -1 neighbours), so the same column-march layout is
// used. In the design region (no conductivity) dEt/d eps_r = -(Et - E_n)/eps_r, and
// the kernel accumulates grad += -e*(E_{n+1} - E_n)/eps_r from captured forward
// fields. The post phase then prepares the input of step n-1:
//   e_{n-1} = mul*(dJ/dE_n + objective term), through the same source operations.
#include "bz_stencil.cuh"

namespace bz {
namespace {

constexpr int BX = 128;
constexpr int RB = 16;
constexpr unsigned FULL = 0xffffffffu;

template <typename T>
struct AdjArgs {
  const T* e_in;
  const T* hx_in;
  const T* hy_in;
  T* e_out;
  T* hx_out;
  T* hy_out;
  const T* ce;
  const T* loss;
  int nx, ny, pitch, n_designs, n_mat;
  long long plane;
  T chx, chy, qy, inv_kd2;
  // gradient
  double* grad;
  const double* eps_region;
  const T* fwd;
  int rx0, ry0, rw, rh, n_fwd;
  long long fwd_step0;
  // operations preparing step n-1
  int n_src, src_steps;
  const int* src_row;
  const int* src_cell;
  const T* src_mul;
  const T* src_w;
  long long w_stride;
  const int* src_sig;
  const T* signals;
};

template <typename T>
__device__ __forceinline__ void cell_coeffs(const AdjArgs<T>& a, const T* lsp, const T* cep, long long r, int x,
                                            int y, T& fh, T& cx, T& cy, T& Fe, T& Ce) {
  const T ls = __ldg(lsp + r), c = __ldg(cep + r);
  h_coeffs(ls, a.chx, a.chy, fh, cx, cy);
  const bool interior = x >= 1 && x <= a.nx - 2 && y >= 1 && y <= a.ny - 2;
  Fe = interior ? T(1) - ls * c * a.inv_kd2 : T(1);
  Ce = interior ? c : T(0);
}

template <typename T>
__global__ void __launch_bounds__(BX) adjoint2d_kernel(AdjArgs<T> a, long long step) {
  const int nx = a.nx, ny = a.ny, pitch = a.pitch;
  const int x = blockIdx.x * BX + threadIdx.x;
  const int wl = threadIdx.x & 31;
  const int d = blockIdx.z;
  const int y0 = blockIdx.y * RB;
  const int nrows = min(RB, ny - y0);
  const bool xin = x < nx;
  const long long fb = (long long)d * a.plane;
  const long long mb = (a.n_mat > 1 ? (long long)d : 0LL) * a.plane;
  const T* lsp = a.loss + mb;
  const T* cep = a.ce + mb;
  const T* E = a.e_in + fb;

  // U(y0, x) and the carried wy(y0-1, x) of the row above the tile
  T fh, cx, cy, Fe, Ce;
  T Uc = T(0), wy_up = T(0);
  if (xin) {
    cell_coeffs(a, lsp, cep, (long long)y0 * pitch + x, x, y0, fh, cx, cy, Fe, Ce);
    Uc = Ce * __ldg(E + (long long)y0 * pitch + x);
    if (y0 >= 1) {
      const long long r = (long long)(y0 - 1) * pitch + x;
      T fhm, cxm, cym, Fem, Cem;
      cell_coeffs(a, lsp, cep, r, x, y0 - 1, fhm, cxm, cym, Fem, Cem);
      const T Um = Cem * __ldg(E + r);
      const T hyp = __ldg(a.hy_in + fb + r) - a.qy * (Uc - Um);
      wy_up = cym * hyp;
    }
  }
  for (int i = 0; i < RB; ++i) {
    const int y = y0 + i;
    if (i >= nrows) break;  // uniform across the block
    const long long r = (long long)y * pitch + x;
    T e = T(0);
    if (xin) {
      cell_coeffs(a, lsp, cep, r, x, y, fh, cx, cy, Fe, Ce);
      e = __ldg(E + r);
    }
    T Un = T(0);  // U(y+1, x)
    if (xin && y + 1 < ny) {
      T fh1, cx1, cy1, Fe1, Ce1;
      cell_coeffs(a, lsp, cep, r + pitch, x, y + 1, fh1, cx1, cy1, Fe1, Ce1);
      Un = Ce1 * __ldg(E + r + pitch);
    }
    T Ur = __shfl_down_sync(FULL, Uc, 1);  // U(y, x+1)
    if (wl == 31) {
      Ur = T(0);
      if (x + 1 < nx) {
        T f1, c1, c2, Fe1, Ce1;
        cell_coeffs(a, lsp, cep, r + 1, x + 1, y, f1, c1, c2, Fe1, Ce1);
        Ur = Ce1 * __ldg(E + r + 1);
      }
    }
    const T hx0 = xin ? __ldg(a.hx_in + fb + r) : T(0);
    const T hy0 = xin ? __ldg(a.hy_in + fb + r) : T(0);
    const T hxp = hx0 + (Ur - Uc);
    const T hyp = hy0 - a.qy * (Un - Uc);
    const T wx = (x < nx - 1) ? cx * hxp : T(0);
    const T wy = (y < ny - 1) ? cy * hyp : T(0);
    T wx_left = __shfl_up_sync(FULL, wx, 1);
    if (wl == 0) {
      wx_left = T(0);
      if (xin && x >= 1) {  // recompute wx(y, x-1) of the lane to the left
        T fl, cxl, cyl, Fel, Cel;
        cell_coeffs(a, lsp, cep, r - 1, x - 1, y, fl, cxl, cyl, Fel, Cel);
        const T Ul = Cel * __ldg(E + r - 1);
        wx_left = cxl * (__ldg(a.hx_in + fb + r - 1) + (Uc - Ul));
      }
    }
    if (xin) {
      const T e_prev = Fe * e - (wx_left - wx) + (wy_up - wy);
      a.e_out[fb + r] = e_prev;
      if (x < nx - 1) a.hx_out[fb + r] = fh * hxp;
      if (y < ny - 1) a.hy_out[fb + r] = fh * hyp;
      if (a.grad != nullptr) {
        const int rx = x - a.rx0, ry = y - a.ry0;
        const long long s1 = step + 1 - a.fwd_step0;
        if (rx >= 0 && rx < a.rw && ry >= 0 && ry < a.rh && s1 >= 1 && s1 < a.n_fwd) {
          const long long cell = (long long)ry * a.rw + rx;
          const long long per = (long long)a.n_designs * a.rh * a.rw;
          const double en1 = (double)a.fwd[s1 * per + (long long)d * a.rh * a.rw + cell];
          const double en0 = (double)a.fwd[(s1 - 1) * per + (long long)d * a.rh * a.rw + cell];
          const double er = a.eps_region[(a.n_mat > 1 ? (long long)d : 0LL) * a.rh * a.rw + cell];
          a.grad[(long long)d * a.rh * a.rw + cell] -= (double)e * (en1 - en0) / er;
        }
      }
    }
    Uc = Un;
    wy_up = wy;
  }

  if (a.n_src == 0 || step == 0) return;
  // ---- post phase: e_{n-1} = mul * (dJ/dE_n + objective term at step n-1) ---------
  __shared__ int s_k0[RB], s_pre[RB + 1];
  const int xlo = blockIdx.x * BX;
  const int xhi = min(xlo + BX, nx);
  __syncthreads();
  const int total = block_op_ranges(a.src_row, a.src_cell, y0, nrows, nx, xlo, xhi, s_k0, s_pre);
  const long long sstep = step - 1;
  for (int i = threadIdx.x; i < total; i += BX) {
    int t;
    const int k = op_at(i, nrows, s_k0, s_pre, t);
    const int cell = __ldg(a.src_cell + k);
    if (i > s_pre[t] && __ldg(a.src_cell + k - 1) == cell) continue;
    const int y = y0 + t;
    const long long rr = fb + (long long)y * pitch + (cell - y * nx);
    T v = a.e_out[rr];
    for (int kk = k; kk < a.n_src && __ldg(a.src_cell + kk) == cell; ++kk) {
      const T s = sstep < a.src_steps ? __ldg(a.signals + (long long)__ldg(a.src_sig + kk) * a.src_steps + sstep) : T(0);
      v = __ldg(a.src_mul + kk) * v + __ldg(a.src_w + d * a.w_stride + kk) * s;
    }
    a.e_out[rr] = v;
  }
}


// ---- several reverse steps per launch (temporal blocking) ---------------------------
// The register tile of the forward step2d_tb kernel, run backwards: a block holds 64
// columns x NW*R rows (lane l: columns X0+l and X0+32+l) with the per-cell factors, and
// performs TS reverse steps m = step, step-1, ..., each one the single-step adjoint
// above: gradient from the incoming e on owned cells of the design box (applied after
// the last sub-step from a shared-memory history of those e), U = Ce*e, the
// H-like pass (U(x+1) by shuffle, U(y+1) from the next row or warp), the E-like pass
// (wx(x-1) by shuffle, wy(y-1) from the previous row or warp), carried fh*hx', fh*hy',
// then the operations preparing step m-1 on every tile cell. Boundary rules enter the
// factors (Ce = 0, Fe = 1 off the interior; cx = 0 in the last column and outside,
// cy = 0 in the last row and outside), and the stale halo of TS cells is not stored.
template <typename T, int TS, int R, int NW>
__global__ void __launch_bounds__(32 * NW) adjoint2d_tb_kernel(AdjArgs<T> a, long long step0) {
  constexpr int TW = 64, TH = NW * R, OW = TW - 2 * TS, OH = TH - 2 * TS;
  static_assert(TS % 2 == 1 && OH > 0 && R * 2 <= 32, "bad temporal tile");
  const int nx = a.nx, ny = a.ny, pitch = a.pitch;
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5, d = blockIdx.z;
  const int X0 = (int)blockIdx.x * OW - TS, Y0 = (int)blockIdx.y * OH - TS;
  const int yb = Y0 + w * R;
  const long long fb = (long long)d * a.plane;
  const long long mb = (a.n_mat > 1 ? (long long)d : 0LL) * a.plane;
  __shared__ T s_top[NW][TW], s_bot[NW][TW];
  __shared__ int s_src[TH][2];

  int xs[2];
  xs[0] = X0 + lane;
  xs[1] = X0 + 32 + lane;
  T e[R][2], hx[R][2], hy[R][2], fh[R][2], cx[R][2], cy[R][2], Fe[R][2], Ce[R][2];
#pragma unroll
  for (int i = 0; i < R; ++i) {
    const int y = yb + i;
#pragma unroll
    for (int j = 0; j < 2; ++j) {
      const int x = xs[j];
      const bool in = x >= 0 && x < nx && y >= 0 && y < ny;
      const long long r = in ? (long long)y * pitch + x : 0LL;
      const T ls = in ? __ldg(a.loss + mb + r) : T(0), c = in ? __ldg(a.ce + mb + r) : T(0);
      h_coeffs(ls, a.chx, a.chy, fh[i][j], cx[i][j], cy[i][j]);
      const bool interior = x >= 1 && x <= nx - 2 && y >= 1 && y <= ny - 2;
      Fe[i][j] = interior ? T(1) - ls * c * a.inv_kd2 : T(1);
      Ce[i][j] = interior ? c : T(0);
      if (!(in && x < nx - 1)) cx[i][j] = T(0);
      if (!(in && y < ny - 1)) cy[i][j] = T(0);
      e[i][j] = in ? __ldg(a.e_in + fb + r) : T(0);
      hx[i][j] = (in && x < nx - 1) ? __ldg(a.hx_in + fb + r) : T(0);
      hy[i][j] = (in && y < ny - 1) ? __ldg(a.hy_in + fb + r) : T(0);
    }
  }
  if (lane < R) {  // operation ranges of the tile's rows over its columns
    const int y = yb + lane, tr = w * R + lane;
    int s0 = 0, s1 = 0;
    if (a.n_src > 0 && y >= 0 && y < ny) {
      const int lo = __ldg(a.src_row + y), hi = __ldg(a.src_row + y + 1);
      if (lo < hi) {
        s0 = lower_bound_i(a.src_cell, lo, hi, y * nx + max(X0, 0));
        s1 = lower_bound_i(a.src_cell, s0, hi, y * nx + min(X0 + TW, nx));
      }
    }
    s_src[tr][0] = s0;
    s_src[tr][1] = s1;
  }
  __syncwarp();
  unsigned src_rows = 0u, gbits = 0u;
  bool own[2];
  own[0] = lane >= TS && xs[0] < nx;
  own[1] = lane < 32 - TS && xs[1] < nx;
#pragma unroll
  for (int i = 0; i < R; ++i) {
    if (s_src[w * R + i][0] < s_src[w * R + i][1]) src_rows |= 1u << i;
    const int tr = w * R + i, y = yb + i;
#pragma unroll
    for (int j = 0; j < 2; ++j) {
      const int rx = xs[j] - a.rx0, ry = y - a.ry0;
      if (a.grad != nullptr && own[j] && tr >= TS && tr < TH - TS && y < ny && rx >= 0 && rx < a.rw && ry >= 0 &&
          ry < a.rh)
        gbits |= 1u << (i * 2 + j);
    }
  }

  // Design-box cells keep each sub-step's incoming e here ([TS][R][2][thread]); the
  // gradient terms are applied after the last sub-step, off the barrier-paced loop.
  extern __shared__ __align__(16) unsigned char s_hist_raw[];
  T* s_hist = reinterpret_cast<T*>(s_hist_raw);
  constexpr int NT = 32 * NW;

#pragma unroll 1
  for (int s = 0; s < TS; ++s) {
    const long long m = step0 - s;  // reverse step taken by this sub-step
    if (gbits) {
#pragma unroll
      for (int i = 0; i < R; ++i)
#pragma unroll
        for (int j = 0; j < 2; ++j)
          if (gbits & (1u << (i * 2 + j))) s_hist[((s * R + i) * 2 + j) * NT + threadIdx.x] = e[i][j];
    }
    T U[R][2];
#pragma unroll
    for (int i = 0; i < R; ++i)
#pragma unroll
      for (int j = 0; j < 2; ++j) U[i][j] = Ce[i][j] * e[i][j];
#pragma unroll
    for (int j = 0; j < 2; ++j) s_top[w][j * 32 + lane] = U[0][j];
    __syncthreads();
    // H-like pass: hx' = hx + U(x+1) - U(x), hy' = hy - qy*(U(y+1) - U(y))
#pragma unroll
    for (int i = 0; i < R; ++i) {
      const T r0 = __shfl_sync(FULL, U[i][0], (lane + 1) & 31);
      const T r1 = __shfl_sync(FULL, U[i][1], (lane + 1) & 31);
      T ur[2], ud[2];
      ur[0] = lane == 31 ? r1 : r0;
      ur[1] = r1;
      if (i + 1 < R) {
        ud[0] = U[i + 1][0];
        ud[1] = U[i + 1][1];
      } else if (w + 1 < NW) {
        ud[0] = s_top[w + 1][lane];
        ud[1] = s_top[w + 1][32 + lane];
      } else {
        ud[0] = ud[1] = T(0);
      }
#pragma unroll
      for (int j = 0; j < 2; ++j) {
        hx[i][j] = hx[i][j] + (ur[j] - U[i][j]);         // hx'
        hy[i][j] = hy[i][j] - a.qy * (ud[j] - U[i][j]);  // hy'
      }
    }
#pragma unroll
    for (int j = 0; j < 2; ++j) s_bot[w][j * 32 + lane] = cy[R - 1][j] * hy[R - 1][j];
    __syncthreads();
    // E-like pass: e_prev = Fe*e - (wx(x-1) - wx) + (wy(y-1) - wy); carried fh*h'
#pragma unroll
    for (int i = 0; i < R; ++i) {
      T wx[2], wy[2], wl[2], wu[2];
#pragma unroll
      for (int j = 0; j < 2; ++j) {
        wx[j] = cx[i][j] * hx[i][j];
        wy[j] = cy[i][j] * hy[i][j];
      }
      const T l0 = __shfl_sync(FULL, wx[0], (lane + 31) & 31);
      const T l1 = __shfl_sync(FULL, wx[1], (lane + 31) & 31);
      wl[0] = l0;
      wl[1] = lane == 0 ? l0 : l1;
      if (i > 0) {
        wu[0] = cy[i - 1][0] * hy[i - 1][0];
        wu[1] = cy[i - 1][1] * hy[i - 1][1];
      } else if (w > 0) {
        wu[0] = s_bot[w - 1][lane];
        wu[1] = s_bot[w - 1][32 + lane];
      } else {
        wu[0] = wu[1] = T(0);
      }
#pragma unroll
      for (int j = 0; j < 2; ++j) e[i][j] = Fe[i][j] * e[i][j] - (wl[j] - wx[j]) + (wu[j] - wy[j]);
    }
#pragma unroll
    for (int i = 0; i < R; ++i)
#pragma unroll
      for (int j = 0; j < 2; ++j) {
        hx[i][j] = fh[i][j] * hx[i][j];
        hy[i][j] = fh[i][j] * hy[i][j];
      }
    // operations preparing step m-1 (none after step 0)
    if (src_rows && m >= 1) {
      const long long sstep = m - 1;
#pragma unroll
      for (int i = 0; i < R; ++i) {
        if (!(src_rows & (1u << i))) continue;  // uniform across the warp
        const int y = yb + i;
        const int k0 = s_src[w * R + i][0], k1 = s_src[w * R + i][1];
        for (int kk = k0; kk < k1; ++kk) {
          const int xo = __ldg(a.src_cell + kk) - y * nx;
          if (xo != xs[0] && xo != xs[1]) continue;
          const T sv =
              sstep < a.src_steps ? __ldg(a.signals + (long long)__ldg(a.src_sig + kk) * a.src_steps + sstep) : T(0);
          const T mul = __ldg(a.src_mul + kk), wv = __ldg(a.src_w + d * a.w_stride + kk);
#pragma unroll
          for (int j = 0; j < 2; ++j)
            if (xo == xs[j]) e[i][j] = mul * e[i][j] + wv * sv;
        }
      }
    }
  }
  // store the owned box
#pragma unroll
  for (int i = 0; i < R; ++i) {
    const int tr = w * R + i, y = yb + i;
    if (tr < TS || tr >= TH - TS || y >= ny) continue;
#pragma unroll
    for (int j = 0; j < 2; ++j) {
      const int x = xs[j];
      if (!own[j]) continue;
      const long long r = fb + (long long)y * pitch + x;
      a.e_out[r] = e[i][j];
      if (x < nx - 1) a.hx_out[r] = hx[i][j];
      if (y < ny - 1) a.hy_out[r] = hy[i][j];
    }
  }
  // grad -= sum over the sub-steps' reverse steps m of e_m * (E_{m+1} - E_m), over
  // eps_r, on the owned design-box cells (no other block writes them)
  if (gbits) {
    const long long per = (long long)a.n_designs * a.rh * a.rw, db = (long long)d * a.rh * a.rw;
    const long long eb = (a.n_mat > 1 ? (long long)d : 0LL) * a.rh * a.rw;
#pragma unroll
    for (int i = 0; i < R; ++i)
#pragma unroll
      for (int j = 0; j < 2; ++j) {
        if (!(gbits & (1u << (i * 2 + j)))) continue;
        const long long cell = (long long)(yb + i - a.ry0) * a.rw + (xs[j] - a.rx0);
        const long long p0 = step0 + 1 - a.fwd_step0;  // captured plane E_{m+1} of sub-step 0
        T f[TS + 1];  // planes p0, p0-1, ..., p0-TS, all loads issued before the sums
#pragma unroll
        for (int k = 0; k <= TS; ++k)
          f[k] = (p0 - k >= 0 && p0 - k < a.n_fwd) ? a.fwd[(p0 - k) * per + db + cell] : T(0);
        const double er = a.eps_region[eb + cell];
        const double gv = a.grad[db + cell];
        T acc = T(0);  // the block's terms in the fields' precision (e and the planes are T)
#pragma unroll
        for (int s = 0; s < TS; ++s)
          if (p0 - s >= 1 && p0 - s < a.n_fwd)
            acc += s_hist[((s * R + i) * 2 + j) * NT + threadIdx.x] * (f[s] - f[s + 1]);
        a.grad[db + cell] = gv - (double)acc / er;
      }
  }
}

template <typename T>
AdjArgs<T> adj_args(const bz_grid2d* g, const bz_adjoint2d* s, const bz_source_ops* ops, int32_t phase) {
  AdjArgs<T> a = {};
  const int src = phase & 1;
  a.e_in = (const T*)s->e[src];
  a.hx_in = (const T*)s->hx[src];
  a.hy_in = (const T*)s->hy[src];
  a.e_out = (T*)s->e[src ^ 1];
  a.hx_out = (T*)s->hx[src ^ 1];
  a.hy_out = (T*)s->hy[src ^ 1];
  a.ce = (const T*)s->ce;
  a.loss = (const T*)s->loss;
  a.nx = g->nx;
  a.ny = g->ny;
  a.pitch = g->pitch;
  a.n_designs = g->n_designs;
  a.n_mat = g->n_mat;
  a.plane = (long long)g->ny * g->pitch;
  a.chx = (T)g->chx;
  a.chy = (T)g->chy;
  a.qy = (T)g->qy;
  a.inv_kd2 = (T)g->inv_kd2;
  a.grad = s->grad;
  a.eps_region = s->eps_region;
  a.fwd = (const T*)s->fwd_region;
  a.rx0 = s->rx0;
  a.ry0 = s->ry0;
  a.rw = s->rw;
  a.rh = s->rh;
  a.n_fwd = s->n_fwd;
  a.fwd_step0 = s->fwd_step0;
  if (ops && ops->n_ops > 0) {
    a.n_src = ops->n_ops;
    a.src_steps = ops->n_steps;
    a.src_row = ops->row_ptr;
    a.src_cell = ops->cell;
    a.src_mul = (const T*)ops->mul;
    a.src_w = (const T*)ops->weight;
    a.w_stride = ops->weight_stride;
    a.src_sig = ops->sig;
    a.signals = (const T*)ops->signals;
  }
  return a;
}

template <typename T>
int launch_adj(const bz_grid2d* g, const bz_adjoint2d* s, const bz_source_ops* ops, int64_t step, int32_t phase,
               cudaStream_t st) {
  const AdjArgs<T> a = adj_args<T>(g, s, ops, phase);
  dim3 grid((unsigned)ceil_div(g->nx, BX), (unsigned)ceil_div(g->ny, RB), (unsigned)g->n_designs);
  adjoint2d_kernel<T><<<grid, BX, 0, st>>>(a, (long long)step);
  return check_launch("bz_adjoint_step2d");
}

template <typename T, int TS>
int launch_adj_tb(const bz_grid2d* g, const bz_adjoint2d* s, const bz_source_ops* ops, int64_t step, int32_t phase,
                  cudaStream_t st) {
  constexpr int R = sizeof(T) == 4 ? 4 : 2, NW = 16;
  constexpr int hist = TS * R * 2 * 32 * NW * (int)sizeof(T);  // at most 147 KB (TS = 9)
  const AdjArgs<T> a = adj_args<T>(g, s, ops, phase);
  dim3 grid((unsigned)ceil_div(g->nx, 64 - 2 * TS), (unsigned)ceil_div(g->ny, NW * R - 2 * TS), (unsigned)g->n_designs);
  static bool opted = false;  // history plus the static tiles pass the default 48 KB
  if (!opted) {
    if (cudaFuncSetAttribute(adjoint2d_tb_kernel<T, TS, R, NW>, cudaFuncAttributeMaxDynamicSharedMemorySize, hist) !=
        cudaSuccess)
      return fail(BZ_ERR_CUDA, "bz_adjoint_step2d_multi: cannot configure the kernel's shared memory");
    opted = true;
  }
  adjoint2d_tb_kernel<T, TS, R, NW><<<grid, 32 * NW, a.grad ? hist : 0, st>>>(a, (long long)step);
  return check_launch("bz_adjoint_step2d_multi");
}

}  // namespace
}  // namespace bz

namespace bz {
namespace {
int check_adj(const char* who, const bz_grid2d* g, const bz_adjoint2d* s, const bz_source_ops* ops, int64_t step) {
  BZ_REQUIRE(g && s, "%s: grid or state is NULL", who);
  BZ_REQUIRE(g->n_comp == 1, "%s: only real fields (n_comp = 1)", who);
  BZ_REQUIRE(g->nx >= 2 && g->ny >= 2 && g->pitch >= g->nx && g->pitch % 32 == 0, "%s: bad grid", who);
  BZ_REQUIRE(g->n_mat == 1 || g->n_mat == g->n_designs, "%s: n_mat must be 1 or n_designs", who);
  for (int i = 0; i < 2; ++i) BZ_REQUIRE(s->e[i] && s->hx[i] && s->hy[i], "%s: NULL state buffer", who);
  BZ_REQUIRE(s->ce && s->loss, "%s: NULL coefficients", who);
  if (s->grad) BZ_REQUIRE(s->eps_region && s->fwd_region && s->rw >= 1 && s->rh >= 1, "%s: bad grad box", who);
  if (ops && ops->n_ops > 0)
    BZ_REQUIRE(ops->row_ptr && ops->cell && ops->mul && ops->weight && ops->sig && ops->signals,
               "%s: incomplete ops", who);
  BZ_REQUIRE(step >= 0, "%s: negative step", who);
  BZ_REQUIRE(g->dtype == BZ_F32 || g->dtype == BZ_F64, "%s: unknown dtype %d", who, g->dtype);
  return BZ_OK;
}
}  // namespace
}  // namespace bz

extern "C" int bz_adjoint_step2d_multi(const bz_grid2d* g, const bz_adjoint2d* s, const bz_source_ops* ops,
                                       int64_t step, int32_t n_sub, int32_t phase, void* stream) {
  const int rc = bz::check_adj("bz_adjoint_step2d_multi", g, s, ops, step);
  if (rc != BZ_OK) return rc;
  BZ_REQUIRE(n_sub == 1 || n_sub == 3 || n_sub == 5 || n_sub == 7 || n_sub == 9,
             "bz_adjoint_step2d_multi: n_sub must be 1, 3, 5, 7 or 9 (got %d)", n_sub);
  BZ_REQUIRE(step + 1 >= n_sub, "bz_adjoint_step2d_multi: %d reverse steps from step %lld pass step 0", n_sub,
             (long long)step);
  if (n_sub == 1) return bz_adjoint_step2d(g, s, ops, step, phase, stream);
  cudaStream_t st = bz::as_stream(stream);
  if (g->dtype == BZ_F32) {
    switch (n_sub) {
      case 3: return bz::launch_adj_tb<float, 3>(g, s, ops, step, phase, st);
      case 5: return bz::launch_adj_tb<float, 5>(g, s, ops, step, phase, st);
      case 9: return bz::launch_adj_tb<float, 9>(g, s, ops, step, phase, st);
      default: return bz::launch_adj_tb<float, 7>(g, s, ops, step, phase, st);
    }
  }
  switch (n_sub) {
    case 3: return bz::launch_adj_tb<double, 3>(g, s, ops, step, phase, st);
    case 5: return bz::launch_adj_tb<double, 5>(g, s, ops, step, phase, st);
    case 9: return bz::launch_adj_tb<double, 9>(g, s, ops, step, phase, st);
    default: return bz::launch_adj_tb<double, 7>(g, s, ops, step, phase, st);
  }
}

extern "C" int bz_adjoint_step2d(const bz_grid2d* g, const bz_adjoint2d* s, const bz_source_ops* ops, int64_t step,
                                 int32_t phase, void* stream) {
  BZ_REQUIRE(g && s, "bz_adjoint_step2d: grid or state is NULL");
  BZ_REQUIRE(g->n_comp == 1, "bz_adjoint_step2d: only real fields (n_comp = 1)");
  BZ_REQUIRE(g->nx >= 2 && g->ny >= 2 && g->pitch >= g->nx && g->pitch % 32 == 0, "bz_adjoint_step2d: bad grid");
  BZ_REQUIRE(g->n_mat == 1 || g->n_mat == g->n_designs, "bz_adjoint_step2d: n_mat must be 1 or n_designs");
  for (int i = 0; i < 2; ++i) BZ_REQUIRE(s->e[i] && s->hx[i] && s->hy[i], "bz_adjoint_step2d: NULL state buffer");
  BZ_REQUIRE(s->ce && s->loss, "bz_adjoint_step2d: NULL coefficients");
  if (s->grad) BZ_REQUIRE(s->eps_region && s->fwd_region && s->rw >= 1 && s->rh >= 1, "bz_adjoint_step2d: bad grad box");
  if (ops && ops->n_ops > 0)
    BZ_REQUIRE(ops->row_ptr && ops->cell && ops->mul && ops->weight && ops->sig && ops->signals,
               "bz_adjoint_step2d: incomplete ops");
  BZ_REQUIRE(step >= 0, "bz_adjoint_step2d: negative step");
  cudaStream_t st = bz::as_stream(stream);
  if (g->dtype == BZ_F32) return bz::launch_adj<float>(g, s, ops, step, phase, st);
  if (g->dtype == BZ_F64) return bz::launch_adj<double>(g, s, ops, step, phase, st);
  return bz::fail(BZ_ERR_INVALID, "bz_adjoint_step2d: unknown dtype %d", g->dtype);
}
