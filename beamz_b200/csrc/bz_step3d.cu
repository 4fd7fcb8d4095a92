// 3D Yee time step, fused H + E (beamz/simulation/fdtd.py:200-310), plus the
// small kernels around it: source injection on one array (helper.py:5-118),
// monitor gathers (helper.py:235-244, monitors.py:317-396) and |S| accumulation
// (helper.py:124-151).
//
// Tiling of bz_step3d: a 32 x 8 thread block covers a 32 x 8 column patch whose
// first column and first row are a halo shared with the neighbouring patch, so it
// owns 31 x 7 columns; it marches along z over tile_z planes. Per plane:
//   1. E(k) of the patch goes to shared memory (y+1 neighbours), x+1 neighbours
//      come from the next lane by warp shuffle (lane 31 and row 7 read global);
//   2. every thread computes H(k) (the halo row/column too);
//   3. H(k) goes to shared memory (y-1 neighbours), x-1 neighbours by shuffle,
//      H(k-1) is carried in registers from the previous plane;
//   4. owned threads compute E(k) and write H(k), E(k).
// The first plane's H(k-1) is recomputed from global memory. Ping-pong copies
// keep every launch reading only the previous step's values. Float32 fields take
// step3d_quad_kernel, the same schedule with four x cells per thread (float4), or on
// request (bz_grid3d.x_cells = 2) step3d_pair_kernel with two.
#include "bz_internal.cuh"

namespace bz {
namespace {

constexpr unsigned FULL = 0xffffffffu;
constexpr int TX = 32;  // tile width; the tile height TY is a template parameter (8 or 16)

template <typename T>
struct Geo3D {
  int nx, ny, nz, pitch, n_designs, n_mat, n_comp, nzb;
  long long plane, vol;  // ny*pitch, nz*plane
  T chx, chy, chz, qx, qz, inv_kd2;
};

template <typename T>
struct Ptr3 {
  const T* e[3];
  const T* h[3];
};

template <typename T>
struct Out3 {
  T* e[3];
  T* h[3];
};

template <typename T>
__device__ __forceinline__ void hfac(T a, const Geo3D<T>& g, T& fh, T& cx, T& cy, T& cz) {
  if (a == T(0)) {
    fh = T(1);
    cx = g.chx;
    cy = g.chy;
    cz = g.chz;
  } else {  // (1-a)/(1+a) and c/(1+a) through one reciprocal
    const T r = T(1) / (T(1) + a);
    fh = (T(1) - a) * r;
    cx = g.chx * r;
    cy = g.chy * r;
    cz = g.chz * r;
  }
}

template <typename T>
__device__ __forceinline__ T ld(const T* p, long long i, bool ok) {
  return ok ? __ldg(p + i) : T(0);
}

// Per-plane inputs of one thread's column: H, coefficients, and the E(x+1) / E(y+1)
// values that the tile's last lane / last row read from memory.
template <typename T, int NC>
struct PlaneIn {
  T hx[NC], hy[NC], hz[NC], ez_x[NC], ey_x[NC], ez_y[NC], ex_y[NC];
  T a, ce;
};

template <typename T, int NC, int ZB, int TY>
__global__ void __launch_bounds__(TX * TY) step3d_kernel(Ptr3<T> in, Out3<T> out, const T* __restrict__ ce,
                                                          const T* __restrict__ loss, Geo3D<T> g) {
  __shared__ T s_ez[NC][TY][TX], s_ex[NC][TY][TX], s_hz[NC][TY][TX], s_hx[NC][TY][TX];
  const int tx = threadIdx.x, ty = threadIdx.y;
  const int nx = g.nx, ny = g.ny, nz = g.nz;
  const int x = blockIdx.x * (TX - 1) - 1 + tx;
  const int y = blockIdx.y * (TY - 1) - 1 + ty;
  const int d = blockIdx.z / g.nzb;
  const int z0 = (blockIdx.z - d * g.nzb) * ZB;
  const int z1 = min(z0 + ZB, nz);
  const bool xin = x >= 0 && x < nx, yin = y >= 0 && y < ny, inb = xin && yin;
  const bool owned = inb && tx >= 1 && ty >= 1;
  const bool xe = tx == TX - 1, ye = ty == TY - 1;
  const bool xnb = yin && x + 1 < nx, ynb = xin && y + 1 < ny;
  const long long P = g.plane;
  const long long mb = (g.n_mat > 1 ? (long long)d : 0LL) * g.vol;
  const long long col = (long long)y * g.pitch + x;  // offset inside a plane
  long long fb[NC];
#pragma unroll
  for (int c = 0; c < NC; ++c) fb[c] = ((long long)d * NC + c) * g.vol;

  // Loads of plane k's inputs; issued one plane ahead so they overlap the arithmetic.
  auto load_plane = [&](int k, PlaneIn<T, NC>& q) {
    const long long po = (long long)k * P + col;
    q.a = ld(loss + mb, po, inb);
    q.ce = ld(ce + mb, po, inb);
#pragma unroll
    for (int c = 0; c < NC; ++c) {
      const long long o = fb[c] + po;
      q.hx[c] = ld(in.h[0], o, inb);
      q.hy[c] = ld(in.h[1], o, inb);
      q.hz[c] = ld(in.h[2], o, inb);
      q.ez_x[c] = ld(in.e[2], o + 1, xe && xnb);
      q.ey_x[c] = ld(in.e[1], o + 1, xe && xnb);
      q.ez_y[c] = ld(in.e[2], o + g.pitch, ye && ynb);
      q.ex_y[c] = ld(in.e[0], o + g.pitch, ye && ynb);
    }
  };

  T exk[NC], eyk[NC], ezk[NC], exn[NC], eyn[NC], ezn[NC], hxm[NC], hym[NC];
  PlaneIn<T, NC> cur, nxt;
  load_plane(z0, cur);
#pragma unroll
  for (int c = 0; c < NC; ++c) {
    const long long o = fb[c] + (long long)z0 * P + col;
    exk[c] = ld(in.e[0], o, inb);
    eyk[c] = ld(in.e[1], o, inb);
    ezk[c] = ld(in.e[2], o, inb);
    exn[c] = ld(in.e[0], o + P, inb && z0 + 1 < nz);
    eyn[c] = ld(in.e[1], o + P, inb && z0 + 1 < nz);
    ezn[c] = ld(in.e[2], o + P, inb && z0 + 1 < nz);
    hxm[c] = T(0);
    hym[c] = T(0);
  }
  if (z0 >= 1 && inb) {  // H(z0-1) at this column, recomputed from global memory
    const int k = z0 - 1;
    T fh, cx, cy, cz;
    hfac(__ldg(loss + mb + (long long)k * P + col), g, fh, cx, cy, cz);
#pragma unroll
    for (int c = 0; c < NC; ++c) {
      const long long o = fb[c] + (long long)k * P + col;
      const T ez = __ldg(in.e[2] + o), ex = __ldg(in.e[0] + o), ey = __ldg(in.e[1] + o);
      const T ez_yp = ld(in.e[2], o + g.pitch, y + 1 < ny);
      const T ez_xp = ld(in.e[2], o + 1, x + 1 < nx);
      const T ey_zp = eyk[c], ex_zp = exk[c];  // plane z0
      hxm[c] = fh * __ldg(in.h[0] + o) - (cy * (ez_yp - ez) - cz * (ey_zp - ey));
      hym[c] = fh * __ldg(in.h[1] + o) - (cz * (ex_zp - ex) - cx * (ez_xp - ez));
    }
  }

  for (int k = z0; k < z1; ++k) {
    const long long po = (long long)k * P + col;
    // prefetch: inputs of plane k+1 and E(k+2)
    T ex2[NC], ey2[NC], ez2[NC];
    if (k + 1 < z1) {
      load_plane(k + 1, nxt);
#pragma unroll
      for (int c = 0; c < NC; ++c) {
        const long long o = fb[c] + po + 2 * P;
        ex2[c] = ld(in.e[0], o, inb && k + 2 < nz);
        ey2[c] = ld(in.e[1], o, inb && k + 2 < nz);
        ez2[c] = ld(in.e[2], o, inb && k + 2 < nz);
      }
    }
    T fh, cx, cy, cz;
    hfac(cur.a, g, fh, cx, cy, cz);
    const T cev = cur.ce;
    const T fe = T(1) - cur.a * cev * g.inv_kd2;
#pragma unroll
    for (int c = 0; c < NC; ++c) {
      s_ez[c][ty][tx] = ezk[c];
      s_ex[c][ty][tx] = exk[c];
    }
    __syncthreads();
    T hxn[NC], hyn[NC], hzn[NC];
#pragma unroll
    for (int c = 0; c < NC; ++c) {
      const T ez_yp = ye ? cur.ez_y[c] : s_ez[c][ty + (ye ? 0 : 1)][tx];
      const T ex_yp = ye ? cur.ex_y[c] : s_ex[c][ty + (ye ? 0 : 1)][tx];
      T ez_xp = __shfl_down_sync(FULL, ezk[c], 1);
      T ey_xp = __shfl_down_sync(FULL, eyk[c], 1);
      if (xe) {
        ez_xp = cur.ez_x[c];
        ey_xp = cur.ey_x[c];
      }
      hxn[c] = fh * cur.hx[c] - (cy * (ez_yp - ezk[c]) - cz * (eyn[c] - eyk[c]));
      hyn[c] = fh * cur.hy[c] - (cz * (exn[c] - exk[c]) - cx * (ez_xp - ezk[c]));
      hzn[c] = fh * cur.hz[c] - (cx * (ey_xp - eyk[c]) - cy * (ex_yp - exk[c]));
      s_hz[c][ty][tx] = hzn[c];
      s_hx[c][ty][tx] = hxn[c];
    }
    __syncthreads();
#pragma unroll
    for (int c = 0; c < NC; ++c) {
      const T hy_xm = __shfl_up_sync(FULL, hyn[c], 1);
      const T hz_xm = __shfl_up_sync(FULL, hzn[c], 1);
      if (owned) {
        const long long o = fb[c] + po;
        const T hz_ym = s_hz[c][ty - 1][tx];
        const T hx_ym = s_hx[c][ty - 1][tx];
        const bool kin = k >= 1 && k <= nz - 2;
        T ex = exk[c], ey = eyk[c], ez = ezk[c];
        if (kin && y >= 1 && y <= ny - 2 && x <= nx - 2)
          ex = fe * exk[c] + cev * ((hzn[c] - hz_ym) - g.qz * (hyn[c] - hym[c]));
        if (kin && y <= ny - 2 && x >= 1 && x <= nx - 2)
          ey = fe * eyk[c] + cev * (g.qz * (hxn[c] - hxm[c]) - g.qx * (hzn[c] - hz_xm));
        if (k <= nz - 2 && y >= 1 && y <= ny - 2 && x >= 1 && x <= nx - 2)
          ez = fe * ezk[c] + cev * (g.qx * (hyn[c] - hy_xm) - (hxn[c] - hx_ym));
        if (x <= nx - 2) out.e[0][o] = ex;
        if (y <= ny - 2) out.e[1][o] = ey;
        if (k <= nz - 2) out.e[2][o] = ez;
        if (k <= nz - 2 && y <= ny - 2) out.h[0][o] = hxn[c];
        if (k <= nz - 2 && x <= nx - 2) out.h[1][o] = hyn[c];
        if (y <= ny - 2 && x <= nx - 2) out.h[2][o] = hzn[c];
      }
      exk[c] = exn[c];
      eyk[c] = eyn[c];
      ezk[c] = ezn[c];
      exn[c] = ex2[c];
      eyn[c] = ey2[c];
      ezn[c] = ez2[c];
      hxm[c] = hxn[c];
      hym[c] = hyn[c];
    }
    cur = nxt;
  }
}

template <typename T, int NC, int ZB, int TY>
int launch3d(const bz_grid3d* gd, const bz_fields3d* f, int64_t step, cudaStream_t st) {
  Geo3D<T> g;
  g.nx = gd->nx;
  g.ny = gd->ny;
  g.nz = gd->nz;
  g.pitch = gd->pitch;
  g.n_designs = gd->n_designs;
  g.n_mat = gd->n_mat;
  g.n_comp = gd->n_comp;
  g.nzb = (int)ceil_div(gd->nz, ZB);
  g.plane = (long long)gd->ny * gd->pitch;
  g.vol = g.plane * gd->nz;
  g.chx = (T)gd->chx;
  g.chy = (T)gd->chy;
  g.chz = (T)gd->chz;
  g.qx = (T)gd->qx;
  g.qz = (T)gd->qz;
  g.inv_kd2 = (T)gd->inv_kd2;
  const int src = (int)(step & 1);
  Ptr3<T> in;
  Out3<T> out;
  for (int i = 0; i < 3; ++i) {
    in.e[i] = (const T*)f->e[src][i];
    in.h[i] = (const T*)f->h[src][i];
    out.e[i] = (T*)f->e[src ^ 1][i];
    out.h[i] = (T*)f->h[src ^ 1][i];
  }
  dim3 block(TX, TY);
  dim3 grid((unsigned)ceil_div(gd->nx, TX - 1), (unsigned)ceil_div(gd->ny, TY - 1), (unsigned)(g.nzb * gd->n_designs));
  step3d_kernel<T, NC, ZB, TY><<<grid, block, 0, st>>>(in, out, (const T*)f->ce, (const T*)f->loss, g);
  return check_launch("bz_step3d");
}

// ---------------------------------------------------------------------------- paired columns (float32)
// The same step with two adjacent x cells per thread, moved as float2: a warp spans 64
// columns whose first two (one pair, to keep 8-byte alignment) are the halo shared
// with the neighbouring tile, so a block owns 62 x (TY-1) columns. Loads, stores,
// shared-memory traffic, shuffles, barriers and index arithmetic are issued once per
// pair. The pair (x, x+1) starts at an even x; when nx is odd the last pair's second
// cell is row padding (pitch > nx), read but never stored, and no stored value
// depends on it. Two-component (complex) fields run as two independent real fields:
// the update is linear with real coefficients, so each block steps one component
// (grid z = z blocks x designs x components) and reads ce and loss for it.
__device__ __forceinline__ float2 ld2(const float* p, long long i, bool ok) {
  return ok ? __ldg(reinterpret_cast<const float2*>(p + i)) : make_float2(0.f, 0.f);
}

// Stores both cells when the second exists (then so does the first), else the first alone.
__device__ __forceinline__ void st2(float* p, long long i, float2 v, bool s0, bool s1) {
  if (s1)
    *reinterpret_cast<float2*>(p + i) = v;
  else if (s0)
    p[i] = v.x;
}

struct PairIn {
  float2 hx, hy, hz, a, ce, ez_y, ex_y;
  float ez_x, ey_x;  // E at x+2 (the warp's last lane)
};

template <int ZB, int TY>
__global__ void __launch_bounds__(TX * TY, TY == 8 ? 3 : 1) step3d_pair_kernel(Ptr3<float> in, Out3<float> out,
                                                               const float* __restrict__ ce,
                                                               const float* __restrict__ loss, Geo3D<float> g) {
  __shared__ float2 s_ez[TY][TX], s_ex[TY][TX], s_hz[TY][TX], s_hx[TY][TX];
  const int tx = threadIdx.x, ty = threadIdx.y;
  const int nx = g.nx, ny = g.ny, nz = g.nz;
  const int x = blockIdx.x * (2 * TX - 2) - 2 + 2 * tx;  // first cell of the pair
  const int y = blockIdx.y * (TY - 1) - 1 + ty;
  const int dc = blockIdx.z / g.nzb;  // design * n_comp + component
  const int d = dc / g.n_comp;
  const int z0 = (blockIdx.z - dc * g.nzb) * ZB;
  const int z1 = min(z0 + ZB, nz);
  const bool xin = x >= 0 && x < nx, yin = y >= 0 && y < ny, inb = xin && yin;
  const bool owned = inb && tx >= 1 && ty >= 1;
  const bool xe = tx == TX - 1, ye = ty == TY - 1;
  const bool xnb = yin && x + 2 < nx, ynb = xin && y + 1 < ny;
  // which cells of the pair exist in each component's extent, and which are updated
  const bool x0m = x <= nx - 2, x1m = x + 1 <= nx - 2, x1in = x + 1 <= nx - 1, x0p = x >= 1;
  const bool yint = y >= 1 && y <= ny - 2, ym = y <= ny - 2;
  const long long P = g.plane;
  const long long mb = (g.n_mat > 1 ? (long long)d : 0LL) * g.vol;
  const long long col = (long long)y * g.pitch + x;
  const long long fb = (long long)dc * g.vol;

  auto load_plane = [&](int k, PairIn& q) {
    const long long po = (long long)k * P + col;
    q.a = ld2(loss + mb, po, inb);
    q.ce = ld2(ce + mb, po, inb);
    const long long o = fb + po;
    q.hx = ld2(in.h[0], o, inb);
    q.hy = ld2(in.h[1], o, inb);
    q.hz = ld2(in.h[2], o, inb);
    q.ez_x = ld(in.e[2], o + 2, xe && xnb);
    q.ey_x = ld(in.e[1], o + 2, xe && xnb);
    q.ez_y = ld2(in.e[2], o + g.pitch, ye && ynb);
    q.ex_y = ld2(in.e[0], o + g.pitch, ye && ynb);
  };

  float2 exk, eyk, ezk, exn, eyn, ezn, hxm = make_float2(0.f, 0.f), hym = make_float2(0.f, 0.f);
  PairIn cur, nxt;
  load_plane(z0, cur);
  {
    const long long o = fb + (long long)z0 * P + col;
    exk = ld2(in.e[0], o, inb);
    eyk = ld2(in.e[1], o, inb);
    ezk = ld2(in.e[2], o, inb);
    exn = ld2(in.e[0], o + P, inb && z0 + 1 < nz);
    eyn = ld2(in.e[1], o + P, inb && z0 + 1 < nz);
    ezn = ld2(in.e[2], o + P, inb && z0 + 1 < nz);
  }
  if (z0 >= 1 && inb) {  // H(z0-1) of the pair, recomputed from global memory
    const long long po = (long long)(z0 - 1) * P + col, o = fb + po;
    const float2 a = __ldg(reinterpret_cast<const float2*>(loss + mb + po));
    const float2 ez = ld2(in.e[2], o, true), ex = ld2(in.e[0], o, true), ey = ld2(in.e[1], o, true);
    const float2 ez_yp = ld2(in.e[2], o + g.pitch, y + 1 < ny);
    const float ez_x2 = ld(in.e[2], o + 2, x + 2 < nx);
    const float2 hx = ld2(in.h[0], o, true), hy = ld2(in.h[1], o, true);
    float fh, cx, cy, cz;
    hfac(a.x, g, fh, cx, cy, cz);
    hxm.x = fh * hx.x - (cy * (ez_yp.x - ez.x) - cz * (eyk.x - ey.x));
    hym.x = fh * hy.x - (cz * (exk.x - ex.x) - cx * (ez.y - ez.x));
    hfac(a.y, g, fh, cx, cy, cz);
    hxm.y = fh * hx.y - (cy * (ez_yp.y - ez.y) - cz * (eyk.y - ey.y));
    hym.y = fh * hy.y - (cz * (exk.y - ex.y) - cx * (ez_x2 - ez.y));
  }

  for (int k = z0; k < z1; ++k) {
    const long long po = (long long)k * P + col;
    float2 ex2, ey2, ez2;  // prefetch: inputs of plane k+1 and E(k+2)
    if (k + 1 < z1) {
      load_plane(k + 1, nxt);
      const long long o = fb + po + 2 * P;
      ex2 = ld2(in.e[0], o, inb && k + 2 < nz);
      ey2 = ld2(in.e[1], o, inb && k + 2 < nz);
      ez2 = ld2(in.e[2], o, inb && k + 2 < nz);
    }
    float fh0, cx0, cy0, cz0, fh1, cx1, cy1, cz1;
    hfac(cur.a.x, g, fh0, cx0, cy0, cz0);
    hfac(cur.a.y, g, fh1, cx1, cy1, cz1);
    s_ez[ty][tx] = ezk;
    s_ex[ty][tx] = exk;
    __syncthreads();
    const float2 ez_yp = ye ? cur.ez_y : s_ez[ty + (ye ? 0 : 1)][tx];
    const float2 ex_yp = ye ? cur.ex_y : s_ex[ty + (ye ? 0 : 1)][tx];
    float ez_x2 = __shfl_down_sync(FULL, ezk.x, 1);
    float ey_x2 = __shfl_down_sync(FULL, eyk.x, 1);
    if (xe) {
      ez_x2 = cur.ez_x;
      ey_x2 = cur.ey_x;
    }
    float2 hxn, hyn, hzn;
    hxn.x = fh0 * cur.hx.x - (cy0 * (ez_yp.x - ezk.x) - cz0 * (eyn.x - eyk.x));
    hyn.x = fh0 * cur.hy.x - (cz0 * (exn.x - exk.x) - cx0 * (ezk.y - ezk.x));
    hzn.x = fh0 * cur.hz.x - (cx0 * (eyk.y - eyk.x) - cy0 * (ex_yp.x - exk.x));
    hxn.y = fh1 * cur.hx.y - (cy1 * (ez_yp.y - ezk.y) - cz1 * (eyn.y - eyk.y));
    hyn.y = fh1 * cur.hy.y - (cz1 * (exn.y - exk.y) - cx1 * (ez_x2 - ezk.y));
    hzn.y = fh1 * cur.hz.y - (cx1 * (ey_x2 - eyk.y) - cy1 * (ex_yp.y - exk.y));
    s_hz[ty][tx] = hzn;
    s_hx[ty][tx] = hxn;
    __syncthreads();
    const float hy_xm = __shfl_up_sync(FULL, hyn.y, 1);
    const float hz_xm = __shfl_up_sync(FULL, hzn.y, 1);
    if (owned) {
      const long long o = fb + po;
      const float2 hz_ym = s_hz[ty - 1][tx];
      const float2 hx_ym = s_hx[ty - 1][tx];
      const bool kin = k >= 1 && k <= nz - 2, kz = k <= nz - 2;
      const float cv0 = cur.ce.x, cv1 = cur.ce.y;
      const float fe0 = 1.f - cur.a.x * cv0 * g.inv_kd2, fe1 = 1.f - cur.a.y * cv1 * g.inv_kd2;
      float2 ex = exk, ey = eyk, ez = ezk;
      if (kin && yint && x0m) ex.x = fe0 * exk.x + cv0 * ((hzn.x - hz_ym.x) - g.qz * (hyn.x - hym.x));
      if (kin && yint && x1m) ex.y = fe1 * exk.y + cv1 * ((hzn.y - hz_ym.y) - g.qz * (hyn.y - hym.y));
      if (kin && ym && x0p && x0m) ey.x = fe0 * eyk.x + cv0 * (g.qz * (hxn.x - hxm.x) - g.qx * (hzn.x - hz_xm));
      if (kin && ym && x1m) ey.y = fe1 * eyk.y + cv1 * (g.qz * (hxn.y - hxm.y) - g.qx * (hzn.y - hzn.x));
      if (kz && yint && x0p && x0m) ez.x = fe0 * ezk.x + cv0 * (g.qx * (hyn.x - hy_xm) - (hxn.x - hx_ym.x));
      if (kz && yint && x1m) ez.y = fe1 * ezk.y + cv1 * (g.qx * (hyn.y - hyn.x) - (hxn.y - hx_ym.y));
      st2(out.e[0], o, ex, x0m, x1m);
      st2(out.e[1], o, ey, ym, ym && x1in);
      st2(out.e[2], o, ez, kz, kz && x1in);
      st2(out.h[0], o, hxn, kz && ym, kz && ym && x1in);
      st2(out.h[1], o, hyn, kz && x0m, kz && x1m);
      st2(out.h[2], o, hzn, ym && x0m, ym && x1m);
    }
    exk = exn;
    eyk = eyn;
    ezk = ezn;
    exn = ex2;
    eyn = ey2;
    ezn = ez2;
    hxm = hxn;
    hym = hyn;
    cur = nxt;
  }
}

template <int ZB, int TY>
int launch3d_pair(const bz_grid3d* gd, const bz_fields3d* f, int64_t step, cudaStream_t st) {
  Geo3D<float> g;
  g.nx = gd->nx;
  g.ny = gd->ny;
  g.nz = gd->nz;
  g.pitch = gd->pitch;
  g.n_designs = gd->n_designs;
  g.n_mat = gd->n_mat;
  g.n_comp = gd->n_comp;
  g.nzb = (int)ceil_div(gd->nz, ZB);
  g.plane = (long long)gd->ny * gd->pitch;
  g.vol = g.plane * gd->nz;
  g.chx = (float)gd->chx;
  g.chy = (float)gd->chy;
  g.chz = (float)gd->chz;
  g.qx = (float)gd->qx;
  g.qz = (float)gd->qz;
  g.inv_kd2 = (float)gd->inv_kd2;
  const int src = (int)(step & 1);
  Ptr3<float> in;
  Out3<float> out;
  for (int i = 0; i < 3; ++i) {
    in.e[i] = (const float*)f->e[src][i];
    in.h[i] = (const float*)f->h[src][i];
    out.e[i] = (float*)f->e[src ^ 1][i];
    out.h[i] = (float*)f->h[src ^ 1][i];
  }
  dim3 block(TX, TY);
  dim3 grid((unsigned)ceil_div(gd->nx, 2 * TX - 2), (unsigned)ceil_div(gd->ny, TY - 1),
            (unsigned)(g.nzb * gd->n_designs * gd->n_comp));
  step3d_pair_kernel<ZB, TY><<<grid, block, 0, st>>>(in, out, (const float*)f->ce, (const float*)f->loss, g);
  return check_launch("bz_step3d");
}

// ---------------------------------------------------------------------------- quad columns (float32)
// The same schedule with four adjacent x cells per thread, moved as float4: a warp spans
// 128 columns whose first four (one quad, to keep 16-byte alignment) are the halo shared
// with the neighbouring tile, so a block owns 124 x (TY-1) columns. Against the pair
// kernel, loads, stores, shared-memory traffic, shuffles and index arithmetic are issued
// once per four cells. The quad starts at x % 4 == 0; cells past the last real column
// (row padding, pitch % 32 == 0) are read as stored (zero) and never written, and no
// written value depends on them.
__device__ __forceinline__ float4 ld4(const float* p, long long i, bool ok) {
  return ok ? __ldg(reinterpret_cast<const float4*>(p + i)) : make_float4(0.f, 0.f, 0.f, 0.f);
}

// Stores the first n (0..4) cells of a quad: one 16-byte store when all four exist.
__device__ __forceinline__ void st4(float* p, long long i, float4 v, int n) {
  if (n >= 4) {
    *reinterpret_cast<float4*>(p + i) = v;
    return;
  }
  if (n >= 1) p[i] = v.x;
  if (n >= 2) p[i + 1] = v.y;
  if (n >= 3) p[i + 2] = v.z;
}

__device__ __forceinline__ float& q_at(float4& v, int j) { return j == 0 ? v.x : (j == 1 ? v.y : (j == 2 ? v.z : v.w)); }
__device__ __forceinline__ float q_get(const float4& v, int j) {
  return j == 0 ? v.x : (j == 1 ? v.y : (j == 2 ? v.z : v.w));
}

struct QuadIn {
  float4 hx, hy, hz, a, ce, ez_y, ex_y;
  float ez_x, ey_x;  // E at x+4 (the warp's last lane)
};

// One column segment: tile (bx, by) of design/component dc, planes [z0, z1).
template <int TY>
__device__ __forceinline__ void quad_segment(const Ptr3<float>& in, const Out3<float>& out,
                                             const float* __restrict__ ce, const float* __restrict__ loss,
                                             const Geo3D<float>& g, int bx, int by, int dc, int z0, int z1,
                                             float4 (*s_ez)[TX], float4 (*s_ex)[TX], float4 (*s_hz)[TX],
                                             float4 (*s_hx)[TX]) {
  const int tx = threadIdx.x, ty = threadIdx.y;
  const int nx = g.nx, ny = g.ny, nz = g.nz;
  const int x = bx * (4 * TX - 4) - 4 + 4 * tx;  // first cell of the quad
  const int y = by * (TY - 1) - 1 + ty;
  const int d = dc / g.n_comp;
  const bool xin = x >= 0 && x < nx, yin = y >= 0 && y < ny, inb = xin && yin;
  const bool owned = inb && tx >= 1 && ty >= 1;
  const bool xe = tx == TX - 1, ye = ty == TY - 1;
  const bool xnb = yin && x + 4 < nx, ynb = xin && y + 1 < ny;
  // cells of the quad inside each component's x extent (x <= nx-2 or x <= nx-1)
  const int n_m = max(0, min(4, nx - 1 - x)), n_a = max(0, min(4, nx - x));
  const bool yint = y >= 1 && y <= ny - 2, ym = y <= ny - 2;
  const long long P = g.plane;
  const long long mb = (g.n_mat > 1 ? (long long)d : 0LL) * g.vol;
  const long long col = (long long)y * g.pitch + x;
  const long long fb = (long long)dc * g.vol;

  auto load_plane = [&](int k, QuadIn& q) {
    const long long po = (long long)k * P + col;
    q.a = ld4(loss + mb, po, inb);
    q.ce = ld4(ce + mb, po, inb);
    const long long o = fb + po;
    q.hx = ld4(in.h[0], o, inb);
    q.hy = ld4(in.h[1], o, inb);
    q.hz = ld4(in.h[2], o, inb);
    q.ez_x = ld(in.e[2], o + 4, xe && xnb);
    q.ey_x = ld(in.e[1], o + 4, xe && xnb);
    q.ez_y = ld4(in.e[2], o + g.pitch, ye && ynb);
    q.ex_y = ld4(in.e[0], o + g.pitch, ye && ynb);
  };

  float4 exk, eyk, ezk, exn, eyn, ezn, hxm = make_float4(0.f, 0.f, 0.f, 0.f), hym = make_float4(0.f, 0.f, 0.f, 0.f);
  QuadIn cur, nxt;
  load_plane(z0, cur);
  {
    const long long o = fb + (long long)z0 * P + col;
    exk = ld4(in.e[0], o, inb);
    eyk = ld4(in.e[1], o, inb);
    ezk = ld4(in.e[2], o, inb);
    exn = ld4(in.e[0], o + P, inb && z0 + 1 < nz);
    eyn = ld4(in.e[1], o + P, inb && z0 + 1 < nz);
    ezn = ld4(in.e[2], o + P, inb && z0 + 1 < nz);
  }
  if (z0 >= 1 && inb) {  // Hx, Hy at plane z0-1 of the quad, recomputed from global memory
    const long long po = (long long)(z0 - 1) * P + col, o = fb + po;
    const float4 a = __ldg(reinterpret_cast<const float4*>(loss + mb + po));
    const float4 ez = ld4(in.e[2], o, true), ex = ld4(in.e[0], o, true), ey = ld4(in.e[1], o, true);
    const float4 ez_yp = ld4(in.e[2], o + g.pitch, y + 1 < ny);
    const float ez_x4 = ld(in.e[2], o + 4, x + 4 < nx);
    const float4 hx = ld4(in.h[0], o, true), hy = ld4(in.h[1], o, true);
#pragma unroll
    for (int j = 0; j < 4; ++j) {
      float fh, cx, cy, cz;
      hfac(q_get(a, j), g, fh, cx, cy, cz);
      const float ez_xp = j < 3 ? q_get(ez, j + 1) : ez_x4;
      q_at(hxm, j) = fh * q_get(hx, j) - (cy * (q_get(ez_yp, j) - q_get(ez, j)) - cz * (q_get(eyk, j) - q_get(ey, j)));
      q_at(hym, j) = fh * q_get(hy, j) - (cz * (q_get(exk, j) - q_get(ex, j)) - cx * (ez_xp - q_get(ez, j)));
    }
  }

  for (int k = z0; k < z1; ++k) {
    const long long po = (long long)k * P + col;
    float4 ex2, ey2, ez2;  // prefetch: inputs of plane k+1 and E(k+2)
    if (k + 1 < z1) {
      load_plane(k + 1, nxt);
      const long long o = fb + po + 2 * P;
      ex2 = ld4(in.e[0], o, inb && k + 2 < nz);
      ey2 = ld4(in.e[1], o, inb && k + 2 < nz);
      ez2 = ld4(in.e[2], o, inb && k + 2 < nz);
    }
    s_ez[ty][tx] = ezk;
    s_ex[ty][tx] = exk;
    __syncthreads();
    const float4 ez_yp = ye ? cur.ez_y : s_ez[ty + (ye ? 0 : 1)][tx];
    const float4 ex_yp = ye ? cur.ex_y : s_ex[ty + (ye ? 0 : 1)][tx];
    float ez_x4 = __shfl_down_sync(FULL, ezk.x, 1);
    float ey_x4 = __shfl_down_sync(FULL, eyk.x, 1);
    if (xe) {
      ez_x4 = cur.ez_x;
      ey_x4 = cur.ey_x;
    }
    float4 hxn, hyn, hzn, fe4;
#pragma unroll
    for (int j = 0; j < 4; ++j) {
      float fh, cx, cy, cz;
      hfac(q_get(cur.a, j), g, fh, cx, cy, cz);
      const float ez_xp = j < 3 ? q_get(ezk, j + 1) : ez_x4;
      const float ey_xp = j < 3 ? q_get(eyk, j + 1) : ey_x4;
      const float ezc = q_get(ezk, j), eyc = q_get(eyk, j), exc = q_get(exk, j);
      q_at(hxn, j) = fh * q_get(cur.hx, j) - (cy * (q_get(ez_yp, j) - ezc) - cz * (q_get(eyn, j) - eyc));
      q_at(hyn, j) = fh * q_get(cur.hy, j) - (cz * (q_get(exn, j) - exc) - cx * (ez_xp - ezc));
      q_at(hzn, j) = fh * q_get(cur.hz, j) - (cx * (ey_xp - eyc) - cy * (q_get(ex_yp, j) - exc));
      q_at(fe4, j) = 1.f - q_get(cur.a, j) * q_get(cur.ce, j) * g.inv_kd2;
    }
    s_hz[ty][tx] = hzn;
    s_hx[ty][tx] = hxn;
    __syncthreads();
    const float hy_xm = __shfl_up_sync(FULL, hyn.w, 1);
    const float hz_xm = __shfl_up_sync(FULL, hzn.w, 1);
    if (owned) {
      const long long o = fb + po;
      const float4 hz_ym = s_hz[ty - 1][tx];
      const float4 hx_ym = s_hx[ty - 1][tx];
      const bool kin = k >= 1 && k <= nz - 2, kz = k <= nz - 2;
      float4 ex = exk, ey = eyk, ez = ezk;
#pragma unroll
      for (int j = 0; j < 4; ++j) {
        const bool xm = x + j <= nx - 2, xp = x + j >= 1;
        const float cv = q_get(cur.ce, j), fe = q_get(fe4, j);
        const float hzl = j > 0 ? q_get(hzn, j - 1) : hz_xm;
        const float hyl = j > 0 ? q_get(hyn, j - 1) : hy_xm;
        if (kin && yint && xm)
          q_at(ex, j) = fe * q_get(exk, j) + cv * ((q_get(hzn, j) - q_get(hz_ym, j)) - g.qz * (q_get(hyn, j) - q_get(hym, j)));
        if (kin && ym && xp && xm)
          q_at(ey, j) = fe * q_get(eyk, j) + cv * (g.qz * (q_get(hxn, j) - q_get(hxm, j)) - g.qx * (q_get(hzn, j) - hzl));
        if (kz && yint && xp && xm)
          q_at(ez, j) = fe * q_get(ezk, j) + cv * (g.qx * (q_get(hyn, j) - hyl) - (q_get(hxn, j) - q_get(hx_ym, j)));
      }
      st4(out.e[0], o, ex, n_m);
      st4(out.e[1], o, ey, ym ? n_a : 0);
      st4(out.e[2], o, ez, kz ? n_a : 0);
      st4(out.h[0], o, hxn, (kz && ym) ? n_a : 0);
      st4(out.h[1], o, hyn, kz ? n_m : 0);
      st4(out.h[2], o, hzn, ym ? n_m : 0);
    }
    exk = exn;
    eyk = eyn;
    ezk = ezn;
    exn = ex2;
    eyn = ey2;
    ezn = ez2;
    hxm = hxn;
    hym = hyn;
    cur = nxt;
  }
}

// One block per (x tile, y tile, z block of ZB planes, design-component).
template <int ZB, int TY>
__global__ void __launch_bounds__(TX * TY, TY == 8 ? 2 : 1) step3d_quad_kernel(Ptr3<float> in, Out3<float> out,
                                                                  const float* __restrict__ ce,
                                                                  const float* __restrict__ loss,
                                                                  Geo3D<float> g) {
  __shared__ float4 s_ez[TY][TX], s_ex[TY][TX], s_hz[TY][TX], s_hx[TY][TX];
  const int dc = blockIdx.z / g.nzb;
  const int z0 = (blockIdx.z - dc * g.nzb) * ZB;
  quad_segment<TY>(in, out, ce, loss, g, blockIdx.x, blockIdx.y, dc, z0, min(z0 + ZB, g.nz), s_ez, s_ex, s_hz, s_hx);
}

template <int TY>
int launch3d_quad(const bz_grid3d* gd, const bz_fields3d* f, int64_t step, cudaStream_t st) {
  Geo3D<float> g;
  g.nx = gd->nx;
  g.ny = gd->ny;
  g.nz = gd->nz;
  g.pitch = gd->pitch;
  g.n_designs = gd->n_designs;
  g.n_mat = gd->n_mat;
  g.n_comp = gd->n_comp;
  g.nzb = 1;
  g.plane = (long long)gd->ny * gd->pitch;
  g.vol = g.plane * gd->nz;
  g.chx = (float)gd->chx;
  g.chy = (float)gd->chy;
  g.chz = (float)gd->chz;
  g.qx = (float)gd->qx;
  g.qz = (float)gd->qz;
  g.inv_kd2 = (float)gd->inv_kd2;
  const int src = (int)(step & 1);
  Ptr3<float> in;
  Out3<float> out;
  for (int i = 0; i < 3; ++i) {
    in.e[i] = (const float*)f->e[src][i];
    in.h[i] = (const float*)f->h[src][i];
    out.e[i] = (float*)f->e[src ^ 1][i];
    out.h[i] = (float*)f->h[src ^ 1][i];
  }
  const int n_xt = (int)ceil_div(gd->nx, 4 * TX - 4), n_yt = (int)ceil_div(gd->ny, TY - 1);
  dim3 block(TX, TY);
  const int zb = gd->tile_z == 8 ? 8 : 16;
  g.nzb = (int)ceil_div(gd->nz, zb);
  dim3 grid((unsigned)n_xt, (unsigned)n_yt, (unsigned)(g.nzb * gd->n_designs * gd->n_comp));
  if (zb == 8)
    step3d_quad_kernel<8, TY><<<grid, block, 0, st>>>(in, out, (const float*)f->ce, (const float*)f->loss, g);
  else
    step3d_quad_kernel<16, TY><<<grid, block, 0, st>>>(in, out, (const float*)f->ce, (const float*)f->loss, g);
  return check_launch("bz_step3d");
}

inline bool vec_aligned(const bz_fields3d* f, uintptr_t bytes) {
  bool ok = ((uintptr_t)f->ce | (uintptr_t)f->loss) % bytes == 0;
  for (int c = 0; c < 2; ++c)
    for (int i = 0; i < 3; ++i) ok = ok && ((uintptr_t)f->e[c][i] | (uintptr_t)f->h[c][i]) % bytes == 0;
  return ok;
}

// float2 accesses need every array 8-byte aligned (offsets are even: pitch % 32 == 0).
inline bool pair_aligned(const bz_fields3d* f) {
  bool ok = ((uintptr_t)f->ce | (uintptr_t)f->loss) % 8 == 0;
  for (int c = 0; c < 2; ++c)
    for (int i = 0; i < 3; ++i) ok = ok && ((uintptr_t)f->e[c][i] | (uintptr_t)f->h[c][i]) % 8 == 0;
  return ok;
}

template <typename T, int TY>
int dispatch3d_ty(const bz_grid3d* g, const bz_fields3d* f, int64_t step, cudaStream_t st) {
  const bool z8 = g->tile_z == 8;  // 0 takes 16-plane z blocks
  if (g->n_comp == 1) return z8 ? launch3d<T, 1, 8, TY>(g, f, step, st) : launch3d<T, 1, 16, TY>(g, f, step, st);
  return z8 ? launch3d<T, 2, 8, TY>(g, f, step, st) : launch3d<T, 2, 16, TY>(g, f, step, st);
}

template <typename T>
int dispatch3d(const bz_grid3d* g, const bz_fields3d* f, int64_t step, cudaStream_t st) {
  const bool zfit = (long long)g->n_designs * g->n_comp * ceil_div(g->nz, 8) <= 65535;
  if (sizeof(T) == 4 && (g->x_cells == 0 || g->x_cells == 4) && vec_aligned(f, 16) && zfit) {
    return g->tile_y == 16 ? launch3d_quad<16>(g, f, step, st) : launch3d_quad<8>(g, f, step, st);
  }
  if (sizeof(T) == 4 && g->x_cells != 1 && pair_aligned(f) && zfit) {
    const bool z8 = g->tile_z == 8;
    if (g->tile_y == 16) return z8 ? launch3d_pair<8, 16>(g, f, step, st) : launch3d_pair<16, 16>(g, f, step, st);
    return z8 ? launch3d_pair<8, 8>(g, f, step, st) : launch3d_pair<16, 8>(g, f, step, st);
  }
  return g->tile_y == 16 ? dispatch3d_ty<T, 16>(g, f, step, st) : dispatch3d_ty<T, 8>(g, f, step, st);
}

// ---------------------------------------------------------------------------- cell ops
template <typename T>
__global__ void cell_ops_kernel(T* __restrict__ field, int n_comp, long long comp_stride, int nx, int pitch,
                                int n_ops, int n_steps, const int* __restrict__ cell, const T* __restrict__ mul,
                                const T* __restrict__ w, long long w_stride, const int* __restrict__ sig,
                                const T* __restrict__ signals, long long step_base,
                                const long long* __restrict__ d_step) {
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= n_ops) return;
  const int c0 = __ldg(cell + k);
  if (k > 0 && __ldg(cell + k - 1) == c0) return;  // the first op of a cell applies its whole run
  const long long step = d_step ? (__ldg(d_step) + step_base) : step_base;
  const int d = blockIdx.y;
  const long long off = (long long)(c0 / nx) * pitch + (c0 % nx);
  for (int c = 0; c < n_comp; ++c) {
    T* p = field + ((long long)d * n_comp + c) * comp_stride + off;
    T v = *p;
    for (int kk = k; kk < n_ops && __ldg(cell + kk) == c0; ++kk) {
      const T s = step < n_steps ? __ldg(signals + (long long)__ldg(sig + kk) * n_steps + step) : T(0);
      v = __ldg(mul + kk) * v + __ldg(w + d * w_stride + (long long)kk * n_comp + c) * s;
    }
    *p = v;
  }
}

// ---------------------------------------------------------------------------- gather
template <typename T>
struct GatherArgs {
  int n_points, n_q, n_designs, n_comp, n_rec, ring_len;
  const T* src[6];
  const long long* offset;
  T* record;
  T* ring;
  long long rec_step0, comp_stride;
};

template <typename T>
__global__ void gather_kernel(GatherArgs<T> a, long long step_base, const long long* __restrict__ d_step) {
  const long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;  // (point, q)
  const long long total = (long long)a.n_points * a.n_q;
  if (i >= total) return;
  const long long step = d_step ? (__ldg(d_step) + step_base) : step_base;
  const int p = (int)(i / a.n_q), q = (int)(i - (long long)p * a.n_q);
  const long long off = __ldg(a.offset + i);
  const int dc = blockIdx.y;  // design * n_comp + comp
  const T v = off >= 0 ? __ldg(a.src[q] + dc * a.comp_stride + off) : T(0);
  const long long tail = ((long long)dc * a.n_points + p) * a.n_q + q;
  const long long per = (long long)a.n_designs * a.n_comp * a.n_points * a.n_q;
  if (a.record && step >= a.rec_step0 && step < a.rec_step0 + a.n_rec) a.record[(step - a.rec_step0) * per + tail] = v;
  if (a.ring) a.ring[(step % a.ring_len) * per + tail] = v;
}

// ---------------------------------------------------------------------------- power
template <typename T, int NC>
__global__ void power3d_kernel(Ptr3<T> f, Geo3D<T> g, double* __restrict__ pw) {
  const int x = blockIdx.x * blockDim.x + threadIdx.x;
  const int y = blockIdx.y;
  const int kd = blockIdx.z;  // design * (nz-1) + k
  const int mz = g.nz - 1, my = g.ny - 1, mx = g.nx - 1;
  if (x >= mx) return;
  const int d = kd / mz, k = kd - d * mz;
  const long long o = (long long)k * g.plane + (long long)y * g.pitch + x;
  double sx = 0, sy = 0, sz = 0;
  for (int c = 0; c < NC; ++c) {  // Re(a conj(b)) summed over the (re, im) parts
    const long long b = ((long long)d * NC + c) * g.vol + o;
    const double ex = __ldg(f.e[0] + b), ey = __ldg(f.e[1] + b), ez = __ldg(f.e[2] + b);
    const double hx = __ldg(f.h[0] + b), hy = __ldg(f.h[1] + b), hz = __ldg(f.h[2] + b);
    sx += ey * hz - ez * hy;
    sy += ez * hx - ex * hz;
    sz += ex * hy - ey * hx;
  }
  pw[(((long long)d * mz + k) * my + y) * mx + x] += sqrt(sx * sx + sy * sy + sz * sz);
}

}  // namespace
}  // namespace bz

extern "C" int bz_step3d(const bz_grid3d* g, const bz_fields3d* f, int64_t step, void* stream) {
  BZ_REQUIRE(g && f, "bz_step3d: grid or fields is NULL");
  BZ_REQUIRE(g->nx >= 2 && g->ny >= 2 && g->nz >= 2, "bz_step3d: grid must be at least 2x2x2");
  BZ_REQUIRE(g->pitch >= g->nx && g->pitch % 32 == 0, "bz_step3d: pitch %d must be >= nx and a multiple of 32",
             g->pitch);
  BZ_REQUIRE(g->n_comp == 1 || g->n_comp == 2, "bz_step3d: n_comp must be 1 or 2");
  BZ_REQUIRE(g->n_designs >= 1 && g->n_designs * bz::ceil_div(g->nz, 8) <= 65535, "bz_step3d: too many designs");
  BZ_REQUIRE(g->n_mat == 1 || g->n_mat == g->n_designs, "bz_step3d: n_mat must be 1 or n_designs");
  BZ_REQUIRE(g->tile_z == 0 || g->tile_z == 8 || g->tile_z == 16, "bz_step3d: tile_z must be 0, 8 or 16");
  BZ_REQUIRE(g->tile_y == 0 || g->tile_y == 8 || g->tile_y == 16, "bz_step3d: tile_y must be 0, 8 or 16");
  BZ_REQUIRE(g->x_cells == 0 || g->x_cells == 1 || g->x_cells == 2 || g->x_cells == 4,
             "bz_step3d: x_cells must be 0, 1, 2 or 4");
  for (int c = 0; c < 2; ++c)
    for (int i = 0; i < 3; ++i) BZ_REQUIRE(f->e[c][i] && f->h[c][i], "bz_step3d: field buffer is NULL");
  BZ_REQUIRE(f->ce && f->loss, "bz_step3d: coefficient arrays are NULL");
  BZ_REQUIRE(step >= 0, "bz_step3d: negative step");
  cudaStream_t st = bz::as_stream(stream);
  if (g->dtype == BZ_F32) return bz::dispatch3d<float>(g, f, step, st);
  if (g->dtype == BZ_F64) return bz::dispatch3d<double>(g, f, step, st);
  return bz::fail(BZ_ERR_INVALID, "bz_step3d: unknown dtype %d", g->dtype);
}

extern "C" int bz_cell_ops(void* field, int32_t dtype, int32_t n_designs, int32_t n_comp, int64_t comp_stride,
                           int32_t nx, int32_t pitch, const bz_source_ops* ops, int64_t step, const int64_t* d_step,
                           void* stream) {
  BZ_REQUIRE(field && ops, "bz_cell_ops: NULL field or ops");
  if (ops->n_ops == 0) return BZ_OK;
  BZ_REQUIRE(ops->cell && ops->mul && ops->weight && ops->sig && ops->signals, "bz_cell_ops: incomplete ops");
  BZ_REQUIRE(nx >= 1 && pitch >= nx && n_designs >= 1 && (n_comp == 1 || n_comp == 2), "bz_cell_ops: bad shape");
  dim3 grid((unsigned)bz::ceil_div(ops->n_ops, 128), (unsigned)n_designs);
  cudaStream_t st = bz::as_stream(stream);
  if (dtype == BZ_F32)
    bz::cell_ops_kernel<float><<<grid, 128, 0, st>>>((float*)field, n_comp, comp_stride, nx, pitch, ops->n_ops,
                                                     ops->n_steps, ops->cell, (const float*)ops->mul,
                                                     (const float*)ops->weight, ops->weight_stride, ops->sig,
                                                     (const float*)ops->signals, step, (const long long*)d_step);
  else if (dtype == BZ_F64)
    bz::cell_ops_kernel<double><<<grid, 128, 0, st>>>((double*)field, n_comp, comp_stride, nx, pitch, ops->n_ops,
                                                      ops->n_steps, ops->cell, (const double*)ops->mul,
                                                      (const double*)ops->weight, ops->weight_stride, ops->sig,
                                                      (const double*)ops->signals, step, (const long long*)d_step);
  else
    return bz::fail(BZ_ERR_INVALID, "bz_cell_ops: unknown dtype %d", dtype);
  return bz::check_launch("bz_cell_ops");
}

template <typename T>
static int gather_t(const bz_gather_ops* o, int32_t n_designs, int32_t n_comp, int64_t comp_stride, int64_t step,
                    const int64_t* d_step, cudaStream_t st) {
  bz::GatherArgs<T> a;
  a.n_points = o->n_points;
  a.n_q = o->n_q;
  a.n_designs = n_designs;
  a.n_comp = n_comp;
  a.n_rec = o->n_rec;
  a.ring_len = o->ring_len;
  for (int q = 0; q < 6; ++q) a.src[q] = (const T*)o->src[q];
  a.offset = (const long long*)o->offset;
  a.record = (T*)o->record;
  a.ring = (T*)o->ring;
  a.rec_step0 = o->rec_step0;
  a.comp_stride = comp_stride;
  const long long total = (long long)o->n_points * o->n_q;
  dim3 grid((unsigned)bz::ceil_div(total, 128), (unsigned)(n_designs * n_comp));
  bz::gather_kernel<T><<<grid, 128, 0, st>>>(a, step, (const long long*)d_step);
  return bz::check_launch("bz_gather");
}

extern "C" int bz_gather(const bz_gather_ops* o, int32_t dtype, int32_t n_designs, int32_t n_comp,
                         int64_t comp_stride, int64_t step, const int64_t* d_step, void* stream) {
  BZ_REQUIRE(o && o->offset, "bz_gather: NULL ops or offsets");
  BZ_REQUIRE(o->n_q >= 1 && o->n_q <= 6 && o->n_points >= 0, "bz_gather: n_q must be 1..6");
  for (int q = 0; q < o->n_q; ++q) BZ_REQUIRE(o->src[q], "bz_gather: source array %d is NULL", q);
  BZ_REQUIRE(o->ring == nullptr || o->ring_len >= 1, "bz_gather: ring without length");
  if (o->n_points == 0 || (!o->record && !o->ring)) return BZ_OK;
  cudaStream_t st = bz::as_stream(stream);
  if (dtype == BZ_F32) return gather_t<float>(o, n_designs, n_comp, comp_stride, step, d_step, st);
  if (dtype == BZ_F64) return gather_t<double>(o, n_designs, n_comp, comp_stride, step, d_step, st);
  return bz::fail(BZ_ERR_INVALID, "bz_gather: unknown dtype %d", dtype);
}

template <typename T>
static int power_t(const bz_grid3d* gd, const bz_fields3d* f, int cur, double* pw, cudaStream_t st) {
  bz::Geo3D<T> g = {};
  g.nx = gd->nx;
  g.ny = gd->ny;
  g.nz = gd->nz;
  g.pitch = gd->pitch;
  g.plane = (long long)gd->ny * gd->pitch;
  g.vol = g.plane * gd->nz;
  bz::Ptr3<T> p;
  for (int i = 0; i < 3; ++i) {
    p.e[i] = (const T*)f->e[cur][i];
    p.h[i] = (const T*)f->h[cur][i];
  }
  dim3 grid((unsigned)bz::ceil_div(gd->nx - 1, 128), (unsigned)(gd->ny - 1), (unsigned)(gd->n_designs * (gd->nz - 1)));
  if (gd->n_comp == 1)
    bz::power3d_kernel<T, 1><<<grid, 128, 0, st>>>(p, g, pw);
  else
    bz::power3d_kernel<T, 2><<<grid, 128, 0, st>>>(p, g, pw);
  return bz::check_launch("bz_power3d");
}

extern "C" int bz_power3d(const bz_grid3d* g, const bz_fields3d* f, int32_t cur, double* power, void* stream) {
  BZ_REQUIRE(g && f && power, "bz_power3d: NULL argument");
  BZ_REQUIRE(cur == 0 || cur == 1, "bz_power3d: cur must be 0 or 1");
  BZ_REQUIRE(g->nx >= 2 && g->ny >= 2 && g->nz >= 2 && (g->n_comp == 1 || g->n_comp == 2), "bz_power3d: bad shape");
  BZ_REQUIRE((long long)g->n_designs * (g->nz - 1) <= 65535 && g->ny - 1 <= 65535, "bz_power3d: grid too large");
  cudaStream_t st = bz::as_stream(stream);
  if (g->dtype == BZ_F32) return power_t<float>(g, f, cur, power, st);
  if (g->dtype == BZ_F64) return power_t<double>(g, f, cur, power, st);
  return bz::fail(BZ_ERR_INVALID, "bz_power3d: unknown dtype %d", g->dtype);
}
