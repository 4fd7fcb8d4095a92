// Design -> (eps, mu, sigma) rasteriser, one thread per cell.
//
// Reproduces beamz/simulation/meshing.py:92-536 (RegularGrid.__rasterize__) cell by
// cell: background fill, then every structure in painter's order through the same
// fast path the reference picks for it (axis-aligned rectangle 193-257, circle
// 259-307, ring 309-361, general polygon 362-477), then the additive PML pass
// (484-531, beamz/design/pml.py:29-62). The host resolves everything that is a
// function of the structure alone (index boxes, which path applies, Python slice
// semantics, the PML grading profile); the kernel does the per-cell arithmetic.
//
// Every floating-point operation uses an explicitly rounded intrinsic so that no
// multiply-add is contracted: the sample tests then round exactly as NumPy does
// and the output is bit-identical to the reference for the same inputs.
#include "bz_internal.cuh"

namespace bz {
namespace {

__device__ __forceinline__ double fadd(double a, double b) { return __dadd_rn(a, b); }
__device__ __forceinline__ double fsub(double a, double b) { return __dsub_rn(a, b); }
__device__ __forceinline__ double fmul(double a, double b) { return __dmul_rn(a, b); }
__device__ __forceinline__ double fdiv(double a, double b) { return __ddiv_rn(a, b); }

// hypot(a, b) by the corrected algorithm of C. F. Borges, "An Improved Algorithm
// for hypot(a,b)" (2019, arXiv:1904.09481), non-fused variant: one square root of
// the rounded sum of squares followed by one correction step. Finite inputs of
// moderate magnitude only (cell coordinates).
__device__ double hypot_borges(double a, double b) {
  double ax = fabs(a), ay = fabs(b);
  if (ax < ay) {
    const double t = ax;
    ax = ay;
    ay = t;
  }
  if (ay <= fmul(ax, 0x1p-54)) return fadd(ax, ay);
  double h = __dsqrt_rn(fadd(fmul(ax, ax), fmul(ay, ay)));
  double t1, t2;
  if (h <= fmul(2.0, ay)) {
    const double delta = fsub(h, ay);
    t1 = fmul(ax, fsub(fmul(2.0, delta), ax));
    t2 = fmul(fsub(delta, fmul(2.0, fsub(ax, ay))), delta);
  } else {
    const double delta = fsub(h, ax);
    t1 = fmul(fmul(2.0, delta), fsub(ax, fmul(2.0, ay)));
    t2 = fadd(fmul(fsub(fmul(4.0, delta), ay), ay), fmul(delta, delta));
  }
  h = fsub(h, fdiv(fadd(t1, t2), fmul(2.0, h)));
  return h;
}

// Even-odd crossing test of one closed path (beamz/design/structures.py:178-196).
__device__ bool in_path(double x, double y, const double* __restrict__ v, int n) {
  if (n <= 0) return false;
  bool inside = false;
  double p1x = v[0], p1y = v[1];
  for (int i = 0; i <= n; ++i) {
    const int k = (i % n) * 2;
    const double p2x = v[k], p2y = v[k + 1];
    if (y > fmin(p1y, p2y) && y <= fmax(p1y, p2y) && x <= fmax(p1x, p2x)) {
      double xint = p1x;
      if (p1y != p2y) xint = fadd(fdiv(fmul(fsub(y, p1y), fsub(p2x, p1x)), fsub(p2y, p1y)), p1x);
      if (p1x == p2x || x <= xint) inside = !inside;
    }
    p1x = p2x;
    p1y = p2y;
  }
  return inside;
}

// structures.py:198-207: inside the exterior path and outside every hole.
__device__ bool in_polygon(double x, double y, const bz_shape2d& s, const int* __restrict__ paths,
                           const double* __restrict__ verts) {
  if (s.npath <= 0) return false;
  const int* p = paths + 2 * s.path0;
  if (!in_path(x, y, verts + 2 * (long long)p[0], p[1])) return false;
  for (int h = 1; h < s.npath; ++h)
    if (in_path(x, y, verts + 2 * (long long)p[2 * h], p[2 * h + 1])) return false;
  return true;
}

__device__ __forceinline__ void blend(double& e, double& m, double& c, double bf, double pe, double pm, double pc) {
  // value * (1 - blend_factor) + material * blend_factor  (meshing.py:251-253)
  const double w = fsub(1.0, bf);
  e = fadd(fmul(e, w), fmul(pe, bf));
  m = fadd(fmul(m, w), fmul(pm, bf));
  c = fadd(fmul(c, w), fmul(pc, bf));
}

__global__ void rasterize2d_kernel(int nx, int ny, const double* __restrict__ xc, const double* __restrict__ yc,
                                   const double* __restrict__ offs, const double* __restrict__ corner,
                                   const double* __restrict__ bg, const bz_shape2d* __restrict__ shapes,
                                   int n_shapes, const int* __restrict__ paths, const double* __restrict__ verts,
                                   const double* __restrict__ custom, const bz_pml2d* __restrict__ pmls, int n_pml,
                                   const double* __restrict__ pml_table, double dx, double eps0, double mu0,
                                   double* __restrict__ eps_out, double* __restrict__ mu_out,
                                   double* __restrict__ sig_out) {
  const int j = blockIdx.x * blockDim.x + threadIdx.x;
  const int i = blockIdx.y * blockDim.y + threadIdx.y;
  if (i >= ny || j >= nx) return;
  const double X = xc[j], Y = yc[i];
  double e = bg[0], m = bg[1], c = bg[2];
  const double o0 = offs[0], o1 = offs[1], o2 = offs[2];
  const double sx[9] = {fadd(X, o0), fadd(X, o1), fadd(X, o2), fadd(X, o0), fadd(X, o1),
                        fadd(X, o2), fadd(X, o0), fadd(X, o1), fadd(X, o2)};
  const double sy[9] = {fadd(Y, o0), fadd(Y, o0), fadd(Y, o0), fadd(Y, o1), fadd(Y, o1),
                        fadd(Y, o1), fadd(Y, o2), fadd(Y, o2), fadd(Y, o2)};

  for (int k = 0; k < n_shapes; ++k) {
    const bz_shape2d s = shapes[k];
    if (s.kind == BZ_SHAPE_RECT) {
      const bool in_box = i >= s.i0 && i < s.i1 && j >= s.j0 && j < s.j1;
      double pe = s.perm, pm = s.permb, pc = s.cond;
      if (s.custom_off >= 0 && in_box) {
        const double* t = custom + 3 * (s.custom_off + (long long)(i - s.i0) * (s.j1 - s.j0) + (j - s.j0));
        pe = t[0];
        pm = t[1];
        pc = t[2];
      }
      if (s.fill && i >= s.fi0 && i < s.fi1 && j >= s.fj0 && j < s.fj1) {
        e = pe;
        m = pm;
        c = pc;
      }
      if (in_box) {
        const int r = i - s.i0, q = j - s.j0;
        if (r < s.top || r >= s.bottom || q < s.left || q >= s.right) {
          int cnt = 0;
#pragma unroll
          for (int t = 0; t < 9; ++t) cnt += (s.p0 <= sx[t] && sx[t] < s.p1 && s.p2 <= sy[t] && sy[t] < s.p3);
          if (cnt > 0) blend(e, m, c, fdiv((double)cnt, 9.0), pe, pm, pc);
        }
      }
    } else {
      if (i < s.i0 || i >= s.i1 || j < s.j0 || j >= s.j1) continue;
      if (s.kind == BZ_SHAPE_CIRCLE || s.kind == BZ_SHAPE_RING) {
        const double ddx = fsub(X, s.p0), ddy = fsub(Y, s.p1);
        const double dist = __dsqrt_rn(fadd(fmul(ddx, ddx), fmul(ddy, ddy)));
        bool full, bnd;
        if (s.kind == BZ_SHAPE_CIRCLE) {
          full = fadd(dist, s.q) <= s.p2;
          bnd = (fsub(dist, s.q) <= s.p2) && !full;
        } else {
          full = (fsub(dist, s.q) >= s.p2) && (fadd(dist, s.q) <= s.p3);
          const bool ib = (fsub(dist, s.q) <= s.p2) && (fadd(dist, s.q) >= s.p2);
          const bool ob = (fsub(dist, s.q) <= s.p3) && (fadd(dist, s.q) >= s.p3);
          bnd = ib || ob;
        }
        if (full) {
          e = s.perm;
          m = s.permb;
          c = s.cond;
        }
        if (bnd) {
          int cnt = 0;
          for (int t = 0; t < 9; ++t) {
            const double h = hypot_borges(fsub(sx[t], s.p0), fsub(sy[t], s.p1));
            cnt += (s.kind == BZ_SHAPE_CIRCLE) ? (h <= s.p2) : (s.p2 <= h && h <= s.p3);
          }
          if (cnt > 0) blend(e, m, c, fdiv((double)cnt, 9.0), s.perm, s.permb, s.cond);
        }
      } else {  // BZ_SHAPE_POLYGON: 5-point classification, then 9-sample blend
        int n5 = in_polygon(X, Y, s, paths, verts) ? 1 : 0;
        const bool centre = n5 == 1;
        const double cs0 = corner[0], cs1 = corner[1];
        n5 += in_polygon(fadd(X, cs0), fadd(Y, cs0), s, paths, verts);
        n5 += in_polygon(fadd(X, cs0), fadd(Y, cs1), s, paths, verts);
        n5 += in_polygon(fadd(X, cs1), fadd(Y, cs0), s, paths, verts);
        n5 += in_polygon(fadd(X, cs1), fadd(Y, cs1), s, paths, verts);
        if (centre && n5 == 5) {
          e = s.perm;
          m = s.permb;
          c = s.cond;
        } else {
          int cnt = 0;
          for (int t = 0; t < 9; ++t) cnt += in_polygon(sx[t], sy[t], s, paths, verts);
          if (cnt > 0) blend(e, m, c, fdiv((double)cnt, 9.0), s.perm, s.permb, s.cond);
        }
      }
    }
  }

  // PML pass: conductivity += sigma_max(eps) * profile * frequency_factor (pml.py:31-62)
  for (int b = 0; b < n_pml; ++b) {
    const bz_pml2d p = pmls[b];
    if (i < p.i0 || i >= p.i1 || j < p.j0 || j >= p.j1) continue;
    const long long idx = p.table_off + (long long)(i - p.i0) * (p.j1 - p.j0) + (j - p.j0);
    const double prof = pml_table[2 * idx], ff = pml_table[2 * idx + 1];
    if (prof < 0.0) continue;
    const double eta = __dsqrt_rn(fdiv(mu0, fmul(eps0, e)));
    double smax = fdiv(1.2, fmul(eta, dx));
    smax = fmul(smax, p.sigma_factor);
    double cond = fmul(smax, prof);
    cond = fmul(cond, ff);
    if (cond > 0.0) c = fadd(c, cond);
  }
  const long long o = (long long)i * nx + j;
  eps_out[o] = e;
  mu_out[o] = m;
  sig_out[o] = c;
}

}  // namespace
}  // namespace bz

extern "C" int bz_rasterize2d(int32_t nx, int32_t ny, const double* xc, const double* yc, const double* offs,
                              const double* corner, const double* bg, const bz_shape2d* shapes, int32_t n_shapes,
                              const int32_t* paths, const double* verts, const double* custom, const bz_pml2d* pmls,
                              int32_t n_pml, const double* pml_table, double dx, double eps0, double mu0,
                              double* eps, double* mu, double* sigma, void* stream) {
  BZ_REQUIRE(nx >= 1 && ny >= 1, "bz_rasterize2d: empty grid %d x %d", nx, ny);
  BZ_REQUIRE(xc && yc && offs && corner && bg && eps && mu && sigma, "bz_rasterize2d: NULL buffer");
  BZ_REQUIRE(n_shapes >= 0 && n_pml >= 0, "bz_rasterize2d: negative counts");
  BZ_REQUIRE(n_shapes == 0 || shapes, "bz_rasterize2d: shapes is NULL");
  BZ_REQUIRE(n_pml == 0 || (pmls && pml_table), "bz_rasterize2d: PML tables are NULL");
  dim3 block(32, 8);
  dim3 grid((unsigned)bz::ceil_div(nx, 32), (unsigned)bz::ceil_div(ny, 8));
  bz::rasterize2d_kernel<<<grid, block, 0, bz::as_stream(stream)>>>(nx, ny, xc, yc, offs, corner, bg, shapes,
                                                                     n_shapes, paths, verts, custom, pmls, n_pml,
                                                                     pml_table, dx, eps0, mu0, eps, mu, sigma);
  return bz::check_launch("bz_rasterize2d");
}

namespace bz {
namespace {

__device__ __forceinline__ double pml_term(double eps, double prof, double ff, double sf, double dx, double eps0,
                                           double mu0) {
  const double eta = __dsqrt_rn(fdiv(mu0, fmul(eps0, eps)));
  double smax = fdiv(1.2, fmul(eta, dx));
  smax = fmul(smax, sf);
  return fmul(fmul(smax, prof), ff);
}

__global__ void rasterize3d_kernel(int nx, int ny, int nz, int n_zs, const double* __restrict__ xc,
                                   const double* __restrict__ yc, const double* __restrict__ offs,
                                   const double* __restrict__ bg, const bz_shape3d* __restrict__ shapes, int n_shapes,
                                   const int* __restrict__ zw, const int* __restrict__ paths,
                                   const double* __restrict__ verts, const bz_pml2d* __restrict__ pmls, int n_pml,
                                   const double* __restrict__ pml_table, const double* __restrict__ prof_z,
                                   double sf_z, double dx, double eps0, double mu0, double* __restrict__ eps_out,
                                   double* __restrict__ mu_out, double* __restrict__ sig_out) {
  const int j = blockIdx.x * blockDim.x + threadIdx.x;
  const int i = blockIdx.y * blockDim.y + threadIdx.y;
  const int k = blockIdx.z;
  if (i >= ny || j >= nx) return;
  const double X = xc[j], Y = yc[i];
  double e = bg[0], m = bg[1], c = bg[2];
  const double o0 = offs[0], o1 = offs[1], o2 = offs[2];
  const double sx[9] = {fadd(X, o0), fadd(X, o1), fadd(X, o2), fadd(X, o0), fadd(X, o1),
                        fadd(X, o2), fadd(X, o0), fadd(X, o1), fadd(X, o2)};
  const double sy[9] = {fadd(Y, o0), fadd(Y, o0), fadd(Y, o0), fadd(Y, o1), fadd(Y, o1),
                        fadd(Y, o1), fadd(Y, o2), fadd(Y, o2), fadd(Y, o2)};
  for (int s_i = 0; s_i < n_shapes; ++s_i) {
    const bz_shape3d s = shapes[s_i];
    if (k < s.k0 || k >= s.k1 || i < s.i0 || i >= s.i1 || j < s.j0 || j >= s.j1) continue;
    const int w = zw[s.zw_off + (k - s.k0)];
    if (w == 0) continue;
    bz_shape2d p;
    p.path0 = s.path0;
    p.npath = s.npath;
    int cnt = 0;
    for (int t = 0; t < 9; ++t) cnt += in_polygon(sx[t], sy[t], p, paths, verts);
    if (cnt > 0) blend(e, m, c, fdiv((double)(cnt * w), (double)(9 * n_zs)), s.perm, s.permb, s.cond);
  }
  for (int b = 0; b < n_pml; ++b) {
    const bz_pml2d p = pmls[b];
    if (i < p.i0 || i >= p.i1 || j < p.j0 || j >= p.j1) continue;
    const long long idx = p.table_off + (long long)(i - p.i0) * (p.j1 - p.j0) + (j - p.j0);
    const double prof = pml_table[2 * idx], ff = pml_table[2 * idx + 1];
    if (prof < 0.0) continue;
    const double cond = pml_term(e, prof, ff, p.sigma_factor, dx, eps0, mu0);
    if (cond > 0.0) c = fadd(c, cond);
  }
  if (prof_z != nullptr && prof_z[2 * k] >= 0.0) {
    const double cond = pml_term(e, prof_z[2 * k], prof_z[2 * k + 1], sf_z, dx, eps0, mu0);
    if (cond > 0.0) c = fadd(c, cond);
  }
  const long long o = ((long long)k * ny + i) * nx + j;
  eps_out[o] = e;
  mu_out[o] = m;
  sig_out[o] = c;
}

}  // namespace
}  // namespace bz

extern "C" int bz_rasterize3d(int32_t nx, int32_t ny, int32_t nz, int32_t n_zs, const double* xc, const double* yc,
                              const double* offs, const double* bg, const bz_shape3d* shapes, int32_t n_shapes,
                              const int32_t* zw, const int32_t* paths, const double* verts, const bz_pml2d* pmls,
                              int32_t n_pml, const double* pml_table, const double* prof_z, double sigma_factor_z,
                              double dx, double eps0, double mu0, double* eps, double* mu, double* sigma,
                              void* stream) {
  BZ_REQUIRE(nx >= 1 && ny >= 1 && nz >= 1 && nz <= 65535, "bz_rasterize3d: bad grid %d x %d x %d", nx, ny, nz);
  BZ_REQUIRE(n_zs == 1 || n_zs == 3, "bz_rasterize3d: n_zs must be 1 or 3");
  BZ_REQUIRE(xc && yc && offs && bg && eps && mu && sigma, "bz_rasterize3d: NULL buffer");
  BZ_REQUIRE(n_shapes == 0 || (shapes && zw && paths && verts), "bz_rasterize3d: shape tables are NULL");
  BZ_REQUIRE(n_pml == 0 || (pmls && pml_table), "bz_rasterize3d: PML tables are NULL");
  dim3 block(32, 8);
  dim3 grid((unsigned)bz::ceil_div(nx, 32), (unsigned)bz::ceil_div(ny, 8), (unsigned)nz);
  bz::rasterize3d_kernel<<<grid, block, 0, bz::as_stream(stream)>>>(
      nx, ny, nz, n_zs, xc, yc, offs, bg, shapes, n_shapes, zw, paths, verts, pmls, n_pml, pml_table, prof_z,
      sigma_factor_z, dx, eps0, mu0, eps, mu, sigma);
  return bz::check_launch("bz_rasterize3d");
}
