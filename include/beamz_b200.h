/*
 * beamz_b200 — C ABI of the B200-native FDTD stepping library (libbeamz_b200.so).
 *
 * Conventions
 *   - Plain C types only: pointers are device pointers unless stated otherwise,
 *     sizes are element counts. No C++ exceptions cross this boundary.
 *   - Every entry returns an int status: BZ_OK (0) or a negative BZ_ERR_* code.
 *     bz_last_error() copies the message of the last failure on this thread.
 *   - The library allocates no device memory. Callers own every buffer.
 *   - Streams are passed as void* (a cudaStream_t); NULL is the legacy stream.
 *   - Layouts: 2D arrays are row-major [y][x] with x contiguous and a row pitch
 *     (elements) that is a multiple of 32; a batch of fields is laid out as
 *     [design][component][ny][pitch]. 3D arrays are [z][y][x], x contiguous,
 *     with the same padded pitch and a plane stride of ny*pitch.
 *   - dtype codes: BZ_F32 (0) or BZ_F64 (1) for field and coefficient arrays.
 *
 * Reference interfaces replaced (paths inside the beamz project):
 *   bz_step2d       beamz/simulation/backends/numpy_backend.py:34-88
 *                   (update_h_fields + update_e_field), beamz/simulation/helper.py:5-118
 *                   (apply_sources), helper.py:120-187 (accumulate_power),
 *                   helper.py:231-256 + beamz/devices/monitors.py:279-315 (record_monitor_data)
 *   bz_step3d       beamz/simulation/fdtd.py:200-310 (_update_3d_fields) + the same helpers
 *   bz_prepare_coeffs  the per-step coefficient arithmetic of numpy_backend.py:52-60,80-84
 *                   and fdtd.py:232-305, hoisted out of the time loop
 *   bz_rasterize2d  beamz/simulation/meshing.py:92-536 (RegularGrid.__rasterize__)
 *   bz_rasterize3d  beamz/simulation/meshing.py:616-781 (RegularGrid3D.__rasterize_3d__)
 */
#ifndef BEAMZ_B200_H
#define BEAMZ_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define BZ_OK 0
#define BZ_ERR_INVALID (-1)     /* bad argument: null pointer, shape, stride, dtype */
#define BZ_ERR_CUDA (-2)        /* a CUDA runtime call failed */
#define BZ_ERR_DIVERGED (-3)    /* non-finite or runaway field detected */
#define BZ_ERR_TIMEOUT (-4)     /* a bounded device wait ran out */
#define BZ_ERR_UNSUPPORTED (-5) /* valid request that this build does not handle */

#define BZ_F32 0
#define BZ_F64 1

/* Library version string, e.g. "beamz_b200 0.1.0 sm_100a". Never fails. */
const char* bz_version(void);

/* Copies the last error message of the calling thread into buf (NUL-terminated,
 * truncated to len). Returns the status code of that error (BZ_OK if none). */
int bz_last_error(char* buf, size_t len);

/* ----------------------------------------------------------------------------
 * Grid description shared by the 2D entries.
 *   nx, ny        cells of the permittivity grid (RegularGrid.permittivity.shape = (ny, nx))
 *   pitch         row pitch in elements (>= nx, multiple of 32)
 *   n_designs     independent designs stepped in one launch
 *   n_comp        field components per design: 1 = real field, 2 = (Re, Im)
 *   n_mat         coefficient sets: 1 (shared by all designs) or n_designs
 *   dtype         BZ_F32 / BZ_F64 for fields and coefficients
 *   chx, chy      dt/(mu0*dy) and dt/(mu0*dx): H-update factors for x- and y-differences
 *                 (the reference divides x-differences by dy and y-differences by dx,
 *                  numpy_backend.py:47-48; the same pairing is kept)
 *   qy            dy/dx: weight of the y-difference in the E curl relative to the x one
 *   inv_kd2       2*eps0*dy/dt: converts (loss * ce) into the E loss factor
 * -------------------------------------------------------------------------- */
typedef struct bz_grid2d {
  int32_t nx, ny, pitch;
  int32_t n_designs, n_comp, n_mat;
  int32_t dtype;
  int32_t tile_rows;        /* rows per thread block: 4, 8, 16 or 32 (0 = 16) */
  double chx, chy, qy, inv_kd2;
} bz_grid2d;

/* Field and coefficient buffers of one 2D problem. ez/hx/hy hold two ping-pong
 * copies each; a launch with host-side step argument n reads copy (n & 1) and
 * writes copy (n & 1) ^ 1.
 * ce   = dt/(eps0*dy*(eps_r + a))   (E update source factor, x-difference units)
 * loss = a = sigma*dt/(2*eps0)      (dimensionless conductivity term)
 * power (optional, float64 [n_designs][ny][pitch]) accumulates |S|^2 per cell as
 * helper.py:153-187 does. */
typedef struct bz_fields2d {
  void* ez[2];
  void* hx[2];
  void* hy[2];
  const void* ce;
  const void* loss;
  double* power;
} bz_fields2d;

/* Source injection after the E update (helper.py:5-118), as a list of cell
 * operations applied in list order: v = mul*v + sum_c weight*signal[sig][step].
 * cell is the linear index y*nx + x (3D: (z*ny + y)*nx + x), sorted ascending with
 * operations on the same cell kept in application order. */
typedef struct bz_source_ops {
  int32_t n_ops;
  int32_t n_steps;          /* length of each signal row; later steps inject nothing */
  const int32_t* row_ptr;   /* [rows+1]: ops of grid row r (2D: y, 3D: z*ny+y) are [row_ptr[r], row_ptr[r+1]) */
  const int32_t* cell;      /* [n_ops] */
  const void* mul;          /* [n_ops] dtype: 1 keeps the old value, 0 zeroes it */
  const void* weight;       /* [n_ops][n_comp] dtype */
  const int32_t* sig;       /* [n_ops] signal row */
  const void* signals;      /* [n_signals][n_steps] dtype */
  int64_t weight_stride;    /* elements between designs' weight tables; 0: one table for all designs */
} bz_source_ops;

/* Monitor sampling after injection (monitors.py:279-315). Each point samples,
 * at its cell: Ez, Hx, Hy (the reference's record_fields_2d triple) and, for the
 * frequency-domain monitors, the two staggered neighbours used to centre H on
 * the E node.
 * record (optional): [n_rec][n_designs][n_comp][n_points][3] dtype, row
 *   (step - rec_step0) for rec_step0 <= step < rec_step0 + n_rec.
 * ring (optional): [ring_len][n_designs][n_comp][n_points][5] dtype, slot
 *   step % ring_len, holding (Ez, Hx(x), Hx(x-1), Hy(y), Hy(y-1)); folded into
 *   float64 DFT sums by bz_dft_fold at least every ring_len steps. */
typedef struct bz_monitor_ops {
  int32_t n_points;
  int32_t ring_len;
  const int32_t* row_ptr;   /* [rows+1] as in bz_source_ops */
  const int32_t* cell;      /* [n_points] sorted ascending */
  const int32_t* point;     /* [n_points] output slot of each sorted entry */
  void* record;
  int64_t rec_step0;
  int32_t n_rec;
  int32_t reserved;
  void* ring;
  /* optional capture of Ez inside a box (design region), for adjoint gradients:
   * region[k][d][c][rh][rw] = Ez after step (reg_step0 + k - 1) for 1 <= k < n_reg
   * (slot 0 is left to the caller, which stores the state at reg_step0); the box must
   * not contain source cells */
  void* region;
  int32_t rx0, ry0, rw, rh;
  int64_t reg_step0;
  int32_t n_reg;
  int32_t reserved2;
} bz_monitor_ops;

/* One full time step of the 2D Ez-mode Yee scheme for every design and component:
 * H update (all H cells), E update (interior, PEC ring), source injection,
 * optional |S|^2 accumulation, monitor record + DFT.
 * step: time-step index n; it also selects the ping-pong copy read (n & 1). If
 * d_step is non-NULL the time index used for signals, records and DFT phasors is
 * *d_step + step (CUDA-graph replay with a device-side step counter) while the
 * copy read stays (step & 1). */
int bz_step2d(const bz_grid2d* g, const bz_fields2d* f, const bz_source_ops* src,
              const bz_monitor_ops* mon, int64_t step, const int64_t* d_step, void* stream);

/* n_sub consecutive steps of bz_step2d in one launch (temporal blocking; replaces
 * n_sub iterations of the reference's step loop, fdtd.py:188-198 + helper.py). Same
 * results as n_sub bz_step2d calls from `step` (same arithmetic per cell; sources,
 * monitor records and ring samples per sub-step). Each block keeps a tile of the
 * grid in registers for all sub-steps and stores the part of it that stays exact.
 * n_sub: 1, 3, 5, 7 or 9 (odd, so the copy read stays (step & 1) and the result lands
 * in copy ((step + n_sub) & 1)); 1 is bz_step2d. tile: 0 = default (4x16), 1..5 =
 * tile shapes of 4x8, 4x16, 8x8, 5x16 and 6x12 (rows per warp x warps) for float32
 * single-component fields. Region capture (mon->region) is taken per sub-step; power
 * accumulation returns BZ_ERR_UNSUPPORTED (use bz_step2d for those steps). */
int bz_step2d_multi(const bz_grid2d* g, const bz_fields2d* f, const bz_source_ops* src,
                    const bz_monitor_ops* mon, int64_t step, int32_t n_sub, int32_t tile,
                    const int64_t* d_step, void* stream);

/* Folds `count` consecutive ring samples, steps step0 .. step0+count-1 (ring slot
 * step % ring_len, count <= ring_len), into float64 DFT sums:
 *   dft[i][f][q] += sum_s ring[s % ring_len][i][q] * phasor[s][f][E or H]
 * for i < n_items (= designs*components*points), q < 5 (q = 0 uses the E phasor,
 * q >= 1 the H phasor). phasor[s][f] = (cos wt_E, -sin wt_E, cos wt_H, -sin wt_H)
 * with t_E = (s+1) dt and t_H = (s+1/2) dt; dft is [n_items][n_freq][5][2]. Steps at
 * or beyond n_phasor contribute nothing. One warp per (item, frequency) reduces
 * over the steps with shuffles. */
int bz_dft_fold(const void* ring, int32_t dtype, int32_t ring_len, int64_t n_items, int32_t n_freq,
                const double* phasor, int64_t n_phasor, int64_t step0, int32_t count, double* dft, void* stream);

/* Allocation-free variant of bz_step2d + bz_dft_fold for callers that cannot call
 * cudaMalloc (for example a binding whose runtime owns all device memory through its
 * own pool, or a host with a fixed device-memory budget). No counterpart in the
 * reference: it has no frequency-domain monitors and no device memory management.
 * Runs n_steps steps from step0 (direct launches) and folds the monitors' samples into
 * dft ([n_designs*n_comp*n_points][n_freq][5][2], float64) exactly as bz_dft_fold does,
 * keeping the sample ring in an 8 MiB array compiled into the library instead of
 * mon->ring, which must be NULL. One step of samples (n_designs*n_comp*n_points*5
 * elements of dtype) must fit in 8 MiB; larger requests return BZ_ERR_INVALID. Calls
 * outside a stream capture look up the array's address on the current device; make the
 * first call on each device before any stream capture. All calls share the array;
 * calls that overlap on the GPU race. */
int bz_step2d_dft_static(const bz_grid2d* g, const bz_fields2d* f, const bz_source_ops* src,
                         const bz_monitor_ops* mon, int64_t step0, int32_t n_steps, int32_t n_freq,
                         const double* phasor, int64_t n_phasor, double* dft, void* stream);

/* Exact discrete adjoint of one 2D step (reverse-mode derivative of bz_step2d), for
 * topology-optimisation gradients. No counterpart in the reference, whose adjoint
 * (examples/4_topo.py:333-341) is a field-overlap heuristic; this one is the
 * transpose of the update, so gradients match finite differences.
 * State (n_comp = 1): e = dJ/dE (after the source zeroing), hx, hy = dJ/dH carried
 * from later steps; two copies each, the launch reads copy (phase & 1) and writes
 * the other. Step `step` = n maps the adjoint of E after step n to that of E_n.
 * Gradient (optional): grad[d][rh][rw] += -e * (E_{n+1} - E_n) / eps_r over the box
 * (rx0, ry0, rw, rh), reading forward captures fwd_region[k][d][rh][rw] = E at step
 * fwd_step0 + k (k < n_fwd) and eps_region[n_mat][rh][rw] (float64); the box must be
 * free of conductivity and sources. ops (optional): per-cell operations
 * v = mul*v + weight*signal[step-1] applied to the output to prepare step n-1 (the
 * source zeroing mask and the objective's dJ/dE_n, weights pre-multiplied by mul). */
typedef struct bz_adjoint2d {
  void* e[2];
  void* hx[2];
  void* hy[2];
  const void* ce;
  const void* loss;
  double* grad;
  const double* eps_region;
  const void* fwd_region;
  int32_t rx0, ry0, rw, rh;
  int64_t fwd_step0;
  int32_t n_fwd;
  int32_t reserved;
} bz_adjoint2d;

int bz_adjoint_step2d(const bz_grid2d* g, const bz_adjoint2d* s, const bz_source_ops* ops, int64_t step,
                      int32_t phase, void* stream);

/* n_sub reverse steps of bz_adjoint_step2d in one launch (step, step-1, ...,
 * step-n_sub+1; temporal blocking with the register tile of bz_step2d_multi): the same
 * gradient and operations per reverse step. n_sub: 1, 3, 5, 7 or 9 (odd, so the copy read
 * is (phase & 1) and the result lands in the other copy, as n_sub single calls with
 * alternating phase leave it); step + 1 >= n_sub. */
int bz_adjoint_step2d_multi(const bz_grid2d* g, const bz_adjoint2d* s, const bz_source_ops* ops, int64_t step,
                            int32_t n_sub, int32_t phase, void* stream);

/* Adds n to the device step counter (*d_step += n). */
int bz_advance_step(int64_t* d_step, int64_t n, void* stream);

/* Coefficients from the rasterised material: float64 eps_r and sigma, dense
 * [rows][nx] (rows = n*ny in 2D, n*nz*ny in 3D), into padded ce/loss arrays of
 * dtype laid out [rows][pitch]; padding columns are written as 0.
 *   ce   = dt/(eps0*dy*(eps_r + a)),  loss = a = sigma*dt/(2*eps0)
 * This is the coefficient arithmetic of numpy_backend.py:52-60,80-84 and
 * fdtd.py:232-305, evaluated once in float64 and rounded once to dtype. */
int bz_prepare_coeffs(const double* eps_r, const double* sigma, int64_t rows, int32_t nx,
                      int32_t pitch, int32_t dtype, double dt, double eps0, double dy,
                      void* ce, void* loss, void* stream);

/* Unfused half-step updates on arrays with the reference's shapes, for callers
 * of the Backend interface (update_h_fields / update_e_field,
 * beamz/simulation/backends/numpy_backend.py:34-88). Dense row-major arrays:
 * Ez (ny, nx), Hx (ny, nx-1), Hy (ny-1, nx), sigma and eps_r (ny, nx), all of
 * dtype; nc = 1 for real fields, 2 for interleaved (re, im) complex fields.
 * H is updated everywhere, Ez in the interior only; both in place. */
int bz_update_h2d(int32_t dtype, int32_t ny, int32_t nx, int32_t nc, void* hx, void* hy, const void* ez,
                  const void* sigma, double dx, double dy, double dt, double mu0, double eps0, void* stream);
int bz_update_e2d(int32_t dtype, int32_t ny, int32_t nx, int32_t nc, void* ez, const void* hx, const void* hy,
                  const void* sigma, const void* eps_r, double dx, double dy, double dt, double eps0, void* stream);

/* ----------------------------------------------------------------------------
 * 3D Yee scheme (beamz/simulation/fdtd.py:200-310). Every component is stored as
 * [n_designs][n_comp][nz][ny][pitch] (x contiguous); positions outside a
 * component's reference shape (Ex (nz, ny, nx-1), Ey (nz, ny-1, nx),
 * Ez (nz-1, ny, nx), Hx (nz-1, ny-1, nx), Hy (nz-1, ny, nx-1), Hz (nz, ny-1, nx-1))
 * stay zero.
 *   chx, chy, chz  dt/(mu0*dx), dt/(mu0*dy), dt/(mu0*dz)
 *   qx, qz         dy/dx, dy/dz (E curl weights relative to the y-difference)
 *   inv_kd2        2*eps0*dy/dt (ce and loss as in bz_prepare_coeffs with dy)
 * -------------------------------------------------------------------------- */
typedef struct bz_grid3d {
  int32_t nx, ny, nz, pitch;
  int32_t n_designs, n_comp, n_mat, dtype;
  int32_t tile_z;           /* z planes per thread block: 8 or 16 (0 = 16) */
  int32_t tile_y;           /* rows per thread block (32 x tile_y threads): 8 or 16 (0 = 8) */
  int32_t x_cells;          /* x cells per thread for float32 fields: 4, 2 or 1 (0 = 4);
                               float64 fields always take 1 */
  double chx, chy, chz, qx, qz, inv_kd2;
} bz_grid3d;

typedef struct bz_fields3d {
  void* e[2][3];            /* [copy][Ex, Ey, Ez] */
  void* h[2][3];            /* [copy][Hx, Hy, Hz] */
  const void* ce;           /* [n_mat][nz][ny][pitch] */
  const void* loss;
} bz_fields3d;

/* One 3D time step (H then E, E on the reference's interior slices) for every
 * design and component; the launch reads copy (step & 1) and writes the other. */
int bz_step3d(const bz_grid3d* g, const bz_fields3d* f, int64_t step, void* stream);

/* Applies source operations (bz_source_ops, cell = (z*ny + y)*nx + x or y*nx + x)
 * in place to one field array laid out [n_designs][n_comp][rows][pitch] with
 * rows of nx cells, as helper.py:5-118 injects after the E update. The time index
 * is step, or *d_step + step when d_step is non-NULL. */
int bz_cell_ops(void* field, int32_t dtype, int32_t n_designs, int32_t n_comp, int64_t comp_stride,
                int32_t nx, int32_t pitch, const bz_source_ops* ops, int64_t step, const int64_t* d_step,
                void* stream);

/* Gathers monitor samples: n_q quantities (<= 6) per point from arrays laid out
 * [n_designs][n_comp][...] (element strides comp_stride between components),
 * offset[p][q] into each quantity's array (-1: the sample is 0). Writes
 * record[step - rec_step0][d][c][p][q] when in range and ring[step % ring_len][d][c][p][q]
 * (either may be NULL). Reference: helper.py:235-244 -> monitors.py:317-396. */
typedef struct bz_gather_ops {
  int32_t n_points, n_q;
  const void* src[6];
  const int64_t* offset;
  void* record;
  int64_t rec_step0;
  int32_t n_rec;
  int32_t ring_len;
  void* ring;
} bz_gather_ops;
int bz_gather(const bz_gather_ops* ops, int32_t dtype, int32_t n_designs, int32_t n_comp, int64_t comp_stride,
              int64_t step, const int64_t* d_step, void* stream);

/* Adds, per cell of the common region (nz-1, ny-1, nx-1), |Re(E x conj(H))| of
 * fields copy `cur` to power[n_designs][nz-1][ny-1][nx-1] (float64), as
 * helper.py:124-151 accumulates it. */
int bz_power3d(const bz_grid3d* g, const bz_fields3d* f, int32_t cur, double* power, void* stream);

/* bz_dft_fold with n_q quantities per item (<= 6), the first n_e on the E phasor and
 * the rest on the H phasor; ring [ring_len][n_items][n_q], dft [n_items][n_freq][n_q][2]. */
int bz_dft_fold_q(const void* ring, int32_t dtype, int32_t ring_len, int64_t n_items, int32_t n_q, int32_t n_e,
                  int32_t n_freq, const double* phasor, int64_t n_phasor, int64_t step0, int32_t count, double* dft,
                  void* stream);

/* Divergence guard (the reference only warns about the Courant number before a run,
 * fdtd.py:375-383, helpers.py:21-53; this checks the fields while they run): scans n
 * values of a field array and, when one is not finite or exceeds `limit` in magnitude,
 * stores BZ_ERR_DIVERGED in status[0] and `step` in status[1] (device int64 words,
 * zeroed by the caller; an earlier detection is kept). Asynchronous: the caller reads
 * the words when it synchronizes and reports BZ_ERR_DIVERGED. */
int bz_field_check(const void* field, int32_t dtype, int64_t n, double limit, int64_t step, int64_t* status,
                   void* stream);

/* ----------------------------------------------------------------------------
 * Rasteriser (meshing.py:92-536): painter's-order supersampled blend of each
 * structure's material, then the additive PML conductivity pass.
 * ------------------------------------------------------------------------- */
#define BZ_SHAPE_RECT 0      /* axis-aligned rectangle fast path, meshing.py:193-257 */
#define BZ_SHAPE_CIRCLE 1    /* circle fast path, meshing.py:259-307 */
#define BZ_SHAPE_RING 2      /* ring fast path, meshing.py:309-361 */
#define BZ_SHAPE_POLYGON 3   /* general polygon path, meshing.py:362-477 */

typedef struct bz_shape2d {
  int32_t kind;
  int32_t i0, i1, j0, j1;        /* cell loop box [i0,i1) x [j0,j1) (rect: the rect box) */
  int32_t fill;                  /* rect: interior fill applies */
  int32_t fi0, fi1, fj0, fj1;    /* rect: interior fill box */
  int32_t top, bottom, left, right; /* rect: boundary strips, rel row < top or >= bottom, rel col < left or >= right */
  int32_t path0, npath;          /* polygon: rows of the path table (exterior first, then holes) */
  int32_t custom_off;            /* rect with CustomMaterial: offset (in triples) into the custom table, else -1 */
  int32_t reserved;
  double p0, p1, p2, p3;         /* rect: x0, x0+w, y0, y0+h; circle: cx, cy, r; ring: cx, cy, rin, rout */
  double q;                      /* circle/ring: 0.3536 * cell_size */
  double perm, permb, cond;      /* material */
} bz_shape2d;

/* PML boundary (beamz/design/pml.py:29-62) over its loop box. table holds, for
 * every cell of the box in row-major order, (profile, frequency_factor) or a
 * negative profile where get_conductivity returns 0 — the position-only part,
 * tabulated by the host. The kernel adds
 *   ((1.2/(sqrt(mu0/(eps0*eps))*dx))*sigma_factor*profile)*frequency_factor
 * when it is > 0. */
typedef struct bz_pml2d {
  int32_t i0, i1, j0, j1;
  int64_t table_off;             /* offset (in pairs) into the pml table */
  double sigma_factor;
} bz_pml2d;

/* eps/mu/sigma: float64 [ny][nx] outputs (fully written). xc[nx], yc[ny]: cell-centre
 * coordinates (float64, the reference's np.linspace values). offs[3]: the
 * supersample offsets (-0.25, 0, 0.25)*cell_size; corner[2]: (-0.4, 0.4)*cell_size.
 * bg: background material triple. shapes, pmls: arrays of the structs above in
 * device memory. paths: [npaths_total][2] (vertex start, count); verts: [nverts][2]
 * float64. custom: [n][3] float64. pml_table: [n][2] float64. All pointers are
 * device pointers. */
int bz_rasterize2d(int32_t nx, int32_t ny, const double* xc, const double* yc,
                   const double* offs, const double* corner, const double* bg,
                   const bz_shape2d* shapes, int32_t n_shapes,
                   const int32_t* paths, const double* verts, const double* custom,
                   const bz_pml2d* pmls, int32_t n_pml, const double* pml_table,
                   double dx, double eps0, double mu0,
                   double* eps, double* mu, double* sigma, void* stream);

/* 3D rasteriser (meshing.py:616-781): for every cell (k, i, j) and every structure
 * in painter's order whose layer range [k0, k1) holds k, count the cell's 9 xy
 * samples inside the structure's polygon, weight by zw[k - k0] of the n_zs z samples
 * (the reference ignores z, so zw = n_zs on its layers; the extrusion mode counts
 * the z samples inside the structure's thickness), and blend with factor
 * count*zw / (9*n_zs). Then add the PML: the 2D boundary tables of bz_rasterize2d
 * applied to every layer with that cell's eps, plus an optional per-layer z-face
 * term prof_z[k] = (profile, frequency factor) (profile < 0: none) with
 * sigma_factor_z. Outputs [nz][ny][nx] float64. */
typedef struct bz_shape3d {
  int32_t i0, i1, j0, j1, k0, k1;
  int32_t path0, npath;
  int32_t zw_off;                /* offset into zw (one entry per layer of [k0, k1)) */
  int32_t reserved;
  double perm, permb, cond;
} bz_shape3d;

int bz_rasterize3d(int32_t nx, int32_t ny, int32_t nz, int32_t n_zs, const double* xc, const double* yc,
                   const double* offs, const double* bg, const bz_shape3d* shapes, int32_t n_shapes,
                   const int32_t* zw, const int32_t* paths, const double* verts, const bz_pml2d* pmls,
                   int32_t n_pml, const double* pml_table, const double* prof_z, double sigma_factor_z, double dx,
                   double eps0, double mu0, double* eps, double* mu, double* sigma, void* stream);

/* ---- learned surrogate kernels ------------------------------------------------
 * No counterpart in the reference (it has no learned surrogate). A Fourier neural
 * operator maps a design density to transmissions; its layers are built from these
 * kernels: bf16 operands and activations, f32 accumulation. */

/* C[b] = epilogue(alpha * op(A[b]) @ op(B[b])) for b < batch, M x N x K:
 * op(A)[m][k] = A[m*lda + k] (ta = 0) or A[k*lda + m] (ta = 1); op(B)[k][n] =
 * B[k*ldb + n] (tb = 0) or B[n*ldb + k] (tb = 1); sa/sb/sc/sadd/spre are batch
 * strides in elements (0 shares an operand across the batch). Epilogue, in order:
 * + cadd[b][m][n] (f32, or bf16 as cadd_h; optional), + bias_m[m], + bias_n[n] (f32, optional), a copy
 * to pre (bf16, optional), act (0 none, 1 GELU tanh form), then store to outf (f32)
 * and/or outh (bf16). atomic = 1 adds alpha*product into outf (f32 only, no other
 * epilogue term), which with sc = 0 reduces over the batch; splitk > 1 splits K
 * across blocks and needs atomic. */
typedef struct bz_gemm {
  int32_t M, N, K, batch, splitk, act;
  int32_t ta, tb, atomic;
  int32_t engine;               /* 0: tcgen05/TMEM kernels where eligible, else mma.sync:
                                   the GEMM kernel for ta = 0, tb = 1, M >= 128, N >= 256,
                                   K >= 64, 16-byte aligned rows (TMA-fed when batch = 1); the
                                   channel-mixing kernel for tb = 0, K and M in {32, 64},
                                   N >= 64, sb = K * ldb, no atomic / split-K; the
                                   weight-gradient kernel for ta = 0, tb = 1, atomic, sc = 0,
                                   M <= 128, N in {32, 64}, sa = M * lda, sb = N * ldb;
                                   1: mma.sync only;
                                   2: the register-staged tcgen05 kernel where eligible */
  const void* A;
  int64_t lda, sa;
  const void* B;
  int64_t ldb, sb;
  float alpha, reserved2;
  const float* cadd;
  int64_t ldadd, sadd;
  const float* bias_m;
  const float* bias_n;
  float* outf;
  void* outh;
  int64_t ldc, sc;
  void* pre;
  int64_t ldpre, spre;
  const void* cadd_h;           /* the added term as bf16 instead of cadd (same ldadd/sadd) */
} bz_gemm;

int bz_gemm_bf16(const bz_gemm* g, void* stream);

/* Error word of the tcgen05 GEMM (non-zero: a pipeline wait ran out; that CTA left
 * its tile unwritten). Synchronous read; reset = 1 clears it. */
int bz_gemm_error(int32_t* value, int32_t reset);

/* Drives the tcgen05 GEMM's bounded-wait error path on one 128 x 256 x 64 tile (no
 * counterpart in the reference, which has no device code: this checks that a wait that
 * never completes ends the kernel cleanly). The control thread issues no MMA for the
 * tile's only K slice, so the wait for that slice's commit gives up after wait_limit
 * polls; the kernel skips its epilogue, frees its tensor memory and raises the error
 * word, which this call reads and clears. A: 128 x 64 bf16, B: 256 x 64 bf16 (row
 * major, K contiguous), C: 128 x 256 f32 (not written). Synchronizes the stream.
 * Returns BZ_ERR_TIMEOUT when the wait ran out, BZ_OK if the word stayed clear. */
int bz_gemm_wait_selftest(const void* A, const void* B, float* C, int32_t wait_limit, void* stream);

/* Spectral channel mixing of one Fourier layer, per mode k < n_modes:
 * O[b][o][k] = sum_c U[b][c][k] * W[k][c][o] (complex, (re, im) pairs, bf16);
 * ci, co <= 32. */
int bz_spectral_mix(const void* U, const void* W, void* O, int32_t B, int32_t ci, int32_t co, int32_t n_modes,
                    void* stream);
/* Its backward: dU = sum_o dO * conj(W); dW (f32, accumulated) += sum_b dO * conj(U). */
int bz_spectral_mix_bwd(const void* dO, const void* U, const void* W, void* dU, float* dW, int32_t B, int32_t ci,
                        int32_t co, int32_t n_modes, void* stream);
/* dx = dy * GELU'(pre) (bf16). */
int bz_gelu_bwd(const void* dy, const void* pre, void* dx, int64_t n, void* stream);
/* out[r] = scale * sum_p x[r][p] (bf16 rows of length P, f32 out). */
int bz_row_mean(const void* x, float* out, int64_t rows, int32_t P, float scale, void* stream);
/* x[r][p] = scale * g[r] (bf16 out). */
int bz_row_broadcast(const float* g, void* x, int64_t rows, int32_t P, float scale, void* stream);
/* out[c] += sum_b sum_p x[b][c][p] (bf16 [B][C][P], f32 out). */
int bz_chan_sum(const void* x, float* out, int32_t B, int32_t C, int32_t P, void* stream);
/* One Adam step (bias-corrected, decoupled weight decay folded into the gradient) on
 * f32 master weights w with moments m, v; refreshes the bf16 copy wh when non-NULL. */
int bz_adam(float* w, const float* g, float* m, float* v, void* wh, int64_t n, float lr, float b1, float b2,
            float eps, int32_t step, float weight_decay, void* stream);
/* y = bf16(x). */
int bz_to_bf16(const float* x, void* y, int64_t n, void* stream);

#ifdef __cplusplus
}
#endif

#endif /* BEAMZ_B200_H */
