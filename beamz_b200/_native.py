"""ctypes binding of libbeamz_b200.so (declarations: include/beamz_b200.h).

The shared library is the only compute path: importing this module fails with
an ImportError naming the missing file when the library has not been built, and
every entry raises ``RuntimeError`` with the library's message on a non-zero
status. There is no fallback implementation.
"""
from __future__ import annotations

import ctypes as C
import os
from pathlib import Path

_LIB_PATH = Path(os.environ.get("BEAMZ_B200_LIB", Path(__file__).resolve().parent / "libbeamz_b200.so"))

if not _LIB_PATH.exists():
    raise ImportError(
        f"libbeamz_b200.so not found at {_LIB_PATH}; build it with `python -m beamz_b200._build` "
        "(needs nvcc for sm_100a)"
    )

try:
    lib = C.CDLL(str(_LIB_PATH))
except OSError as exc:  # e.g. libcudart missing on a machine without CUDA
    raise ImportError(f"cannot load {_LIB_PATH}: {exc}") from exc

BZ_OK = 0
BZ_ERR_INVALID = -1
BZ_ERR_CUDA = -2
BZ_ERR_DIVERGED = -3
BZ_ERR_TIMEOUT = -4
BZ_ERR_UNSUPPORTED = -5
BZ_F32 = 0
BZ_F64 = 1
BZ_SHAPE_RECT, BZ_SHAPE_CIRCLE, BZ_SHAPE_RING, BZ_SHAPE_POLYGON = 0, 1, 2, 3

i32, i64, f64, vp = C.c_int32, C.c_int64, C.c_double, C.c_void_p


class Grid2D(C.Structure):
    _fields_ = [("nx", i32), ("ny", i32), ("pitch", i32), ("n_designs", i32), ("n_comp", i32), ("n_mat", i32),
                ("dtype", i32), ("tile_rows", i32), ("chx", f64), ("chy", f64), ("qy", f64), ("inv_kd2", f64)]


class Fields2D(C.Structure):
    _fields_ = [("ez", vp * 2), ("hx", vp * 2), ("hy", vp * 2), ("ce", vp), ("loss", vp), ("power", vp)]


class SourceOps(C.Structure):
    _fields_ = [("n_ops", i32), ("n_steps", i32), ("row_ptr", vp), ("cell", vp), ("mul", vp), ("weight", vp),
                ("sig", vp), ("signals", vp), ("weight_stride", i64)]


class MonitorOps(C.Structure):
    _fields_ = [("n_points", i32), ("ring_len", i32), ("row_ptr", vp), ("cell", vp), ("point", vp), ("record", vp),
                ("rec_step0", i64), ("n_rec", i32), ("reserved", i32), ("ring", vp), ("region", vp), ("rx0", i32),
                ("ry0", i32), ("rw", i32), ("rh", i32), ("reg_step0", i64), ("n_reg", i32), ("reserved2", i32)]


class Adjoint2D(C.Structure):
    _fields_ = [("e", vp * 2), ("hx", vp * 2), ("hy", vp * 2), ("ce", vp), ("loss", vp), ("grad", vp),
                ("eps_region", vp), ("fwd_region", vp), ("rx0", i32), ("ry0", i32), ("rw", i32), ("rh", i32),
                ("fwd_step0", i64), ("n_fwd", i32), ("reserved", i32)]


class Gemm(C.Structure):
    _fields_ = [("M", i32), ("N", i32), ("K", i32), ("batch", i32), ("splitk", i32), ("act", i32), ("ta", i32),
                ("tb", i32), ("atomic", i32), ("engine", i32), ("A", vp), ("lda", i64), ("sa", i64), ("B", vp),
                ("ldb", i64), ("sb", i64), ("alpha", C.c_float), ("reserved2", C.c_float), ("cadd", vp),
                ("ldadd", i64), ("sadd", i64), ("bias_m", vp), ("bias_n", vp), ("outf", vp), ("outh", vp),
                ("ldc", i64), ("sc", i64), ("pre", vp), ("ldpre", i64), ("spre", i64), ("cadd_h", vp)]


class Grid3D(C.Structure):
    _fields_ = [("nx", i32), ("ny", i32), ("nz", i32), ("pitch", i32), ("n_designs", i32), ("n_comp", i32),
                ("n_mat", i32), ("dtype", i32), ("tile_z", i32), ("tile_y", i32), ("x_cells", i32),
                ("chx", f64), ("chy", f64), ("chz", f64), ("qx", f64), ("qz", f64), ("inv_kd2", f64)]


class Fields3D(C.Structure):
    _fields_ = [("e", (vp * 3) * 2), ("h", (vp * 3) * 2), ("ce", vp), ("loss", vp)]


class GatherOps(C.Structure):
    _fields_ = [("n_points", i32), ("n_q", i32), ("src", vp * 6), ("offset", vp), ("record", vp), ("rec_step0", i64),
                ("n_rec", i32), ("ring_len", i32), ("ring", vp)]


class Shape2D(C.Structure):
    _fields_ = [("kind", i32), ("i0", i32), ("i1", i32), ("j0", i32), ("j1", i32), ("fill", i32), ("fi0", i32),
                ("fi1", i32), ("fj0", i32), ("fj1", i32), ("top", i32), ("bottom", i32), ("left", i32),
                ("right", i32), ("path0", i32), ("npath", i32), ("custom_off", i32), ("reserved", i32),
                ("p0", f64), ("p1", f64), ("p2", f64), ("p3", f64), ("q", f64), ("perm", f64), ("permb", f64),
                ("cond", f64)]


class Shape3D(C.Structure):
    _fields_ = [("i0", i32), ("i1", i32), ("j0", i32), ("j1", i32), ("k0", i32), ("k1", i32), ("path0", i32),
                ("npath", i32), ("zw_off", i32), ("reserved", i32), ("perm", f64), ("permb", f64), ("cond", f64)]


class Pml2D(C.Structure):
    _fields_ = [("i0", i32), ("i1", i32), ("j0", i32), ("j1", i32), ("table_off", i64), ("sigma_factor", f64)]


def _sig(name, restype, argtypes):
    fn = getattr(lib, name)
    fn.restype = restype
    fn.argtypes = argtypes
    return fn


_version = _sig("bz_version", C.c_char_p, [])
_last_error = _sig("bz_last_error", C.c_int, [C.c_char_p, C.c_size_t])
_step2d = _sig("bz_step2d", C.c_int, [C.POINTER(Grid2D), C.POINTER(Fields2D), C.POINTER(SourceOps),
                                       C.POINTER(MonitorOps), i64, vp, vp])
_step2d_multi = _sig("bz_step2d_multi", C.c_int, [C.POINTER(Grid2D), C.POINTER(Fields2D), C.POINTER(SourceOps),
                                                   C.POINTER(MonitorOps), i64, i32, i32, vp, vp])
_dft_fold = _sig("bz_dft_fold", C.c_int, [vp, i32, i32, i64, i32, vp, i64, i64, i32, vp, vp])
_step2d_dft_static = _sig("bz_step2d_dft_static", C.c_int,
                          [C.POINTER(Grid2D), C.POINTER(Fields2D), C.POINTER(SourceOps), C.POINTER(MonitorOps), i64,
                           i32, i32, vp, i64, vp, vp])
_step3d = _sig("bz_step3d", C.c_int, [C.POINTER(Grid3D), C.POINTER(Fields3D), i64, vp])
_cell_ops = _sig("bz_cell_ops", C.c_int, [vp, i32, i32, i32, i64, i32, i32, C.POINTER(SourceOps), i64, vp, vp])
_gather = _sig("bz_gather", C.c_int, [C.POINTER(GatherOps), i32, i32, i32, i64, i64, vp, vp])
_power3d = _sig("bz_power3d", C.c_int, [C.POINTER(Grid3D), C.POINTER(Fields3D), i32, vp, vp])
_dft_fold_q = _sig("bz_dft_fold_q", C.c_int, [vp, i32, i32, i64, i32, i32, i32, vp, i64, i64, i32, vp, vp])
_raster3d = _sig("bz_rasterize3d", C.c_int, [i32, i32, i32, i32, vp, vp, vp, vp, vp, i32, vp, vp, vp, vp, i32, vp,
                                              vp, f64, f64, f64, f64, vp, vp, vp, vp])
_adjoint2d = _sig("bz_adjoint_step2d", C.c_int, [C.POINTER(Grid2D), C.POINTER(Adjoint2D), C.POINTER(SourceOps), i64,
                                                  i32, vp])
_adjoint2d_multi = _sig("bz_adjoint_step2d_multi", C.c_int, [C.POINTER(Grid2D), C.POINTER(Adjoint2D),
                                                              C.POINTER(SourceOps), i64, i32, i32, vp])
_advance = _sig("bz_advance_step", C.c_int, [vp, i64, vp])
_prepare = _sig("bz_prepare_coeffs", C.c_int, [vp, vp, i64, i32, i32, i32, f64, f64, f64, vp, vp, vp])
_upd_h2d = _sig("bz_update_h2d", C.c_int, [i32, i32, i32, i32, vp, vp, vp, vp, f64, f64, f64, f64, f64, vp])
_upd_e2d = _sig("bz_update_e2d", C.c_int, [i32, i32, i32, i32, vp, vp, vp, vp, vp, f64, f64, f64, f64, vp])
_raster2d = _sig("bz_rasterize2d", C.c_int, [i32, i32, vp, vp, vp, vp, vp, vp, i32, vp, vp, vp, vp, i32, vp,
                                              f64, f64, f64, vp, vp, vp, vp])
_gemm = _sig("bz_gemm_bf16", C.c_int, [C.POINTER(Gemm), vp])
_spec = _sig("bz_spectral_mix", C.c_int, [vp, vp, vp, i32, i32, i32, i32, vp])
_spec_bwd = _sig("bz_spectral_mix_bwd", C.c_int, [vp, vp, vp, vp, vp, i32, i32, i32, i32, vp])
_gelu_bwd = _sig("bz_gelu_bwd", C.c_int, [vp, vp, vp, i64, vp])
_row_mean = _sig("bz_row_mean", C.c_int, [vp, vp, i64, i32, C.c_float, vp])
_row_bcast = _sig("bz_row_broadcast", C.c_int, [vp, vp, i64, i32, C.c_float, vp])
_chan_sum = _sig("bz_chan_sum", C.c_int, [vp, vp, i32, i32, i32, vp])
_adam = _sig("bz_adam", C.c_int, [vp, vp, vp, vp, vp, i64, C.c_float, C.c_float, C.c_float, C.c_float, i32,
                                  C.c_float, vp])
_to_bf16 = _sig("bz_to_bf16", C.c_int, [vp, vp, i64, vp])
_gemm_err = _sig("bz_gemm_error", C.c_int, [C.POINTER(i32), i32])
_gemm_selftest = _sig("bz_gemm_wait_selftest", C.c_int, [vp, vp, vp, i32, vp])
_field_check = _sig("bz_field_check", C.c_int, [vp, i32, i64, f64, i64, vp, vp])

#: every symbol include/beamz_b200.h declares (checked by the CPU test suite)
EXPORTED = ["bz_version", "bz_last_error", "bz_step2d", "bz_step2d_multi", "bz_dft_fold", "bz_step2d_dft_static", "bz_advance_step",
            "bz_adjoint_step2d", "bz_adjoint_step2d_multi", "bz_step3d", "bz_cell_ops", "bz_gather", "bz_power3d", "bz_dft_fold_q", "bz_rasterize3d", "bz_prepare_coeffs", "bz_update_h2d",
            "bz_update_e2d", "bz_rasterize2d", "bz_gemm_bf16", "bz_spectral_mix", "bz_spectral_mix_bwd", "bz_gelu_bwd",
            "bz_row_mean", "bz_row_broadcast", "bz_chan_sum", "bz_adam", "bz_to_bf16", "bz_gemm_error",
            "bz_gemm_wait_selftest", "bz_field_check"]


class NativeError(RuntimeError):
    def __init__(self, code: int, message: str):
        super().__init__(f"libbeamz_b200 error {code}: {message}")
        self.code = code


def last_error() -> tuple[int, str]:
    buf = C.create_string_buffer(512)
    code = _last_error(buf, len(buf))
    return code, buf.value.decode(errors="replace")


def check(status: int) -> None:
    if status != BZ_OK:
        code, msg = last_error()
        raise NativeError(status, msg or f"status {status}")


def version() -> str:
    return _version().decode()


def step2d(grid, fields, src, mon, step: int, d_step: int | None, stream: int) -> None:
    check(_step2d(C.byref(grid), C.byref(fields), C.byref(src) if src is not None else None,
                  C.byref(mon) if mon is not None else None, step, d_step, stream))


def step2d_multi(grid, fields, src, mon, step: int, n_sub: int, tile: int, d_step: int | None, stream: int) -> None:
    check(_step2d_multi(C.byref(grid), C.byref(fields), C.byref(src) if src is not None else None,
                        C.byref(mon) if mon is not None else None, step, n_sub, tile, d_step, stream))


def advance_step(d_step: int, n: int, stream: int) -> None:
    check(_advance(d_step, n, stream))


def prepare_coeffs(eps, sigma, rows, nx, pitch, dtype, dt, eps0, dy, ce, loss, stream) -> None:
    check(_prepare(eps, sigma, rows, nx, pitch, dtype, dt, eps0, dy, ce, loss, stream))


def rasterize2d(*args) -> None:
    check(_raster2d(*args))


def update_h2d(*args) -> None:
    check(_upd_h2d(*args))


def update_e2d(*args) -> None:
    check(_upd_e2d(*args))


def dft_fold(*args) -> None:
    check(_dft_fold(*args))


def step3d(grid, fields, step, stream) -> None:
    check(_step3d(C.byref(grid), C.byref(fields), step, stream))


def cell_ops(field, dtype, n_designs, n_comp, comp_stride, nx, pitch, ops, step, d_step, stream) -> None:
    check(_cell_ops(field, dtype, n_designs, n_comp, comp_stride, nx, pitch, C.byref(ops), step, d_step, stream))


def gather(ops, dtype, n_designs, n_comp, comp_stride, step, d_step, stream) -> None:
    check(_gather(C.byref(ops), dtype, n_designs, n_comp, comp_stride, step, d_step, stream))


def power3d(grid, fields, cur, power, stream) -> None:
    check(_power3d(C.byref(grid), C.byref(fields), cur, power, stream))


def dft_fold_q(*args) -> None:
    check(_dft_fold_q(*args))


def rasterize3d(*args) -> None:
    check(_raster3d(*args))


def adjoint_step2d(grid, state, ops, step, phase, stream) -> None:
    check(_adjoint2d(C.byref(grid), C.byref(state), C.byref(ops) if ops is not None else None, step, phase, stream))


def adjoint_step2d_multi(grid, state, ops, step: int, n_sub: int, phase: int, stream: int) -> None:
    check(_adjoint2d_multi(C.byref(grid), C.byref(state), C.byref(ops) if ops is not None else None, step, n_sub,
                           phase, stream))


# ---- surrogate kernels -------------------------------------------------------------
def gemm(g: Gemm, stream: int) -> None:
    check(_gemm(C.byref(g), stream))


def spectral_mix(U, W, O, B, ci, co, n_modes, stream) -> None:
    check(_spec(U, W, O, B, ci, co, n_modes, stream))


def spectral_mix_bwd(dO, U, W, dU, dW, B, ci, co, n_modes, stream) -> None:
    check(_spec_bwd(dO, U, W, dU, dW, B, ci, co, n_modes, stream))


def gelu_bwd(dy, pre, dx, n, stream) -> None:
    check(_gelu_bwd(dy, pre, dx, n, stream))


def row_mean(x, out, rows, P, scale, stream) -> None:
    check(_row_mean(x, out, rows, P, scale, stream))


def row_broadcast(g, x, rows, P, scale, stream) -> None:
    check(_row_bcast(g, x, rows, P, scale, stream))


def chan_sum(x, out, B, C_, P, stream) -> None:
    check(_chan_sum(x, out, B, C_, P, stream))


def adam(w, g, m, v, wh, n, lr, b1, b2, eps, step, wd, stream) -> None:
    check(_adam(w, g, m, v, wh, n, lr, b1, b2, eps, step, wd, stream))


def to_bf16(x, y, n, stream) -> None:
    check(_to_bf16(x, y, n, stream))


def field_check(ptr: int, dtype: int, n: int, limit: float, step: int, status_ptr: int, stream) -> None:
    check(_field_check(vp(ptr), dtype, n, float(limit), int(step), vp(status_ptr), vp(stream)))


def gemm_wait_selftest(a_ptr: int, b_ptr: int, c_ptr: int, wait_limit: int, stream) -> int:
    """Status of the tcgen05 GEMM's withheld-slice run (BZ_ERR_TIMEOUT expected); does not raise."""
    return _gemm_selftest(vp(a_ptr), vp(b_ptr), vp(c_ptr), int(wait_limit), vp(stream))


def gemm_error(reset: bool = True) -> int:
    """Error word of the tcgen05 GEMM (non-zero: a bounded pipeline wait ran out)."""
    v = i32(0)
    check(_gemm_err(C.byref(v), 1 if reset else 0))
    return v.value
