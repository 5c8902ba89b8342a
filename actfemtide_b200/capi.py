"""ctypes binding of libactfem_gpu.so (include/afem.h).

The library is built in-tree by ``actfemtide_b200.build`` (or
``__graft_entry__.build()``); this module never falls back to anything else:
if the shared object is missing, loading raises.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "_lib", "libactfem_gpu.so")

AFEM_OK = 0
STATUS = {
    0: "AFEM_OK", -1: "AFEM_EINVAL", -2: "AFEM_EVOLUME", -3: "AFEM_EPATTERN", -4: "AFEM_EMAXITER",
    -5: "AFEM_EBREAKDOWN", -6: "AFEM_ENONFINITE", -7: "AFEM_ECUDA", -8: "AFEM_ESTATE", -9: "AFEM_ETIMEOUT",
    -10: "AFEM_EIO", -11: "AFEM_ENOPRECOND", -12: "AFEM_ESITE", -13: "AFEM_ESTAGNATION",
}
STATUS_CODE = {v: k for k, v in STATUS.items()}
PRECOND = {"IC": 0, "SSOR": 1, "DIAG": 2, "NONE": 3, "LEARNED": 4, "SSOR_MC": 5, "HYBRID": 6}
PRECISION = {"fp64": 0, "mixed": 1, "pc32": 2}

# Every entry point declared in include/afem.h.
EXPORTS = (
    "afem_create", "afem_destroy", "afem_last_error", "afem_stream", "afem_set_mesh", "afem_get_lines",
    "afem_set_cond", "afem_set_sigma", "afem_set_source", "afem_set_bounds", "afem_assemble",
    "afem_export_system", "afem_solve", "afem_get_solution", "afem_sites", "afem_site_coeffs", "afem_load_ctl",
    "afem_ctl_info", "afem_run_ctl", "afem_fortran_g", "afem_set_profiling", "afem_profile_count",
    "afem_profile_entry", "afem_cocg13_single", "afem_set_system", "afem_get_residual", "afem_mpnn_nparam",
    "afem_mpnn_set_params", "afem_mpnn_get_params", "afem_mpnn_forward", "afem_mpnn_loss_grad", "afem_mpnn_train",
    "afem_solve_rhs", "afem_jacobian", "afem_sweep_schedule", "afem_coloring", "afem_set_segments",
    "afem_segment_info", "afem_launch_count", "afem_hybrid_matrix", "afem_sites_grid", "afem_site_coeffs_grid",
    "afem_xy_points", "afem_sort_index", "afem_mesh_info", "afem_solution_count", "afem_sites_noalloc",
    "afem_set_wait_limit", "afem_set_spmv_rows_per_warp", "afem_utm_xy",
    "afem_mpnn_set_base", "afem_precond_apply", "afem_mt_forward", "afem_mt_boundary", "afem_mt_face",
)


class SolveOpts(C.Structure):
    _fields_ = [("precond", C.c_int), ("precision", C.c_int), ("tol", C.c_double), ("maxit", C.c_int),
                ("sigma_diag", C.c_double), ("check_every", C.c_int), ("inner_tol", C.c_double),
                ("use_graph", C.c_int)]


class SolveStats(C.Structure):
    _fields_ = [("iterations", C.c_int), ("refinements", C.c_int), ("resid_recursive", C.c_double),
                ("resid_true", C.c_double), ("seconds", C.c_double), ("status", C.c_int)]


class MtCond(C.Structure):
    """afem_mt_cond: the MT forward's conductivity (GENMAT_MT / COND3DTO2D selections)."""
    _fields_ = [("sigma_air", C.c_double), ("condflag", C.c_int), ("nvolume", C.c_int), ("sigma_land", C.c_void_p),
                ("nphys2", C.c_int), ("sigma_file", C.c_void_p), ("tag_phys", C.c_void_p)]


class AfemError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__(f"{STATUS.get(code, code)}: {msg}")
        self.code = code


_LIB = None
_vp = C.c_void_p
_i32p = np.ctypeslib.ndpointer(dtype=np.int32, flags="C_CONTIGUOUS")
_f64p = np.ctypeslib.ndpointer(dtype=np.float64, flags="C_CONTIGUOUS")


def lib():
    """Load the in-tree library (raises OSError when it has not been built)."""
    global _LIB
    if _LIB is not None:
        return _LIB
    if not os.path.exists(LIB_PATH):
        raise OSError(f"{LIB_PATH} is missing: run `python -m actfemtide_b200.build`")
    L = C.CDLL(LIB_PATH)
    L.afem_create.restype = _vp
    L.afem_create.argtypes = [C.c_int]
    L.afem_destroy.argtypes = [_vp]
    L.afem_last_error.restype = C.c_char_p
    L.afem_last_error.argtypes = [_vp]
    L.afem_stream.restype = _vp
    L.afem_stream.argtypes = [_vp]
    L.afem_set_mesh.argtypes = [_vp, C.c_int, _vp, C.c_int, _vp, _vp, C.c_int, _vp, _vp]
    L.afem_get_lines.argtypes = [_vp, C.POINTER(C.c_int), _vp, _vp]
    L.afem_mpnn_set_base.argtypes = [_vp, C.c_int]
    L.afem_mpnn_set_base.restype = C.c_int
    L.afem_precond_apply.argtypes = [_vp, C.c_double, _vp, _vp]
    L.afem_precond_apply.restype = C.c_int
    L.afem_sites_noalloc.argtypes = [_vp, C.c_int, _vp, _vp]
    L.afem_sites_noalloc.restype = C.c_int
    L.afem_utm_xy.argtypes = [C.c_double, C.c_double, C.c_double, C.c_double, C.c_int, _vp]
    L.afem_utm_xy.restype = C.c_int
    L.afem_set_wait_limit.argtypes = [_vp, C.c_uint]
    L.afem_set_wait_limit.restype = C.c_int
    L.afem_set_spmv_rows_per_warp.argtypes = [_vp, C.c_int]
    L.afem_set_spmv_rows_per_warp.restype = C.c_int
    L.afem_sites_grid.argtypes = [_vp, C.c_int, _vp, _vp]
    L.afem_sites_grid.restype = C.c_int
    L.afem_site_coeffs_grid.argtypes = [_vp, C.c_int, _vp, _vp, _vp, _vp, _vp]
    L.afem_site_coeffs_grid.restype = C.c_int
    L.afem_xy_points.argtypes = [C.c_double, C.c_double, C.c_double, C.c_double, C.c_int, C.c_int, C.c_double, _vp]
    L.afem_xy_points.restype = C.c_int
    L.afem_sort_index.argtypes = [C.c_int, _vp, _vp]
    L.afem_sort_index.restype = C.c_int
    L.afem_hybrid_matrix.argtypes = [_vp, C.POINTER(C.c_int), C.POINTER(C.c_long), _vp, _vp, _vp]
    L.afem_hybrid_matrix.restype = C.c_int
    L.afem_launch_count.argtypes = []
    L.afem_launch_count.restype = C.c_long
    L.afem_mesh_info.argtypes = [_vp, C.POINTER(C.c_int), C.POINTER(C.c_int), C.POINTER(C.c_int)]
    L.afem_mesh_info.restype = C.c_int
    L.afem_solution_count.argtypes = [_vp, C.POINTER(C.c_int)]
    L.afem_solution_count.restype = C.c_int
    L.afem_set_segments.argtypes = [_vp, C.c_int, _vp]
    L.afem_segment_info.argtypes = [_vp, C.POINTER(C.c_int), _vp, _vp]
    L.afem_set_cond.argtypes = [_vp, C.c_double, C.c_double, C.c_int, C.c_int, _vp, C.c_int, _vp]
    L.afem_set_sigma.argtypes = [_vp, _vp]
    L.afem_set_source.argtypes = [_vp, C.c_int, C.c_int, _vp, _vp]
    L.afem_set_bounds.argtypes = [_vp, C.c_double, C.c_double, C.c_double, C.c_double]
    L.afem_assemble.argtypes = [_vp]
    L.afem_export_system.argtypes = [_vp, C.c_double, C.c_int, C.POINTER(C.c_int), C.POINTER(C.c_long), _vp, _vp,
                                     _vp, _vp, _vp, _vp, _vp, _vp, _vp]
    L.afem_solve.argtypes = [_vp, C.c_int, _vp, _vp, C.POINTER(SolveOpts), C.POINTER(SolveStats)]
    L.afem_get_solution.argtypes = [_vp, C.c_int, _vp]
    L.afem_sites.argtypes = [_vp, C.c_int, _vp, _vp]
    L.afem_site_coeffs.argtypes = [_vp, C.c_int, _vp, _vp, _vp, _vp, _vp]
    L.afem_load_ctl.argtypes = [_vp, C.c_char_p]
    L.afem_ctl_info.argtypes = [_vp, C.POINTER(C.c_int), _vp, C.POINTER(C.c_int), _vp]
    L.afem_run_ctl.argtypes = [_vp, C.POINTER(SolveOpts)]
    L.afem_fortran_g.argtypes = [C.c_double, C.c_int, C.c_int, C.c_char_p, C.c_int]
    L.afem_cocg13_single.argtypes = [_vp, C.c_int, C.c_int, C.c_int, _vp, _vp, _vp, _vp, _vp, _vp, _vp, _vp, _vp,
                                     C.c_char_p, C.c_double, C.c_double, C.POINTER(C.c_double), C.POINTER(C.c_int),
                                     C.POINTER(C.c_int), C.c_int]
    L.afem_set_system.argtypes = [_vp, C.c_int, _vp, _vp, _vp, _vp, _vp, _vp, _vp, _vp]
    L.afem_get_residual.argtypes = [_vp, C.c_int, _vp]
    L.afem_coloring.argtypes = [C.c_int, _vp, _vp, _vp, _vp, _vp]
    L.afem_coloring.restype = C.c_int
    L.afem_sweep_schedule.argtypes = [C.c_int, _vp, _vp, _vp, _vp, _vp, C.POINTER(C.c_int), C.POINTER(C.c_int)]
    L.afem_solve_rhs.argtypes = [_vp, C.c_int, _vp, _vp, C.POINTER(SolveOpts), C.POINTER(SolveStats)]
    L.afem_jacobian.argtypes = [_vp, C.c_double, _vp, C.c_int, _vp]
    L.afem_mpnn_nparam.argtypes = []
    L.afem_mpnn_set_params.argtypes = [_vp, _vp, C.c_int]
    L.afem_mpnn_get_params.argtypes = [_vp, _vp]
    L.afem_mpnn_forward.argtypes = [_vp, C.c_int, _vp, _vp, _vp]
    L.afem_mpnn_loss_grad.argtypes = [_vp, C.c_double, C.c_int, _vp, C.POINTER(C.c_double), _vp]
    L.afem_mpnn_train.argtypes = [_vp, C.c_double, C.c_int, _vp, C.c_int, C.c_float, _vp]
    L.afem_set_profiling.argtypes = [_vp, C.c_int]
    L.afem_profile_count.argtypes = [_vp]
    L.afem_profile_entry.argtypes = [_vp, C.c_int, C.c_char_p, C.c_int, C.POINTER(C.c_double), C.POINTER(C.c_long)]
    L.afem_mt_forward.argtypes = [_vp, C.POINTER(MtCond), C.c_int, _vp, C.c_int, _vp, C.POINTER(SolveOpts), _vp, _vp,
                                  _vp, _vp, C.POINTER(SolveStats)]
    L.afem_mt_forward.restype = C.c_int
    L.afem_mt_boundary.argtypes = [_vp, C.POINTER(MtCond), C.c_double, _vp, _vp]
    L.afem_mt_boundary.restype = C.c_int
    L.afem_mt_face.argtypes = [_vp, C.POINTER(MtCond), C.c_int, C.c_double, C.POINTER(C.c_int), C.POINTER(C.c_long),
                               _vp, _vp, _vp, _vp, _vp, _vp]
    L.afem_mt_face.restype = C.c_int
    for name in ("afem_set_mesh", "afem_get_lines", "afem_set_cond", "afem_set_sigma", "afem_set_source",
                 "afem_set_bounds", "afem_assemble", "afem_export_system", "afem_solve", "afem_get_solution",
                 "afem_sites", "afem_site_coeffs", "afem_load_ctl", "afem_ctl_info", "afem_run_ctl",
                 "afem_fortran_g", "afem_set_profiling", "afem_profile_count", "afem_profile_entry", "afem_cocg13_single",
                 "afem_set_system", "afem_get_residual", "afem_mpnn_nparam", "afem_mpnn_set_params",
                 "afem_mpnn_get_params", "afem_mpnn_forward", "afem_mpnn_loss_grad", "afem_mpnn_train",
                 "afem_solve_rhs", "afem_jacobian", "afem_sweep_schedule", "afem_set_segments", "afem_segment_info"):
        getattr(L, name).restype = C.c_int
    _LIB = L
    return L


def xy_points(xmin, xmax, ymin, ymax, nx, ny, z):
    """PREPOBSCOEFF_XY's plan-view points (nx*ny, 3), point (j-1)*ny + i for x cell j and y cell i."""
    out = np.zeros((nx * ny, 3))
    if lib().afem_xy_points(xmin, xmax, ymin, ymax, nx, ny, z, out.ctypes.data_as(_vp)) != 0:
        raise ValueError("xy_points: bad grid")
    return out


def utm_xy(lon, lat, lonorigin, latorigin, zone):
    """UTMXY: km east/north of the origin in UTM zone `zone` (host only)."""
    out = np.zeros(2)
    rc = lib().afem_utm_xy(float(lon), float(lat), float(lonorigin), float(latorigin), int(zone), out.ctypes.data)
    if rc != AFEM_OK:
        raise AfemError(rc, "utm_xy: bad zone")
    return out


def launch_count() -> int:
    """Kernels the library has launched in this process."""
    return int(lib().afem_launch_count())


def ptr(a):
    return None if a is None else a.ctypes.data_as(_vp)


def fortran_g(x: float, w: int = 15, d: int = 7) -> str:
    buf = C.create_string_buffer(64)
    n = lib().afem_fortran_g(float(x), w, d, buf, 64)
    if n < 0:
        raise ValueError("format overflow")
    return buf.value.decode()
