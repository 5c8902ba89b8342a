"""ctypes front end of the CPU oracle (``afem_oracle.cpp``) -- TEST INFRASTRUCTURE ONLY.

Only ``tests/``, ``__graft_entry__.smoke()`` and the CPU-baseline leg of
``bench.py`` use this module, and only as the checker / timed CPU reference.
Each function names the reference routine it restates; see the C++ source for
file:line citations.  Parity status: unpinned against the reference itself
(no compiler for it here, no golden data shipped with it); pinned by the
reference's two in-source known-answer examples and by identities.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "_build", "liborc.so")

_i32p = np.ctypeslib.ndpointer(dtype=np.int32, flags="C_CONTIGUOUS")
_f64p = np.ctypeslib.ndpointer(dtype=np.float64, flags="C_CONTIGUOUS")
_u8p = np.ctypeslib.ndpointer(dtype=np.uint8, flags="C_CONTIGUOUS")
_c128p = np.ctypeslib.ndpointer(dtype=np.complex128, flags="C_CONTIGUOUS")


def build(force: bool = False) -> str:
    srcs = [os.path.join(HERE, f) for f in ("afem_oracle.cpp", "afem_oracle_mt.cpp", "Makefile")]
    if force or not os.path.exists(LIB_PATH) or os.path.getmtime(LIB_PATH) < max(map(os.path.getmtime, srcs)):
        subprocess.run(["make", "-s", "-C", HERE], check=True)
    return LIB_PATH


_LIB = None


def lib():
    global _LIB
    if _LIB is None:
        build()
        L = C.CDLL(LIB_PATH)
        L.orc_sort_index.argtypes = [C.c_int, _i32p, _f64p]
        L.orc_mul_matcrs_cv.argtypes = [C.c_int, _i32p, _i32p, _f64p, _c128p, _c128p]
        L.orc_mkline.restype = C.c_long
        L.orc_mkline.argtypes = [C.c_int, C.c_long, _i32p, C.c_long, _i32p, _i32p]
        L.orc_pattern.restype = C.c_long
        L.orc_pattern.argtypes = [C.c_int, C.c_long, _i32p, _i32p, _i32p, C.c_void_p, C.c_void_p]
        L.orc_resolve_sigma.restype = C.c_long
        L.orc_resolve_sigma.argtypes = [C.c_long, _i32p, C.c_double, C.c_double, C.c_int, C.c_int, _f64p, C.c_long,
                                        _f64p, _f64p]
        L.orc_forward_assemble.restype = C.c_int
        L.orc_forward_assemble.argtypes = [C.c_int, _f64p, C.c_long, _i32p, _i32p, C.c_int, _i32p, _i32p, _i32p, _i32p,
                                           _i32p, _i32p, _f64p, C.c_int, _f64p, _c128p, C.c_double, C.c_double,
                                           C.c_double, C.c_double, C.c_double, C.c_int, _c128p, _c128p, _c128p, _c128p,
                                           _u8p, C.POINTER(C.c_long)]
        L.orc_assemble_split.restype = C.c_int
        L.orc_assemble_split.argtypes = [C.c_long, _f64p, _i32p, _i32p, C.c_int, _i32p, _i32p, _f64p, _f64p, _f64p,
                                         _f64p, _f64p]
        L.orc_cocg13_single.restype = None
        L.orc_cocg13_single.argtypes = [C.c_int, C.c_int, C.c_int, _c128p, _c128p, _i32p, _i32p, _c128p, _i32p, _i32p,
                                        _c128p, _c128p, C.c_char_p, C.c_double, C.c_double, C.POINTER(C.c_double),
                                        C.POINTER(C.c_int), C.POINTER(C.c_int), C.c_int, C.c_void_p]
        L.orc_cocg_begin.restype = C.c_void_p
        L.orc_cocg_begin.argtypes = [C.c_int, _c128p, _c128p, _i32p, _i32p, _c128p, _i32p, _i32p, _c128p, _c128p,
                                     C.c_char_p, C.c_double, C.c_int]
        L.orc_cocg_advance.restype = C.c_double
        L.orc_cocg_advance.argtypes = [C.c_void_p, C.c_int]
        L.orc_cocg_iterations.restype = C.c_int
        L.orc_cocg_iterations.argtypes = [C.c_void_p]
        L.orc_cocg_end.restype = None
        L.orc_cocg_end.argtypes = [C.c_void_p]
        L.orc_utm_lonlat2xy.restype = None
        L.orc_utm_lonlat2xy.argtypes = [C.c_double, C.c_double, C.c_int, C.c_int, C.POINTER(C.c_double),
                                        C.POINTER(C.c_double)]
        L.orc_utmxy.restype = None
        L.orc_utmxy.argtypes = [C.c_double, C.c_double, C.c_double, C.c_double, C.c_int, _f64p]
        L.orc_true_residual.restype = C.c_double
        L.orc_true_residual.argtypes = [C.c_int, _c128p, _c128p, _i32p, _i32p, _c128p, _i32p, _i32p, _c128p, _c128p]
        L.orc_findelement0.restype = C.c_long
        L.orc_findelement0.argtypes = [_f64p, _f64p, C.c_long, _i32p, _f64p]
        L.orc_prepobscoeff.restype = C.c_long
        L.orc_prepobscoeff.argtypes = [_f64p, C.c_long, _i32p, _i32p, C.c_int, _f64p, _i32p, _f64p, _f64p, _i32p]
        L.orc_prepobscoeff_grid.restype = C.c_long
        L.orc_prepobscoeff_grid.argtypes = [_f64p, C.c_long, C.c_long, _i32p, _i32p, C.c_int, _f64p, _i32p, _f64p,
                                            _f64p, _i32p]
        L.orc_prepobscoeff_grid_nz.restype = C.c_long
        L.orc_prepobscoeff_grid_nz.argtypes = [_f64p, C.c_long, C.c_long, _i32p, _i32p, C.c_int, _f64p, C.c_int,
                                               _i32p, _f64p, _f64p, _i32p]
        L.orc_findtri_grid.restype = C.c_long
        L.orc_findtri_grid.argtypes = [_f64p, C.c_long, _i32p, _f64p, C.c_int, C.c_int, C.c_int, _f64p, _i32p,
                                       _f64p]
        L.orc_calobsebcomp.restype = None
        L.orc_calobsebcomp.argtypes = [C.c_int, C.c_int, C.c_double, _c128p, C.c_int, _i32p, _f64p, _f64p, _c128p,
                                       _f64p, _f64p]
        L.orc_mt_surfaces.restype = C.c_void_p
        L.orc_mt_surfaces.argtypes = [C.c_int, _f64p, C.c_long, _i32p, C.c_int, _i32p, _i32p]
        L.orc_mt_free.argtypes = [C.c_void_p]
        L.orc_mt_error.restype = C.c_int
        L.orc_mt_error.argtypes = [C.c_void_p]
        L.orc_mt_minmax.argtypes = [C.c_void_p, _f64p]
        L.orc_mt_surface_sizes.argtypes = [C.c_void_p, C.c_int] + [C.POINTER(C.c_int)] * 3
        L.orc_mt_surface_get.argtypes = [C.c_void_p, C.c_int] + [C.c_void_p] * 7
        L.orc_mt_cond2d.restype = C.c_long
        L.orc_mt_cond2d.argtypes = [C.c_void_p, C.c_int, _i32p, C.c_double, C.c_int, C.c_double, C.c_long, _f64p,
                                    _f64p]
        L.orc_mt_face_system.restype = C.c_int
        L.orc_mt_face_system.argtypes = [C.c_void_p, C.c_int, _f64p, C.c_double, C.c_int, C.POINTER(C.c_long)] + \
            [C.c_void_p] * 10
        L.orc_mt_genbcmt.argtypes = [C.c_void_p, C.c_double, C.c_int, _c128p, _c128p, _c128p, _c128p, _c128p, _u8p]
        L.orc_mt_set_bc3d.argtypes = [C.c_int, C.c_int, _c128p, _c128p, _i32p, _i32p, _c128p, _i32p, _i32p, _c128p,
                                      _u8p, _c128p]
        L.orc_mt_calrespmt.argtypes = [C.c_int, C.c_double, _c128p, _c128p, _f64p, _f64p]
        _LIB = L
    return _LIB


def _c(a, dt):
    return np.ascontiguousarray(a, dtype=dt)


def sort_index(na, ra):
    """SORT_INDEX: heap sort of ra carrying na (src/solver/sort_index.f90:13-56)."""
    na = _c(na, np.int32).copy(); ra = _c(ra, np.float64).copy()
    lib().orc_sort_index(len(na), na, ra)
    return na, ra


def mul_matcrs_cv(stack, item, val, cv):
    """mul_matcrs_cv (src/common/m_matrix.f90:83-102); stack 0-based prefix, item 1-based."""
    stack = _c(stack, np.int32); out = np.zeros(len(stack) - 1, dtype=np.complex128)
    lib().orc_mul_matcrs_cv(len(stack) - 1, stack, _c(item, np.int32), _c(val, np.float64), _c(cv, np.complex128), out)
    return out


def mkline(node: int, n4):
    """MKLINE_V2 + MKN6: returns line (nline, 2) and n6line (ntet, 6), 1-based."""
    n4 = _c(n4, np.int32)
    ntet = n4.shape[0]
    cap = 6 * ntet + 6
    line = np.zeros((cap, 2), dtype=np.int32)
    n6 = np.zeros((ntet, 6), dtype=np.int32)
    nline = lib().orc_mkline(node, ntet, n4, cap, line, n6)
    if nline < 0:
        raise RuntimeError(f"orc_mkline failed: {nline}")
    return np.ascontiguousarray(line[:nline]), n6


def pattern(nline: int, n6line):
    """set_iccg_var7_dofn/C_set_dof2: INU, IAU, INL, IAL (prefix arrays length n+1, columns 1-based)."""
    n6 = _c(n6line, np.int32)
    INU = np.zeros(nline + 1, dtype=np.int32); INL = np.zeros(nline + 1, dtype=np.int32)
    tot = lib().orc_pattern(nline, n6.shape[0], n6, INU, INL, None, None)
    if tot < 0:
        raise RuntimeError("orc_pattern overflow")
    IAU = np.zeros(tot, dtype=np.int32); IAL = np.zeros(tot, dtype=np.int32)
    lib().orc_pattern(nline, n6.shape[0], n6, INU, INL, IAU.ctypes.data, IAL.ctypes.data)
    return INU, IAU, INL, IAL


def resolve_sigma(tag, sigma_air, sigma_ocean, condflag, sigma_land=None, nphys1=0, sigma_file=None):
    """Per-tetrahedron sigma as GENMAT selects it (forward_bxyz_mpi.f90:196-208)."""
    tag = _c(tag, np.int32)
    sl = _c(sigma_land if sigma_land is not None else [0.0], np.float64)
    sf = _c(sigma_file if sigma_file is not None else [0.0], np.float64)
    out = np.zeros(tag.shape[0], dtype=np.float64)
    rc = lib().orc_resolve_sigma(tag.shape[0], tag, sigma_air, sigma_ocean, condflag, len(sl), sl, nphys1, sf, out)
    if rc != 0:
        raise RuntimeError(f"resolve_sigma: tetrahedron {-rc} has no conductivity")
    return out


class Assembled:
    def __init__(self, D, AU, AL, b, bc, INU, IAU, INL, IAL):
        self.D, self.AU, self.AL, self.b, self.bc = D, AU, AL, b, bc
        self.INU, self.IAU, self.INL, self.IAL = INU, IAU, INL, IAL

    @property
    def n(self):
        return self.D.shape[0]

    def to_scipy(self):
        import scipy.sparse as sp
        n = self.n
        rows_u = np.repeat(np.arange(n), np.diff(self.INU))
        rows_l = np.repeat(np.arange(n), np.diff(self.INL))
        r = np.concatenate([np.arange(n), rows_u, rows_l])
        c = np.concatenate([np.arange(n), self.IAU - 1, self.IAL - 1])
        v = np.concatenate([self.D, self.AU, self.AL])
        return sp.csr_matrix((v, (r, c)), shape=(n, n))


def forward_assemble(m, line, n6line, pat, freq, sigma_tet, apply_bc=True) -> Assembled:
    """INITIALIZE+GENMAT+COPY_UL_ICCG12+GENBCCSEM+SET_BC_ICCG for one frequency."""
    INU, IAU, INL, IAL = pat
    n = line.shape[0]
    D = np.zeros(n, np.complex128); b = np.zeros(n, np.complex128)
    AU = np.zeros(len(IAU), np.complex128); AL = np.zeros(len(IAL), np.complex128)
    bc = np.zeros(n, np.uint8)
    bad = C.c_long(0)
    F = _c(m.F, np.float64).reshape(-1)
    v = _c(m.v, np.complex128).reshape(-1)
    rc = lib().orc_forward_assemble(m.node, _c(m.xyz, np.float64).reshape(-1), m.ntet, _c(m.n4, np.int32), _c(m.tag, np.int32),
                                    n, _c(line, np.int32), _c(n6line, np.int32), INU, IAU, INL, IAL,
                                    _c(sigma_tet, np.float64), m.nodes, F, v, float(freq), m.bounds["zmin"],
                                    m.bounds["zmax"], m.bounds["xout"], m.bounds["yout"], int(apply_bc), D, AU, AL, b,
                                    bc, C.byref(bad))
    if rc != 0:
        raise RuntimeError(f"orc_forward_assemble failed rc={rc} at element {bad.value}")
    return Assembled(D, AU, AL, b, bc, INU, IAU, INL, IAL)


def assemble_split(m, n6line, pat, sigma_tet):
    INU, IAU, _, _ = pat
    n = len(INU) - 1
    Kd = np.zeros(n); Md = np.zeros(n); Ku = np.zeros(len(IAU)); Mu = np.zeros(len(IAU))
    rc = lib().orc_assemble_split(m.ntet, _c(m.xyz, np.float64).reshape(-1), _c(m.n4, np.int32), _c(n6line, np.int32),
                                  n, INU, IAU, _c(sigma_tet, np.float64), Kd, Ku, Md, Mu)
    if rc != 0:
        raise RuntimeError(f"orc_assemble_split rc={rc}")
    return Kd, Ku, Md, Mu


def cocg13_single(A: Assembled, b=None, x0=None, precond="IC", resid=1e-8, maxit=20000, sigma_diag=1.0, sigma=0.0,
                  nset=1, history=False):
    """COCG13_single on copies of A (the reference mutates its arguments)."""
    n = A.n
    D = A.D.copy(); AL = A.AL.copy(); AU = A.AU.copy()
    B = (A.b if b is None else np.asarray(b, np.complex128)).copy()
    X = np.zeros(n, np.complex128) if x0 is None else np.asarray(x0, np.complex128).copy()
    R = C.c_double(resid); IT = C.c_int(maxit); ER = C.c_int(0)
    hist = np.zeros(maxit + 1) if history else None
    lib().orc_cocg13_single(n, len(AL), len(AU), D, AL, A.INL, A.IAL, AU, A.INU, A.IAU, B, X, precond.encode(),
                            sigma_diag, sigma, C.byref(R), C.byref(IT), C.byref(ER), nset,
                            hist.ctypes.data if history else None)
    out = dict(x=X, resid=R.value, iter=IT.value, error=ER.value)
    if history:
        out["history"] = hist[: min(IT.value, maxit)]
    return out


class CocgSlices:
    """COCG13_single run in slices: the same iterations as cocg13_single, with the
    Krylov state kept between advance() calls (the reference's solver timed on a
    bounded sample).  A is read, not modified (NSET 1); b defaults to A.b."""

    def __init__(self, A: Assembled, b=None, precond="SSOR", sigma_diag=1.0):
        self.A = A
        self.b = (A.b if b is None else np.asarray(b, np.complex128)).copy()
        self.x = np.zeros(A.n, np.complex128)
        self.h = lib().orc_cocg_begin(A.n, A.D, A.AL, A.INL, A.IAL, A.AU, A.INU, A.IAU, self.b, self.x,
                                      precond.encode(), sigma_diag, 1)
        if not self.h:
            raise ValueError("CocgSlices: ||b|| = 0")
        self.resid = 1.0

    def advance(self, k: int) -> float:
        """k more iterations (ctypes releases the GIL, so threads run in parallel)."""
        self.resid = lib().orc_cocg_advance(self.h, int(k))
        return self.resid

    @property
    def iterations(self) -> int:
        return lib().orc_cocg_iterations(self.h)

    def close(self):
        if self.h:
            lib().orc_cocg_end(self.h)
            self.h = None
        return self.x


def true_residual(A: Assembled, x, b=None):
    B = A.b if b is None else _c(b, np.complex128)
    return lib().orc_true_residual(A.n, A.D, A.AL, A.INL, A.IAL, A.AU, A.INU, A.IAU, _c(B, np.complex128),
                                   _c(x, np.complex128))


def utm_lonlat2xy(lon, lat, zone, reference_series=True):
    """utm_geo_tm LONLAT2UTM: easting, northing [m]; reference_series=False uses Snyder's series."""
    x = C.c_double(); y = C.c_double()
    lib().orc_utm_lonlat2xy(float(lon), float(lat), int(zone), int(bool(reference_series)), C.byref(x), C.byref(y))
    return x.value, y.value


def utmxy(lon, lat, lonorigin, latorigin, zone):
    """UTMXY: km east/north of the origin."""
    out = np.zeros(2)
    lib().orc_utmxy(float(lon), float(lat), float(lonorigin), float(latorigin), int(zone), out)
    return out


def findelement0(m, x3):
    a = np.zeros(4)
    i = lib().orc_findelement0(_c(x3, np.float64), _c(m.xyz, np.float64).reshape(-1), m.ntet, _c(m.n4, np.int32), a)
    return int(i), a


def prepobscoeff(m, n6line, sites):
    """PREPOBSCOEFF: item (nobs,6) 1-based sorted edge ids; val_e/val_f (3, nobs, 6); iele (nobs,)."""
    sites = _c(sites, np.float64)
    nobs = sites.shape[0]
    item = np.zeros((nobs, 6), np.int32)
    ve = np.zeros((3, nobs, 6)); vf = np.zeros((3, nobs, 6)); iele = np.zeros(nobs, np.int32)
    rc = lib().orc_prepobscoeff(_c(m.xyz, np.float64).reshape(-1), m.ntet, _c(m.n4, np.int32), _c(n6line, np.int32), nobs,
                                sites.reshape(-1), item, ve, vf, iele)
    if rc != 0:
        raise RuntimeError(f"site {-rc} is outside the mesh")
    return item, ve, vf, iele


def prepobscoeff_grid(m, n6line, sites):
    """PREPOBSCOEFF_XY's search: FINDELEWITHGRID over the grid list (m_mesh_type.f90:56-277), same rows."""
    sites = _c(sites, np.float64)
    nobs = sites.shape[0]
    item = np.zeros((nobs, 6), np.int32)
    ve = np.zeros((3, nobs, 6)); vf = np.zeros((3, nobs, 6)); iele = np.zeros(nobs, np.int32)
    rc = lib().orc_prepobscoeff_grid(_c(m.xyz, np.float64).reshape(-1), m.node, m.ntet, _c(m.n4, np.int32),
                                     _c(n6line, np.int32), nobs, sites.reshape(-1), item, ve, vf, iele)
    if rc != 0:
        raise RuntimeError(f"site {-rc} is outside the mesh")
    return item, ve, vf, iele


def prepobscoeff_grid_nz(m, n6line, sites, nz):
    """prepobscoeff_grid with the grid list's nz boxes in z (PREPOBSCOEFF_XYSBTM uses 300)."""
    sites = _c(sites, np.float64)
    nobs = sites.shape[0]
    item = np.zeros((nobs, 6), np.int32)
    ve = np.zeros((3, nobs, 6)); vf = np.zeros((3, nobs, 6)); iele = np.zeros(nobs, np.int32)
    rc = lib().orc_prepobscoeff_grid_nz(_c(m.xyz, np.float64).reshape(-1), m.node, m.ntet, _c(m.n4, np.int32),
                                        _c(n6line, np.int32), nobs, sites.reshape(-1), int(nz), item, ve, vf, iele)
    if rc != 0:
        raise RuntimeError(f"site {-rc} is outside the mesh")
    return item, ve, vf, iele


def findtri_grid(xyz, n3, minmax, pts2, nx=200, ny=200):
    """findtriwithgrid over a triangle mesh (m_triangle.f90:11-260): 1-based triangle and a3 per point."""
    pts2 = _c(np.asarray(pts2)[:, :2], np.float64)
    npts = pts2.shape[0]
    iele = np.zeros(npts, np.int32)
    a3 = np.zeros((npts, 3))
    rc = lib().orc_findtri_grid(_c(xyz, np.float64).reshape(-1), int(n3.shape[0]), _c(n3, np.int32).reshape(-1),
                                _c(minmax, np.float64), nx, ny, npts, pts2.reshape(-1), iele, a3)
    if rc != 0:
        raise RuntimeError(f"findtri_grid failed: {rc}")
    return iele, a3


def xyz_minmax(xyz):
    """GENXYZMINMAX (n_ebfem_bxyz_mpi.f90:533-565): node extent xmin, xmax, ymin, ymax, zmin, zmax."""
    return np.array([xyz[:, 0].min(), xyz[:, 0].max(), xyz[:, 1].min(), xyz[:, 1].max(), xyz[:, 2].min(),
                     xyz[:, 2].max()])


def prepzobs(xyz3d, ki_xyz, ki_n3, ki23dptr, pts):
    """PREPZOBS with iflag 1 (n_ebfem_bxyz_mpi.f90:1181-1267): each plan-view point 1 m below the seafloor
    under it (the triangle of the polygon_ki mesh that holds it, its nodes' seafloor nodes ki23dptr(2,:)),
    and the coeff_vF rows (3 seafloor nodes, the triangle's coordinates).  Returns xyz, items (1-based), vals."""
    iele, a3 = findtri_grid(ki_xyz, ki_n3, xyz_minmax(xyz3d)[:4], pts, 200, 200)
    m = ki23dptr[ki_n3[iele - 1] - 1, 1]  # (npts, 3) 1-based 3-D seafloor nodes
    out = np.array(pts, np.float64).copy()
    z = xyz3d[:, 2]
    out[:, 2] = a3[:, 0] * z[m[:, 0] - 1] + a3[:, 1] * z[m[:, 1] - 1] + a3[:, 2] * z[m[:, 2] - 1] - 0.001
    return out, m.astype(np.int32), a3


def xysbtm_points(xyz3d, ki_n3, ki23dptr):
    """PREPOBSCOEFF_XYSBTM's points (n_ebfem_bxyz_mpi.f90:1064-1078): per polygon_ki triangle, the mean of its
    three seafloor nodes raised by 1 m, and coeff_vF rows of 1/3 on those nodes."""
    m = ki23dptr[ki_n3 - 1, 1].astype(np.int32)  # (ntri, 3)
    x3 = np.zeros((ki_n3.shape[0], 3))
    up = np.array([0.0, 0.0, 0.001])
    for j in range(3):
        x3 = x3 + xyz3d[m[:, j] - 1] / 3.0 + up / 3.0
    return x3, m, np.full(m.shape, 1.0 / 3.0)


def ixyhout(pts, fields5, F, v, items, vals):
    """IXYHOUT (n_ebfem_bxyz_mpi.f90:192-302): the 26 columns of ixyh_xy2D<freq>.dat per plan-view point.

    fields5: complex (5, npts) bx, by, bz, ex, ey of source 1; F (node, 3) nT and v (node, 3) m/s over the
    3-D mesh nodes (zero past the ocean nodes), items/vals the coeff_vF rows."""
    pi = 4.0 * np.arctan(1.0)
    d2r, r2d = pi / 180.0, 180.0 / pi
    amp = np.sqrt(fields5.real ** 2.0 + fields5.imag ** 2.0)
    ph = np.arctan2(fields5.imag, fields5.real) * r2d
    rec = amp * np.exp(1j * ph * d2r)             # CALOBSRESP amp/phase read back as in IXYHOUT
    bxyz, exy = rec[0:3], rec[3:5]
    sig = float(np.float32(3.3))                    # sigma_ocean = 3.3, a default-real literal
    h = -np.asarray(pts)[:, 2]
    h = np.where(h <= 0.0, 0.0, h)
    vF = np.stack([v[:, 1] * F[:, 2] - v[:, 2] * F[:, 1], v[:, 2] * F[:, 0] - v[:, 0] * F[:, 2],
                   v[:, 0] * F[:, 1] - v[:, 1] * F[:, 0]])
    npts = len(h)
    vF_obs = np.zeros((3, npts), np.complex128)
    vh = np.zeros((2, npts), np.complex128)
    for k in range(items.shape[1]):               # mul_matcrs_cv, in the row's entry order
        vF_obs = vF_obs + vals[:, k] * vF[:, items[:, k] - 1]
        vh = vh + vals[:, k] * v[items[:, k] - 1, :2].T
    ixyh = sig * h * (exy + vF_obs[:2] * 1e-3)
    ixyh_e = sig * h * exy
    ixyh_vF = sig * h * vF_obs[:2] * 1e-3
    vh = h * vh
    cols = [np.asarray(pts)[:, j] for j in range(3)]
    for arr in (ixyh_e, ixyh_vF, ixyh, vh, bxyz):
        for c in range(arr.shape[0]):
            cols += [arr[c].real, arr[c].imag]
    cols.append(h)
    return np.stack(cols, axis=1)


def calobsebcomp(fs, omega, item, ve, vf):
    """CALOBSEBCOMP with fp = 0: returns complex (nsr, 5, nobs) [bx,by,bz,ex,ey], amp, phase (deg)."""
    fs = np.asarray(fs, np.complex128)
    if fs.ndim == 1:
        fs = fs[None, :]
    nsr, nline = fs.shape
    nobs = item.shape[0]
    out = np.zeros((nsr, 5, nobs), np.complex128); amp = np.zeros((nsr, 5, nobs)); ph = np.zeros((nsr, 5, nobs))
    lib().orc_calobsebcomp(nline, nsr, float(omega), _c(fs, np.complex128), nobs, _c(item, np.int32),
                           _c(ve, np.float64), _c(vf, np.float64), out, amp, ph)
    return out, amp, ph


class OracleForward:
    """The whole reference path for one model on the CPU: numbering, pattern, assembly, COCG, sites."""

    def __init__(self, m, line=None, n6line=None):
        self.m = m
        if line is None:
            line, n6line = mkline(m.node, m.n4)
        self.line, self.n6line = line, n6line
        self.pat = pattern(line.shape[0], n6line)
        self.sigma_tet = m.sigma_per_tet()

    def assemble(self, freq, apply_bc=True) -> Assembled:
        return forward_assemble(self.m, self.line, self.n6line, self.pat, freq, self.sigma_tet, apply_bc)

    def sites(self, x, freq):
        item, ve, vf, _ = prepobscoeff(self.m, self.n6line, self.m.sites)
        omega = 2.0 * (4.0 * np.arctan(1.0)) * freq
        return calobsebcomp(x, omega, item, ve, vf)


# ----------------------------------------------------------------------------- 3-D MT forward
def mt_sigma(m):
    """GENMAT_MT's conductivity per tetrahedron (src/src_3DMT/forward_3DMT.f90:239-252): physical tags
    1 and 2 -> sigma_air, >= 3 -> the per-element file value (condflag 1)."""
    return resolve_sigma(m.tag, m.sigma_air, m.sigma_air, 1, None, m.nphys1, m.sigma_land)


class Face:
    """The 2-D TM system of one side surface at one frequency (split storage, after SET_BC_ICCG)."""

    def __init__(self, A: Assembled, rf, gval, line3d, flag):
        self.A, self.rf, self.gval, self.line3d, self.flag = A, rf, gval, line3d, flag

    def solve(self):
        """The direct solve the reference leaves to PARDISO (forward_2DTM.f90:160), here SuperLU."""
        import scipy.sparse.linalg as sla
        return sla.spsolve(self.A.to_scipy().tocsc(), self.rf)


class MTOracle:
    """EXTRACT6SURFACES, the 2-D TM boundary solves, GENBCMT, GENMAT_MT + SET_BC_3DJoint and
    CALRESPMT (src/src_3DMT/n_ebfem_3DMT.f90:38-113) on a model m with numbering (line, n6line)."""

    def __init__(self, m, line, n6line):
        self.m = m
        self.line = _c(line, np.int32)
        self.n6line = _c(n6line, np.int32)
        self.nline = self.line.shape[0]
        self.h = lib().orc_mt_surfaces(m.node, _c(m.xyz, np.float64).reshape(-1), m.ntet, _c(m.n4, np.int32),
                                       self.nline, self.line, self.n6line)
        err = lib().orc_mt_error(self.h)
        if err != 0:
            raise RuntimeError(f"orc_mt_surfaces failed: {err}")
        self.pat = pattern(self.nline, self.n6line)

    def __del__(self):
        if getattr(self, "h", None):
            lib().orc_mt_free(self.h)
            self.h = None

    def minmax(self):
        mm = np.zeros(6)
        lib().orc_mt_minmax(self.h, mm)
        return mm

    def surface(self, j: int) -> dict:
        a, b, c = C.c_int(), C.c_int(), C.c_int()
        lib().orc_mt_surface_sizes(self.h, j, C.byref(a), C.byref(b), C.byref(c))
        node, ntri, nl = a.value, b.value, c.value
        d = dict(x1x2=np.zeros((node, 2)), n3=np.zeros((ntri, 3), np.int32), n3line=np.zeros((ntri, 3), np.int32),
                 tet=np.zeros(ntri, np.int32), line=np.zeros((nl, 2), np.int32), line3d=np.zeros(nl, np.int32),
                 flag=np.zeros(nl, np.int32))
        lib().orc_mt_surface_get(self.h, j, *[d[k].ctypes.data for k in ("x1x2", "n3", "n3line", "tet", "line",
                                                                         "line3d", "flag")])
        return d

    def cond2d(self, j: int):
        m = self.m
        ntri = self.surface(j)["tet"].shape[0]
        out = np.zeros(ntri)
        rc = lib().orc_mt_cond2d(self.h, j, _c(m.tag, np.int32), m.sigma_air, 1, 0.0, m.nphys1,
                                 _c(m.sigma_land, np.float64), out)
        if rc != 0:
            raise RuntimeError(f"cond3dto2d: triangle {-rc} has no conductivity")
        return out

    def face(self, j: int, freq: float, apply_bc: bool = True) -> Face:
        cond = self.cond2d(j)
        tot = C.c_long(0)
        L = lib()
        nul = [None] * 10
        rc = L.orc_mt_face_system(self.h, j, cond, float(freq), int(apply_bc), C.byref(tot), *nul)
        s = self.surface(j)
        n = s["line3d"].shape[0]
        INU = np.zeros(n + 1, np.int32); INL = np.zeros(n + 1, np.int32)
        IAU = np.zeros(tot.value, np.int32); IAL = np.zeros(tot.value, np.int32)
        D = np.zeros(n, np.complex128); AU = np.zeros(tot.value, np.complex128); AL = np.zeros(tot.value, np.complex128)
        rf = np.zeros(n, np.complex128); bc = np.zeros(n, np.uint8); gv = np.zeros(n, np.complex128)
        rc = L.orc_mt_face_system(self.h, j, cond, float(freq), int(apply_bc), C.byref(tot),
                                  *[x.ctypes.data for x in (INU, IAU, INL, IAL, D, AU, AL, rf, bc, gv)])
        if rc != 0:
            raise RuntimeError(f"orc_mt_face_system({j}) rc={rc}")
        return Face(Assembled(D, AU, AL, rf, bc, INU, IAU, INL, IAL), rf, gv, s["line3d"], s["flag"])

    def boundary(self, freq: float, bs=None):
        """GENBCMT after the four 2-D solves: (Avalue (2, nline) complex, line_bc (nline,)) and the bs used."""
        if bs is None:
            bs = [self.face(j, freq).solve() for j in (2, 3, 4, 5)]
        av = np.zeros((2, self.nline), np.complex128)
        bc = np.zeros(self.nline, np.uint8)
        lib().orc_mt_genbcmt(self.h, 2.0 * np.pi * freq, self.nline, *[_c(b, np.complex128) for b in bs], av, bc)
        return av, bc, bs

    def system(self, freq: float, av, bc):
        """INITIALIZE + GENMAT_MT + COPY_UL_ICCG12 + SET_BC_3DJoint: the split system and rf (2, nline)."""
        import types
        m = self.m
        src = types.SimpleNamespace(**{k: getattr(m, k) for k in ("node", "xyz", "ntet", "n4", "tag", "bounds")})
        src.nodes = 0
        src.F = np.zeros((1, 3)); src.v = np.zeros((1, 3), np.complex128)
        A = forward_assemble(src, self.line, self.n6line, self.pat, freq, mt_sigma(m), apply_bc=False)
        rf = np.zeros((2, self.nline), np.complex128)
        lib().orc_mt_set_bc3d(self.nline, 2, A.D, A.AL, A.INL, A.IAL, A.AU, A.INU, A.IAU, _c(av, np.complex128),
                              _c(bc, np.uint8), rf)
        A.bc = _c(bc, np.uint8)
        return A, rf

    def forward(self, freqs, sites, solver="direct", tol=1e-10):
        """Fields at the sites for both polarisations, impedances and apparent resistivity/phase:
        be (nfreq, 2, 5, nobs), z (nfreq, 4, nobs), rho, pha (nfreq, 4, nobs), and the solutions."""
        import scipy.sparse.linalg as sla
        item, ve, vf, _ = prepobscoeff(self.m, self.n6line, sites)
        nobs = item.shape[0]
        out = dict(be=[], z=[], rho=[], pha=[], x=[], resid=[])
        for f in np.atleast_1d(freqs):
            av, bc, _ = self.boundary(f)
            A, rf = self.system(f, av, bc)
            X = np.zeros((2, self.nline), np.complex128)
            if solver == "direct":
                lu = sla.splu(A.to_scipy().tocsc())
                for k in range(2):
                    X[k] = lu.solve(rf[k])
            else:
                for k in range(2):
                    X[k] = cocg13_single(A, b=rf[k], precond="SSOR", resid=tol, maxit=200000)["x"]
            om = 2.0 * np.pi * f
            be = np.zeros((2, 5, nobs), np.complex128)
            lib().orc_calobsebcomp(self.nline, 2, om, X.reshape(-1), nobs, item, ve, vf, be, np.zeros(10 * nobs),
                                   np.zeros(10 * nobs))
            z = np.zeros((4, nobs), np.complex128); rho = np.zeros((4, nobs)); pha = np.zeros((4, nobs))
            lib().orc_mt_calrespmt(nobs, om, be, z, rho, pha)
            out["be"].append(be); out["z"].append(z); out["rho"].append(rho); out["pha"].append(pha)
            out["x"].append(X)
            out["resid"].append([true_residual(A, X[k], rf[k]) for k in range(2)])
        return {k: np.asarray(v) for k, v in out.items()}
