"""Host-side API of the B200 tidal forward path, over the C ABI (include/afem.h).

Mirrors the reference's seams (src/solver_mpi/forward_bxyz_mpi.f90:3,
src/solver/COCG13_single.f90:9, src/solver_mpi/n_ebfem_bxyz_mpi.f90:397/653):
a ``Forward`` object holds one device context with the mesh, conductivity,
tidal source and Dirichlet bounds; ``assemble`` builds the system once for
every frequency, ``solve`` runs batched COCG, ``sites`` evaluates B and E.
Errors raise ``AfemError`` with the library's status code, as the reference
reports ``ERROR`` / stops.
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass

import numpy as np

from . import capi
from .capi import AfemError, SolveOpts, SolveStats, ptr


def _c(a, dt):
    return np.ascontiguousarray(a, dtype=dt)


@dataclass
class SolveResult:
    iterations: int
    refinements: int
    resid_recursive: float
    resid_true: float
    seconds: float
    status: int

    @property
    def ok(self) -> bool:
        return self.status == capi.AFEM_OK


class Forward:
    """One device context (one CUDA stream) holding one forward problem."""

    def __init__(self, device: int = 0):
        self._L = capi.lib()
        self.ctx = self._L.afem_create(device)
        if not self.ctx:
            raise AfemError(-7, f"afem_create({device}) failed: no usable CUDA device")
        self.node = self.ntet = self.nline = 0
        self.row_ptr = None

    def close(self):
        if self.ctx:
            self._L.afem_destroy(self.ctx)
            self.ctx = None

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _check(self, rc):
        if rc != capi.AFEM_OK:
            raise AfemError(rc, self._L.afem_last_error(self.ctx).decode())

    # ------------------------------------------------------------ inputs
    def set_mesh(self, xyz, n4, tag, line=None, n6line=None):
        """readmsh2 + READLINE; without line/n6line the MKLINE_V2 numbering is built on the device."""
        xyz = _c(xyz, np.float64); n4 = _c(n4, np.int32); tag = _c(tag, np.int32)
        self.node, self.ntet = xyz.shape[0], n4.shape[0]
        if line is None:
            self._check(self._L.afem_set_mesh(self.ctx, self.node, ptr(xyz), self.ntet, ptr(n4), ptr(tag), 0, None, None))
        else:
            line = _c(line, np.int32); n6line = _c(n6line, np.int32)
            self._check(self._L.afem_set_mesh(self.ctx, self.node, ptr(xyz), self.ntet, ptr(n4), ptr(tag), line.shape[0],
                                              ptr(line), ptr(n6line)))
        self._sizes()
        self.row_ptr = None

    def _sizes(self):
        """Mesh sizes as the library holds them (host buffers are always sized from these)."""
        node = C.c_int(0); ntet = C.c_int(0); nline = C.c_int(0)
        self._check(self._L.afem_mesh_info(self.ctx, C.byref(node), C.byref(ntet), C.byref(nline)))
        self.node, self.ntet, self.nline = node.value, ntet.value, nline.value

    def set_segments(self, node_ptr):
        """Declare the mesh as a packed batch of independent meshes (0-based node-range prefix)."""
        self.row_ptr = None
        if node_ptr is None or len(node_ptr) <= 1:
            self._check(self._L.afem_set_segments(self.ctx, 0, None))
            return
        npt = _c(node_ptr, np.int32)
        self._check(self._L.afem_set_segments(self.ctx, len(npt) - 1, ptr(npt)))
        self.row_ptr, self.tet_ptr = self.segment_info()

    def segment_info(self):
        """(row_ptr, tet_ptr) of the declared meshes."""
        k = C.c_int(0)
        self._check(self._L.afem_segment_info(self.ctx, C.byref(k), None, None))
        rp = np.zeros(k.value + 1, np.int32); tp = np.zeros(k.value + 1, np.int32)
        self._check(self._L.afem_segment_info(self.ctx, C.byref(k), ptr(rp), ptr(tp)))
        return rp, tp

    def load_packed(self, pk):
        """Load a synth.PackedModels batch: union mesh, mesh declaration, conductivity, source, bounds."""
        self.set_mesh(pk.xyz, pk.n4, pk.tag)
        self.set_segments(pk.node_ptr)
        self.set_sigma(pk.sigma_tet)
        self.set_source(pk.F, pk.v, 0)
        b = pk.bounds
        self.set_bounds(b["zmin"], b["zmax"], b["xout"], b["yout"])

    def _rows(self, k):
        return self.nline if self.row_ptr is None else int(self.row_ptr[k + 1] - self.row_ptr[k])

    def lines(self):
        self._sizes()
        line = np.zeros((self.nline, 2), np.int32); n6 = np.zeros((self.ntet, 6), np.int32)
        self._check(self._L.afem_get_lines(self.ctx, None, ptr(line), ptr(n6)))
        return line, n6

    def set_cond(self, sigma_air, sigma_ocean, condflag, sigma_land=None, sigma_file=None):
        sl = None if sigma_land is None else _c(sigma_land, np.float64)
        sf = None if sigma_file is None else _c(sigma_file, np.float64)
        self._check(self._L.afem_set_cond(self.ctx, float(sigma_air), float(sigma_ocean), int(condflag),
                                          0 if sl is None else len(sl), ptr(sl), 0 if sf is None else len(sf), ptr(sf)))

    def set_sigma(self, sigma_tet):
        s = _c(sigma_tet, np.float64)
        self._check(self._L.afem_set_sigma(self.ctx, ptr(s)))

    def set_source(self, F, v, isrc: int = 0):
        F = _c(F, np.float64); v = _c(v, np.complex128)
        self._check(self._L.afem_set_source(self.ctx, isrc, F.shape[0], ptr(F), ptr(v)))

    def set_bounds(self, zmin, zmax, xout, yout):
        self._check(self._L.afem_set_bounds(self.ctx, zmin, zmax, xout, yout))

    def load_model(self, m, with_lines=None, sources=None):
        """Load a synthetic TidalModel (actfemtide_b200.synth) with per-land-tetrahedron conductivity."""
        if with_lines is not None:
            self.set_mesh(m.xyz, m.n4, m.tag, *with_lines)
        else:
            self.set_mesh(m.xyz, m.n4, m.tag)
        self.set_cond(m.sigma_air, m.sigma_ocean, 1, sigma_file=m.sigma_land)
        if sources is None:
            sources = [(m.F, m.v)]
        for k, (F, v) in enumerate(sources):
            self.set_source(F, v, k)
        b = m.bounds
        self.set_bounds(b["zmin"], b["zmax"], b["xout"], b["yout"])

    # ------------------------------------------------------------ assembly
    def assemble(self):
        self._check(self._L.afem_assemble(self.ctx))

    def export_system(self, freq: float, isrc: int = 0):
        """The assembled system in the reference's split layout (type global_matrix)."""
        n = C.c_int(0); tot = C.c_long(0)
        self._check(self._L.afem_export_system(self.ctx, freq, isrc, C.byref(n), C.byref(tot), *([None] * 9)))
        n, tot = n.value, tot.value
        INU = np.zeros(n + 1, np.int32); INL = np.zeros(n + 1, np.int32)
        IAU = np.zeros(tot, np.int32); IAL = np.zeros(tot, np.int32)
        D = np.zeros(n, np.complex128); AU = np.zeros(tot, np.complex128); AL = np.zeros(tot, np.complex128)
        b = np.zeros(n, np.complex128); bc = np.zeros(n, np.uint8)
        self._check(self._L.afem_export_system(self.ctx, freq, isrc, None, None, ptr(INU), ptr(IAU), ptr(INL), ptr(IAL),
                                               ptr(D), ptr(AU), ptr(AL), ptr(b), ptr(bc)))
        return dict(INU=INU, IAU=IAU, INL=INL, IAL=IAL, D=D, AU=AU, AL=AL, b=b, bc=bc)

    def export_pattern(self):
        n = C.c_int(0); tot = C.c_long(0)
        self._check(self._L.afem_export_system(self.ctx, 0.0, 0, C.byref(n), C.byref(tot), *([None] * 9)))
        n, tot = n.value, tot.value
        INU = np.zeros(n + 1, np.int32); INL = np.zeros(n + 1, np.int32)
        IAU = np.zeros(tot, np.int32); IAL = np.zeros(tot, np.int32)
        self._check(self._L.afem_export_system(self.ctx, 0.0, 0, None, None, ptr(INU), ptr(IAU), ptr(INL), ptr(IAL),
                                               None, None, None, None, None))
        return INU, IAU, INL, IAL

    # ------------------------------------------------------------ solve
    def solve(self, freqs, srcs=None, precond="SSOR", precision="fp64", tol=1e-8, maxit=100000, sigma_diag=1.0,
              check_every=0, inner_tol=0.0, use_graph=True) -> SolveResult:
        f = _c(np.atleast_1d(freqs), np.float64)
        s = None if srcs is None else _c(srcs, np.int32)
        o = SolveOpts(capi.PRECOND[precond], capi.PRECISION[precision], tol, maxit, sigma_diag, check_every, inner_tol,
                      int(use_graph))
        st = SolveStats()
        rc = self._L.afem_solve(self.ctx, len(f), ptr(f), ptr(s), C.byref(o), C.byref(st))
        res = SolveResult(st.iterations, st.refinements, st.resid_recursive, st.resid_true, st.seconds, st.status)
        if rc not in (capi.AFEM_OK, -4, -13):  # max-iter / stagnation are reported in the result
            self._check(rc)
        res.status = rc
        return res

    def cocg13_single(self, INU, IAU, INL, IAL, D, AU, AL, B, X=None, precond="IC", resid=1e-8, maxit=3000,
                      sigma_diag=1.0, sigma=0.0, nset=1):
        """COCG13_single with the reference's argument list, on the device (arrays are copied, not mutated)."""
        n = len(D)
        D = _c(D, np.complex128).copy(); AU = _c(AU, np.complex128).copy(); AL = _c(AL, np.complex128).copy()
        B = _c(B, np.complex128).copy()
        X = np.zeros(n, np.complex128) if X is None else _c(X, np.complex128).copy()
        INU = _c(INU, np.int32); IAU = _c(IAU, np.int32); INL = _c(INL, np.int32); IAL = _c(IAL, np.int32)
        R = C.c_double(resid); IT = C.c_int(maxit); ER = C.c_int(0)
        self._check(self._L.afem_cocg13_single(self.ctx, n, len(AL), len(AU), ptr(D), ptr(AL), ptr(INL), ptr(IAL),
                                               ptr(AU), ptr(INU), ptr(IAU), ptr(B), ptr(X), precond.encode(),
                                               sigma_diag, sigma, C.byref(R), C.byref(IT), C.byref(ER), nset))
        self._sizes()
        self.row_ptr = None
        return dict(x=X, resid=R.value, iter=IT.value, error=ER.value)

    def solve_rhs(self, freqs, rhs, precond="SSOR", precision="fp64", tol=1e-8, maxit=100000) -> SolveResult:
        """Solve A(freq_k) u_k = rhs[:, k] for caller right-hand sides rhs (n, nsys)."""
        f = _c(np.atleast_1d(freqs), np.float64)
        b = _c(np.asarray(rhs).reshape(self.nline, len(f)), np.complex128)
        o = SolveOpts(capi.PRECOND[precond], capi.PRECISION[precision], tol, maxit, 1.0, 0, 0.0, 1)
        st = SolveStats()
        rc = self._L.afem_solve_rhs(self.ctx, len(f), ptr(f), ptr(b), C.byref(o), C.byref(st))
        if rc not in (capi.AFEM_OK, -4, -13):
            self._check(rc)
        return SolveResult(st.iterations, st.refinements, st.resid_recursive, st.resid_true, st.seconds, rc)

    def jacobian(self, freq, x, nadj):
        """J[k, t] = d(datum k)/d log(sigma_t) from the nadj adjoint solutions of the last solve_rhs."""
        xx = _c(x, np.complex128)
        J = np.zeros((nadj, self.ntet), np.complex128)
        self._check(self._L.afem_jacobian(self.ctx, float(freq), ptr(xx), nadj, ptr(J)))
        return J

    def adjoint_sources(self, freq, sites, comps=(3, 4)):
        """Adjoint right-hand sides c with datum = c^T x for the site components (0..2 = B, 3..4 = E)."""
        item, ve, vf, _ = self.site_coeffs(sites)
        om = 2.0 * (4.0 * np.arctan(1.0)) * freq
        cols = []
        for s_ in range(len(sites)):
            for comp in comps:
                c = np.zeros(self.nline, np.complex128)
                if comp < 3:
                    c[item[s_] - 1] += vf[comp, s_]
                else:
                    c[item[s_] - 1] += -1j * om * ve[comp - 3, s_]
                cols.append(c)
        return np.stack(cols, axis=1)

    def residual(self, k: int = 0):
        """FP64 b - A x of system k after the last solve."""
        r = np.zeros(self._rows(k), np.complex128)
        self._check(self._L.afem_get_residual(self.ctx, k, ptr(r)))
        return r

    # ------------------------------------------------------------ learned preconditioner
    def mpnn_set_base(self, hybrid: bool):
        """The network's base: False -> Jacobi (a preconditioner on its own), True -> z = H(r) + N(r)."""
        self._check(self._L.afem_mpnn_set_base(self.ctx, 1 if hybrid else 0))

    def precond_apply(self, freq, r):
        """z = H(r): one application of the gradient-corrected multicolour SSOR."""
        r = _c(np.asarray(r).reshape(self.nline), np.complex128)
        z = np.zeros_like(r)
        self._check(self._L.afem_precond_apply(self.ctx, float(freq), ptr(r), ptr(z)))
        return z

    def mpnn_set_params(self, p):
        p = _c(p, np.float32)
        self._check(self._L.afem_mpnn_set_params(self.ctx, ptr(p), len(p)))

    def mpnn_get_params(self):
        p = np.zeros(self._L.afem_mpnn_nparam(), np.float32)
        self._check(self._L.afem_mpnn_get_params(self.ctx, ptr(p)))
        return p

    def mpnn_forward(self, freqs, r):
        """z = P(r); r (n,) or (n, nsys) complex."""
        f = _c(np.atleast_1d(freqs), np.float64)
        r2 = _c(np.asarray(r).reshape(self.nline, len(f)), np.complex128)
        z = np.zeros_like(r2)
        self._check(self._L.afem_mpnn_forward(self.ctx, len(f), ptr(f), ptr(r2), ptr(z)))
        return z.reshape(np.asarray(r).shape)

    def mpnn_loss_grad(self, freq, samples):
        s = _c(np.atleast_2d(samples), np.complex128)
        g = np.zeros(self._L.afem_mpnn_nparam(), np.float32)
        loss = C.c_double(0)
        self._check(self._L.afem_mpnn_loss_grad(self.ctx, float(freq), s.shape[0], ptr(s), C.byref(loss), ptr(g)))
        return loss.value, g

    def mpnn_train(self, freq, samples, steps, lr=1e-3):
        s = _c(np.atleast_2d(samples), np.complex128)
        hist = np.zeros(steps)
        self._check(self._L.afem_mpnn_train(self.ctx, float(freq), s.shape[0], ptr(s), steps, lr, ptr(hist)))
        return hist

    def solution(self, k: int = 0):
        x = np.zeros(self._rows(k), np.complex128)
        self._check(self._L.afem_get_solution(self.ctx, k, ptr(x)))
        return x

    # ------------------------------------------------------------ sites
    def _nsys(self, nsys):
        k = C.c_int(0)
        self._check(self._L.afem_solution_count(self.ctx, C.byref(k)))
        if nsys is not None and nsys != k.value:
            raise ValueError(f"the last solve holds {k.value} system(s), not {nsys}")
        return k.value

    def sites(self, xyz_obs, nsys=None):
        """Complex (nsys, 5, nobs): bx, by, bz (B = curl A), ex, ey (E = -i omega A) for every solved system."""
        o = _c(xyz_obs, np.float64)
        out = np.zeros((self._nsys(nsys), 5, o.shape[0]), np.complex128)
        self._check(self._L.afem_sites(self.ctx, o.shape[0], ptr(o), ptr(out)))
        return out

    def sites_noalloc(self, xyz_obs, nsys=None):
        """As sites(), through the entry point that allocates nothing (at most 1024 sites, 32 systems)."""
        o = _c(xyz_obs, np.float64)
        out = np.zeros((self._nsys(nsys), 5, o.shape[0]), np.complex128)
        self._check(self._L.afem_sites_noalloc(self.ctx, o.shape[0], ptr(o), ptr(out)))
        return out

    def sites_grid(self, xyz_obs, nsys=None):
        """As sites(), with PREPOBSCOEFF_XY's grid-list element search (FINDELEWITHGRID)."""
        o = _c(xyz_obs, np.float64)
        out = np.zeros((self._nsys(nsys), 5, o.shape[0]), np.complex128)
        self._check(self._L.afem_sites_grid(self.ctx, o.shape[0], ptr(o), ptr(out)))
        return out

    def site_coeffs_grid(self, xyz_obs):
        o = _c(xyz_obs, np.float64)
        nobs = o.shape[0]
        item = np.zeros((nobs, 6), np.int32); ve = np.zeros((3, nobs, 6)); vf = np.zeros((3, nobs, 6))
        iele = np.zeros(nobs, np.int32)
        self._check(self._L.afem_site_coeffs_grid(self.ctx, nobs, ptr(o), ptr(item), ptr(ve), ptr(vf), ptr(iele)))
        return item, ve, vf, iele

    def site_coeffs(self, xyz_obs):
        o = _c(xyz_obs, np.float64)
        nobs = o.shape[0]
        item = np.zeros((nobs, 6), np.int32); ve = np.zeros((3, nobs, 6)); vf = np.zeros((3, nobs, 6))
        iele = np.zeros(nobs, np.int32)
        self._check(self._L.afem_site_coeffs(self.ctx, nobs, ptr(o), ptr(item), ptr(ve), ptr(vf), ptr(iele)))
        return item, ve, vf, iele

    # ------------------------------------------------------------ measurement
    def set_wait_limit(self, polls: int):
        """Bound of the sync-free sweeps' waits in polls (0: the built-in bound)."""
        self._check(self._L.afem_set_wait_limit(self.ctx, int(polls)))

    def set_spmv_rows_per_warp(self, rpw: int):
        """Pin the SpMV variant for the same bits in every process: 1, 2, 4 rows per warp, 8 (two
        systems per lane, 16-system batches), 16 (tiles staged in shared memory, 16-system FP64
        batches); a variant that does not fit the batch falls back to 1; 0: tuned."""
        self._check(self._L.afem_set_spmv_rows_per_warp(self.ctx, int(rpw)))

    def set_profiling(self, enable: bool):
        self._check(self._L.afem_set_profiling(self.ctx, int(enable)))

    def profile(self):
        """{kernel name: (total ms, launches)} accumulated since profiling was enabled."""
        out = {}
        buf = C.create_string_buffer(64)
        for i in range(self._L.afem_profile_count(self.ctx)):
            ms = C.c_double(0); n = C.c_long(0)
            self._check(self._L.afem_profile_entry(self.ctx, i, buf, 64, C.byref(ms), C.byref(n)))
            out[buf.value.decode()] = (ms.value, n.value)
        return out

    def hybrid_matrix(self):
        """(rowptr, col, K_G, M_G) of the gradient-space correction's nodal matrix."""
        node = C.c_int(0); nnz = C.c_long(0)
        self._check(self._L.afem_hybrid_matrix(self.ctx, C.byref(node), C.byref(nnz), None, None, None))
        rp = np.zeros(node.value + 1, np.int32); col = np.zeros(nnz.value, np.int32); km = np.zeros((nnz.value, 2))
        self._check(self._L.afem_hybrid_matrix(self.ctx, None, None, ptr(rp), ptr(col), ptr(km)))
        return rp, col, km[:, 0].copy(), km[:, 1].copy()

    def stream_ptr(self) -> int:
        return int(self._L.afem_stream(self.ctx) or 0)

    # ------------------------------------------------------------ drop-in driver
    def load_ctl(self, path: str):
        self._check(self._L.afem_load_ctl(self.ctx, path.encode()))
        self._sizes()
        self.row_ptr = None

    def ctl_info(self):
        nf = C.c_int(0); no = C.c_int(0)
        self._check(self._L.afem_ctl_info(self.ctx, C.byref(nf), None, C.byref(no), None))
        f = np.zeros(nf.value); x = np.zeros((no.value, 3))
        self._check(self._L.afem_ctl_info(self.ctx, None, ptr(f), None, ptr(x)))
        return f, x

    def run_ctl(self, precond="SSOR", precision="fp64", tol=1e-8, maxit=100000):
        o = SolveOpts(capi.PRECOND[precond], capi.PRECISION[precision], tol, maxit, 1.0, 0, 0.0, 1)
        self._check(self._L.afem_run_ctl(self.ctx, C.byref(o)))


def amp_phase(c):
    """CALOBSRESP's amplitude and phase in degrees (n_ebfem_bxyz_mpi.f90:611-626)."""
    c = np.asarray(c)
    return np.sqrt(c.real ** 2 + c.imag ** 2), np.arctan2(c.imag, c.real) * (180.0 / (4.0 * np.arctan(1.0)))


@dataclass
class MTResult:
    """afem_mt_forward's outputs: be (nfreq, 2, 5, nobs) fields of the Ex / Ey polarisations
    (bx, by, bz, ex, ey), z (nfreq, 4, nobs) impedances Zxx, Zxy, Zyx, Zyy in (mV/km)/nT,
    rho / pha (nfreq, 4, nobs) apparent resistivity (Ohm m) and phase (degrees)."""
    be: np.ndarray
    z: np.ndarray
    rho: np.ndarray
    pha: np.ndarray
    solve: SolveResult


class MTForward(Forward):
    """The 3-D MT forward (src/src_3DMT/n_ebfem_3DMT.f90) over the same device context: a mesh,
    a conductivity (afem_mt_cond), frequencies and sites."""

    def set_mt_cond(self, sigma_air, condflag=1, sigma_land=None, sigma_file=None, tag_phys=None):
        self._keep = [None if a is None else _c(a, dt) for a, dt in
                      ((sigma_land, np.float64), (sigma_file, np.float64), (tag_phys, np.int32))]
        sl, sf, tg = self._keep
        self._cond = capi.MtCond(float(sigma_air), int(condflag), 0 if sl is None else len(sl),
                                 None if sl is None else sl.ctypes.data, 0 if sf is None else len(sf),
                                 None if sf is None else sf.ctypes.data, None if tg is None else tg.ctypes.data)

    def load_mt_model(self, m, with_lines=None):
        """A synthetic MT model (actfemtide_b200.synth.mt_box): mesh with physical tags, per-element sigma."""
        if with_lines is not None:
            self.set_mesh(m.xyz, m.n4, m.tag, *with_lines)
        else:
            self.set_mesh(m.xyz, m.n4, m.tag)
        self.set_mt_cond(m.sigma_air, 1, sigma_file=m.sigma_land)

    def mt_forward(self, freqs, sites, precond="HYBRID", precision="fp64", tol=1e-8, maxit=100000,
                   use_graph=True) -> MTResult:
        f = _c(np.atleast_1d(freqs), np.float64)
        o = _c(sites, np.float64)
        nf, nobs = len(f), o.shape[0]
        be = np.zeros((nf, 2, 5, nobs), np.complex128)
        z = np.zeros((nf, 4, nobs), np.complex128)
        rho = np.zeros((nf, 4, nobs)); pha = np.zeros((nf, 4, nobs))
        opts = SolveOpts(capi.PRECOND[precond], capi.PRECISION[precision], tol, maxit, 1.0, 0, 0.0, int(use_graph))
        st = SolveStats()
        rc = self._L.afem_mt_forward(self.ctx, C.byref(self._cond), nf, ptr(f), nobs, ptr(o), C.byref(opts), ptr(be),
                                     ptr(z), ptr(rho), ptr(pha), C.byref(st))
        if rc not in (capi.AFEM_OK, -4, -13):
            self._check(rc)
        res = SolveResult(st.iterations, st.refinements, st.resid_recursive, st.resid_true, st.seconds, rc)
        self._sizes()
        return MTResult(be, z, rho, pha, res)

    def mt_boundary(self, freq):
        """GENBCMT's values at freq: (av (2, nline) complex, bc (nline,) uint8)."""
        av = np.zeros((2, self.nline), np.complex128)
        bc = np.zeros(self.nline, np.uint8)
        self._check(self._L.afem_mt_boundary(self.ctx, C.byref(self._cond), float(freq), ptr(av), ptr(bc)))
        return av, bc

    def mt_face(self, j, freq):
        """The 2-D TM system of side surface j at freq in the device's band order:
        dict(line3d, A (scipy CSR), rhs, bs)."""
        import scipy.sparse as sp
        n = C.c_int(0); nnz = C.c_long(0)
        self._check(self._L.afem_mt_face(self.ctx, C.byref(self._cond), int(j), float(freq), C.byref(n),
                                         C.byref(nnz), None, None, None, None, None, None))
        n, nnz = n.value, nnz.value
        line3d = np.zeros(n, np.int32); rp = np.zeros(n + 1, np.int32); cl = np.zeros(nnz, np.int32)
        val = np.zeros(nnz, np.complex128); rhs = np.zeros(n, np.complex128); bs = np.zeros(n, np.complex128)
        self._check(self._L.afem_mt_face(self.ctx, C.byref(self._cond), int(j), float(freq), C.byref(C.c_int()),
                                         C.byref(C.c_long()), ptr(line3d), ptr(rp), ptr(cl), ptr(val), ptr(rhs),
                                         ptr(bs)))
        return dict(line3d=line3d, A=sp.csr_matrix((val, cl, rp), shape=(n, n)), rhs=rhs, bs=bs)
