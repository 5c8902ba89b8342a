/*
 * afem.h -- C ABI of libactfem_gpu.so, the B200 (sm_100a) implementation of
 * the ActFEMtide tidal forward path: assemble the complex-symmetric
 * first-order Nedelec system, solve it with COCG, evaluate E/B at sites.
 *
 * The reference is a Fortran program with no plugin layer; its seams are the
 * subroutines below.  Each entry point names the reference interface it
 * replaces.  Conventions:
 *   - node / edge / tetrahedron ids are 1-based, exactly as in the reference
 *     files and arrays; 2-D Fortran arrays are passed element-major:
 *     xyz[3*(i-1)+c] = xyz(c+1,i), n4[4*(t-1)+k] = n4(t,k+1),
 *     n6line[6*(t-1)+j] = n6line(t,j+1), line[2*(e-1)+k] = line(k+1,e).
 *   - complex numbers are interleaved doubles (re, im), i.e. C99
 *     `double _Complex` / Fortran complex(8) layout.
 *   - every call returns 0 (AFEM_OK) or a negative afem_status; the message of
 *     the last failure on a context is afem_last_error(ctx).  No call exits.
 *   - host pointers are borrowed for the duration of the call and copied;
 *     device buffers belong to the context.  One context per host thread;
 *     each context owns one CUDA stream on the device given to afem_create.
 */
#ifndef AFEM_H
#define AFEM_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct afem_ctx afem_ctx;

typedef enum afem_status {
  AFEM_OK = 0,
  AFEM_EINVAL = -1,         /* bad argument (null pointer, size, id out of range) */
  AFEM_EVOLUME = -2,        /* non-positive tetrahedron volume (m_fem_util.f90:23) */
  AFEM_EPATTERN = -3,       /* row longer than the pattern limit / dof not found */
  AFEM_EMAXITER = -4,       /* iteration cap reached (COCG13_single ERROR = -100) */
  AFEM_EBREAKDOWN = -5,     /* rho or p^T q vanished */
  AFEM_ENONFINITE = -6,     /* NaN/Inf in the iterates */
  AFEM_ECUDA = -7,          /* CUDA runtime error */
  AFEM_ESTATE = -8,         /* call out of order (e.g. solve before assemble) */
  AFEM_ETIMEOUT = -9,       /* a device wait exceeded its bound */
  AFEM_EIO = -10,           /* file could not be read or parsed */
  AFEM_ENOPRECOND = -11,    /* NSET = 0 (COCG13_single ERROR = 101) */
  AFEM_ESITE = -12,         /* a site lies outside every tetrahedron (FINDELEMENT0) */
  AFEM_ESTAGNATION = -13    /* the true residual stopped decreasing above the tolerance (the
                               solutions of the last refinement are kept) */
} afem_status;

/* Preconditioners of COCG13_single (COCG13_single.f90:107-130, 202-241). */
typedef enum afem_precond {
  AFEM_PRECOND_IC = 0,    /* diagonal-modified IC(0): DD_i = 1/(D_i*sd - sum AL_k^2 DD_col) */
  AFEM_PRECOND_SSOR = 1,  /* DD_i = 1/(sd*D_i), same forward/backward sweeps */
  AFEM_PRECOND_DIAG = 2,  /* z = DD * r */
  AFEM_PRECOND_NONE = 3,
  AFEM_PRECOND_LEARNED = 4,  /* flexible COCG with the learned network; SSOR-COCG restart when it stalls */
  AFEM_PRECOND_SSOR_MC = 5,  /* SSOR of the colour-permuted matrix: every sweep is ~10 parallel passes */
  AFEM_PRECOND_HYBRID = 6    /* multicolour SSOR plus a gradient-space correction G SSOR_node(G^T r)
                                (Hiptmair's hybrid smoother, additive); needs the mesh */
} afem_precond;

typedef enum afem_precision {
  AFEM_FP64 = 0,          /* every kernel in complex FP64 */
  AFEM_MIXED = 1,         /* inner COCG in complex FP32, FP64 iterative refinement outside */
  AFEM_FP32_PRECOND = 2   /* COCG in complex FP64 (SpMV, residuals, x, p, alpha/beta, the true-residual
                             check) with the multicolour preconditioner (SSOR_MC, HYBRID: its sweeps,
                             matrix copies, nodal correction and vectors) in complex FP32 */
} afem_precision;

typedef struct afem_solve_opts {
  int precond;            /* afem_precond */
  int precision;          /* afem_precision */
  double tol;             /* relative FP64 true residual to reach, ||b-Ax||/||b|| (1e-8) */
  int maxit;              /* total COCG iteration cap */
  double sigma_diag;      /* SIGMA_DIAG of COCG13_single (1.0) */
  int check_every;        /* iterations between host-visible convergence checks (0 = auto) */
  double inner_tol;       /* MIXED: relative reduction per refinement step (0 = auto) */
  int use_graph;          /* 1: capture the iteration loop in a CUDA graph */
} afem_solve_opts;

typedef struct afem_solve_stats {
  int iterations;         /* COCG iterations (summed over refinement steps) */
  int refinements;        /* MIXED: outer refinement steps */
  double resid_recursive; /* last recursive ||r||/||b|| */
  double resid_true;      /* FP64 ||b - A x|| / ||b|| computed on the device */
  double seconds;         /* device time of the solve */
  int status;             /* afem_status of the solve */
} afem_solve_stats;

/* ---- context -------------------------------------------------------------- */
afem_ctx *afem_create(int device);
void afem_destroy(afem_ctx *ctx);
const char *afem_last_error(const afem_ctx *ctx);
/* Device pointer of the context's stream (cudaStream_t), for callers that order work with it. */
void *afem_stream(afem_ctx *ctx);

/* ---- mesh, edges, conductivity, source ------------------------------------ */
/* Replaces READMESH_TOTAL/readmsh2 (m_mesh_type.f90:281-468) + READLINE
 * (m_line_type.f90:28-48): the em3d.msh tetrahedra with their elementary tag
 * (n4flag(:,2)) and the lineinfo.dat edge list.  line/n6line may be NULL
 * (nline = 0): the edge numbering of MKLINE_V2/MKN6 (tmtgem/common/
 * m_line_type.f90:120-277) is then built on the device. */
int afem_set_mesh(afem_ctx *ctx, int node, const double *xyz, int ntet, const int32_t *n4, const int32_t *tag,
                  int nline, const int32_t *line, const int32_t *n6line);
/* Sizes of the loaded mesh (any pointer may be NULL). */
int afem_mesh_info(afem_ctx *ctx, int *node, int *ntet, int *nline);
/* Systems held by the last solve (afem_sites writes 5*nobs values for each). */
int afem_solution_count(afem_ctx *ctx, int *nsys);
/* Number of edges and the numbering in use (line: 2*nline, n6line: 6*ntet; either may be NULL). */
int afem_get_lines(afem_ctx *ctx, int *nline, int32_t *line, int32_t *n6line);

/* Packed batch of independent meshes (no counterpart in the reference, which
 * runs one mesh per process).  After afem_set_mesh of the union of nseg
 * meshes, with mesh k owning the 1-based node ids node_ptr[k]+1 ..
 * node_ptr[k+1] (node_ptr[0] = 0, node_ptr[nseg] = node) and the
 * tetrahedra grouped mesh by mesh, this declares the meshes.  The edge
 * numbering of the union then runs mesh by mesh as well.  A later
 * afem_solve takes nsys = nseg: system k is mesh k at freq_hz[k] with
 * source src[k], with its own COCG scalars and convergence test, all meshes
 * in one launch sequence.  afem_get_solution / afem_get_residual return
 * the rows of mesh k only, and afem_sites searches system k's sites in
 * mesh k's tetrahedra.  nseg <= 32; nseg = 0 removes the declaration
 * (so does afem_set_mesh). */
int afem_set_segments(afem_ctx *ctx, int nseg, const int32_t *node_ptr);
/* The declared meshes: *nseg, and the row (edge) and tetrahedron ranges, 0-based prefixes
 * row_ptr[nseg+1], tet_ptr[nseg+1] (either may be NULL). */
int afem_segment_info(afem_ctx *ctx, int *nseg, int32_t *row_ptr, int32_t *tet_ptr);

/* Replaces param_cond + SETNPHYS1INDEX2COND + READCOND (m_param.f90:449-485,
 * n_ebfem_bxyz_mpi.f90:470-527) and GENMAT's selection (forward_bxyz_mpi.f90:196-208):
 * tag 1 -> sigma_air, tag 2 -> sigma_ocean (the reference hard-codes 3.33),
 * tag j >= 3 -> sigma_land[j-2] (condflag 0, sigma_land(j-1) in Fortran) or
 * sigma_file[t-nphys1-1] for 1-based tetrahedron t (condflag 1, nphys2 values). */
int afem_set_cond(afem_ctx *ctx, double sigma_air, double sigma_ocean, int condflag, int nvolume,
                  const double *sigma_land, int nphys2, const double *sigma_file);
/* Direct per-tetrahedron conductivity override (ntet values, S/m). */
int afem_set_sigma(afem_ctx *ctx, const double *sigma_tet);

/* Replaces readfxyz/readvxyz (m_readfvxyz.f90:7-62): F (3*nodes, nT) and
 * v (3*nodes complex, m/s) for mesh nodes 1..nodes; later nodes are zero.
 * Several source patterns may be set (isrc = 0..), each one RHS column. */
int afem_set_source(afem_ctx *ctx, int isrc, int nodes, const double *F, const double *v_complex);

/* Replaces the bounds forward_bxyz passes to GENBCCSEM (forward_bxyz_mpi.f90:34-37,
 * 467-519): zmin = zbound(1), zmax = zbound(4), xout = xbound(4), yout = ybound(4). */
int afem_set_bounds(afem_ctx *ctx, double zmin, double zmax, double xout, double yout);

/* ---- assembly ------------------------------------------------------------- */
/* Replaces set_iccg_var7_dofn (m_iccg_var_takuto.f90:277-359) and, per call,
 * INITIALIZE + GENMAT + COPY_UL_ICCG12 + GENBCCSEM + SET_BC_ICCG
 * (forward_bxyz_mpi.f90:46-58).  The device keeps K (curl-curl) and
 * M (sigma-weighted mass * mu0 * L0^2) so that A(omega) = K + i*omega*M
 * serves every frequency without re-assembly. */
int afem_assemble(afem_ctx *ctx);

/* Export the assembled system for one frequency in the reference's split
 * layout (type global_matrix, m_iccg_var_takuto.f90:9-18): INU/INL (n+1,
 * INU[0] = 0), IAU/IAL 1-based columns, complex D (n), AU/AL (iau_tot),
 * b (n, source isrc).  Any pointer may be NULL.  *n and *iau_tot receive sizes. */
int afem_export_system(afem_ctx *ctx, double freq_hz, int isrc, int *n, long *iau_tot, int32_t *INU, int32_t *IAU,
                       int32_t *INL, int32_t *IAL, double *D, double *AU, double *AL, double *b, uint8_t *bc);

/* ---- solve ---------------------------------------------------------------- */
/* Replaces solveCG -> COCG13_single (forward_bxyz_mpi.f90:70-94,
 * COCG13_single.f90:9-340) and, as the production solver, solvePARDISO
 * (forward_bxyz_mpi.f90:63).  Solves nsys systems A(freq[k]) x_k = b_{src[k]}
 * in one batched launch sequence; src may be NULL (all source 0).  Solutions
 * stay on the device (afem_get_solution copies them out). */
int afem_solve(afem_ctx *ctx, int nsys, const double *freq_hz, const int *src, const afem_solve_opts *opts,
               afem_solve_stats *stats);
/* The solver seam with the reference's own argument list: COCG13_single
 * (src/solver/COCG13_single.f90:9-12) on the device.  D/AL/AU/B/X complex
 * (interleaved), INL/INU (0:NP) prefix arrays, IAL/IAU 1-based columns;
 * PRECOND "IC" / "SSOR" / "DIAG" (anything else: none); X is the initial
 * guess and the solution; RESID in: tolerance on the recursive residual,
 * out: reached value; ITER in: MAXIT, out: iterations (MAXIT+1 at the cap,
 * as the Fortran loop variable); ERROR 0, 101 (NSET = 0) or -100 (cap).
 * NSET = 2 scales D/AL/AU/B in place as the reference does.  IC with
 * SIGMA != 0 is rejected (AFEM_EINVAL).  Returns an afem_status. */
int afem_cocg13_single(afem_ctx *ctx, int NP, int NPL, int NPU, double *D, double *AL, const int32_t *INL,
                       const int32_t *IAL, double *AU, const int32_t *INU, const int32_t *IAU, double *B, double *X,
                       const char *PRECOND, double SIGMA_DIAG, double SIGMA, double *RESID, int *ITER, int *ERROR,
                       int NSET);
/* Bound of the waits in the sync-free triangular sweeps (IC, SSOR, DIAG set-up
 * and sweeps in natural row order; COCG13_single's sweeps are serial, so the
 * reference has no counterpart): after `polls` back-off polls (32 ns doubling to
 * 1 us) on a row the sweep depends on, the kernel records a timeout, every
 * waiting row gives up, and the solve returns AFEM_ETIMEOUT with the context
 * still usable.  0 restores the built-in bound (2^21 polls, about 2 s). */
int afem_set_wait_limit(afem_ctx *ctx, unsigned polls);
/* Pin the SpMV variant: rows per warp 1, 2 or 4; 8 = two systems per lane and four
 * rows per warp (16-system batches); 16 = tiles of 32 rows whose distinct p rows are
 * staged in shared memory (16-system FP64 batches).  A value that does not fit the
 * batch falls back to 1; 0: the autotuner picks per pattern by timing.  The choice sets how a row's products are split over lanes and so
 * the order of the floating-point additions: with the tuner, two processes may
 * pick different variants and their results differ in the last bits; a pinned
 * value gives the same bits in every process.  No counterpart in the reference. */
int afem_set_spmv_rows_per_warp(afem_ctx *ctx, int rows_per_warp);
/* Load a system in the same split layout for afem_solve (freq_hz = 1/(2*pi) gives A itself). */
int afem_set_system(afem_ctx *ctx, int n, const int32_t *INU, const int32_t *IAU, const int32_t *INL,
                    const int32_t *IAL, const double *D, const double *AU, const double *AL, const double *b);
/* afem_solve with caller right-hand sides rhs[(row*nsys + k)] (complex), e.g. adjoint
 * sources P^T of site data (src/src_inv/solvePARDISOinv.f90:154-196). */
int afem_solve_rhs(afem_ctx *ctx, int nsys, const double *freq_hz, const double *rhs, const afem_solve_opts *opts,
                   afem_solve_stats *stats);
/* Sensitivities of nadj site data to log(sigma) of every tetrahedron (m_jacobian.f90:120-218):
 * after afem_solve_rhs solved the nadj adjoint systems A u_k = c_k at freq_hz,
 * J[k*ntet + t] = -u_k^T (dA/dlog sigma_t) x for the forward solution x (n complex). */
int afem_jacobian(afem_ctx *ctx, double freq_hz, const double *x_complex, int nadj, double *J_complex);
/* FP64 true residual b - A x of system k after the last afem_solve (n complex values). */
int afem_get_residual(afem_ctx *ctx, int k, double *r_complex);
/* Solution of system k (n complex values, [nT*km] like bs in forward_bxyz; a packed batch: the rows of mesh k). */
int afem_get_solution(afem_ctx *ctx, int k, double *x_complex);

/* ---- sites ---------------------------------------------------------------- */
/* Replaces PREPOBSCOEFF (n_ebfem_bxyz_mpi.f90:653-726, FINDELEMENT0 +
 * EDGEBASISFUN/FACEBASISFUN) and CALOBSEBCOMP/CALOBSRESP (:397-423, :570-626)
 * with the primary field 0: for each solved system k and site s,
 * out[(k*5 + c)*nobs + s] for c = bx, by, bz (B = curl A) and ex, ey
 * (E = -i*omega*A), complex. */
int afem_sites(afem_ctx *ctx, int nobs, const double *xyz_obs, double *out_complex);
/* afem_sites without any device or host allocation (no counterpart in the
 * reference): the same kernels and results as afem_sites, with the device
 * buffers in one fixed, statically allocated scratch array of 2.9 MB, so at
 * most 1024 sites per call and 32 solved systems (AFEM_EINVAL above that) and
 * no packed batches.  The first call on a device looks the scratch up
 * (cudaGetSymbolAddress); make that first call before any stream capture.
 * The scratch is shared by every context on the device: calls that overlap in
 * time (from two host threads or two contexts) race on it. */
int afem_sites_noalloc(afem_ctx *ctx, int nobs, const double *xyz_obs, double *out_complex);
/* The site coefficient rows (item: 6*nobs 1-based edge ids ascending; val_e, val_f: 3*nobs*6,
 * [(c*nobs + s)*6 + j]; iele: containing tetrahedron) for parity checks. */
int afem_site_coeffs(afem_ctx *ctx, int nobs, const double *xyz_obs, int32_t *item, double *val_e, double *val_f,
                     int32_t *iele);

/* The same with the element search of PREPOBSCOEFF_XY / CALCOEFF_LINE: FINDELEWITHGRID
 * (m_mesh_type.f90:204-277) over the grid list of gengridforlist / classifyelement2grd
 * (300 x 300 x 50 boxes over the node extent +-1 km, tetrahedra sorted by the box of
 * their centroid with SORT_INDEX): the first tetrahedron holding the site in the
 * list's search order.  Sites whose tetrahedron lies more than 64 box shells away
 * are reported as outside the mesh (AFEM_ESITE). */
int afem_sites_grid(afem_ctx *ctx, int nobs, const double *xyz_obs, double *out_complex);
int afem_site_coeffs_grid(afem_ctx *ctx, int nobs, const double *xyz_obs, int32_t *item, double *val_e,
                          double *val_f, int32_t *iele);
/* Host only: SORT_INDEX (src/solver/sort_index.f90:13-56), the heapsort that orders the
 * grid list: ra ascending, na carried along (equal keys in the heapsort's own order). */
int afem_sort_index(int n, int32_t *na, double *ra);
/* Host only: the plan-view points of PREPOBSCOEFF_XY (n_ebfem_bxyz_mpi.f90:769-784),
 * nx*ny cell centres over [xmin,xmax]x[ymin,ymax] at depth z, point (j-1)*ny + i
 * for x cell j and y cell i; xyz holds 3*nx*ny values. */
int afem_xy_points(double xmin, double xmax, double ymin, double ymax, int nx, int ny, double z, double *xyz);

/* ---- learned preconditioner (no counterpart in the reference) ---------------- */
/* A message-passing network over the matrix graph (6 layers, width 48, BF16
 * weights, FP32 accumulation) that maps a residual r to z ~ A^-1 r; used by
 * afem_solve with AFEM_PRECOND_LEARNED inside flexible COCG.  Parameters are
 * one flat FP32 vector of afem_mpnn_nparam() values (W_in 8x48, then per
 * layer W 144x48 and c 48, then W_out 48x2, all row-major). */
int afem_mpnn_nparam(void);
int afem_mpnn_set_params(afem_ctx *ctx, const float *params, int nparam);
int afem_mpnn_get_params(afem_ctx *ctx, float *params);
/* The network's base: 0 (default) z = r/|A_ii| + correction, a preconditioner on its
 * own; 1: z = H(r) + correction with H the gradient-corrected multicolour SSOR
 * (AFEM_PRECOND_HYBRID), so the network learns what H leaves; inside afem_solve the
 * fallback on a stall is then H.  Training and afem_mpnn_forward follow the base. */
int afem_mpnn_set_base(afem_ctx *ctx, int base);
/* z = H(r), one application of the gradient-corrected multicolour SSOR to n complex values
 * of the assembled system at freq_hz (the learned base; also for tests). */
int afem_precond_apply(afem_ctx *ctx, double freq_hz, const double *r, double *z);
/* z = P(r) for nsys systems at freq[k]; r, z: [row][system] interleaved complex. */
int afem_mpnn_forward(afem_ctx *ctx, int nsys, const double *freq, const double *r, double *z);
/* Sum over nsamp residuals (each n complex values) of ||A P(r) - r||^2/||r||^2 and its gradient. */
int afem_mpnn_loss_grad(afem_ctx *ctx, double freq_hz, int nsamp, const double *r, double *loss, float *grad);
/* steps Adam updates (lr) on the mean loss over the samples; hist[steps] receives the loss per step. */
int afem_mpnn_train(afem_ctx *ctx, double freq_hz, int nsamp, const double *r, int steps, float lr, double *hist);

/* ---- measurement (no counterpart in the reference, which only prints banners) -- */
/* Accumulate per-kernel device time (CUDA events on the context's stream)
 * while enabled; enabling or disabling clears the table. */
int afem_set_profiling(afem_ctx *ctx, int enable);
int afem_profile_count(afem_ctx *ctx);
/* Entry i: kernel name, total milliseconds, launches. */
int afem_profile_entry(afem_ctx *ctx, int i, char *name, int cap, double *ms, long *launches);

/* The nodal matrix of the gradient-space correction (AFEM_PRECOND_HYBRID) for the
 * assembled system: A_G = G^T P A P G with G the edge-node incidence (+1 at
 * line(2,e), -1 at line(1,e)) and P dropping the Dirichlet edges, split as
 * (K_G, M_G) pairs per entry like A (km: 2*nnz doubles); rowptr[node+1] and
 * 0-based ascending col[nnz] over the node graph.  Any pointer may be NULL.
 * No counterpart in the reference. */
int afem_hybrid_matrix(afem_ctx *ctx, int *node, long *nnz, int32_t *rowptr, int32_t *col, double *km);

/* Kernels this library has launched in this process (each kernel of a CUDA
 * graph launch counts once per launch).  Host only. */
long afem_launch_count(void);

/* Host only: the triangular-sweep schedules of a CSR pattern (0-based columns
 * ascending, diagonal included): rows sorted by dependency level of the
 * forward (lower) and backward (upper) sweeps; the sweep kernels visit rows
 * in these orders.  No counterpart in the reference (its sweeps are serial). */
int afem_sweep_schedule(int n, const int32_t *rowptr, const int32_t *col, const int32_t *diagpos, int32_t *perm_f,
                        int32_t *perm_b, int *levels_f, int *levels_b);

/* Host only: greedy distance-1 colouring of a CSR pattern; color[n], perm[n]
 * (rows sorted by colour), cptr[ncolors+1] (cptr must hold 256).  Returns ncolors. */
int afem_coloring(int n, const int32_t *rowptr, const int32_t *col, uint8_t *color, int32_t *perm, int32_t *cptr);

/* ---- 3-D MT forward ------------------------------------------------------------ */
/* Conductivity of the MT forward as READPARAM_MT + SETNPHYS1INDEX2COND deliver it
 * (src/src_3DMT/m_param_mt.f90, n_ebfem_3DMT.f90:291-340).  The 3-D system uses
 * GENMAT_MT's selection (forward_3DMT.f90:239-252): tags 1 and 2 -> sigma_air,
 * tag j >= 3 -> sigma_land[j-2] (condflag 0) or sigma_file[t-nphys1-1] for 1-based
 * tetrahedron t (condflag 1, nphys2 values, the land tetrahedra last).  The 2-D
 * side faces use COND3DTO2D's (src/src_2D/m_surface_type.f90:76-120): tag 1 ->
 * sigma_air, tag 2 -> 3.31 (a default-real literal there), tag >= 3 ->
 * sigma_land[0] or the file value of the triangle's tetrahedron. */
typedef struct afem_mt_cond {
  double sigma_air;
  int condflag;               /* 0: per tag, 1: per element */
  int nvolume;                /* entries of sigma_land (condflag 0) */
  const double *sigma_land;
  int nphys2;                 /* entries of sigma_file (condflag 1): the tetrahedra with tag >= 3 */
  const double *sigma_file;
  const int32_t *tag_phys;    /* physical tags n4flag(:,1), ntet values; NULL: the tags of afem_set_mesh */
} afem_mt_cond;

/* Replaces the frequency loop of program ebfem_3DMT (src/src_3DMT/n_ebfem_3DMT.f90:85-113):
 * per frequency the 2-D TM boundary solves of the four side faces (forward_2DTM,
 * src/src_2D/forward_2DTM.f90:17-170; a banded LDL^T on the device in place of PARDISO),
 * GENBCMT + GENMAT_MT + SET_BC_3DJoint (forward_3DMT.f90:5-88, 92-177, 553-623), the solve of
 * the Ex and Ey polarisations of every frequency in batches (in place of solvePARDISO),
 * CALOBSEBCOMP at the sites and CALRESPMT (n_ebfem_3DMT.f90:179-237).  Outputs (any may be
 * NULL): be[((f*2 + pol)*5 + c)*nobs + s] complex (c = bx, by, bz, ex, ey; pol 0 = Ex
 * source, 1 = Ey), z[(f*4 + k)*nobs + s] complex (k = xx, xy, yx, yy, Z = E B^-1 in
 * (mV/km)/nT), rho[(f*4 + k)*nobs + s] (Ohm m) and pha[...] (degrees).  The context's
 * conductivity, matrix and right-hand sides become the MT ones (column 2f+pol is frequency
 * f, polarisation pol; afem_export_system shows them); the last batch's solutions stay for
 * afem_get_solution.  stats: iterations summed over the batches, worst residuals. */
int afem_mt_forward(afem_ctx *ctx, const afem_mt_cond *cond, int nfreq, const double *freq_hz, int nobs,
                    const double *xyz_obs, const afem_solve_opts *opts, double *be_complex, double *z_complex,
                    double *rho, double *pha, afem_solve_stats *stats);
/* GENBCMT's Dirichlet values at one frequency after the four 2-D solves (for parity checks):
 * av[pol*nline + i] complex (Avalue_bc(i, pol+1)), bc[nline] (line_bc(:,1)).  Either may be NULL. */
int afem_mt_boundary(afem_ctx *ctx, const afem_mt_cond *cond, double freq_hz, double *av_complex, uint8_t *bc);
/* The 2-D TM system of side surface j (2 north, 3 west, 4 south, 5 east) at one frequency,
 * after GENBC2D + SET_BC_ICCG, over the surface's lines in the device's band order:
 * line3d[n] (1-based 3-D line ids), full CSR rowptr[n+1] / col[nnz] (0-based, ascending) /
 * val[nnz] complex, rhs[n] complex and the solution bs[n] complex.  Call with line3d NULL to
 * get *n and *nnz only.  (GENMAT2DTM, forward_2DTM.f90:253-363.) */
int afem_mt_face(afem_ctx *ctx, const afem_mt_cond *cond, int j, double freq_hz, int *n, long *nnz,
                 int32_t *line3d, int32_t *rowptr, int32_t *col, double *val_complex, double *rhs_complex,
                 double *bs_complex);

/* ---- drop-in driver --------------------------------------------------------- */
/* Replaces the rank-0 input stage of program n_ebfem_bxyz (n_ebfem_bxyz_mpi.f90:55-90):
 * reads the forward ctl file (readcontrolfile + readparam, m_param.f90:145-446,
 * 939-999) and every file it names (mesh, polygonz surface, lineinfo, ocean
 * mesh node count, vxyz/fxyz, cond file), lifts the sites onto the surface
 * (PREPZSRCOBS, n_ebfem_bxyz_mpi.f90:937-1030) and loads it all. */
int afem_load_ctl(afem_ctx *ctx, const char *ctl_path);
/* Frequencies and sites from the last afem_load_ctl (either pointer may be NULL). */
int afem_ctl_info(afem_ctx *ctx, int *nfreq, double *freq, int *nobs, double *xyz_obs);
/* Run every frequency of the loaded ctl and write <outputfolder><site>_<src>.dat
 * exactly as OUTOBSFILESFWD (m_outresp.f90:221-262). */
int afem_run_ctl(afem_ctx *ctx, const afem_solve_opts *opts);
/* Host only: a site's position in km east and north of the origin (lonorigin,
 * latorigin), both projected to UTM zone `zone` (1..60): UTMXY + UTMGMT +
 * utm_geo_tm (src/common/m_param.f90:609-661, 741-936), which readparam applies
 * to lonlatflag-1 sites (m_param.f90:316-323).  xy_km[2]. */
int afem_utm_xy(double lon, double lat, double lonorigin, double latorigin, int zone, double *xy_km);
/* Fortran Gw.d formatting of x as OUTOBSFILESFWD writes it ('(11g15.7)'); host only. */
int afem_fortran_g(double x, int w, int d, char *out, int cap);

#ifdef __cplusplus
}
#endif
#endif /* AFEM_H */
