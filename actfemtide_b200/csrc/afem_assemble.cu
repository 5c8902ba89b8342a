// Element assembly: GENMAT + COPY_UL_ICCG12 + GENBCCSEM + SET_BC_ICCG on the device.
//
// Reference: src/solver_mpi/forward_bxyz_mpi.f90:99-311 (GENMAT), :467-519
// (GENBCCSEM), :567-636 (SET_BC_ICCG), :642-699 (sup_iccg), and
// src/solver/m_iccg_var_takuto.f90:107-167 (COPY_UL_ICCG12).
//
// Instead of scattering 36 element entries per tetrahedron with a linear
// row search (sup_iccg), every matrix row -- one edge -- gathers the
// contributions of the tetrahedra around it in ascending tetrahedron id, the
// order in which the serial element loop adds them.  Each value is written
// once, no atomics are needed, and the upper and lower halves come out
// mirrored by construction (the reference mirrors them in COPY_UL_ICCG12).
// For an entry (e, c) with local edges (a, b) the element value taken is
// elm_k(max(a,b), min(a,b)), the one sup_iccg adds for the pair.
//
// Storage is frequency independent: K = curl-curl (real) and
// M = sigma-weighted mass * mu0 * L0^2 (real), A(omega) = K + i*omega*M.
// This file is compiled with -fmad=false so that every product and sum rounds
// separately, as in the reference's AVX (no FMA) build.
#include "afem_internal.h"

namespace afem {

namespace {

constexpr int MAXSRC = 16;

struct SrcArgs {
  int nsrc;
  int nodes[MAXSRC];
  const double* F[MAXSRC];
  const double2* v[MAXSRC];
};

__constant__ int c_kl[6][2] = {{1, 2}, {2, 3}, {1, 3}, {1, 4}, {2, 4}, {3, 4}};

struct V3 {
  double x, y, z;
};
__device__ __forceinline__ V3 vsub(const V3& a, const V3& b) { return V3{a.x - b.x, a.y - b.y, a.z - b.z}; }
__device__ __forceinline__ V3 vneg(const V3& a) { return V3{-a.x, -a.y, -a.z}; }
__device__ __forceinline__ V3 vouter(const V3& a, const V3& b) {
  return V3{a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x};
}
__device__ __forceinline__ double vinner(const V3& a, const V3& b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
__device__ __forceinline__ V3 vscale(double c, const V3& a) { return V3{c * a.x, c * a.y, c * a.z}; }
__device__ __forceinline__ double intv(int k, int m, double v) { return (k != m) ? v / 20.0 : v / 10.0; }

// GENBCCSEM (forward_bxyz_mpi.f90:483-511)
__global__ void k_bc_flags(const int32_t* __restrict__ line, const double* __restrict__ xyz, int nline, double zmin,
                           double zmax, double xout, double yout, uint8_t* __restrict__ bc) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= nline) return;
  const double xout1 = xout - 1.0, yout1 = yout - 1.0, zmin1 = zmin + 1.0, zmax1 = zmax - 1.0;
  const double* p1 = xyz + 3L * (line[2L * i] - 1);
  const double* p2 = xyz + 3L * (line[2L * i + 1] - 1);
  const double x1 = p1[0], y1 = p1[1], z1 = p1[2], x2 = p2[0], y2 = p2[1], z2 = p2[2];
  int g = 0;
  if (x1 <= -xout1 && x2 <= -xout1) g = 3;
  else if (x1 >= xout1 && x2 >= xout1) g = 5;
  else if (y1 <= -yout1 && y2 <= -yout1) g = 4;
  else if (y1 >= yout1 && y2 >= yout1) g = 2;
  else if (z1 <= zmin1 && z2 <= zmin1) g = 6;
  else if (z1 >= zmax1 && z2 >= zmax1) g = 1;
  bc[i] = (g != 0);
}

__device__ __forceinline__ int find_slot(const int32_t* __restrict__ col, int r0, int r1, int c) {
  int lo = r0, hi = r1;
  while (lo < hi) {
    int mid = (lo + hi) >> 1;
    if (__ldg(col + mid) < c) lo = mid + 1;
    else hi = mid;
  }
  return (lo < r1 && __ldg(col + lo) == c) ? lo - r0 : -1;
}

// One thread per row (edge).  Accumulators live in local memory (ROW_MAX slots).
__global__ void __launch_bounds__(128)
    k_assemble_rows(const double* __restrict__ xyz, const int32_t* __restrict__ n4, const int32_t* __restrict__ tag,
                    const int32_t* __restrict__ n6line, const double* __restrict__ sigma,
                    const int32_t* __restrict__ etp, const int32_t* __restrict__ etl,
                    const int32_t* __restrict__ rowptr, const int32_t* __restrict__ col,
                    const uint8_t* __restrict__ bc, int nline, SrcArgs src, double2* __restrict__ km,
                    double2* __restrict__ rhs, DevStatus* st) {
  const int e = blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= nline) return;
  const double pi = 4.0 * atan(1.0);
  const double dmu = 4.0 * pi * 1.0e-7;
  const double L0 = 1.0e3;
  const int r0 = rowptr[e], r1 = rowptr[e + 1];
  const int len = r1 - r0;
  if (len > ROW_MAX) {
    raise_status(st, DEV_ROWLEN, e);
    return;
  }
  double accK[ROW_MAX], accM[ROW_MAX];
  for (int s = 0; s < len; ++s) { accK[s] = 0.0; accM[s] = 0.0; }
  double2 acc_b[MAXSRC];
  for (int s = 0; s < src.nsrc; ++s) acc_b[s] = make_double2(0.0, 0.0);

  for (int q = etp[e]; q < etp[e + 1]; ++q) {
    const int code = etl[q];
    const long t = code >> 3;
    const int a = code & 7;  // local edge of this row in tetrahedron t
    V3 p[4];
    int nd[4];
    for (int j = 0; j < 4; ++j) {
      nd[j] = n4[4 * t + j];
      const double* P = xyz + 3L * (nd[j] - 1);
      p[j] = V3{P[0], P[1], P[2]};
    }
    int gl[6], d[6];
    for (int j = 0; j < 6; ++j) {
      const int s6 = n6line[6 * t + j];
      d[j] = (s6 < 0) ? -1 : 1;
      gl[j] = (s6 < 0) ? -s6 : s6;
    }
    // calxmn (m_fem_util.f90:42-53)
    V3 xx[6];
    xx[0] = vsub(p[3], p[2]);
    xx[1] = vsub(p[3], p[0]);
    xx[2] = vsub(p[1], p[3]);
    xx[3] = vsub(p[2], p[1]);
    xx[4] = vsub(p[0], p[2]);
    xx[5] = vsub(p[1], p[0]);
    // gradnodebasisfun (m_fem_util.f90:12-40)
    const double vol = 1.0 / 6.0 * vinner(vouter(xx[0], xx[4]), vneg(xx[3]));
    if (!(vol > 0.0)) {
      raise_status(st, DEV_VOLUME, (int)t);
      continue;
    }
    const double cg = 1.0 / 6.0 / vol;
    V3 gn[4];
    gn[0] = vscale(cg, vouter(vsub(p[3], p[1]), vsub(p[2], p[1])));
    gn[1] = vscale(cg, vouter(vsub(p[2], p[0]), vsub(p[3], p[0])));
    gn[2] = vscale(cg, vouter(vsub(p[3], p[0]), vsub(p[1], p[0])));
    gn[3] = vscale(cg, vouter(vsub(p[1], p[0]), vsub(p[2], p[0])));
    const double AA = 1.0 / 9.0 / vol;
    const double sg = sigma[t];
    const double ms = dmu * sg * L0 * L0;
    for (int b = 0; b < 6; ++b) {
      const int i = (a > b) ? a : b, j = (a > b) ? b : a;  // elm_k(max, min)
      const double kv = vinner(xx[i], xx[j]) * d[i] * d[j] * AA;
      const int k = c_kl[i][0], l = c_kl[i][1], m = c_kl[j][0], n = c_kl[j][1];
      const double yy = intv(k, m, vol) * vinner(gn[l - 1], gn[n - 1]) - intv(k, n, vol) * vinner(gn[l - 1], gn[m - 1]) -
                        intv(l, m, vol) * vinner(gn[k - 1], gn[n - 1]) + intv(l, n, vol) * vinner(gn[k - 1], gn[m - 1]);
      const double mv = yy * d[i] * d[j] * ms;
      const int slot = find_slot(col, r0, r1, gl[b] - 1);
      if (slot < 0) {
        raise_status(st, DEV_NOTFOUND, e);
        continue;
      }
      accK[slot] += kv;
      accM[slot] += mv;
    }
    // right-hand side, ocean tetrahedra only (forward_bxyz_mpi.f90:267-299)
    if (tag[t] == 2) {
      const int k = c_kl[a][0], l = c_kl[a][1];
      for (int s = 0; s < src.nsrc; ++s) {
        double2 S2 = make_double2(0.0, 0.0);
        for (int jn = 1; jn <= 4; ++jn) {
          const int no = nd[jn - 1];
          double Fv[3] = {0.0, 0.0, 0.0};
          double2 vv[3] = {make_double2(0.0, 0.0), make_double2(0.0, 0.0), make_double2(0.0, 0.0)};
          if (no <= src.nodes[s]) {
            for (int cc = 0; cc < 3; ++cc) {
              Fv[cc] = src.F[s][3L * (no - 1) + cc];
              vv[cc] = src.v[s][3L * (no - 1) + cc];
            }
          }
          // cr_outer (m_outerinnerproduct.f90:52-60)
          double2 vF[3];
          vF[0] = make_double2(vv[1].x * Fv[2] - vv[2].x * Fv[1], vv[1].y * Fv[2] - vv[2].y * Fv[1]);
          vF[1] = make_double2(vv[2].x * Fv[0] - vv[0].x * Fv[2], vv[2].y * Fv[0] - vv[0].y * Fv[2]);
          vF[2] = make_double2(vv[0].x * Fv[1] - vv[1].x * Fv[0], vv[0].y * Fv[1] - vv[1].y * Fv[0]);
          // rc_inner (m_outerinnerproduct.f90:78-84)
          const V3& gL = gn[l - 1];
          const V3& gK = gn[k - 1];
          const double2 rl = make_double2(gL.x * vF[0].x + gL.y * vF[1].x + gL.z * vF[2].x,
                                          gL.x * vF[0].y + gL.y * vF[1].y + gL.z * vF[2].y);
          const double2 rk = make_double2(gK.x * vF[0].x + gK.y * vF[1].x + gK.z * vF[2].x,
                                          gK.x * vF[0].y + gK.y * vF[1].y + gK.z * vF[2].y);
          const double ik = intv(k, jn, vol), il = intv(l, jn, vol);
          const double2 tm = make_double2(ik * rl.x - il * rk.x, ik * rl.y - il * rk.y);
          const double c0 = dmu * sg;
          double2 term = make_double2(c0 * tm.x, c0 * tm.y);
          term = make_double2(term.x * (double)d[a], term.y * (double)d[a]);
          term = make_double2(term.x * 1.0e3, term.y * 1.0e3);
          S2 = make_double2(S2.x + term.x, S2.y + term.y);
        }
        acc_b[s] = make_double2(acc_b[s].x + S2.x, acc_b[s].y + S2.y);
      }
    }
  }
  // SET_BC_ICCG with Dirichlet value 0 (forward_bxyz_mpi.f90:592-633)
  const bool dir_row = bc[e] != 0;
  for (int s = 0; s < len; ++s) {
    const int c = col[r0 + s];
    double kv = accK[s], mv = accM[s];
    if (dir_row) {
      kv = (c == e) ? 1.0 : 0.0;
      mv = 0.0;
    } else if (bc[c]) {
      kv = 0.0;
      mv = 0.0;
    }
    km[r0 + s] = make_double2(kv, mv);
  }
  for (int s = 0; s < src.nsrc; ++s) rhs[(long)s * nline + e] = dir_row ? make_double2(0.0, 0.0) : acc_b[s];
}

}  // namespace

void assemble_device(afem_ctx* c) {
  AFEM_REQUIRE(c->pattern_ready, AFEM_ESTATE, "assemble: pattern not built");
  AFEM_REQUIRE(c->sigma_set, AFEM_ESTATE, "assemble: conductivity not set");
  AFEM_REQUIRE(c->bounds_set, AFEM_ESTATE, "assemble: Dirichlet bounds not set");
  AFEM_REQUIRE(!c->src.empty(), AFEM_ESTATE, "assemble: no tidal source set");
  AFEM_REQUIRE((int)c->src.size() <= MAXSRC, AFEM_EINVAL, "assemble: at most 16 source patterns");
  cudaStream_t s = c->stream;
  c->bc.alloc(c->nline);
  k_bc_flags<<<(c->nline + 255) / 256, 256, 0, s>>>(c->line.p, c->xyz.p, c->nline, c->zmin, c->zmax, c->xout, c->yout,
                                                  c->bc.p);
  count_launch();
  SrcArgs sa{};
  sa.nsrc = (int)c->src.size();
  for (int i = 0; i < sa.nsrc; ++i) {
    AFEM_REQUIRE(c->src[i] != nullptr, AFEM_ESTATE, "assemble: source patterns must be numbered 0..nsrc-1");
    sa.nodes[i] = c->src[i]->nodes;
    sa.F[i] = c->src[i]->F.p;
    sa.v[i] = c->src[i]->v.p;
  }
  c->km.alloc(c->nnz);
  c->rhs.alloc((size_t)c->nline * sa.nsrc);
  c->rhs_nsrc = sa.nsrc;
  cudaEvent_t e0 = nullptr, e1 = nullptr;
  if (c->prof.on) {
    AFEM_CUDA(cudaEventCreate(&e0));
    AFEM_CUDA(cudaEventCreate(&e1));
    AFEM_CUDA(cudaEventRecord(e0, s));
  }
  k_assemble_rows<<<(c->nline + 127) / 128, 128, 0, s>>>(c->xyz.p, c->n4.p, c->tag.p, c->n6line.p, c->sigma.p,
                                                         c->etp.p, c->etl.p, c->rowptr.p, c->col.p, c->bc.p, c->nline,
                                                         sa, c->km.p, c->rhs.p, c->status.p);
  count_launch();
  if (c->prof.on) {
    AFEM_CUDA(cudaEventRecord(e1, s));
    AFEM_CUDA(cudaEventSynchronize(e1));
    float ms = 0;
    cudaEventElapsedTime(&ms, e0, e1);
    c->prof.add("assemble_rows", ms);
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
  }
  check_status(c, "assemble");
  c->assembled = true;
  c->assemble_gen += 1;
}

}  // namespace afem

namespace afem {
namespace {

// SET_BC_3DJoint's lifting (src/src_3DMT/forward_3DMT.f90:581-596) on the uncleared
// system: rhs[k*n + e] = g_k[e] on a Dirichlet row; otherwise -(D*g_k[e] + the row's
// products in ascending column order), the order of the reference's AL then AU loops.
__global__ void k_lift_dirichlet(const int32_t* __restrict__ rowptr, const int32_t* __restrict__ col,
                                 const int32_t* __restrict__ diagpos, const double2* __restrict__ km,
                                 const uint8_t* __restrict__ bc, int n, int nsys,
                                 const double* __restrict__ omega, const double2* __restrict__ g,
                                 double2* __restrict__ rhs) {
  const long total = (long)n * nsys;
  for (long q = blockIdx.x * (long)blockDim.x + threadIdx.x; q < total; q += (long)gridDim.x * blockDim.x) {
    const int k = (int)(q / n), e = (int)(q % n);
    const double2* gk = g + (long)k * n;
    if (bc[e]) {
      rhs[q] = gk[e];
      continue;
    }
    const double om = omega[k];
    double2 t = make_double2(0.0, 0.0);
    {
      const int dpos = diagpos[e];
      const double ar = km[dpos].x, ai = om * km[dpos].y;
      const double2 v = gk[e];
      t = make_double2(ar * v.x - ai * v.y, ar * v.y + ai * v.x);
    }
    for (int p = rowptr[e]; p < rowptr[e + 1]; ++p) {
      const int c = col[p];
      if (c == e) continue;
      const double ar = km[p].x, ai = om * km[p].y;
      const double2 v = gk[c];
      t = make_double2(t.x + (ar * v.x - ai * v.y), t.y + (ar * v.y + ai * v.x));
    }
    rhs[q] = make_double2(0.0 - t.x, 0.0 - t.y);
  }
}

// SET_BC_3DJoint's matrix part (forward_3DMT.f90:599-620): Dirichlet rows become the
// identity row, Dirichlet columns of the other rows are cleared.
__global__ void k_apply_dirichlet(const int32_t* __restrict__ rowptr, const int32_t* __restrict__ col,
                                  const uint8_t* __restrict__ bc, int n, double2* __restrict__ km) {
  for (int e = blockIdx.x * blockDim.x + threadIdx.x; e < n; e += gridDim.x * blockDim.x) {
    const bool dr = bc[e] != 0;
    for (int p = rowptr[e]; p < rowptr[e + 1]; ++p) {
      const int c = col[p];
      if (dr) km[p] = make_double2(c == e ? 1.0 : 0.0, 0.0);
      else if (bc[c]) km[p] = make_double2(0.0, 0.0);
    }
  }
}

}  // namespace

void assemble_dirichlet_device(afem_ctx* c, const uint8_t* bc, int nsys, const double* omega_host,
                               const double2* g) {
  AFEM_REQUIRE(c->pattern_ready, AFEM_ESTATE, "assemble: pattern not built");
  AFEM_REQUIRE(c->sigma_set, AFEM_ESTATE, "assemble: conductivity not set");
  AFEM_REQUIRE(nsys >= 1, AFEM_EINVAL, "assemble: no system");
  cudaStream_t s = c->stream;
  const int n = c->nline;
  // K and M with every row complete: no Dirichlet flag for the element gather
  DBuf<uint8_t> nobc;
  nobc.alloc(n);
  nobc.zero(s);
  SrcArgs sa{};
  sa.nsrc = 0;
  c->km.alloc(c->nnz);
  c->rhs.alloc((size_t)n * nsys);
  c->rhs_nsrc = nsys;
  k_assemble_rows<<<(n + 127) / 128, 128, 0, s>>>(c->xyz.p, c->n4.p, c->tag.p, c->n6line.p, c->sigma.p, c->etp.p,
                                                  c->etl.p, c->rowptr.p, c->col.p, nobc.p, n, sa, c->km.p, c->rhs.p,
                                                  c->status.p);
  count_launch();
  check_status(c, "assemble");
  DBuf<double> om;
  om.upload(omega_host, nsys, s);
  k_lift_dirichlet<<<c->num_sms * 8, 256, 0, s>>>(c->rowptr.p, c->col.p, c->diagpos.p, c->km.p, bc, n, nsys, om.p,
                                                  g, c->rhs.p);
  count_launch();
  k_apply_dirichlet<<<c->num_sms * 8, 256, 0, s>>>(c->rowptr.p, c->col.p, bc, n, c->km.p);
  count_launch();
  c->bc.alloc(n);
  AFEM_CUDA(cudaMemcpyAsync(c->bc.p, bc, n, cudaMemcpyDeviceToDevice, s));
  AFEM_CUDA(cudaStreamSynchronize(s));
  c->assembled = true;
  c->assemble_gen += 1;
}

}  // namespace afem
