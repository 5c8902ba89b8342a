// Site evaluation: PREPOBSCOEFF + CALOBSEBCOMP on the device.
//
// Reference: src/solver_mpi/n_ebfem_bxyz_mpi.f90:653-726 (PREPOBSCOEFF),
// :397-423 and :570-626 (CALOBSEBCOMP / CALOBSRESP), src/common/
// m_mesh_type.f90:697-734 (FINDELEMENT0), src/solver/m_fem_util.f90:56-83
// (nodebasisfun), src/solver/m_fem_edge_util.f90:27-82 (FACEBASISFUN,
// EDGEBASISFUN), src/solver/sort_index.f90 (SORT_INDEX).
//
// FINDELEMENT0 returns the FIRST tetrahedron in id order whose barycentric
// coordinates are all >= 0; on the device every tetrahedron is tested in
// parallel and the smallest qualifying id wins (atomicMin).  Compiled with
// -fmad=false so the >= 0 decisions round exactly like the serial code.
#include "afem_internal.h"

namespace afem {

namespace {

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
__device__ __forceinline__ double volume(const V3& a, const V3& b, const V3& c) {
  return 1.0 / 6.0 * vinner(vouter(a, b), c);
}

__constant__ int c_kl[6][2] = {{1, 2}, {2, 3}, {1, 3}, {1, 4}, {2, 4}, {3, 4}};
__constant__ int c_lmn[4][3] = {{2, 3, 4}, {1, 4, 3}, {1, 2, 4}, {1, 3, 2}};
__constant__ int c_rot[4][6] = {{0, 1, 0, 0, -1, 1}, {0, 0, -1, 1, 0, -1}, {1, 0, 0, -1, 1, 0}, {-1, -1, 1, 0, 0, 0}};

__device__ __forceinline__ void load_tet(const double* xyz, const int32_t* n4, long t, V3 p[4]) {
  for (int j = 0; j < 4; ++j) {
    const double* P = xyz + 3L * (n4[4 * t + j] - 1);
    p[j] = V3{P[0], P[1], P[2]};
  }
}

// nodebasisfun (m_fem_util.f90:56-83)
__device__ __forceinline__ void nodebasis(const V3 e[4], const V3& x3, double a[4]) {
  const V3 v1 = vsub(e[0], x3), v2 = vsub(e[1], x3);
  const V3 x12 = vsub(e[1], e[0]), x13 = vsub(e[2], e[0]), x14 = vsub(e[3], e[0]);
  const V3 x24 = vsub(e[3], e[1]), x23 = vsub(e[2], e[1]);
  const double a5 = volume(x12, x13, x14);
  const double a4 = volume(x12, x13, vneg(v1)) / a5;
  const double a3 = volume(x14, x12, vneg(v1)) / a5;
  const double a2 = volume(x13, x14, vneg(v1)) / a5;
  const double a1 = volume(x24, x23, vneg(v2)) / a5;
  a[0] = a1; a[1] = a2; a[2] = a3; a[3] = a4;
}

// Searches tetrahedra t0 <= t < t1 (a packed batch restricts the search to one mesh).
__global__ void k_find(const double* __restrict__ xyz, const int32_t* __restrict__ n4, long t0, long t1,
                       const double* __restrict__ obs, int nobs, int* __restrict__ best) {
  const int s = blockIdx.y;
  if (s >= nobs) return;
  const V3 x3{obs[3 * s], obs[3 * s + 1], obs[3 * s + 2]};
  for (long t = t0 + blockIdx.x * (long)blockDim.x + threadIdx.x; t < t1; t += (long)gridDim.x * blockDim.x) {
    if (t >= *(volatile int*)(best + s)) break;
    V3 e[4];
    load_tet(xyz, n4, t, e);
    double a[4];
    nodebasis(e, x3, a);
    if (a[0] >= 0.0 && a[1] >= 0.0 && a[2] >= 0.0 && a[3] >= 0.0) {
      atomicMin(best + s, (int)t);
      break;
    }
  }
}

// Coefficient rows of one site (PREPOBSCOEFF :681-721).
__global__ void k_coeffs(const double* __restrict__ xyz, const int32_t* __restrict__ n4,
                         const int32_t* __restrict__ n6line, const double* __restrict__ obs, int nobs,
                         const int* __restrict__ best, int32_t* __restrict__ item, double* __restrict__ val_e,
                         double* __restrict__ val_f, DevStatus* st) {
  const int s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= nobs) return;
  const int tb = best[s];
  if (tb == 0x7fffffff) {
    raise_status(st, DEV_NOTFOUND, s);
    return;
  }
  const long t = tb;
  const V3 x3{obs[3 * s], obs[3 * s + 1], obs[3 * s + 2]};
  V3 e[4];
  load_tet(xyz, n4, t, e);
  // gradnodebasisfun (m_fem_util.f90:12-40)
  const V3 xx1 = vsub(e[3], e[2]), xx4 = vsub(e[2], e[1]), xx5 = vsub(e[0], e[2]);
  const double vol = volume(xx1, xx5, vneg(xx4));
  const double cg = 1.0 / 6.0 / vol;
  V3 gn[4];
  gn[0] = vscale(cg, vouter(vsub(e[3], e[1]), vsub(e[2], e[1])));
  gn[1] = vscale(cg, vouter(vsub(e[2], e[0]), vsub(e[3], e[0])));
  gn[2] = vscale(cg, vouter(vsub(e[3], e[0]), vsub(e[1], e[0])));
  gn[3] = vscale(cg, vouter(vsub(e[1], e[0]), vsub(e[2], e[0])));
  double lam[4];
  nodebasis(e, x3, lam);
  double w[6][3], wf[4][3], wfe[6][3];
  for (int i = 0; i < 6; ++i) {
    const int k = c_kl[i][0] - 1, l = c_kl[i][1] - 1;
    w[i][0] = lam[k] * gn[l].x - lam[l] * gn[k].x;
    w[i][1] = lam[k] * gn[l].y - lam[l] * gn[k].y;
    w[i][2] = lam[k] * gn[l].z - lam[l] * gn[k].z;
  }
  for (int i = 0; i < 4; ++i) {
    const int l = c_lmn[i][0] - 1, m = c_lmn[i][1] - 1, n = c_lmn[i][2] - 1;
    const V3 o1 = vouter(gn[m], gn[n]), o2 = vouter(gn[l], gn[m]), o3 = vouter(gn[n], gn[l]);
    wf[i][0] = 2.0 * (lam[l] * o1.x + lam[n] * o2.x + lam[m] * o3.x);
    wf[i][1] = 2.0 * (lam[l] * o1.y + lam[n] * o2.y + lam[m] * o3.y);
    wf[i][2] = 2.0 * (lam[l] * o1.z + lam[n] * o2.z + lam[m] * o3.z);
  }
  for (int c = 0; c < 3; ++c)  // mul_ab (m_matrix.f90:1106-1126)
    for (int j = 0; j < 6; ++j) {
      double acc = 0.0;
      for (int k = 0; k < 4; ++k) acc = acc + wf[k][c] * (c_rot[k][j] * 1.0);
      wfe[j][c] = acc;
    }
  // sort the 6 local edges by global id (distinct keys: any sort gives SORT_INDEX's order)
  int ord[6], gid[6];
  for (int j = 0; j < 6; ++j) {
    ord[j] = j;
    gid[j] = abs(n6line[6 * t + j]);
  }
  for (int i = 1; i < 6; ++i) {
    int v = ord[i], j = i - 1;
    while (j >= 0 && gid[ord[j]] > gid[v]) { ord[j + 1] = ord[j]; --j; }
    ord[j + 1] = v;
  }
  for (int j = 0; j < 6; ++j) {
    const int lj = ord[j];
    const double sg = (n6line[6 * t + lj] < 0) ? -1.0 : 1.0;
    item[6 * s + j] = gid[lj];
    for (int c = 0; c < 3; ++c) {
      val_e[((long)c * nobs + s) * 6 + j] = w[lj][c] * sg;
      val_f[((long)c * nobs + s) * 6 + j] = wfe[lj][c] * sg;
    }
  }
}

// CALOBSEBCOMP with fp = 0: B = coeff(2,c) A, E = coeff(1,c) (-i omega A).
__global__ void k_eval(const double2* __restrict__ X, int nline, int nsys, const double* __restrict__ omega,
                       int nobs, const int32_t* __restrict__ item, const double* __restrict__ val_e,
                       const double* __restrict__ val_f, double2* __restrict__ out) {
  const long i = blockIdx.x * (long)blockDim.x + threadIdx.x;
  if (i >= (long)nsys * 5 * nobs) return;
  const int s = (int)(i % nobs);
  const int comp = (int)((i / nobs) % 5);
  const int k = (int)(i / (5L * nobs));
  const double om = omega[k];
  const double* val = (comp < 3) ? val_f + (long)comp * nobs * 6 : val_e + (long)(comp - 3) * nobs * 6;
  double2 acc = make_double2(0.0, 0.0);
  for (int j = 0; j < 6; ++j) {
    const double2 a = X[(long)(item[6 * s + j] - 1) * nsys + k];
    double2 f = a;
    if (comp >= 3) {
      // fss = -((0,1)*omega*fs): ((0,1)*omega) = (0, omega); times fs; negated
      const double2 io = make_double2(0.0, om);
      const double2 pr = make_double2(io.x * a.x - io.y * a.y, io.x * a.y + io.y * a.x);
      f = make_double2(-pr.x, -pr.y);
    }
    const double v = val[s * 6 + j];
    acc = make_double2(acc.x + v * f.x, acc.y + v * f.y);
  }
  out[i] = acc;
}

}  // namespace

namespace {

void site_coeffs_range(afem_ctx* c, int nobs, const double* xyz_obs, long t0, long t1, int32_t* item, double* val_e,
                       double* val_f, int32_t* iele) {
  cudaStream_t s = c->stream;
  DBuf<double> obs;
  obs.upload(xyz_obs, 3L * nobs, s);
  DBuf<int> best;
  best.alloc(nobs);
  std::vector<int> init(nobs, 0x7fffffff);
  AFEM_CUDA(cudaMemcpyAsync(best.p, init.data(), sizeof(int) * nobs, cudaMemcpyHostToDevice, s));
  dim3 grid(std::max(1, std::min(2 * c->num_sms, (int)((t1 - t0 + 255) / 256))), nobs);
  k_find<<<grid, 256, 0, s>>>(c->xyz.p, c->n4.p, t0, t1, obs.p, nobs, best.p);
  count_launch();
  DBuf<int32_t> ditem;
  DBuf<double> dve, dvf;
  ditem.alloc(6L * nobs);
  dve.alloc(18L * nobs);
  dvf.alloc(18L * nobs);
  k_coeffs<<<(nobs + 63) / 64, 64, 0, s>>>(c->xyz.p, c->n4.p, c->n6line.p, obs.p, nobs, best.p, ditem.p, dve.p, dvf.p,
                                          c->status.p);
  count_launch();
  check_status(c, "sites: a site lies outside every tetrahedron");
  if (item) ditem.download(item, 6L * nobs, s);
  if (val_e) dve.download(val_e, 18L * nobs, s);
  if (val_f) dvf.download(val_f, 18L * nobs, s);
  if (iele) {
    std::vector<int> h(nobs);
    best.download(h.data(), nobs, s);
    AFEM_CUDA(cudaStreamSynchronize(s));
    for (int i = 0; i < nobs; ++i) iele[i] = h[i] + 1;
  }
  AFEM_CUDA(cudaStreamSynchronize(s));
}

}  // namespace

void site_coeffs_device(afem_ctx* c, int nobs, const double* xyz_obs, int32_t* item, double* val_e, double* val_f,
                        int32_t* iele) {
  site_coeffs_range(c, nobs, xyz_obs, 0, c->ntet, item, val_e, val_f, iele);
}

void sites_device(afem_ctx* c, int nobs, const double* xyz_obs, double* out) {
  AFEM_REQUIRE(c->nsys > 0 && c->X.p, AFEM_ESTATE, "sites: no solution");
  cudaStream_t s = c->stream;
  if (c->sol_packed) {
    // packed batch: system k is mesh k; its sites are searched in its own tetrahedra
    AFEM_REQUIRE((int)c->seg_tet_ptr.size() == c->nsys + 1, AFEM_ESTATE, "sites: the packed meshes changed");
    const double pi = 4.0 * std::atan(1.0);
    std::vector<int32_t> item(6L * nobs);
    std::vector<double> ve(18L * nobs), vf(18L * nobs);
    DBuf<int32_t> ditem;
    DBuf<double> dve, dvf, dom;
    DBuf<double2> dout;
    dout.alloc((long)c->nsys * 5 * nobs);
    for (int k = 0; k < c->nsys; ++k) {
      site_coeffs_range(c, nobs, xyz_obs, c->seg_tet_ptr[k], c->seg_tet_ptr[k + 1], item.data(), ve.data(), vf.data(),
                        nullptr);
      ditem.upload(item.data(), item.size(), s);
      dve.upload(ve.data(), ve.size(), s);
      dvf.upload(vf.data(), vf.size(), s);
      const double om = 2.0 * pi * c->sol_freq[k];
      dom.upload(&om, 1, s);
      const long tot = 5L * nobs;
      k_eval<<<(unsigned)((tot + 127) / 128), 128, 0, s>>>(c->X.p, c->nline, 1, dom.p, nobs, ditem.p, dve.p, dvf.p,
                                                           dout.p + (long)k * 5 * nobs);
      count_launch();
      AFEM_CUDA(cudaStreamSynchronize(s));
    }
    dout.download(reinterpret_cast<double2*>(out), (long)c->nsys * 5 * nobs, s);
    AFEM_CUDA(cudaStreamSynchronize(s));
    return;
  }
  std::vector<int32_t> item(6L * nobs);
  std::vector<double> ve(18L * nobs), vf(18L * nobs);
  site_coeffs_device(c, nobs, xyz_obs, item.data(), ve.data(), vf.data(), nullptr);
  DBuf<int32_t> ditem;
  DBuf<double> dve, dvf, dom;
  ditem.upload(item.data(), item.size(), s);
  dve.upload(ve.data(), ve.size(), s);
  dvf.upload(vf.data(), vf.size(), s);
  std::vector<double> om(c->nsys);
  const double pi = 4.0 * std::atan(1.0);
  for (int k = 0; k < c->nsys; ++k) om[k] = 2.0 * pi * c->sol_freq[k];
  dom.upload(om.data(), om.size(), s);
  DBuf<double2> dout;
  const long tot = (long)c->nsys * 5 * nobs;
  dout.alloc(tot);
  k_eval<<<(unsigned)((tot + 127) / 128), 128, 0, s>>>(c->X.p, c->nline, c->nsys, dom.p, nobs, ditem.p, dve.p, dvf.p,
                                                       dout.p);
  count_launch();
  dout.download(reinterpret_cast<double2*>(out), tot, s);
  AFEM_CUDA(cudaStreamSynchronize(s));
}

}  // namespace afem
