// Adjoint sensitivities of site fields to the conductivity of each tetrahedron.
//
// Reference pattern: src/src_inv/m_jacobian.f90:120-218 and
// src/src_inv/solvePARDISOinv.f90:154-196 (one factorisation, adjoint right-
// hand sides K u = P^T, J = u^T (-dK/dm) A).  Here, for a site datum
// d = c^T x with A x = b and A = A^T (complex symmetric):
//   dd/dlog(sigma_t) = -u^T (dA/dlog sigma_t) x,   A u = c,
//   dA/dlog sigma_t = i omega sigma_t mu0 L0^2 Y_t   (Y_t: the element mass
//   matrix of GENMAT with its orientation signs, forward_bxyz_mpi.f90:223-232),
// restricted to non-Dirichlet rows and columns (SET_BC_ICCG removes the others).
// The adjoint systems are solved as one batch; this kernel then forms every
// (datum, tetrahedron) entry from the 6 edge values of the tetrahedron.
// Compiled with -fmad=false like the assembly it mirrors.
#include "afem_internal.h"

namespace afem {

namespace {

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

// J[k * ntet + t] for the nadj adjoint solutions U ([row][nadj]) and the forward solution x.
__global__ void k_jacobian(const double* __restrict__ xyz, const int32_t* __restrict__ n4,
                           const int32_t* __restrict__ n6line, const double* __restrict__ sigma,
                           const uint8_t* __restrict__ bc, int ntet, double omega, const double2* __restrict__ x,
                           const double2* __restrict__ U, int nadj, double2* __restrict__ J, DevStatus* st) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= ntet) return;
  const double pi = 4.0 * atan(1.0);
  const double dmu = 4.0 * pi * 1.0e-7;
  V3 p[4];
  for (int j = 0; j < 4; ++j) {
    const double* P = xyz + 3L * (n4[4L * t + j] - 1);
    p[j] = V3{P[0], P[1], P[2]};
  }
  int gl[6], d[6];
  bool live[6];
  for (int j = 0; j < 6; ++j) {
    const int s6 = n6line[6L * t + j];
    d[j] = (s6 < 0) ? -1 : 1;
    gl[j] = ((s6 < 0) ? -s6 : s6) - 1;
    live[j] = bc[gl[j]] == 0;
  }
  const V3 xx0 = vsub(p[3], p[2]), xx3 = vsub(p[2], p[1]), xx4 = vsub(p[0], p[2]);
  const double vol = 1.0 / 6.0 * vinner(vouter(xx0, xx4), vneg(xx3));
  if (!(vol > 0.0)) {
    raise_status(st, DEV_VOLUME, t);
    return;
  }
  const double cg = 1.0 / 6.0 / vol;
  V3 gn[4];
  gn[0] = vscale(cg, vouter(vsub(p[3], p[1]), vsub(p[2], p[1])));
  gn[1] = vscale(cg, vouter(vsub(p[2], p[0]), vsub(p[3], p[0])));
  gn[2] = vscale(cg, vouter(vsub(p[3], p[0]), vsub(p[1], p[0])));
  gn[3] = vscale(cg, vouter(vsub(p[1], p[0]), vsub(p[2], p[0])));
  double Y[6][6];
  for (int i = 0; i < 6; ++i)
    for (int j = 0; j < 6; ++j) {
      const int a = i > j ? i : j, b = i > j ? j : i;
      const int k = c_kl[a][0], l = c_kl[a][1], m = c_kl[b][0], n = c_kl[b][1];
      const double yy = intv(k, m, vol) * vinner(gn[l - 1], gn[n - 1]) - intv(k, n, vol) * vinner(gn[l - 1], gn[m - 1]) -
                        intv(l, m, vol) * vinner(gn[k - 1], gn[n - 1]) + intv(l, n, vol) * vinner(gn[k - 1], gn[m - 1]);
      Y[i][j] = (live[i] && live[j]) ? yy * d[a] * d[b] : 0.0;
    }
  // w = Y x (local), then J_k = -(i omega sigma mu0 L0^2) u_k^T w
  double2 w[6];
  for (int i = 0; i < 6; ++i) {
    double wr = 0.0, wi = 0.0;
    for (int j = 0; j < 6; ++j) {
      const double2 xj = x[gl[j]];
      wr += Y[i][j] * xj.x;
      wi += Y[i][j] * xj.y;
    }
    w[i] = make_double2(wr, wi);
  }
  const double c0 = omega * sigma[t] * dmu * 1.0e3 * 1.0e3;  // -(i c0) u^T w
  for (int k = 0; k < nadj; ++k) {
    double sr = 0.0, si = 0.0;
    for (int i = 0; i < 6; ++i) {
      const double2 u = U[(long)gl[i] * nadj + k];
      sr += u.x * w[i].x - u.y * w[i].y;
      si += u.x * w[i].y + u.y * w[i].x;
    }
    // -(i c0)(sr + i si) = c0 si - i c0 sr
    J[(long)k * ntet + t] = make_double2(c0 * si, -c0 * sr);
  }
}

}  // namespace

void jacobian_device(afem_ctx* c, double freq, const double* x_host, int nadj, double* J_host) {
  AFEM_REQUIRE(c->assembled && c->ntet > 0, AFEM_ESTATE, "jacobian: no assembled mesh system");
  AFEM_REQUIRE(c->nsys == nadj && c->X.p && !c->sol_packed, AFEM_ESTATE,
               "jacobian: solve the nadj adjoint systems first");
  cudaStream_t s = c->stream;
  DBuf<double2> x;
  x.upload(reinterpret_cast<const double2*>(x_host), c->nline, s);
  DBuf<double2> J;
  J.alloc((size_t)nadj * c->ntet);
  const double omega = 2.0 * (4.0 * atan(1.0)) * freq;
  k_jacobian<<<(c->ntet + 127) / 128, 128, 0, s>>>(c->xyz.p, c->n4.p, c->n6line.p, c->sigma.p, c->bc.p, c->ntet, omega,
                                                  x.p, c->X.p, nadj, J.p, c->status.p);
  count_launch();
  check_status(c, "jacobian");
  J.download(reinterpret_cast<double2*>(J_host), (size_t)nadj * c->ntet, s);
  AFEM_CUDA(cudaStreamSynchronize(s));
}

}  // namespace afem
