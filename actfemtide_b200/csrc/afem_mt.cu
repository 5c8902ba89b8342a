// 3-D magnetotelluric forward on the device: the boundary surfaces of the mesh, the
// 2-D TM solves on the four side faces that give the Dirichlet values, GENBCMT,
// and the batched solve of both polarisations of every frequency.
//
// Reference: src/src_3DMT/n_ebfem_3DMT.f90:38-113 (the program), forward_3DMT.f90
// (forward_3DMT, GENBCMT, GENMAT_MT, SET_BC_3DJoint), src/src_2D/forward_2DTM.f90
// (forward_2DTM, GENMAT2DTM, GENBC2D, SET_BC_ICCG) and src/src_2D/m_surface_type.f90
// (EXTRACT6SURFACES, FINDBOUNDARYLINE, COND3DTO2D and the triangle element functions).
//
// Layout.  A side surface's lines are numbered in a band order (sorted by the midpoint
// along one face axis, then the other; the order with the smaller bandwidth wins), so
// its complex-symmetric 2-D system is a band matrix of half-bandwidth b stored by
// columns: L[c*(b+1) + d] = A[c+d][c].  Every (surface, frequency) system is factored
// as L D L^T by one thread block (no pivoting: -i*A has the positive definite
// Hermitian part omega*mu0*sigma*M, so every leading block is non-singular), which
// replaces the reference's PARDISO call.  The element values and their sums are
// the reference's bit for bit (this file is built without FMA contraction): each
// off-diagonal entry receives one triangle's value and each diagonal at most two,
// so the atomic accumulation is order independent.
#include <algorithm>
#include <cmath>
#include <complex>
#include <numeric>

#include "afem_internal.h"

namespace afem {

namespace {

constexpr int MT_BAND_MAX = 2048;  // half-bandwidth limit of a side surface's band matrix

// A boundary triangle of a side surface as the device finds it (EXTRACT6SURFACES):
// nodes smallest first and anticlockwise in the surface plane, edges n[l] -> n[l+1]
// as signed 1-based 3-D line ids, the plane coordinates of the nodes.
struct MtTri {
  int surf;   // 2..5
  int tet;    // 0-based tetrahedron
  int n[3];   // 1-based 3-D node ids
  int e[3];   // signed 1-based 3-D line ids
  double y[3], z[3];
};

// One side surface: triangles with band-local signed edges, the band-ordered lines.
struct MtSurface {
  int n = 0, ntri = 0, bw = 0;
  std::vector<int32_t> line3d;    // n, 1-based 3-D ids in band order
  std::vector<uint8_t> bc;        // n, GENBC2D's Dirichlet flags
  std::vector<double> gval;       // n, Dirichlet values (real)
  std::vector<int32_t> nbr_ptr;   // n+1: pattern neighbours of each line, ascending 3-D id
  std::vector<int32_t> nbr;       // band-local ids
  std::vector<int> tet;           // ntri, 0-based tetrahedron of each triangle
  std::vector<int32_t> tedge;     // 3*ntri, signed 1-based band-local edges
  std::vector<double> tyz;        // 6*ntri: y[3], z[3]
};

}  // namespace

struct MtState {
  bool ready = false;
  double minmax[6] = {0, 0, 0, 0, 0, 0};
  DBuf<uint8_t> bits;         // node: bit j-1 set when the node lies on surface j (1..6)
  MtSurface s[4];             // surfaces 2..5
  // device copies, all surfaces concatenated
  DBuf<int32_t> tedge, tsurf, line3d, nbr_ptr, nbr;
  DBuf<double> tyz, gval;
  DBuf<uint8_t> bc2;
  DBuf<uint8_t> lbits;        // 3-D line: bit j-1 set when both its nodes lie on surface j
  DBuf<uint8_t> bc3;          // 3-D line: Dirichlet in the MT solve (on any surface)
  long tri_off[5] = {0, 0, 0, 0, 0}, row_off[5] = {0, 0, 0, 0, 0};
};

namespace {

// ---------------------------------------------------------------- 2-D element (m_surface_type.f90:727-907)
__constant__ int c_id3[3][3] = {{1, 2, 3}, {2, 3, 1}, {3, 1, 2}};

__device__ __forceinline__ double area_tri(const double* y, const double* z) {
  return 0.5 * fabs((y[2] - y[0]) * (z[1] - z[0]) - (y[1] - y[0]) * (z[2] - z[0]));
}
__device__ __forceinline__ void outer3(const double* a, const double* b, double* c) {
  c[0] = a[1] * b[2] - a[2] * b[1];
  c[1] = a[2] * b[0] - a[0] * b[2];
  c[2] = a[0] * b[1] - a[1] * b[0];
}
__device__ __forceinline__ double inner3(const double* a, const double* b) {
  return a[0] * b[0] + a[1] * b[1] + a[2] * b[2];
}
// grcgr: grad lambda_l x grad lambda_m of edge i_edge (x component; the others are zeros)
__device__ void grcgr(int ie, const double* y, const double* z, double* g) {
  const int l = c_id3[ie - 1][0], m = c_id3[ie - 1][1], n = c_id3[ie - 1][2];
  const double rl[3] = {0.0, y[l - 1], z[l - 1]}, rm[3] = {0.0, y[m - 1], z[m - 1]},
               rn[3] = {0.0, y[n - 1], z[n - 1]};
  double rnl[3], rmn[3], c[3];
  for (int k = 0; k < 3; ++k) { rnl[k] = rl[k] - rn[k]; rmn[k] = rn[k] - rm[k]; }
  const double s = area_tri(y, z);
  const double coef = -(0.25 / (s * s));
  outer3(rnl, rmn, c);
  for (int k = 0; k < 3; ++k) g[k] = coef * c[k];
}
// gradnodebasisfun_tri, with the reference's ex = (1, 0, 1)
__device__ void gradnode_tri(const double* y, const double* z, double gn[3][2]) {
  const double ex[3] = {1.0, 0.0, 1.0};
  const double s = area_tri(y, z);
  for (int l = 1; l <= 3; ++l) {
    const int m = c_id3[l - 1][1], n = c_id3[l - 1][2];
    const double xmn[3] = {0.0 - 0.0, y[n - 1] - y[m - 1], z[n - 1] - z[m - 1]};
    double c[3];
    outer3(ex, xmn, c);
    const double coef = 0.5 / s;
    gn[l - 1][0] = coef * c[1];
    gn[l - 1][1] = coef * c[2];
  }
}
__device__ __forceinline__ double grdgr(const double gn[3][2], int i, int j) {
  const double a[3] = {0.0, gn[i - 1][0], gn[i - 1][1]}, b[3] = {0.0, gn[j - 1][0], gn[j - 1][1]};
  return inner3(a, b);
}
// NlNmdS with the reference's default-real 1./6. and 1./12.
__device__ __forceinline__ double nlnm(int l, int m, double s) {
  return (l == m) ? (double)(1.0f / 6.0f) * s : (double)(1.0f / 12.0f) * s;
}
__device__ double wiwjds(int ie, int je, const double* y, const double* z) {
  const int l = c_id3[ie - 1][0], m = c_id3[ie - 1][1];
  const int lp = c_id3[je - 1][0], mp = c_id3[je - 1][1];
  double gn[3][2];
  gradnode_tri(y, z, gn);
  const double s = area_tri(y, z);
  return nlnm(l, lp, s) * grdgr(gn, m, mp) - nlnm(m, lp, s) * grdgr(gn, l, mp) - nlnm(l, mp, s) * grdgr(gn, m, lp) +
         nlnm(m, mp, s) * grdgr(gn, l, lp);
}

// ---------------------------------------------------------------- surfaces (EXTRACT6SURFACES)
__global__ void k_mt_minmax(const double* __restrict__ xyz, int node, double* __restrict__ part) {
  double mm[6] = {xyz[0], xyz[0], xyz[1], xyz[1], xyz[2], xyz[2]};
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < node; i += gridDim.x * blockDim.x)
    for (int c = 0; c < 3; ++c) {
      const double v = xyz[3L * i + c];
      mm[2 * c] = fmin(mm[2 * c], v);
      mm[2 * c + 1] = fmax(mm[2 * c + 1], v);
    }
  __shared__ double red[6][256];
  for (int k = 0; k < 6; ++k) red[k][threadIdx.x] = mm[k];
  __syncthreads();
  for (int w = blockDim.x / 2; w > 0; w >>= 1) {
    if ((int)threadIdx.x < w)
      for (int k = 0; k < 6; ++k)
        red[k][threadIdx.x] = (k & 1) ? fmax(red[k][threadIdx.x], red[k][threadIdx.x + w])
                                      : fmin(red[k][threadIdx.x], red[k][threadIdx.x + w]);
    __syncthreads();
  }
  if (threadIdx.x == 0)
    for (int k = 0; k < 6; ++k) part[6L * blockIdx.x + k] = red[k][0];
}

// node_on_surface (m_surface_type.f90:247-258): bounds are the extent -+ the default-real 0.1
__global__ void k_mt_node_bits(const double* __restrict__ xyz, int node, double xmin, double xmax, double ymin,
                               double ymax, double zmin, double zmax, uint8_t* __restrict__ bits) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < node; i += gridDim.x * blockDim.x) {
    const double x = xyz[3L * i], y = xyz[3L * i + 1], z = xyz[3L * i + 2];
    uint8_t b = 0;
    if (z >= zmax) b |= 1;
    if (y >= ymax) b |= 2;
    if (x <= xmin) b |= 4;
    if (y <= ymin) b |= 8;
    if (x >= xmax) b |= 16;
    if (z <= zmin) b |= 32;
    bits[i] = b;
  }
}

__constant__ int c_lmn[4][3] = {{2, 3, 4}, {1, 4, 3}, {1, 2, 4}, {1, 3, 2}};

// Boundary triangles of the side surfaces 2..5: tetrahedron faces whose three nodes lie
// on one side plane.  count_only: only the number per surface (cnt[0..3]).
__global__ void k_mt_side_tris(const int32_t* __restrict__ n4, const int32_t* __restrict__ n6line,
                               const int32_t* __restrict__ line, const double* __restrict__ xyz,
                               const uint8_t* __restrict__ bits, int ntet, int* __restrict__ cnt,
                               MtTri* __restrict__ out, int cap, DevStatus* st) {
  for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < ntet; t += gridDim.x * blockDim.x) {
    for (int f = 0; f < 4; ++f) {
      int nd[3];
      for (int k = 0; k < 3; ++k) nd[k] = n4[4L * t + c_lmn[f][k] - 1];
      const int common = bits[nd[0] - 1] & bits[nd[1] - 1] & bits[nd[2] - 1] & 0x1e;  // surfaces 2..5
      if (!common) continue;
      for (int j = 2; j <= 5; ++j) {
        if (!(common & (1 << (j - 1)))) continue;
        if (!out) {
          atomicAdd(&cnt[j - 2], 1);
          continue;
        }
        const int q = atomicAdd(&cnt[4], 1);
        if (q >= cap) { raise_status(st, DEV_NOTFOUND, t); continue; }
        // smallest node first (MKFACE lists (n1 < n2 < n3)), then anticlockwise
        int a = nd[0], b = nd[1], c = nd[2], tmp;
        if (a > b) { tmp = a; a = b; b = tmp; }
        if (b > c) { tmp = b; b = c; c = tmp; }
        if (a > b) { tmp = a; a = b; b = tmp; }
        int v[3] = {a, b, c};
        double yy[3], zz[3];
        for (int k = 0; k < 3; ++k) {
          const double* P = xyz + 3L * (v[k] - 1);
          // x1x2_face: xz on north/south, yz on west/east
          yy[k] = (j == 2 || j == 4) ? P[0] : P[1];
          zz[k] = P[2];
        }
        double x1[3] = {yy[1] - yy[0], zz[1] - zz[0], 0.0}, x2[3] = {yy[2] - yy[0], zz[2] - zz[0], 0.0}, x3[3];
        x1[2] = 0.0;
        x2[2] = 0.0;
        outer3(x1, x2, x3);
        if (x3[2] < 0.0) {
          tmp = v[1]; v[1] = v[2]; v[2] = tmp;
          double d = yy[1]; yy[1] = yy[2]; yy[2] = d;
          d = zz[1]; zz[1] = zz[2]; zz[2] = d;
        }
        MtTri r;
        r.surf = j;
        r.tet = t;
        for (int k = 0; k < 3; ++k) { r.n[k] = v[k]; r.y[k] = yy[k]; r.z[k] = zz[k]; }
        // n3line: each edge v[l] -> v[l+1] matched against the tetrahedron's six lines
        for (int l = 0; l < 3; ++l) {
          const int p = v[l], pq = v[(l + 1) % 3];
          int got = 0;
          for (int k = 0; k < 6 && !got; ++k) {
            const int s6 = n6line[6L * t + k];
            const int e = s6 < 0 ? -s6 : s6;
            const int la = line[2L * (e - 1)], lb = line[2L * (e - 1) + 1];
            if (p == la && pq == lb) got = e;
            else if (p == lb && pq == la) got = -e;
          }
          if (!got) raise_status(st, DEV_NOTFOUND, t);
          r.e[l] = got;
        }
        out[q] = r;
      }
    }
  }
}

// Lines with both nodes on surface j, per surface 1..6 (for the counts and the 3-D flags).
__global__ void k_mt_line_bits(const int32_t* __restrict__ line, const uint8_t* __restrict__ bits, int nline,
                               uint8_t* __restrict__ lbits, uint8_t* __restrict__ bc3, int* __restrict__ cnt) {
  for (int e = blockIdx.x * blockDim.x + threadIdx.x; e < nline; e += gridDim.x * blockDim.x) {
    const uint8_t b = bits[line[2L * e] - 1] & bits[line[2L * e + 1] - 1];
    lbits[e] = b;
    bc3[e] = b != 0;
    for (int j = 0; j < 6; ++j)
      if (b & (1 << j)) atomicAdd(&cnt[j], 1);
  }
}

}  // namespace

namespace {

// One (side surface, frequency) band system.
struct BandSys {
  long boff;  // first band entry
  long roff;  // first row of the right-hand side / solution
  long lro;   // the surface's first line in the concatenated per-line arrays
  int n, bw, surf, f;
};

__device__ __forceinline__ void atomic_add2(double2* p, double re, double im) {
  atomicAdd(&p->x, re);
  atomicAdd(&p->y, im);
}

// GENMAT2DTM (forward_2DTM.f90:272-355) for every (triangle, frequency): the element matrix
// (A1 + i*omega*mu0*sigma*L0^2 * B1) * d_i * d_j added to the band as sup_iccg adds it:
// D gets elm_k(i,i), the pair (i, j) gets elm_k(max, min).
__global__ void k_mt2d_assemble(const int32_t* __restrict__ tedge, const double* __restrict__ tyz,
                                const double* __restrict__ tsig, const int32_t* __restrict__ tsurf, long ntri_all,
                                int nf, const double* __restrict__ om, double dmu, const BandSys* __restrict__ sys,
                                double2* __restrict__ band) {
  const long total = ntri_all * nf;
  for (long q = blockIdx.x * (long)blockDim.x + threadIdx.x; q < total; q += (long)gridDim.x * blockDim.x) {
    const long t = q % ntri_all;
    const int f = (int)(q / ntri_all);
    const BandSys S = sys[tsurf[t] * nf + f];
    const int ld = S.bw + 1;
    double y[3], z[3];
    for (int k = 0; k < 3; ++k) { y[k] = tyz[6 * t + k]; z[k] = tyz[6 * t + 3 + k]; }
    int loc[3];
    double dir[3];
    for (int k = 0; k < 3; ++k) {
      const int e = tedge[3 * t + k];
      dir[k] = (e < 0) ? -1.0 : 1.0;
      loc[k] = (e < 0 ? -e : e) - 1;
    }
    // BB = iunit*omega*dmu*sigma*L0**2: real part 0*..., imaginary ((omega*dmu)*sigma)*1e6
    const double bbr = ((0.0 * om[f]) * dmu) * tsig[t] * 1.0e6;
    const double bbi = ((1.0 * om[f]) * dmu) * tsig[t] * 1.0e6;
    const double sa = area_tri(y, z);
    double g[3][3];
    for (int k = 0; k < 3; ++k) grcgr(k + 1, y, z, g[k]);
    for (int a = 0; a < 3; ++a)
      for (int b = 0; b <= a; ++b) {
        const double A1 = 4.0 * sa * inner3(g[a], g[b]);
        const double B1 = wiwjds(a + 1, b + 1, y, z);
        // (A1 + BB*B1) * idir(a) * idir(b), BB*B1 = (bbr*B1 - 0, bbi*B1)
        double re = A1 + bbr * B1, im = bbi * B1;
        re = re * dir[a]; im = im * dir[a];
        re = re * dir[b]; im = im * dir[b];
        const int r = max(loc[a], loc[b]), c = min(loc[a], loc[b]);
        atomic_add2(band + S.boff + (long)c * ld + (r - c), re, im);
      }
  }
}

// SET_BC_ICCG's lifting (forward_2DTM.f90:429-447): rf = g on Dirichlet rows, else
// -(D*g_i + the row's products in ascending surface-line order).
__global__ void k_mt2d_lift(const BandSys* __restrict__ sys, const double2* __restrict__ band,
                            const uint8_t* __restrict__ bc2, const double* __restrict__ gval,
                            const int32_t* __restrict__ nbr_ptr, const int32_t* __restrict__ nbr,
                            double2* __restrict__ rf) {
  const BandSys S = sys[blockIdx.y];
  const long ro = S.lro;
  const int ld = S.bw + 1;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < S.n; i += gridDim.x * blockDim.x) {
    double2 out;
    if (bc2[ro + i]) {
      out = make_double2(gval[ro + i], 0.0);
    } else {
      const double2 di = band[S.boff + (long)i * ld];
      const double gr = gval[ro + i], gi = 0.0;
      double tr = di.x * gr - di.y * gi, ti = di.x * gi + di.y * gr;
      for (int p = nbr_ptr[ro + i]; p < nbr_ptr[ro + i + 1]; ++p) {
        const int c = nbr[p];
        const int hi = max(i, c), lo = min(i, c);
        const double2 a = band[S.boff + (long)lo * ld + (hi - lo)];
        const double vr = gval[ro + c], vi = 0.0;
        tr = tr + (a.x * vr - a.y * vi);
        ti = ti + (a.x * vi + a.y * vr);
      }
      out = make_double2(0.0 - tr, 0.0 - ti);
    }
    rf[S.roff + i] = out;
  }
}

// SET_BC_ICCG's matrix part (forward_2DTM.f90:449-468) on the band.
__global__ void k_mt2d_zero(const BandSys* __restrict__ sys, const uint8_t* __restrict__ bc2,
                            double2* __restrict__ band) {
  const BandSys S = sys[blockIdx.y];
  const long ro = S.lro;
  const int ld = S.bw + 1;
  const long tot = (long)S.n * ld;
  for (long q = blockIdx.x * (long)blockDim.x + threadIdx.x; q < tot; q += (long)gridDim.x * blockDim.x) {
    const int c = (int)(q / ld), d = (int)(q % ld), r = c + d;
    if (r >= S.n) continue;
    const bool br = bc2[ro + r] != 0, bcc = bc2[ro + c] != 0;
    if (d == 0) {
      if (br) band[S.boff + q] = make_double2(1.0, 0.0);
    } else if (br || bcc) {
      band[S.boff + q] = make_double2(0.0, 0.0);
    }
  }
}

// A = L D L^T of one band system per block, the forward substitution folded in, then
// D^-1 and the back substitution by warp 0.  L overwrites the band (unit diagonal
// implied, D kept on the diagonal); rf becomes L^-1 rf; x receives the solution.
__global__ void __launch_bounds__(512) k_band_ldlt(const BandSys* __restrict__ sys, double2* __restrict__ band,
                                                   double2* __restrict__ rf, double2* __restrict__ x,
                                                   DevStatus* st) {
  const BandSys S = sys[blockIdx.x];
  const int n = S.n, b = S.bw, ld = b + 1;
  double2* L = band + S.boff;
  double2* y = rf + S.roff;
  double2* X = x + S.roff;
  extern __shared__ double2 shm[];
  double2* cb = shm;           // column k below the pivot, unscaled
  double2* lb = shm + ld;      // the same divided by the pivot
  for (int k = 0; k < n; ++k) {
    const int m = min(b, n - 1 - k);
    const double2 dk = L[(long)k * ld];
    if (threadIdx.x == 0 && !(isfinite(dk.x) && isfinite(dk.y) && (dk.x != 0.0 || dk.y != 0.0)))
      raise_status(st, DEV_PIVOT, k);
    const double2 yk = y[k];
    for (int d = 1 + threadIdx.x; d <= m; d += blockDim.x) {
      const double2 c = L[(long)k * ld + d];
      const double2 l = cdiv(c, dk);
      cb[d] = c;
      lb[d] = l;
      L[(long)k * ld + d] = l;
      y[k + d] = csub(y[k + d], cmul(l, yk));
    }
    __syncthreads();
    // trailing update A[k+i][k+j] -= l_i * c_j (j <= i): warps take the columns k+j in turn,
    // lanes run down a column (contiguous in the band)
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, nw = blockDim.x >> 5;
    for (int j = 1 + warp; j <= m; j += nw) {
      const double2 cj = cb[j];
      double2* colp = L + (long)(k + j) * ld - j;
      for (int i = j + lane; i <= m; i += 32) colp[i] = csub(colp[i], cmul(lb[i], cj));
    }
    __syncthreads();
  }
  if (threadIdx.x >= 32) return;
  const int lane = threadIdx.x;
  for (int k = n - 1; k >= 0; --k) {
    const int m = min(b, n - 1 - k);
    double sr = 0.0, si = 0.0;
    for (int d = 1 + lane; d <= m; d += 32) {
      const double2 p = cmul(L[(long)k * ld + d], X[k + d]);
      sr += p.x;
      si += p.y;
    }
    for (int o = 16; o > 0; o >>= 1) {
      sr += __shfl_xor_sync(0xffffffffu, sr, o);
      si += __shfl_xor_sync(0xffffffffu, si, o);
    }
    if (lane == 0) {
      const double2 zk = cdiv(y[k], L[(long)k * ld]);
      X[k] = make_double2(zk.x - sr, zk.y - si);
    }
    __syncwarp();
  }
}

// GENBCMT (forward_3DMT.f90:113-176) into g[sys*nline + e], sys = 2f + pol.  Top lines:
// (i/omega) * (dx, dy) . (xhat, yhat).  Run before the side and bottom kernels.
__global__ void k_mt_g_top(const int32_t* __restrict__ line, const double* __restrict__ xyz,
                           const uint8_t* __restrict__ lbits, int nline, int nf, const double* __restrict__ om,
                           double2* __restrict__ g) {
  for (int e = blockIdx.x * blockDim.x + threadIdx.x; e < nline; e += gridDim.x * blockDim.x) {
    if (!(lbits[e] & 1)) continue;
    const double* P1 = xyz + 3L * (line[2L * e] - 1);
    const double* P2 = xyz + 3L * (line[2L * e + 1] - 1);
    const double dxy[3] = {P2[0] - P1[0], P2[1] - P1[1], 0.0};
    const double xh[3] = {1.0, 0.0, 0.0}, yh[3] = {0.0, 1.0, 0.0};
    const double ix = inner3(dxy, xh), iy = inner3(dxy, yh);
    for (int f = 0; f < nf; ++f) {
      const double ur = 0.0 / om[f], ui = 1.0 / om[f];  // iunit/omega
      g[(long)(2 * f) * nline + e] = make_double2(ur * ix * 1.0, ui * ix * 1.0);
      g[(long)(2 * f + 1) * nline + e] = make_double2(ur * iy * 1.0, ui * iy * 1.0);
    }
  }
}

// Side surface js (0..3 for surfaces 2..5): Avalue_bc(iline, isr) = (i/omega) * bs(l).
__global__ void k_mt_g_side(const int32_t* __restrict__ line3d, int nl, long sol_stride_f,
                            const double2* __restrict__ xs, int isr, int nf, const double* __restrict__ om, int nline,
                            double2* __restrict__ g) {
  for (int l = blockIdx.x * blockDim.x + threadIdx.x; l < nl; l += gridDim.x * blockDim.x) {
    const int e = line3d[l] - 1;
    for (int f = 0; f < nf; ++f) {
      const double2 v = xs[f * sol_stride_f + l];
      const double ur = 0.0 / om[f], ui = 1.0 / om[f];
      g[(long)(2 * f + isr) * nline + e] = make_double2(ur * v.x - ui * v.y, ur * v.y + ui * v.x);
    }
  }
}

// Bottom lines: only the column the side loop left behind (Ey) is reset.
__global__ void k_mt_g_bottom(const uint8_t* __restrict__ lbits, int nline, int nf, double2* __restrict__ g) {
  for (int e = blockIdx.x * blockDim.x + threadIdx.x; e < nline; e += gridDim.x * blockDim.x) {
    if (!(lbits[e] & 32)) continue;
    for (int f = 0; f < nf; ++f) g[(long)(2 * f + 1) * nline + e] = make_double2(0.0, 0.0);
  }
}

}  // namespace

namespace {

inline int nblk(long n, int t) { return (int)std::max<long>(1, std::min<long>((n + t - 1) / t, 1L << 20)); }

MtState& state(afem_ctx* c) {
  if (!c->mt) c->mt = new MtState();
  return *c->mt;
}

// GENMAT_MT's and COND3DTO2D's conductivities per tetrahedron.
void resolve_cond(afem_ctx* c, const afem_mt_cond* cd, std::vector<double>& s3, std::vector<double>& s2) {
  AFEM_REQUIRE(cd, AFEM_EINVAL, "mt: null conductivity");
  AFEM_REQUIRE(cd->condflag == 0 || cd->condflag == 1, AFEM_EINVAL, "mt: condflag must be 0 or 1");
  const int ntet = c->ntet;
  const int32_t* tag = cd->tag_phys ? cd->tag_phys : c->h_tag.data();
  long nphys2 = 0;
  for (int t = 0; t < ntet; ++t) nphys2 += tag[t] >= 3;
  const long nphys1 = ntet - nphys2;
  if (cd->condflag == 1) {
    AFEM_REQUIRE(cd->sigma_file, AFEM_EINVAL, "mt: condflag 1 needs sigma_file");
    AFEM_REQUIRE(cd->nphys2 == nphys2, AFEM_EINVAL, "mt: nphys2 differs from the tetrahedra with tag >= 3");
  } else {
    AFEM_REQUIRE(cd->sigma_land && cd->nvolume >= 1, AFEM_EINVAL, "mt: condflag 0 needs sigma_land");
  }
  s3.resize(ntet);
  s2.resize(ntet);
  for (int t = 0; t < ntet; ++t) {
    const int g = tag[t];
    AFEM_REQUIRE(g >= 1, AFEM_EINVAL, "mt: a tetrahedron's tag selects no conductivity");
    if (g <= 2) {
      s3[t] = cd->sigma_air;
      s2[t] = (g == 1) ? cd->sigma_air : (double)3.31f;
    } else if (cd->condflag == 0) {
      AFEM_REQUIRE(g - 1 <= cd->nvolume, AFEM_EINVAL, "mt: tag beyond sigma_land");
      s3[t] = cd->sigma_land[g - 2];
      s2[t] = cd->sigma_land[0];
    } else {
      AFEM_REQUIRE(t >= nphys1, AFEM_EINVAL, "mt: a land tetrahedron before the last nphys2");
      s3[t] = s2[t] = cd->sigma_file[t - nphys1];
    }
  }
}

struct LineEnds {
  int id;
  double y1, z1, y2, z2;  // plane coordinates of line(1) and line(2)
};

void build_surfaces(afem_ctx* c) {
  MtState& M = state(c);
  if (M.ready) return;
  cudaStream_t s = c->stream;
  const int node = c->node, ntet = c->ntet, nline = c->nline;
  // extent (GENXYZMINMAX_MT)
  const int nb = std::min(nblk(node, 256), 1024);
  DBuf<double> part;
  part.alloc(6L * nb);
  k_mt_minmax<<<nb, 256, 0, s>>>(c->xyz.p, node, part.p);
  count_launch();
  std::vector<double> hp(6L * nb);
  part.download(hp.data(), hp.size(), s);
  AFEM_CUDA(cudaStreamSynchronize(s));
  double mm[6] = {hp[0], hp[1], hp[2], hp[3], hp[4], hp[5]};
  for (int b = 1; b < nb; ++b)
    for (int k = 0; k < 6; ++k) mm[k] = (k & 1) ? std::max(mm[k], hp[6L * b + k]) : std::min(mm[k], hp[6L * b + k]);
  std::copy(mm, mm + 6, M.minmax);
  const double d01 = (double)0.1f;
  const double xmin = mm[0] + d01, xmax = mm[1] - d01, ymin = mm[2] + d01, ymax = mm[3] - d01;
  const double zmin = mm[4] + d01, zmax = mm[5] - d01;
  M.bits.alloc(node);
  k_mt_node_bits<<<nblk(node, 256), 256, 0, s>>>(c->xyz.p, node, xmin, xmax, ymin, ymax, zmin, zmax, M.bits.p);
  count_launch();
  // side triangles: count, then emit
  DBuf<int> cnt;
  cnt.alloc(8);
  cnt.zero(s);
  k_mt_side_tris<<<nblk(ntet, 256), 256, 0, s>>>(c->n4.p, c->n6line.p, c->line.p, c->xyz.p, M.bits.p, ntet, cnt.p,
                                                 nullptr, 0, c->status.p);
  count_launch();
  int hc[8];
  cnt.download(hc, 8, s);
  AFEM_CUDA(cudaStreamSynchronize(s));
  const long ntri_all = (long)hc[0] + hc[1] + hc[2] + hc[3];
  AFEM_REQUIRE(hc[0] > 0 && hc[1] > 0 && hc[2] > 0 && hc[3] > 0, AFEM_EINVAL,
               "mt: a side surface of the mesh extent holds no boundary triangle");
  DBuf<MtTri> tri;
  tri.alloc(ntri_all);
  cnt.zero(s);
  k_mt_side_tris<<<nblk(ntet, 256), 256, 0, s>>>(c->n4.p, c->n6line.p, c->line.p, c->xyz.p, M.bits.p, ntet, cnt.p,
                                                 tri.p, (int)ntri_all, c->status.p);
  count_launch();
  check_status(c, "mt surfaces");
  std::vector<MtTri> ht(ntri_all);
  tri.download(ht.data(), ntri_all, s);
  // lines on each plane
  M.lbits.alloc(nline);
  M.bc3.alloc(nline);
  cnt.zero(s);
  k_mt_line_bits<<<nblk(nline, 256), 256, 0, s>>>(c->line.p, M.bits.p, nline, M.lbits.p, M.bc3.p, cnt.p);
  count_launch();
  cnt.download(hc, 8, s);
  AFEM_CUDA(cudaStreamSynchronize(s));
  std::sort(ht.begin(), ht.end(), [](const MtTri& a, const MtTri& b) {
    if (a.surf != b.surf) return a.surf < b.surf;
    if (a.n[0] != b.n[0]) return a.n[0] < b.n[0];
    if (a.n[1] != b.n[1]) return a.n[1] < b.n[1];
    return a.n[2] < b.n[2];
  });
  long t0 = 0;
  for (int js = 0; js < 4; ++js) {
    MtSurface& S = M.s[js];
    long t1 = t0;
    while (t1 < ntri_all && ht[t1].surf == js + 2) ++t1;
    S.ntri = (int)(t1 - t0);
    // the surface's lines with their plane coordinates, oriented as the 3-D line
    std::vector<LineEnds> L;
    L.reserve(3 * S.ntri);
    for (long t = t0; t < t1; ++t)
      for (int l = 0; l < 3; ++l) {
        const int e = ht[t].e[l], a = l, b = (l + 1) % 3;
        LineEnds le;
        le.id = std::abs(e);
        if (e > 0) { le.y1 = ht[t].y[a]; le.z1 = ht[t].z[a]; le.y2 = ht[t].y[b]; le.z2 = ht[t].z[b]; }
        else { le.y1 = ht[t].y[b]; le.z1 = ht[t].z[b]; le.y2 = ht[t].y[a]; le.z2 = ht[t].z[a]; }
        L.push_back(le);
      }
    std::sort(L.begin(), L.end(), [](const LineEnds& a, const LineEnds& b) { return a.id < b.id; });
    L.erase(std::unique(L.begin(), L.end(), [](const LineEnds& a, const LineEnds& b) { return a.id == b.id; }),
            L.end());
    S.n = (int)L.size();
    AFEM_REQUIRE(S.n == hc[js + 1], AFEM_EPATTERN,
                 "mt: a line on a side plane belongs to no boundary triangle (the surface is not a plane face)");
    // band order: midpoints sorted along one plane axis, then the other; keep the narrower
    std::vector<int> byid(S.n);
    std::iota(byid.begin(), byid.end(), 0);
    auto bandwidth = [&](const std::vector<int>& order) {
      std::vector<int> pos(S.n);
      for (int k = 0; k < S.n; ++k) pos[order[k]] = k;
      int bw = 0;
      for (long t = t0; t < t1; ++t) {
        int lo = S.n, hi = -1;
        for (int l = 0; l < 3; ++l) {
          const int id = std::abs(ht[t].e[l]);
          const int k = (int)(std::lower_bound(L.begin(), L.end(), id,
                                               [](const LineEnds& a, int v) { return a.id < v; }) - L.begin());
          lo = std::min(lo, pos[k]);
          hi = std::max(hi, pos[k]);
        }
        bw = std::max(bw, hi - lo);
      }
      return bw;
    };
    std::vector<int> best;
    int bestbw = -1;
    for (int axis = 0; axis < 2; ++axis) {
      std::vector<int> order = byid;
      std::stable_sort(order.begin(), order.end(), [&](int a, int b) {
        const double ua = L[a].y1 + L[a].y2, ub = L[b].y1 + L[b].y2;
        const double va = L[a].z1 + L[a].z2, vb = L[b].z1 + L[b].z2;
        const double pa = axis ? va : ua, pb = axis ? vb : ub, qa = axis ? ua : va, qb = axis ? ub : vb;
        if (pa != pb) return pa < pb;
        return qa < qb;
      });
      const int bw = bandwidth(order);
      if (bestbw < 0 || bw < bestbw) { bestbw = bw; best = order; }
    }
    AFEM_REQUIRE(bestbw <= MT_BAND_MAX, AFEM_EINVAL, "mt: a side surface's band is wider than 2048 lines");
    S.bw = bestbw;
    std::vector<int> pos(S.n);
    for (int k = 0; k < S.n; ++k) pos[best[k]] = k;
    S.line3d.resize(S.n);
    S.bc.assign(S.n, 0);
    S.gval.assign(S.n, 0.0);
    // FINDBOUNDARYLINE + GENBC2D; the plane axes of a side face: (x or y, z)
    const double yl = (js == 0 || js == 2) ? xmin : ymin, yr = (js == 0 || js == 2) ? xmax : ymax;
    for (int k = 0; k < S.n; ++k) {
      const LineEnds& le = L[best[k]];
      S.line3d[k] = le.id;
      int fl = 0;
      if (le.y1 < yl && le.y2 < yl) fl = 3;
      if (le.y1 > yr && le.y2 > yr) fl = 4;
      if (le.z1 < zmin && le.z2 < zmin) fl = 2;
      if (le.z1 > zmax && le.z2 > zmax) fl = 1;
      if (fl == 1) {
        AFEM_REQUIRE(le.z1 == le.z2, AFEM_EINVAL, "mt: a top boundary line of a side face is not horizontal");
        S.bc[k] = 1;
        S.gval[k] = (le.y2 - le.y1) * 1.0;
      } else if (fl != 0) {
        S.bc[k] = 1;
      }
    }
    // triangles in band-local edges; pattern neighbours for the lifting
    S.tet.resize(S.ntri);
    S.tedge.resize(3L * S.ntri);
    S.tyz.resize(6L * S.ntri);
    std::vector<std::vector<int>> nb(S.n);
    for (long t = t0; t < t1; ++t) {
      const long q = t - t0;
      S.tet[q] = ht[t].tet;
      int loc[3];
      for (int l = 0; l < 3; ++l) {
        const int id = std::abs(ht[t].e[l]);
        const int k = (int)(std::lower_bound(L.begin(), L.end(), id,
                                             [](const LineEnds& a, int v) { return a.id < v; }) - L.begin());
        loc[l] = pos[k];
        S.tedge[3 * q + l] = (ht[t].e[l] < 0 ? -1 : 1) * (loc[l] + 1);
        S.tyz[6 * q + l] = ht[t].y[l];
        S.tyz[6 * q + 3 + l] = ht[t].z[l];
      }
      for (int a = 0; a < 3; ++a)
        for (int b = 0; b < 3; ++b)
          if (a != b) nb[loc[a]].push_back(loc[b]);
    }
    S.nbr_ptr.assign(S.n + 1, 0);
    S.nbr.clear();
    for (int k = 0; k < S.n; ++k) {
      auto& v = nb[k];
      std::sort(v.begin(), v.end(), [&](int a, int b) { return S.line3d[a] < S.line3d[b]; });
      v.erase(std::unique(v.begin(), v.end()), v.end());
      S.nbr.insert(S.nbr.end(), v.begin(), v.end());
      S.nbr_ptr[k + 1] = (int32_t)S.nbr.size();
    }
    t0 = t1;
  }
  // concatenated device copies
  std::vector<int32_t> tedge, tsurf, line3d, nbr_ptr, nbr;
  std::vector<double> tyz, gval;
  std::vector<uint8_t> bc2;
  nbr_ptr.push_back(0);
  for (int js = 0; js < 4; ++js) {
    const MtSurface& S = M.s[js];
    M.tri_off[js] = (long)tsurf.size();
    M.row_off[js] = (long)line3d.size();
    tedge.insert(tedge.end(), S.tedge.begin(), S.tedge.end());
    tsurf.insert(tsurf.end(), S.ntri, js);
    tyz.insert(tyz.end(), S.tyz.begin(), S.tyz.end());
    line3d.insert(line3d.end(), S.line3d.begin(), S.line3d.end());
    gval.insert(gval.end(), S.gval.begin(), S.gval.end());
    bc2.insert(bc2.end(), S.bc.begin(), S.bc.end());
    const int32_t base = nbr_ptr.back();
    for (int k = 0; k < S.n; ++k) nbr_ptr.push_back(base + S.nbr_ptr[k + 1]);
    nbr.insert(nbr.end(), S.nbr.begin(), S.nbr.end());
  }
  M.tri_off[4] = (long)tsurf.size();
  M.row_off[4] = (long)line3d.size();
  M.tedge.upload(tedge.data(), tedge.size(), s);
  M.tsurf.upload(tsurf.data(), tsurf.size(), s);
  M.tyz.upload(tyz.data(), tyz.size(), s);
  M.line3d.upload(line3d.data(), line3d.size(), s);
  M.gval.upload(gval.data(), gval.size(), s);
  M.bc2.upload(bc2.data(), bc2.size(), s);
  M.nbr_ptr.upload(nbr_ptr.data(), nbr_ptr.size(), s);
  M.nbr.upload(nbr.data(), nbr.size(), s);
  AFEM_CUDA(cudaStreamSynchronize(s));
  M.ready = true;
}

// The 2-D TM systems of the four side surfaces at nf frequencies (system js*nf + f):
// assembly, lifting, Dirichlet rows, L D L^T and the solutions X (row js*nf + f at
// roff).  keep: the band and right-hand side before the factorisation, for export.
struct FaceRun {
  std::vector<BandSys> sys;
  DBuf<BandSys> dsys;
  DBuf<double2> band, rf, X, band0, rf0;
  long nrow = 0;
};

void run_faces(afem_ctx* c, const std::vector<double>& s2tet, int nf, const double* freq, FaceRun& R, bool keep) {
  MtState& M = state(c);
  cudaStream_t s = c->stream;
  const double pi = 4.0 * std::atan(1.0), dmu = 4.0 * pi * 1.0e-7;
  R.sys.clear();
  long boff = 0, roff = 0;
  int maxbw = 0;
  for (int js = 0; js < 4; ++js)
    for (int f = 0; f < nf; ++f) {
      const MtSurface& S = M.s[js];
      BandSys b;
      b.boff = boff;
      b.roff = roff;
      b.lro = M.row_off[js];
      b.n = S.n;
      b.bw = S.bw;
      b.surf = js;
      b.f = f;
      R.sys.push_back(b);
      boff += (long)S.n * (S.bw + 1);
      roff += S.n;
      maxbw = std::max(maxbw, S.bw);
    }
  R.nrow = roff;
  const int nsys = (int)R.sys.size();
  R.dsys.upload(R.sys.data(), nsys, s);
  R.band.alloc(boff);
  R.band.zero(s);
  R.rf.alloc(roff);
  R.X.alloc(roff);
  std::vector<double> om(nf), tsig(M.tri_off[4]);
  for (int f = 0; f < nf; ++f) om[f] = 2.0 * pi * freq[f];
  for (int js = 0; js < 4; ++js)
    for (int q = 0; q < M.s[js].ntri; ++q) tsig[M.tri_off[js] + q] = s2tet[M.s[js].tet[q]];
  DBuf<double> dom, dsig;
  dom.upload(om.data(), nf, s);
  dsig.upload(tsig.data(), tsig.size(), s);
  const long ntri_all = M.tri_off[4];
  k_mt2d_assemble<<<nblk(ntri_all * nf, 128), 128, 0, s>>>(M.tedge.p, M.tyz.p, dsig.p, M.tsurf.p, ntri_all, nf, dom.p,
                                                           dmu, R.dsys.p, R.band.p);
  count_launch();
  int maxn = 0;
  for (int js = 0; js < 4; ++js) maxn = std::max(maxn, M.s[js].n);
  k_mt2d_lift<<<dim3(nblk(maxn, 256), nsys), 256, 0, s>>>(R.dsys.p, R.band.p, M.bc2.p, M.gval.p, M.nbr_ptr.p, M.nbr.p,
                                                          R.rf.p);
  count_launch();
  long maxb = 0;
  for (const auto& b : R.sys) maxb = std::max(maxb, (long)b.n * (b.bw + 1));
  k_mt2d_zero<<<dim3(nblk(maxb, 256), nsys), 256, 0, s>>>(R.dsys.p, M.bc2.p, R.band.p);
  count_launch();
  if (keep) {
    R.band0.alloc(boff);
    R.rf0.alloc(roff);
    AFEM_CUDA(cudaMemcpyAsync(R.band0.p, R.band.p, sizeof(double2) * boff, cudaMemcpyDeviceToDevice, s));
    AFEM_CUDA(cudaMemcpyAsync(R.rf0.p, R.rf.p, sizeof(double2) * roff, cudaMemcpyDeviceToDevice, s));
  }
  const size_t shm = 2 * sizeof(double2) * (size_t)(maxbw + 1);
  AFEM_CUDA(cudaFuncSetAttribute(k_band_ldlt, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)shm));
  cudaEvent_t e0 = nullptr, e1 = nullptr;
  if (c->prof.on) {
    AFEM_CUDA(cudaEventCreate(&e0));
    AFEM_CUDA(cudaEventCreate(&e1));
    AFEM_CUDA(cudaEventRecord(e0, s));
  }
  k_band_ldlt<<<nsys, 512, shm, s>>>(R.dsys.p, R.band.p, R.rf.p, R.X.p, c->status.p);
  count_launch();
  if (c->prof.on) {
    AFEM_CUDA(cudaEventRecord(e1, s));
    AFEM_CUDA(cudaEventSynchronize(e1));
    float ms = 0;
    cudaEventElapsedTime(&ms, e0, e1);
    c->prof.add("mt_band_ldlt", ms);
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
  }
  check_status(c, "mt 2-D TM solve");
}

// GENBCMT for nf frequencies into g[(2f + pol)*nline + e] from the face solutions of R.
void genbc(afem_ctx* c, int nf, const double* freq, const FaceRun& R, double2* g) {
  MtState& M = state(c);
  cudaStream_t s = c->stream;
  const int nline = c->nline;
  const double pi = 4.0 * std::atan(1.0);
  std::vector<double> om(nf);
  for (int f = 0; f < nf; ++f) om[f] = 2.0 * pi * freq[f];
  DBuf<double> dom;
  dom.upload(om.data(), nf, s);
  AFEM_CUDA(cudaMemsetAsync(g, 0, sizeof(double2) * 2L * nf * nline, s));
  k_mt_g_top<<<nblk(nline, 256), 256, 0, s>>>(c->line.p, c->xyz.p, M.lbits.p, nline, nf, dom.p, g);
  count_launch();
  for (int js = 0; js < 4; ++js) {
    const MtSurface& S = M.s[js];
    const BandSys& b0 = R.sys[js * nf];
    const int isr = (js == 0 || js == 2) ? 0 : 1;  // north/south: Ex polarisation, west/east: Ey
    k_mt_g_side<<<nblk(S.n, 256), 256, 0, s>>>(M.line3d.p + M.row_off[js], S.n, S.n, R.X.p + b0.roff, isr, nf, dom.p,
                                               nline, g);
    count_launch();
  }
  k_mt_g_bottom<<<nblk(nline, 256), 256, 0, s>>>(M.lbits.p, nline, nf, g);
  count_launch();
}

constexpr int MT_FREQ_GROUP = 8;  // frequencies whose face systems are held at once

}  // namespace

void mt_destroy(afem_ctx* c) {
  delete c->mt;
  c->mt = nullptr;
}

int mt_forward_device(afem_ctx* c, const afem_mt_cond* cond, int nfreq, const double* freq, int nobs,
                      const double* xyz_obs, const afem_solve_opts* o, double* be, double* z, double* rho,
                      double* pha, afem_solve_stats* st) {
  AFEM_REQUIRE(c->pattern_ready, AFEM_ESTATE, "mt: set the mesh first");
  AFEM_REQUIRE(c->nseg == 0, AFEM_EINVAL, "mt: packed batches are not supported");
  AFEM_REQUIRE(nfreq >= 1 && freq && o, AFEM_EINVAL, "mt: no frequencies or options");
  AFEM_REQUIRE(nobs >= 0 && (nobs == 0 || xyz_obs), AFEM_EINVAL, "mt: bad sites");
  for (int f = 0; f < nfreq; ++f) AFEM_REQUIRE(freq[f] > 0.0, AFEM_EINVAL, "mt: frequencies must be positive");
  cudaStream_t s = c->stream;
  build_surfaces(c);
  MtState& M = state(c);
  std::vector<double> s3, s2;
  resolve_cond(c, cond, s3, s2);
  c->sigma.upload(s3.data(), s3.size(), s);
  c->sigma_set = true;
  const int nline = c->nline, nsys = 2 * nfreq;
  DBuf<double2> G;
  G.alloc((size_t)nsys * nline);
  for (int f0 = 0; f0 < nfreq; f0 += MT_FREQ_GROUP) {
    const int nf = std::min(MT_FREQ_GROUP, nfreq - f0);
    FaceRun R;
    run_faces(c, s2, nf, freq + f0, R, false);
    genbc(c, nf, freq + f0, R, G.p + 2L * f0 * nline);
  }
  const double pi = 4.0 * std::atan(1.0);
  std::vector<double> om(nsys), fs(nsys);
  for (int k = 0; k < nsys; ++k) { fs[k] = freq[k / 2]; om[k] = 2.0 * pi * fs[k]; }
  assemble_dirichlet_device(c, M.bc3.p, nsys, om.data(), G.p);
  invalidate_work(c);
  std::vector<double> hbe;
  double* bev = be;
  if (!bev && (z || rho || pha) && nobs > 0) {
    hbe.resize(2L * 5 * nobs * nsys);
    bev = hbe.data();
  }
  int status = AFEM_OK, its = 0, refs = 0;
  double rrec = 0.0, rtrue = 0.0, secs = 0.0;
  for (int k0 = 0; k0 < nsys;) {
    int ns = 16;
    while (ns > nsys - k0) ns /= 2;
    std::vector<int> src(ns);
    for (int k = 0; k < ns; ++k) src[k] = k0 + k;
    afem_solve_stats sk{};
    const int rc = solve_device(c, ns, fs.data() + k0, src.data(), o, &sk, nullptr);
    if (rc != AFEM_OK && status == AFEM_OK) status = rc;
    its += sk.iterations;
    refs += sk.refinements;
    rrec = std::max(rrec, sk.resid_recursive);
    rtrue = std::max(rtrue, sk.resid_true);
    secs += sk.seconds;
    if (bev && nobs > 0) sites_device(c, nobs, xyz_obs, bev + 2L * 5 * nobs * k0);
    k0 += ns;
  }
  // CALRESPMT (n_ebfem_3DMT.f90:179-237)
  if (bev && nobs > 0 && (z || rho || pha)) {
    const double dmu = 4.0 * pi * 1.0e-7, r2d = 180.0 / pi;
    typedef std::complex<double> cx;
    const cx* B = reinterpret_cast<const cx*>(bev);
    for (int f = 0; f < nfreq; ++f) {
      const double omega = 2.0 * pi * freq[f];
      for (int j = 0; j < nobs; ++j) {
        auto ex = [&](int cc) { return B[((2L * f + 0) * 5 + cc) * nobs + j]; };
        auto ey = [&](int cc) { return B[((2L * f + 1) * 5 + cc) * nobs + j]; };
        const cx a = ex(0), cc = ex(1), b = ey(0), d = ey(1);
        const cx det = a * d - b * cc;
        cx bi[2][2] = {{d, -b}, {-cc, a}};
        for (int p = 0; p < 2; ++p)
          for (int q = 0; q < 2; ++q) bi[p][q] = bi[p][q] / det;
        const cx e[2][2] = {{ex(3), ey(3)}, {ex(4), ey(4)}};
        cx zz[4];
        for (int p = 0; p < 2; ++p)
          for (int q = 0; q < 2; ++q) zz[2 * p + q] = e[p][0] * bi[0][q] + e[p][1] * bi[1][q];
        const double coef = dmu / omega * 1.0e6;
        for (int k = 0; k < 4; ++k) {
          const long oi = (4L * f + k) * nobs + j;
          if (z) { z[2 * oi] = zz[k].real(); z[2 * oi + 1] = zz[k].imag(); }
          const double amp = std::sqrt(std::pow(zz[k].real(), 2.0) + std::pow(zz[k].imag(), 2.0));
          if (rho) rho[oi] = coef * std::pow(amp, 2.0);
          if (pha) pha[oi] = std::atan2(zz[k].imag(), zz[k].real()) * r2d;
        }
      }
    }
  }
  if (st) {
    st->iterations = its;
    st->refinements = refs;
    st->resid_recursive = rrec;
    st->resid_true = rtrue;
    st->seconds = secs;
    st->status = status;
  }
  return status;
}

void mt_boundary_device(afem_ctx* c, const afem_mt_cond* cond, double freq, double* av, uint8_t* bc) {
  AFEM_REQUIRE(c->pattern_ready, AFEM_ESTATE, "mt: set the mesh first");
  AFEM_REQUIRE(freq > 0.0, AFEM_EINVAL, "mt: the frequency must be positive");
  build_surfaces(c);
  MtState& M = state(c);
  std::vector<double> s3, s2;
  resolve_cond(c, cond, s3, s2);
  FaceRun R;
  run_faces(c, s2, 1, &freq, R, false);
  DBuf<double2> G;
  G.alloc(2L * c->nline);
  genbc(c, 1, &freq, R, G.p);
  cudaStream_t s = c->stream;
  if (av) G.download(reinterpret_cast<double2*>(av), 2L * c->nline, s);
  if (bc) M.bc3.download(bc, c->nline, s);
  AFEM_CUDA(cudaStreamSynchronize(s));
}

void mt_face_device(afem_ctx* c, const afem_mt_cond* cond, int j, double freq, int* n, long* nnz, int32_t* line3d,
                    int32_t* rowptr, int32_t* col, double* val, double* rhs, double* bs) {
  AFEM_REQUIRE(c->pattern_ready, AFEM_ESTATE, "mt: set the mesh first");
  AFEM_REQUIRE(j >= 2 && j <= 5, AFEM_EINVAL, "mt: side surfaces are 2..5");
  AFEM_REQUIRE(freq > 0.0, AFEM_EINVAL, "mt: the frequency must be positive");
  build_surfaces(c);
  MtState& M = state(c);
  const MtSurface& S = M.s[j - 2];
  long nz = S.n;
  for (int k = 0; k < S.n; ++k) nz += S.nbr_ptr[k + 1] - S.nbr_ptr[k];
  if (n) *n = S.n;
  if (nnz) *nnz = nz;
  if (!line3d) return;
  AFEM_REQUIRE(rowptr && col && val && rhs && bs, AFEM_EINVAL, "mt face: null output");
  std::vector<double> s3, s2;
  resolve_cond(c, cond, s3, s2);
  FaceRun R;
  run_faces(c, s2, 1, &freq, R, true);
  cudaStream_t s = c->stream;
  const BandSys& b = R.sys[j - 2];  // nf = 1: system js
  const int ld = b.bw + 1;
  std::vector<double2> band((size_t)b.n * ld), r0(b.n), x(b.n);
  AFEM_CUDA(cudaMemcpyAsync(band.data(), R.band0.p + b.boff, sizeof(double2) * band.size(), cudaMemcpyDeviceToHost,
                            s));
  AFEM_CUDA(cudaMemcpyAsync(r0.data(), R.rf0.p + b.roff, sizeof(double2) * b.n, cudaMemcpyDeviceToHost, s));
  AFEM_CUDA(cudaMemcpyAsync(x.data(), R.X.p + b.roff, sizeof(double2) * b.n, cudaMemcpyDeviceToHost, s));
  AFEM_CUDA(cudaStreamSynchronize(s));
  std::copy(S.line3d.begin(), S.line3d.end(), line3d);
  long p = 0;
  rowptr[0] = 0;
  for (int r = 0; r < S.n; ++r) {
    std::vector<int> cols(S.nbr.begin() + S.nbr_ptr[r], S.nbr.begin() + S.nbr_ptr[r + 1]);
    cols.push_back(r);
    std::sort(cols.begin(), cols.end());
    for (int cc : cols) {
      const int hi = std::max(r, cc), lo = std::min(r, cc);
      const double2 v = band[(size_t)lo * ld + (hi - lo)];
      col[p] = cc;
      val[2 * p] = v.x;
      val[2 * p + 1] = v.y;
      ++p;
    }
    rowptr[r + 1] = (int32_t)p;
    rhs[2 * r] = r0[r].x;
    rhs[2 * r + 1] = r0[r].y;
    bs[2 * r] = x[r].x;
    bs[2 * r + 1] = x[r].y;
  }
}

}  // namespace afem
