// CPU oracle for the ActFEMtide tidal forward path -- TEST INFRASTRUCTURE ONLY.
//
// A statement-by-statement C++ restatement of the reference's Fortran path,
// used by tests/ (as the parity checker) and by bench.py (the timed CPU
// baseline).  Nothing in the product library links or calls this file.
//
// Parity status: the reference ships no tests, golden vectors or data for
// this path and cannot be compiled here (Fortran + MKL), so this oracle is
// pinned only by the two known-answer examples the reference carries in its
// sources (SORT_INDEX, src/solver/sort_index.f90:3-10; the CRS product of
// src/common/test.f90:5-20), by the reference-shipped tide files
// (src/src_tide/{f,v}xyz_mesh, parsed by the product readers) and by
// mathematical identities (curl-curl annihilates discrete gradients, direct
// solves).  Parity against the reference itself is therefore "unpinned".
//
// Conventions: node / edge / tetrahedron ids are 1-based exactly as in the
// reference; arrays that are 2-D in Fortran are passed row-major by element
// (n4[t*4+k] = n4(t+1,k+1), n6line[t*6+j] = n6line(t+1,j+1),
// xyz[3*(i-1)+c] = xyz(c+1,i)); complex arrays are interleaved (re, im).
// Compile with -ffp-contract=off: the reference is built for AVX without FMA
// (src/solver_mpi/Makefile:8), so products and sums round separately.

#include <cmath>
#include <complex>
#include <cstdint>
#include <cstring>
#include <vector>
#include <algorithm>

typedef std::complex<double> cplx;

namespace {

// edge table kl (src/solver/m_fem_edge_util.f90:5-11), 1-based local nodes
const int KL[6][2] = {{1, 2}, {2, 3}, {1, 3}, {1, 4}, {2, 4}, {3, 4}};
// face table lmn (m_fem_edge_util.f90:13-17)
const int LMN[4][3] = {{2, 3, 4}, {1, 4, 3}, {1, 2, 4}, {1, 3, 2}};
// rotation matrix C(4,6) (m_fem_edge_util.f90:19-23)
const int CROT[4][6] = {{0, 1, 0, 0, -1, 1}, {0, 0, -1, 1, 0, -1}, {1, 0, 0, -1, 1, 0}, {-1, -1, 1, 0, 0, 0}};

inline double PI() { return 4.0 * std::atan(1.0); }      // constants :: pi (m_constants.f90:6)
inline double DMU() { return 4.0 * PI() * 1.0e-7; }     // constants :: dmu (m_constants.f90:9)

struct V3 { double x[3]; };
inline V3 sub(const double* a, const double* b) { return V3{{a[0] - b[0], a[1] - b[1], a[2] - b[2]}}; }
inline V3 neg(const V3& a) { return V3{{-a.x[0], -a.x[1], -a.x[2]}}; }
// outer / inner (src/common/m_outerinnerproduct.f90:4-19)
inline V3 outer(const V3& a, const V3& b) {
  return V3{{a.x[1] * b.x[2] - a.x[2] * b.x[1], a.x[2] * b.x[0] - a.x[0] * b.x[2], a.x[0] * b.x[1] - a.x[1] * b.x[0]}};
}
inline double inner(const V3& a, const V3& b) { return a.x[0] * b.x[0] + a.x[1] * b.x[1] + a.x[2] * b.x[2]; }
inline V3 scale(double c, const V3& a) { return V3{{c * a.x[0], c * a.x[1], c * a.x[2]}}; }

// volume (src/solver/m_fem_util.f90:101-109)
inline double volume(const V3& a, const V3& b, const V3& c) { return 1.0 / 6.0 * inner(outer(a, b), c); }

// calxmn (m_fem_util.f90:42-53): xx(:,1..6)
inline void calxmn(const double e[4][3], V3 xx[6]) {
  xx[0] = sub(e[3], e[2]);
  xx[1] = sub(e[3], e[0]);
  xx[2] = sub(e[1], e[3]);
  xx[3] = sub(e[2], e[1]);
  xx[4] = sub(e[0], e[2]);
  xx[5] = sub(e[1], e[0]);
}

// gradnodebasisfun (m_fem_util.f90:12-40).  Returns false for v <= 0 (the reference stops).
inline bool gradnodebasisfun(const double e[4][3], V3 gn[4], double* v) {
  V3 xx[6];
  calxmn(e, xx);
  *v = volume(xx[0], xx[4], neg(xx[3]));
  if (*v <= 0) return false;
  const double c = 1.0 / 6.0 / *v;
  gn[0] = scale(c, outer(sub(e[3], e[1]), sub(e[2], e[1])));
  gn[1] = scale(c, outer(sub(e[2], e[0]), sub(e[3], e[0])));
  gn[2] = scale(c, outer(sub(e[3], e[0]), sub(e[1], e[0])));
  gn[3] = scale(c, outer(sub(e[1], e[0]), sub(e[2], e[0])));
  return true;
}

// intv (m_fem_util.f90:86-96), k/m 1-based
inline double intv(int k, int m, double v) { return (k != m) ? v / 20.0 : v / 10.0; }

// nodebasisfun (m_fem_util.f90:56-83)
inline void nodebasisfun(const double e[4][3], const double x3[3], double a[4]) {
  V3 v[4];
  for (int j = 0; j < 4; ++j) v[j] = sub(e[j], x3);
  V3 x12 = sub(e[1], e[0]), x13 = sub(e[2], e[0]), x14 = sub(e[3], e[0]);
  V3 x24 = sub(e[3], e[1]), x23 = sub(e[2], e[1]);
  double a5 = volume(x12, x13, x14);
  double a4 = volume(x12, x13, neg(v[0])) / a5;
  double a3 = volume(x14, x12, neg(v[0])) / a5;
  double a2 = volume(x13, x14, neg(v[0])) / a5;
  double a1 = volume(x24, x23, neg(v[1])) / a5;
  a[0] = a1; a[1] = a2; a[2] = a3; a[3] = a4;
}

inline void load_tet(const double* xyz, const int* n4, long t, double e[4][3]) {
  for (int j = 0; j < 4; ++j) {
    const double* p = xyz + 3 * (long)(n4[t * 4 + j] - 1);
    e[j][0] = p[0]; e[j][1] = p[1]; e[j][2] = p[2];
  }
}

// SORT_INDEX (src/solver/sort_index.f90:13-56): heap sort of RA carrying NA.
void sort_index(int n, int* na, double* ra) {
  // 1-based views
  int* NA = na - 1;
  double* RA = ra - 1;
  if (n < 2) return;
  int L = n / 2 + 1, IR = n, I, J;
  double RRA; int IIA;
  for (;;) {
    if (L > 1) {
      L = L - 1; RRA = RA[L]; IIA = NA[L];
    } else {
      RRA = RA[IR]; IIA = NA[IR];
      RA[IR] = RA[1]; NA[IR] = NA[1];
      IR = IR - 1;
      if (IR == 1) { RA[1] = RRA; NA[1] = IIA; return; }
    }
    I = L; J = L + L;
    while (J <= IR) {
      if (J < IR) { if (RA[J] < RA[J + 1]) J = J + 1; }
      if (RRA < RA[J]) { RA[I] = RA[J]; NA[I] = NA[J]; I = J; J = J + J; }
      else J = IR + 1;
    }
    RA[I] = RRA; NA[I] = IIA;
  }
}

}  // namespace

extern "C" {

int orc_version() { return 1; }

void orc_sort_index(int n, int* na, double* ra) { sort_index(n, na, ra); }

// mul_matcrs_cv (src/common/m_matrix.f90:83-102): vout = crs * cv, 1-based items.
void orc_mul_matcrs_cv(int nrow, const int* stack, const int* item, const double* val, const double* cv,
                       double* vout) {
  const cplx* x = reinterpret_cast<const cplx*>(cv);
  cplx* y = reinterpret_cast<cplx*>(vout);
  for (int r = 0; r < nrow; ++r) {
    cplx s(0.0, 0.0);
    for (int j = stack[r]; j < stack[r + 1]; ++j) s = s + val[j] * x[item[j] - 1];
    y[r] = s;
  }
}

// MKLINE_V2 + MKN6 (tmtgem/common/m_line_type.f90:120-222, 224-277).
// Edges grouped by their smaller node n1 ascending; inside a group, in order
// of first encounter scanning the tetrahedra that contain n1 by ascending id
// and their local nodes 1..4.  n6line(t,j) = +-id, sign = orientation of kl(j).
// Returns nline, or -1 if a node is shared by more than maxnele=100
// tetrahedra, -2 if cap is too small, -3 if an edge is missing.
long orc_mkline(int node, long ntet, const int* n4, long cap, int* line, int* n6line) {
  const int maxnele = 100;
  std::vector<int> nele(node + 1, 0);
  std::vector<long> node2ele((size_t)maxnele * (node + 1));
  for (long i = 0; i < ntet; ++i)
    for (int j = 0; j < 4; ++j) {
      int n1 = n4[i * 4 + j];
      if (nele[n1] == maxnele) return -1;
      nele[n1]++;
      node2ele[(size_t)maxnele * n1 + nele[n1] - 1] = i;
    }
  std::vector<long> stack(node + 1, 0);
  std::vector<int> item;
  item.reserve((size_t)ntet * 2);
  long nline = 0;
  for (int n1 = 1; n1 <= node; ++n1) {
    stack[n1] = stack[n1 - 1];
    for (int j = 0; j < nele[n1]; ++j) {
      long iele = node2ele[(size_t)maxnele * n1 + j];
      for (int k = 0; k < 4; ++k) {
        int n2 = n4[iele * 4 + k];
        if (n2 <= n1) continue;
        bool found = false;
        for (long l = stack[n1 - 1]; l < stack[n1]; ++l)
          if (item[l] == n2) { found = true; break; }
        if (found) continue;
        stack[n1]++;
        item.push_back(n2);
        nline++;
      }
    }
  }
  if (nline > cap) return -2;
  for (int i = 1; i <= node; ++i)
    for (long j = stack[i - 1]; j < stack[i]; ++j) { line[2 * j] = i; line[2 * j + 1] = item[j]; }
  for (long i = 0; i < ntet; ++i)
    for (int j = 0; j < 6; ++j) {
      int n11 = n4[i * 4 + KL[j][0] - 1], n12 = n4[i * 4 + KL[j][1] - 1], dir = 1;
      if (n11 > n12) { std::swap(n11, n12); dir = -1; }
      long id = -1;
      for (long k = stack[n11 - 1]; k < stack[n11]; ++k)
        if (item[k] == n12) { id = k + 1; break; }
      if (id < 0) return -3;
      n6line[i * 6 + j] = (int)(dir * id);
    }
  return nline;
}

// set_iccg_var7_dofn / C_set_dof2 (src/solver/m_iccg_var_takuto.f90:277-485)
// with table_dof = identity (n_ebfem_bxyz_mpi.f90:104-107).  Strictly upper
// (IAU) and strictly lower (IAL) column lists per row, ascending, built by the
// reference's search-then-insert.  INU/INL hold n+1 prefix counts (INU[0]=0),
// IAU/IAL 1-based columns.  Call with IAU==NULL to get the counts only.
// Returns iau_tot (== ial_tot), or -1 when a row exceeds max_inum = 1000.
long orc_pattern(int n, long ntet, const int* n6line, int* INU, int* INL, int* IAU, int* IAL) {
  const int max_inum = 1000;
  std::vector<std::vector<int>> up(n + 1), lo(n + 1);
  for (long elm = 0; elm < ntet; ++elm) {
    int dof[6];
    for (int j = 0; j < 6; ++j) dof[j] = std::abs(n6line[elm * 6 + j]);
    for (int kf = 0; kf < 6; ++kf) {
      int i = dof[kf];
      for (int lf = 0; lf < 6; ++lf) {
        int j = dof[lf];
        if (i == j) continue;
        std::vector<int>& row = (i < j) ? up[i] : lo[i];
        bool exist = false;
        for (size_t num = 0; num < row.size(); ++num) {
          if (j == row[num]) { exist = true; break; }
          else if (j < row[num]) break;
        }
        if (exist) continue;
        if ((int)row.size() + 1 > max_inum) return -1;
        size_t pos = row.size();
        for (size_t num = 0; num < row.size(); ++num)
          if (j < row[num]) { pos = num; break; }
        row.insert(row.begin() + pos, j);
      }
    }
  }
  INU[0] = 0; INL[0] = 0;
  for (int i = 1; i <= n; ++i) {
    INU[i] = INU[i - 1] + (int)up[i].size();
    INL[i] = INL[i - 1] + (int)lo[i].size();
  }
  if (IAU && IAL)
    for (int i = 1; i <= n; ++i) {
      std::copy(up[i].begin(), up[i].end(), IAU + INU[i - 1]);
      std::copy(lo[i].begin(), lo[i].end(), IAL + INL[i - 1]);
    }
  return INU[n];
}

// Conductivity per tetrahedron as GENMAT selects it (forward_bxyz_mpi.f90:196-208):
// tag 1 -> sigma_air; 2 -> sigma_ocean (the reference hard-codes the default-real
// literal 3.33); >=3 -> sigma_land(tag-1) for condflag 0, sigma(iele-nphys1) for
// condflag 1.  Returns 0, or -(t+1) for a tetrahedron whose tag selects nothing.
long orc_resolve_sigma(long ntet, const int* tag, double sigma_air, double sigma_ocean, int condflag, int nvolume,
                       const double* sigma_land, long nphys1, const double* sigma_file, double* sigma_tet) {
  for (long t = 0; t < ntet; ++t) {
    int j = tag[t];
    if (j == 1) sigma_tet[t] = sigma_air;
    else if (j == 2) sigma_tet[t] = sigma_ocean;
    else if (j >= 3) {
      if (condflag == 0) {
        if (j - 1 > nvolume) return -(t + 1);
        sigma_tet[t] = sigma_land[j - 2];
      } else {
        if (t + 1 - nphys1 < 1) return -(t + 1);
        sigma_tet[t] = sigma_file[t - nphys1];
      }
    } else return -(t + 1);
  }
  return 0;
}

// INITIALIZE + GENMAT + COPY_UL_ICCG12 + GENBCCSEM + SET_BC_ICCG for one
// frequency (forward_bxyz_mpi.f90:42-58, 99-311, 467-519, 567-636;
// m_iccg_var_takuto.f90:23-37, 107-167).  sup_iccg's linear row search
// (forward_bxyz_mpi.f90:642-699) scatters into D and AU.  Source: fxyz/vxyz
// hold nodes 1..nodes, later nodes are zero (m_readfvxyz.f90:21,47).
// Returns 0; -1 non-positive volume (tet id in *bad); -2 dof not found;
// -3 copy_ul mismatch.
int orc_forward_assemble(int node, const double* xyz, long ntet, const int* n4, const int* tag, int nline,
                         const int* line, const int* n6line, const int* INU, const int* IAU, const int* INL,
                         const int* IAL, const double* sigma_tet, int nodes, const double* F, const double* vc,
                         double freq, double zmin, double zmax, double xout, double yout, int apply_bc,
                         double* D_, double* AU_, double* AL_, double* b_, unsigned char* bc_flag, long* bad) {
  const double pi = PI(), dmu = DMU();
  const double omega = 2.0 * pi * freq;
  const double L0 = 1.0e3;
  cplx* D = reinterpret_cast<cplx*>(D_);
  cplx* AU = reinterpret_cast<cplx*>(AU_);
  cplx* AL = reinterpret_cast<cplx*>(AL_);
  cplx* b = reinterpret_cast<cplx*>(b_);
  const long iau_tot = INU[nline];
  for (int i = 0; i < nline; ++i) { D[i] = 0.0; b[i] = 0.0; }
  for (long i = 0; i < iau_tot; ++i) { AU[i] = 0.0; AL[i] = 0.0; }
  const cplx* v = reinterpret_cast<const cplx*>(vc);
  const cplx iunit(0.0, 1.0);
  for (long iele = 0; iele < ntet; ++iele) {
    int idir[6];
    for (int j = 0; j < 6; ++j) idir[j] = (n6line[iele * 6 + j] < 0) ? -1 : 1;
    double e[4][3];
    load_tet(xyz, n4, iele, e);
    V3 xx[6], gn[4];
    double vol;
    calxmn(e, xx);
    if (!gradnodebasisfun(e, gn, &vol)) { if (bad) *bad = iele + 1; return -1; }
    const double AA = 1.0 / 9.0 / vol;
    double S[6][6];
    for (int j = 0; j < 6; ++j)
      for (int k = 0; k < 6; ++k) S[j][k] = inner(xx[j], xx[k]) * idir[j] * idir[k] * AA;
    const double sigma = sigma_tet[iele];
    const cplx BB = iunit * omega * dmu * sigma * std::pow(L0, 2.0);
    cplx elm_k[6][6];
    for (int i = 0; i < 6; ++i)
      for (int j = 0; j < 6; ++j) {
        int k = KL[i][0], l = KL[i][1], m = KL[j][0], n = KL[j][1];
        double yy = intv(k, m, vol) * inner(gn[l - 1], gn[n - 1]) - intv(k, n, vol) * inner(gn[l - 1], gn[m - 1]) -
                    intv(l, m, vol) * inner(gn[k - 1], gn[n - 1]) + intv(l, n, vol) * inner(gn[k - 1], gn[m - 1]);
        cplx S1 = (yy * idir[i] * idir[j]) * BB;
        elm_k[i][j] = S[i][j] + S1;
      }
    // sup_iccg
    int tdof[6];
    for (int i = 0; i < 6; ++i) tdof[i] = n6line[iele * 6 + i] * idir[i];
    for (int ie = 0; ie < 6; ++ie) {
      int igl = tdof[ie];
      for (int je = 0; je < 6; ++je) {
        int jgl = tdof[je];
        if (igl == jgl) D[igl - 1] += elm_k[ie][je];
        else if (igl < jgl) {
          long pos = -1;
          for (int num = INU[igl - 1]; num < INU[igl]; ++num)
            if (jgl == IAU[num]) { pos = num; break; }
          if (pos < 0) { if (bad) *bad = iele + 1; return -2; }
          if (ie > je) AU[pos] += elm_k[ie][je];
          else AU[pos] += elm_k[je][ie];
        }
      }
    }
    // right-hand side, ocean tetrahedra only (forward_bxyz_mpi.f90:267-299)
    cplx S2[6] = {0.0, 0.0, 0.0, 0.0, 0.0, 0.0};
    if (tag[iele] == 2) {
      cplx vF[4][3];
      for (int i = 0; i < 4; ++i) {
        int no = n4[iele * 4 + i];
        double Fv[3] = {0.0, 0.0, 0.0};
        cplx vv[3] = {0.0, 0.0, 0.0};
        if (no <= nodes) {
          for (int c = 0; c < 3; ++c) { Fv[c] = F[3 * (no - 1) + c]; vv[c] = v[3 * (no - 1) + c]; }
        }
        // cr_outer (m_outerinnerproduct.f90:52-60)
        vF[i][0] = vv[1] * Fv[2] - vv[2] * Fv[1];
        vF[i][1] = vv[2] * Fv[0] - vv[0] * Fv[2];
        vF[i][2] = vv[0] * Fv[1] - vv[1] * Fv[0];
      }
      for (int i = 0; i < 6; ++i) {
        int k = KL[i][0], l = KL[i][1];
        for (int j = 1; j <= 4; ++j) {
          // rc_inner (m_outerinnerproduct.f90:78-84)
          cplx gl = gn[l - 1].x[0] * vF[j - 1][0] + gn[l - 1].x[1] * vF[j - 1][1] + gn[l - 1].x[2] * vF[j - 1][2];
          cplx gk = gn[k - 1].x[0] * vF[j - 1][0] + gn[k - 1].x[1] * vF[j - 1][1] + gn[k - 1].x[2] * vF[j - 1][2];
          S2[i] = S2[i] + dmu * sigma * (intv(k, j, vol) * gl - intv(l, j, vol) * gk) * (double)idir[i] * 1.0e3;
        }
      }
    }
    for (int i = 0; i < 6; ++i) {
      int ii = n6line[iele * 6 + i] * idir[i];
      b[ii - 1] = b[ii - 1] + S2[i];
    }
  }
  // COPY_UL_ICCG12
  {
    std::vector<char> assigned(iau_tot, 0);
    for (int igl = 1; igl <= nline; ++igl)
      for (int num = INU[igl - 1]; num < INU[igl]; ++num) {
        int jgl = IAU[num];
        long pos = -1;
        for (int num2 = INL[jgl - 1]; num2 < INL[jgl]; ++num2)
          if (igl == IAL[num2]) { pos = num2; break; }
        if (pos < 0) return -3;
        AL[pos] = AU[num];
        assigned[pos] = 1;
      }
    for (long i = 0; i < INL[nline]; ++i)
      if (!assigned[i]) return -3;
  }
  // GENBCCSEM
  const double xout1 = xout - 1.0, yout1 = yout - 1.0, zmin1 = zmin + 1.0, zmax1 = zmax - 1.0;
  for (int i = 0; i < nline; ++i) {
    const double* p1 = xyz + 3 * (long)(line[2 * i] - 1);
    const double* p2 = xyz + 3 * (long)(line[2 * i + 1] - 1);
    int g = 0;
    if (p1[0] <= -xout1 && p2[0] <= -xout1) g = 3;
    else if (p1[0] >= xout1 && p2[0] >= xout1) g = 5;
    else if (p1[1] <= -yout1 && p2[1] <= -yout1) g = 4;
    else if (p1[1] >= yout1 && p2[1] >= yout1) g = 2;
    else if (p1[2] <= zmin1 && p2[2] <= zmin1) g = 6;
    else if (p1[2] >= zmax1 && p2[2] >= zmax1) g = 1;
    bc_flag[i] = (g != 0);
  }
  if (!apply_bc) return 0;
  // SET_BC_ICCG with Dirichlet value 0, one source column
  for (int i = 0; i < nline; ++i) {
    if (bc_flag[i]) b[i] = 0.0;
    else {
      cplx temp = D[i] * cplx(0.0, 0.0);
      for (int p = INL[i]; p < INL[i + 1]; ++p) temp = temp + AL[p] * cplx(0.0, 0.0);
      for (int p = INU[i]; p < INU[i + 1]; ++p) temp = temp + AU[p] * cplx(0.0, 0.0);
      b[i] = b[i] - temp;
    }
  }
  for (int i = 0; i < nline; ++i) {
    if (bc_flag[i]) {
      D[i] = 1.0;
      for (int p = INL[i]; p < INL[i + 1]; ++p) AL[p] = 0.0;
      for (int p = INU[i]; p < INU[i + 1]; ++p) AU[p] = 0.0;
    } else {
      for (int p = INL[i]; p < INL[i + 1]; ++p)
        if (bc_flag[IAL[p] - 1]) AL[p] = 0.0;
      for (int p = INU[i]; p < INU[i + 1]; ++p)
        if (bc_flag[IAU[p] - 1]) AU[p] = 0.0;
    }
  }
  return 0;
}

// Split assembly used to check the product's frequency-independent storage:
// K (curl-curl, real) and Msig (sigma-weighted mass times mu0*L0^2, real),
// with A(omega) = K + i*omega*Msig, in the same D/AU layout.
int orc_assemble_split(long ntet, const double* xyz, const int* n4, const int* n6line, int nline, const int* INU,
                       const int* IAU, const double* sigma_tet, double* Kd, double* Ku, double* Md, double* Mu) {
  const double dmu = DMU(), L0 = 1.0e3;
  const long tot = INU[nline];
  std::fill(Kd, Kd + nline, 0.0); std::fill(Md, Md + nline, 0.0);
  std::fill(Ku, Ku + tot, 0.0); std::fill(Mu, Mu + tot, 0.0);
  for (long iele = 0; iele < ntet; ++iele) {
    int idir[6];
    for (int j = 0; j < 6; ++j) idir[j] = (n6line[iele * 6 + j] < 0) ? -1 : 1;
    double e[4][3];
    load_tet(xyz, n4, iele, e);
    V3 xx[6], gn[4];
    double vol;
    calxmn(e, xx);
    if (!gradnodebasisfun(e, gn, &vol)) return -1;
    const double AA = 1.0 / 9.0 / vol;
    const double ms = dmu * sigma_tet[iele] * L0 * L0;
    for (int ie = 0; ie < 6; ++ie)
      for (int je = 0; je < 6; ++je) {
        int gi = std::abs(n6line[iele * 6 + ie]), gj = std::abs(n6line[iele * 6 + je]);
        if (gi > gj) continue;
        // sup_iccg adds elm_k(max(ie,je), min(ie,je)) to the upper entry
        const int i = std::max(ie, je), j = std::min(ie, je);
        int k = KL[i][0], l = KL[i][1], m = KL[j][0], n = KL[j][1];
        double s = inner(xx[i], xx[j]) * idir[i] * idir[j] * AA;
        double yy = intv(k, m, vol) * inner(gn[l - 1], gn[n - 1]) - intv(k, n, vol) * inner(gn[l - 1], gn[m - 1]) -
                    intv(l, m, vol) * inner(gn[k - 1], gn[n - 1]) + intv(l, n, vol) * inner(gn[k - 1], gn[m - 1]);
        double mm = yy * idir[i] * idir[j] * ms;
        if (gi == gj) { Kd[gi - 1] += s; Md[gi - 1] += mm; }
        else {
          long pos = -1;
          for (int num = INU[gi - 1]; num < INU[gi]; ++num)
            if (gj == IAU[num]) { pos = num; break; }
          if (pos < 0) return -2;
          Ku[pos] += s; Mu[pos] += mm;
        }
      }
  }
  return 0;
}

}  // extern "C"

namespace {

// COCG13_single (src/solver/COCG13_single.f90:9-340) as a resumable run: the
// set-up (NSET scaling, DD, initial residual, ||b||^2), one iteration at a time,
// and the final unscaling.  orc_cocg13_single drives it exactly as the
// reference's DO loop; orc_cocg_begin/advance/end let a caller time the same
// iterations in slices (the Krylov state carries over between slices).
struct CocgRun {
  int NP = 0;
  cplx *D = nullptr, *AL = nullptr, *AU = nullptr, *B = nullptr, *X = nullptr;
  const int *INL = nullptr, *IAL = nullptr, *INU = nullptr, *IAU = nullptr;
  bool ic = false, ssor = false, diag = false;
  std::vector<cplx> R, Z, P, DD;
  std::vector<double> SCALE;
  double BNRM2 = 0.0;
  cplx RHO1 = 0.0;
  int iter = 0;  // iterations done

  // COCG13_single.f90:80-180: NSET 2 scaling (in place), DD, R = B - A X, ||B||^2
  void setup(const char* PRECOND, double SIGMA_DIAG, double SIGMA, int NSET) {
    R.assign(NP, 0.0);
    Z.assign(NP, 0.0);
    P.assign(NP, 0.0);
    DD.assign(NP, 0.0);
    SCALE.assign(NP, 1.0);
    ic = (std::strncmp(PRECOND, "IC", 2) == 0) || (std::strncmp(PRECOND, "ILU", 3) == 0);
    ssor = std::strncmp(PRECOND, "SSOR", 4) == 0;
    diag = std::strncmp(PRECOND, "DIAG", 4) == 0;
    if (NSET >= 1) {
      if (NSET == 2) {
        for (int i = 0; i < NP; ++i) SCALE[i] = 1.0 / std::sqrt(std::abs(D[i]));
        for (int j = 0; j < NP; ++j) {
          D[j] = std::abs(D[j]) / D[j];
          for (int i = INU[j]; i < INU[j + 1]; ++i) AU[i] = AU[i] * SCALE[IAU[i] - 1] * SCALE[j];
          for (int i = INL[j]; i < INL[j + 1]; ++i) AL[i] = AL[i] * SCALE[IAL[i] - 1] * SCALE[j];
        }
      }
      for (int i = 0; i < NP; ++i) B[i] = B[i] * SCALE[i];
      for (int i = 0; i < NP; ++i) DD[i] = 0.0;
      if (ic) {
        for (int i = 0; i < NP; ++i) {
          cplx W = D[i] * SIGMA_DIAG;
          for (int k = INL[i]; k < INL[i + 1]; ++k) {
            cplx SS = AL[k];
            int id = IAL[k];
            for (int kk = INU[id - 1]; kk < INU[id]; ++kk) SS = SS + AU[kk] * SIGMA;
            W = W - AL[k] * SS * DD[id - 1];
          }
          DD[i] = cplx(1.0, 0.0) / W;
        }
      }
      if (ssor || diag)
        for (int i = 0; i < NP; ++i) DD[i] = cplx(1.0, 0.0) / (SIGMA_DIAG * D[i]);
    }
    for (int j = 0; j < NP; ++j) {
      cplx W = B[j] - D[j] * X[j];
      for (int i = INU[j]; i < INU[j + 1]; ++i) W = W - AU[i] * X[IAU[i] - 1];
      for (int i = INL[j]; i < INL[j + 1]; ++i) W = W - AL[i] * X[IAL[i] - 1];
      R[j] = W;
    }
    BNRM2 = 0.0;
    for (int i = 0; i < NP; ++i) BNRM2 = BNRM2 + (B[i] * std::conj(B[i])).real();
  }

  // One pass of the DO loop body (COCG13_single.f90:195-330); returns RESID.
  double step() {
    ++iter;
    std::vector<cplx>& Q = Z;  // Q shares the Z column (COCG13_single.f90:64-67)
    for (int i = 0; i < NP; ++i) Z[i] = R[i];
    if (ic || ssor) {
      for (int i = 0; i < NP; ++i) {
        cplx W = R[i];
        for (int j = INL[i]; j < INL[i + 1]; ++j) W = W - AL[j] * Z[IAL[j] - 1];
        Z[i] = W * DD[i];
      }
      for (int i = NP - 1; i >= 0; --i) {
        cplx SW(0.0, 0.0);
        for (int j = INU[i]; j < INU[i + 1]; ++j) SW = SW + AU[j] * Z[IAU[j] - 1];
        Z[i] = Z[i] - DD[i] * SW;
      }
    }
    if (diag)
      for (int i = 0; i < NP; ++i) Z[i] = R[i] * DD[i];
    cplx RHO0(0.0, 0.0);
    for (int i = 0; i < NP; ++i) RHO0 = RHO0 + R[i] * Z[i];
    const cplx RHO = RHO0;
    if (iter == 1) {
      for (int i = 0; i < NP; ++i) P[i] = Z[i];
    } else {
      cplx BETA = RHO / RHO1;
      for (int i = 0; i < NP; ++i) P[i] = Z[i] + BETA * P[i];
    }
    for (int j = 0; j < NP; ++j) {
      cplx W = D[j] * P[j];
      for (int i = INU[j]; i < INU[j + 1]; ++i) W = W + AU[i] * P[IAU[i] - 1];
      for (int i = INL[j]; i < INL[j + 1]; ++i) W = W + AL[i] * P[IAL[i] - 1];
      Q[j] = W;
    }
    cplx C10(0.0, 0.0);
    for (int i = 0; i < NP; ++i) C10 = C10 + P[i] * Q[i];
    const cplx ALPHA = RHO / C10;
    for (int i = 0; i < NP; ++i) {
      X[i] = X[i] + ALPHA * P[i];
      R[i] = R[i] - ALPHA * Q[i];
    }
    double DNRM2 = 0.0;
    for (int i = 0; i < NP; ++i) DNRM2 = DNRM2 + (R[i] * std::conj(R[i])).real();
    RHO1 = RHO;
    return std::sqrt(DNRM2 / BNRM2);
  }

  // COCG13_single.f90:332-338: X and B back to the unscaled system
  void finish() {
    for (int i = 0; i < NP; ++i) {
      X[i] = X[i] * SCALE[i];
      B[i] = B[i] / SCALE[i];
    }
  }
};

}  // namespace

extern "C" {

// COCG13_single (src/solver/COCG13_single.f90:9-340): preconditioned COCG on
// split D/L/U storage, unconjugated r^T z and p^T q, conjugated norms, stop on
// the recursive residual ||r||/||b|| <= RESID.  PRECOND "IC" (diagonal-modified
// IC(0)), "SSOR", "DIAG".  NSET 0 -> ERROR 101 on first use, 1 -> precondition,
// 2 -> symmetric diagonal scaling as well.  ITER in: max iterations; out: count
// (MAXIT+1 after a full loop, as the Fortran DO variable).  ERROR -100 at the cap.
// The reference SAVEs DD/SCALE across calls; here they are fresh each call.
void orc_cocg13_single(int NP, int NPL, int NPU, double* D_, double* AL_, const int* INL, const int* IAL,
                       double* AU_, const int* INU, const int* IAU, double* B_, double* X_, const char* PRECOND,
                       double SIGMA_DIAG, double SIGMA, double* RESID, int* ITER, int* ERROR, int NSET,
                       double* history) {
  (void)NPL; (void)NPU;
  *ERROR = 0;
  if (NSET == 0) { *ERROR = 101; return; }
  CocgRun run;
  run.NP = NP;
  run.D = reinterpret_cast<cplx*>(D_);
  run.AL = reinterpret_cast<cplx*>(AL_);
  run.AU = reinterpret_cast<cplx*>(AU_);
  run.B = reinterpret_cast<cplx*>(B_);
  run.X = reinterpret_cast<cplx*>(X_);
  run.INL = INL; run.IAL = IAL; run.INU = INU; run.IAU = IAU;
  const int MAXIT = *ITER;
  const double TOL = *RESID;
  run.setup(PRECOND, SIGMA_DIAG, SIGMA, NSET);
  if (run.BNRM2 == 0.0) {
    for (int i = 0; i < NP; ++i) run.X[i] = 0.0;
    *RESID = 0.0; *ITER = 0;
    return;
  }
  int iter;
  for (iter = 1; iter <= MAXIT; ++iter) {
    *RESID = run.step();
    if (history) history[iter - 1] = *RESID;
    if (*RESID <= TOL) break;
    if (iter == MAXIT) *ERROR = -100;
  }
  *ITER = iter;
  run.finish();
}

// The same solver in slices (measurement of the reference's solver on a bounded
// sample): begin does COCG13_single's set-up on the caller's arrays (kept
// borrowed until end; NSET 2 scales them in place), advance runs k more
// iterations of the same loop and returns the recursive residual, end unscales
// X (and B) and frees the state.  Returns nullptr when ||b|| = 0 or NSET = 0.
void* orc_cocg_begin(int NP, double* D_, double* AL_, const int* INL, const int* IAL, double* AU_, const int* INU,
                     const int* IAU, double* B_, double* X_, const char* PRECOND, double SIGMA_DIAG, int NSET) {
  if (NSET == 0) return nullptr;
  CocgRun* run = new CocgRun();
  run->NP = NP;
  run->D = reinterpret_cast<cplx*>(D_);
  run->AL = reinterpret_cast<cplx*>(AL_);
  run->AU = reinterpret_cast<cplx*>(AU_);
  run->B = reinterpret_cast<cplx*>(B_);
  run->X = reinterpret_cast<cplx*>(X_);
  run->INL = INL; run->IAL = IAL; run->INU = INU; run->IAU = IAU;
  run->setup(PRECOND, SIGMA_DIAG, 0.0, NSET);
  if (run->BNRM2 == 0.0) {
    delete run;
    return nullptr;
  }
  return run;
}

double orc_cocg_advance(void* h, int k) {
  CocgRun* run = static_cast<CocgRun*>(h);
  double resid = -1.0;
  for (int i = 0; i < k; ++i) resid = run->step();
  return resid;
}

int orc_cocg_iterations(void* h) { return static_cast<CocgRun*>(h)->iter; }

void orc_cocg_end(void* h) {
  CocgRun* run = static_cast<CocgRun*>(h);
  run->finish();
  delete run;
}

// utm_geo_tm, LONLAT2UTM branch (src/common/m_param.f90:741-936): Snyder's
// ellipsoidal transverse Mercator on Clarke 1866, k0 0.9996, false easting
// 500 km.  reference_series = 1 keeps the reference's sin(4 phi) coefficient
// (15 e4/256 * 45 e6/1024, a product), 0 uses Snyder's sum (for checking the
// restatement against Snyder's published worked example).
void orc_utm_lonlat2xy(double rlon_deg, double rlat_deg, int zone, int reference_series, double* rx, double* ry) {
  const double PI = 3.141592653589793;
  const double degrad = PI / 180.0;
  const double semimaj = 6378206.4, semimin = 6356583.8, scfa = 0.9996, north = 0.0, east = 500000.0;
  const double e2 = 1.0 - std::pow(semimin / semimaj, 2.0);
  const double e4 = e2 * e2, e6 = e2 * e4, ep2 = e2 / (1.0 - e2);
  const double dlon = rlon_deg, dlat = rlat_deg;
  const double cm = (double)zone * 6.0 - 183.0;
  const double rlat = degrad * dlat;
  double delam = dlon - cm;
  if (delam < -180.0) delam = delam + 360.0;
  if (delam > 180.0) delam = delam - 360.0;
  delam = delam * degrad;
  double f1 = (1.0 - e2 / 4.0 - 3.0 * e4 / 64.0 - 5.0 * e6 / 256) * rlat;
  double f2 = 3.0 * e2 / 8.0 + 3.0 * e4 / 32.0 + 45.0 * e6 / 1024.0;
  f2 = f2 * std::sin(2.0 * rlat);
  double f3 = reference_series ? 15.0 * e4 / 256.0 * 45.0 * e6 / 1024.0 : 15.0 * e4 / 256.0 + 45.0 * e6 / 1024.0;
  f3 = f3 * std::sin(4.0 * rlat);
  double f4 = 35.0 * e6 / 3072.0;
  f4 = f4 * std::sin(6.0 * rlat);
  const double rm = semimaj * (f1 - f2 + f3 - f4);
  double xx, yy;
  if (dlat == 90.0 || dlat == -90.0) {
    xx = 0.0;
    yy = scfa * rm;
  } else {
    const double rn = semimaj / std::sqrt(1.0 - e2 * std::pow(std::sin(rlat), 2));
    const double t = std::pow(std::tan(rlat), 2);
    const double c = ep2 * std::pow(std::cos(rlat), 2);
    const double a = std::cos(rlat) * delam;
    f1 = (1.0 - t + c) * std::pow(a, 3) / 6.0;
    f2 = 5.0 - 18.0 * t + std::pow(t, 2) + 72.0 * c - 58.0 * ep2;
    f2 = f2 * std::pow(a, 5) / 120.0;
    xx = scfa * rn * (a + f1 + f2);
    f1 = std::pow(a, 2) / 2.0;
    f2 = 5.0 - t + 9.0 * c + 4.0 * std::pow(c, 2);
    f2 = f2 * std::pow(a, 4) / 24.0;
    f3 = 61.0 - 58.0 * t + std::pow(t, 2) + 600.0 * c - 330.0 * ep2;
    f3 = f3 * std::pow(a, 6) / 720.0;
    yy = scfa * (rm + rn * std::tan(rlat) * (f1 + f2 + f3));
  }
  *rx = xx + east;
  *ry = yy + north;
}

// UTMXY (src/common/m_param.f90:609-627): (x - xorigin)/1e3, (y - yorigin)/1e3 [km]
void orc_utmxy(double lon, double lat, double lonorigin, double latorigin, int zone, double* xy) {
  double x, y, xo, yo;
  orc_utm_lonlat2xy(lon, lat, zone, 1, &x, &y);
  orc_utm_lonlat2xy(lonorigin, latorigin, zone, 1, &xo, &yo);
  xy[0] = (x - xo) / 1.0e3;
  xy[1] = (y - yo) / 1.0e3;
}

// ||b - A x|| / ||b|| on split storage (the build's acceptance criterion).
double orc_true_residual(int NP, const double* D_, const double* AL_, const int* INL, const int* IAL,
                         const double* AU_, const int* INU, const int* IAU, const double* B_, const double* X_) {
  const cplx* D = reinterpret_cast<const cplx*>(D_);
  const cplx* AL = reinterpret_cast<const cplx*>(AL_);
  const cplx* AU = reinterpret_cast<const cplx*>(AU_);
  const cplx* B = reinterpret_cast<const cplx*>(B_);
  const cplx* X = reinterpret_cast<const cplx*>(X_);
  double rn = 0.0, bn = 0.0;
  for (int j = 0; j < NP; ++j) {
    cplx W = B[j] - D[j] * X[j];
    for (int i = INU[j]; i < INU[j + 1]; ++i) W = W - AU[i] * X[IAU[i] - 1];
    for (int i = INL[j]; i < INL[j + 1]; ++i) W = W - AL[i] * X[IAL[i] - 1];
    rn += std::norm(W);
    bn += std::norm(B[j]);
  }
  return bn > 0 ? std::sqrt(rn / bn) : 0.0;
}

// FINDELEMENT0 (src/common/m_mesh_type.f90:697-734): first tetrahedron in id
// order whose four barycentric coordinates are >= 0.  Returns 1-based id or 0.
long orc_findelement0(const double* x3, const double* xyz, long ntet, const int* n4, double* a) {
  for (long i = 0; i < ntet; ++i) {
    double e[4][3];
    load_tet(xyz, n4, i, e);
    nodebasisfun(e, x3, a);
    if (a[0] >= 0.0 && a[1] >= 0.0 && a[2] >= 0.0 && a[3] >= 0.0) return i + 1;
  }
  return 0;
}

}  // extern "C"

namespace {

// The coefficient rows of one site in tetrahedron t (0-based): PREPOBSCOEFF
// :681-721 / CALCOEFF_LINE (n_ebfem_bxyz_mpi.f90:880-929) with EDGEBASISFUN /
// FACEBASISFUN (m_fem_edge_util.f90:27-82), entries sorted by edge id.
void coeff_rows(const double* xyz, const int* n4, const int* n6line, int nobs, int s, long t, const double* x3,
                int* item, double* val_e, double* val_f) {
  double e[4][3];
  load_tet(xyz, n4, t, e);
  V3 gn[4];
  double vol, lam[4];
  gradnodebasisfun(e, gn, &vol);
  nodebasisfun(e, x3, lam);
  double w[6][3], wf[4][3], wfe[6][3];
  for (int i = 0; i < 6; ++i) {
    int k = KL[i][0], l = KL[i][1];
    for (int c = 0; c < 3; ++c) w[i][c] = lam[k - 1] * gn[l - 1].x[c] - lam[l - 1] * gn[k - 1].x[c];
  }
  for (int i = 0; i < 4; ++i) {
    int l = LMN[i][0], m = LMN[i][1], n = LMN[i][2];
    V3 o1 = outer(gn[m - 1], gn[n - 1]), o2 = outer(gn[l - 1], gn[m - 1]), o3 = outer(gn[n - 1], gn[l - 1]);
    for (int c = 0; c < 3; ++c)
      wf[i][c] = 2.0 * (lam[l - 1] * o1.x[c] + lam[n - 1] * o2.x[c] + lam[m - 1] * o3.x[c]);
  }
  for (int c = 0; c < 3; ++c)  // mul_ab (m_matrix.f90:1106-1126)
    for (int j = 0; j < 6; ++j) {
      double acc = 0.0;
      for (int k = 0; k < 4; ++k) acc = acc + wf[k][c] * (CROT[k][j] * 1.0);
      wfe[j][c] = acc;
    }
  double r6[6];
  int n6[6];
  double ce[6][3], cf[6][3];
  for (int j = 0; j < 6; ++j) {
    int sg = (n6line[t * 6 + j] < 0) ? -1 : 1;
    for (int c = 0; c < 3; ++c) { ce[j][c] = w[j][c] * sg; cf[j][c] = wfe[j][c] * sg; }
    r6[j] = std::abs(n6line[t * 6 + j]) * 1.0;
    n6[j] = j + 1;
  }
  sort_index(6, n6, r6);
  for (int j = 0; j < 6; ++j) {
    int jj = std::abs(n6line[t * 6 + n6[j] - 1]);
    item[s * 6 + j] = jj;
    for (int c = 0; c < 3; ++c) {
      val_e[((long)c * nobs + s) * 6 + j] = ce[n6[j] - 1][c];
      val_f[((long)c * nobs + s) * 6 + j] = cf[n6[j] - 1][c];
    }
  }
}

// Grid list of gengridforlist + classifyelement2grd (m_mesh_type.f90:56-202).
struct GridList {
  int nx, ny, nz;
  std::vector<double> xg, yg, zg;   // 1-based: xg[1..nx+1]
  std::vector<int> stack;           // 0..nx*ny*nz
  std::vector<int> ordered;         // 1-based tetrahedron ids, ordered[1..ntet]
};

GridList make_grid_list(const double* xyz, long node, long ntet, const int* n4, int nz = 50) {
  GridList g;
  // PREPOBSCOEFF_XY (n_ebfem_bxyz_mpi.f90:822): 300 x 300 x 50; PREPOBSCOEFF_XYSBTM (:1097): 300 x 300 x 300
  g.nx = 300; g.ny = 300; g.nz = nz;
  // GENXYZMINMAX (src/src_inv_ap/n_inv_ap.f90:1175-1205)
  double xmin = xyz[0], xmax = xyz[0], ymin = xyz[1], ymax = xyz[1], zmin = xyz[2], zmax = xyz[2];
  for (long i = 0; i < node; ++i) {
    xmin = std::min(xmin, xyz[3 * i]); xmax = std::max(xmax, xyz[3 * i]);
    ymin = std::min(ymin, xyz[3 * i + 1]); ymax = std::max(ymax, xyz[3 * i + 1]);
    zmin = std::min(zmin, xyz[3 * i + 2]); zmax = std::max(zmax, xyz[3 * i + 2]);
  }
  // gengridforlist (:73-107): the extent widened by the default-real literal 1.
  xmin = xmin - 1.0; xmax = xmax + 1.0; ymin = ymin - 1.0; ymax = ymax + 1.0; zmin = zmin - 1.0; zmax = zmax + 1.0;
  g.zg.assign(g.nz + 2, 0.0); g.yg.assign(g.ny + 2, 0.0); g.xg.assign(g.nx + 2, 0.0);
  for (int i = 1; i <= g.nz + 1; ++i) g.zg[i] = (i - 1) * (zmax - zmin) / (double)(float)g.nz + zmin;
  for (int i = 1; i <= g.ny + 1; ++i) g.yg[i] = (i - 1) * (ymax - ymin) / (double)(float)g.ny + ymin;
  for (int i = 1; i <= g.nx + 1; ++i) g.xg[i] = (i - 1) * (xmax - xmin) / (double)(float)g.nx + xmin;
  // classifyelement2grd (:110-202)
  std::vector<double> order(ntet + 1, 0.0);  // order(0) stays 0
  std::vector<int> index(ntet);
  for (long ii = 1; ii <= ntet; ++ii) {
    double x3[3] = {0.0, 0.0, 0.0};
    for (int j = 0; j < 4; ++j)
      for (int c = 0; c < 3; ++c) x3[c] = x3[c] + xyz[3L * (n4[(ii - 1) * 4 + j] - 1) + c] / 4.0;
    int ix = 0, iy = 0, iz = 0;
    for (int k = 1; k <= g.nz && !ix; ++k) {
      if (g.zg[k] < x3[2] && x3[2] <= g.zg[k + 1]) {
        iz = k;
        for (int j = 1; j <= g.ny && !ix; ++j) {
          if (g.yg[j] < x3[1] && x3[1] <= g.yg[j + 1]) {
            iy = j;
            for (int i = 1; i <= g.nx; ++i)
              if (g.xg[i] < x3[0] && x3[0] <= g.xg[i + 1]) { ix = i; break; }
          }
        }
      }
    }
    order[ii] = ((g.nx * g.ny) * (iz - 1) + g.nx * (iy - 1) + ix) * 1.0;
    index[ii - 1] = (int)ii;
  }
  sort_index((int)ntet, index.data(), order.data() + 1);
  g.ordered.assign(ntet + 1, 0);
  for (long i = 1; i <= ntet; ++i) g.ordered[i] = index[i - 1];
  // the stack loop as written (:170-190)
  const long nxyz = (long)g.nx * g.ny * g.nz;
  g.stack.assign(nxyz + 1, 0);
  long ipre = 0, ii = 0;
  for (ii = 0; ii <= nxyz - 1; ++ii) {
    for (;;) {
      if (ipre == ntet) goto done;
      if (order[ipre] < order[ipre + 1]) {
        g.stack[ii] = (int)ipre;
        if (ii + 1 == (long)order[ipre + 1]) ipre = ipre + 1;
        break;
      } else {
        ipre = ipre + 1;
      }
    }
  }
done:
  for (long k = ii; k <= nxyz; ++k) g.stack[k] = (int)ntet;
  return g;
}

// findelewithgrid (m_mesh_type.f90:204-277) + FINDELEMENT (:739-790); 1-based id or 0
long findelewithgrid(const GridList& g, const double* xyz, const int* n4, const double* x3) {
  int ix = 0, iy = 0, iz = 0;
  for (int l = 1; l <= g.nz && !ix; ++l) {
    if (g.zg[l] < x3[2] && x3[2] <= g.zg[l + 1]) {
      iz = l;
      for (int k = 1; k <= g.ny && !ix; ++k) {
        if (g.yg[k] < x3[1] && x3[1] <= g.yg[k + 1]) {
          iy = k;
          for (int j = 1; j <= g.nx; ++j)
            if (g.xg[j] < x3[0] && x3[0] <= g.xg[j + 1]) { ix = j; break; }
        }
      }
    }
  }
  if (!ix) return 0;
  std::vector<int> elist;
  for (int iside = 0; iside <= 64; ++iside) {  // the reference grows iside without bound
    elist.clear();
    for (int l = std::max(iz - iside, 1); l <= std::min(iz + iside, g.nz); ++l)
      for (int k = std::max(iy - iside, 1); k <= std::min(iy + iside, g.ny); ++k)
        for (int j = std::max(ix - iside, 1); j <= std::min(ix + iside, g.nx); ++j) {
          if (iz - (iside - 1) <= l && l <= iz + (iside - 1) && iy - (iside - 1) <= k && k <= iy + (iside - 1) &&
              ix - (iside - 1) <= j && j <= ix + (iside - 1))
            continue;
          const long index = (long)(g.nx * g.ny) * (l - 1) + g.nx * (k - 1) + j;
          const int num = g.stack[index] - g.stack[index - 1];
          for (int i = 1; i <= num; ++i) elist.push_back(g.ordered[g.stack[index - 1] + i]);
        }
    for (int ii : elist) {
      double e[4][3], a[4];
      load_tet(xyz, n4, ii - 1, e);
      nodebasisfun(e, x3, a);
      if (a[0] >= 0.0 && a[1] >= 0.0 && a[2] >= 0.0 && a[3] >= 0.0) return ii;
    }
  }
  return 0;
}

}  // namespace

extern "C" {

// PREPOBSCOEFF (n_ebfem_bxyz_mpi.f90:653-726) with EDGEBASISFUN/FACEBASISFUN
// (m_fem_edge_util.f90:27-82): per site, 6 entries sorted by edge id (item,
// 1-based) with edge-basis values val_e (3 comps) and face-basis*C values val_f.
// Layout: item[s*6+j], val_e[(c*nobs + s)*6 + j], val_f likewise (c = x,y,z).
// Returns 0 or -(s+1) for a site outside the mesh.
long orc_prepobscoeff(const double* xyz, long ntet, const int* n4, const int* n6line, int nobs,
                      const double* xyzobs, int* item, double* val_e, double* val_f, int* iele_out) {
  for (int s = 0; s < nobs; ++s) {
    const double* x3 = xyzobs + 3 * s;
    double a4[4];
    long iele = orc_findelement0(x3, xyz, ntet, n4, a4);
    if (iele == 0) return -(s + 1);
    if (iele_out) iele_out[s] = (int)iele;
    coeff_rows(xyz, n4, n6line, nobs, s, iele - 1, x3, item, val_e, val_f);
  }
  return 0;
}

// PREPOBSCOEFF_XY's element search and CALCOEFF_LINE (n_ebfem_bxyz_mpi.f90:792-929):
// the grid list over the node extent, FINDELEWITHGRID per site, the same rows.
long orc_prepobscoeff_grid(const double* xyz, long node, long ntet, const int* n4, const int* n6line, int nobs,
                           const double* xyzobs, int* item, double* val_e, double* val_f, int* iele_out) {
  GridList g = make_grid_list(xyz, node, ntet, n4);
  for (int s = 0; s < nobs; ++s) {
    const double* x3 = xyzobs + 3 * s;
    long iele = findelewithgrid(g, xyz, n4, x3);
    if (iele == 0) return -(s + 1);
    if (iele_out) iele_out[s] = (int)iele;
    coeff_rows(xyz, n4, n6line, nobs, s, iele - 1, x3, item, val_e, val_f);
  }
  return 0;
}

// The same with the grid list's vertical box count nz (XYSBTM's 300).
long orc_prepobscoeff_grid_nz(const double* xyz, long node, long ntet, const int* n4, const int* n6line, int nobs,
                              const double* xyzobs, int nz, int* item, double* val_e, double* val_f, int* iele_out) {
  GridList g = make_grid_list(xyz, node, ntet, n4, nz);
  for (int s = 0; s < nobs; ++s) {
    const double* x3 = xyzobs + 3 * s;
    long iele = findelewithgrid(g, xyz, n4, x3);
    if (iele == 0) return -(s + 1);
    if (iele_out) iele_out[s] = (int)iele;
    coeff_rows(xyz, n4, n6line, nobs, s, iele - 1, x3, item, val_e, val_f);
  }
  return 0;
}

// Triangle search of PREPZOBS (n_ebfem_bxyz_mpi.f90:1218-1223) over a 2-D mesh:
// allocate_2Dgrid_list + gen2Dgridforlist + classifytri2grd + findtriwithgrid +
// FINDTRI (src/common/m_triangle.f90:11-260).  xyz: 3 per node (x, y used);
// n3: 3 per triangle, 1-based; minmax: xmin, xmax, ymin, ymax (GENXYZMINMAX of
// the 3-D mesh, not widened here); nx x ny boxes.  Per point: iele (1-based) and
// a3.  Returns 0; -(j+1) when point j lies in no box or in no triangle of the
// shells searched (the reference stops or searches forever); -1000000 - t when
// triangle t's centroid lies on a box boundary (the reference stops).
long orc_findtri_grid(const double* xyz, long ntri, const int* n3, const double* minmax, int nx, int ny, int npts,
                      const double* pts, int* iele_out, double* a3_out) {
  // gen2Dgridforlist (:28-54)
  std::vector<double> xg(nx + 2, 0.0), yg(ny + 2, 0.0);
  const double xmin = minmax[0], xmax = minmax[1], ymin = minmax[2], ymax = minmax[3];
  for (int i = 1; i <= ny + 1; ++i) yg[i] = (i - 1) * (ymax - ymin) / (double)(float)ny + ymin;
  for (int i = 1; i <= nx + 1; ++i) xg[i] = (i - 1) * (xmax - xmin) / (double)(float)nx + xmin;
  // classifytri2grd (:56-131): the centroid's box, strict on both sides
  std::vector<double> order(ntri + 1, 0.0);
  std::vector<int> index(ntri);
  for (long ii = 1; ii <= ntri; ++ii) {
    double x2[2] = {0.0, 0.0};
    for (int j = 0; j < 3; ++j)
      for (int c = 0; c < 2; ++c) x2[c] = x2[c] + xyz[3L * (n3[(ii - 1) * 3 + j] - 1) + c] / 3.0;
    int ix = 0, iy = 0;
    for (int j = 1; j <= ny && !ix; ++j) {
      if (yg[j] < x2[1] && x2[1] < yg[j + 1]) {
        iy = j;
        for (int i = 1; i <= nx; ++i)
          if (xg[i] < x2[0] && x2[0] < xg[i + 1]) { ix = i; break; }
      }
    }
    if (!ix) return -1000000 - ii;
    order[ii] = (nx * (iy - 1) + ix) * 1.0;
    index[ii - 1] = (int)ii;
  }
  sort_index((int)ntri, index.data(), order.data() + 1);
  std::vector<int> ordered(ntri + 1, 0);
  for (long i = 1; i <= ntri; ++i) ordered[i] = index[i - 1];
  const long nxy = (long)nx * ny;
  std::vector<int> stack(nxy + 1, 0);
  long ipre = 0, ii = 0;
  for (ii = 0; ii <= nxy - 1; ++ii) {
    for (;;) {
      if (ipre == ntri) goto done;
      if (order[ipre] < order[ipre + 1]) {
        stack[ii] = (int)ipre;
        if (ii + 1 == (long)order[ipre + 1]) ipre = ipre + 1;
        break;
      } else {
        ipre = ipre + 1;
      }
    }
  }
done:
  for (long k = ii; k <= nxy; ++k) stack[k] = (int)ntri;
  // findtriwithgrid (:133-204) per point: the box (half-open), then growing shells
  for (int p = 0; p < npts; ++p) {
    const double* x2 = pts + 2L * p;
    int ix = 0, iy = 0;
    for (int k = 1; k <= ny && !ix; ++k) {
      if (yg[k] < x2[1] && x2[1] <= yg[k + 1]) {
        iy = k;
        for (int j = 1; j <= nx; ++j)
          if (xg[j] < x2[0] && x2[0] <= xg[j + 1]) { ix = j; break; }
      }
    }
    if (!ix) return -(p + 1);
    long found = 0;
    double a[3] = {0.0, 0.0, 0.0};
    std::vector<int> elist;
    for (int iside = 0; iside <= std::max(nx, ny) && !found; ++iside) {
      elist.clear();
      for (int k = std::max(iy - iside, 1); k <= std::min(iy + iside, ny); ++k)
        for (int j = std::max(ix - iside, 1); j <= std::min(ix + iside, nx); ++j) {
          if (iy - (iside - 1) <= k && k <= iy + (iside - 1) && ix - (iside - 1) <= j && j <= ix + (iside - 1))
            continue;
          const long idx = (long)nx * (k - 1) + j;
          const int num = stack[idx] - stack[idx - 1];
          for (int i = 1; i <= num; ++i) elist.push_back(ordered[stack[idx - 1] + i]);
        }
      // FINDTRI (:208-258): the first listed triangle with all three coordinates >= 0
      for (int t : elist) {
        const double* P[3];
        for (int j = 0; j < 3; ++j) P[j] = xyz + 3L * (n3[(t - 1) * 3 + j] - 1);
        const double x12[2] = {P[1][0] - P[0][0], P[1][1] - P[0][1]};
        const double x13[2] = {P[2][0] - P[0][0], P[2][1] - P[0][1]};
        const double x23[2] = {P[2][0] - P[1][0], P[2][1] - P[1][1]};
        const double v1[2] = {x2[0] - P[0][0], x2[1] - P[0][1]};
        const double v2[2] = {x2[0] - P[1][0], x2[1] - P[1][1]};
        const double a0 = (x13[0] * x12[1] - x13[1] * x12[0]);
        a[1] = (x13[0] * v1[1] - x13[1] * v1[0]) / a0;
        a[2] = (v1[0] * x12[1] - v1[1] * x12[0]) / a0;
        a[0] = (v2[0] * x23[1] - v2[1] * x23[0]) / a0;
        if (a[0] >= 0.0 && a[1] >= 0.0 && a[2] >= 0.0) { found = t; break; }
      }
    }
    if (!found) return -(p + 1);
    iele_out[p] = (int)found;
    for (int j = 0; j < 3; ++j) a3_out[3L * p + j] = a[j];
  }
  return 0;
}

// CALOBSEBCOMP + CALOBSRESP (n_ebfem_bxyz_mpi.f90:397-423, 570-626) with the
// primary field fp = 0: for each source column k, bx,by,bz = coeff(2,c)*A and
// ex,ey = coeff(1,c)*(-i*omega*A).  out: complex [(k*5 + comp)*nobs + s];
// amp/phase (deg) alongside, same indexing.
void orc_calobsebcomp(int nline, int nsr, double omega, const double* fs_, int nobs, const int* item,
                      const double* val_e, const double* val_f, double* out_, double* amp, double* phase) {
  const cplx* fs = reinterpret_cast<const cplx*>(fs_);
  cplx* out = reinterpret_cast<cplx*>(out_);
  const double pi = 4.0 * std::atan(1.0), r2d = 180.0 / pi;
  std::vector<cplx> fss(nline);
  for (int k = 0; k < nsr; ++k) {
    const cplx* f = fs + (long)k * nline;
    for (int i = 0; i < nline; ++i) fss[i] = -(cplx(0.0, 1.0) * omega * f[i]);
    for (int comp = 0; comp < 5; ++comp) {
      const double* val = (comp < 3) ? val_f + (long)comp * nobs * 6 : val_e + (long)(comp - 3) * nobs * 6;
      const cplx* src = (comp < 3) ? f : fss.data();
      for (int s = 0; s < nobs; ++s) {
        cplx acc(0.0, 0.0);
        for (int j = 0; j < 6; ++j) acc = acc + val[s * 6 + j] * src[item[s * 6 + j] - 1];
        long o = ((long)k * 5 + comp) * nobs + s;
        out[o] = acc;
        if (amp) amp[o] = std::sqrt(std::pow(acc.real(), 2.0) + std::pow(acc.imag(), 2.0));
        if (phase) phase[o] = std::atan2(acc.imag(), acc.real()) * r2d;
      }
    }
  }
}

}  // extern "C"
