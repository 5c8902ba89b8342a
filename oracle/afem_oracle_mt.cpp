// CPU oracle for the 3-D MT forward -- TEST INFRASTRUCTURE ONLY.
//
// A statement-by-statement C++ restatement of the reference's MT forward
// (src/src_3DMT/n_ebfem_3DMT.f90, forward_3DMT.f90) and of the 2-D TM
// boundary solves it runs on the four side faces (src/src_2D/m_surface_type.f90,
// forward_2DTM.f90; src/common/m_face_type.f90 for the face list).  Used by
// tests/ as the parity checker; nothing in the product library links or calls
// this file.  The direct solves the reference hands to PARDISO are left to the
// caller (the tests use SciPy's SuperLU on the exported systems).
//
// Parity status: unpinned against the reference itself (no Fortran compiler,
// no MT data shipped with it).  Pinned by identities (the 2-D curl-curl
// annihilates discrete gradients, the 2-D mass matrix is SPD) and by the
// known answer of MT over a uniform half-space (apparent resistivity 1/sigma,
// phase 45 degrees), which the whole chain reproduces.
//
// Literals: the reference is compiled without -r8, so its default-real
// constants (1./6., 1./12., 0.1, 3.31) are single precision; they are kept
// as (double)(float) here.  Compile with -ffp-contract=off (no FMA).
#include <algorithm>
#include <cmath>
#include <complex>
#include <cstdint>
#include <cstring>
#include <string>
#include <vector>

typedef std::complex<double> cplx;

namespace {

// lmn face table (src/solver/m_fem_edge_util.f90:13-17), 1-based local nodes
const int LMN_MT[4][3] = {{2, 3, 4}, {1, 4, 3}, {1, 2, 4}, {1, 3, 2}};

inline double pi_mt() { return 4.0 * std::atan(1.0); }
inline double dmu_mt() { return 4.0 * pi_mt() * 1.0e-7; }

struct Surface {
  int facetype = 0;  // 0 "xy", 1 "yz", 2 "xz"
  int node = 0, ntri = 0, nline = 0;
  std::vector<double> x1x2;          // 2*node
  std::vector<int> inodeface_to_3D;  // node, 1-based 3-D ids
  std::vector<int> n3;               // 3*ntri, 1-based surface node ids
  std::vector<int> n3line;           // 3*ntri, signed 1-based surface line ids
  std::vector<int> ifacetri_to_face; // ntri, 1-based 3-D face ids
  std::vector<int> ifacetri_to_tet;  // ntri, 1-based tetrahedra
  std::vector<int> line;             // 2*nline, 1-based surface node ids
  std::vector<int> ilineface_to_3D;  // nline, 1-based 3-D line ids
  std::vector<int> iflag_bound;      // nline: 0 none, 1 top, 2 bottom, 3 left, 4 right
};

struct Surfaces {
  Surface s[6];
  double minmax[6];
  int err = 0;
};

// MKFACE (src/common/m_face_type.f90:43-141): faces grouped by their smallest
// node n1, in order of first encounter scanning the tetrahedra of n1 (by id)
// and their local node pairs (k, m).  face_stack[0..node], face_item[2*nface].
int mkface(int node, long ntet, const int* n4, std::vector<int>& face_stack, std::vector<int>& face_item) {
  const int maxnele = 200;
  std::vector<int> nele(node + 1, 0);
  std::vector<int> node2ele((size_t)maxnele * (node + 1));
  for (long i = 1; i <= ntet; ++i)
    for (int j = 0; j < 4; ++j) {
      const int n1 = n4[(i - 1) * 4 + j];
      if (nele[n1] == maxnele) return -1;
      nele[n1] += 1;
      node2ele[(size_t)n1 * maxnele + nele[n1] - 1] = (int)i;
    }
  face_stack.assign(node + 1, 0);
  face_item.clear();
  for (int n1 = 1; n1 <= node; ++n1) {
    face_stack[n1] = face_stack[n1 - 1];
    for (int j = 1; j <= nele[n1]; ++j) {
      const long iele = node2ele[(size_t)n1 * maxnele + j - 1];
      for (int k = 0; k < 4; ++k)
        for (int m = 0; m < 4; ++m) {
          const int n2 = n4[(iele - 1) * 4 + k], n3 = n4[(iele - 1) * 4 + m];
          if (n1 < n2 && n2 < n3) {
            bool found = false;
            for (int l = face_stack[n1 - 1] + 1; l <= face_stack[n1]; ++l)
              if (n2 == face_item[2 * (l - 1)] && n3 == face_item[2 * (l - 1) + 1]) { found = true; break; }
            if (found) continue;
            face_stack[n1] += 1;
            face_item.push_back(n2);
            face_item.push_back(n3);
          }
        }
    }
  }
  return 0;
}

// MKN4FACE + FACE2ELEMENT (m_face_type.f90:145-236): n4face(i,j) = +-face id
// (+ when the face's nodes lmn(j,:) run in cyclically ascending order);
// face2ele(1,f) = the tetrahedron seeing f outward, face2ele(2,f) inward.
int face2element(int node, long ntet, const int* n4, const std::vector<int>& face_stack,
                 const std::vector<int>& face_item, std::vector<int>& face2ele) {
  const long nface = (long)face_item.size() / 2;
  face2ele.assign(2 * nface, 0);
  for (long i = 1; i <= ntet; ++i)
    for (int j = 0; j < 4; ++j) {
      const int n11 = n4[(i - 1) * 4 + LMN_MT[j][0] - 1];
      const int n12 = n4[(i - 1) * 4 + LMN_MT[j][1] - 1];
      const int n13 = n4[(i - 1) * 4 + LMN_MT[j][2] - 1];
      int idir;
      if ((n11 < n12 && n12 < n13) || (n12 < n13 && n13 < n11) || (n13 < n11 && n11 < n12)) idir = 1;
      else idir = -1;
      int s3[3] = {n11, n12, n13};
      std::sort(s3, s3 + 3);  // SORT_INDEX of three distinct ids: ascending
      int faceid = 0;
      for (int k = face_stack[s3[0] - 1] + 1; k <= face_stack[s3[0]]; ++k)
        if (face_item[2 * (k - 1)] == s3[1] && face_item[2 * (k - 1) + 1] == s3[2]) { faceid = k; break; }
      if (faceid == 0) return -2;
      if (idir > 0) face2ele[2 * (faceid - 1)] = (int)i;
      else face2ele[2 * (faceid - 1) + 1] = (int)i;
    }
  (void)node;
  return 0;
}

// area_tri (src/src_2D/m_surface_type.f90:816-826)
inline double area_tri(const double y[3], const double z[3]) {
  return 0.5 * std::fabs((y[2] - y[0]) * (z[1] - z[0]) - (y[1] - y[0]) * (z[2] - z[0]));
}

const int ID3[3][3] = {{1, 2, 3}, {2, 3, 1}, {3, 1, 2}};

// outer (src/common/m_outerinnerproduct.f90:4-12) of 3-vectors
inline void outer3(const double a[3], const double b[3], double c[3]) {
  c[0] = a[1] * b[2] - a[2] * b[1];
  c[1] = a[2] * b[0] - a[0] * b[2];
  c[2] = a[0] * b[1] - a[1] * b[0];
}
inline double inner3(const double a[3], const double b[3]) { return a[0] * b[0] + a[1] * b[1] + a[2] * b[2]; }

// grcgr (m_surface_type.f90:783-813): grad lambda_l x grad lambda_m of edge i_edge
inline void grcgr(int i_edge, const double y[3], const double z[3], double g[3]) {
  const int l = ID3[i_edge - 1][0], m = ID3[i_edge - 1][1], n = ID3[i_edge - 1][2];
  const double r[3][3] = {{0.0, y[0], z[0]}, {0.0, y[1], z[1]}, {0.0, y[2], z[2]}};
  double rnl[3], rmn[3], c[3];
  for (int k = 0; k < 3; ++k) { rnl[k] = r[l - 1][k] - r[n - 1][k]; rmn[k] = r[n - 1][k] - r[m - 1][k]; }
  const double s = area_tri(y, z);
  const double coef = -(0.25 / (s * s));
  outer3(rnl, rmn, c);
  for (int k = 0; k < 3; ++k) g[k] = coef * c[k];
}

// gradnodebasisfun_tri (m_surface_type.f90:727-753): gn[l] = (y, z) gradient of lambda_l
inline void gradnodebasisfun_tri(const double y[3], const double z[3], double gn[3][2]) {
  const double ex[3] = {1.0, 0.0, 1.0};
  const double exyz[3][3] = {{0.0, y[0], z[0]}, {0.0, y[1], z[1]}, {0.0, y[2], z[2]}};
  const double s = area_tri(y, z);
  for (int l = 1; l <= 3; ++l) {
    const int m = ID3[l - 1][1], n = ID3[l - 1][2];
    double xmn[3], c[3];
    for (int k = 0; k < 3; ++k) xmn[k] = exyz[n - 1][k] - exyz[m - 1][k];
    outer3(ex, xmn, c);
    const double coef = 0.5 / s;
    gn[l - 1][0] = coef * c[1];
    gn[l - 1][1] = coef * c[2];
  }
}

// grdgr (m_surface_type.f90:887-907)
inline double grdgr(int i, int j, const double y[3], const double z[3]) {
  double gn[3][2];
  gradnodebasisfun_tri(y, z, gn);
  const double a[3] = {0.0, gn[i - 1][0], gn[i - 1][1]}, b[3] = {0.0, gn[j - 1][0], gn[j - 1][1]};
  return inner3(a, b);
}

// NlNmdS (m_surface_type.f90:871-883): the default-real 1./6. and 1./12.
inline double nlnmds(int l, int m, const double y[3], const double z[3]) {
  const double s = area_tri(y, z);
  return (l == m) ? (double)(1.0f / 6.0f) * s : (double)(1.0f / 12.0f) * s;
}

// wiwjdS (m_surface_type.f90:845-868)
inline double wiwjds(int i_edge, int j_edge, const double y[3], const double z[3]) {
  const int l = ID3[i_edge - 1][0], m = ID3[i_edge - 1][1];
  const int lp = ID3[j_edge - 1][0], mp = ID3[j_edge - 1][1];
  return nlnmds(l, lp, y, z) * grdgr(m, mp, y, z) - nlnmds(m, lp, y, z) * grdgr(l, mp, y, z) -
         nlnmds(l, mp, y, z) * grdgr(m, lp, y, z) + nlnmds(m, mp, y, z) * grdgr(l, lp, y, z);
}

}  // namespace

extern "C" {

// EXTRACT6SURFACES + FINDBOUNDARYLINE (src/src_2D/m_surface_type.f90:189-502, 123-186)
// on the mesh extent (GENXYZMINMAX_MT, src/src_3DMT/n_ebfem_3DMT.f90:488-521).
// Surfaces 1..6: top (xy), north (xz), west (yz), south (xz), east (yz), bottom (xy).
// Returns a handle (free with orc_mt_free); its err is nonzero on a failure the
// reference stops on (-1: a node in more than 200 tetrahedra, -2: face not found,
// -3: a boundary face seen by two tetrahedra, -4: a triangle edge missing in its tetrahedron).
void* orc_mt_surfaces(int node, const double* xyz, long ntet, const int* n4, int nline, const int* line,
                      const int* n6line) {
  Surfaces* S = new Surfaces();
  double mm[6] = {xyz[0], xyz[0], xyz[1], xyz[1], xyz[2], xyz[2]};
  for (int i = 0; i < node; ++i) {
    mm[0] = std::min(mm[0], xyz[3 * i]); mm[1] = std::max(mm[1], xyz[3 * i]);
    mm[2] = std::min(mm[2], xyz[3 * i + 1]); mm[3] = std::max(mm[3], xyz[3 * i + 1]);
    mm[4] = std::min(mm[4], xyz[3 * i + 2]); mm[5] = std::max(mm[5], xyz[3 * i + 2]);
  }
  for (int k = 0; k < 6; ++k) S->minmax[k] = mm[k];
  std::vector<int> face_stack, face_item, face2ele;
  if (mkface(node, ntet, n4, face_stack, face_item) != 0) { S->err = -1; return S; }
  if (face2element(node, ntet, n4, face_stack, face_item, face2ele) != 0) { S->err = -2; return S; }
  const double d01 = (double)0.1f;
  const double xmin = mm[0] + d01, xmax = mm[1] - d01, ymin = mm[2] + d01, ymax = mm[3] - d01;
  const double zmin = mm[4] + d01, zmax = mm[5] - d01;
  const int ftype[6] = {0, 2, 1, 2, 1, 0};
  std::vector<unsigned char> on((size_t)6 * (node + 1), 0);
  for (int i = 1; i <= node; ++i) {
    const double x = xyz[3 * (i - 1)], y = xyz[3 * (i - 1) + 1], z = xyz[3 * (i - 1) + 2];
    on[0 * (node + 1) + i] = z >= zmax;
    on[1 * (node + 1) + i] = y >= ymax;
    on[2 * (node + 1) + i] = x <= xmin;
    on[3 * (node + 1) + i] = y <= ymin;
    on[4 * (node + 1) + i] = x >= xmax;
    on[5 * (node + 1) + i] = z <= zmin;
  }
  std::vector<int> n3d2f((size_t)6 * (node + 1), 0);
  for (int j = 0; j < 6; ++j) {
    Surface& s = S->s[j];
    s.facetype = ftype[j];
    const unsigned char* onj = &on[(size_t)j * (node + 1)];
    int* i2f = &n3d2f[(size_t)j * (node + 1)];
    for (int i = 1; i <= node; ++i)
      if (onj[i]) {
        s.node += 1;
        s.inodeface_to_3D.push_back(i);
        i2f[i] = s.node;
        const double x = xyz[3 * (i - 1)], y = xyz[3 * (i - 1) + 1], z = xyz[3 * (i - 1) + 2];
        if (s.facetype == 0) { s.x1x2.push_back(x); s.x1x2.push_back(y); }
        if (s.facetype == 1) { s.x1x2.push_back(y); s.x1x2.push_back(z); }
        if (s.facetype == 2) { s.x1x2.push_back(x); s.x1x2.push_back(z); }
      }
    // triangles: faces whose smallest node is on the surface and whose other two are too
    for (int i = 1; i <= s.node; ++i) {
      const int i3d = s.inodeface_to_3D[i - 1];
      for (int k = face_stack[i3d - 1] + 1; k <= face_stack[i3d]; ++k) {
        const int a = face_item[2 * (k - 1)], b = face_item[2 * (k - 1) + 1];
        if (onj[a] && onj[b]) {
          s.ntri += 1;
          s.n3.push_back(i); s.n3.push_back(i2f[a]); s.n3.push_back(i2f[b]);
          s.ifacetri_to_face.push_back(k);
        }
      }
    }
    // smallest node first, then anticlockwise in the surface plane
    for (int t = 0; t < s.ntri; ++t) {
      int* q = &s.n3[3 * t];
      int i1 = q[0], i2 = q[1], i3 = q[2];
      if (q[0] >= q[1]) { i1 = q[1]; i2 = q[0]; }
      if (i1 >= q[2]) { i3 = i1; i1 = q[2]; }
      q[0] = i1; q[1] = i2; q[2] = i3;
      double x1[3] = {0, 0, 0}, x2[3] = {0, 0, 0}, x3[3];
      for (int c = 0; c < 2; ++c) {
        x1[c] = s.x1x2[2 * (i2 - 1) + c] - s.x1x2[2 * (i1 - 1) + c];
        x2[c] = s.x1x2[2 * (i3 - 1) + c] - s.x1x2[2 * (i1 - 1) + c];
      }
      outer3(x1, x2, x3);
      if (x3[2] < 0.0) { q[1] = i3; q[2] = i2; }
    }
    for (int t = 0; t < s.ntri; ++t) {
      const int f = s.ifacetri_to_face[t];
      const int f1 = face2ele[2 * (f - 1)], f2 = face2ele[2 * (f - 1) + 1];
      int tet = 0;
      if (f1 != 0) tet = f1;
      if (f2 != 0) tet = f2;
      if (f1 != 0 && f2 != 0) { S->err = -3; return S; }
      s.ifacetri_to_tet.push_back(tet);
    }
  }
  // surface lines, in 3-D line order
  std::vector<int> l3d2f((size_t)6 * (nline + 1), 0);
  for (int i = 1; i <= nline; ++i)
    for (int j = 0; j < 6; ++j) {
      const int a = line[2 * (i - 1)], b = line[2 * (i - 1) + 1];
      if (on[(size_t)j * (node + 1) + a] && on[(size_t)j * (node + 1) + b]) {
        Surface& s = S->s[j];
        s.nline += 1;
        s.line.push_back(n3d2f[(size_t)j * (node + 1) + a]);
        s.line.push_back(n3d2f[(size_t)j * (node + 1) + b]);
        s.ilineface_to_3D.push_back(i);
        l3d2f[(size_t)j * (nline + 1) + i] = s.nline;
      }
    }
  // n3line: each triangle edge matched against its tetrahedron's six lines
  for (int j = 0; j < 6; ++j) {
    Surface& s = S->s[j];
    s.n3line.assign(3 * (size_t)s.ntri, 0);
    for (int t = 0; t < s.ntri; ++t) {
      const int v3[3] = {s.inodeface_to_3D[s.n3[3 * t] - 1], s.inodeface_to_3D[s.n3[3 * t + 1] - 1],
                         s.inodeface_to_3D[s.n3[3 * t + 2] - 1]};
      const long tet = s.ifacetri_to_tet[t];
      for (int l = 0; l < 3; ++l) {
        const int p = v3[l], q = v3[(l + 1) % 3];
        bool got = false;
        for (int k = 0; k < 6 && !got; ++k) {
          const int e = std::abs(n6line[(tet - 1) * 6 + k]);
          const int la = line[2 * (e - 1)], lb = line[2 * (e - 1) + 1];
          if (p == la && q == lb) { s.n3line[3 * t + l] = l3d2f[(size_t)j * (nline + 1) + e]; got = true; }
          else if (p == lb && q == la) { s.n3line[3 * t + l] = -l3d2f[(size_t)j * (nline + 1) + e]; got = true; }
        }
        if (!got) { S->err = -4; return S; }
      }
    }
  }
  // FINDBOUNDARYLINE
  for (int j = 0; j < 6; ++j) {
    Surface& s = S->s[j];
    s.iflag_bound.assign(s.nline, 0);
    double yl, yr, zb, zt;
    if (s.facetype == 0) { yl = xmin; yr = xmax; zb = ymin; zt = ymax; }
    else if (s.facetype == 1) { yl = ymin; yr = ymax; zb = zmin; zt = zmax; }
    else { yl = xmin; yr = xmax; zb = zmin; zt = zmax; }
    for (int l = 0; l < s.nline; ++l) {
      const int i1 = s.line[2 * l], i2 = s.line[2 * l + 1];
      const double y1 = s.x1x2[2 * (i1 - 1)], y2 = s.x1x2[2 * (i2 - 1)];
      const double z1 = s.x1x2[2 * (i1 - 1) + 1], z2 = s.x1x2[2 * (i2 - 1) + 1];
      if (y1 < yl && y2 < yl) s.iflag_bound[l] = 3;
      if (y1 > yr && y2 > yr) s.iflag_bound[l] = 4;
      if (z1 < zb && z2 < zb) s.iflag_bound[l] = 2;
      if (z1 > zt && z2 > zt) s.iflag_bound[l] = 1;
    }
  }
  return S;
}

void orc_mt_free(void* h) { delete static_cast<Surfaces*>(h); }
int orc_mt_error(void* h) { return static_cast<Surfaces*>(h)->err; }
void orc_mt_minmax(void* h, double* mm) { std::memcpy(mm, static_cast<Surfaces*>(h)->minmax, 6 * sizeof(double)); }

// Sizes of surface j (1..6): node, ntri, nline.
void orc_mt_surface_sizes(void* h, int j, int* node, int* ntri, int* nline) {
  const Surface& s = static_cast<Surfaces*>(h)->s[j - 1];
  *node = s.node; *ntri = s.ntri; *nline = s.nline;
}

// Arrays of surface j (any pointer may be NULL): x1x2[2*node], n3[3*ntri], n3line[3*ntri],
// tet[ntri] (ifacetri_to_tet), line[2*nline], line3d[nline] (ilineface_to_3D), flag[nline].
void orc_mt_surface_get(void* h, int j, double* x1x2, int* n3, int* n3line, int* tet, int* line, int* line3d,
                        int* flag) {
  const Surface& s = static_cast<Surfaces*>(h)->s[j - 1];
  if (x1x2) std::copy(s.x1x2.begin(), s.x1x2.end(), x1x2);
  if (n3) std::copy(s.n3.begin(), s.n3.end(), n3);
  if (n3line) std::copy(s.n3line.begin(), s.n3line.end(), n3line);
  if (tet) std::copy(s.ifacetri_to_tet.begin(), s.ifacetri_to_tet.end(), tet);
  if (line) std::copy(s.line.begin(), s.line.end(), line);
  if (line3d) std::copy(s.ilineface_to_3D.begin(), s.ilineface_to_3D.end(), line3d);
  if (flag) std::copy(s.iflag_bound.begin(), s.iflag_bound.end(), flag);
}

// COND3DTO2D (m_surface_type.f90:76-120) for surface j: tag 1 -> sigma_air,
// tag 2 -> the default-real literal 3.31, tag >= 3 -> sigma_land(1) (condflag 0)
// or sigma(tet - nphys1) (condflag 1).  Returns 0, or -(t+1) for a triangle whose
// tetrahedron's tag selects nothing.
long orc_mt_cond2d(void* h, int j, const int* tag, double sigma_air, int condflag, double sigma_land1, long nphys1,
                   const double* sigma_file, double* cond) {
  const Surface& s = static_cast<Surfaces*>(h)->s[j - 1];
  for (int t = 0; t < s.ntri; ++t) {
    const long tet = s.ifacetri_to_tet[t];
    const int g = tag[tet - 1];
    if (g == 1) cond[t] = sigma_air;
    else if (g == 2) cond[t] = (double)3.31f;
    else if (g >= 3) cond[t] = (condflag == 0) ? sigma_land1 : sigma_file[tet - nphys1 - 1];
    else return -(t + 1);
  }
  return 0;
}

// The 2-D TM system of surface j at freq: PREPAOFSURFACE's pattern
// (forward_2DTM.f90:226-250, set_iccg_var7_dofn with three dofs per triangle),
// INITIALIZE + GENMAT2DTM (:253-363) + COPY_UL_ICCG12 + GENBC2D (:366-410) +
// SET_BC_ICCG (:414-470, nsr = 1); apply_bc = 0 stops after COPY_UL (bc, gval
// and rf zero).  cond[ntri] from orc_mt_cond2d.  With
// INU == NULL only *iau_tot is set (the pattern size).  Outputs: INU/INL[n+1],
// IAU/IAL[iau_tot] (1-based), complex D[n], AU/AL[iau_tot], rf[n] (the
// right-hand side after the Dirichlet lifting), bc[n], gval[n] (complex
// Dirichlet values).  Returns 0, -1 on a row longer than 1000, -2 on a dof
// missing from the pattern, -3 when a top boundary line is not horizontal.
int orc_mt_face_system(void* h, int j, const double* cond, double freq, int apply_bc, long* iau_tot, int* INU,
                       int* IAU, int* INL,
                       int* IAL, double* D_, double* AU_, double* AL_, double* rf_, unsigned char* bc,
                       double* gval_) {
  const Surface& s = static_cast<Surfaces*>(h)->s[j - 1];
  const int n = s.nline;
  std::vector<std::vector<int>> up(n + 1), lo(n + 1);
  for (int t = 0; t < s.ntri; ++t) {
    int dof[3];
    for (int k = 0; k < 3; ++k) dof[k] = std::abs(s.n3line[3 * t + k]);
    for (int kf = 0; kf < 3; ++kf)
      for (int lf = 0; lf < 3; ++lf) {
        const int i = dof[kf], c = dof[lf];
        if (i == c) continue;
        std::vector<int>& row = (i < c) ? up[i] : lo[i];
        size_t pos = row.size();
        bool exist = false;
        for (size_t q = 0; q < row.size(); ++q) {
          if (row[q] == c) { exist = true; break; }
          if (c < row[q]) { pos = q; break; }
        }
        if (exist) continue;
        if (row.size() + 1 > 1000) return -1;
        row.insert(row.begin() + pos, c);
      }
  }
  std::vector<int> inu(n + 1, 0), inl(n + 1, 0);
  for (int i = 1; i <= n; ++i) {
    inu[i] = inu[i - 1] + (int)up[i].size();
    inl[i] = inl[i - 1] + (int)lo[i].size();
  }
  *iau_tot = inu[n];
  if (!INU) return 0;
  std::copy(inu.begin(), inu.end(), INU);
  std::copy(inl.begin(), inl.end(), INL);
  for (int i = 1; i <= n; ++i) {
    std::copy(up[i].begin(), up[i].end(), IAU + inu[i - 1]);
    std::copy(lo[i].begin(), lo[i].end(), IAL + inl[i - 1]);
  }
  cplx* D = reinterpret_cast<cplx*>(D_);
  cplx* AU = reinterpret_cast<cplx*>(AU_);
  cplx* AL = reinterpret_cast<cplx*>(AL_);
  cplx* rf = reinterpret_cast<cplx*>(rf_);
  cplx* gv = reinterpret_cast<cplx*>(gval_);
  const long nnzu = inu[n];
  for (int i = 0; i < n; ++i) { D[i] = 0.0; rf[i] = 0.0; }
  for (long p = 0; p < nnzu; ++p) { AU[p] = 0.0; AL[p] = 0.0; }
  const double omega = 2.0 * pi_mt() * freq, dmu = dmu_mt(), L0 = 1.0e3;
  const cplx iunit(0.0, 1.0);
  // GENMAT2DTM
  for (int t = 0; t < s.ntri; ++t) {
    int idir[3];
    for (int k = 0; k < 3; ++k) idir[k] = (s.n3line[3 * t + k] < 0) ? -1 : 1;
    double y[3], z[3];
    for (int k = 0; k < 3; ++k) {
      y[k] = s.x1x2[2 * (s.n3[3 * t + k] - 1)];
      z[k] = s.x1x2[2 * (s.n3[3 * t + k] - 1) + 1];
    }
    const double sigma = cond[t];
    const cplx BB = iunit * omega * dmu * sigma * std::pow(L0, 2.0);
    const double sa = area_tri(y, z);
    double A1[3][3], B1[3][3];
    for (int ie = 1; ie <= 3; ++ie) {
      double gi[3];
      grcgr(ie, y, z, gi);
      for (int je = 1; je <= 3; ++je) {
        double gj[3];
        grcgr(je, y, z, gj);
        A1[ie - 1][je - 1] = 4.0 * sa * inner3(gi, gj);
        B1[ie - 1][je - 1] = wiwjds(ie, je, y, z);
      }
    }
    cplx ek[3][3];
    for (int a = 0; a < 3; ++a)
      for (int b = 0; b < 3; ++b) ek[a][b] = (A1[a][b] + BB * B1[a][b]) * (double)idir[a] * (double)idir[b];
    int tdof[3];
    for (int k = 0; k < 3; ++k) tdof[k] = s.n3line[3 * t + k] * idir[k];
    // sup_iccg (forward_bxyz_mpi.f90:642-699)
    for (int ie = 0; ie < 3; ++ie)
      for (int je = 0; je < 3; ++je) {
        const int igl = tdof[ie], jgl = tdof[je];
        if (igl == jgl) D[igl - 1] += ek[ie][je];
        else if (igl < jgl) {
          long pos = -1;
          for (int q = inu[igl - 1]; q < inu[igl]; ++q)
            if (IAU[q] == jgl) { pos = q; break; }
          if (pos < 0) return -2;
          AU[pos] += (ie > je) ? ek[ie][je] : ek[je][ie];
        }
      }
  }
  // COPY_UL_ICCG12
  for (int igl = 1; igl <= n; ++igl)
    for (int q = inu[igl - 1]; q < inu[igl]; ++q) {
      const int jgl = IAU[q];
      for (int q2 = inl[jgl - 1]; q2 < inl[jgl]; ++q2)
        if (IAL[q2] == igl) { AL[q2] = AU[q]; break; }
    }
  for (int i = 0; i < n; ++i) { bc[i] = 0; gv[i] = 0.0; }
  if (!apply_bc) return 0;
  // GENBC2D
  for (int i = 0; i < n; ++i) {
    const int fl = s.iflag_bound[i];
    if (fl == 1) {
      const int a = s.line[2 * i], b = s.line[2 * i + 1];
      const double y1 = s.x1x2[2 * (a - 1)], y2 = s.x1x2[2 * (b - 1)];
      const double z1 = s.x1x2[2 * (a - 1) + 1], z2 = s.x1x2[2 * (b - 1) + 1];
      if (z1 != z2) return -3;
      bc[i] = 1;
      gv[i] = (y2 - y1) * 1.0;
    } else if (fl == 2 || fl == 3 || fl == 4) {
      bc[i] = 1;
      gv[i] = 0.0;
    }
  }
  // SET_BC_ICCG
  for (int i = 0; i < n; ++i) {
    if (bc[i]) rf[i] = gv[i];
    else {
      cplx temp = D[i] * gv[i];
      for (int q = inl[i]; q < inl[i + 1]; ++q) temp = temp + AL[q] * gv[IAL[q] - 1];
      for (int q = inu[i]; q < inu[i + 1]; ++q) temp = temp + AU[q] * gv[IAU[q] - 1];
      rf[i] = rf[i] - temp;
    }
  }
  for (int i = 0; i < n; ++i) {
    if (bc[i]) {
      D[i] = 1.0;
      for (int q = inl[i]; q < inl[i + 1]; ++q) AL[q] = 0.0;
      for (int q = inu[i]; q < inu[i + 1]; ++q) AU[q] = 0.0;
    } else {
      for (int q = inl[i]; q < inl[i + 1]; ++q)
        if (bc[IAL[q] - 1]) AL[q] = 0.0;
      for (int q = inu[i]; q < inu[i + 1]; ++q)
        if (bc[IAU[q] - 1]) AU[q] = 0.0;
    }
  }
  return 0;
}

// GENBCMT (forward_3DMT.f90:92-177): the Dirichlet values of both polarisations,
// Avalue[isr*nline + i] (complex, isr 0 = Ex, 1 = Ey), and line_bc[nline].  bs[k]
// (k = 0..3) holds the 2-D solution of surface k+2 (its nline values, complex).
void orc_mt_genbcmt(void* h, double omega, int nline, const double* bs2, const double* bs3, const double* bs4,
                    const double* bs5, double* aval_, unsigned char* line_bc) {
  const Surfaces* S = static_cast<Surfaces*>(h);
  cplx* av = reinterpret_cast<cplx*>(aval_);
  const cplx* bs[4] = {reinterpret_cast<const cplx*>(bs2), reinterpret_cast<const cplx*>(bs3),
                       reinterpret_cast<const cplx*>(bs4), reinterpret_cast<const cplx*>(bs5)};
  const cplx iunit(0.0, 1.0);
  for (int i = 0; i < 2 * nline; ++i) av[i] = 0.0;
  for (int i = 0; i < nline; ++i) line_bc[i] = 0;
  // top
  {
    const Surface& s = S->s[0];
    for (int l = 0; l < s.nline; ++l) {
      const int iline = s.ilineface_to_3D[l];
      const int np1 = s.line[2 * l], np2 = s.line[2 * l + 1];
      double dxy[3] = {0.0, 0.0, 0.0};
      for (int c = 0; c < 2; ++c) dxy[c] = s.x1x2[2 * (np2 - 1) + c] - s.x1x2[2 * (np1 - 1) + c];
      const double xhat[3] = {1.0, 0.0, 0.0}, yhat[3] = {0.0, 1.0, 0.0};
      av[iline - 1] = iunit / omega * inner3(dxy, xhat) * 1.0;
      av[nline + iline - 1] = iunit / omega * inner3(dxy, yhat) * 1.0;
      line_bc[iline - 1] = 1;
    }
  }
  // side surfaces 2..5: Ex polarisation on north/south, Ey on west/east
  int isr = 0;
  for (int j = 2; j <= 5; ++j) {
    const Surface& s = S->s[j - 1];
    if (j == 2 || j == 4) isr = 1;
    if (j == 3 || j == 5) isr = 2;
    for (int l = 0; l < s.nline; ++l) {
      const int iline = s.ilineface_to_3D[l];
      av[(long)(isr - 1) * nline + iline - 1] = iunit / omega * bs[j - 2][l];
      line_bc[iline - 1] = 1;
    }
  }
  // bottom: only the column isr left by the side loop (2) is reset
  {
    const Surface& s = S->s[5];
    for (int l = 0; l < s.nline; ++l) {
      const int iline = s.ilineface_to_3D[l];
      av[(long)(isr - 1) * nline + iline - 1] = 0.0;
      line_bc[iline - 1] = 1;
    }
  }
}

// SET_BC_3DJoint (forward_3DMT.f90:553-623): lifts the Dirichlet values of nsr
// columns into rf[isr*n + i] (rf starts at zero, GENMAT_MT's b_vec) and clears the
// Dirichlet rows and columns of the split matrix in place.
void orc_mt_set_bc3d(int n, int nsr, double* D_, double* AL_, const int* INL, const int* IAL, double* AU_,
                     const int* INU, const int* IAU, const double* dval_, const unsigned char* dir, double* rf_) {
  cplx* D = reinterpret_cast<cplx*>(D_);
  cplx* AL = reinterpret_cast<cplx*>(AL_);
  cplx* AU = reinterpret_cast<cplx*>(AU_);
  const cplx* dv = reinterpret_cast<const cplx*>(dval_);
  cplx* rf = reinterpret_cast<cplx*>(rf_);
  for (long i = 0; i < (long)n * nsr; ++i) rf[i] = 0.0;
  for (int i = 0; i < n; ++i) {
    if (dir[i]) {
      for (int j = 0; j < nsr; ++j) rf[(long)j * n + i] = dv[(long)j * n + i];
    } else {
      for (int j = 0; j < nsr; ++j) {
        const cplx* g = dv + (long)j * n;
        cplx temp = D[i] * g[i];
        for (int q = INL[i]; q < INL[i + 1]; ++q) temp = temp + AL[q] * g[IAL[q] - 1];
        for (int q = INU[i]; q < INU[i + 1]; ++q) temp = temp + AU[q] * g[IAU[q] - 1];
        rf[(long)j * n + i] = rf[(long)j * n + i] - temp;
      }
    }
  }
  for (int i = 0; i < n; ++i) {
    if (dir[i]) {
      D[i] = 1.0;
      for (int q = INL[i]; q < INL[i + 1]; ++q) AL[q] = 0.0;
      for (int q = INU[i]; q < INU[i + 1]; ++q) AU[q] = 0.0;
    } else {
      for (int q = INL[i]; q < INL[i + 1]; ++q)
        if (dir[IAL[q] - 1]) AL[q] = 0.0;
      for (int q = INU[i]; q < INU[i + 1]; ++q)
        if (dir[IAU[q] - 1]) AU[q] = 0.0;
    }
  }
}

// CALRESPMT (n_ebfem_3DMT.f90:179-237): Z = E B^-1 per site from the two
// polarisations' fields resp5[(isr*5 + c)*nobs + s] (c = bx, by, bz, ex, ey);
// z[(k*nobs + s)] for k = xx, xy, yx, yy (complex), rho[k*nobs + s] (Ohm m) and
// pha[k*nobs + s] (degrees) with rho = mu0/omega*1e6*|Z|^2.
void orc_mt_calrespmt(int nobs, double omega, const double* resp5_, double* z_, double* rho, double* pha) {
  const cplx* r = reinterpret_cast<const cplx*>(resp5_);
  cplx* zo = reinterpret_cast<cplx*>(z_);
  const double pi = pi_mt(), r2d = 180.0 / pi, dmu = dmu_mt();
  for (int j = 0; j < nobs; ++j) {
    auto ex = [&](int c) { return r[(0 * 5 + c) * (long)nobs + j]; };
    auto ey = [&](int c) { return r[(1 * 5 + c) * (long)nobs + j]; };
    const cplx a = ex(0), c = ex(1), b = ey(0), d = ey(1);
    const cplx det = a * d - b * c;
    cplx bi[2][2] = {{d, -b}, {-c, a}};
    for (int p = 0; p < 2; ++p)
      for (int q = 0; q < 2; ++q) bi[p][q] = bi[p][q] / det;
    const cplx e[2][2] = {{ex(3), ey(3)}, {ex(4), ey(4)}};
    cplx z[2][2];
    for (int p = 0; p < 2; ++p)
      for (int q = 0; q < 2; ++q) z[p][q] = e[p][0] * bi[0][q] + e[p][1] * bi[1][q];
    const double coef = dmu / omega * 1.0e6;
    const cplx zz[4] = {z[0][0], z[0][1], z[1][0], z[1][1]};
    for (int k = 0; k < 4; ++k) {
      zo[(long)k * nobs + j] = zz[k];
      const double amp = std::sqrt(std::pow(zz[k].real(), 2.0) + std::pow(zz[k].imag(), 2.0));
      rho[(long)k * nobs + j] = coef * std::pow(amp, 2.0);
      pha[(long)k * nobs + j] = std::atan2(zz[k].imag(), zz[k].real()) * r2d;
    }
  }
}

}  // extern "C"
