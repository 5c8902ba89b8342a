// Drop-in driver: the reference's forward ctl file and the files it names.
//
// Reference: src/common/m_param.f90:145-446 (readparam), :449-485 (READCOND),
// :939-999 (readcontrolfile / subtractcommentout); src/common/
// m_mesh_type.f90:379-468 (readmsh2); src/common/m_line_type.f90:28-48
// (READLINE); src/src_tide/m_readfvxyz.f90:7-62 (readfxyz / readvxyz);
// src/solver_mpi/n_ebfem_bxyz_mpi.f90:55-183 (driver), :937-1030
// (PREPZSRCOBS), :470-527 (SETNPHYS1INDEX2COND), :570-626 (CALOBSRESP);
// src/common/m_outresp.f90:221-262 (OUTOBSFILESFWD).
#include <cmath>
#include <complex>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <sstream>
#include <string>
#include <vector>

#include "afem_internal.h"

namespace afem {

struct CtlInfo {
  std::string dir;  // directory of the ctl file (relative paths resolve against the working directory, as in Fortran)
  std::string g_meshfile, z_meshfile, lineinfofile, ocean_meshfile, meshctlfile, vxyz_file, fxyz_file,
      outputfolder, header2d, header3d, condfile;
  std::vector<double> freq;
  double xbound[4] = {0, 0, 0, 0}, ybound[4] = {0, 0, 0, 0}, zbound[4] = {0, 0, 0, 0};
  double lenout = 0, upzin = 0, downzin = 0, zmax = 0, zmin = 0;
  int nobs = 0, lonlatflag = 2, ixyflag = 0, nsource = 0, condflag = 0, nvolume = 0;
  double lonorigin = 0, latorigin = 0;
  std::vector<std::string> obsname, sourcename;
  std::vector<double> xyzobs;  // 3*nobs, after PREPZSRCOBS
  double sigma_air = 1e-8;
  std::vector<double> sigma_land;
  int nodes = 0;
  // plan view (ixyflag = 1, 2): OUTFREQFILES2 files <outputfolder><xyfilehead><freq>_S<k>.dat
  std::string xyfilehead;
  int xy_nx = 0, xy_ny = 0, ixydepth = 0;
  double depth_xy = 0.0;
  // seafloor plan views (ixydepth 2, ixyflag 2): the polygon_ki triangle mesh and ki23dptr,
  // its nodes' surface and seafloor nodes of the 3-D mesh (READKI23DPTR, 1-based)
  std::string pokimsh, ki23dfile;
  std::vector<double> ki_xyz;
  std::vector<int32_t> ki_n3, ki23dptr;
  std::vector<double> xyz3d;  // 3-D mesh nodes (PREPZOBS heights, XYSBTM points, GENXYZMINMAX)
  std::vector<double> F, v;   // readfxyz / readvxyz records of the ocean nodes (IXYHOUT)
  bool seafloor() const { return ixyflag == 2 || (ixyflag == 1 && ixydepth == 2); }
};

namespace {

std::string rtrim(const std::string& s) {
  size_t e = s.find_last_not_of(" \t\r\n");
  return e == std::string::npos ? std::string() : s.substr(0, e + 1);
}
std::string ltrim(const std::string& s) {
  size_t b = s.find_first_not_of(" \t\r\n");
  return b == std::string::npos ? std::string() : s.substr(b);
}
std::string trim(const std::string& s) { return ltrim(rtrim(s)); }

// Fortran list-directed tokens: blanks/commas separate; "(a,b)" is one complex item.
std::vector<std::string> tokens(const std::string& line) {
  std::vector<std::string> out;
  size_t i = 0, n = line.size();
  while (i < n) {
    while (i < n && (line[i] == ' ' || line[i] == '\t' || line[i] == ',' || line[i] == '\r')) ++i;
    if (i >= n) break;
    if (line[i] == '/') break;  // list-directed terminator
    size_t j = i;
    if (line[i] == '(') {
      while (j < n && line[j] != ')') ++j;
      out.push_back(line.substr(i, j - i + 1));
      i = j + 1;
      continue;
    }
    if (line[i] == '\'' || line[i] == '"') {
      char q = line[i];
      j = i + 1;
      while (j < n && line[j] != q) ++j;
      out.push_back(line.substr(i + 1, j - i - 1));
      i = j + 1;
      continue;
    }
    while (j < n && line[j] != ' ' && line[j] != '\t' && line[j] != ',' && line[j] != '\r') ++j;
    out.push_back(line.substr(i, j - i));
    i = j;
  }
  return out;
}

double fnum(const std::string& t) {
  std::string s = t;
  for (auto& ch : s)
    if (ch == 'd' || ch == 'D') ch = 'e';
  char* end = nullptr;
  double v = std::strtod(s.c_str(), &end);
  if (end == s.c_str()) throw Error{AFEM_EIO, "cannot read a number from '" + t + "'"};
  return v;
}

void fcomplex(const std::string& t, double* re, double* im) {
  // "(re,im)"
  std::string s = t;
  if (s.size() < 5 || s.front() != '(' || s.back() != ')') throw Error{AFEM_EIO, "bad complex item '" + t + "'"};
  s = s.substr(1, s.size() - 2);
  size_t c = s.find(',');
  if (c == std::string::npos) throw Error{AFEM_EIO, "bad complex item '" + t + "'"};
  *re = fnum(trim(s.substr(0, c)));
  *im = fnum(trim(s.substr(c + 1)));
}

// Sequential record reader over the ctl lines (after readcontrolfile's cut).
struct Records {
  std::vector<std::string> lines;
  size_t pos = 0;
  const std::string& next(const char* what) {
    if (pos >= lines.size()) throw Error{AFEM_EIO, std::string("ctl file ends before ") + what};
    return lines[pos++];
  }
  std::string str(const char* what) { return trim(next(what)); }          // '(a)' read, trimmed
  std::string word(const char* what) {                                     // list-directed character item
    auto t = tokens(next(what));
    return t.empty() ? std::string() : t[0];
  }
  std::vector<double> nums(const char* what, size_t k) {
    auto t = tokens(next(what));
    if (t.size() < k) throw Error{AFEM_EIO, std::string("ctl: too few values for ") + what};
    std::vector<double> v(k);
    for (size_t i = 0; i < k; ++i) v[i] = fnum(t[i]);
    return v;
  }
  double num(const char* what) { return nums(what, 1)[0]; }
  void skip(const char* what) { next(what); }
};

// readcontrolfile + subtractcommentout (m_param.f90:939-999): drop "##"
// lines, keep columns 21.. of the others.
Records read_ctl_records(const std::string& path) {
  std::ifstream f(path);
  if (!f) throw Error{AFEM_EIO, "cannot open ctl file " + path};
  Records r;
  std::string line;
  while (std::getline(f, line)) {
    if (!line.empty() && line.back() == '\r') line.pop_back();
    if (line.size() >= 2 && line[0] == '#' && line[1] == '#') continue;
    r.lines.push_back(line.size() > 20 ? line.substr(20) : std::string());
  }
  return r;
}

struct Msh {
  int node = 0;
  std::vector<double> xyz;
  std::vector<int32_t> n4, n4flag;  // n4flag: (physical, elementary) per tet
  std::vector<int32_t> n3;          // triangles
};

// readmsh2 (m_mesh_type.f90:379-468): Gmsh 2.2 ASCII, two tags per element.
Msh read_msh(const std::string& path, bool want_tets, bool want_tris) {
  std::ifstream f(path);
  if (!f) throw Error{AFEM_EIO, "cannot open mesh file " + path};
  Msh m;
  std::string line;
  for (int i = 0; i < 4; ++i)
    if (!std::getline(f, line)) throw Error{AFEM_EIO, "truncated mesh header in " + path};
  if (!(f >> m.node)) throw Error{AFEM_EIO, "no node count in " + path};
  m.xyz.resize(3L * m.node);
  for (int i = 0; i < m.node; ++i) {
    long id;
    std::string a, b, c;
    if (!(f >> id >> a >> b >> c)) throw Error{AFEM_EIO, "truncated node list in " + path};
    m.xyz[3L * i] = fnum(a);
    m.xyz[3L * i + 1] = fnum(b);
    m.xyz[3L * i + 2] = fnum(c);
  }
  std::getline(f, line);
  std::getline(f, line);  // $EndNodes
  std::getline(f, line);  // $Elements
  long nele = 0;
  if (!(f >> nele)) throw Error{AFEM_EIO, "no element count in " + path};
  static const int etype[16] = {0, 2, 3, 0, 4, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 1};
  for (long e = 0; e < nele; ++e) {
    long id;
    int itype, ntag, jj, kk;
    if (!(f >> id >> itype >> ntag >> jj >> kk)) throw Error{AFEM_EIO, "truncated element list in " + path};
    int nn = (itype >= 0 && itype < 16) ? etype[itype] : 0;
    if (nn == 0) throw Error{AFEM_EIO, "unsupported element type in " + path};
    int nd[4];
    for (int k = 0; k < nn; ++k) f >> nd[k];
    if (itype == 4 && want_tets) {
      for (int k = 0; k < 4; ++k) m.n4.push_back(nd[k]);
      m.n4flag.push_back(jj);
      m.n4flag.push_back(kk);
    } else if (itype == 2 && want_tris) {
      for (int k = 0; k < 3; ++k) m.n3.push_back(nd[k]);
    }
  }
  return m;
}

int count_msh_nodes(const std::string& path) {
  std::ifstream f(path);
  if (!f) throw Error{AFEM_EIO, "cannot open mesh file " + path};
  std::string line;
  for (int i = 0; i < 4; ++i) std::getline(f, line);
  int n = 0;
  if (!(f >> n)) throw Error{AFEM_EIO, "no node count in " + path};
  return n;
}

// READLINE (m_line_type.f90:28-48)
void read_lineinfo(const std::string& path, std::vector<int32_t>& line, std::vector<int32_t>& n6, int& nline,
                   int& ntet) {
  std::ifstream f(path);
  if (!f) throw Error{AFEM_EIO, "cannot open line file " + path};
  if (!(f >> nline)) throw Error{AFEM_EIO, "no nline in " + path};
  line.resize(2L * nline);
  for (long i = 0; i < 2L * nline; ++i)
    if (!(f >> line[i])) throw Error{AFEM_EIO, "truncated line list in " + path};
  if (!(f >> ntet)) throw Error{AFEM_EIO, "no ntet in " + path};
  n6.resize(6L * ntet);
  for (long i = 0; i < 6L * ntet; ++i)
    if (!(f >> n6[i])) throw Error{AFEM_EIO, "truncated n6line in " + path};
}

// readfxyz / readvxyz (m_readfvxyz.f90:7-62): first `nodes` records.
void read_fv(const std::string& fpath, const std::string& vpath, int nodes, std::vector<double>& F,
             std::vector<double>& v) {
  F.assign(3L * nodes, 0.0);
  v.assign(6L * nodes, 0.0);
  std::ifstream ff(fpath), fv(vpath);
  if (!ff) throw Error{AFEM_EIO, "cannot open " + fpath};
  if (!fv) throw Error{AFEM_EIO, "cannot open " + vpath};
  std::string line;
  for (int i = 0; i < nodes; ++i) {
    if (!std::getline(ff, line)) throw Error{AFEM_EIO, "fxyz file has fewer than nodes records"};
    auto t = tokens(line);
    if (t.size() < 6) throw Error{AFEM_EIO, "fxyz record with fewer than 6 values"};
    for (int c = 0; c < 3; ++c) F[3L * i + c] = fnum(t[3 + c]);
  }
  for (int i = 0; i < nodes; ++i) {
    if (!std::getline(fv, line)) throw Error{AFEM_EIO, "vxyz file has fewer than nodes records"};
    auto t = tokens(line);
    if (t.size() < 5) throw Error{AFEM_EIO, "vxyz record with fewer than 5 values"};
    fcomplex(t[3], &v[6L * i + 0], &v[6L * i + 1]);
    fcomplex(t[4], &v[6L * i + 2], &v[6L * i + 3]);
    v[6L * i + 4] = 0.0;
    v[6L * i + 5] = 0.0;
  }
}

// READCOND (m_param.f90:449-485): 11 header lines, nphys2, then "index rho".
void read_cond(const std::string& path, std::vector<double>& sigma) {
  std::ifstream f(path);
  if (!f) throw Error{AFEM_EIO, "cannot open cond file " + path};
  std::string line;
  for (int i = 0; i < 11; ++i)
    if (!std::getline(f, line)) throw Error{AFEM_EIO, "truncated cond header in " + path};
  int nphys2 = 0;
  if (!(f >> nphys2)) throw Error{AFEM_EIO, "no nphys2 in " + path};
  sigma.assign(nphys2, -9999.0);
  for (int i = 0; i < nphys2; ++i) {
    long idx;
    std::string r;
    if (!(f >> idx >> r)) throw Error{AFEM_EIO, "truncated cond list in " + path};
    const double rho = fnum(r);
    if (std::fabs(rho) > 1e-10) sigma[i] = 1.0 / rho;
  }
}

// PREPZSRCOBS (n_ebfem_bxyz_mpi.f90:976-998) with findtri's barycentrics
// (m_triangle.f90:133-260): z += surface height interpolated in the first
// triangle (id order) that contains (x, y).  The reference visits candidate
// triangles bucket by bucket; on a shared edge both triangles give the same
// height up to rounding.
void lift_sites(const Msh& h, std::vector<double>& xyzobs) {
  const long ntri = (long)h.n3.size() / 3;
  const int nobs = (int)xyzobs.size() / 3;
  for (int s = 0; s < nobs; ++s) {
    const double x = xyzobs[3 * s], y = xyzobs[3 * s + 1];
    bool found = false;
    for (long t = 0; t < ntri && !found; ++t) {
      const double* p[3];
      for (int j = 0; j < 3; ++j) p[j] = &h.xyz[3L * (h.n3[3 * t + j] - 1)];
      const double x12[2] = {p[1][0] - p[0][0], p[1][1] - p[0][1]};
      const double x13[2] = {p[2][0] - p[0][0], p[2][1] - p[0][1]};
      const double x23[2] = {p[2][0] - p[1][0], p[2][1] - p[1][1]};
      const double v1[2] = {x - p[0][0], y - p[0][1]};
      const double v2[2] = {x - p[1][0], y - p[1][1]};
      const double a0 = (x13[0] * x12[1] - x13[1] * x12[0]);
      double a[3];
      a[1] = (x13[0] * v1[1] - x13[1] * v1[0]) / a0;
      a[2] = (v1[0] * x12[1] - v1[1] * x12[0]) / a0;
      a[0] = (v2[0] * x23[1] - v2[1] * x23[0]) / a0;
      if (a[0] >= 0.0 && a[1] >= 0.0 && a[2] >= 0.0) {
        xyzobs[3 * s + 2] = a[0] * p[0][2] + a[1] * p[1][2] + a[2] * p[2][2] + xyzobs[3 * s + 2];
        found = true;
      }
    }
    if (!found) throw Error{AFEM_EIO, "site outside the surface mesh (PREPZSRCOBS)"};
  }
}

}  // namespace

// Longitude/latitude (deg) to UTM easting/northing (m) in `zone`: the ellipsoidal
// transverse Mercator of Snyder ("Map Projections -- A Working Manual", USGS
// Professional Paper 1395, 1987, eqs. 8-9 to 8-13, Clarke 1866 ellipsoid, scale
// 0.9996, false easting 500 km) in the form utm_geo_tm evaluates it for
// LONLAT2UTM (src/common/m_param.f90:741-936, called by UTMGMT, :629-661).  One
// term is kept as the reference has it: the sin(4 phi) coefficient of the
// meridional arc multiplies 15 e^4/256 by 45 e^6/1024 where Snyder adds them, so
// northings differ from Snyder's by up to ~17 m; the sites must land where the
// reference puts them.
void utm_lonlat2xy(double lon, double lat, int zone, double* x, double* y) {
  const double pi = 3.141592653589793, degrad = pi / 180.0;
  const double a_ = 6378206.4, b_ = 6356583.8, k0 = 0.9996;
  const double e2 = 1.0 - std::pow(b_ / a_, 2.0), e4 = e2 * e2, e6 = e2 * e4, ep2 = e2 / (1.0 - e2);
  const double cm = zone * 6.0 - 183.0;
  const double rlat = degrad * lat;
  double delam = lon - cm;
  if (delam < -180.0) delam += 360.0;
  if (delam > 180.0) delam -= 360.0;
  delam *= degrad;
  const double f1 = (1.0 - e2 / 4.0 - 3.0 * e4 / 64.0 - 5.0 * e6 / 256.0) * rlat;
  const double f2 = (3.0 * e2 / 8.0 + 3.0 * e4 / 32.0 + 45.0 * e6 / 1024.0) * std::sin(2.0 * rlat);
  const double f3 = (15.0 * e4 / 256.0 * 45.0 * e6 / 1024.0) * std::sin(4.0 * rlat);  // the reference's product
  const double f4 = 35.0 * e6 / 3072.0 * std::sin(6.0 * rlat);
  const double rm = a_ * (f1 - f2 + f3 - f4);
  double xx, yy;
  if (lat == 90.0 || lat == -90.0) {
    xx = 0.0;
    yy = k0 * rm;
  } else {
    const double sl = std::sin(rlat), cl = std::cos(rlat), tl = std::tan(rlat);
    const double rn = a_ / std::sqrt(1.0 - e2 * sl * sl);
    const double t = tl * tl, c = ep2 * cl * cl, A = cl * delam;
    const double A2 = A * A, A3 = A2 * A, A4 = A2 * A2, A5 = A4 * A, A6 = A4 * A2;
    xx = k0 * rn * (A + (1.0 - t + c) * A3 / 6.0 + (5.0 - 18.0 * t + t * t + 72.0 * c - 58.0 * ep2) * A5 / 120.0);
    yy = k0 * (rm + rn * tl * (A2 / 2.0 + (5.0 - t + 9.0 * c + 4.0 * c * c) * A4 / 24.0 +
                               (61.0 - 58.0 * t + t * t + 600.0 * c - 330.0 * ep2) * A6 / 720.0));
  }
  *x = xx + 500000.0;
  *y = yy;
}

namespace {

// UTMXY (m_param.f90:609-627): site position in km east/north of the origin, both in UTM zone `zone`
void utmxy(double lon, double lat, double lonorigin, double latorigin, int zone, double* xkm, double* ykm) {
  double x, y, x0, y0;
  utm_lonlat2xy(lon, lat, zone, &x, &y);
  utm_lonlat2xy(lonorigin, latorigin, zone, &x0, &y0);
  *xkm = (x - x0) / 1e3;
  *ykm = (y - y0) / 1e3;
}

// The 2-D grid list of a triangle mesh and its point search (allocate_2Dgrid_list,
// gen2Dgridforlist, classifytri2grd, findtriwithgrid, FINDTRI; src/common/
// m_triangle.f90:11-260), as PREPZOBS uses it to find the seafloor under a
// plan-view point: nx x ny boxes over [xmin, xmax] x [ymin, ymax] (the 3-D mesh's
// node extent), each triangle listed in the box of its centroid (strictly
// inside; a centroid on a box boundary stops the reference), the list in
// SORT_INDEX (heap) order; a point's box is half-open (lo, hi], and shells of
// boxes grow around it until a listed triangle holds the point.
struct TriGrid {
  int nx = 0, ny = 0;
  std::vector<double> xg, yg;     // nx+1 / ny+1 boundaries
  std::vector<int32_t> stack;     // 0..nx*ny: triangles in boxes <= b
  std::vector<int32_t> ordered;   // 0-based triangle ids in list order
};

TriGrid make_tri_grid(const std::vector<double>& xyz, const std::vector<int32_t>& n3, const double mm[4], int nx,
                      int ny) {
  TriGrid g;
  g.nx = nx;
  g.ny = ny;
  g.xg.resize(nx + 1);
  g.yg.resize(ny + 1);
  for (int i = 0; i <= ny; ++i) g.yg[i] = (double)i * (mm[3] - mm[2]) / (double)ny + mm[2];
  for (int i = 0; i <= nx; ++i) g.xg[i] = (double)i * (mm[1] - mm[0]) / (double)nx + mm[0];
  const long ntri = (long)n3.size() / 3;
  // strict box of a centroid coordinate: g[i-1] < v < g[i], 1-based i, 0 if none
  auto sbox = [](const std::vector<double>& gr, double v) {
    const int pos = (int)(std::lower_bound(gr.begin(), gr.end(), v) - gr.begin());  // count of gr < v
    return (pos >= 1 && pos < (int)gr.size() && v < gr[pos]) ? pos : 0;
  };
  std::vector<double> order(ntri);
  std::vector<int32_t> index(ntri);
  for (long t = 0; t < ntri; ++t) {
    double x2[2] = {0.0, 0.0};
    for (int j = 0; j < 3; ++j)
      for (int c = 0; c < 2; ++c) x2[c] = x2[c] + xyz[3L * (n3[3 * t + j] - 1) + c] / 3.0;
    const int iy = sbox(g.yg, x2[1]), ix = sbox(g.xg, x2[0]);
    AFEM_REQUIRE(ix && iy, AFEM_EIO,
                 "seafloor plan view: a polygon_ki triangle's centroid lies on a box boundary or outside the "
                 "3-D mesh (classifytri2grd)");
    order[t] = (double)((long)nx * (iy - 1) + ix);
    index[t] = (int32_t)(t + 1);
  }
  sort_index_heap((int)ntri, index.data(), order.data());
  g.stack.assign((long)nx * ny + 1, 0);
  for (long t = 0; t < ntri; ++t) g.stack[(long)order[t]] += 1;
  for (long b = 1; b <= (long)nx * ny; ++b) g.stack[b] += g.stack[b - 1];
  g.ordered.resize(ntri);
  for (long t = 0; t < ntri; ++t) g.ordered[t] = index[t] - 1;
  return g;
}

// findtriwithgrid + FINDTRI: 0-based triangle holding (x, y) and its coordinates a[3]; false if none
bool find_tri(const TriGrid& g, const std::vector<double>& xyz, const std::vector<int32_t>& n3, double x, double y,
              int* tri, double a[3]) {
  auto hbox = [](const std::vector<double>& gr, double v) {  // gr[i-1] < v <= gr[i]
    const int pos = (int)(std::lower_bound(gr.begin(), gr.end(), v) - gr.begin());
    return (pos >= 1 && pos < (int)gr.size()) ? pos : 0;
  };
  const int iy = hbox(g.yg, y), ix = hbox(g.xg, x);
  if (!ix || !iy) return false;
  for (int iside = 0; iside <= std::max(g.nx, g.ny); ++iside) {  // the reference grows iside without bound
    for (int k = std::max(iy - iside, 1); k <= std::min(iy + iside, g.ny); ++k)
      for (int j = std::max(ix - iside, 1); j <= std::min(ix + iside, g.nx); ++j) {
        if (iy - (iside - 1) <= k && k <= iy + (iside - 1) && ix - (iside - 1) <= j && j <= ix + (iside - 1))
          continue;
        const long idx = (long)g.nx * (k - 1) + j;
        for (int q = g.stack[idx - 1]; q < g.stack[idx]; ++q) {
          const int t = g.ordered[q];
          const double* p[3];
          for (int m = 0; m < 3; ++m) p[m] = &xyz[3L * (n3[3 * t + m] - 1)];
          const double x12[2] = {p[1][0] - p[0][0], p[1][1] - p[0][1]};
          const double x13[2] = {p[2][0] - p[0][0], p[2][1] - p[0][1]};
          const double x23[2] = {p[2][0] - p[1][0], p[2][1] - p[1][1]};
          const double v1[2] = {x - p[0][0], y - p[0][1]};
          const double v2[2] = {x - p[1][0], y - p[1][1]};
          const double a0 = (x13[0] * x12[1] - x13[1] * x12[0]);
          a[1] = (x13[0] * v1[1] - x13[1] * v1[0]) / a0;
          a[2] = (v1[0] * x12[1] - v1[1] * x12[0]) / a0;
          a[0] = (v2[0] * x23[1] - v2[1] * x23[0]) / a0;
          if (a[0] >= 0.0 && a[1] >= 0.0 && a[2] >= 0.0) {
            *tri = t;
            return true;
          }
        }
      }
  }
  return false;
}

// Fortran Gw.d edit descriptor (G15.7 of OUTOBSFILESFWD) for finite values.
std::string fortran_g(double x, int w, int d) {
  char buf[64];
  const double ax = std::fabs(x);
  if (x == 0.0) {
    std::snprintf(buf, sizeof(buf), "%*.*f%*s", w - 4, d - 1, 0.0, 4, "");
    return buf;
  }
  // F editing when 0.1 - 0.5e-(d+1) <= |x| < 10^d - 0.5
  if (ax >= 0.1 - 0.5 * std::pow(10.0, -(d + 1)) && ax < std::pow(10.0, d) - 0.5) {
    int k = 0;
    // smallest k with |x| < 10^k - 0.5*10^(k-d)
    for (k = 0; k <= d; ++k)
      if (ax < std::pow(10.0, k) - 0.5 * std::pow(10.0, k - d)) break;
    std::snprintf(buf, sizeof(buf), "%*.*f%*s", w - 4, d - k, x, 4, "");
    return buf;
  }
  // Ew.d: [-]0.ddddddE+ee
  int e10 = (int)std::floor(std::log10(ax)) + 1;
  double mant = ax / std::pow(10.0, e10);
  double r = std::round(mant * std::pow(10.0, d)) / std::pow(10.0, d);
  if (r >= 1.0) { r /= 10.0; e10 += 1; }
  char mb[32];
  std::snprintf(mb, sizeof(mb), "%.*f", d, r);  // "0.ddddddd"
  char eb[16];
  std::snprintf(eb, sizeof(eb), "E%c%02d", e10 < 0 ? '-' : '+', std::abs(e10));
  std::string s = std::string(x < 0 ? "-" : "") + mb + eb;
  if ((int)s.size() < w) s = std::string(w - s.size(), ' ') + s;
  return s;
}

}  // namespace

int load_ctl(afem_ctx* c, const char* path) {
  AFEM_REQUIRE(path, AFEM_EINVAL, "load_ctl: null path");
  destroy_ctl(c);
  CtlInfo* ci = new CtlInfo();
  c->ctl = ci;
  Records r = read_ctl_records(path);
  const int itopoflag = (int)r.num("itopoflag");
  if (itopoflag == 1) {
    const int nfile = (int)r.num("nfile");
    for (int i = 0; i < nfile; ++i) {
      r.skip("topofile");
      r.skip("lonlatshift");
    }
  } else if (itopoflag != 0) {
    throw Error{AFEM_EIO, "ctl: itopoflag should be 0 or 1"};
  }
  ci->g_meshfile = r.str("mesh file");
  ci->z_meshfile = r.str("2d triangle z file");
  ci->lineinfofile = r.str("line file");
  ci->ocean_meshfile = r.str("ocean mesh file");
  ci->meshctlfile = r.str("mesh ctl file");
  ci->vxyz_file = r.str("vxyz file");
  ci->fxyz_file = r.str("fxyz file");
  ci->outputfolder = r.str("output folder");
  ci->header2d = r.str("header2d");
  ci->header3d = r.str("header3d");
  const int nfreq = (int)r.num("nfreq");
  for (int i = 0; i < nfreq; ++i) ci->freq.push_back(r.num("frequency"));
  ci->xbound[1] = r.num("west bound");
  ci->xbound[2] = r.num("east bound");
  ci->ybound[1] = r.num("south bound");
  ci->ybound[2] = r.num("north bound");
  ci->lenout = r.num("lenout");
  ci->upzin = r.num("upzin");
  ci->downzin = r.num("downzin");
  ci->zmax = r.num("zmax");
  ci->zmin = r.num("zmin");
  for (int i = 0; i < 7; ++i) r.skip("mesh size / obs / source parameters");
  // zbound / xbound / ybound (m_param.f90:259-264)
  ci->zbound[0] = ci->zmin; ci->zbound[1] = ci->downzin; ci->zbound[2] = ci->upzin; ci->zbound[3] = ci->zmax;
  ci->xbound[0] = ci->xbound[1] - ci->lenout;
  ci->xbound[3] = -ci->xbound[0];
  ci->ybound[0] = ci->ybound[1] - ci->lenout;
  ci->ybound[3] = -ci->ybound[0];
  ci->nobs = (int)r.num("nobs");
  ci->lonlatflag = (int)r.num("lonlatflag");
  AFEM_REQUIRE(ci->lonlatflag >= 0 && ci->lonlatflag <= 2, AFEM_EIO, "ctl: lonlatflag should be 0, 1 or 2");
  int utm_zone = 0;
  if (ci->lonlatflag == 1) {
    // read(input,*) c_param%UTM (character(3)); UTMGMT reads the zone number from its first two characters
    const std::string z = r.word("UTM zone");
    const std::string z2 = z.substr(0, 2);
    char* end = nullptr;
    utm_zone = (int)std::strtol(z2.c_str(), &end, 10);
    AFEM_REQUIRE(end != z2.c_str() && utm_zone >= 1 && utm_zone <= 60, AFEM_EIO, "ctl: bad UTM zone '" + z + "'");
  } else {
    r.skip("UTM zone line");
  }
  auto org = r.nums("lonlatorigin", 2);
  ci->lonorigin = org[0];
  ci->latorigin = org[1];
  const double pi = 4.0 * std::atan(1.0), d2r = pi / 180.0, radius = 6371.2;
  for (int i = 0; i < ci->nobs; ++i) {
    ci->obsname.push_back(r.str("site name"));
    auto v = r.nums("site coordinates", 3);
    if (ci->lonlatflag == 0) {
      ci->xyzobs.push_back((v[0] - ci->lonorigin) * d2r * radius * std::cos(ci->latorigin * d2r));
      ci->xyzobs.push_back((v[1] - ci->latorigin) * d2r * radius);
      ci->xyzobs.push_back(v[2]);
    } else if (ci->lonlatflag == 1) {  // UTMXY (m_param.f90:316-323)
      double xk, yk;
      utmxy(v[0], v[1], ci->lonorigin, ci->latorigin, utm_zone, &xk, &yk);
      ci->xyzobs.push_back(xk);
      ci->xyzobs.push_back(yk);
      ci->xyzobs.push_back(v[2]);
    } else {
      ci->xyzobs.insert(ci->xyzobs.end(), v.begin(), v.end());
    }
  }
  ci->ixyflag = (int)r.num("ixyflag");
  AFEM_REQUIRE(ci->ixyflag >= 0 && ci->ixyflag <= 2, AFEM_EIO, "ctl: ixyflag should be 0, 1 or 2");
  if (ci->ixyflag == 1) {
    ci->xyfilehead = r.word("xyfilehead");
    auto nxy = r.nums("nx ny", 2);
    ci->xy_nx = (int)nxy[0];
    ci->xy_ny = (int)nxy[1];
    ci->ixydepth = (int)r.num("ixydepth");
    AFEM_REQUIRE(ci->ixydepth == 1 || ci->ixydepth == 2, AFEM_EIO, "ctl: ixydepth should be 1 or 2");
    if (ci->ixydepth == 1) ci->depth_xy = r.num("depth_xy");
    ci->pokimsh = r.str("pokimsh");
    ci->ki23dfile = r.str("ki23dfile");
  } else if (ci->ixyflag == 2) {
    ci->xyfilehead = r.word("xyfilehead");
    ci->pokimsh = r.str("pokimsh");
    ci->ki23dfile = r.str("ki23dfile");
  }
  ci->nsource = (int)r.num("nsource");
  for (int i = 0; i < ci->nsource; ++i) {
    ci->sourcename.push_back(r.word("source name"));
    r.skip("source start");
    r.skip("source end");
  }
  r.skip("source current");
  ci->sigma_air = r.num("sigma_air");
  ci->condflag = (int)r.num("condflag");
  std::vector<double> sigma_file;
  if (ci->condflag == 0) {
    ci->nvolume = (int)r.num("nvolume");
    for (int i = 0; i < ci->nvolume; ++i) ci->sigma_land.push_back(r.num("sigma_land"));
  } else if (ci->condflag == 1) {
    ci->condfile = trim(r.next("condfile").substr(0, 50));
    read_cond(ci->condfile, sigma_file);
  } else {
    throw Error{AFEM_EIO, "ctl: condflag should be 0 or 1"};
  }
  // mesh, surface, ocean node count, edges
  Msh g = read_msh(ci->g_meshfile, true, false);
  Msh h = read_msh(ci->z_meshfile, false, true);
  ci->xyz3d = g.xyz;
  if (ci->seafloor()) {
    // READMESH_TOTAL(ki_mesh, pokimsh) + READKI23DPTR (n_ebfem_bxyz_mpi.f90:67-70, 305-328); the
    // constant-depth view does not use them, so they are read only for the seafloor views
    Msh k = read_msh(ci->pokimsh, false, true);
    ci->ki_xyz = k.xyz;
    ci->ki_n3 = k.n3;
    std::ifstream f(ci->ki23dfile);
    AFEM_REQUIRE((bool)f, AFEM_EIO, "cannot open ki23dfile " + ci->ki23dfile);
    long ndat = 0;
    AFEM_REQUIRE((bool)(f >> ndat), AFEM_EIO, "no count in " + ci->ki23dfile);
    AFEM_REQUIRE(ndat == k.node, AFEM_EIO, "ki23dfile: the count differs from the polygon_ki node count");
    ci->ki23dptr.resize(2 * ndat);
    for (long i = 0; i < 2 * ndat; ++i) {
      std::string tok;
      AFEM_REQUIRE((bool)(f >> tok), AFEM_EIO, "truncated " + ci->ki23dfile);
      ci->ki23dptr[i] = (int32_t)fnum(tok);  // read as real(8), used as integer(4)
      AFEM_REQUIRE(ci->ki23dptr[i] >= 1 && ci->ki23dptr[i] <= g.node, AFEM_EIO,
                   "ki23dfile: a node id outside the 3-D mesh");
    }
    for (int32_t id : ci->ki_n3)
      AFEM_REQUIRE(id >= 1 && id <= k.node, AFEM_EIO, "polygon_ki mesh: a triangle node id out of range");
  }
  ci->nodes = count_msh_nodes(ci->ocean_meshfile);
  lift_sites(h, ci->xyzobs);
  std::vector<int32_t> line, n6;
  int nline = 0, ntet_l = 0;
  read_lineinfo(ci->lineinfofile, line, n6, nline, ntet_l);
  const int ntet = (int)g.n4.size() / 4;
  AFEM_REQUIRE(ntet_l == ntet, AFEM_EIO, "lineinfo ntet differs from the mesh");
  std::vector<int32_t> tag(ntet);
  for (int t = 0; t < ntet; ++t) tag[t] = g.n4flag[2 * t + 1];  // n4flag(:,2): elementary tag
  int rc = afem_set_mesh(c, g.node, g.xyz.data(), ntet, g.n4.data(), tag.data(), nline, line.data(), n6.data());
  if (rc) throw Error{rc, c->err};
  // GENMAT's ocean value is the default-real literal 3.33
  rc = afem_set_cond(c, ci->sigma_air, (double)3.33f, ci->condflag, ci->nvolume,
                     ci->sigma_land.empty() ? nullptr : ci->sigma_land.data(), (int)sigma_file.size(),
                     sigma_file.empty() ? nullptr : sigma_file.data());
  if (rc) throw Error{rc, c->err};
  std::vector<double>& F = ci->F;
  std::vector<double>& v = ci->v;
  read_fv(ci->fxyz_file, ci->vxyz_file, ci->nodes, F, v);
  rc = afem_set_source(c, 0, ci->nodes, F.data(), v.data());
  if (rc) throw Error{rc, c->err};
  // forward_bxyz: zmin = zbound(1), zmax = zbound(4), xout = xbound(4), yout = ybound(4)
  rc = afem_set_bounds(c, ci->zbound[0], ci->zbound[3], ci->xbound[3], ci->ybound[3]);
  if (rc) throw Error{rc, c->err};
  return AFEM_OK;
}

int ctl_info(afem_ctx* c, int* nfreq, double* freq, int* nobs, double* xyz) {
  AFEM_REQUIRE(c->ctl, AFEM_ESTATE, "ctl_info: no ctl loaded");
  CtlInfo* ci = c->ctl;
  if (nfreq) *nfreq = (int)ci->freq.size();
  if (freq) std::memcpy(freq, ci->freq.data(), sizeof(double) * ci->freq.size());
  if (nobs) *nobs = ci->nobs;
  if (xyz) std::memcpy(xyz, ci->xyzobs.data(), sizeof(double) * ci->xyzobs.size());
  return AFEM_OK;
}

// Fortran Ew.d as write(num,'(e9.2)') prints a frequency for the plan-view file names
// (OUTFREQFILES2, m_outresp.f90:192): [sign]0.ddE+ee, mantissa in [0.1, 1).
std::string fortran_e(double x, int w, int d) {
  char buf[64];
  const double ax = std::fabs(x);
  int e = 0;
  double m = 0.0;
  if (ax > 0.0) {
    e = (int)std::floor(std::log10(ax)) + 1;
    m = ax / std::pow(10.0, e);
    if (m < 0.1) { m *= 10.0; e -= 1; }
    if (m >= 1.0) { m /= 10.0; e += 1; }
    const double scale = std::pow(10.0, d);
    double r = std::nearbyint(m * scale) / scale;
    if (r >= 1.0) { r /= 10.0; e += 1; }
    m = r;
  }
  std::snprintf(buf, sizeof(buf), "%s0.%0*lldE%c%02d", x < 0 ? "-" : "", d, (long long)std::llround(m * std::pow(10.0, d)),
                e < 0 ? '-' : '+', std::abs(e));
  std::string s(buf);
  if ((int)s.size() < w) s = std::string(w - s.size(), ' ') + s;
  return s;
}

// Fortran Fw.d: right-justified fixed point, asterisks when it does not fit.
std::string fortran_f(double x, int w, int d) {
  char buf[96];
  std::snprintf(buf, sizeof(buf), "%*.*f", w, d, x);
  std::string s(buf);
  if ((int)s.size() > w) s = std::string(w, '*');
  return s;
}

namespace {

// GENXYZMINMAX (n_ebfem_bxyz_mpi.f90:533-565): xmin, xmax, ymin, ymax of the 3-D mesh nodes
void xy_extent(const std::vector<double>& xyz, double mm[4]) {
  mm[0] = mm[1] = xyz[0];
  mm[2] = mm[3] = xyz[1];
  for (size_t i = 0; i < xyz.size() / 3; ++i) {
    mm[0] = std::min(mm[0], xyz[3 * i]);
    mm[1] = std::max(mm[1], xyz[3 * i]);
    mm[2] = std::min(mm[2], xyz[3 * i + 1]);
    mm[3] = std::max(mm[3], xyz[3 * i + 1]);
  }
}

// PREPZOBS with iflag 1 (n_ebfem_bxyz_mpi.f90:1181-1267): each plan-view point goes
// 1 m below the seafloor under it (the polygon_ki triangle holding it, interpolating
// the heights of its nodes' seafloor nodes ki23dptr(2,:)); the same three nodes and
// weights are IXYHOUT's coeff_vF row of the point.
void prepzobs(const CtlInfo* ci, std::vector<double>& xy, std::vector<int32_t>& item, std::vector<double>& val) {
  const int np = (int)xy.size() / 3;
  double mm[4];
  xy_extent(ci->xyz3d, mm);
  const TriGrid g = make_tri_grid(ci->ki_xyz, ci->ki_n3, mm, 200, 200);
  item.resize(3L * np);
  val.resize(3L * np);
  for (int p = 0; p < np; ++p) {
    int t = 0;
    double a[3];
    AFEM_REQUIRE(find_tri(g, ci->ki_xyz, ci->ki_n3, xy[3L * p], xy[3L * p + 1], &t, a), AFEM_EIO,
                 "seafloor plan view: a point lies outside the polygon_ki mesh (findtriwithgrid)");
    double z[3];
    for (int j = 0; j < 3; ++j) {
      const int m = ci->ki23dptr[2L * (ci->ki_n3[3L * t + j] - 1) + 1];
      item[3L * p + j] = m;
      val[3L * p + j] = a[j];
      z[j] = ci->xyz3d[3L * (m - 1) + 2];
    }
    xy[3L * p + 2] = a[0] * z[0] + a[1] * z[1] + a[2] * z[2] - 0.001;
  }
}

// PREPOBSCOEFF_XYSBTM's points (n_ebfem_bxyz_mpi.f90:1064-1078): per polygon_ki
// triangle the mean of its nodes' seafloor nodes, raised by 1 m, with coeff_vF
// weights 1/3 on those nodes.
void xysbtm_points(const CtlInfo* ci, std::vector<double>& xy, std::vector<int32_t>& item, std::vector<double>& val) {
  const long ntri = (long)ci->ki_n3.size() / 3;
  xy.assign(3 * ntri, 0.0);
  item.resize(3 * ntri);
  val.resize(3 * ntri);
  const double up[3] = {0.0, 0.0, 0.001};
  for (long i = 0; i < ntri; ++i) {
    double x3[3] = {0.0, 0.0, 0.0};
    for (int j = 0; j < 3; ++j) {
      const int m = ci->ki23dptr[2L * (ci->ki_n3[3 * i + j] - 1) + 1];
      for (int c = 0; c < 3; ++c) x3[c] = x3[c] + ci->xyz3d[3L * (m - 1) + c] / 3.0 + up[c] / 3.0;
      item[3 * i + j] = m;
      val[3 * i + j] = 1.0 / 3.0;
    }
    for (int c = 0; c < 3; ++c) xy[3 * i + c] = x3[c];
  }
}

// IXYHOUT (n_ebfem_bxyz_mpi.f90:192-302): the depth-integrated ocean current of each
// plan-view point, <outputfolder>ixyh_xy2D<freq>.dat with 26 E15.7 columns: x, y, z,
// sigma h E, sigma h (v x F), their sum, h v (x, y, complex), B (3 complex), h.
// fields: complex bx, by, bz, ex, ey of source 1 (5 x np); the reference reads them
// back from amplitude and phase, and takes sigma_ocean from the default-real 3.3.
void write_ixyhout(const CtlInfo* ci, double freq, const std::vector<double>& xy, const double* fields,
                   const std::vector<int32_t>& item, const std::vector<double>& val) {
  const int np = (int)xy.size() / 3;
  const double pi = 4.0 * std::atan(1.0), d2r = pi / 180.0, r2d = 180.0 / pi;
  const double sig = (double)3.3f;
  using cx = std::complex<double>;
  auto vnode = [&](int m, int c) {  // readvxyz: ocean nodes 1..nodes, zero beyond
    return m <= ci->nodes ? cx(ci->v[6L * (m - 1) + 2 * c], ci->v[6L * (m - 1) + 2 * c + 1]) : cx(0.0, 0.0);
  };
  auto fnode = [&](int m, int c) { return m <= ci->nodes ? ci->F[3L * (m - 1) + c] : 0.0; };
  const std::string num = trim(fortran_e(freq, 9, 2));
  const std::string fn = rtrim(ci->outputfolder.substr(0, 70)) + "ixyh_xy2D" + num + ".dat";
  FILE* f = std::fopen(fn.c_str(), "w");
  if (!f) throw Error{AFEM_EIO, "cannot write " + fn};
  for (int i = 0; i < np; ++i) {
    double h = -xy[3L * i + 2];
    if (h <= 0.0) h = 0.0;
    cx rec[5];
    for (int comp = 0; comp < 5; ++comp) {
      const double re = fields[2 * ((long)comp * np + i)], im = fields[2 * ((long)comp * np + i) + 1];
      const double amp = std::sqrt(std::pow(re, 2.0) + std::pow(im, 2.0));
      const double ph = std::atan2(im, re) * r2d;
      rec[comp] = amp * std::exp(cx(0.0, ph * d2r));
    }
    cx vf[3] = {0.0, 0.0, 0.0}, vh[2] = {0.0, 0.0};
    for (int k = 0; k < 3; ++k) {
      const int m = item[3L * i + k];
      const double w = val[3L * i + k];
      const cx v1 = vnode(m, 0), v2 = vnode(m, 1), v3 = vnode(m, 2);
      const double F1 = fnode(m, 0), F2 = fnode(m, 1), F3 = fnode(m, 2);
      const cx c1 = v2 * F3 - v3 * F2, c2 = v3 * F1 - v1 * F3, c3 = v1 * F2 - v2 * F1;  // cr_outer(v, F)
      vf[0] = vf[0] + w * c1;
      vf[1] = vf[1] + w * c2;
      vf[2] = vf[2] + w * c3;
      vh[0] = vh[0] + w * v1;
      vh[1] = vh[1] + w * v2;
    }
    cx out[9];
    for (int c = 0; c < 2; ++c) {
      out[c] = sig * h * rec[3 + c];                         // ixyh_e
      out[2 + c] = sig * h * vf[c] * 1e-3;                   // ixyh_vF
      out[4 + c] = sig * h * (rec[3 + c] + vf[c] * 1e-3);    // ixyh
      out[6 + c] = h * vh[c];                                // vh_obs
    }
    std::string row;
    for (int j = 0; j < 3; ++j) row += fortran_e(xy[3L * i + j], 15, 7);
    for (int j = 0; j < 8; ++j) row += fortran_e(out[j].real(), 15, 7) + fortran_e(out[j].imag(), 15, 7);
    for (int c = 0; c < 3; ++c) row += fortran_e(rec[c].real(), 15, 7) + fortran_e(rec[c].imag(), 15, 7);
    row += fortran_e(h, 15, 7);
    std::fprintf(f, "%s\n", row.c_str());
  }
  std::fclose(f);
}

}  // namespace

// Frequency loop of n_ebfem_bxyz (n_ebfem_bxyz_mpi.f90:144-183): one forward
// solve per frequency, CALOBSEBCOMP, then OUTOBSFILESFWD.  GENMAT fills
// right-hand-side column 1 only, so sources 2..nsr have zero fields.
int run_ctl(afem_ctx* c, const afem_solve_opts* o) {
  AFEM_REQUIRE(c->ctl, AFEM_ESTATE, "run_ctl: no ctl loaded");
  AFEM_REQUIRE(o, AFEM_EINVAL, "run_ctl: null options");
  CtlInfo* ci = c->ctl;
  int rc = afem_assemble(c);
  if (rc) throw Error{rc, c->err};
  const int nf = (int)ci->freq.size(), nobs = ci->nobs;
  // plan-view points: PREPOBSCOEFF_XY's cells of [xbound(2), xbound(3)] x [ybound(2), ybound(3)]
  // at depth_xy (ixydepth 1) or 1 m below the seafloor (ixydepth 2, PREPZOBS), or
  // PREPOBSCOEFF_XYSBTM's polygon_ki triangles (ixyflag 2); the seafloor views also
  // write IXYHOUT's file (with ixydepth 1 the reference's IXYHOUT reads coeff_vF rows
  // that nothing built, so that file is not written there)
  std::vector<double> xy;
  std::vector<int32_t> vf_item;
  std::vector<double> vf_val;
  int nxy = 0, grid_nz = 50;
  if (ci->ixyflag == 1) {
    nxy = ci->xy_nx * ci->xy_ny;
    xy.resize(3L * nxy);
    rc = afem_xy_points(ci->xbound[1], ci->xbound[2], ci->ybound[1], ci->ybound[2], ci->xy_nx, ci->xy_ny,
                        ci->ixydepth == 1 ? ci->depth_xy : 0.0, xy.data());
    if (rc) throw Error{rc, "run_ctl: plan-view grid"};
    if (ci->ixydepth == 2) prepzobs(ci, xy, vf_item, vf_val);
  } else if (ci->ixyflag == 2) {
    xysbtm_points(ci, xy, vf_item, vf_val);
    nxy = (int)xy.size() / 3;
    grid_nz = 300;  // PREPOBSCOEFF_XYSBTM's grid list (n_ebfem_bxyz_mpi.f90:1097)
  }
  std::vector<double> amp((size_t)nf * 5 * nobs), ph((size_t)nf * 5 * nobs);
  const double pi = 4.0 * std::atan(1.0), r2d = 180.0 / pi;
  for (int i = 0; i < nf; ++i) {
    if (ci->freq[i] < 0.0) continue;
    afem_solve_stats st{};
    rc = afem_solve(c, 1, &ci->freq[i], nullptr, o, &st);
    if (rc) throw Error{rc, std::string("run_ctl: solve failed: ") + c->err};
    std::vector<double> out(2L * 5 * nobs);
    rc = afem_sites(c, nobs, ci->xyzobs.data(), out.data());
    if (rc) throw Error{rc, c->err};
    if (nxy > 0) {
      // OUTFREQFILES2 (m_outresp.f90:181-217): x, y, z and (amp, phase) of bx..ey per plan-view point
      std::vector<double> o2(2L * 5 * nxy);
      reset_status(c);
      sites_device(c, nxy, xy.data(), o2.data(), true, grid_nz);
      const std::string num = fortran_e(ci->freq[i], 9, 2);
      for (int k = 0; k < ci->nsource; ++k) {
        // the reference assembles the name in a character(50) variable
        const std::string fn = (rtrim(ci->outputfolder) + rtrim(ci->xyfilehead) + num.substr(1, 8) + "_S" +
                                std::to_string((k + 1) % 10) + ".dat").substr(0, 50);
        FILE* f = std::fopen(fn.c_str(), "w");
        if (!f) throw Error{AFEM_EIO, "cannot write " + fn};
        for (int sidx = 0; sidx < nxy; ++sidx) {
          std::string row;
          for (int j = 0; j < 3; ++j) row += fortran_f(xy[3L * sidx + j], 15, 7);
          for (int comp = 0; comp < 5; ++comp) {
            double a = 0.0, p = 0.0;
            if (k == 0) {
              const double re = o2[2 * ((long)comp * nxy + sidx)], im = o2[2 * ((long)comp * nxy + sidx) + 1];
              a = std::sqrt(std::pow(re, 2.0) + std::pow(im, 2.0));
              p = std::atan2(im, re) * r2d;
            }
            row += fortran_f(a, 15, 7) + fortran_f(p, 15, 7);
          }
          std::fprintf(f, "%s\n", row.c_str());
        }
        std::fclose(f);
      }
      if (ci->seafloor()) write_ixyhout(ci, ci->freq[i], xy, o2.data(), vf_item, vf_val);
    }
    for (int comp = 0; comp < 5; ++comp)
      for (int s = 0; s < nobs; ++s) {
        const double re = out[2 * ((long)comp * nobs + s)], im = out[2 * ((long)comp * nobs + s) + 1];
        amp[((size_t)i * 5 + comp) * nobs + s] = std::sqrt(std::pow(re, 2.0) + std::pow(im, 2.0));
        ph[((size_t)i * 5 + comp) * nobs + s] = std::atan2(im, re) * r2d;
      }
  }
  for (int l = 0; l < nobs; ++l)
    for (int k = 0; k < ci->nsource; ++k) {
      // OUTOBSFILESFWD (m_outresp.f90:228-247): head, site and source names are character(50), the name (70)
      const std::string fn = (rtrim(ci->outputfolder.substr(0, 50)) + rtrim(ci->obsname[l].substr(0, 50)) + "_" +
                              rtrim(ci->sourcename[k].substr(0, 50)) + ".dat").substr(0, 70);
      FILE* f = std::fopen(fn.c_str(), "w");
      if (!f) throw Error{AFEM_EIO, "cannot write " + fn};
      for (int i = 0; i < nf; ++i) {
        std::string row = fortran_g(ci->freq[i], 15, 7);
        for (int comp = 0; comp < 5; ++comp) {
          const double a = (k == 0) ? amp[((size_t)i * 5 + comp) * nobs + l] : 0.0;
          const double p = (k == 0) ? ph[((size_t)i * 5 + comp) * nobs + l] : 0.0;
          row += fortran_g(a, 15, 7) + fortran_g(p, 15, 7);
        }
        std::fprintf(f, "%s\n", row.c_str());
      }
      std::fclose(f);
    }
  return AFEM_OK;
}

void destroy_ctl(afem_ctx* c) {
  delete c->ctl;
  c->ctl = nullptr;
}

}  // namespace afem

// Host only: UTMXY of one site (m_param.f90:609-627): km east/north of the origin.
extern "C" int afem_utm_xy(double lon, double lat, double lonorigin, double latorigin, int zone, double* xy_km) {
  if (!xy_km || zone < 1 || zone > 60) return AFEM_EINVAL;
  afem::utmxy(lon, lat, lonorigin, latorigin, zone, &xy_km[0], &xy_km[1]);
  return AFEM_OK;
}

// Host-only helpers exported for the test-suite (no device work).
extern "C" int afem_fortran_g(double x, int w, int d, char* out, int cap) {
  std::string s = afem::fortran_g(x, w, d);
  if ((int)s.size() + 1 > cap) return AFEM_EINVAL;
  std::memcpy(out, s.c_str(), s.size() + 1);
  return (int)s.size();
}
