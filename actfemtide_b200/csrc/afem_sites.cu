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
#include <algorithm>

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

// FINDELEWITHGRID (m_mesh_type.f90:204-277): the site's box, then growing
// shells of boxes (iside = 0, 1, ...; z outer, y, x inner; the boxes of the
// previous shells skipped), each box's tetrahedra in list order; the first
// tetrahedron with all barycentrics >= 0 wins (FINDELEMENT, :739-790).  One
// warp per site: boxes are visited in order, a box's tetrahedra 32 at a time,
// and the lowest lane that holds the site wins, which is the list order.
constexpr int GRID_SIDE_MAX = 64;  // shells searched before a site is declared outside the mesh

__device__ __forceinline__ int grid_box(const double* g, int n, double v) {
  // the box i (1-based) with g(i) < v <= g(i+1): the number of boundaries below v
  int lo = 0, hi = n + 1;  // count of g[0..n] that are < v
  while (lo < hi) {
    const int mid = (lo + hi) >> 1;
    if (g[mid] < v) lo = mid + 1;
    else hi = mid;
  }
  return (lo >= 1 && lo <= n) ? lo : 0;
}

__global__ void k_find_grid(const double* __restrict__ xyz, const int32_t* __restrict__ n4,
                            const double* __restrict__ xg, const double* __restrict__ yg,
                            const double* __restrict__ zg, int nx, int ny, int nz, const int32_t* __restrict__ stack,
                            const int32_t* __restrict__ ordered, const double* __restrict__ obs, int nobs,
                            int* __restrict__ best) {
  const int s = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int lane = threadIdx.x & 31;
  if (s >= nobs) return;
  const V3 x3{obs[3 * s], obs[3 * s + 1], obs[3 * s + 2]};
  const int ix = grid_box(xg, nx, x3.x), iy = grid_box(yg, ny, x3.y), iz = grid_box(zg, nz, x3.z);
  if (!ix || !iy || !iz) return;  // outside the grid: left not found
  for (int iside = 0; iside <= GRID_SIDE_MAX; ++iside) {
    for (int l = max(iz - iside, 1); l <= min(iz + iside, nz); ++l)
      for (int k = max(iy - iside, 1); k <= min(iy + iside, ny); ++k)
        for (int j = max(ix - iside, 1); j <= min(ix + iside, nx); ++j) {
          if (iz - (iside - 1) <= l && l <= iz + (iside - 1) && iy - (iside - 1) <= k && k <= iy + (iside - 1) &&
              ix - (iside - 1) <= j && j <= ix + (iside - 1))
            continue;  // searched in an inner shell
          const long b = (long)nx * ny * (l - 1) + (long)nx * (k - 1) + j;
          const int e0 = stack[b - 1], e1 = stack[b];
          for (int base = e0; base < e1; base += 32) {
            const int e = base + lane;
            bool ok = false;
            int t = 0;
            if (e < e1) {
              t = ordered[e];
              V3 el[4];
              load_tet(xyz, n4, t, el);
              double a[4];
              nodebasis(el, x3, a);
              ok = a[0] >= 0.0 && a[1] >= 0.0 && a[2] >= 0.0 && a[3] >= 0.0;
            }
            const unsigned hit = __ballot_sync(0xffffffffu, ok);
            if (hit) {
              const int w = __ffs(hit) - 1;
              const int tw = __shfl_sync(0xffffffffu, t, w);
              if (lane == 0) best[s] = tw;
              return;
            }
          }
        }
    if (iz - iside <= 1 && iz + iside >= nz && iy - iside <= 1 && iy + iside >= ny && ix - iside <= 1 &&
        ix + iside >= nx)
      return;  // every box searched
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

// SORT_INDEX (src/solver/sort_index.f90:13-56): heapsort of ra (ascending)
// carrying na along, after Numerical Recipes' SORT.  Equal keys leave in the
// order this heapsort produces, which the grid list inherits; hence the same
// hire / retire steps.
void sort_index_heap(int n, int32_t* na, double* ra) {
  if (n < 2) return;
  // 1-based views
  int32_t* NA = na - 1;
  double* RA = ra - 1;
  int l = n / 2 + 1, ir = n;
  for (;;) {
    double rra;
    int32_t iia;
    if (l > 1) {
      --l;
      rra = RA[l];
      iia = NA[l];
    } else {
      rra = RA[ir];
      iia = NA[ir];
      RA[ir] = RA[1];
      NA[ir] = NA[1];
      if (--ir == 1) {
        RA[1] = rra;
        NA[1] = iia;
        return;
      }
    }
    int i = l, j = l + l;
    while (j <= ir) {
      if (j < ir && RA[j] < RA[j + 1]) ++j;
      if (rra < RA[j]) {
        RA[i] = RA[j];
        NA[i] = NA[j];
        i = j;
        j += j;
      } else {
        j = ir + 1;
      }
    }
    RA[i] = rra;
    NA[i] = iia;
  }
}

namespace {

// gengridforlist + classifyelement2grd (m_mesh_type.f90:73-202) on the host:
// the grid over the node extent (GENXYZMINMAX) widened by 1 km, each
// tetrahedron's box by its centroid, the list sorted by box with SORT_INDEX.
void build_grid(afem_ctx* c, int nz) {
  if (!c->grid) c->grid = new GridList();
  GridList* g = c->grid;
  if (g->ready && g->nz == nz) return;
  g->nz = nz;
  g->ready = false;
  cudaStream_t s = c->stream;
  const int node = c->node, ntet = c->ntet;
  std::vector<double> xyz(3L * node);
  std::vector<int32_t> n4(4L * ntet);
  c->xyz.download(xyz.data(), xyz.size(), s);
  c->n4.download(n4.data(), n4.size(), s);
  AFEM_CUDA(cudaStreamSynchronize(s));
  double mn[3] = {xyz[0], xyz[1], xyz[2]}, mx[3] = {xyz[0], xyz[1], xyz[2]};
  for (int i = 0; i < node; ++i)
    for (int k = 0; k < 3; ++k) {
      mn[k] = std::min(mn[k], xyz[3L * i + k]);
      mx[k] = std::max(mx[k], xyz[3L * i + k]);
    }
  const int nn[3] = {g->nx, g->ny, g->nz};
  std::vector<double> grd[3];
  for (int k = 0; k < 3; ++k) {
    const double lo = mn[k] - 1.0, hi = mx[k] + 1.0;
    grd[k].resize(nn[k] + 1);
    for (int i = 0; i <= nn[k]; ++i) grd[k][i] = ((double)i * (hi - lo)) / (double)nn[k] + lo;
  }
  auto box = [&](int k, double v) {
    const std::vector<double>& gr = grd[k];
    const int pos = (int)(std::lower_bound(gr.begin(), gr.end(), v) - gr.begin());  // count of gr < v
    return (pos >= 1 && pos <= nn[k]) ? pos : 0;
  };
  std::vector<double> order(ntet);
  std::vector<int32_t> index(ntet);
  const long nxy = (long)g->nx * g->ny;
  for (int t = 0; t < ntet; ++t) {
    double cen[3] = {0.0, 0.0, 0.0};
    for (int j = 0; j < 4; ++j) {
      const double* P = &xyz[3L * (n4[4L * t + j] - 1)];
      for (int k = 0; k < 3; ++k) cen[k] = cen[k] + P[k] / 4.0;
    }
    const int ix = box(0, cen[0]), iy = box(1, cen[1]), iz = box(2, cen[2]);
    AFEM_REQUIRE(ix && iy && iz, AFEM_EINVAL, "grid list: a centroid lies outside the node extent");
    order[t] = (double)(nxy * (iz - 1) + (long)g->nx * (iy - 1) + ix);
    index[t] = t + 1;
  }
  sort_index_heap(ntet, index.data(), order.data());
  const long nbox = nxy * g->nz;
  std::vector<int32_t> stack(nbox + 1, 0);
  for (int t = 0; t < ntet; ++t) stack[(long)order[t]] += 1;
  for (long b = 1; b <= nbox; ++b) stack[b] += stack[b - 1];
  for (int t = 0; t < ntet; ++t) index[t] -= 1;
  g->xg.upload(grd[0].data(), grd[0].size(), s);
  g->yg.upload(grd[1].data(), grd[1].size(), s);
  g->zg.upload(grd[2].data(), grd[2].size(), s);
  g->stack.upload(stack.data(), stack.size(), s);
  g->ordered.upload(index.data(), index.size(), s);
  AFEM_CUDA(cudaStreamSynchronize(s));
  g->ready = true;
}

void site_coeffs_range(afem_ctx* c, int nobs, const double* xyz_obs, long t0, long t1, int32_t* item, double* val_e,
                       double* val_f, int32_t* iele, bool grid_search = false, int grid_nz = 50) {
  cudaStream_t s = c->stream;
  DBuf<double> obs;
  obs.upload(xyz_obs, 3L * nobs, s);
  DBuf<int> best;
  best.alloc(nobs);
  std::vector<int> init(nobs, 0x7fffffff);
  AFEM_CUDA(cudaMemcpyAsync(best.p, init.data(), sizeof(int) * nobs, cudaMemcpyHostToDevice, s));
  if (grid_search) {
    build_grid(c, grid_nz);
    GridList* g = c->grid;
    k_find_grid<<<(nobs * 32 + 127) / 128, 128, 0, s>>>(c->xyz.p, c->n4.p, g->xg.p, g->yg.p, g->zg.p, g->nx, g->ny,
                                                         g->nz, g->stack.p, g->ordered.p, obs.p, nobs, best.p);
    count_launch();
  } else {
    // one grid row per site; sites beyond the 65,535 rows of a grid go to further launches
    constexpr int ROWS = 65535;
    for (int s0 = 0; s0 < nobs; s0 += ROWS) {
      const int cnt = std::min(ROWS, nobs - s0);
      dim3 grid(std::max(1, std::min(2 * c->num_sms, (int)((t1 - t0 + 255) / 256))), cnt);
      k_find<<<grid, 256, 0, s>>>(c->xyz.p, c->n4.p, t0, t1, obs.p + 3L * s0, cnt, best.p + s0);
      count_launch();
    }
  }
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

void site_coeffs_grid_device(afem_ctx* c, int nobs, const double* xyz_obs, int32_t* item, double* val_e,
                             double* val_f, int32_t* iele) {
  site_coeffs_range(c, nobs, xyz_obs, 0, c->ntet, item, val_e, val_f, iele, true);
}

void grid_destroy(afem_ctx* c) {
  delete c->grid;
  c->grid = nullptr;
}

void sites_device(afem_ctx* c, int nobs, const double* xyz_obs, double* out, bool grid, int grid_nz) {
  AFEM_REQUIRE(c->nsys > 0 && c->X.p, AFEM_ESTATE, "sites: no solution");
  cudaStream_t s = c->stream;
  if (c->sol_packed) {
    AFEM_REQUIRE(!grid, AFEM_EINVAL, "sites: the grid search covers one mesh, not a packed batch");
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
  site_coeffs_range(c, nobs, xyz_obs, 0, c->ntet, item.data(), ve.data(), vf.data(), nullptr, grid, grid_nz);
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

// ---------------------------------------------------------------- sites without allocation
// A variant of the site evaluation (FINDELEMENT0 + PREPOBSCOEFF rows + CALOBSEBCOMP)
// whose device buffers live in one file-scope __device__ array, so a call
// allocates nothing: at most NOALLOC_SITES sites and NOALLOC_SYS solved systems.
// The array's address is taken once per device (cudaGetSymbolAddress) by the
// first call; make that first call before any stream capture.  All calls share
// the one array, so calls that overlap in time (two host threads, or two
// contexts on one device) race on it.
constexpr int NOALLOC_SITES = 1024;
constexpr int NOALLOC_SYS = 32;
constexpr size_t na_align(size_t b) { return (b + 255) / 256 * 256; }
constexpr size_t NA_OBS = 0;                                                        // 3*S doubles
constexpr size_t NA_BEST = na_align(NA_OBS + 3 * sizeof(double) * NOALLOC_SITES);   // S ints
constexpr size_t NA_ITEM = na_align(NA_BEST + sizeof(int) * NOALLOC_SITES);          // 6*S ints
constexpr size_t NA_VE = na_align(NA_ITEM + 6 * sizeof(int) * NOALLOC_SITES);        // 18*S doubles
constexpr size_t NA_VF = na_align(NA_VE + 18 * sizeof(double) * NOALLOC_SITES);      // 18*S doubles
constexpr size_t NA_OM = na_align(NA_VF + 18 * sizeof(double) * NOALLOC_SITES);      // SYS doubles
constexpr size_t NA_OUT = na_align(NA_OM + sizeof(double) * NOALLOC_SYS);            // 5*S*SYS double2
constexpr size_t NA_BYTES = na_align(NA_OUT + 5 * sizeof(double2) * NOALLOC_SITES * NOALLOC_SYS);  // 2.9 MB

static __device__ __align__(256) unsigned char g_sites_scratch[NA_BYTES];

namespace {

constexpr int NA_MAX_DEVICES = 64;
// device address of g_sites_scratch per device, looked up once; atomic because
// contexts on several host threads may make their first call at the same time
std::atomic<unsigned char*> g_sites_scratch_ptr[NA_MAX_DEVICES] = {};

__global__ void k_fill_int(int* __restrict__ p, int n, int v) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) p[i] = v;
}

}  // namespace

void sites_noalloc_device(afem_ctx* c, int nobs, const double* xyz_obs, double* out) {
  AFEM_REQUIRE(c->nsys > 0 && c->X.p, AFEM_ESTATE, "sites_noalloc: no solution");
  AFEM_REQUIRE(!c->sol_packed, AFEM_EINVAL, "sites_noalloc: packed batches are not supported (use afem_sites)");
  AFEM_REQUIRE(nobs <= NOALLOC_SITES, AFEM_EINVAL,
               "sites_noalloc: at most " + std::to_string(NOALLOC_SITES) + " sites per call (got " +
                   std::to_string(nobs) + ")");
  AFEM_REQUIRE(c->nsys <= NOALLOC_SYS, AFEM_EINVAL,
               "sites_noalloc: at most " + std::to_string(NOALLOC_SYS) + " solved systems (got " +
                   std::to_string(c->nsys) + ")");
  AFEM_REQUIRE(c->device >= 0 && c->device < NA_MAX_DEVICES, AFEM_EINVAL, "sites_noalloc: device id out of range");
  unsigned char* base = g_sites_scratch_ptr[c->device].load(std::memory_order_acquire);
  if (!base) {  // the device is current (every entry point sets it)
    AFEM_CUDA(cudaGetSymbolAddress(reinterpret_cast<void**>(&base), g_sites_scratch));
    g_sites_scratch_ptr[c->device].store(base, std::memory_order_release);
  }
  double* obs = reinterpret_cast<double*>(base + NA_OBS);
  int* best = reinterpret_cast<int*>(base + NA_BEST);
  int32_t* item = reinterpret_cast<int32_t*>(base + NA_ITEM);
  double* ve = reinterpret_cast<double*>(base + NA_VE);
  double* vf = reinterpret_cast<double*>(base + NA_VF);
  double* om = reinterpret_cast<double*>(base + NA_OM);
  double2* dout = reinterpret_cast<double2*>(base + NA_OUT);
  cudaStream_t s = c->stream;
  const double pi = 4.0 * std::atan(1.0);
  double hom[NOALLOC_SYS];
  for (int k = 0; k < c->nsys; ++k) hom[k] = 2.0 * pi * c->sol_freq[k];
  AFEM_CUDA(cudaMemcpyAsync(obs, xyz_obs, sizeof(double) * 3 * nobs, cudaMemcpyHostToDevice, s));
  AFEM_CUDA(cudaMemcpyAsync(om, hom, sizeof(double) * c->nsys, cudaMemcpyHostToDevice, s));
  // the search keeps the smallest holder: every site starts with none
  k_fill_int<<<(nobs + 255) / 256, 256, 0, s>>>(best, nobs, 0x7fffffff);
  count_launch();
  dim3 grid(std::max(1, std::min(2 * c->num_sms, (c->ntet + 255) / 256)), nobs);
  k_find<<<grid, 256, 0, s>>>(c->xyz.p, c->n4.p, 0, c->ntet, obs, nobs, best);
  count_launch();
  k_coeffs<<<(nobs + 63) / 64, 64, 0, s>>>(c->xyz.p, c->n4.p, c->n6line.p, obs, nobs, best, item, ve, vf, c->status.p);
  count_launch();
  check_status(c, "sites_noalloc: a site lies outside every tetrahedron");
  const long tot = (long)c->nsys * 5 * nobs;
  k_eval<<<(unsigned)((tot + 127) / 128), 128, 0, s>>>(c->X.p, c->nline, c->nsys, om, nobs, item, ve, vf, dout);
  count_launch();
  AFEM_CUDA(cudaMemcpyAsync(out, dout, sizeof(double2) * tot, cudaMemcpyDeviceToHost, s));
  AFEM_CUDA(cudaStreamSynchronize(s));
}

}  // namespace afem
