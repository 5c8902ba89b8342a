// C ABI entry points (include/afem.h): context, inputs, assembly, solve, sites.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <exception>

#include "afem_hybrid.h"
#include "afem_internal.h"

namespace afem {

void reset_status(afem_ctx* c) { AFEM_CUDA(cudaMemsetAsync(c->status.p, 0, sizeof(DevStatus), c->stream)); }

void check_status(afem_ctx* c, const char* what) {
  DevStatus h{};
  AFEM_CUDA(cudaMemcpyAsync(&h, c->status.p, sizeof(DevStatus), cudaMemcpyDeviceToHost, c->stream));
  AFEM_CUDA(cudaStreamSynchronize(c->stream));
  AFEM_CUDA(cudaGetLastError());
  if (h.code == DEV_OK) return;
  reset_status(c);
  int code = AFEM_EINVAL;
  const char* kind = "error";
  switch (h.code) {
    case DEV_VOLUME: code = AFEM_EVOLUME; kind = "non-positive volume"; break;
    case DEV_ROWLEN: code = AFEM_EPATTERN; kind = "row longer than 64 nonzeros"; break;
    case DEV_TIMEOUT: code = AFEM_ETIMEOUT; kind = "device wait exceeded its bound"; break;
    case DEV_NOTFOUND: code = AFEM_EPATTERN; kind = "id not found"; break;
    case DEV_DEGREE: code = AFEM_EPATTERN; kind = "adjacency longer than the kernel limit"; break;
    case DEV_NOSIGMA: code = AFEM_EINVAL; kind = "no conductivity for tag"; break;
    case DEV_PIVOT: code = AFEM_EBREAKDOWN; kind = "zero or non-finite pivot"; break;
    default: break;
  }
  char buf[256];
  snprintf(buf, sizeof(buf), "%s: %s (index %d, 0-based)", what, kind, h.where);
  throw Error{code, buf};
}

HostTimer::HostTimer(afem_ctx* ctx, const char* nm) : c(ctx), name(nm), on(ctx->prof.on) {
  if (on) {
    cudaStreamSynchronize(c->stream);
    t0 = std::chrono::steady_clock::now();
  }
}
HostTimer::~HostTimer() {
  if (!on) return;
  cudaStreamSynchronize(c->stream);
  const double ms = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
  c->prof.add(name, ms);
}

std::atomic<long> g_launches{0};
thread_local int g_capturing = 0;

}  // namespace afem

using afem::Error;

namespace afem {

// A complex system given in the reference's split storage (type global_matrix,
// m_iccg_var_takuto.f90:9-18) becomes the device CSR with (K, M) = (Re, Im)
// and omega = 1.  Rows keep their column order sorted ascending.
void load_split_system(afem_ctx* c, int n, const int32_t* INU, const int32_t* IAU, const int32_t* INL,
                       const int32_t* IAL, const double* D, const double* AU, const double* AL, const double* b) {
  AFEM_REQUIRE(n > 0 && INU && IAU && INL && IAL && D && AU && AL && b, AFEM_EINVAL, "split system: null array");
  AFEM_REQUIRE(INU[0] == 0 && INL[0] == 0, AFEM_EINVAL, "split system: INU(0) and INL(0) must be 0");
  clear_segments(c);
  std::vector<int32_t> rp(n + 1), cl, dp(n);
  std::vector<double2> km;
  const long tot = (long)INU[n] + INL[n] + n;
  cl.reserve(tot);
  km.reserve(tot);
  rp[0] = 0;
  std::vector<std::pair<int, double2>> row;
  for (int i = 0; i < n; ++i) {
    row.clear();
    for (int k = INL[i]; k < INL[i + 1]; ++k) {
      const int j = IAL[k] - 1;
      AFEM_REQUIRE(j >= 0 && j < i, AFEM_EINVAL, "split system: IAL column not below the diagonal");
      row.push_back({j, make_double2(AL[2L * k], AL[2L * k + 1])});
    }
    row.push_back({i, make_double2(D[2L * i], D[2L * i + 1])});
    for (int k = INU[i]; k < INU[i + 1]; ++k) {
      const int j = IAU[k] - 1;
      AFEM_REQUIRE(j > i && j < n, AFEM_EINVAL, "split system: IAU column not above the diagonal");
      row.push_back({j, make_double2(AU[2L * k], AU[2L * k + 1])});
    }
    std::stable_sort(row.begin(), row.end(), [](const auto& a, const auto& b) { return a.first < b.first; });
    AFEM_REQUIRE((long)row.size() <= ROW_MAX, AFEM_EPATTERN, "split system: row longer than 64 entries");
    for (auto& e : row) {
      if (e.first == i) dp[i] = (int32_t)cl.size();
      cl.push_back(e.first);
      km.push_back(e.second);
    }
    rp[i + 1] = (int32_t)cl.size();
  }
  cudaStream_t s = c->stream;
  c->nline = n;
  c->ntet = 0;
  c->node = 0;
  c->nnz = (long)cl.size();
  c->rowptr.upload(rp.data(), n + 1, s);
  c->col.upload(cl.data(), cl.size(), s);
  c->diagpos.upload(dp.data(), n, s);
  c->km.upload(km.data(), km.size(), s);
  c->rhs.upload(reinterpret_cast<const double2*>(b), n, s);
  c->rhs_nsrc = 1;
  c->bc.alloc(n);
  c->bc.zero(s);
  AFEM_CUDA(cudaStreamSynchronize(s));
  c->pattern_ready = true;
  c->schedule_ready = false;
  c->levels_ready = false;
  c->assembled = true;
  c->assemble_gen += 1;
  afem::hybrid_invalidate(c);
  invalidate_pattern_work(c);
}

}  // namespace afem

namespace {

template <class F>
int guarded(afem_ctx* c, F&& f) {
  if (!c) return AFEM_EINVAL;
  try {
    cudaSetDevice(c->device);
    int rc = f();
    return rc;
  } catch (const Error& e) {
    c->err = e.msg;
    return e.code;
  } catch (const std::exception& e) {
    c->err = e.what();
    return AFEM_EINVAL;
  }
}

void invalidate_assembly(afem_ctx* c) { c->assembled = false; }

}  // namespace

extern "C" {

afem_ctx* afem_create(int device) {
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || device < 0 || device >= ndev) return nullptr;
  if (cudaSetDevice(device) != cudaSuccess) return nullptr;
  afem_ctx* c = new afem_ctx();
  c->device = device;
  try {
    AFEM_CUDA(cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking));
    AFEM_CUDA(cudaDeviceGetAttribute(&c->num_sms, cudaDevAttrMultiProcessorCount, device));
    c->status.alloc(1);
    c->status.zero(c->stream);
    AFEM_CUDA(cudaStreamSynchronize(c->stream));
  } catch (const Error&) {
    delete c;
    return nullptr;
  }
  return c;
}

void afem_destroy(afem_ctx* c) {
  if (!c) return;
  cudaSetDevice(c->device);
  afem::destroy_work(c);
  afem::destroy_ctl(c);
  afem::mpnn_destroy(c);
  afem::hybrid_destroy(c);
  afem::grid_destroy(c);
  afem::mt_destroy(c);
  for (auto* s : c->src) delete s;
  c->src.clear();
    if (c->stream) {
    cudaStreamSynchronize(c->stream);
    cudaStreamDestroy(c->stream);
  }
  delete c;
}

const char* afem_last_error(const afem_ctx* c) { return c ? c->err.c_str() : "null context"; }

long afem_launch_count(void) { return afem::g_launches.load(); }

int afem_hybrid_matrix(afem_ctx* c, int* node, long* nnz, int32_t* rowptr, int32_t* col, double* km) {
  return guarded(c, [&]() {
    afem::hybrid_export(c, node, nnz, rowptr, col, km);
    return (int)AFEM_OK;
  });
}

void* afem_stream(afem_ctx* c) { return c ? (void*)c->stream : nullptr; }

int afem_set_mesh(afem_ctx* c, int node, const double* xyz, int ntet, const int32_t* n4, const int32_t* tag,
                  int nline, const int32_t* line, const int32_t* n6line) {
  return guarded(c, [&]() {
    AFEM_REQUIRE(node > 0 && ntet > 0 && xyz && n4 && tag, AFEM_EINVAL, "set_mesh: empty mesh or null array");
    AFEM_REQUIRE(nline >= 0, AFEM_EINVAL, "set_mesh: negative nline");
    afem::HostTimer ht(c, "host_set_mesh");
    for (long i = 0; i < 4L * ntet; ++i)
      AFEM_REQUIRE(n4[i] >= 1 && n4[i] <= node, AFEM_EINVAL, "set_mesh: node id outside 1..node in n4");
    if (nline > 0) {
      AFEM_REQUIRE(line && n6line, AFEM_EINVAL, "set_mesh: nline > 0 needs line and n6line");
      for (long i = 0; i < 2L * nline; ++i)
        AFEM_REQUIRE(line[i] >= 1 && line[i] <= node, AFEM_EINVAL, "set_mesh: node id outside 1..node in line");
      for (long i = 0; i < 6L * ntet; ++i)
        AFEM_REQUIRE(n6line[i] != 0 && std::abs(n6line[i]) <= nline, AFEM_EINVAL,
                     "set_mesh: n6line entry outside +-1..nline");
    }
    cudaStream_t s = c->stream;
    c->node = node;
    c->ntet = ntet;
    c->xyz.upload(xyz, 3L * node, s);
    c->n4.upload(n4, 4L * ntet, s);
    c->tag.upload(tag, ntet, s);
    c->h_tag.assign(tag, tag + ntet);
    c->pattern_ready = false;
    c->assembled = false;
    c->sigma_set = false;
    afem::clear_segments(c);
    afem::hybrid_invalidate(c);
    afem::invalidate_pattern_work(c);
    if (c->grid) c->grid->ready = false;
    afem::mt_destroy(c);
    afem::reset_status(c);
    if (nline > 0) {
      c->nline = nline;
      c->line.upload(line, 2L * nline, s);
      c->n6line.upload(n6line, 6L * ntet, s);
    } else {
      afem::build_lines_device(c);
    }
    AFEM_CUDA(cudaStreamSynchronize(s));
    afem::build_pattern_device(c);
    return (int)AFEM_OK;
  });
}

int afem_mesh_info(afem_ctx* c, int* node, int* ntet, int* nline) {
  return guarded(c, [&]() {
    if (node) *node = c->node;
    if (ntet) *ntet = c->ntet;
    if (nline) *nline = c->nline;
    return (int)AFEM_OK;
  });
}

int afem_solution_count(afem_ctx* c, int* nsys) {
  return guarded(c, [&]() {
    AFEM_REQUIRE(nsys, AFEM_EINVAL, "solution_count: null output");
    *nsys = c->nsys;
    return (int)AFEM_OK;
  });
}

int afem_get_lines(afem_ctx* c, int* nline, int32_t* line, int32_t* n6line) {
  return guarded(c, [&]() {
    AFEM_REQUIRE(c->nline > 0, AFEM_ESTATE, "get_lines: no mesh");
    if (nline) *nline = c->nline;
    if (line) c->line.download(line, 2L * c->nline, c->stream);
    if (n6line) c->n6line.download(n6line, 6L * c->ntet, c->stream);
    AFEM_CUDA(cudaStreamSynchronize(c->stream));
    return (int)AFEM_OK;
  });
}

int afem_set_segments(afem_ctx* c, int nseg, const int32_t* node_ptr) {
  return guarded(c, [&]() {
    AFEM_REQUIRE(c->nline > 0 && c->ntet > 0, AFEM_ESTATE, "set_segments: set the mesh first");
    AFEM_REQUIRE(nseg >= 0 && nseg <= 32, AFEM_EINVAL, "set_segments: nseg must be 0..32");
    afem::clear_segments(c);
    if (nseg == 0) return (int)AFEM_OK;
    AFEM_REQUIRE(node_ptr, AFEM_EINVAL, "set_segments: null node_ptr");
    AFEM_REQUIRE(node_ptr[0] == 0 && node_ptr[nseg] == c->node, AFEM_EINVAL,
                 "set_segments: node_ptr must run from 0 to node");
    for (int k = 0; k < nseg; ++k)
      AFEM_REQUIRE(node_ptr[k + 1] > node_ptr[k], AFEM_EINVAL, "set_segments: empty or decreasing node range");
    cudaStream_t s = c->stream;
    // segment of a 1-based node id
    auto seg_of = [&](int32_t id) {
      return (int)(std::upper_bound(node_ptr, node_ptr + nseg + 1, id - 1) - node_ptr) - 1;
    };
    // tetrahedra: all four nodes in one mesh, meshes in order
    std::vector<int32_t> n4(4L * c->ntet);
    c->n4.download(n4.data(), n4.size(), s);
    std::vector<int32_t> line(2L * c->nline);
    c->line.download(line.data(), line.size(), s);
    AFEM_CUDA(cudaStreamSynchronize(s));
    std::vector<int32_t> tet_ptr(nseg + 1, 0), row_ptr(nseg + 1, 0);
    int prev = 0;
    for (long t = 0; t < c->ntet; ++t) {
      const int k = seg_of(n4[4 * t]);
      for (int j = 1; j < 4; ++j)
        AFEM_REQUIRE(seg_of(n4[4 * t + j]) == k, AFEM_EINVAL, "set_segments: a tetrahedron joins two meshes");
      AFEM_REQUIRE(k >= prev, AFEM_EINVAL, "set_segments: tetrahedra are not grouped mesh by mesh");
      prev = k;
      tet_ptr[k + 1] += 1;
    }
    std::vector<uint8_t> seg(c->nline);
    prev = 0;
    for (long e = 0; e < c->nline; ++e) {
      const int k = seg_of(line[2 * e]);
      AFEM_REQUIRE(seg_of(line[2 * e + 1]) == k, AFEM_EINVAL, "set_segments: an edge joins two meshes");
      AFEM_REQUIRE(k >= prev, AFEM_EINVAL, "set_segments: edges are not numbered mesh by mesh");
      prev = k;
      row_ptr[k + 1] += 1;
      seg[e] = (uint8_t)k;
    }
    for (int k = 0; k < nseg; ++k) {
      AFEM_REQUIRE(tet_ptr[k + 1] > 0 && row_ptr[k + 1] > 0, AFEM_EINVAL, "set_segments: a mesh has no tetrahedra");
      tet_ptr[k + 1] += tet_ptr[k];
      row_ptr[k + 1] += row_ptr[k];
    }
    c->seg_node_ptr.assign(node_ptr, node_ptr + nseg + 1);
    c->seg_tet_ptr = tet_ptr;
    c->seg_row_ptr = row_ptr;
    c->seg_of_row.upload(seg.data(), seg.size(), s);
    AFEM_CUDA(cudaStreamSynchronize(s));
    c->nseg = nseg;
    afem::invalidate_pattern_work(c);
    c->nsys = 0;
    return (int)AFEM_OK;
  });
}

int afem_segment_info(afem_ctx* c, int* nseg, int32_t* row_ptr, int32_t* tet_ptr) {
  return guarded(c, [&]() {
    if (nseg) *nseg = c->nseg;
    if (c->nseg > 0) {
      if (row_ptr) std::copy(c->seg_row_ptr.begin(), c->seg_row_ptr.end(), row_ptr);
      if (tet_ptr) std::copy(c->seg_tet_ptr.begin(), c->seg_tet_ptr.end(), tet_ptr);
    }
    return (int)AFEM_OK;
  });
}

int afem_set_cond(afem_ctx* c, double sigma_air, double sigma_ocean, int condflag, int nvolume,
                  const double* sigma_land, int nphys2, const double* sigma_file) {
  return guarded(c, [&]() {
    AFEM_REQUIRE(c->ntet > 0, AFEM_ESTATE, "set_cond: set the mesh first");
    AFEM_REQUIRE(condflag == 0 || condflag == 1, AFEM_EINVAL, "set_cond: condflag must be 0 or 1");
    const std::vector<int32_t>& tag = c->h_tag;
    const long ntet = c->ntet;
    long count3 = 0;
    for (long t = 0; t < ntet; ++t) count3 += tag[t] >= 3;
    if (condflag == 1) {
      AFEM_REQUIRE(sigma_file && nphys2 == count3, AFEM_EINVAL,
                   "set_cond: nphys2 differs from the number of tetrahedra with tag >= 3 (SETNPHYS1INDEX2COND)");
    }
    const long nphys1 = ntet - count3;
    std::vector<double> sig(ntet);
    for (long t = 0; t < ntet; ++t) {
      const int j = tag[t];
      if (j == 1) sig[t] = sigma_air;
      else if (j == 2) sig[t] = sigma_ocean;
      else if (j >= 3) {
        if (condflag == 0) {
          AFEM_REQUIRE(sigma_land && j - 1 <= nvolume, AFEM_EINVAL, "set_cond: tag beyond nvolume + 1");
          sig[t] = sigma_land[j - 2];
        } else {
          AFEM_REQUIRE(t >= nphys1, AFEM_EINVAL, "set_cond: land tetrahedra must come last (sigma(iele - nphys1))");
          sig[t] = sigma_file[t - nphys1];
        }
      } else {
        throw Error{AFEM_EINVAL, "set_cond: tetrahedron tag < 1 selects no conductivity"};
      }
    }
    c->sigma.upload(sig.data(), ntet, c->stream);
    AFEM_CUDA(cudaStreamSynchronize(c->stream));
    c->sigma_set = true;
    invalidate_assembly(c);
    return (int)AFEM_OK;
  });
}

int afem_set_sigma(afem_ctx* c, const double* sigma_tet) {
  return guarded(c, [&]() {
    AFEM_REQUIRE(c->ntet > 0 && sigma_tet, AFEM_EINVAL, "set_sigma: set the mesh first / null array");
    c->sigma.upload(sigma_tet, c->ntet, c->stream);
    AFEM_CUDA(cudaStreamSynchronize(c->stream));
    c->sigma_set = true;
    invalidate_assembly(c);
    return (int)AFEM_OK;
  });
}

int afem_set_source(afem_ctx* c, int isrc, int nodes, const double* F, const double* v) {
  return guarded(c, [&]() {
    AFEM_REQUIRE(c->node > 0, AFEM_ESTATE, "set_source: set the mesh first");
    AFEM_REQUIRE(isrc >= 0 && isrc < 16, AFEM_EINVAL, "set_source: isrc must be 0..15");
    AFEM_REQUIRE(nodes >= 0 && nodes <= c->node, AFEM_EINVAL, "set_source: nodes must be 0..node");
    AFEM_REQUIRE(nodes == 0 || (F && v), AFEM_EINVAL, "set_source: null F or v");
    if ((int)c->src.size() <= isrc) c->src.resize(isrc + 1, nullptr);
    if (!c->src[isrc]) c->src[isrc] = new afem::SourceSet();
    afem::SourceSet* S = c->src[isrc];
    S->nodes = nodes;
    S->F.upload(F, 3L * nodes, c->stream);
    S->v.upload(reinterpret_cast<const double2*>(v), 3L * nodes, c->stream);
    AFEM_CUDA(cudaStreamSynchronize(c->stream));
    invalidate_assembly(c);
    return (int)AFEM_OK;
  });
}

int afem_set_bounds(afem_ctx* c, double zmin, double zmax, double xout, double yout) {
  return guarded(c, [&]() {
    c->zmin = zmin; c->zmax = zmax; c->xout = xout; c->yout = yout;
    c->bounds_set = true;
    invalidate_assembly(c);
    return (int)AFEM_OK;
  });
}

int afem_assemble(afem_ctx* c) {
  return guarded(c, [&]() {
    AFEM_REQUIRE(c->pattern_ready, AFEM_ESTATE, "assemble: set the mesh first");
    afem::reset_status(c);
    afem::assemble_device(c);
    afem::invalidate_work(c);
    return (int)AFEM_OK;
  });
}

int afem_export_system(afem_ctx* c, double freq, int isrc, int* n_out, long* iau_tot, int32_t* INU, int32_t* IAU,
                       int32_t* INL, int32_t* IAL, double* D, double* AU, double* AL, double* b, uint8_t* bc) {
  return guarded(c, [&]() {
    AFEM_REQUIRE(c->pattern_ready, AFEM_ESTATE, "export: no pattern");
    const int n = c->nline;
    cudaStream_t s = c->stream;
    std::vector<int32_t> rp(n + 1), cl(c->nnz), dp(n);
    c->rowptr.download(rp.data(), n + 1, s);
    c->col.download(cl.data(), c->nnz, s);
    c->diagpos.download(dp.data(), n, s);
    std::vector<double2> km;
    std::vector<double2> rh;
    if (c->assembled) {
      km.resize(c->nnz);
      c->km.download(km.data(), c->nnz, s);
      AFEM_REQUIRE(isrc >= 0 && isrc < c->rhs_nsrc, AFEM_EINVAL, "export: isrc out of range");
      rh.resize(n);
      AFEM_CUDA(cudaMemcpyAsync(rh.data(), c->rhs.p + (long)isrc * n, sizeof(double2) * n, cudaMemcpyDeviceToHost, s));
      if (bc) c->bc.download(bc, n, s);
    } else {
      AFEM_REQUIRE(!(D || AU || AL || b || bc), AFEM_ESTATE, "export: values requested before assembly");
    }
    AFEM_CUDA(cudaStreamSynchronize(s));
    const double omega = 2.0 * (4.0 * std::atan(1.0)) * freq;
    long tot = 0;
    for (int i = 0; i < n; ++i) tot += rp[i + 1] - dp[i] - 1;
    if (n_out) *n_out = n;
    if (iau_tot) *iau_tot = tot;
    long pu = 0, pl = 0;
    if (INU) INU[0] = 0;
    if (INL) INL[0] = 0;
    for (int i = 0; i < n; ++i) {
      for (int k = rp[i]; k < rp[i + 1]; ++k) {
        const int j = cl[k];
        double re = 0, im = 0;
        if (!km.empty()) { re = km[k].x; im = omega * km[k].y; }
        if (j < i) {
          if (IAL) IAL[pl] = j + 1;
          if (AL) { AL[2 * pl] = re; AL[2 * pl + 1] = im; }
          ++pl;
        } else if (j > i) {
          if (IAU) IAU[pu] = j + 1;
          if (AU) { AU[2 * pu] = re; AU[2 * pu + 1] = im; }
          ++pu;
        } else if (D) {
          D[2 * i] = re; D[2 * i + 1] = im;
        }
      }
      if (INU) INU[i + 1] = (int32_t)pu;
      if (INL) INL[i + 1] = (int32_t)pl;
      if (b && !rh.empty()) { b[2 * i] = rh[i].x; b[2 * i + 1] = rh[i].y; }
    }
    return (int)AFEM_OK;
  });
}

namespace {
void check_opts(const afem_solve_opts* o) {
  AFEM_REQUIRE(o->precond >= 0 && o->precond <= 6, AFEM_EINVAL, "solve: unknown preconditioner");
  AFEM_REQUIRE(o->precision >= 0 && o->precision <= 2, AFEM_EINVAL, "solve: unknown precision");
  AFEM_REQUIRE(o->precision != AFEM_FP32_PRECOND || o->precond == AFEM_PRECOND_SSOR_MC ||
                   o->precond == AFEM_PRECOND_HYBRID,
               AFEM_EINVAL, "solve: the FP32 preconditioner applies to SSOR_MC and HYBRID");
}
}  // namespace

int afem_set_wait_limit(afem_ctx* c, unsigned polls) {
  return guarded(c, [&]() {
    c->wait_limit = polls;
    return (int)AFEM_OK;
  });
}

int afem_set_spmv_rows_per_warp(afem_ctx* c, int rpw) {
  return guarded(c, [&]() {
    AFEM_REQUIRE(rpw == 0 || rpw == 1 || rpw == 2 || rpw == 4 || rpw == 8 || rpw == 16, AFEM_EINVAL,
                 "set_spmv_rows_per_warp: 0 (tuned), 1, 2, 4, 8 or 16 (tiles staged in shared memory)");
    c->spmv_rpw = rpw;
    afem::reset_spmv_tuning(c);
    return (int)AFEM_OK;
  });
}

int afem_solve(afem_ctx* c, int nsys, const double* freq, const int* src, const afem_solve_opts* opts,
               afem_solve_stats* stats) {
  return guarded(c, [&]() {
    AFEM_REQUIRE(freq && opts, AFEM_EINVAL, "solve: null freq or opts");
    check_opts(opts);
    afem::reset_status(c);
    return afem::solve_device(c, nsys, freq, src, opts, stats);
  });
}

int afem_get_solution(afem_ctx* c, int k, double* x) {
  return guarded(c, [&]() {
    AFEM_REQUIRE(k >= 0 && k < c->nsys && x, AFEM_EINVAL, "get_solution: no such system");
    if (c->sol_packed) {  // packed batch: the rows of mesh k
      const int r0 = c->seg_row_ptr[k], r1 = c->seg_row_ptr[k + 1];
      AFEM_CUDA(cudaMemcpyAsync(x, c->X.p + r0, sizeof(double2) * (r1 - r0), cudaMemcpyDeviceToHost, c->stream));
      AFEM_CUDA(cudaStreamSynchronize(c->stream));
      return (int)AFEM_OK;
    }
    // stored [row][system]
    std::vector<double2> all((size_t)c->nline * c->nsys);
    c->X.download(all.data(), all.size(), c->stream);
    AFEM_CUDA(cudaStreamSynchronize(c->stream));
    for (int i = 0; i < c->nline; ++i) {
      x[2 * i] = all[(size_t)i * c->nsys + k].x;
      x[2 * i + 1] = all[(size_t)i * c->nsys + k].y;
    }
    return (int)AFEM_OK;
  });
}

int afem_solve_rhs(afem_ctx* c, int nsys, const double* freq, const double* rhs, const afem_solve_opts* opts,
                   afem_solve_stats* stats) {
  return guarded(c, [&]() {
    AFEM_REQUIRE(freq && opts && rhs, AFEM_EINVAL, "solve_rhs: null argument");
    check_opts(opts);
    afem::reset_status(c);
    afem::SolveExtra ex;
    ex.rhs = rhs;
    return afem::solve_device(c, nsys, freq, nullptr, opts, stats, &ex);
  });
}

int afem_jacobian(afem_ctx* c, double freq, const double* x, int nadj, double* J) {
  return guarded(c, [&]() {
    AFEM_REQUIRE(x && J && nadj > 0, AFEM_EINVAL, "jacobian: null argument");
    afem::reset_status(c);
    afem::jacobian_device(c, freq, x, nadj, J);
    return (int)AFEM_OK;
  });
}

int afem_get_residual(afem_ctx* c, int k, double* r) {
  return guarded(c, [&]() {
    AFEM_REQUIRE(r, AFEM_EINVAL, "get_residual: null output");
    afem::get_residual(c, k, r);
    return (int)AFEM_OK;
  });
}

int afem_sites(afem_ctx* c, int nobs, const double* xyz_obs, double* out) {
  return guarded(c, [&]() {
    AFEM_REQUIRE(nobs > 0 && xyz_obs && out, AFEM_EINVAL, "sites: empty or null");
    afem::reset_status(c);
    afem::sites_device(c, nobs, xyz_obs, out);
    return (int)AFEM_OK;
  });
}

int afem_site_coeffs(afem_ctx* c, int nobs, const double* xyz_obs, int32_t* item, double* val_e, double* val_f,
                     int32_t* iele) {
  return guarded(c, [&]() {
    AFEM_REQUIRE(nobs > 0 && xyz_obs, AFEM_EINVAL, "site_coeffs: empty or null");
    AFEM_REQUIRE(c->ntet > 0 && c->nline > 0, AFEM_ESTATE, "site_coeffs: no mesh");
    afem::reset_status(c);
    afem::site_coeffs_device(c, nobs, xyz_obs, item, val_e, val_f, iele);
    return (int)AFEM_OK;
  });
}

int afem_mpnn_set_base(afem_ctx* c, int base) {
  return guarded(c, [&]() {
    afem::mpnn_set_base(c, base);
    return (int)AFEM_OK;
  });
}

int afem_precond_apply(afem_ctx* c, double freq, const double* r, double* z) {
  return guarded(c, [&]() {
    AFEM_REQUIRE(r && z && freq > 0, AFEM_EINVAL, "precond_apply: null vector or bad frequency");
    AFEM_REQUIRE(c->assembled && c->nline > 0, AFEM_ESTATE, "precond_apply: assemble first");
    afem::reset_status(c);
    afem::DBuf<double2> dr, dz;
    dr.upload(reinterpret_cast<const double2*>(r), c->nline, c->stream);
    dz.alloc(c->nline);
    afem::precond_apply_device(c, 2.0 * (4.0 * std::atan(1.0)) * freq, dr.p, dz.p);
    dz.download(reinterpret_cast<double2*>(z), c->nline, c->stream);
    AFEM_CUDA(cudaStreamSynchronize(c->stream));
    return (int)AFEM_OK;
  });
}

int afem_sites_noalloc(afem_ctx* c, int nobs, const double* xyz_obs, double* out) {
  return guarded(c, [&]() {
    AFEM_REQUIRE(nobs > 0 && xyz_obs && out, AFEM_EINVAL, "sites_noalloc: empty or null");
    afem::reset_status(c);
    afem::sites_noalloc_device(c, nobs, xyz_obs, out);
    return (int)AFEM_OK;
  });
}

int afem_sites_grid(afem_ctx* c, int nobs, const double* xyz_obs, double* out) {
  return guarded(c, [&]() {
    AFEM_REQUIRE(nobs > 0 && xyz_obs && out, AFEM_EINVAL, "sites_grid: empty or null");
    AFEM_REQUIRE(c->ntet > 0 && c->nline > 0, AFEM_ESTATE, "sites_grid: no mesh");
    afem::reset_status(c);
    afem::sites_device(c, nobs, xyz_obs, out, true);
    return (int)AFEM_OK;
  });
}

int afem_site_coeffs_grid(afem_ctx* c, int nobs, const double* xyz_obs, int32_t* item, double* val_e, double* val_f,
                          int32_t* iele) {
  return guarded(c, [&]() {
    AFEM_REQUIRE(nobs > 0 && xyz_obs, AFEM_EINVAL, "site_coeffs_grid: empty or null");
    AFEM_REQUIRE(c->ntet > 0 && c->nline > 0, AFEM_ESTATE, "site_coeffs_grid: no mesh");
    afem::reset_status(c);
    afem::site_coeffs_grid_device(c, nobs, xyz_obs, item, val_e, val_f, iele);
    return (int)AFEM_OK;
  });
}

int afem_sort_index(int n, int32_t* na, double* ra) {
  if (n < 0 || (n > 0 && (!na || !ra))) return AFEM_EINVAL;
  afem::sort_index_heap(n, na, ra);
  return AFEM_OK;
}

int afem_xy_points(double xmin, double xmax, double ymin, double ymax, int nx, int ny, double z, double* xyz) {
  if (nx <= 0 || ny <= 0 || !xyz) return AFEM_EINVAL;
  // PREPOBSCOEFF_XY (n_ebfem_bxyz_mpi.f90:769-784): cell centres, ii = (j-1)*ny + i;
  // dx = (xmax - xmin)/float(nx) divides by a default-real count
  const double dx = (xmax - xmin) / (double)(float)nx, dy = (ymax - ymin) / (double)(float)ny;
  for (int j = 1; j <= nx; ++j)
    for (int i = 1; i <= ny; ++i) {
      const long ii = (long)(j - 1) * ny + i - 1;
      xyz[3 * ii] = (j - 1) * dx + xmin + dx / 2.0;
      xyz[3 * ii + 1] = (i - 1) * dy + ymin + dy / 2.0;
      xyz[3 * ii + 2] = z;
    }
  return AFEM_OK;
}

int afem_set_system(afem_ctx* c, int n, const int32_t* INU, const int32_t* IAU, const int32_t* INL,
                    const int32_t* IAL, const double* D, const double* AU, const double* AL, const double* b) {
  return guarded(c, [&]() {
    afem::load_split_system(c, n, INU, IAU, INL, IAL, D, AU, AL, b);
    return (int)AFEM_OK;
  });
}

int afem_cocg13_single(afem_ctx* c, int NP, int NPL, int NPU, double* D, double* AL, const int32_t* INL,
                       const int32_t* IAL, double* AU, const int32_t* INU, const int32_t* IAU, double* B, double* X,
                       const char* PRECOND, double SIGMA_DIAG, double SIGMA, double* RESID, int* ITER, int* ERROR,
                       int NSET) {
  return guarded(c, [&]() {
    AFEM_REQUIRE(RESID && ITER && ERROR && PRECOND && B && X, AFEM_EINVAL, "cocg13_single: null argument");
    (void)NPL;
    (void)NPU;
    *ERROR = 0;
    if (NSET == 0) {  // COCG13_single.f90:49-52
      *ERROR = 101;
      return (int)AFEM_OK;
    }
    int prec = AFEM_PRECOND_NONE;
    if (!std::strncmp(PRECOND, "IC", 2) || !std::strncmp(PRECOND, "ILU", 3)) prec = AFEM_PRECOND_IC;
    else if (!std::strncmp(PRECOND, "SSOR", 4)) prec = AFEM_PRECOND_SSOR;
    else if (!std::strncmp(PRECOND, "DIAG", 4)) prec = AFEM_PRECOND_DIAG;
    AFEM_REQUIRE(!(prec == AFEM_PRECOND_IC && SIGMA != 0.0), AFEM_EINVAL,
                 "cocg13_single: IC with SIGMA != 0 is not supported on the device");
    std::vector<double> scale(NP, 1.0);
    if (NSET == 2) {  // COCG13_single.f90:77-97, the caller's arrays are scaled in place
      for (int i = 0; i < NP; ++i) scale[i] = 1.0 / std::sqrt(std::hypot(D[2 * i], D[2 * i + 1]));
      for (int j = 0; j < NP; ++j) {
        const double a = std::hypot(D[2 * j], D[2 * j + 1]);
        const double dr = D[2 * j], di = D[2 * j + 1], den = dr * dr + di * di;
        D[2 * j] = a * dr / den;
        D[2 * j + 1] = -a * di / den;
        for (int k = INU[j]; k < INU[j + 1]; ++k) {
          const double f = scale[IAU[k] - 1] * scale[j];
          AU[2L * k] *= f;
          AU[2L * k + 1] *= f;
        }
        for (int k = INL[j]; k < INL[j + 1]; ++k) {
          const double f = scale[IAL[k] - 1] * scale[j];
          AL[2L * k] *= f;
          AL[2L * k + 1] *= f;
        }
      }
    }
    double bn = 0.0;
    for (int i = 0; i < NP; ++i) {
      B[2 * i] *= scale[i];
      B[2 * i + 1] *= scale[i];
      bn += B[2 * i] * B[2 * i] + B[2 * i + 1] * B[2 * i + 1];
    }
    const int maxit = *ITER;
    if (bn == 0.0) {  // COCG13_single.f90:171-177
      for (int i = 0; i < 2 * NP; ++i) X[i] = 0.0;
      *RESID = 0.0;
      *ITER = 0;
      for (int i = 0; i < NP; ++i) { B[2 * i] /= scale[i]; B[2 * i + 1] /= scale[i]; }
      return (int)AFEM_OK;
    }
    afem::load_split_system(c, NP, INU, IAU, INL, IAL, D, AU, AL, B);
    afem_solve_opts o{};
    o.precond = prec;
    o.precision = AFEM_FP64;
    o.tol = *RESID;
    o.maxit = maxit;
    o.sigma_diag = SIGMA_DIAG;
    o.use_graph = 1;
    afem::SolveExtra ex;
    ex.x0 = X;
    ex.recursive_only = true;
    afem_solve_stats st{};
    const double freq = 1.0 / (8.0 * std::atan(1.0));  // omega = 1: the values are A itself
    afem::reset_status(c);
    const int rc = afem::solve_device(c, 1, &freq, nullptr, &o, &st, &ex);
    if (rc != AFEM_OK && rc != AFEM_EMAXITER) return rc;
    std::vector<double2> x(NP);
    c->X.download(x.data(), NP, c->stream);
    AFEM_CUDA(cudaStreamSynchronize(c->stream));
    for (int i = 0; i < NP; ++i) {
      X[2 * i] = x[i].x * scale[i];
      X[2 * i + 1] = x[i].y * scale[i];
      B[2 * i] /= scale[i];
      B[2 * i + 1] /= scale[i];
    }
    *RESID = st.resid_recursive;
    if (rc == AFEM_EMAXITER) {
      *ERROR = -100;
      *ITER = maxit + 1;  // value of the Fortran DO variable after a full loop
    } else {
      *ITER = st.iterations;
    }
    return (int)AFEM_OK;
  });
}

int afem_mpnn_nparam(void) { return afem::mpnn_nparam(); }

int afem_mpnn_set_params(afem_ctx* c, const float* p, int np) {
  return guarded(c, [&]() {
    afem::mpnn_set_params(c, p, np);
    return (int)AFEM_OK;
  });
}

int afem_mpnn_get_params(afem_ctx* c, float* p) {
  return guarded(c, [&]() {
    afem::mpnn_get_params(c, p);
    return (int)AFEM_OK;
  });
}

int afem_mpnn_forward(afem_ctx* c, int nsys, const double* freq, const double* r, double* z) {
  return guarded(c, [&]() {
    AFEM_REQUIRE(c->assembled, AFEM_ESTATE, "mpnn_forward: system not assembled");
    AFEM_REQUIRE(nsys >= 1 && nsys <= 16 && freq && r && z, AFEM_EINVAL, "mpnn_forward: bad arguments");
    afem::mpnn_forward_host(c, nsys, freq, r, z);
    return (int)AFEM_OK;
  });
}

int afem_mpnn_loss_grad(afem_ctx* c, double freq, int nsamp, const double* r, double* loss, float* grad) {
  return guarded(c, [&]() {
    AFEM_REQUIRE(c->assembled, AFEM_ESTATE, "mpnn_loss_grad: system not assembled");
    AFEM_REQUIRE(nsamp >= 1 && r, AFEM_EINVAL, "mpnn_loss_grad: bad arguments");
    const double L = afem::mpnn_loss_grad_host(c, freq, nsamp, r, grad);
    if (loss) *loss = L;
    return (int)AFEM_OK;
  });
}

int afem_mpnn_train(afem_ctx* c, double freq, int nsamp, const double* r, int steps, float lr, double* hist) {
  return guarded(c, [&]() {
    AFEM_REQUIRE(c->assembled, AFEM_ESTATE, "mpnn_train: system not assembled");
    AFEM_REQUIRE(nsamp >= 1 && r && steps >= 1, AFEM_EINVAL, "mpnn_train: bad arguments");
    afem::mpnn_train_host(c, freq, nsamp, r, steps, lr, hist);
    return (int)AFEM_OK;
  });
}

int afem_set_profiling(afem_ctx* c, int enable) {
  return guarded(c, [&]() {
    c->prof.on = enable != 0;
    c->prof.e.clear();
    return (int)AFEM_OK;
  });
}

int afem_profile_count(afem_ctx* c) { return c ? (int)c->prof.e.size() : 0; }

int afem_profile_entry(afem_ctx* c, int i, char* name, int cap, double* ms, long* launches) {
  return guarded(c, [&]() {
    AFEM_REQUIRE(i >= 0 && i < (int)c->prof.e.size(), AFEM_EINVAL, "profile_entry: index out of range");
    const afem::ProfEntry& e = c->prof.e[i];
    if (name && cap > 0) {
      std::strncpy(name, e.name.c_str(), cap - 1);
      name[cap - 1] = 0;
    }
    if (ms) *ms = e.ms;
    if (launches) *launches = e.launches;
    return (int)AFEM_OK;
  });
}

int afem_load_ctl(afem_ctx* c, const char* path) {
  return guarded(c, [&]() { return afem::load_ctl(c, path); });
}

int afem_ctl_info(afem_ctx* c, int* nfreq, double* freq, int* nobs, double* xyz) {
  return guarded(c, [&]() { return afem::ctl_info(c, nfreq, freq, nobs, xyz); });
}

int afem_run_ctl(afem_ctx* c, const afem_solve_opts* o) {
  return guarded(c, [&]() { return afem::run_ctl(c, o); });
}

}  // extern "C"

// ---- 3-D MT forward
int afem_mt_forward(afem_ctx* c, const afem_mt_cond* cond, int nfreq, const double* freq, int nobs,
                    const double* xyz_obs, const afem_solve_opts* opts, double* be, double* z, double* rho,
                    double* pha, afem_solve_stats* stats) {
  return guarded(c, [&]() {
    AFEM_REQUIRE(opts, AFEM_EINVAL, "mt_forward: null options");
    check_opts(opts);
    afem::reset_status(c);
    return afem::mt_forward_device(c, cond, nfreq, freq, nobs, xyz_obs, opts, be, z, rho, pha, stats);
  });
}

int afem_mt_boundary(afem_ctx* c, const afem_mt_cond* cond, double freq, double* av, uint8_t* bc) {
  return guarded(c, [&]() {
    afem::reset_status(c);
    afem::mt_boundary_device(c, cond, freq, av, bc);
    return (int)AFEM_OK;
  });
}

int afem_mt_face(afem_ctx* c, const afem_mt_cond* cond, int j, double freq, int* n, long* nnz, int32_t* line3d,
                 int32_t* rowptr, int32_t* col, double* val, double* rhs, double* bs) {
  return guarded(c, [&]() {
    afem::reset_status(c);
    afem::mt_face_device(c, cond, j, freq, n, nnz, line3d, rowptr, col, val, rhs, bs);
    return (int)AFEM_OK;
  });
}
