// Internal declarations shared by the translation units of libactfem_gpu.so.
#pragma once

#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <chrono>
#include <cstdint>
#include <cstdio>
#include <string>
#include <thread>
#include <vector>

#include "../../include/afem.h"

namespace afem {

// ---------------------------------------------------------------- errors
struct Error {
  int code;
  std::string msg;
};

#define AFEM_CUDA(call)                                                                       \
  do {                                                                                        \
    cudaError_t e_ = (call);                                                                  \
    if (e_ != cudaSuccess)                                                                    \
      throw ::afem::Error{AFEM_ECUDA, std::string(#call) + ": " + cudaGetErrorString(e_)};   \
  } while (0)

#define AFEM_REQUIRE(cond, code, msg)                 \
  do {                                                \
    if (!(cond)) throw ::afem::Error{(code), (msg)};  \
  } while (0)

// ---------------------------------------------------------------- device buffer
template <class T>
struct DBuf {
  T* p = nullptr;
  size_t n = 0;
  DBuf() = default;
  DBuf(const DBuf&) = delete;
  DBuf& operator=(const DBuf&) = delete;
  ~DBuf() { release(); }
  void release() {
    if (p) cudaFree(p);
    p = nullptr;
    n = 0;
  }
  void alloc(size_t count) {
    if (count == n && p) return;
    release();
    if (count == 0) return;
    AFEM_CUDA(cudaMalloc(&p, count * sizeof(T)));
    n = count;
  }
  void upload(const T* h, size_t count, cudaStream_t s) {
    alloc(count);
    if (count) AFEM_CUDA(cudaMemcpyAsync(p, h, count * sizeof(T), cudaMemcpyHostToDevice, s));
  }
  void download(T* h, size_t count, cudaStream_t s) const {
    if (count) AFEM_CUDA(cudaMemcpyAsync(h, p, count * sizeof(T), cudaMemcpyDeviceToHost, s));
  }
  void zero(cudaStream_t s) {
    if (n) AFEM_CUDA(cudaMemsetAsync(p, 0, n * sizeof(T), s));
  }
  size_t bytes() const { return n * sizeof(T); }
};

// Error / status words written by kernels (never trap).
enum DevErr : int {
  DEV_OK = 0,
  DEV_VOLUME = 1,      // non-positive volume
  DEV_ROWLEN = 2,      // row longer than the kernel's limit
  DEV_TIMEOUT = 3,     // bounded wait expired
  DEV_NOTFOUND = 4,    // id missing (edge search / pattern slot)
  DEV_DEGREE = 5,      // adjacency longer than the kernel's limit
  DEV_NOSIGMA = 6,     // tetrahedron tag selects no conductivity
  DEV_PIVOT = 7        // zero or non-finite pivot in a direct factorisation
};

struct DevStatus {
  int code;   // first DevErr raised
  int where;  // kernel-specific index (0-based row / tet) of the first error
  int aux;
  int pad;
};

// ---------------------------------------------------------------- limits
constexpr int ROW_MAX = 64;      // maximum nonzeros of one matrix row (diagonal included)
constexpr int EDGE_DEG_MAX = 64; // maximum tetrahedra sharing one edge
constexpr int NODE_DEG_MAX = 100;// maximum tetrahedra sharing one node (MKLINE_V2 maxnele)
constexpr int NODE_NBR_MAX = 128;// maximum edges leaving one node towards larger ids

struct SourceSet {
  int nodes = 0;
  DBuf<double> F;   // 3*nodes
  DBuf<double2> v;  // 3*nodes
};

struct CtlInfo;  // drop-in driver state (afem_io.cpp)

// Gridded element list of gengridforlist / classifyelement2grd
// (m_mesh_type.f90:56-202): nx*ny*nz boxes over the node extent +-1 km,
// tetrahedra sorted by the box of their centroid (SORT_INDEX heap order).
struct GridList {
  int nx = 300, ny = 300, nz = 50;
  DBuf<double> xg, yg, zg;       // box boundaries, nx+1 / ny+1 / nz+1 values
  DBuf<int32_t> stack;           // 0..nx*ny*nz: tetrahedra with box <= b
  DBuf<int32_t> ordered;         // ntet, 0-based tetrahedra in list order
  bool ready = false;
};

// Per-kernel device time accumulated with CUDA events while profiling is on.
struct ProfEntry {
  std::string name;
  double ms = 0.0;
  long launches = 0;
};
struct Profile {
  bool on = false;
  std::vector<ProfEntry> e;
  void add(const char* name, double ms, long n = 1) {
    for (auto& x : e)
      if (x.name == name) { x.ms += ms; x.launches += n; return; }
    e.push_back(ProfEntry{name, ms, n});
  }
};

// Kernel launches of this library in this process (measurement).  Launches
// enqueued while a stream is captured into a CUDA graph are not counted
// there; each launch of the graph counts its kernel nodes instead.
extern std::atomic<long> g_launches;
extern thread_local int g_capturing;
// Every launch site calls this right after the launch, so a launch that the
// runtime refused (bad configuration, too many resources) is reported at once
// instead of leaving its outputs unwritten.
inline void count_launch(long n = 1) {
  const cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) throw Error{AFEM_ECUDA, std::string("kernel launch: ") + cudaGetErrorString(e)};
  if (!g_capturing) g_launches.fetch_add(n, std::memory_order_relaxed);
}

// Host wall time of a set-up phase, added to the profile table while profiling is on
// (the stream is drained on both sides then, so the phase's device work is included).
struct HostTimer {
  afem_ctx* c;
  const char* name;
  std::chrono::steady_clock::time_point t0;
  bool on;
  HostTimer(afem_ctx* ctx, const char* nm);
  ~HostTimer();
};

struct SolverWork;   // afem_solver.cu
struct MpnnState;    // afem_mpnn.cu
struct HybridState;  // afem_hybrid.cu
struct MtState;      // afem_mt.cu

}  // namespace afem

struct afem_ctx {
  int device = 0;
  cudaStream_t stream = nullptr;
  std::string err;
  int num_sms = 0;

  // mesh
  int node = 0, ntet = 0, nline = 0;
  afem::DBuf<double> xyz;      // 3*node
  afem::DBuf<int32_t> n4;      // 4*ntet, 1-based
  afem::DBuf<int32_t> tag;     // ntet
  std::vector<int32_t> h_tag;  // host copy of the tags (conductivity selection)
  afem::DBuf<int32_t> line;    // 2*nline, 1-based
  afem::DBuf<int32_t> n6line;  // 6*ntet, signed 1-based

  // conductivity
  afem::DBuf<double> sigma;  // ntet
  bool sigma_set = false;

  // sources
  std::vector<afem::SourceSet*> src;

  // Dirichlet bounds
  double zmin = 0, zmax = 0, xout = 0, yout = 0;
  bool bounds_set = false;

  // pattern (full CSR, sorted columns, 0-based)
  long nnz = 0;
  afem::DBuf<int32_t> rowptr;   // nline+1
  afem::DBuf<int32_t> col;      // nnz
  afem::DBuf<int32_t> diagpos;  // nline
  afem::DBuf<int32_t> etp;      // nline+1, edge -> (tet, local edge) adjacency
  afem::DBuf<int32_t> etl;      // 6*ntet, value = tet*8 + local edge, ascending per edge
  bool pattern_ready = false;
  // triangular-sweep schedules: rows in dependency-level order (a topological order)
  afem::DBuf<int32_t> perm_f;   // forward sweep: lower-triangle levels ascending, ties by row
  afem::DBuf<int32_t> perm_b;   // backward sweep: upper-triangle levels ascending, ties by row descending
  int levels_f = 0, levels_b = 0;
  // multicolour sweeps: greedy colouring, rows sorted by colour
  afem::DBuf<uint8_t> color;    // nline
  afem::DBuf<int32_t> perm_mc;  // nline
  afem::DBuf<int32_t> color_ptr;// ncolors + 1
  int ncolors = 0;
  // the same rows in colour order, split: entries of earlier colours (mc_l*) and of
  // later colours (mc_u*); *src = index of the entry in the CSR, *km the values
  afem::DBuf<int32_t> mc_lptr, mc_lcol, mc_lsrc, mc_uptr, mc_ucol, mc_usrc;
  afem::DBuf<int32_t> mc_dsrc;  // CSR index of the diagonal of the row at each colour position
  afem::DBuf<double2> mc_lkm, mc_ukm, mc_dkm;
  long mc_vals_gen = -1;        // assembly generation of mc_lkm / mc_ukm / mc_dkm
  bool schedule_ready = false;  // colouring and colour-ordered split rows
  bool levels_ready = false;    // perm_f / perm_b (natural-order sweeps only)
  // tiled SpMV (16 systems): per tile of 32 rows its distinct columns and the entries'
  // positions among them (k_spt_build); spt_fb flags tiles summed from global memory
  afem::DBuf<int32_t> spt_ptr, spt_uniq;
  afem::DBuf<uint16_t> spt_lidx;
  afem::DBuf<uint8_t> spt_fb;
  int spt_ntiles = 0;
  bool spt_ready = false;

  // values: A(omega) = K + i*omega*M, stored interleaved (K_k, M_k)
  afem::DBuf<double2> km;       // nnz
  afem::DBuf<uint8_t> bc;       // nline Dirichlet flags
  afem::DBuf<double2> rhs;      // nline * nsrc
  int rhs_nsrc = 0;
  bool assembled = false;
  long assemble_gen = 0;        // increases with every new set of matrix values

  // packed batch of independent meshes (segments): mesh k owns nodes
  // [seg_node_ptr[k], seg_node_ptr[k+1]), tetrahedra [seg_tet_ptr[k], ..) and
  // rows [seg_row_ptr[k], ..) of the union; system k of a solve is mesh k
  int nseg = 0;
  std::vector<int32_t> seg_node_ptr, seg_tet_ptr, seg_row_ptr;
  afem::DBuf<uint8_t> seg_of_row;  // nline: segment of each row

  // solutions of the last solve: x[k*nline + i]
  afem::DBuf<double2> X;
  std::vector<double> sol_freq;
  int nsys = 0;
  bool sol_packed = false;  // X holds a packed batch: one system per row, x[i]

  afem::SolverWork* work = nullptr;
  afem::MpnnState* mpnn = nullptr;
  afem::HybridState* hyb = nullptr;
  afem::GridList* grid = nullptr;   // element locator of the plan-view sites
  int last_learned_its = 0;  // iterations the last solve ran with the learned preconditioner
  afem::CtlInfo* ctl = nullptr;
  afem::MtState* mt = nullptr;   // boundary surfaces of the MT forward (built per mesh)

  unsigned wait_limit = 0;   // polls of the sync-free sweeps' bounded wait (0: the built-in limit)
  int spmv_rpw = 0;          // SpMV rows per warp pinned by the caller (0: chosen by the tuner)

  afem::DBuf<afem::DevStatus> status;  // one status word
  afem::Profile prof;
};

namespace afem {

// afem_mesh.cu
void build_lines_device(afem_ctx* c);     // MKLINE_V2 + MKN6 on the device
void build_pattern_device(afem_ctx* c);   // adjacency + full CSR pattern
void build_schedule(afem_ctx* c, bool levels);  // colouring + split rows; the level schedules when asked
void exclusive_scan(const int32_t* in, int32_t* out, int n, cudaStream_t s, long* total_host);
int compute_coloring(int n, const int32_t* rp, const int32_t* cl, uint8_t* color, int32_t* perm, int32_t* cptr,
                     int max_colors);  // greedy distance-1 colouring, rows sorted by colour
// Colour-ordered split rows of a CSR pattern on the device (rp, cl, dp, color, perm: device):
// position p holds row perm[p], its entries of earlier colours (lptr/lcol/lsrc) and of later
// colours (uptr/ucol/usrc) in the row's CSR order with their CSR indices; dsrc (optional)
// the CSR index of the row's diagonal.
void split_rows_device(afem_ctx* c, const int32_t* rp, const int32_t* cl, const int32_t* dp, const uint8_t* color,
                       const int32_t* perm, int n, DBuf<int32_t>& lptr, DBuf<int32_t>& lcol, DBuf<int32_t>& lsrc,
                       DBuf<int32_t>& uptr, DBuf<int32_t>& ucol, DBuf<int32_t>& usrc, DBuf<int32_t>* dsrc);

// Host loop over [0, n) in contiguous chunks on up to 32 threads: f(begin, end).
// Each index's work must be independent (and not throw); small n runs inline.
template <class F>
void host_parallel_for(long n, F f) {
  const unsigned hw = std::thread::hardware_concurrency();
  const long nt = std::min<long>(std::max(1u, hw), 32);
  if (n < 200000 || nt == 1) {
    f(0L, n);
    return;
  }
  const long chunk = (n + nt - 1) / nt;
  std::vector<std::thread> th;
  for (long t = 0; t < nt; ++t) {
    const long a = t * chunk, b = std::min(n, a + chunk);
    if (a >= b) break;
    th.emplace_back(f, a, b);
  }
  for (auto& x : th) x.join();
}

// afem_assemble.cu
void assemble_device(afem_ctx* c);        // K, M, rhs, bc (GENMAT + COPY_UL + GENBCCSEM + SET_BC)

// packed batches
inline void clear_segments(afem_ctx* c) {
  c->nseg = 0;
  c->seg_node_ptr.clear();
  c->seg_tet_ptr.clear();
  c->seg_row_ptr.clear();
  c->seg_of_row.release();
}

// afem_solver.cu
struct SolveExtra {
  const double* x0 = nullptr;   // initial guess, [row][system] interleaved complex (host)
  bool recursive_only = false;  // stop on the recursive residual, no refinement (COCG13_single)
  const double* rhs = nullptr;  // caller right-hand sides, [row][system] interleaved complex (host)
};
int solve_device(afem_ctx* c, int nsys, const double* freq, const int* src, const afem_solve_opts* o,
                 afem_solve_stats* st, const SolveExtra* ex = nullptr);
void load_split_system(afem_ctx* c, int n, const int32_t* INU, const int32_t* IAU, const int32_t* INL,
                       const int32_t* IAL, const double* D, const double* AU, const double* AL, const double* b);
void destroy_work(afem_ctx* c);
void invalidate_work(afem_ctx* c);          // new matrix values
void invalidate_pattern_work(afem_ctx* c);  // new pattern
void reset_spmv_tuning(afem_ctx* c);        // the SpMV rows per warp is chosen again at the next solve
void get_residual(afem_ctx* c, int k, double* r);  // b - A x of system k after the last solve

// afem_mpnn.cu (learned preconditioner)
void mpnn_destroy(afem_ctx* c);
int mpnn_nparam();
void mpnn_set_params(afem_ctx* c, const float* p, int np);
void mpnn_get_params(afem_ctx* c, float* p);
bool mpnn_ready(afem_ctx* c);
int mpnn_base(afem_ctx* c);                 // 0: Jacobi base, 1: gradient-corrected SSOR base
void mpnn_set_base(afem_ctx* c, int base);
// z = H(r) for one system at angular frequency omega: the gradient-corrected multicolour
// SSOR of the assembled system (the learned preconditioner's base), device vectors of n values
void precond_apply_device(afem_ctx* c, double omega, const double2* r, double2* z);
void mpnn_prepare(afem_ctx* c, int ns, const double* d_omega);
template <class V>
void mpnn_run(afem_ctx* c, int ns, const double* d_rms, const V* r, V* z, const int* skip);
void mpnn_forward_host(afem_ctx* c, int ns, const double* freq, const double* r_host, double* z_host);
double mpnn_loss_grad_host(afem_ctx* c, double freq, int nsamp, const double* r_host, float* grad_host);
double mpnn_train_host(afem_ctx* c, double freq, int nsamp, const double* r_host, int steps, float lr,
                       double* hist);

// afem_adjoint.cu
void jacobian_device(afem_ctx* c, double freq, const double* x_host, int nadj, double* J_host);

// afem_assemble.cu: the system with non-zero Dirichlet values g_k (SET_BC_3DJoint): K and M
// without the boundary rows cleared, rhs column k = -A(omega_k) g_k on interior rows and g_k on
// Dirichlet rows, then the Dirichlet rows and columns cleared.  bc, g: device; g[k*nline + row].
void assemble_dirichlet_device(afem_ctx* c, const uint8_t* bc, int nsys, const double* omega_host,
                               const double2* g);

// afem_mt.cu (3-D MT forward)
void mt_destroy(afem_ctx* c);
int mt_forward_device(afem_ctx* c, const afem_mt_cond* cond, int nfreq, const double* freq, int nobs,
                      const double* xyz_obs, const afem_solve_opts* o, double* be, double* z, double* rho,
                      double* pha, afem_solve_stats* st);
void mt_boundary_device(afem_ctx* c, const afem_mt_cond* cond, double freq, double* av, uint8_t* bc);
void mt_face_device(afem_ctx* c, const afem_mt_cond* cond, int j, double freq, int* n, long* nnz, int32_t* line3d,
                    int32_t* rowptr, int32_t* col, double* val, double* rhs, double* bs);

// afem_sites.cu
void site_coeffs_device(afem_ctx* c, int nobs, const double* xyz_obs, int32_t* item, double* val_e, double* val_f,
                        int32_t* iele);
// grid: FINDELEWITHGRID search over a 300 x 300 x grid_nz grid list (PREPOBSCOEFF_XY: 50, _XYSBTM: 300)
void sites_device(afem_ctx* c, int nobs, const double* xyz_obs, double* out, bool grid = false, int grid_nz = 50);
void site_coeffs_grid_device(afem_ctx* c, int nobs, const double* xyz_obs, int32_t* item, double* val_e,
                             double* val_f, int32_t* iele);
void sort_index_heap(int n, int32_t* na, double* ra);  // SORT_INDEX (sort_index.f90:13-56)
void sites_noalloc_device(afem_ctx* c, int nobs, const double* xyz_obs, double* out);  // afem_sites_noalloc
void grid_destroy(afem_ctx* c);

// status helpers
void reset_status(afem_ctx* c);
void check_status(afem_ctx* c, const char* what);

// afem_io.cpp
int load_ctl(afem_ctx* c, const char* path);
int ctl_info(afem_ctx* c, int* nfreq, double* freq, int* nobs, double* xyz);
int run_ctl(afem_ctx* c, const afem_solve_opts* o);
void destroy_ctl(afem_ctx* c);

}  // namespace afem

// ---------------------------------------------------------------- device helpers
#ifdef __CUDACC__
namespace afem {

__device__ __forceinline__ double2 cadd(double2 a, double2 b) { return make_double2(a.x + b.x, a.y + b.y); }
__device__ __forceinline__ double2 csub(double2 a, double2 b) { return make_double2(a.x - b.x, a.y - b.y); }
__device__ __forceinline__ double2 cmul(double2 a, double2 b) {
  return make_double2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
__device__ __forceinline__ double2 cscale(double s, double2 a) { return make_double2(s * a.x, s * a.y); }
// Smith's algorithm (R. L. Smith, CACM 5(8), 1962) for a / b.
__device__ __forceinline__ double2 cdiv(double2 a, double2 b) {
  if (fabs(b.x) >= fabs(b.y)) {
    double r = b.y / b.x, den = b.x + b.y * r;
    return make_double2((a.x + a.y * r) / den, (a.y - a.x * r) / den);
  } else {
    double r = b.x / b.y, den = b.x * r + b.y;
    return make_double2((a.x * r + a.y) / den, (a.y * r - a.x) / den);
  }
}

__device__ __forceinline__ void raise_status(DevStatus* st, int code, int where) {
  if (atomicCAS(&st->code, 0, code) == 0) st->where = where;
}

__device__ __forceinline__ unsigned ld_acquire(const unsigned* p) {
  unsigned v;
  asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
  return v;
}
// Polling load: coherent at GPU scope (served by L2), no fence.  The data a
// flag publishes is read after the poll loop exits (control dependency) with
// ld.global.cg, and the writer fences before it stores the flag.
__device__ __forceinline__ unsigned ld_relaxed(const unsigned* p) {
  unsigned v;
  asm volatile("ld.relaxed.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
  return v;
}
__device__ __forceinline__ void st_release(unsigned* p, unsigned v) {
  asm volatile("st.release.gpu.global.u32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}

}  // namespace afem
#endif
