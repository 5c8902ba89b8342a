// Batched preconditioned COCG (COCG13_single) on the device.
//
// Reference: src/solver/COCG13_single.f90:9-340.  Per iteration the reference
// does: z = M^-1 r (forward + backward sweep with DD), rho = r^T z, p = z +
// (rho/rho1) p, q = A p, alpha = rho / p^T q, x += alpha p, r -= alpha q,
// RESID = ||r|| / ||b||.  Here one iteration is four streaming kernels and
// three single-block scalar kernels:
//   k_fwd   : x += alpha p, r -= alpha q (previous iteration), ||r||^2, forward sweep
//   k_scal_r: RESID, convergence / iteration cap / non-finite checks
//   k_bwd   : backward sweep, rho = r^T z (unconjugated)
//   k_scal_rho: beta = rho / rho1
//   k_pupd  : p = z + beta p
//   k_spmv  : q = A p, p^T q
//   k_scal_pq: alpha = rho / p^T q, rho1 = rho, epoch++
// Every kernel returns at once after the batch has finished, so a captured
// chunk of iterations can run past convergence harmlessly.
//
// Storage: A(omega_s) = K + i omega_s M for system s; K and M are read once
// per entry for all NS systems of a batch.  Vectors are laid out [row][system]
// so the NS values of one row are contiguous.  A warp handles one row: lane =
// g * NS + s works on system s and on entries g, g + G, ... (G = 32 / NS).
//
// The triangular sweeps are sync-free: each row waits (bounded) on a per-row
// flag of every row it depends on.  Rows are statically interleaved over the
// warps of a cooperative (co-resident) grid, each warp in increasing
// dependency order, so the lowest unfinished row can always proceed.
#include <cooperative_groups.h>

#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstring>
#include <type_traits>

#include "afem_hybrid.h"
#include "afem_internal.h"

namespace afem {

template <class T>
struct Cx;
template <>
struct Cx<double> {
  using V = double2;
  __host__ __device__ static V make(double a, double b) { return make_double2(a, b); }
};
template <>
struct Cx<float> {
  using V = float2;
  __host__ __device__ static V make(float a, float b) { return make_float2(a, b); }
};

constexpr int MAX_SYS = 32;  // systems of one solve: NS, or the meshes of a packed batch
constexpr unsigned SPIN_LIMIT = 1u << 21;  // x ~1 us back-off: a wait gives up after ~2 s

// per-system scalars (always FP64)
struct SysScal {
  double2 rho, rho1, alpha, beta, pq;
  double rr, bnrm2, resid, omega;
  int active;     // 1 while iterating
  int status;     // afem_status of this system
  int iter;       // iterations done
  int xpend;      // multicolour path: this iteration's x += alpha p waits for the p update
};

struct Ctrl {
  unsigned epoch;  // flag generation, increases by one per sweep pair, never reset
  int done;        // all systems finished
  int iter;        // iterations of the current inner solve
  int maxit;
  double tol;
  unsigned spin_limit;  // polls of a bounded wait before DEV_TIMEOUT (0: SPIN_LIMIT)
};

struct SolverWork {
  int n = 0, ns = 0, prec_bits = 64;
  int nsys = 0;     // systems of the current solve: ns, or the meshes of a packed batch
  bool seg = false; // packed batch: vectors hold one system per row
  int nblocks = 0;  // persistent grid size (blocks of 256 threads)
  DBuf<double2> x, b;               // FP64 solution and right-hand side [row][sys]
  DBuf<double2> xacc;               // FP64 solution accumulated over the refinement steps (kept between solves)
  DBuf<double2> r64;                // FP64 true residual
  DBuf<double2> r, z, p, q, dd;     // FP64 inner vectors
  DBuf<float2> rf, zf, pf, qf, ddf; // FP32 inner vectors
  DBuf<float2> kmf;                 // FP32 copy of (K, M)
  DBuf<float2> mc_lkmf, mc_ukmf;    // FP32 copies of the colour-ordered split rows
  DBuf<double2> rprev;              // flexible COCG: previous residual (FP64 inner)
  DBuf<float2> rprevf;              // flexible COCG: previous residual (FP32 inner)
  DBuf<double> rms;                 // per-system rms(r) for the learned preconditioner
  DBuf<double2> ht, hy, hdd;        // gradient-space correction: nodal rhs, solution, 1/diag (FP64 inner)
  DBuf<float2> htf, hyf, hddf;      // the same for the FP32 inner solve
  int nmc_blocks = 0;               // co-resident grid of the nodal multicolour sweeps
  int rpw64 = 0, rpw32 = 0;         // SpMV rows per warp chosen by tune_spmv (0 = not tuned; 8: 4 systems per lane)
  int spmv_grid[2][5] = {};         // one-wave grid of each SpMV variant (FP64 / FP32), 0 = not known yet
  int mc_blocks = 0;                // co-resident grid of the forward multicolour sweep
  int mcb_blocks = 0;               // and of the backward one (fewer registers: more blocks)
  double sd = 1.0;                  // SSOR diagonal scale of the current solve (DD = 1 / (sd D))
  bool no_window = false;           // COCG13_single semantics: no stagnation window, run to the cap
  bool kmf_valid = false;            // kmf matches the assembly
  bool mcf_valid = false;            // mc_lkmf / mc_ukmf match the assembly
  DBuf<unsigned> flag_f, flag_b;
  DBuf<double> part;                // partial sums [block][sys][4]
  DBuf<double> part2;               // nodal share of rho (hybrid), same layout
  DBuf<SysScal> sc;
  DBuf<Ctrl> ctrl;
  Ctrl* h_ctrl = nullptr;           // pinned mirror
  SysScal* h_sc = nullptr;          // pinned mirror
  unsigned epoch_host = 0;
  ~SolverWork() {
    if (h_ctrl) cudaFreeHost(h_ctrl);
    if (h_sc) cudaFreeHost(h_sc);
  }
};

namespace {

__device__ __forceinline__ bool wait_flag(const unsigned* f, unsigned epoch, DevStatus* st, int row,
                                          unsigned limit) {
  if (ld_relaxed(f) >= epoch) return true;
  // exponential back-off keeps the poll traffic from crowding L2
  unsigned spins = 0, ns = 32;
  for (;;) {
    __nanosleep(ns);
    if (ns < 1024) ns <<= 1;
    if (ld_relaxed(f) >= epoch) return true;
    ++spins;
    if ((spins & 63) == 0 && *(volatile int*)&st->code == DEV_TIMEOUT) return false;
    if (spins > limit) {
      raise_status(st, DEV_TIMEOUT, row);
      return false;
    }
  }
}

template <class V>
__device__ __forceinline__ V ldcg(const V* p);
template <>
__device__ __forceinline__ double2 ldcg<double2>(const double2* p) { return __ldcg(p); }
template <>
__device__ __forceinline__ float2 ldcg<float2>(const float2* p) { return __ldcg(p); }

template <class T>
__device__ __forceinline__ T shfl_xor(T v, int m) { return __shfl_xor_sync(0xffffffffu, v, m); }

// Reduce complex (t1, t2) over the G lane groups of a warp (lanes differing in g).
template <class T, int NS>
__device__ __forceinline__ void group_reduce(T& a, T& b, T& c, T& d) {
#pragma unroll
  for (int m = NS; m < 32; m <<= 1) {
    a += shfl_xor(a, m);
    b += shfl_xor(b, m);
    c += shfl_xor(c, m);
    d += shfl_xor(d, m);
  }
}

// The values a gather reads may sit in L1 when every row's NS values fill whole
// 128-byte lines: a line then holds one row only, and a row is read only after
// this kernel wrote it (earlier colours of a sweep) or never written in it (the
// SpMV's p), so no SM can hold a stale copy.  Narrower rows share lines with
// rows still to be written and are read at L2 (ld.cg).
template <class V, int NS>
struct GatherL1 {
  static constexpr bool ok = (NS * sizeof(V)) % 128 == 0;
};
template <class V, int NS>
__device__ __forceinline__ V gather_ld(const V* p) {
  if constexpr (GatherL1<V, NS>::ok) return *p;
  else return ldcg(p);
}

// Sum over a row's entries k0, k0+G, ... < k1 of A_k * v_col(k) for system s, split
// as t1 = sum K*v and t2 = sum M*v.  Four entries at a time: their columns,
// then their values and gathers, so four independent gathers are in flight
// per lane; the additions keep the entries' order (the sums do not change).
template <class T, int NS, int G>
__device__ __forceinline__ void row_gather(const int32_t* __restrict__ cols, const typename Cx<T>::V* __restrict__ vals,
                                           const typename Cx<T>::V* vec, int k0, int k1, int s, T& t1x, T& t1y,
                                           T& t2x, T& t2y) {
  using V = typename Cx<T>::V;
  int k = k0;
  // four loads in flight only where one lane owns the row: with G > 1 lanes per row each
  // holds few entries and the unrolled registers cost occupancy
  if constexpr (G == 1)
    for (; k + 3 < k1; k += 4) {
      const int j0 = __ldg(cols + k), j1 = __ldg(cols + k + 1), j2 = __ldg(cols + k + 2), j3 = __ldg(cols + k + 3);
      const V a0 = vals[k], a1 = vals[k + 1], a2 = vals[k + 2], a3 = vals[k + 3];
      const V v0 = gather_ld<V, NS>(vec + (long)j0 * NS + s), v1 = gather_ld<V, NS>(vec + (long)j1 * NS + s);
      const V v2 = gather_ld<V, NS>(vec + (long)j2 * NS + s), v3 = gather_ld<V, NS>(vec + (long)j3 * NS + s);
      t1x += a0.x * v0.x; t1y += a0.x * v0.y; t2x += a0.y * v0.x; t2y += a0.y * v0.y;
      t1x += a1.x * v1.x; t1y += a1.x * v1.y; t2x += a1.y * v1.x; t2y += a1.y * v1.y;
      t1x += a2.x * v2.x; t1y += a2.x * v2.y; t2x += a2.y * v2.x; t2y += a2.y * v2.y;
      t1x += a3.x * v3.x; t1y += a3.x * v3.y; t2x += a3.y * v3.x; t2y += a3.y * v3.y;
    }
  for (; k < k1; k += G) {
    const int j = __ldg(cols + k);
    const V a = vals[k];
    const V v = gather_ld<V, NS>(vec + (long)j * NS + s);
    t1x += a.x * v.x; t1y += a.x * v.y;
    t2x += a.y * v.x; t2y += a.y * v.y;
  }
}

// Row schedule of the persistent kernels: [p0, p1) is cut into chunks of CH
// rounds of the block's warps (CH * warps * RPW rows), dealt to the blocks
// round-robin.  All SMs then work inside a band of gridDim * chunk rows that
// moves through the range (the neighbours they gather stay in L2), and inside a
// chunk the warps of one SM gather from overlapping neighbourhoods (L1 serves
// the repeats).  CH = 1 is a plain grid-wide stride.
#ifndef AFEM_SWEEP_CHUNK
#define AFEM_SWEEP_CHUNK 1  // rounds per chunk in the multicolour sweeps
#endif
#ifndef AFEM_SPMV_CHUNK
#define AFEM_SPMV_CHUNK 4  // rounds per chunk in the SpMV
#endif
// The first row of this warp's first round in for_rows<RPW, CH>(p0, ..).
template <int RPW, int CH>
__device__ __forceinline__ int first_round(int p0) {
  return p0 + (int)blockIdx.x * CH * (int)(blockDim.x >> 5) * RPW + (int)(threadIdx.x >> 5) * RPW;
}

// Calls body(pos0, end, next) for every warp round of this block: the round's rows
// are pos0 + sub (sub < RPW), live below `end`; `next` is the first row of the
// warp's following round (-1 after the last), so that a body can load the next
// rows' indices while it gathers for the current ones.
template <int RPW, int CH, class F>
__device__ __forceinline__ void for_rows(int p0, int p1, F body) {
  const int wib = threadIdx.x >> 5, nwb = blockDim.x >> 5;
  const int chunk = CH * nwb * RPW, cstride = (int)gridDim.x * chunk;
  int cb = p0 + (int)blockIdx.x * chunk, pos0 = cb + wib * RPW;
  if (cb < p1 && pos0 >= min(cb + chunk, p1)) cb = p1;  // no round of this warp in the (last, partial) chunk
  while (cb < p1) {
    const int ce = min(cb + chunk, p1);
    int ncb = cb, npos = pos0 + nwb * RPW;
    if (npos >= ce) {
      ncb = cb + cstride;
      npos = ncb + wib * RPW;
      if (ncb < p1 && npos >= min(ncb + chunk, p1)) ncb = p1;
    }
    body(pos0, ce, ncb < p1 ? npos : -1);
    cb = ncb;
    pos0 = npos;
  }
}

// Block-reduce NS-per-lane doubles into part[blockIdx][s*4 + slot]; lanes with g == 0 hold system s values.
template <int NS, int NVAL>
__device__ __forceinline__ void block_partials(const double (&v)[NVAL], double* part) {
  __shared__ double red[8][32][NVAL];
  const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
#pragma unroll
  for (int k = 0; k < NVAL; ++k) red[w][lane][k] = v[k];
  __syncthreads();
  if (threadIdx.x < NS) {
    const int s = threadIdx.x;
    double acc[NVAL];
#pragma unroll
    for (int k = 0; k < NVAL; ++k) acc[k] = 0.0;
    for (int ww = 0; ww < (int)(blockDim.x >> 5); ++ww)
#pragma unroll
      for (int k = 0; k < NVAL; ++k) acc[k] += red[ww][s][k];
#pragma unroll
    for (int k = 0; k < NVAL; ++k) part[((long)blockIdx.x * MAX_SYS + s) * 4 + k] = acc[k];
  }
}

// Packed batches of independent meshes (NS = 1, SEG): the system of a row is
// seg[row].  Each warp slot adds its rows' values to its own per-system sums
// in shared memory; the block then adds the slots in a fixed order, so the
// partial sums stay deterministic.
template <int SLOTS, int NVAL>
__device__ __forceinline__ double (*seg_sums())[MAX_SYS][NVAL] {
  __shared__ double red[SLOTS][MAX_SYS][NVAL];
  for (int i = threadIdx.x; i < SLOTS * MAX_SYS * NVAL; i += blockDim.x) (&red[0][0][0])[i] = 0.0;
  __syncthreads();
  return red;
}

template <int SLOTS, int NVAL>
__device__ __forceinline__ void seg_partials(double (*red)[MAX_SYS][NVAL], double* part) {
  __syncthreads();
  for (int t = threadIdx.x; t < MAX_SYS * NVAL; t += blockDim.x) {
    const int sid = t / NVAL, k = t % NVAL;
    double acc = 0.0;
    for (int sl = 0; sl < SLOTS; ++sl) acc += red[sl][sid][k];
    part[((long)blockIdx.x * MAX_SYS + sid) * 4 + k] = acc;
  }
}

// ------------------------------------------------------------------ forward sweep
// For iteration > 1 first applies the previous update to the row, then
// y_i = (r_i - sum_{j<i} A_ij y_j) * DD_i  (COCG13_single.f90:203-212, 304-307).
template <class T, int NS, bool SEG = false>
__global__ void __launch_bounds__(256)
    k_fwd(const int32_t* __restrict__ rowptr, const int32_t* __restrict__ col, const int32_t* __restrict__ diagpos,
          const typename Cx<T>::V* __restrict__ km, int n, typename Cx<T>::V* __restrict__ r,
          typename Cx<T>::V* __restrict__ y, const typename Cx<T>::V* __restrict__ p,
          const typename Cx<T>::V* __restrict__ q, double2* __restrict__ x, const typename Cx<T>::V* __restrict__ dd,
          unsigned* __restrict__ flag, int mode, SysScal* __restrict__ sc, Ctrl* __restrict__ ctrl,
          double* __restrict__ part, DevStatus* st, typename Cx<T>::V* __restrict__ rprev,
          const int32_t* __restrict__ perm, const uint8_t* __restrict__ seg) {
  using V = typename Cx<T>::V;
  static_assert(!SEG || NS == 1, "packed batches hold one system per row");
  if (ctrl->done) return;
  constexpr int G = 32 / NS;
  const unsigned epoch = ctrl->epoch;
  const unsigned lim = ctrl->spin_limit ? ctrl->spin_limit : SPIN_LIMIT;
  const bool update = ctrl->iter > 0;
  const int lane = threadIdx.x & 31, s = lane % NS, g = lane / NS;
  const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int nwarps = (gridDim.x * blockDim.x) >> 5;
  double om = sc[s].omega;
  double2 al = sc[s].alpha;
  bool act = sc[s].active;
  double rr = 0.0;
  double (*red)[MAX_SYS][1] = nullptr;
  if constexpr (SEG) red = seg_sums<8, 1>();
  for (int pos = warp; pos < n; pos += nwarps) {
    const int row = __ldg(perm + pos);
    int sid = s;
    if constexpr (SEG) {
      sid = __ldg(seg + row);
      om = sc[sid].omega;
      al = sc[sid].alpha;
      act = sc[sid].active;
    }
    V ri = r[(long)row * NS + s];
    if (rprev && g == 0) rprev[(long)row * NS + s] = ri;  // flexible COCG keeps r_k
    if (update && act && g == 0) {
      const V qi = q[(long)row * NS + s], pi = p[(long)row * NS + s];
      ri = Cx<T>::make((T)((double)ri.x - (al.x * (double)qi.x - al.y * (double)qi.y)),
                       (T)((double)ri.y - (al.x * (double)qi.y + al.y * (double)qi.x)));
      r[(long)row * NS + s] = ri;
      double2 xi = x[(long)row * NS + s];
      xi.x += al.x * (double)pi.x - al.y * (double)pi.y;
      xi.y += al.x * (double)pi.y + al.y * (double)pi.x;
      x[(long)row * NS + s] = xi;
    }
    if (g == 0) {
      const double v = (double)ri.x * (double)ri.x + (double)ri.y * (double)ri.y;
      if constexpr (SEG) red[threadIdx.x >> 5][sid][0] += v;
      else rr += v;
    }
    if (mode == 2) {  // DIAG: z = DD r
      if (g == 0) {
        const V d = dd[(long)row * NS + s];
        y[(long)row * NS + s] = Cx<T>::make(ri.x * d.x - ri.y * d.y, ri.x * d.y + ri.y * d.x);
      }
      continue;
    }
    if (mode >= 3) {  // no preconditioner (3) / learned network applied after this kernel (4)
      if (g == 0) y[(long)row * NS + s] = ri;
      continue;
    }
    const int k0 = rowptr[row], k1 = diagpos[row];
    T t1x = 0, t1y = 0, t2x = 0, t2y = 0;
    for (int k = k0 + g; k < k1; k += G) {
      const int j = col[k];
      const V a = km[k];
      if (!wait_flag(flag + j, epoch, st, row, lim)) break;
      const V yj = ldcg(y + (long)j * NS + s);
      t1x += a.x * yj.x; t1y += a.x * yj.y;
      t2x += a.y * yj.x; t2y += a.y * yj.y;
    }
    group_reduce<T, NS>(t1x, t1y, t2x, t2y);
    if (g == 0) {
      const T o = (T)om;
      const T ax = t1x - o * t2y, ay = t1y + o * t2x;
      const T wx = ri.x - ax, wy = ri.y - ay;
      const V d = dd[(long)row * NS + s];
      y[(long)row * NS + s] = Cx<T>::make(wx * d.x - wy * d.y, wx * d.y + wy * d.x);
    }
    __syncwarp();
    if (lane == 0) st_release(flag + row, epoch);  // release: the row's values are visible first
  }
  if constexpr (SEG) {
    seg_partials<8, 1>(red, part);
  } else {
    double v[1] = {rr};
    block_partials<NS, 1>(v, part);
  }
}

// ------------------------------------------------------------------ backward sweep
// z_i = y_i - DD_i * sum_{j>i} A_ij z_j (COCG13_single.f90:214-225), rho += r_i z_i.
template <class T, int NS, bool SEG = false>
__global__ void __launch_bounds__(256)
    k_bwd(const int32_t* __restrict__ rowptr, const int32_t* __restrict__ col, const int32_t* __restrict__ diagpos,
          const typename Cx<T>::V* __restrict__ km, int n, const typename Cx<T>::V* __restrict__ r,
          typename Cx<T>::V* __restrict__ z, const typename Cx<T>::V* __restrict__ dd, unsigned* __restrict__ flag,
          int mode, SysScal* __restrict__ sc, Ctrl* __restrict__ ctrl, double* __restrict__ part, DevStatus* st,
          const typename Cx<T>::V* __restrict__ rprev, const int32_t* __restrict__ perm,
          const uint8_t* __restrict__ seg) {
  using V = typename Cx<T>::V;
  static_assert(!SEG || NS == 1, "packed batches hold one system per row");
  if (ctrl->done) return;
  constexpr int G = 32 / NS;
  const unsigned epoch = ctrl->epoch;
  const unsigned lim = ctrl->spin_limit ? ctrl->spin_limit : SPIN_LIMIT;
  const int lane = threadIdx.x & 31, s = lane % NS, g = lane / NS;
  const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int nwarps = (gridDim.x * blockDim.x) >> 5;
  double om = sc[s].omega;
  double rx = 0.0, ry = 0.0, px = 0.0, py = 0.0;
  double (*red)[MAX_SYS][4] = nullptr;
  if constexpr (SEG) red = seg_sums<8, 4>();
  for (int pos = warp; pos < n; pos += nwarps) {
    const int row = __ldg(perm + pos);
    int sid = s;
    if constexpr (SEG) {
      sid = __ldg(seg + row);
      om = sc[sid].omega;
    }
    V zi = z[(long)row * NS + s];
    if (mode <= 1) {
      const int k0 = diagpos[row] + 1, k1 = rowptr[row + 1];
      T t1x = 0, t1y = 0, t2x = 0, t2y = 0;
      for (int k = k0 + g; k < k1; k += G) {
        const int j = col[k];
        const V a = km[k];
        if (!wait_flag(flag + j, epoch, st, row, lim)) break;
        const V zj = ldcg(z + (long)j * NS + s);
        t1x += a.x * zj.x; t1y += a.x * zj.y;
        t2x += a.y * zj.x; t2y += a.y * zj.y;
      }
      group_reduce<T, NS>(t1x, t1y, t2x, t2y);
      if (g == 0) {
        const T o = (T)om;
        const T swx = t1x - o * t2y, swy = t1y + o * t2x;
        const V d = dd[(long)row * NS + s];
        zi = Cx<T>::make(zi.x - (d.x * swx - d.y * swy), zi.y - (d.x * swy + d.y * swx));
        z[(long)row * NS + s] = zi;
      }
      __syncwarp();
      if (lane == 0) st_release(flag + row, epoch);
    }
    if (g == 0) {
      const V ri = r[(long)row * NS + s];
      const double ex = (double)ri.x * (double)zi.x - (double)ri.y * (double)zi.y;
      const double ey = (double)ri.x * (double)zi.y + (double)ri.y * (double)zi.x;
      if constexpr (SEG) {
        red[threadIdx.x >> 5][sid][0] += ex;
        red[threadIdx.x >> 5][sid][1] += ey;
      } else {
        rx += ex;
        ry += ey;
        if (rprev) {
          const V rp = rprev[(long)row * NS + s];
          px += (double)rp.x * (double)zi.x - (double)rp.y * (double)zi.y;
          py += (double)rp.x * (double)zi.y + (double)rp.y * (double)zi.x;
        }
      }
    }
  }
  if constexpr (SEG) {
    seg_partials<8, 4>(red, part);
  } else {
    double v[4] = {rx, ry, px, py};
    block_partials<NS, 4>(v, part);
  }
}

// ------------------------------------------------------------------ multicolour sweeps
// SSOR of the colour-permuted matrix: rows of one colour share no nonzero, so
// the forward sweep updates colour 0, 1, ... in turn (each a parallel pass over
// its rows, summing only entries of earlier colours) and the backward sweep
// goes through the colours in reverse.  The rows are stored a second time in
// colour order and split into their earlier-colour part (forward) and their
// later-colour part (backward), so a sweep reads half the entries, row data is
// contiguous by position and no entry needs a colour test.  RPW rows share a
// warp (lane = sub * 32/RPW + g * NS + s), which keeps several rows' loads in
// flight per warp.  One persistent cooperative kernel per sweep with a grid
// barrier between colours; no flags, no waits.
// A lane per (row, system): the earlier- or later-colour part of a row holds ~8
// entries, so a row per lane keeps 32/NS rows' dependent loads in flight per
// warp (the sweeps are latency-bound, not bandwidth-bound).  Packed batches
// keep 4 rows per warp so that each row's per-mesh sums have their own slot.
// With 16 systems a lane carries SPL of them (2 by default): a row's 16 values are
// read by its 16/SPL lanes as one contiguous run, and a warp works on 2*SPL rows at
// once (SPL times the independent load chains of a lane per system), with the row's
// column indices and matrix values loaded by 16/SPL lanes instead of 16.
#ifndef AFEM_MC_SPL
#define AFEM_MC_SPL 2  // systems per lane at 16 systems (1, 2 or 4)
#endif
constexpr int MC_MIN_BLOCKS = 4;

template <int NS, bool SEG = false>
struct McShape {
  static constexpr int SPL = (NS == 16 && !SEG) ? AFEM_MC_SPL : 1;  // systems per lane
  static constexpr int NG = NS / SPL;                      // lanes of a row that hold different systems
  static constexpr int RPW = SEG ? 4 : 32 / NG;            // rows per warp
  static constexpr int LPR = 32 / RPW;                     // lanes per row
  static constexpr int G = LPR / NG;                       // entry groups per row
};

// Minimum resident blocks of 256 threads asked of the compiler: the 4-systems-per-lane
// kernels get at most 64 registers a thread, so that 4 blocks (32 warps, 256 rows) stay
// resident per SM; the lane-per-system kernels keep the compiler's choice.
template <int NS, bool SEG>
constexpr int mc_min_blocks() {
  return McShape<NS, SEG>::SPL > 1 ? MC_MIN_BLOCKS : 0;
}

// Two consecutive complex doubles (32 bytes, 32-byte aligned) in one 256-bit access
// (sm_100 ld/st .v4.f64).  A row's 16 FP64 values are then read by 8 lanes as two
// whole 128-byte lines per instruction instead of 16-byte pieces at a 32-byte
// stride, which halves the L1 wavefronts of a gather.  CG: at L2 only (ld.cg).
// RO: the data are not written during the launch, and the load may be scheduled
// freely; otherwise (values other threads write between grid barriers, as in the
// sweeps) the load is also a compiler memory barrier, so it is never moved across a
// grid barrier or a store.
template <bool CG, bool RO>
__device__ __forceinline__ void ld_v4d(const double2* p, double2& a, double2& b) {
  if constexpr (RO) {
    if constexpr (CG)
      asm("ld.global.cg.v4.f64 {%0,%1,%2,%3}, [%4];" : "=d"(a.x), "=d"(a.y), "=d"(b.x), "=d"(b.y) : "l"(p));
    else
      asm("ld.global.v4.f64 {%0,%1,%2,%3}, [%4];" : "=d"(a.x), "=d"(a.y), "=d"(b.x), "=d"(b.y) : "l"(p));
  } else {
    if constexpr (CG)
      asm volatile("ld.global.cg.v4.f64 {%0,%1,%2,%3}, [%4];"
                   : "=d"(a.x), "=d"(a.y), "=d"(b.x), "=d"(b.y) : "l"(p) : "memory");
    else
      asm volatile("ld.global.v4.f64 {%0,%1,%2,%3}, [%4];"
                   : "=d"(a.x), "=d"(a.y), "=d"(b.x), "=d"(b.y) : "l"(p) : "memory");
  }
}
__device__ __forceinline__ void st_v4d(double2* p, double2 a, double2 b) {
  asm volatile("st.global.v4.f64 [%0], {%1,%2,%3,%4};" ::"l"(p), "d"(a.x), "d"(a.y), "d"(b.x), "d"(b.y)
               : "memory");
}

#ifndef AFEM_REFINE_PROGRESS
#define AFEM_REFINE_PROGRESS 0.9  // a refinement must cut the worst true residual below this fraction
#endif

#ifndef AFEM_V4D
#define AFEM_V4D 1  // 256-bit accesses for FP64 pairs (0: two 128-bit accesses)
#endif

// SPL consecutive complex values of one row (systems s0 .. s0+SPL-1) at p: FP32 pairs
// as one 16-byte load, FP64 pairs as one 32-byte load (s0 even, rows 256-byte aligned);
// GATHER: a neighbour's values (L1 or L2, see GatherL1), else the row's own (plain load);
// RO: values nothing writes during the launch (see ld_v4d).
template <class V, int NS, int SPL, bool GATHER, bool RO = false>
__device__ __forceinline__ void load_spl(const V* p, V (&v)[SPL]) {
  if constexpr (AFEM_V4D && SPL > 1 && sizeof(V) == 16) {  // double2 pairs as 32 bytes
#pragma unroll
    for (int i = 0; i < SPL; i += 2) ld_v4d<GATHER && !GatherL1<V, NS>::ok, RO>(p + i, v[i], v[i + 1]);
  } else if constexpr (SPL > 1 && sizeof(V) == 8) {  // float2 pairs as float4
#pragma unroll
    for (int i = 0; i < SPL; i += 2) {
      const float4* q = reinterpret_cast<const float4*>(p + i);
      float4 f;
      if constexpr (GATHER && !GatherL1<V, NS>::ok) f = __ldcg(q);
      else f = *q;
      v[i] = V{f.x, f.y};
      v[i + 1] = V{f.z, f.w};
    }
  } else {
#pragma unroll
    for (int i = 0; i < SPL; ++i) {
      if constexpr (GATHER) v[i] = gather_ld<V, NS>(p + i);
      else v[i] = p[i];
    }
  }
}
template <class V, int SPL>
__device__ __forceinline__ void store_spl(V* p, const V (&v)[SPL]) {
  if constexpr (AFEM_V4D && SPL > 1 && sizeof(V) == 16) {
#pragma unroll
    for (int i = 0; i < SPL; i += 2) st_v4d(p + i, v[i], v[i + 1]);
  } else if constexpr (SPL > 1 && sizeof(V) == 8) {
#pragma unroll
    for (int i = 0; i < SPL; i += 2)
      *reinterpret_cast<float4*>(p + i) = make_float4(v[i].x, v[i].y, v[i + 1].x, v[i + 1].y);
  } else {
#pragma unroll
    for (int i = 0; i < SPL; ++i) p[i] = v[i];
  }
}

// row_gather for a lane carrying SPL systems: sums A_k v_col(k) for systems s0..s0+SPL-1
// over entries k0, k0+G, ... < k1, two entries' loads in flight (SPL = 1: row_gather).
template <class T, int NS, int G, int SPL, bool RO = false>
__device__ __forceinline__ void row_gather_spl(const int32_t* __restrict__ cols,
                                               const typename Cx<T>::V* __restrict__ vals,
                                               const typename Cx<T>::V* vec, int k0, int k1, int s0,
                                               T (&t1x)[SPL], T (&t1y)[SPL], T (&t2x)[SPL], T (&t2y)[SPL]) {
  using V = typename Cx<T>::V;
  if constexpr (SPL == 1) {
    row_gather<T, NS, G>(cols, vals, vec, k0, k1, s0, t1x[0], t1y[0], t2x[0], t2y[0]);
  } else {
    int k = k0;
    if constexpr (G == 1)
      for (; k + 1 < k1; k += 2) {
        const int j0 = __ldg(cols + k), j1 = __ldg(cols + k + 1);
        const V a0 = vals[k], a1 = vals[k + 1];
        V v0[SPL], v1[SPL];
        load_spl<V, NS, SPL, true, RO>(vec + (long)j0 * NS + s0, v0);
        load_spl<V, NS, SPL, true, RO>(vec + (long)j1 * NS + s0, v1);
#pragma unroll
        for (int i = 0; i < SPL; ++i) {
          t1x[i] += a0.x * v0[i].x; t1y[i] += a0.x * v0[i].y; t2x[i] += a0.y * v0[i].x; t2y[i] += a0.y * v0[i].y;
          t1x[i] += a1.x * v1[i].x; t1y[i] += a1.x * v1[i].y; t2x[i] += a1.y * v1[i].x; t2y[i] += a1.y * v1[i].y;
        }
      }
    for (; k < k1; k += G) {
      const int j = __ldg(cols + k);
      const V a = vals[k];
      V v[SPL];
      load_spl<V, NS, SPL, true, RO>(vec + (long)j * NS + s0, v);
#pragma unroll
      for (int i = 0; i < SPL; ++i) {
        t1x[i] += a.x * v[i].x; t1y[i] += a.x * v[i].y; t2x[i] += a.y * v[i].x; t2y[i] += a.y * v[i].y;
      }
    }
  }
}

// Row sums for rows whose LPR lanes hold different systems (G == 1): the row's columns
// and values are loaded once, lane m of the row taking entry m of each block of LPR
// entries (one coalesced load per row instead of LPR copies of every entry), and are
// handed to the row's other lanes by shuffles; a block's gathers are then issued
// BATCH at a time before their products are summed, so a row waits on one column
// load and len/BATCH gathers instead of a column load before every pair of gathers.
// Warp-uniform (shuffles): every lane runs the blocks of the longest row of its warp,
// len = 0 for a lane whose row is not live.  Each lane adds its row's entries in CSR
// order, as row_gather_spl does, so the sums are the same bits.  Used by the nodal
// sweeps (0.84 -> 0.62 ms a pair on the 96x96x64 batch); the edge sweeps measured
// slower with it (forward 1.29 -> 1.51 ms, backward 0.89 -> 1.17 ms) and keep
// row_gather_spl.
#ifndef AFEM_COOP_GATHER
#define AFEM_COOP_GATHER 1
#endif
template <class T, int NS, int SPL, int LPR, int BATCH>
__device__ __forceinline__ void row_gather_coop(const int32_t* __restrict__ cols,
                                                const typename Cx<T>::V* __restrict__ vals,
                                                const typename Cx<T>::V* vec, int k0, int len, int s0,
                                                T (&t1x)[SPL], T (&t1y)[SPL], T (&t2x)[SPL], T (&t2y)[SPL]) {
  using V = typename Cx<T>::V;
  static_assert(LPR % BATCH == 0 && LPR <= 32, "a batch stays inside a block");
  const int ql = threadIdx.x & (LPR - 1);
  const int maxlen = (int)__reduce_max_sync(0xffffffffu, (unsigned)len);
  for (int b = 0; b < maxlen; b += LPR) {
    const bool have = b + ql < len;
    const int jm = have ? __ldg(cols + k0 + b + ql) : 0;
    const V am = have ? vals[k0 + b + ql] : Cx<T>::make(0, 0);
    const int nb = min(LPR, maxlen - b);
    for (int e0 = 0; e0 < nb; e0 += BATCH) {
      V a[BATCH], v[BATCH][SPL];
#pragma unroll
      for (int u = 0; u < BATCH; ++u) {
        const int e = e0 + u;
        const int j = __shfl_sync(0xffffffffu, jm, e, LPR);
        a[u] = Cx<T>::make(__shfl_sync(0xffffffffu, am.x, e, LPR), __shfl_sync(0xffffffffu, am.y, e, LPR));
        if (b + e < len) {
          load_spl<V, NS, SPL, true>(vec + (long)j * NS + s0, v[u]);
        } else {
#pragma unroll
          for (int i = 0; i < SPL; ++i) v[u][i] = Cx<T>::make(0, 0);
        }
      }
#pragma unroll
      for (int u = 0; u < BATCH; ++u)
        if (b + e0 + u < len)
#pragma unroll
          for (int i = 0; i < SPL; ++i) {
            t1x[i] += a[u].x * v[u][i].x; t1y[i] += a[u].x * v[u][i].y;
            t2x[i] += a[u].y * v[u][i].x; t2y[i] += a[u].y * v[u][i].y;
          }
    }
  }
}

// Sum the G entry groups of a row (lanes of one row that hold the same systems).
template <class T, int SPL, int NG, int LPR>
__device__ __forceinline__ void group_sum(T (&a)[SPL], T (&b)[SPL], T (&c)[SPL], T (&d)[SPL]) {
#pragma unroll
  for (int m = NG; m < LPR; m <<= 1)
#pragma unroll
    for (int i = 0; i < SPL; ++i) {
      a[i] += shfl_xor(a[i], m); b[i] += shfl_xor(b[i], m);
      c[i] += shfl_xor(c[i], m); d[i] += shfl_xor(d[i], m);
    }
}

// Block partial sums when a lane carries systems s0..s0+SPL-1 (values nonzero only
// on lanes with g == 0): the rows of each warp are folded with shuffles, the lanes
// of its first row hand their systems' values to shared memory, and threads s < NS
// add the warps in order into part[blockIdx][s][slot].
template <int NS, int SPL, int LPR, int NVAL>
__device__ __forceinline__ void block_partials_spl(double (&v)[SPL][NVAL], int s0, bool g0, double* part) {
  __shared__ double red[8][NS][NVAL];
  const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
#pragma unroll
  for (int m = LPR; m < 32; m <<= 1)
#pragma unroll
    for (int i = 0; i < SPL; ++i)
#pragma unroll
      for (int k = 0; k < NVAL; ++k) v[i][k] += __shfl_xor_sync(0xffffffffu, v[i][k], m);
  if (lane < LPR && g0)
#pragma unroll
    for (int i = 0; i < SPL; ++i)
#pragma unroll
      for (int k = 0; k < NVAL; ++k) red[w][s0 + i][k] = v[i][k];
  __syncthreads();
  if (threadIdx.x < NS) {
    const int sy = threadIdx.x;
    double acc[NVAL];
#pragma unroll
    for (int k = 0; k < NVAL; ++k) acc[k] = 0.0;
    for (int ww = 0; ww < (int)(blockDim.x >> 5); ++ww)
#pragma unroll
      for (int k = 0; k < NVAL; ++k) acc[k] += red[ww][sy][k];
#pragma unroll
    for (int k = 0; k < NVAL; ++k) part[((long)blockIdx.x * MAX_SYS + sy) * 4 + k] = acc[k];
  }
}

// 1 / (sd (K_ii + i omega M_ii)): the SSOR diagonal of the system at omega, from the
// row's (K, M) diagonal pair (COCG13_single.f90:126-130), computed where it is used
// instead of being read from a per-(row, system) array
__device__ __forceinline__ double2 ssor_dd(double2 a, double om, double sd) {
  const double dx = sd * a.x, dy = sd * om * a.y;
  const double inv = 1.0 / (dx * dx + dy * dy);
  return make_double2(dx * inv, -dy * inv);
}

// T: the COCG vectors (r, q); PT: the preconditioner's matrix copy, output y and
// the values gathered from it (PT = float: the FP32 preconditioner of an FP64 solve)
template <class T, class PT, int NS, bool SEG = false>
__global__ void __launch_bounds__(256, (mc_min_blocks<NS, SEG>()))
    k_fwd_mc(const int32_t* __restrict__ lptr, const int32_t* __restrict__ lcol,
             const typename Cx<PT>::V* __restrict__ lkm, int n, typename Cx<T>::V* __restrict__ r,
             typename Cx<PT>::V* __restrict__ y, const typename Cx<T>::V* __restrict__ q,
             const double2* __restrict__ dkm, double sd, const int32_t* __restrict__ perm,
             const int32_t* __restrict__ cptr, int ncolors, SysScal* __restrict__ sc, Ctrl* __restrict__ ctrl,
             double* __restrict__ part, const uint8_t* __restrict__ seg, typename Cx<T>::V* __restrict__ rprev) {
  using V = typename Cx<T>::V;
  using PV = typename Cx<PT>::V;
  using S = McShape<NS, SEG>;
  constexpr int SPL = S::SPL;
  static_assert(!SEG || NS == 1, "packed batches hold one system per row");
  if (ctrl->done) return;  // uniform over the grid
  cooperative_groups::grid_group grid = cooperative_groups::this_grid();
  const bool update = ctrl->iter > 0;
  const int lane = threadIdx.x & 31, sub = lane / S::LPR, ql = lane % S::LPR;
  const int s0 = (ql % S::NG) * SPL, g = ql / S::NG;
  const int slot = (threadIdx.x >> 5) * S::RPW + sub;  // this row's per-warp slot
  double om[SPL], rr[SPL][1];
#pragma unroll
  for (int i = 0; i < SPL; ++i) {
    om[i] = sc[s0 + i].omega;
    rr[i][0] = 0.0;
  }
  double (*red)[MAX_SYS][1] = nullptr;
  if constexpr (SEG) red = seg_sums<8 * S::RPW, 1>();
  for (int c = 0; c < ncolors; ++c) {
    const int p0 = cptr[c], p1 = cptr[c + 1];
    // the next row's id, diagonal pair and pointers, loaded one round ahead
    int nrow = 0, nk0 = 0, nk1 = 0;
    double2 ndg = make_double2(1.0, 0.0);
    auto fetch = [&](int ps) {
      if (ps < p1) {
        nrow = __ldg(perm + ps);
        ndg = __ldg(dkm + ps);
        nk0 = __ldg(lptr + ps);
        nk1 = __ldg(lptr + ps + 1);
      }
    };
    fetch(first_round<S::RPW, AFEM_SWEEP_CHUNK>(p0) + sub);
    for_rows<S::RPW, AFEM_SWEEP_CHUNK>(p0, p1, [&](int pos0, int cend, int next) {
      const int pos = pos0 + sub;
      const bool live = pos < cend;
      const int row = live ? nrow : 0;
      const int k0 = nk0, k1 = nk1;
      const double2 dg = live ? ndg : make_double2(1.0, 0.0);
      if (next >= 0) fetch(next + sub);
      int sid = s0;
      if constexpr (SEG) {
        sid = live ? (int)__ldg(seg + row) : 0;
        om[0] = sc[sid].omega;
      }
      V ri[SPL];
      if (live) load_spl<V, NS, SPL, false>(r + (long)row * NS + s0, ri);
      else
#pragma unroll
        for (int i = 0; i < SPL; ++i) ri[i] = Cx<T>::make(0, 0);
      if (rprev && live && g == 0) store_spl<V, SPL>(rprev + (long)row * NS + s0, ri);  // flexible COCG keeps r_k
      if (live && update && g == 0) {  // x += alpha p follows in the p update
        V qi[SPL];
        load_spl<V, NS, SPL, false>(q + (long)row * NS + s0, qi);
        bool any = false;
#pragma unroll
        for (int i = 0; i < SPL; ++i)
          if (sc[sid + i].active) {  // the system's scalars (read-only here, L1)
            any = true;
            const double2 al = sc[sid + i].alpha;
            ri[i] = Cx<T>::make((T)((double)ri[i].x - (al.x * (double)qi[i].x - al.y * (double)qi[i].y)),
                                (T)((double)ri[i].y - (al.x * (double)qi[i].y + al.y * (double)qi[i].x)));
          }
        if (any) store_spl<V, SPL>(r + (long)row * NS + s0, ri);
      }
      if (live && g == 0)
#pragma unroll
        for (int i = 0; i < SPL; ++i) {
          const double v = (double)ri[i].x * (double)ri[i].x + (double)ri[i].y * (double)ri[i].y;
          if constexpr (SEG) red[slot][sid][0] += v;
          else rr[i][0] += v;
        }
      PT t1x[SPL], t1y[SPL], t2x[SPL], t2y[SPL];
#pragma unroll
      for (int i = 0; i < SPL; ++i) t1x[i] = t1y[i] = t2x[i] = t2y[i] = 0;
      if (live)
        row_gather_spl<PT, NS, S::G, SPL>(lcol, lkm, y, k0 + g, k1, s0, t1x, t1y,
                                          t2x, t2y);
      group_sum<PT, SPL, S::NG, S::LPR>(t1x, t1y, t2x, t2y);
      if (live && g == 0) {
        PV yo[SPL];
#pragma unroll
        for (int i = 0; i < SPL; ++i) {
          const PT o = (PT)om[i];
          const PT wx = (PT)ri[i].x - (t1x[i] - o * t2y[i]), wy = (PT)ri[i].y - (t1y[i] + o * t2x[i]);
          const double2 dd = ssor_dd(dg, om[i], sd);
          const PT dx = (PT)dd.x, dy = (PT)dd.y;
          yo[i] = Cx<PT>::make(wx * dx - wy * dy, wx * dy + wy * dx);
        }
        store_spl<PV, SPL>(y + (long)row * NS + s0, yo);
      }
    });
    grid.sync();
  }
  if constexpr (SEG) {
    seg_partials<8 * S::RPW, 1>(red, part);
  } else {
    block_partials_spl<NS, SPL, S::LPR, 1>(rr, s0, g == 0, part);
  }
}

// Backward sweep in place on z (the forward sweep's y).  r (COCG type T) is read
// only by packed batches, for their per-mesh rho = r^T z.
template <class T, class PT, int NS, bool SEG = false>
__global__ void __launch_bounds__(256, (mc_min_blocks<NS, SEG>()))
    k_bwd_mc(const int32_t* __restrict__ uptr, const int32_t* __restrict__ ucol,
             const typename Cx<PT>::V* __restrict__ ukm, int n, const typename Cx<T>::V* __restrict__ r,
             typename Cx<PT>::V* __restrict__ z, const int32_t* __restrict__ perm,
             const int32_t* __restrict__ cptr, int ncolors, SysScal* __restrict__ sc, Ctrl* __restrict__ ctrl,
             double* __restrict__ part, const uint8_t* __restrict__ seg, const double2* __restrict__ dkm,
             double sd) {
  using V = typename Cx<T>::V;
  using PV = typename Cx<PT>::V;
  using S = McShape<NS, SEG>;
  constexpr int SPL = S::SPL;
  static_assert(!SEG || NS == 1, "packed batches hold one system per row");
  if (ctrl->done) return;
  cooperative_groups::grid_group grid = cooperative_groups::this_grid();
  const int lane = threadIdx.x & 31, sub = lane / S::LPR, ql = lane % S::LPR;
  const int s0 = (ql % S::NG) * SPL, g = ql / S::NG;
  const int slot = (threadIdx.x >> 5) * S::RPW + sub;  // this row's per-warp slot
  double om[SPL], rh[SPL][4];
#pragma unroll
  for (int i = 0; i < SPL; ++i) {
    om[i] = sc[s0 + i].omega;
    rh[i][0] = rh[i][1] = rh[i][2] = rh[i][3] = 0.0;
  }
  double (*red)[MAX_SYS][4] = nullptr;
  if constexpr (SEG) red = seg_sums<8 * S::RPW, 4>();
  for (int c = ncolors - 1; c >= 0; --c) {
    const int p0 = cptr[c], p1 = cptr[c + 1];
    // the next row's id, diagonal pair and pointers, loaded one round ahead
    int nrow = 0, nk0 = 0, nk1 = 0;
    double2 ndg = make_double2(1.0, 0.0);
    auto fetch = [&](int ps) {
      if (ps < p1) {
        nrow = __ldg(perm + ps);
        ndg = __ldg(dkm + ps);
        nk0 = __ldg(uptr + ps);
        nk1 = __ldg(uptr + ps + 1);
      }
    };
    fetch(first_round<S::RPW, AFEM_SWEEP_CHUNK>(p0) + sub);
    for_rows<S::RPW, AFEM_SWEEP_CHUNK>(p0, p1, [&](int pos0, int cend, int next) {
      const int pos = pos0 + sub;
      const bool live = pos < cend;
      const int row = live ? nrow : 0;
      const int k0 = nk0, k1 = nk1;
      const double2 dg = live ? ndg : make_double2(1.0, 0.0);
      if (next >= 0) fetch(next + sub);
      int sid = s0;
      if constexpr (SEG) {
        sid = live ? (int)__ldg(seg + row) : 0;
        om[0] = sc[sid].omega;
      }
      PT t1x[SPL], t1y[SPL], t2x[SPL], t2y[SPL];
#pragma unroll
      for (int i = 0; i < SPL; ++i) t1x[i] = t1y[i] = t2x[i] = t2y[i] = 0;
      if (live)
        row_gather_spl<PT, NS, S::G, SPL>(ucol, ukm, z, k0 + g, k1, s0, t1x, t1y,
                                          t2x, t2y);
      group_sum<PT, SPL, S::NG, S::LPR>(t1x, t1y, t2x, t2y);
      if (live && g == 0) {
        PV zi[SPL];
        load_spl<PV, NS, SPL, false>(z + (long)row * NS + s0, zi);
#pragma unroll
        for (int i = 0; i < SPL; ++i) {
          if constexpr (!SEG) {
            // rho = r^T z = y^T D' y (U = L^T, D' = sd diag(A), y = the forward sweep's output in z)
            const double dx = sd * dg.x, dy = sd * om[i] * dg.y;
            const double y2x = (double)zi[i].x * (double)zi[i].x - (double)zi[i].y * (double)zi[i].y;
            const double y2y = 2.0 * (double)zi[i].x * (double)zi[i].y;
            rh[i][0] += dx * y2x - dy * y2y;
            rh[i][1] += dx * y2y + dy * y2x;
          }
          const PT o = (PT)om[i];
          const PT swx = t1x[i] - o * t2y[i], swy = t1y[i] + o * t2x[i];
          const double2 dd = ssor_dd(dg, om[i], sd);
          const PT dx = (PT)dd.x, dy = (PT)dd.y;
          zi[i] = Cx<PT>::make(zi[i].x - (dx * swx - dy * swy), zi[i].y - (dx * swy + dy * swx));
        }
        store_spl<PV, SPL>(z + (long)row * NS + s0, zi);
        if constexpr (SEG) {  // packed batches: per-mesh rho = r^T z
          const V ri = r[(long)row * NS + s0];
          red[slot][sid][0] += (double)ri.x * (double)zi[0].x - (double)ri.y * (double)zi[0].y;
          red[slot][sid][1] += (double)ri.x * (double)zi[0].y + (double)ri.y * (double)zi[0].x;
        }
      }
    });
    grid.sync();
  }
  if constexpr (SEG) {
    seg_partials<8 * S::RPW, 4>(red, part);
  } else {
    block_partials_spl<NS, SPL, S::LPR, 4>(rh, s0, g == 0, part);
  }
}

// values of the colour-ordered split rows: out[k] = km[src[k]]
template <class Vd>
__global__ void k_gather_entries(const double2* __restrict__ km, const int32_t* __restrict__ src, long cnt,
                                 Vd* __restrict__ out) {
  for (long k = blockIdx.x * (long)blockDim.x + threadIdx.x; k < cnt; k += (long)gridDim.x * blockDim.x) {
    const double2 v = km[__ldg(src + k)];
    if constexpr (sizeof(Vd) == 16) out[k] = v;
    else out[k] = make_float2((float)v.x, (float)v.y);
  }
}

// ------------------------------------------------------------------ gradient-space correction
// z += G SSOR_node(G^T r) (Hiptmair's hybrid smoother in additive form): the
// nodal right-hand side t = G^T r, two multicolour sweeps on A_G = K_G + i omega M_G,
// then z += G u and the rho = r^T z partial sums of the corrected z.

// t_a = sum over the non-Dirichlet edges e at node a of g_ea r_e (g = +1 at the head, -1 at the tail)
// (r in the COCG type T, t in the preconditioner type PT; the sum runs in T)
template <class T, class PT, int NS>
__global__ void k_grad_t(int node, const int32_t* __restrict__ nptr, const int32_t* __restrict__ nlist,
                         const uint8_t* __restrict__ bc, const typename Cx<T>::V* __restrict__ r,
                         typename Cx<PT>::V* __restrict__ t, const Ctrl* __restrict__ ctrl) {
  if (ctrl->done) return;
  const long total = (long)node * NS;
  for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < total; i += (long)gridDim.x * blockDim.x) {
    const int a = (int)(i / NS), s = (int)(i % NS);
    T ax = 0, ay = 0;
    for (int q = __ldg(nptr + a); q < __ldg(nptr + a + 1); ++q) {
      const int v = __ldg(nlist + q), e = v >> 1;
      if (__ldg(bc + e)) continue;
      const typename Cx<T>::V re = r[(long)e * NS + s];
      if (v & 1) { ax -= re.x; ay -= re.y; }
      else { ax += re.x; ay += re.y; }
    }
    t[i] = Cx<PT>::make((PT)ax, (PT)ay);
  }
}

// One multicolour SSOR sweep on the nodal matrix, over its colour-ordered split
// rows (as the edge sweeps): forward y_a = (t_a - sum_{col(b)<col(a)} A_ab y_b) dd_a,
// backward (in place) y_a -= dd_a sum_{col(b)>col(a)} A_ab y_b.  Grid barrier between colours.
// part (backward, nullable): partial sums of t^T y over the final y, the share
// r^T G u of rho = r^T (z + G u) (since t = G^T r), slots 0, 1.
template <class T, int NS, bool SEG>
__global__ void __launch_bounds__(256, (mc_min_blocks<NS, SEG>()))
    k_nsweep_mc(const int32_t* __restrict__ xptr, const int32_t* __restrict__ xcol,
                const typename Cx<T>::V* __restrict__ xkm, const typename Cx<T>::V* __restrict__ t,
                typename Cx<T>::V* __restrict__ y, const typename Cx<T>::V* __restrict__ dd,
                const int32_t* __restrict__ perm, const int32_t* __restrict__ cptr, int ncolors,
                const SysScal* __restrict__ sc, const Ctrl* __restrict__ ctrl, const uint8_t* __restrict__ seg,
                int backward, double* __restrict__ part) {
  using V = typename Cx<T>::V;
  using S = McShape<NS, SEG>;
  constexpr int SPL = S::SPL;
  static_assert(!SEG || NS == 1, "packed batches hold one system per row");
  if (ctrl->done) return;
  cooperative_groups::grid_group grid = cooperative_groups::this_grid();
  const int lane = threadIdx.x & 31, sub = lane / S::LPR, ql = lane % S::LPR;
  const int s0 = (ql % S::NG) * SPL, g = ql / S::NG;
  double om[SPL], tu[SPL][4];
#pragma unroll
  for (int i = 0; i < SPL; ++i) {
    om[i] = sc[s0 + i].omega;
    tu[i][0] = tu[i][1] = tu[i][2] = tu[i][3] = 0.0;
  }
  for (int cc = 0; cc < ncolors; ++cc) {
    const int c = backward ? ncolors - 1 - cc : cc;
    const int p0 = cptr[c], p1 = cptr[c + 1];
    // the next row's id and pointers, loaded one round ahead
    int nrow = 0, nk0 = 0, nk1 = 0;

    auto fetch = [&](int ps) {
      if (ps < p1) {
        nrow = __ldg(perm + ps);

        nk0 = __ldg(xptr + ps);
        nk1 = __ldg(xptr + ps + 1);
      }
    };
    fetch(first_round<S::RPW, AFEM_SWEEP_CHUNK>(p0) + sub);
    for_rows<S::RPW, AFEM_SWEEP_CHUNK>(p0, p1, [&](int pos0, int cend, int next) {
      const int pos = pos0 + sub;
      const bool live = pos < cend;
      const int row = live ? nrow : 0;
      const int k0 = nk0, k1 = nk1;
      if (next >= 0) fetch(next + sub);
      if constexpr (SEG) om[0] = sc[live ? (int)__ldg(seg + row) : 0].omega;
      T t1x[SPL], t1y[SPL], t2x[SPL], t2y[SPL];
#pragma unroll
      for (int i = 0; i < SPL; ++i) t1x[i] = t1y[i] = t2x[i] = t2y[i] = 0;
      if constexpr (AFEM_COOP_GATHER && S::G == 1 && S::LPR == 8 && !SEG)
        row_gather_coop<T, NS, SPL, S::LPR, (sizeof(T) == 4 ? 4 : 2)>(xcol, xkm, y, k0, live ? k1 - k0 : 0, s0, t1x,
                                                                      t1y, t2x, t2y);
      else if (live)
        row_gather_spl<T, NS, S::G, SPL>(xcol, xkm, y, k0 + g, k1, s0, t1x, t1y,
                                         t2x, t2y);
      group_sum<T, SPL, S::NG, S::LPR>(t1x, t1y, t2x, t2y);
      if (live && g == 0) {
        const long base = (long)row * NS + s0;
        V d[SPL], yo[SPL];
        load_spl<V, NS, SPL, false>(dd + base, d);
        if (!backward) {
          V ti[SPL];
          load_spl<V, NS, SPL, false>(t + base, ti);
#pragma unroll
          for (int i = 0; i < SPL; ++i) {
            const T o = (T)om[i];
            const T sx = t1x[i] - o * t2y[i], sy = t1y[i] + o * t2x[i];
            const T wx = ti[i].x - sx, wy = ti[i].y - sy;
            yo[i] = Cx<T>::make(wx * d[i].x - wy * d[i].y, wx * d[i].y + wy * d[i].x);
          }
        } else {
          V yi[SPL];
          load_spl<V, NS, SPL, false>(y + base, yi);
#pragma unroll
          for (int i = 0; i < SPL; ++i) {
            const T o = (T)om[i];
            const T sx = t1x[i] - o * t2y[i], sy = t1y[i] + o * t2x[i];
            yo[i] = Cx<T>::make(yi[i].x - (d[i].x * sx - d[i].y * sy), yi[i].y - (d[i].x * sy + d[i].y * sx));
          }
          if (part) {
            V ti[SPL];
            load_spl<V, NS, SPL, false>(t + base, ti);
#pragma unroll
            for (int i = 0; i < SPL; ++i) {
              tu[i][0] += (double)ti[i].x * (double)yo[i].x - (double)ti[i].y * (double)yo[i].y;
              tu[i][1] += (double)ti[i].x * (double)yo[i].y + (double)ti[i].y * (double)yo[i].x;
            }
          }
        }
        store_spl<V, SPL>(y + base, yo);
      }
    });
    grid.sync();
  }
  if (part) block_partials_spl<NS, SPL, S::LPR, 4>(tu, s0, g == 0, part);  // uniform over the grid
}

// Packed batches: the lanes of a warp hold rows of possibly different meshes;
// lane 0 adds them to the warp's per-mesh slots in lane order (deterministic).
template <int NVAL>
__device__ __forceinline__ void seg_warp_add(double (*red)[MAX_SYS][NVAL], int slot, int sid, const double (&v)[NVAL]) {
  const int lane = threadIdx.x & 31;
  for (int l = 0; l < 32; ++l) {
    const int sl = __shfl_sync(0xffffffffu, sid, l);
    double vl[NVAL];
#pragma unroll
    for (int k = 0; k < NVAL; ++k) vl[k] = __shfl_sync(0xffffffffu, v[k], l);
    if (lane == 0 && sl >= 0) {
#pragma unroll
      for (int k = 0; k < NVAL; ++k) red[slot][sl][k] += vl[k];
    }
  }
}

// z_e += u_head(e) - u_tail(e) on the non-Dirichlet edges, then rho = r^T z partial sums (slots 0, 1)
// (u, z in the preconditioner type PT, r in the COCG type T)
template <class T, class PT, int NS, bool SEG>
__global__ void __launch_bounds__(256)
    k_grad_add(int n, const int32_t* __restrict__ line, const uint8_t* __restrict__ bc,
               const typename Cx<PT>::V* __restrict__ u, typename Cx<PT>::V* __restrict__ z,
               const typename Cx<T>::V* __restrict__ r, const Ctrl* __restrict__ ctrl, double* __restrict__ part,
               const uint8_t* __restrict__ seg) {
  using V = typename Cx<T>::V;
  using PV = typename Cx<PT>::V;
  static_assert(!SEG || NS == 1, "packed batches hold one system per row");
  if (ctrl->done) return;
  const long total = (long)n * NS;
  const long stride = (long)gridDim.x * blockDim.x;  // a multiple of NS: lane % NS is the system
  double rx = 0.0, ry = 0.0;
  double (*red)[MAX_SYS][4] = nullptr;
  if constexpr (SEG) red = seg_sums<8, 4>();
  const long span = (total + stride - 1) / stride * stride;  // every lane runs the same trip count
  for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < span; i += stride) {
    double ex = 0.0, ey = 0.0;
    int sid = -1;
    if (i < total) {
      const int e = (int)(i / NS), s = (int)(i % NS);
      PV zi = z[i];
      if (!__ldg(bc + e)) {
        const PV uh = u[(long)(__ldg(line + 2 * e + 1) - 1) * NS + s];
        const PV ut = u[(long)(__ldg(line + 2 * e) - 1) * NS + s];
        zi = Cx<PT>::make(zi.x + (uh.x - ut.x), zi.y + (uh.y - ut.y));
        z[i] = zi;
      }
      const V ri = r[i];
      ex = (double)ri.x * (double)zi.x - (double)ri.y * (double)zi.y;
      ey = (double)ri.x * (double)zi.y + (double)ri.y * (double)zi.x;
      sid = SEG ? (int)__ldg(seg + e) : s;
    }
    if constexpr (SEG) {
      const double v[4] = {ex, ey, 0.0, 0.0};
      seg_warp_add<4>(red, threadIdx.x >> 5, sid, v);
    } else {
      rx += ex;
      ry += ey;
    }
  }
  if constexpr (SEG) {
    seg_partials<8, 4>(red, part);
  } else {
#pragma unroll
    for (int m = NS; m < 32; m <<= 1) {
      rx += __shfl_xor_sync(0xffffffffu, rx, m);
      ry += __shfl_xor_sync(0xffffffffu, ry, m);
    }
    double v[4] = {rx, ry, 0.0, 0.0};
    block_partials<NS, 4>(v, part);
  }
}

// rho = r^T z and rprev^T z partial sums (slots 0..3) after the learned correction
// changed z (flexible COCG's beta needs both); NS systems per row, no packed batches
template <class T, int NS>
__global__ void __launch_bounds__(256)
    k_dots(int n, const typename Cx<T>::V* __restrict__ r, const typename Cx<T>::V* __restrict__ z,
           const typename Cx<T>::V* __restrict__ rprev, const Ctrl* __restrict__ ctrl, double* __restrict__ part) {
  if (ctrl->done) return;
  const long total = (long)n * NS;
  double v[4] = {0.0, 0.0, 0.0, 0.0};
  for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < total; i += (long)gridDim.x * blockDim.x) {
    const typename Cx<T>::V ri = r[i], zi = z[i], pi = rprev[i];
    v[0] += (double)ri.x * (double)zi.x - (double)ri.y * (double)zi.y;
    v[1] += (double)ri.x * (double)zi.y + (double)ri.y * (double)zi.x;
    v[2] += (double)pi.x * (double)zi.x - (double)pi.y * (double)zi.y;
    v[3] += (double)pi.x * (double)zi.y + (double)pi.y * (double)zi.x;
  }
#pragma unroll
  for (int m = NS; m < 32; m <<= 1)
#pragma unroll
    for (int k = 0; k < 4; ++k) v[k] += __shfl_xor_sync(0xffffffffu, v[k], m);
  block_partials<NS, 4>(v, part);
}

// dd_a = 1 / A_G(omega)_aa for nodes with a non-Dirichlet edge, 0 for the others
template <class T, int NS>
__global__ void k_dd_node(const double2* __restrict__ km, const int32_t* __restrict__ diagpos,
                          const uint8_t* __restrict__ live, int node, const SysScal* __restrict__ sc,
                          typename Cx<T>::V* __restrict__ dd, const uint8_t* __restrict__ seg) {
  const long total = (long)node * NS;
  for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < total; i += (long)gridDim.x * blockDim.x) {
    const int a = (int)(i / NS), s = seg ? (int)__ldg(seg + a) : (int)(i % NS);
    const double2 v = km[diagpos[a]];
    const double2 D = make_double2(v.x, sc[s].omega * v.y);
    double2 w = make_double2(0.0, 0.0);
    if (live[a] && (D.x != 0.0 || D.y != 0.0)) w = cdiv(make_double2(1.0, 0.0), D);
    dd[i] = Cx<T>::make((T)w.x, (T)w.y);
  }
}

// ------------------------------------------------------------------ p update, SpMV
// Multicolour path (x != nullptr): first x += alpha p with the old p for the
// systems whose update is pending (also after the residual check ended the
// solve).  Hybrid preconditioner with the gradient add folded in (u != nullptr):
// z_e + u_head(e) - u_tail(e) on the non-Dirichlet edges stands for z.
// (p in the COCG type T; z and u in the preconditioner type PT)
template <class T, class PT, int NS, bool SEG = false>
__global__ void k_pupd(int n, const typename Cx<PT>::V* __restrict__ z, typename Cx<T>::V* __restrict__ p,
                       const SysScal* __restrict__ sc, const Ctrl* __restrict__ ctrl, const uint8_t* __restrict__ seg,
                       double2* __restrict__ x, int nsys, const int32_t* __restrict__ line,
                       const uint8_t* __restrict__ bc, const typename Cx<PT>::V* __restrict__ u) {
  using V = typename Cx<T>::V;
  using PV = typename Cx<PT>::V;
  const bool done = ctrl->done;
  if (done) {
    if (!x) return;
    bool any = false;
    for (int k = 0; k < nsys; ++k) any |= sc[k].xpend != 0;
    if (!any) return;
  }
  const bool first = ctrl->iter == 0;
  const long total = (long)n * NS;
  for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < total; i += (long)gridDim.x * blockDim.x) {
    const int s = SEG ? (int)__ldg(seg + i) : (int)(i % NS);
    V pi = Cx<T>::make(0, 0);
    bool have_p = false;
    if (x && sc[s].xpend) {
      pi = p[i];
      have_p = true;
      const double2 al = sc[s].alpha;
      double2 xi = x[i];
      xi.x += al.x * (double)pi.x - al.y * (double)pi.y;
      xi.y += al.x * (double)pi.y + al.y * (double)pi.x;
      x[i] = xi;
    }
    if (done) continue;
    const PV zp = z[i];
    V zi = Cx<T>::make((T)zp.x, (T)zp.y);
    if (u) {
      const int e = (int)(i / NS);
      if (!__ldg(bc + e)) {
        const int sn = SEG ? 0 : s;
        const PV uh = u[(long)(__ldg(line + 2 * e + 1) - 1) * NS + sn];
        const PV ut = u[(long)(__ldg(line + 2 * e) - 1) * NS + sn];
        zi = Cx<T>::make(zi.x + (T)(uh.x - ut.x), zi.y + (T)(uh.y - ut.y));
      }
    }
    if (first) {
      p[i] = zi;
    } else {
      const double2 be = sc[s].beta;
      if (!have_p) pi = p[i];
      p[i] = Cx<T>::make((T)((double)zi.x + (be.x * (double)pi.x - be.y * (double)pi.y)),
                         (T)((double)zi.y + (be.x * (double)pi.y + be.y * (double)pi.x)));
    }
  }
}

// k_pupd for 16 systems sharing a matrix: a thread takes 2 consecutive systems of
// one row, so the 8 threads of a row read and write its FP64 values (p, x) as one
// 256-byte run of 32-byte accesses and its FP32 values (z, u) as one 128-byte run
// of 16-byte accesses; the systems' scalars stay in registers.  The grid-stride is
// a multiple of 8, so a thread keeps the same 2 systems throughout.
template <class T, class PT, int NS>
__global__ void k_pupd_spl(int n, const typename Cx<PT>::V* __restrict__ z, typename Cx<T>::V* __restrict__ p,
                           const SysScal* __restrict__ sc, const Ctrl* __restrict__ ctrl, double2* __restrict__ x,
                           int nsys, const int32_t* __restrict__ line, const uint8_t* __restrict__ bc,
                           const typename Cx<PT>::V* __restrict__ u) {
  using V = typename Cx<T>::V;
  using PV = typename Cx<PT>::V;
  constexpr int SP = 2, GPR = NS / SP;  // systems per thread, threads per row
  const bool done = ctrl->done;
  if (done) {
    if (!x) return;
    bool any = false;
    for (int k = 0; k < nsys; ++k) any |= sc[k].xpend != 0;
    if (!any) return;
  }
  const bool first = ctrl->iter == 0;
  const long total = (long)n * GPR;
  const long stride = (long)gridDim.x * blockDim.x;
  const long i0 = blockIdx.x * (long)blockDim.x + threadIdx.x;
  const int s0 = (int)(i0 % GPR) * SP;
  double2 al[SP], be[SP];
  bool xp[SP], anyx = false;
#pragma unroll
  for (int j = 0; j < SP; ++j) {
    xp[j] = x && sc[s0 + j].xpend;
    al[j] = sc[s0 + j].alpha;
    be[j] = sc[s0 + j].beta;
    anyx |= xp[j];
  }
  for (long i = i0; i < total; i += stride) {
    const int e = (int)(i / GPR);
    const long base = (long)e * NS + s0;
    V pi[SP];
    bool have_p = false;
    if (anyx) {
      load_spl<V, NS, SP, false>(p + base, pi);
      have_p = true;
      double2 xi[SP];
      load_spl<double2, NS, SP, false>(x + base, xi);
#pragma unroll
      for (int j = 0; j < SP; ++j)
        if (xp[j]) {
          xi[j].x += al[j].x * (double)pi[j].x - al[j].y * (double)pi[j].y;
          xi[j].y += al[j].x * (double)pi[j].y + al[j].y * (double)pi[j].x;
        }
      store_spl<double2, SP>(x + base, xi);  // a system not pending keeps its value
    }
    if (done) continue;
    PV zp[SP];
    load_spl<PV, NS, SP, false>(z + base, zp);
    V zi[SP];
#pragma unroll
    for (int j = 0; j < SP; ++j) zi[j] = Cx<T>::make((T)zp[j].x, (T)zp[j].y);
    if (u && !__ldg(bc + e)) {
      PV uh[SP], ut[SP];
      load_spl<PV, NS, SP, false>(u + (long)(__ldg(line + 2 * e + 1) - 1) * NS + s0, uh);
      load_spl<PV, NS, SP, false>(u + (long)(__ldg(line + 2 * e) - 1) * NS + s0, ut);
#pragma unroll
      for (int j = 0; j < SP; ++j)
        zi[j] = Cx<T>::make(zi[j].x + (T)(uh[j].x - ut[j].x), zi[j].y + (T)(uh[j].y - ut[j].y));
    }
    if (first) {
      store_spl<V, SP>(p + base, zi);
    } else {
      if (!have_p) load_spl<V, NS, SP, false>(p + base, pi);
      V po[SP];
#pragma unroll
      for (int j = 0; j < SP; ++j)
        po[j] = Cx<T>::make((T)((double)zi[j].x + (be[j].x * (double)pi[j].x - be[j].y * (double)pi[j].y)),
                            (T)((double)zi[j].y + (be[j].x * (double)pi[j].y + be[j].y * (double)pi[j].x)));
      store_spl<V, SP>(p + base, po);
    }
  }
}

// q = A p (COCG13_single.f90:273-288) and p^T q partial sums.  With
// resid_mode, computes r = b - A x in FP64 instead and ||r||^2 (and ||b||^2).
// RPW rows per warp, SPL systems per lane: lane = sub * (32/RPW) + g * (NS/SPL) +
// s0/SPL, so rows of ~16 nonzeros do not leave half a warp idle (RPW and SPL are
// picked by tune_spmv; SPL = 4 at 16 systems gives 8 rows per warp).
template <class T, int NS, int RPW = 1, bool SEG = false, int SPL = 1>
__global__ void __launch_bounds__(256, (SPL > 1 ? MC_MIN_BLOCKS : 0))
    k_spmv(const int32_t* __restrict__ rowptr, const int32_t* __restrict__ col,
           const typename Cx<T>::V* __restrict__ km, int n, const typename Cx<T>::V* __restrict__ p,
           typename Cx<T>::V* __restrict__ q, const SysScal* __restrict__ sc, const Ctrl* __restrict__ ctrl,
           double* __restrict__ part, const typename Cx<T>::V* __restrict__ bvec, const uint8_t* __restrict__ seg) {
  using V = typename Cx<T>::V;
  constexpr int NG = NS / SPL;   // lanes of a row that hold different systems
  static_assert(NG * RPW <= 32, "rows per warp times lanes per row must fit a warp");
  static_assert(!SEG || (NS == 1 && SPL == 1), "packed batches hold one system per row");
  if (ctrl && ctrl->done) return;
  constexpr int LPR = 32 / RPW;  // lanes per row
  constexpr int G = LPR / NG;    // entry groups per row
  const int lane = threadIdx.x & 31, sub = lane / LPR, ql = lane % LPR;
  const int s0 = (ql % NG) * SPL, g = ql / NG;
  // SPL > 1 never runs in resid_mode (the true residual uses one system per lane):
  // two sums per system (p^T q) keep the 64-register variant free of spills
  constexpr int NACC = SPL > 1 ? 2 : 3;
  double om1 = sc[s0].omega;  // SPL = 1: this lane's system (SEG: set per row)
  double acc[SPL][NACC];
#pragma unroll
  for (int i = 0; i < SPL; ++i)
#pragma unroll
    for (int k = 0; k < NACC; ++k) acc[i][k] = 0.0;
  double (*red)[MAX_SYS][3] = nullptr;
  if constexpr (SEG) red = seg_sums<8 * RPW, 3>();
  const int slot = (threadIdx.x >> 5) * RPW + sub;
  // row pointers of the warp's next row, loaded one round ahead
  int nk0 = 0, nk1 = 0;
  {
    const int wib = threadIdx.x >> 5;
    const int first = (int)blockIdx.x * AFEM_SPMV_CHUNK * (int)(blockDim.x >> 5) * RPW + wib * RPW + sub;
    if (first < n) { nk0 = __ldg(rowptr + first); nk1 = __ldg(rowptr + first + 1); }
  }
  for_rows<RPW, AFEM_SPMV_CHUNK>(0, n, [&](int row0, int cend, int next) {
    const int row = row0 + sub;
    const bool live = row < cend;
    int sid = s0;
    if constexpr (SEG) {
      sid = live ? (int)__ldg(seg + row) : 0;
      om1 = sc[sid].omega;
    }
    const int k0 = live ? nk0 : 0, k1 = live ? nk1 : 0;
    if (next >= 0 && next + sub < n) { nk0 = __ldg(rowptr + next + sub); nk1 = __ldg(rowptr + next + sub + 1); }
    T t1x[SPL], t1y[SPL], t2x[SPL], t2y[SPL];
#pragma unroll
    for (int i = 0; i < SPL; ++i) t1x[i] = t1y[i] = t2x[i] = t2y[i] = 0;
    row_gather_spl<T, NS, G, SPL, true>(col, km, p, k0 + g, k1, s0, t1x, t1y, t2x, t2y);
    group_sum<T, SPL, NG, LPR>(t1x, t1y, t2x, t2y);
    if (g == 0 && live) {
      const long base = (long)row * NS + s0;
      V qi[SPL], own[SPL];
#pragma unroll
      for (int i = 0; i < SPL; ++i) {
        const T o = (T)(SPL == 1 ? om1 : __ldg(&sc[s0 + i].omega));
        qi[i] = Cx<T>::make(t1x[i] - o * t2y[i], t1y[i] + o * t2x[i]);
      }
      if (SPL == 1 && bvec) {  // r = b - A x
        load_spl<V, NS, SPL, false>(bvec + base, own);
#pragma unroll
        for (int i = 0; i < SPL; ++i) {
          const V ri = Cx<T>::make(own[i].x - qi[i].x, own[i].y - qi[i].y);
          qi[i] = ri;
          const double e0 = (double)ri.x * (double)ri.x + (double)ri.y * (double)ri.y;
          const double e2 = (double)own[i].x * (double)own[i].x + (double)own[i].y * (double)own[i].y;
          if constexpr (SEG) { red[slot][sid][0] += e0; red[slot][sid][2] += e2; }
          else { acc[i][0] += e0; acc[i][NACC - 1] += e2; }
        }
      } else {
        load_spl<V, NS, SPL, false, true>(p + base, own);
#pragma unroll
        for (int i = 0; i < SPL; ++i) {
          const double e0 = (double)own[i].x * (double)qi[i].x - (double)own[i].y * (double)qi[i].y;
          const double e1 = (double)own[i].x * (double)qi[i].y + (double)own[i].y * (double)qi[i].x;
          if constexpr (SEG) { red[slot][sid][0] += e0; red[slot][sid][1] += e1; }
          else { acc[i][0] += e0; acc[i][1] += e1; }
        }
      }
      store_spl<V, SPL>(q + base, qi);
    }
  });
  if constexpr (SEG) {
    seg_partials<8 * RPW, 3>(red, part);
    return;
  }
  block_partials_spl<NS, SPL, LPR, NACC>(acc, s0, g == 0, part);
}

// ------------------------------------------------------------------ tiled SpMV (16 systems, FP64)
// Rows in tiles of SPT_ROWS consecutive rows.  The distinct columns of a tile's
// entries (the rows of p its sums gather: ~154 for the ~520 entries of 32 rows of a
// tetrahedral edge mesh) are listed once (spt_uniq from spt_ptr[t]), and every entry
// holds the position of its column in that list (spt_lidx, 16 bits).  The tile's
// block copies those p rows into shared memory with independent, coalesced 256-bit
// loads, then each row sums its entries in CSR order from shared memory: a row's
// gathers no longer wait on global loads one pair at a time, and each distinct p row
// crosses L2 once per tile instead of once per entry.  A tile with more than
// SPT_UCAP distinct columns (or more entries than the builder's table takes) is
// flagged and summed from global memory as in k_spmv.  The sums, and so q, are the
// same bits as k_spmv's two-systems-per-lane variant (same entry order, same FMAs).
constexpr int SPT_ROWS = 32;    // rows per tile: 8 warps x 4 rows
constexpr int SPT_UCAP = 192;   // distinct columns staged per tile (48 KB of FP64 p rows)
constexpr int SPT_HASH = 2048;  // builder's open-addressing table; tiles of > SPT_HASH/2 entries fall back
constexpr int SPT_PIECES = (SPT_UCAP * 8 + 255) / 256;  // 32-byte pieces a thread copies at most
#ifndef SPT_GROUP
#define SPT_GROUP 3  // pieces a thread has in flight while staging
#endif

__device__ __forceinline__ unsigned spt_hash(int j) { return ((unsigned)j * 2654435761u) >> 21; }  // 11 bits

// One block per tile (grid-stride).  fill = false: count[t] = distinct columns, or 0
// with fb[t] = 1 when the tile falls back; fill = true: list the columns from
// ptr[t] and the entries' positions.  Positions depend on the order of the atomic
// insertions; the SpMV's result does not (it sums in CSR order).
__global__ void __launch_bounds__(256) k_spt_build(const int32_t* __restrict__ rowptr, const int32_t* __restrict__ col,
                                                   int n, int ntiles, bool fill, int32_t* __restrict__ count,
                                                   uint8_t* __restrict__ fb, const int32_t* __restrict__ ptr,
                                                   int32_t* __restrict__ uniq, uint16_t* __restrict__ lidx) {
  __shared__ int32_t key[SPT_HASH];
  __shared__ int32_t pos[SPT_HASH];
  __shared__ int nu;
  for (int t = blockIdx.x; t < ntiles; t += gridDim.x) {
    const int r0 = t * SPT_ROWS, r1 = min(r0 + SPT_ROWS, n);
    const int k0 = rowptr[r0], k1 = rowptr[r1];
    const bool big = k1 - k0 > SPT_HASH / 2;  // keeps the table at most half full: every probe ends
    for (int i = threadIdx.x; i < SPT_HASH; i += blockDim.x) key[i] = -1;
    if (threadIdx.x == 0) nu = 0;
    __syncthreads();
    if (!big)
      for (int k = k0 + (int)threadIdx.x; k < k1; k += blockDim.x) {
        const int j = col[k];
        unsigned h = spt_hash(j);
        for (;;) {
          const int prev = atomicCAS(&key[h], -1, j);
          if (prev == -1) { pos[h] = atomicAdd(&nu, 1); break; }
          if (prev == j) break;
          h = (h + 1) & (SPT_HASH - 1);
        }
      }
    __syncthreads();
    const bool over = big || nu > SPT_UCAP;
    if (!fill) {
      if (threadIdx.x == 0) { count[t] = over ? 0 : nu; fb[t] = over ? 1 : 0; }
    } else if (!over) {
      const int u0 = ptr[t];
      for (int h = threadIdx.x; h < SPT_HASH; h += blockDim.x)
        if (key[h] >= 0) uniq[u0 + pos[h]] = key[h];
      for (int k = k0 + (int)threadIdx.x; k < k1; k += blockDim.x) {
        const int j = col[k];
        unsigned h = spt_hash(j);
        while (key[h] != j) h = (h + 1) & (SPT_HASH - 1);
        lidx[k] = (uint16_t)pos[h];
      }
    }
    __syncthreads();
  }
}

// 3 blocks of 256 threads per SM: 80 registers without spills, 3 x 48 KB of staged rows.
template <int NS>
__global__ void __launch_bounds__(256, 3)
    k_spmv_tile(const int32_t* __restrict__ rowptr, const int32_t* __restrict__ col,
                const double2* __restrict__ km, int n, const int32_t* __restrict__ sptr,
                const int32_t* __restrict__ suniq, const uint16_t* __restrict__ slidx,
                const uint8_t* __restrict__ sfb, int ntiles, const double2* __restrict__ p,
                double2* __restrict__ q, const SysScal* __restrict__ sc, const Ctrl* __restrict__ ctrl,
                double* __restrict__ part) {
  static_assert(NS == 16, "tiles hold 16 systems per row");
  constexpr int SPL = 2, LPR = NS / SPL;  // 8 lanes per row, 2 systems per lane, 4 rows per warp
  // SPT_UCAP rows x NS values; a row's system 2m + h sits at 8h + m, so the 8 lanes of
  // a row read its values for their first (second) systems as one 128-byte run
  extern __shared__ double2 sp[];
  if (ctrl && ctrl->done) return;
  const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5, sub = lane / LPR, ql = lane % LPR;
  const int s0 = ql * SPL;
  double acc[SPL][2];
#pragma unroll
  for (int i = 0; i < SPL; ++i) acc[i][0] = acc[i][1] = 0.0;
  for (int t = blockIdx.x; t < ntiles; t += gridDim.x) {
    const bool fb = __ldg(sfb + t) != 0;  // block-uniform
    if (!fb) {
      const int u0 = __ldg(sptr + t), nu = __ldg(sptr + t + 1) - u0;
      // piece i: 32 bytes (systems 2(i%8), +1) of the tile's column i/8; a thread's
      // pieces in groups of SPT_GROUP loads in flight, then their stores
#pragma unroll
      for (int m0 = 0; m0 < SPT_PIECES; m0 += SPT_GROUP) {
        double2 va[SPT_GROUP], vb[SPT_GROUP];
#pragma unroll
        for (int m = 0; m < SPT_GROUP; ++m) {
          const int i = (int)threadIdx.x + 256 * (m0 + m);
          if (m0 + m < SPT_PIECES && i < nu * 8) {
            const int j = __ldg(suniq + u0 + (i >> 3));
            ld_v4d<false, true>(p + (long)j * NS + (i & 7) * 2, va[m], vb[m]);
          }
        }
#pragma unroll
        for (int m = 0; m < SPT_GROUP; ++m) {
          const int i = (int)threadIdx.x + 256 * (m0 + m);
          if (m0 + m < SPT_PIECES && i < nu * 8) {
            sp[(i >> 3) * NS + (i & 7)] = va[m];
            sp[(i >> 3) * NS + 8 + (i & 7)] = vb[m];
          }
        }
      }
      __syncthreads();
    }
    const int row = t * SPT_ROWS + wib * 4 + sub;
    if (row < n) {
      const int k0 = __ldg(rowptr + row), k1 = __ldg(rowptr + row + 1);
      double t1x[SPL], t1y[SPL], t2x[SPL], t2y[SPL];
#pragma unroll
      for (int i = 0; i < SPL; ++i) t1x[i] = t1y[i] = t2x[i] = t2y[i] = 0.0;
      if (!fb) {
        int k = k0;
        for (; k + 1 < k1; k += 2) {
          const int l0 = __ldg(slidx + k), l1 = __ldg(slidx + k + 1);
          const double2 a0 = km[k], a1 = km[k + 1];
          const double2* v0 = sp + l0 * NS + ql;
          const double2* v1 = sp + l1 * NS + ql;
#pragma unroll
          for (int i = 0; i < SPL; ++i) {
            const double2 w0 = v0[8 * i], w1 = v1[8 * i];
            t1x[i] += a0.x * w0.x; t1y[i] += a0.x * w0.y; t2x[i] += a0.y * w0.x; t2y[i] += a0.y * w0.y;
            t1x[i] += a1.x * w1.x; t1y[i] += a1.x * w1.y; t2x[i] += a1.y * w1.x; t2y[i] += a1.y * w1.y;
          }
        }
        if (k < k1) {
          const int l0 = __ldg(slidx + k);
          const double2 a = km[k];
          const double2* v = sp + l0 * NS + ql;
#pragma unroll
          for (int i = 0; i < SPL; ++i) {
            const double2 w = v[8 * i];
            t1x[i] += a.x * w.x; t1y[i] += a.x * w.y; t2x[i] += a.y * w.x; t2y[i] += a.y * w.y;
          }
        }
      } else {
        row_gather_spl<double, NS, 1, SPL, true>(col, km, p, k0, k1, s0, t1x, t1y, t2x, t2y);
      }
      const long base = (long)row * NS + s0;
      double2 qi[SPL], own[SPL];
#pragma unroll
      for (int i = 0; i < SPL; ++i) {
        const double o = __ldg(&sc[s0 + i].omega);
        qi[i] = make_double2(t1x[i] - o * t2y[i], t1y[i] + o * t2x[i]);
      }
      load_spl<double2, NS, SPL, false, true>(p + base, own);
#pragma unroll
      for (int i = 0; i < SPL; ++i) {
        acc[i][0] += own[i].x * qi[i].x - own[i].y * qi[i].y;
        acc[i][1] += own[i].x * qi[i].y + own[i].y * qi[i].x;
      }
      store_spl<double2, SPL>(q + base, qi);
    }
    __syncthreads();  // the next tile overwrites the staged rows
  }
  block_partials_spl<NS, SPL, LPR, 2>(acc, s0, true, part);
}

// ------------------------------------------------------------------ scalar kernels
__device__ __forceinline__ void sum_partials(const double* part, int nblocks, int s, int k, double* out,
                                             int nvals) {
  // one warp per system; deterministic order
  __shared__ double sh[32][4];
  const int lane = threadIdx.x & 31;
  for (int v = 0; v < nvals; ++v) {
    double acc = 0.0;
    for (int b = lane; b < nblocks; b += 32) acc += part[((long)b * MAX_SYS + s) * 4 + k + v];
    for (int m = 16; m > 0; m >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, m);
    sh[threadIdx.x >> 5][v] = acc;
  }
  __syncwarp();
  for (int v = 0; v < nvals; ++v) out[v] = sh[threadIdx.x >> 5][v];
}

// defer_x (multicolour path): the sweep updated r only; x += alpha p of an active
// system is marked pending and applied by the p update of the same iteration,
// which also runs when this kernel ends the solve.
__global__ void k_scal_r(SysScal* sc, Ctrl* ctrl, const double* part, int nblocks, int ns, double* rms, int n,
                         int defer_x) {
  if (ctrl->done) {
    // the update pending when the solve ended was applied by that iteration's p update
    if (defer_x && threadIdx.x < ns) sc[threadIdx.x].xpend = 0;
    return;
  }
  const int s = threadIdx.x >> 5;
  bool finished = true;
  if (s < ns) {
    double rr;
    sum_partials(part, nblocks, s, 0, &rr, 1);
    if ((threadIdx.x & 31) == 0) {
      SysScal& S = sc[s];
      S.xpend = defer_x && S.active && ctrl->iter > 0;
      if (S.active) {
        S.rr = rr;
        if (rms) rms[s] = sqrt(rr / n) > 0.0 ? sqrt(rr / n) : 1.0;
        S.resid = sqrt(rr / S.bnrm2);
        if (ctrl->iter > 0) S.iter += 1;
        if (!isfinite(S.resid)) { S.active = 0; S.status = AFEM_ENONFINITE; }
        else if (S.resid <= ctrl->tol && ctrl->iter > 0) { S.active = 0; S.status = AFEM_OK; }
        else if (ctrl->iter >= ctrl->maxit) { S.active = 0; S.status = AFEM_EMAXITER; }
      }
    }
  }
  __syncthreads();
  __shared__ int any_active;
  if (threadIdx.x == 0) any_active = 0;
  __syncthreads();
  if (s < ns && (threadIdx.x & 31) == 0 && sc[s].active) atomicOr(&any_active, 1);
  __syncthreads();
  finished = !any_active;
  if (threadIdx.x == 0 && finished) ctrl->done = 1;
}

__device__ __forceinline__ double2 d_cdiv(double2 a, double2 b) { return cdiv(a, b); }

// part2 (nullable): the nodal correction's share r^T G u = t^T u of rho, summed by
// the backward nodal sweep when the gradient add is folded into the p update
__global__ void k_scal_rho(SysScal* sc, Ctrl* ctrl, const double* part, int nblocks, int ns, int flexible,
                           const double* part2, int nblocks2) {
  if (ctrl->done) return;
  const int s = threadIdx.x >> 5;
  if (s >= ns) return;
  double v[4];
  sum_partials(part, nblocks, s, 0, v, 4);
  if (part2) {
    double v2[2];
    __syncwarp();
    sum_partials(part2, nblocks2, s, 0, v2, 2);
    v[0] += v2[0];
    v[1] += v2[1];
  }
  if ((threadIdx.x & 31) == 0) {
    SysScal& S = sc[s];
    S.rho = make_double2(v[0], v[1]);
    if (S.active) {
      if (S.rho.x == 0.0 && S.rho.y == 0.0) { S.active = 0; S.status = AFEM_EBREAKDOWN; }
      else if (ctrl->iter > 0) {
        // flexible (Polak-Ribiere) form for a variable preconditioner: z^T (r_k+1 - r_k) / z_k^T r_k
        const double2 num = flexible ? make_double2(S.rho.x - v[2], S.rho.y - v[3]) : S.rho;
        S.beta = d_cdiv(num, S.rho1);
      }
    }
  }
}

__global__ void k_scal_pq(SysScal* sc, Ctrl* ctrl, const double* part, int nblocks, int ns) {
  if (ctrl->done) return;
  const int s = threadIdx.x >> 5;
  if (s < ns) {
    double v[2];
    sum_partials(part, nblocks, s, 0, v, 2);
    if ((threadIdx.x & 31) == 0) {
      SysScal& S = sc[s];
      S.pq = make_double2(v[0], v[1]);
      if (S.active) {
        if (S.pq.x == 0.0 && S.pq.y == 0.0) { S.active = 0; S.status = AFEM_EBREAKDOWN; S.alpha = make_double2(0, 0); }
        else S.alpha = d_cdiv(S.rho, S.pq);
        S.rho1 = S.rho;
      } else {
        S.alpha = make_double2(0.0, 0.0);
      }
    }
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    ctrl->iter += 1;
    ctrl->epoch += 1;
  }
}

// ------------------------------------------------------------------ preconditioner set-up
// SSOR / DIAG: DD_i = 1 / (sd * D_i) (COCG13_single.f90:126-130).
template <class T, int NS>
__global__ void k_dd_diag(const typename Cx<T>::V* __restrict__ km, const int32_t* __restrict__ diagpos, int n,
                          double sd, const SysScal* __restrict__ sc, typename Cx<T>::V* __restrict__ dd,
                          const uint8_t* __restrict__ seg) {
  const long total = (long)n * NS;
  for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < total; i += (long)gridDim.x * blockDim.x) {
    const int row = (int)(i / NS), s = seg ? (int)__ldg(seg + row) : (int)(i % NS);
    const double2 a = make_double2((double)km[diagpos[row]].x, (double)km[diagpos[row]].y);
    const double om = sc[s].omega;
    const double2 D = make_double2(sd * a.x, sd * om * a.y);
    const double2 w = cdiv(make_double2(1.0, 0.0), D);
    dd[i] = Cx<T>::make((T)w.x, (T)w.y);
  }
}

// IC: DD_i = 1 / (sd*D_i - sum_{k in L(i)} AL_k * AL_k * DD_col(k)) (COCG13_single.f90:107-124, SIGMA = 0).
template <class T, int NS>
__global__ void __launch_bounds__(256)
    k_dd_ic(const int32_t* __restrict__ rowptr, const int32_t* __restrict__ col, const int32_t* __restrict__ diagpos,
            const typename Cx<T>::V* __restrict__ km, int n, double sd, const SysScal* __restrict__ sc,
            typename Cx<T>::V* __restrict__ dd, unsigned* __restrict__ flag, const Ctrl* __restrict__ ctrl,
            DevStatus* st, const int32_t* __restrict__ perm, const uint8_t* __restrict__ seg) {
  using V = typename Cx<T>::V;
  constexpr int G = 32 / NS;
  const unsigned epoch = ctrl->epoch;
  const unsigned lim = ctrl->spin_limit ? ctrl->spin_limit : SPIN_LIMIT;
  const int lane = threadIdx.x & 31, s = lane % NS, g = lane / NS;
  const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int nwarps = (gridDim.x * blockDim.x) >> 5;
  double om = sc[s].omega;
  for (int pos = warp; pos < n; pos += nwarps) {
    const int row = __ldg(perm + pos);
    if (seg) om = sc[__ldg(seg + row)].omega;  // packed batch (NS = 1)
    const int k0 = rowptr[row], k1 = diagpos[row];
    double wx = 0, wy = 0;
    for (int k = k0 + g; k < k1; k += G) {
      const int j = col[k];
      const V a = km[k];
      if (!wait_flag(flag + j, epoch, st, row, lim)) break;
      const V d = ldcg(dd + (long)j * NS + s);
      const double2 al = make_double2((double)a.x, om * (double)a.y);
      const double2 a2 = cmul(al, al);
      const double2 t = cmul(a2, make_double2((double)d.x, (double)d.y));
      wx += t.x; wy += t.y;
    }
    for (int m = NS; m < 32; m <<= 1) {
      wx += __shfl_xor_sync(0xffffffffu, wx, m);
      wy += __shfl_xor_sync(0xffffffffu, wy, m);
    }
    if (g == 0) {
      const V a = km[diagpos[row]];
      const double2 W = make_double2(sd * (double)a.x - wx, sd * om * (double)a.y - wy);
      const double2 dv = cdiv(make_double2(1.0, 0.0), W);
      dd[(long)row * NS + s] = Cx<T>::make((T)dv.x, (T)dv.y);
    }
    __syncwarp();
    if (lane == 0) st_release(flag + row, epoch);  // release: the row's values are visible first
  }
}

// ------------------------------------------------------------------ helpers
template <class Vd, class Vs>
__global__ void k_convert(const Vs* __restrict__ in, Vd* __restrict__ out, long total);
template <>
__global__ void k_convert<float2, double2>(const double2* __restrict__ in, float2* __restrict__ out, long total) {
  for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < total; i += (long)gridDim.x * blockDim.x)
    out[i] = make_float2((float)in[i].x, (float)in[i].y);
}

__global__ void k_gather_rhs(const double2* __restrict__ rhs, int n, int ns, const int* __restrict__ src,
                             double2* __restrict__ b, const uint8_t* __restrict__ seg) {
  const long total = (long)n * ns;
  for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < total; i += (long)gridDim.x * blockDim.x) {
    const int row = (int)(i / ns), s = seg ? (int)seg[row] : (int)(i % ns);
    b[i] = rhs[(long)src[s] * n + row];
  }
}

__global__ void k_add_x(double2* __restrict__ x, const double2* __restrict__ dx, long total) {
  for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < total; i += (long)gridDim.x * blockDim.x)
    x[i] = make_double2(x[i].x + dx[i].x, x[i].y + dx[i].y);
}

template <class V>
__global__ void k_copy_r(const double2* __restrict__ in, V* __restrict__ out, long total);
template <>
__global__ void k_copy_r<double2>(const double2* __restrict__ in, double2* __restrict__ out, long total) {
  for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < total; i += (long)gridDim.x * blockDim.x)
    out[i] = in[i];
}
template <>
__global__ void k_copy_r<float2>(const double2* __restrict__ in, float2* __restrict__ out, long total) {
  for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < total; i += (long)gridDim.x * blockDim.x)
    out[i] = make_float2((float)in[i].x, (float)in[i].y);
}

// Start of an inner solve: x_inner = 0, ||b||^2 from the partials of the residual SpMV.
__global__ void k_init_sys(SysScal* sc, Ctrl* ctrl, const double* part, int nblocks, int ns, double tol, int maxit,
                           const double* omega, unsigned spin_limit) {
  const int s = threadIdx.x >> 5;
  if (s < ns) {
    double v[1];
    sum_partials(part, nblocks, s, 0, v, 1);
    if ((threadIdx.x & 31) == 0) {
      SysScal& S = sc[s];
      S.omega = omega[s];
      S.bnrm2 = v[0];
      S.rr = v[0];
      S.resid = 1.0;
      S.rho = S.rho1 = S.alpha = S.beta = S.pq = make_double2(0.0, 0.0);
      S.iter = 0;
      S.xpend = 0;
      // a NaN / Inf in the matrix or the right-hand side shows in ||b - A 0||^2
      const bool finite = isfinite(v[0]);
      S.active = finite && v[0] > 0.0;
      S.status = finite ? AFEM_OK : AFEM_ENONFINITE;
    }
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    ctrl->done = 0;
    ctrl->iter = 0;
    ctrl->tol = tol;
    ctrl->maxit = maxit;
    ctrl->spin_limit = spin_limit;
  }
}

// Residual norms after a true-residual SpMV: part[.][0] = ||b - Ax||^2, part[.][2] = ||b||^2.
__global__ void k_true_resid(const double* part, int nblocks, int ns, double* out /* 2*ns */) {
  const int s = threadIdx.x >> 5;
  if (s >= ns) return;
  double v[3];
  sum_partials(part, nblocks, s, 0, v, 3);
  if ((threadIdx.x & 31) == 0) {
    out[2 * s] = v[0];
    out[2 * s + 1] = v[2];
  }
}

}  // namespace

// ======================================================================== host side
namespace {

struct Launch {
  afem_ctx* c;
  SolverWork* w;
};

template <class K, class... Args>
void launch_coop(K kernel, int blocks, cudaStream_t s, Args... args) {
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3(blocks);
  cfg.blockDim = dim3(256);
  cfg.stream = s;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeCooperative;
  attr[0].val.cooperative = 1;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  AFEM_CUDA(cudaLaunchKernelEx(&cfg, kernel, args...));
  count_launch();
}

template <class K>
int coresident_blocks(K kernel, int num_sms) {
  int per_sm = 0;
  AFEM_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kernel, 256, 0));
  AFEM_REQUIRE(per_sm > 0, AFEM_ECUDA, "sweep kernel cannot be resident");
  return per_sm * num_sms;
}

template <class T, int NS>
struct Inner {
  using V = typename Cx<T>::V;
  static V* vec(SolverWork* w, int which);
};
template <int NS>
struct Inner<double, NS> {
  using V = double2;
  static V* R(SolverWork* w) { return w->r.p; }
  static V* Z(SolverWork* w) { return w->z.p; }
  static V* P(SolverWork* w) { return w->p.p; }
  static V* Q(SolverWork* w) { return w->q.p; }
  static V* DD(SolverWork* w) { return w->dd.p; }
  static V* RP(SolverWork* w) { return w->rprev.p; }
  static const V* KM(afem_ctx* c, SolverWork*) { return c->km.p; }
  static V* HT(SolverWork* w) { return w->ht.p; }
  static V* HY(SolverWork* w) { return w->hy.p; }
  static V* HDD(SolverWork* w) { return w->hdd.p; }
  static const V* HKM(afem_ctx* c) { return c->hyb->km.p; }
  static const V* HLKM(afem_ctx* c) { return c->hyb->lkm.p; }
  static const V* HUKM(afem_ctx* c) { return c->hyb->ukm.p; }
  static const V* LKM(afem_ctx* c, SolverWork*) { return c->mc_lkm.p; }
  static const V* UKM(afem_ctx* c, SolverWork*) { return c->mc_ukm.p; }
};
template <int NS>
struct Inner<float, NS> {
  using V = float2;
  static V* R(SolverWork* w) { return w->rf.p; }
  static V* Z(SolverWork* w) { return w->zf.p; }
  static V* P(SolverWork* w) { return w->pf.p; }
  static V* Q(SolverWork* w) { return w->qf.p; }
  static V* DD(SolverWork* w) { return w->ddf.p; }
  static V* RP(SolverWork* w) { return w->rprevf.p; }
  static const V* KM(afem_ctx*, SolverWork* w) { return w->kmf.p; }
  static V* HT(SolverWork* w) { return w->htf.p; }
  static V* HY(SolverWork* w) { return w->hyf.p; }
  static V* HDD(SolverWork* w) { return w->hddf.p; }
  static const V* HKM(afem_ctx* c) { return c->hyb->kmf.p; }
  static const V* HLKM(afem_ctx* c) { return c->hyb->lkmf.p; }
  static const V* HUKM(afem_ctx* c) { return c->hyb->ukmf.p; }
  static const V* LKM(afem_ctx*, SolverWork* w) { return w->mc_lkmf.p; }
  static const V* UKM(afem_ctx*, SolverWork* w) { return w->mc_ukmf.p; }
};

// Co-resident blocks of a kernel on this device (256 threads), at most `cap`: a
// persistent grid of that size runs in one wave with every block's slice of rows.
template <class K>
int one_wave_grid(afem_ctx* c, K kernel, int cap, size_t smem = 0) {
  int per_sm = 0;
  AFEM_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kernel, 256, smem));
  return std::max(1, std::min(cap, std::max(1, per_sm) * c->num_sms));
}

// The SpMV variants: rpw rows per warp with a lane per system (1, 2, 4), or, at 16
// systems, 8 rows per warp with 4 systems per lane (rpw = 8).  Returns the grid it
// used (the number of partial sums its consumer adds).
// Build the tiled SpMV's column lists once per pattern (two passes of k_spt_build:
// count, scan, fill).  Synchronises the stream; called before any graph capture.
void ensure_spmv_tiles(afem_ctx* c) {
  if (c->spt_ready) return;
  cudaStream_t s = c->stream;
  const int n = c->nline;
  const int ntiles = (n + SPT_ROWS - 1) / SPT_ROWS;
  c->spt_ptr.alloc(ntiles + 1);
  c->spt_fb.alloc(ntiles);
  DBuf<int32_t> cnt;
  cnt.alloc(ntiles);
  const int grid = std::max(1, std::min(ntiles, c->num_sms * 8));
  k_spt_build<<<grid, 256, 0, s>>>(c->rowptr.p, c->col.p, n, ntiles, false, cnt.p, c->spt_fb.p, nullptr, nullptr,
                                   nullptr);
  count_launch();
  long total = 0;
  exclusive_scan(cnt.p, c->spt_ptr.p, ntiles, s, &total);
  c->spt_uniq.alloc(std::max(1L, total));
  c->spt_lidx.alloc(std::max(1L, c->nnz));
  k_spt_build<<<grid, 256, 0, s>>>(c->rowptr.p, c->col.p, n, ntiles, true, nullptr, c->spt_fb.p, c->spt_ptr.p,
                                   c->spt_uniq.p, c->spt_lidx.p);
  count_launch();
  AFEM_CUDA(cudaStreamSynchronize(s));
  c->spt_ntiles = ntiles;
  c->spt_ready = true;
}

template <class T, int NS, bool SEG>
int launch_spmv(afem_ctx* c, SolverWork* w, int rpw, const typename Cx<T>::V* km, const typename Cx<T>::V* p,
                typename Cx<T>::V* q, const Ctrl* ctrl, const typename Cx<T>::V* bvec) {
  cudaStream_t s = c->stream;
  const int n = w->n;
  const int32_t* rp = c->rowptr.p;
  const int32_t* cl = c->col.p;
  const uint8_t* sg = SEG ? c->seg_of_row.p : nullptr;
  const int vi = rpw == 16 ? 4 : rpw == 8 ? 3 : rpw == 4 ? 2 : rpw == 2 ? 1 : 0;
  int& grid = w->spmv_grid[sizeof(T) == 8 ? 0 : 1][vi];
  if constexpr (NS == 16 && !SEG && sizeof(T) == 8) {
    if (rpw == 16 && !bvec) {  // tiles staged in shared memory (built by ensure_spmv_tiles)
      AFEM_REQUIRE(c->spt_ready, AFEM_ESTATE, "SpMV: tiles not built");
      auto k = k_spmv_tile<NS>;
      constexpr size_t smem = sizeof(double2) * SPT_UCAP * NS;
      if (!grid) {
        AFEM_CUDA(cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
        grid = one_wave_grid(c, k, w->nblocks, smem);
      }
      k<<<grid, 256, smem, s>>>(rp, cl, (const double2*)km, n, c->spt_ptr.p, c->spt_uniq.p, c->spt_lidx.p,
                                c->spt_fb.p, c->spt_ntiles, (const double2*)p, (double2*)q, w->sc.p, ctrl, w->part.p);
      count_launch();
      return grid;
    }
  }
  if constexpr (NS == 16 && !SEG) {
    if (rpw == 8 && !bvec) {  // AFEM_MC_SPL systems per lane, 2 * AFEM_MC_SPL rows per warp (q = A p only)
      auto k = k_spmv<T, NS, 2 * AFEM_MC_SPL, SEG, AFEM_MC_SPL>;
      if (!grid) grid = one_wave_grid(c, k, w->nblocks);
      k<<<grid, 256, 0, s>>>(rp, cl, km, n, p, q, w->sc.p, ctrl, w->part.p, bvec, sg);
      count_launch();
      return grid;
    }
  }
  if (rpw == 4 && NS * 4 <= 32) {
    auto k = k_spmv<T, NS, (NS * 4 <= 32 ? 4 : 1), SEG>;
    if (!grid) grid = one_wave_grid(c, k, w->nblocks);
    k<<<grid, 256, 0, s>>>(rp, cl, km, n, p, q, w->sc.p, ctrl, w->part.p, bvec, sg);
  } else if (rpw == 2 && NS * 2 <= 32) {
    auto k = k_spmv<T, NS, (NS * 2 <= 32 ? 2 : 1), SEG>;
    if (!grid) grid = one_wave_grid(c, k, w->nblocks);
    k<<<grid, 256, 0, s>>>(rp, cl, km, n, p, q, w->sc.p, ctrl, w->part.p, bvec, sg);
  } else {
    auto k = k_spmv<T, NS, 1, SEG>;
    if (!grid) grid = one_wave_grid(c, k, w->nblocks);
    k<<<grid, 256, 0, s>>>(rp, cl, km, n, p, q, w->sc.p, ctrl, w->part.p, bvec, sg);
  }
  count_launch();
  return grid;
}

// Rows-per-warp autotuner: times each variant on this matrix (q = A p with the
// current p) in three interleaved rounds and keeps the fastest by its best
// round (one round alone flipped between close variants from run to run);
// cached per workspace and precision.
template <class T, int NS, bool SEG>
int tune_spmv(afem_ctx* c, SolverWork* w) {
  using I = Inner<T, NS>;
  int& slot = sizeof(T) == 8 ? w->rpw64 : w->rpw32;
  if (slot) return slot;
  auto valid = [](int rpw) {
    return rpw == 16 ? (NS == 16 && !SEG && sizeof(T) == 8) : rpw == 8 ? (NS == 16 && !SEG) : NS * rpw <= 32;
  };
  // the tiles are built here, outside any graph capture (the build synchronises); the
  // tiled variant is only run when pinned: on these meshes it is slower than two
  // systems per lane (2.24 against 1.69 ms on the 96x96x64 batch), so the tuner skips it
  if (valid(16) && c->spmv_rpw == 16) ensure_spmv_tiles(c);
  if (c->spmv_rpw > 0) {  // pinned by the caller: the same reduction order in every process
    slot = valid(c->spmv_rpw) ? c->spmv_rpw : 1;
    return slot;
  }
  cudaStream_t s = c->stream;
  cudaEvent_t a, b;
  AFEM_CUDA(cudaEventCreate(&a));
  AFEM_CUDA(cudaEventCreate(&b));
  const int cand[4] = {1, 2, 4, 8};
  float tbest[4] = {1e30f, 1e30f, 1e30f, 1e30f};
  for (int round = 0; round < 3; ++round)
    for (int ci = 0; ci < 4; ++ci) {
      const int rpw = cand[ci];
      if (!valid(rpw)) continue;
      launch_spmv<T, NS, SEG>(c, w, rpw, I::KM(c, w), I::P(w), I::Q(w), nullptr, nullptr);  // warm
      AFEM_CUDA(cudaEventRecord(a, s));
      for (int k = 0; k < 3; ++k) launch_spmv<T, NS, SEG>(c, w, rpw, I::KM(c, w), I::P(w), I::Q(w), nullptr, nullptr);
      AFEM_CUDA(cudaEventRecord(b, s));
      AFEM_CUDA(cudaEventSynchronize(b));
      float ms = 0;
      AFEM_CUDA(cudaEventElapsedTime(&ms, a, b));
      tbest[ci] = std::min(tbest[ci], ms);
    }
  float best = 1e30f;
  int pick = 1;
  for (int ci = 0; ci < 4; ++ci)
    if (tbest[ci] < best * 0.97f) { best = tbest[ci]; pick = cand[ci]; }
  cudaEventDestroy(a);
  cudaEventDestroy(b);
  slot = pick;
  return pick;
}

// One COCG iteration (7 launches; the learned preconditioner adds the network's 8).
// T: COCG vectors and the SpMV; PT: the multicolour preconditioner (its matrix
// copies and vectors); PT differs from T only on the multicolour path.
template <class T, class PT, int NS, bool SEG>
void enqueue_iteration(afem_ctx* c, SolverWork* w, int mode, int sweep_blocks, cudaEvent_t* ev) {
  using I = Inner<T, NS>;
  using P = Inner<PT, NS>;
  using V = typename I::V;
  using PV = typename P::V;
  constexpr bool same = std::is_same<T, PT>::value;
  cudaStream_t s = c->stream;
  const int n = w->n;
  const int nsys = w->nsys;
  const uint8_t* sg = SEG ? c->seg_of_row.p : nullptr;
  const bool learned = mode == AFEM_PRECOND_LEARNED;
  V* rp = learned ? I::RP(w) : nullptr;
  // the learned network either replaces the preconditioner (Jacobi base) or adds its
  // correction to the gradient-corrected SSOR (hybrid base): z = H(r) + N(r)
  const bool lbase = learned && mpnn_base(c) == 1;
  const bool hyb = mode == AFEM_PRECOND_HYBRID || lbase;
  const bool mc = mode == AFEM_PRECOND_SSOR_MC || hyb;  // the hybrid's edge part is the multicolour SSOR
  // hybrid alone (one matrix): z + G u is formed inside the p update, and the
  // backward nodal sweep sums t^T u, the nodal share of rho
  const bool fold_grad = hyb && !lbase && !SEG;
  if (ev) AFEM_CUDA(cudaEventRecord(ev[0], s));
  if (mc) {  // the multicolour sweep updates r only: x += alpha p moves to the p update
    launch_coop(k_fwd_mc<T, PT, NS, SEG>, w->mc_blocks, s, (const int32_t*)c->mc_lptr.p,
                (const int32_t*)c->mc_lcol.p, P::LKM(c, w), n, I::R(w), P::Z(w), (const V*)I::Q(w),
                (const double2*)c->mc_dkm.p, w->sd, (const int32_t*)c->perm_mc.p, (const int32_t*)c->color_ptr.p,
                c->ncolors, w->sc.p, w->ctrl.p, w->part.p, sg, rp);
  } else if constexpr (same) {
    launch_coop(k_fwd<T, NS, SEG>, sweep_blocks, s, (const int32_t*)c->rowptr.p, (const int32_t*)c->col.p,
                (const int32_t*)c->diagpos.p, I::KM(c, w), n, I::R(w), I::Z(w), (const V*)I::P(w), (const V*)I::Q(w),
                w->x.p, (const V*)I::DD(w), w->flag_f.p, mode, w->sc.p, w->ctrl.p, w->part.p, c->status.p, rp,
                (const int32_t*)c->perm_f.p, sg);
  }
  if (ev) AFEM_CUDA(cudaEventRecord(ev[1], s));
  const int swb = mc ? w->mc_blocks : sweep_blocks;
  k_scal_r<<<1, 32 * MAX_SYS, 0, s>>>(w->sc.p, w->ctrl.p, w->part.p, swb, nsys, learned ? w->rms.p : nullptr, n,
                                      mc ? 1 : 0);
  count_launch();
  if constexpr (same)
    if (learned && !lbase) mpnn_run<V>(c, NS, w->rms.p, (const V*)I::R(w), I::Z(w), &w->ctrl.p->done);
  if (ev) AFEM_CUDA(cudaEventRecord(ev[2], s));
  if (mc) {
    launch_coop(k_bwd_mc<T, PT, NS, SEG>, w->mcb_blocks, s, (const int32_t*)c->mc_uptr.p,
                (const int32_t*)c->mc_ucol.p, P::UKM(c, w), n, (const V*)I::R(w), P::Z(w),
                (const int32_t*)c->perm_mc.p, (const int32_t*)c->color_ptr.p, c->ncolors, w->sc.p, w->ctrl.p,
                w->part.p, sg, (const double2*)c->mc_dkm.p, w->sd);
  } else if constexpr (same) {
    launch_coop(k_bwd<T, NS, SEG>, sweep_blocks, s, (const int32_t*)c->rowptr.p, (const int32_t*)c->col.p,
                (const int32_t*)c->diagpos.p, I::KM(c, w), n, (const V*)I::R(w), I::Z(w), (const V*)I::DD(w),
                w->flag_b.p, mode, w->sc.p, w->ctrl.p, w->part.p, c->status.p, (const V*)rp,
                (const int32_t*)c->perm_b.p, sg);
  }
  if (ev) AFEM_CUDA(cudaEventRecord(ev[3], s));
  int rho_blocks = mc ? w->mcb_blocks : sweep_blocks;
  if (hyb) {
    // z += G SSOR_node(G^T r): folded into the p update, or (packed batches, learned
    // base) a pass of its own that takes the rho partials again from the corrected z
    HybridState* h = c->hyb;
    const int node = h->node;
    const uint8_t* hs = SEG ? h->seg.p : nullptr;
    k_grad_t<T, PT, NS><<<c->num_sms * 8, 256, 0, s>>>(node, h->nptr.p, h->nlist.p, c->bc.p, (const V*)I::R(w),
                                                        P::HT(w), w->ctrl.p);
    count_launch();
    for (int bwd = 0; bwd < 2; ++bwd)
      launch_coop(k_nsweep_mc<PT, NS, SEG>, w->nmc_blocks, s, (const int32_t*)(bwd ? h->uptr.p : h->lptr.p),
                  (const int32_t*)(bwd ? h->ucol.p : h->lcol.p), bwd ? P::HUKM(c) : P::HLKM(c),
                  (const PV*)P::HT(w), P::HY(w), (const PV*)P::HDD(w), (const int32_t*)h->perm.p,
                  (const int32_t*)h->cptr.p, h->ncolors, (const SysScal*)w->sc.p, (const Ctrl*)w->ctrl.p, hs, bwd,
                  (fold_grad && bwd) ? w->part2.p : (double*)nullptr);
    if (!fold_grad) {
      k_grad_add<T, PT, NS, SEG><<<w->nblocks, 256, 0, s>>>(n, c->line.p, c->bc.p, (const PV*)P::HY(w), P::Z(w),
                                                              (const V*)I::R(w), w->ctrl.p, w->part.p, sg);
      count_launch();
      rho_blocks = w->nblocks;
    }
  }
  if constexpr (same)
    if (lbase) {
      // z += N(r), then rho = r^T z and rprev^T z of the final z for the flexible beta
      mpnn_run<V>(c, NS, w->rms.p, (const V*)I::R(w), I::Z(w), &w->ctrl.p->done);
      k_dots<T, NS><<<w->nblocks, 256, 0, s>>>(n, (const V*)I::R(w), (const V*)I::Z(w), (const V*)rp, w->ctrl.p,
                                               w->part.p);
      count_launch();
      rho_blocks = w->nblocks;
    }
  if (ev) AFEM_CUDA(cudaEventRecord(ev[4], s));
  k_scal_rho<<<1, 32 * MAX_SYS, 0, s>>>(w->sc.p, w->ctrl.p, w->part.p, rho_blocks, nsys, learned ? 1 : 0,
                                        fold_grad ? w->part2.p : (const double*)nullptr, w->nmc_blocks);
  count_launch();
  if (ev) AFEM_CUDA(cudaEventRecord(ev[5], s));
  if constexpr (NS == 16 && !SEG)
    k_pupd_spl<T, PT, NS><<<c->num_sms * 8, 256, 0, s>>>(
        n, (const PV*)P::Z(w), I::P(w), w->sc.p, w->ctrl.p, mc ? w->x.p : (double2*)nullptr, nsys,
        fold_grad ? (const int32_t*)c->line.p : (const int32_t*)nullptr,
        fold_grad ? c->bc.p : (const uint8_t*)nullptr, fold_grad ? (const PV*)P::HY(w) : (const PV*)nullptr);
  else
    k_pupd<T, PT, NS, SEG><<<c->num_sms * 8, 256, 0, s>>>(
        n, (const PV*)P::Z(w), I::P(w), w->sc.p, w->ctrl.p, sg, mc ? w->x.p : (double2*)nullptr, nsys,
        fold_grad ? (const int32_t*)c->line.p : (const int32_t*)nullptr, fold_grad ? c->bc.p : (const uint8_t*)nullptr,
        fold_grad ? (const PV*)P::HY(w) : (const PV*)nullptr);
  count_launch();
  if (ev) AFEM_CUDA(cudaEventRecord(ev[6], s));
  const int spmv_grid = launch_spmv<T, NS, SEG>(c, w, sizeof(T) == 8 ? w->rpw64 : w->rpw32, I::KM(c, w),
                                                (const V*)I::P(w), I::Q(w), w->ctrl.p, (const V*)nullptr);
  if (ev) AFEM_CUDA(cudaEventRecord(ev[7], s));
  k_scal_pq<<<1, 32 * MAX_SYS, 0, s>>>(w->sc.p, w->ctrl.p, w->part.p, spmv_grid, nsys);
  count_launch();
}

// FP64 true residual r64 = b - A x; returns per-system ||r||^2 and ||b||^2 on the host.
template <int NS, bool SEG>
void true_residual(afem_ctx* c, SolverWork* w, std::vector<double>& rr, std::vector<double>& bb) {
  cudaStream_t s = c->stream;
  const int nsys = w->nsys;
  k_spmv<double, NS, 1, SEG><<<w->nblocks, 256, 0, s>>>((const int32_t*)c->rowptr.p, (const int32_t*)c->col.p, c->km.p,
                                                        w->n, w->x.p, w->r64.p, w->sc.p, (const Ctrl*)nullptr,
                                                        w->part.p, w->b.p, SEG ? c->seg_of_row.p : nullptr);
  count_launch();
  DBuf<double> out;
  out.alloc(2 * nsys);
  k_true_resid<<<1, 32 * MAX_SYS, 0, s>>>(w->part.p, w->nblocks, nsys, out.p);
  count_launch();
  std::vector<double> h(2 * nsys);
  out.download(h.data(), 2 * nsys, s);
  AFEM_CUDA(cudaStreamSynchronize(s));
  rr.resize(nsys);
  bb.resize(nsys);
  for (int k = 0; k < nsys; ++k) { rr[k] = h[2 * k]; bb[k] = h[2 * k + 1]; }
}

// DD of the natural-order sweeps (IC, SSOR, DIAG) in the COCG type T; the
// multicolour sweeps compute theirs from the diagonal, and the hybrid's nodal
// diagonal goes to the preconditioner type PT.
template <class T, class PT, int NS, bool SEG>
void setup_dd(afem_ctx* c, SolverWork* w, int precond, double sd) {
  using I = Inner<T, NS>;
  using P = Inner<PT, NS>;
  cudaStream_t s = c->stream;
  const uint8_t* sg = SEG ? c->seg_of_row.p : nullptr;
  if (precond == AFEM_PRECOND_IC) {
    // fresh epoch for the set-up recurrence
    w->epoch_host += 1;
    AFEM_CUDA(cudaMemcpyAsync(&w->ctrl.p->epoch, &w->epoch_host, sizeof(unsigned), cudaMemcpyHostToDevice, s));
    const int blocks = coresident_blocks(k_dd_ic<T, NS>, c->num_sms);
    launch_coop(k_dd_ic<T, NS>, blocks, s, (const int32_t*)c->rowptr.p, (const int32_t*)c->col.p,
                (const int32_t*)c->diagpos.p, I::KM(c, w), w->n, sd, (const SysScal*)w->sc.p, I::DD(w), w->flag_f.p,
                (const Ctrl*)w->ctrl.p, c->status.p, (const int32_t*)c->perm_f.p, sg);
    w->epoch_host += 1;
    AFEM_CUDA(cudaMemcpyAsync(&w->ctrl.p->epoch, &w->epoch_host, sizeof(unsigned), cudaMemcpyHostToDevice, s));
  } else if (precond == AFEM_PRECOND_SSOR || precond == AFEM_PRECOND_DIAG) {
    k_dd_diag<T, NS><<<c->num_sms * 8, 256, 0, s>>>(I::KM(c, w), (const int32_t*)c->diagpos.p, w->n, sd,
                                                    (const SysScal*)w->sc.p, I::DD(w), sg);
    count_launch();
  }
  if (precond == AFEM_PRECOND_HYBRID) {
    HybridState* h = c->hyb;
    k_dd_node<PT, NS><<<c->num_sms * 8, 256, 0, s>>>(h->km.p, h->diagpos.p, h->live.p, h->node,
                                                     (const SysScal*)w->sc.p, P::HDD(w), SEG ? h->seg.p : nullptr);
    count_launch();
  }
}

// Inner COCG from x_inner = 0 on right-hand side r64 (FP64, converted to T).
// Returns iterations; fills per-system status/resid.
template <class T, class PT, int NS, bool SEG>
int inner_cocg(afem_ctx* c, SolverWork* w, const afem_solve_opts* o, int precond, double tol, int maxit,
               int check_every, const double* d_omega, std::vector<SysScal>& hs, bool* stalled) {
  using I = Inner<T, NS>;
  cudaStream_t s = c->stream;
  const int n = w->n;
  const int nsys = w->nsys;
  const long total = (long)n * NS;
  // r = rhs (as T), x = 0, ||b||^2
  k_copy_r<typename I::V><<<c->num_sms * 8, 256, 0, s>>>(w->r64.p, I::R(w), total);
  count_launch();
  // ||r64||^2 via partials of a dedicated pass
  {
    // reuse SpMV-with-b path on x = 0: part[0] = ||b||^2
    AFEM_CUDA(cudaMemsetAsync(w->x.p, 0, sizeof(double2) * total, s));
    k_spmv<double, NS, 1, SEG><<<w->nblocks, 256, 0, s>>>((const int32_t*)c->rowptr.p, (const int32_t*)c->col.p,
                                                          c->km.p, n, w->x.p, w->q.p, w->sc.p, (const Ctrl*)nullptr,
                                                          w->part.p, w->r64.p, SEG ? c->seg_of_row.p : nullptr);
    count_launch();
  }
  k_init_sys<<<1, 32 * MAX_SYS, 0, s>>>(w->sc.p, w->ctrl.p, w->part.p, w->nblocks, nsys, tol, maxit, d_omega,
                                       c->wait_limit);
  count_launch();
  const bool use_hyb = precond == AFEM_PRECOND_HYBRID || (precond == AFEM_PRECOND_LEARNED && mpnn_base(c) == 1);
  if (use_hyb) {
    HybridState* h = c->hyb;
    const long nt = (long)h->node * NS;
    if (sizeof(PT) == 8) {
      w->ht.alloc(nt); w->hy.alloc(nt); w->hdd.alloc(nt);
    } else {
      w->htf.alloc(nt); w->hyf.alloc(nt); w->hddf.alloc(nt);
      if (!h->kmf_valid || h->kmf.n != (size_t)h->nnz) {
        h->kmf.alloc(h->nnz);
        k_convert<float2, double2><<<c->num_sms * 8, 256, 0, s>>>(h->km.p, h->kmf.p, h->nnz);
        count_launch();
        h->lkmf.alloc(h->lkm.n);
        h->ukmf.alloc(h->ukm.n);
        if (h->lkm.n) {
          k_convert<float2, double2><<<c->num_sms * 8, 256, 0, s>>>(h->lkm.p, h->lkmf.p, (long)h->lkm.n);
          count_launch();
        }
        if (h->ukm.n) {
          k_convert<float2, double2><<<c->num_sms * 8, 256, 0, s>>>(h->ukm.p, h->ukmf.p, (long)h->ukm.n);
          count_launch();
        }
        h->kmf_valid = true;
      }
    }
  }
  w->sd = o->sigma_diag > 0 ? o->sigma_diag : 1.0;
  setup_dd<T, PT, NS, SEG>(c, w, use_hyb ? AFEM_PRECOND_HYBRID : precond, w->sd);
  const int mode = precond;
  {
    HostTimer ht(c, "host_setup_spmv_tuner");
    tune_spmv<T, NS, SEG>(c, w);
  }
  const bool learned = mode == AFEM_PRECOND_LEARNED;
  if (learned) {
    using V = typename I::V;
    if (sizeof(V) == 8) w->rprevf.alloc(total); else w->rprev.alloc(total);
    w->rms.alloc(NS);
    mpnn_prepare(c, NS, d_omega);
  }
  if (stalled) *stalled = false;
  double watch = 1e300, win_min = 1e300;  // stagnation windows (see below)
  const int sweep_blocks = coresident_blocks(k_fwd<T, NS, SEG>, c->num_sms);
  const int sb2 = coresident_blocks(k_bwd<T, NS, SEG>, c->num_sms);
  const int sblocks = std::min(std::min(sweep_blocks, sb2), w->nblocks);
  if (mode == AFEM_PRECOND_SSOR_MC || use_hyb) {
    w->mc_blocks = std::min(coresident_blocks(k_fwd_mc<T, PT, NS, SEG>, c->num_sms), w->nblocks);
    w->mcb_blocks = std::min(coresident_blocks(k_bwd_mc<T, PT, NS, SEG>, c->num_sms), w->nblocks);
  }
  if (use_hyb)
    w->nmc_blocks = std::min(coresident_blocks(k_nsweep_mc<PT, NS, SEG>, c->num_sms), w->nblocks);
  // every solve starts a fresh flag generation: a solve that stopped inside a
  // chunk left its last forward-sweep flags at the epoch it ended on
  w->epoch_host += 1;
  AFEM_CUDA(cudaMemcpyAsync(&w->ctrl.p->epoch, &w->epoch_host, sizeof(unsigned), cudaMemcpyHostToDevice, s));
  int iters_done = 0;
  const int chunk = check_every > 0 ? check_every : 32;
  // profiling: 8 events per iteration of a chunk (fwd | scal | bwd | nodal correction | scal | pupd | spmv)
  const bool prof = c->prof.on;
  std::vector<cudaEvent_t> evs;
  if (prof) {
    evs.resize(8L * chunk);
    for (auto& e : evs) AFEM_CUDA(cudaEventCreate(&e));
  }
  auto ev_of = [&](int k) -> cudaEvent_t* { return prof ? &evs[8L * k] : nullptr; };
  cudaGraphExec_t gexec = nullptr;
  long graph_kernels = 0;  // kernel nodes of the captured chunk (launch count per graph launch)
  bool use_graph = o->use_graph != 0 && !prof;
  if (use_graph) {
    cudaGraph_t graph = nullptr;
    cudaError_t e = cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal);
    if (e == cudaSuccess) {
      bool ok = true;
      g_capturing = 1;
      try {
        for (int k = 0; k < chunk; ++k) enqueue_iteration<T, PT, NS, SEG>(c, w, mode, sblocks, ev_of(k));
      } catch (const Error&) {
        ok = false;
      }
      g_capturing = 0;
      e = cudaStreamEndCapture(s, &graph);
      if (ok && e == cudaSuccess && graph) {
        if (cudaGraphInstantiate(&gexec, graph, 0) != cudaSuccess) gexec = nullptr;
        size_t nn = 0;
        if (gexec && cudaGraphGetNodes(graph, nullptr, &nn) == cudaSuccess && nn > 0) {
          std::vector<cudaGraphNode_t> nodes(nn);
          if (cudaGraphGetNodes(graph, nodes.data(), &nn) == cudaSuccess)
            for (size_t k = 0; k < nn; ++k) {
              cudaGraphNodeType t;
              if (cudaGraphNodeGetType(nodes[k], &t) == cudaSuccess && t == cudaGraphNodeTypeKernel) ++graph_kernels;
            }
        }
      }
      if (graph) cudaGraphDestroy(graph);
    }
    cudaGetLastError();
    if (!gexec) use_graph = false;
  }
  int iter_before = 0;
  // On an error inside the loop (a device status such as a wait timeout, a CUDA
  // error) the graph and events are released and the host's flag epoch is brought
  // up to the device's, so that the next solve's epoch is above every flag written.
  struct LoopGuard {
    SolverWork* w;
    cudaStream_t s;
    cudaGraphExec_t* g;
    std::vector<cudaEvent_t>* evs;
    bool armed = true;
    ~LoopGuard() {
      if (!armed) return;
      if (*g) cudaGraphExecDestroy(*g);
      for (auto& e : *evs) cudaEventDestroy(e);
      if (cudaMemcpyAsync(w->h_ctrl, w->ctrl.p, sizeof(Ctrl), cudaMemcpyDeviceToHost, s) == cudaSuccess &&
          cudaStreamSynchronize(s) == cudaSuccess)
        w->epoch_host = std::max(w->epoch_host, w->h_ctrl->epoch);
      cudaGetLastError();
    }
  } guard{w, s, &gexec, &evs};
  // every chunk either advances the iteration count or ends the solve; the
  // chunk budget is a host-side backstop against a device state that does neither
  const long chunk_budget = (long)maxit / chunk + 4;
  for (long nchunk = 0;; ++nchunk) {
    AFEM_REQUIRE(nchunk < chunk_budget, AFEM_ESTATE, "COCG: inner solve made no progress");
    if (use_graph) {
      AFEM_CUDA(cudaGraphLaunch(gexec, s));
      count_launch(graph_kernels);
    } else {
      for (int k = 0; k < chunk; ++k) enqueue_iteration<T, PT, NS, SEG>(c, w, mode, sblocks, ev_of(k));
    }
    AFEM_CUDA(cudaMemcpyAsync(w->h_ctrl, w->ctrl.p, sizeof(Ctrl), cudaMemcpyDeviceToHost, s));
    AFEM_CUDA(cudaStreamSynchronize(s));
    check_status(c, "COCG iteration");
    if (prof) {
      // count only iterations that ran to their last kernel
      const int executed = std::min(chunk, w->h_ctrl->iter - iter_before);
      const char* tag = sizeof(T) == 8 ? (sizeof(PT) == 8 ? "fp64" : "fp64pc32") : "fp32";
      char nf[64], nb[64], nh[64], np_[64], ns_[64];
      const char* kind = SEG ? "seg" : "ns";
      const int cnt = SEG ? nsys : NS;
      const bool mcs = mode == AFEM_PRECOND_SSOR_MC || use_hyb;
      snprintf(nf, sizeof nf, "cocg_fwd_sweep%s_%s_%s%d", mcs ? "_mc" : "", tag, kind, cnt);
      snprintf(nb, sizeof nb, "cocg_bwd_sweep%s_%s_%s%d", mcs ? "_mc" : "", tag, kind, cnt);
      snprintf(nh, sizeof nh, "cocg_nodal_correction_%s_%s%d", tag, kind, cnt);
      snprintf(np_, sizeof np_, "cocg_p_update_%s_%s%d", tag, kind, cnt);
      snprintf(ns_, sizeof ns_, "cocg_spmv_%s_%s%d_rpw%d", tag, kind, cnt, sizeof(T) == 8 ? w->rpw64 : w->rpw32);
      for (int k = 0; k < executed; ++k) {
        float a = 0, b = 0, h = 0, d = 0, e = 0;
        cudaEvent_t* E = &evs[8L * k];
        if (cudaEventElapsedTime(&a, E[0], E[1]) != cudaSuccess || cudaEventElapsedTime(&b, E[2], E[3]) != cudaSuccess ||
            cudaEventElapsedTime(&h, E[3], E[4]) != cudaSuccess || cudaEventElapsedTime(&d, E[5], E[6]) != cudaSuccess ||
            cudaEventElapsedTime(&e, E[6], E[7]) != cudaSuccess) {
          cudaGetLastError();
          continue;
        }
        c->prof.add(nf, a);
        c->prof.add(nb, b);
        if (use_hyb) c->prof.add(nh, h);
        c->prof.add(np_, d);
        c->prof.add(ns_, e);
      }
    }
    iter_before = w->h_ctrl->iter;
    if (w->h_ctrl->done) break;
    // stagnation detector: the smallest worst-system residual seen in a window
    // of `win` chunks (learned: 4, FP32 inner: 16) must be 10% below
    // the previous window's, else the inner solve ends and the refinement /
    // fallback loop takes over (COCG residuals oscillate: windows, not samples)
    // FP64 inner solves get a long window (64 chunks, 2048 iterations): on the
    // air-dominated systems the recursive residual can flatten out near 1e-7,
    // and a restart from the true residual resumes the descent
    const int win = learned ? 4 : (sizeof(T) == 4 ? 16 : 64);
    if (!w->no_window) {
      AFEM_CUDA(cudaMemcpyAsync(w->h_sc, w->sc.p, sizeof(SysScal) * nsys, cudaMemcpyDeviceToHost, s));
      AFEM_CUDA(cudaStreamSynchronize(s));
      double worst = 0.0;
      for (int k = 0; k < nsys; ++k)
        if (w->h_sc[k].active) worst = std::max(worst, w->h_sc[k].resid);
      win_min = std::min(win_min, worst);
      if ((w->h_ctrl->iter / chunk) % win == 0) {
        if (!(win_min < 0.9 * watch) && watch < 1e300) {
          const int one = 1;
          AFEM_CUDA(cudaMemcpyAsync(&w->ctrl.p->done, &one, sizeof(int), cudaMemcpyHostToDevice, s));
          AFEM_CUDA(cudaStreamSynchronize(s));
          if (stalled) *stalled = true;
          break;
        }
        watch = win_min;
        win_min = 1e300;
      }
    }
  }
  guard.armed = false;
  if (gexec) cudaGraphExecDestroy(gexec);
  for (auto& e : evs) cudaEventDestroy(e);
  w->epoch_host = w->h_ctrl->epoch;
  hs.resize(nsys);
  AFEM_CUDA(cudaMemcpyAsync(w->h_sc, w->sc.p, sizeof(SysScal) * nsys, cudaMemcpyDeviceToHost, s));
  AFEM_CUDA(cudaStreamSynchronize(s));
  for (int k = 0; k < nsys; ++k) hs[k] = w->h_sc[k];
  iters_done = 0;
  for (int k = 0; k < nsys; ++k) iters_done = std::max(iters_done, hs[k].iter);
  return iters_done;
}

// The solve workspace for NS systems per row (SEG: a packed batch), FP32 copies when mixed.
template <int NS, bool SEG>
SolverWork* ensure_work(afem_ctx* c, int nsys, bool mixed, bool pc32 = false) {
  SolverWork* w = c->work;
  cudaStream_t s = c->stream;
  const int n = c->nline;
  const long total = (long)n * NS;
  if (!w) {
    w = new SolverWork();
    c->work = w;
  }
  if (w->n != n || w->ns != NS || w->seg != SEG) {
    w->n = n;
    w->ns = NS;
    w->seg = SEG;
    w->x.alloc(total); w->b.alloc(total); w->r64.alloc(total);
    w->r.alloc(total); w->z.alloc(total); w->p.alloc(total); w->q.alloc(total); w->dd.alloc(total);
    w->rf.release(); w->zf.release(); w->pf.release(); w->qf.release(); w->ddf.release();
    w->flag_f.alloc(n); w->flag_b.alloc(n);
    w->rpw64 = w->rpw32 = 0;
    w->flag_f.zero(s); w->flag_b.zero(s);
    w->sc.alloc(MAX_SYS);
    w->ctrl.alloc(1);
    w->ctrl.zero(s);
    w->epoch_host = 1;
    if (!w->h_ctrl) AFEM_CUDA(cudaMallocHost(&w->h_ctrl, sizeof(Ctrl)));
    if (!w->h_sc) AFEM_CUDA(cudaMallocHost(&w->h_sc, sizeof(SysScal) * MAX_SYS));
  }
  w->nsys = nsys;
  if (mixed && w->rf.n != (size_t)total) {
    w->rf.alloc(total); w->pf.alloc(total); w->qf.alloc(total); w->ddf.alloc(total);
  }
  if ((mixed || pc32) && w->zf.n != (size_t)total) w->zf.alloc(total);
  if (mixed && (!w->kmf_valid || w->kmf.n != (size_t)c->nnz)) {
    w->kmf.alloc(c->nnz);
    k_convert<float2, double2><<<c->num_sms * 8, 256, 0, s>>>(c->km.p, w->kmf.p, c->nnz);
    count_launch();
    w->kmf_valid = true;
  }
  // FP32 copies of the colour-ordered split rows (mixed inner solve, FP32 preconditioner)
  if ((mixed || pc32) && (!w->mcf_valid || w->mc_lkmf.n != c->mc_lcol.n)) {
    const long nl = (long)c->mc_lcol.n, nu = (long)c->mc_ucol.n;
    w->mc_lkmf.alloc(nl);
    w->mc_ukmf.alloc(nu);
    if (nl) {
      k_gather_entries<float2><<<c->num_sms * 8, 256, 0, s>>>(c->km.p, c->mc_lsrc.p, nl, w->mc_lkmf.p);
      count_launch();
    }
    if (nu) {
      k_gather_entries<float2><<<c->num_sms * 8, 256, 0, s>>>(c->km.p, c->mc_usrc.p, nu, w->mc_ukmf.p);
      count_launch();
    }
    w->mcf_valid = true;
  }
  {
    int b1 = 0;
    AFEM_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b1, k_spmv<double, NS, 1, SEG>, 256, 0));
    w->nblocks = std::max(1, b1) * c->num_sms;
    w->nblocks = std::max(w->nblocks, coresident_blocks(k_fwd_mc<double, double, NS, SEG>, c->num_sms));
    w->nblocks = std::max(w->nblocks, coresident_blocks(k_bwd_mc<double, double, NS, SEG>, c->num_sms));
    if (pc32) {
      w->nblocks = std::max(w->nblocks, coresident_blocks(k_fwd_mc<double, float, NS, SEG>, c->num_sms));
      w->nblocks = std::max(w->nblocks, coresident_blocks(k_bwd_mc<double, float, NS, SEG>, c->num_sms));
    }
    int bf = coresident_blocks(k_fwd<double, NS, SEG>, c->num_sms);
    int bb = coresident_blocks(k_bwd<double, NS, SEG>, c->num_sms);
    w->nblocks = std::max(w->nblocks, std::max(bf, bb));
    if (mixed) {
      w->nblocks = std::max(w->nblocks, coresident_blocks(k_fwd<float, NS, SEG>, c->num_sms));
      w->nblocks = std::max(w->nblocks, coresident_blocks(k_bwd<float, NS, SEG>, c->num_sms));
    }
    w->part.alloc((size_t)w->nblocks * MAX_SYS * 4);
    w->part2.alloc((size_t)w->nblocks * MAX_SYS * 4);
  }
  return w;
}

template <int NS, bool SEG>
int solve_ns(afem_ctx* c, const double* freq, const int* srcs, const afem_solve_opts* o, afem_solve_stats* st,
             const SolveExtra* ex) {
  cudaStream_t s = c->stream;
  const int n = c->nline;
  const long total = (long)n * NS;
  const int nsys = SEG ? c->nseg : NS;
  const bool mixed = o->precision == AFEM_MIXED;
  const bool pc32 = o->precision == AFEM_FP32_PRECOND;
  SolverWork* w = nullptr;
  {
    HostTimer ht(c, "host_setup_work");
    w = ensure_work<NS, SEG>(c, nsys, mixed, pc32);
  }
  // ---- right-hand sides and omegas
  {
    DBuf<int> dsrc;
    std::vector<int> hsrc(nsys);
    for (int k = 0; k < nsys; ++k) {
      hsrc[k] = srcs ? srcs[k] : 0;
      AFEM_REQUIRE((ex && ex->rhs) || (hsrc[k] >= 0 && hsrc[k] < c->rhs_nsrc), AFEM_EINVAL,
                   "solve: source index out of range");
    }
    if (ex && ex->rhs) {
      w->b.upload(reinterpret_cast<const double2*>(ex->rhs), total, s);
    } else {
      dsrc.upload(hsrc.data(), nsys, s);
      k_gather_rhs<<<c->num_sms * 8, 256, 0, s>>>(c->rhs.p, n, NS, dsrc.p, w->b.p, SEG ? c->seg_of_row.p : nullptr);
      count_launch();
    }
    AFEM_CUDA(cudaStreamSynchronize(s));
  }
  std::vector<double> om(nsys);
  const double pi = 4.0 * std::atan(1.0);
  for (int k = 0; k < nsys; ++k) om[k] = 2.0 * pi * freq[k];
  DBuf<double> d_om;
  d_om.upload(om.data(), nsys, s);
  // SysScal.omega must be valid for the residual SpMV before k_init_sys runs
  {
    std::vector<SysScal> tmp(MAX_SYS);
    for (int k = 0; k < nsys; ++k) { memset(&tmp[k], 0, sizeof(SysScal)); tmp[k].omega = om[k]; }
    AFEM_CUDA(cudaMemcpyAsync(w->sc.p, tmp.data(), sizeof(SysScal) * nsys, cudaMemcpyHostToDevice, s));
    AFEM_CUDA(cudaStreamSynchronize(s));
  }
  cudaEvent_t e0, e1;
  AFEM_CUDA(cudaEventCreate(&e0));
  AFEM_CUDA(cudaEventCreate(&e1));
  AFEM_CUDA(cudaEventRecord(e0, s));

  DBuf<double2>& xacc = w->xacc;  // accumulated FP64 solution (allocated once per size)
  xacc.alloc(total);
  std::vector<double> rr, bb;
  double tol_scale = 1.0;  // inner tolerances are relative to ||r0||; the target is relative to ||b||
  if (ex && ex->x0) {
    xacc.upload(reinterpret_cast<const double2*>(ex->x0), total, s);
    AFEM_CUDA(cudaMemcpyAsync(w->x.p, xacc.p, sizeof(double2) * total, cudaMemcpyDeviceToDevice, s));
    true_residual<NS, SEG>(c, w, rr, bb);  // r64 = b - A x0
    double worst_r = 0.0;
    for (int k = 0; k < nsys; ++k)
      if (bb[k] > 0) worst_r = std::max(worst_r, std::sqrt(rr[k] / bb[k]));
    if (worst_r > 0) tol_scale = 1.0 / worst_r;
  } else {
    xacc.zero(s);
    // r64 = b (x = 0)
    AFEM_CUDA(cudaMemcpyAsync(w->r64.p, w->b.p, sizeof(double2) * total, cudaMemcpyDeviceToDevice, s));
  }
  const bool recursive_only = ex && ex->recursive_only;
  w->no_window = recursive_only;
  const double tol = o->tol > 0 ? o->tol : 1e-8;
  const int maxit = o->maxit > 0 ? o->maxit : 100000;
  int it_total = 0, refinements = 0;
  std::vector<SysScal> hs;
  std::vector<int> status(nsys, AFEM_EMAXITER);
  double worst = 0.0, rec = 0.0;
  double prev = 1.0;  // current ||b - A x|| / ||b|| (worst system)
  int precond_now = o->precond;
  int learned_its = 0;
  bool fell_back = false;
  if (precond_now == AFEM_PRECOND_LEARNED)
    AFEM_REQUIRE(mpnn_ready(c), AFEM_ESTATE, "solve: the learned preconditioner has no weights");
  for (int outer = 0; outer < 64; ++outer) {
    // The inner solve starts from x = 0 on r64 and stops at a recursive
    // residual relative to ||r64||; ask for the reduction still missing,
    // never below what FP32 can deliver in the mixed mode.
    double inner_tol = std::min(0.5, 0.5 * tol / prev);
    if (outer == 0) inner_tol = tol * tol_scale;
    if (mixed) inner_tol = std::max(inner_tol, o->inner_tol > 0 ? o->inner_tol : 1e-5);
    const int left = maxit - it_total;
    if (left <= 0) break;
    int its;
    bool stalled = false;
    const bool mc_now = precond_now == AFEM_PRECOND_SSOR_MC || precond_now == AFEM_PRECOND_HYBRID;
    if (mixed)
      its = inner_cocg<float, float, NS, SEG>(c, w, o, precond_now, inner_tol, left, o->check_every, d_om.p, hs,
                                              &stalled);
    else if (pc32 && mc_now)
      its = inner_cocg<double, float, NS, SEG>(c, w, o, precond_now, inner_tol, left, o->check_every, d_om.p, hs,
                                               &stalled);
    else
      its = inner_cocg<double, double, NS, SEG>(c, w, o, precond_now, inner_tol, left, o->check_every, d_om.p, hs,
                                                &stalled);
    if (precond_now != AFEM_PRECOND_LEARNED && stalled) {
      for (int k = 0; k < nsys; ++k)
        if (hs[k].active) hs[k].status = AFEM_ESTAGNATION;
    }
    if (precond_now == AFEM_PRECOND_LEARNED) {
      learned_its += its;
      if (stalled) {
        // fallback: continue from the current iterate without the network (its base: the
        // gradient-corrected SSOR, or the reference's SSOR)
        precond_now = mpnn_base(c) == 1 ? AFEM_PRECOND_HYBRID : AFEM_PRECOND_SSOR;
        fell_back = true;
      }
    }
    it_total += its;
    refinements += 1;
    k_add_x<<<c->num_sms * 8, 256, 0, s>>>(xacc.p, w->x.p, total);
    count_launch();
    AFEM_CUDA(cudaMemcpyAsync(w->x.p, xacc.p, sizeof(double2) * total, cudaMemcpyDeviceToDevice, s));
    true_residual<NS, SEG>(c, w, rr, bb);  // r64 = b - A x_acc
    worst = 0.0;
    rec = 0.0;
    bool all_ok = true, any_fatal = false;
    for (int k = 0; k < nsys; ++k) {
      double rel = bb[k] > 0 ? std::sqrt(rr[k] / bb[k]) : 0.0;
      if (!std::isfinite(rr[k]) || !std::isfinite(bb[k])) rel = std::nan("");
      worst = std::max(worst, rel);
      rec = std::max(rec, hs[k].resid);
      if (!(rel <= tol)) all_ok = false;
      if (!std::isfinite(rel)) hs[k].status = AFEM_ENONFINITE;
      if (hs[k].status == AFEM_ENONFINITE || hs[k].status == AFEM_EBREAKDOWN) any_fatal = true;
      // OK only at the true residual: an inner solve that met its own (recursive)
      // target while the true residual stays above tol is a stagnation
      status[k] = (rel <= tol) ? AFEM_OK : (hs[k].status == AFEM_OK ? AFEM_ESTAGNATION : hs[k].status);
    }
    if (recursive_only) {
      // COCG13_single semantics: one Krylov run judged on its recursive residual
      for (int k = 0; k < nsys; ++k) status[k] = hs[k].status;
      rec = 0.0;
      for (int k = 0; k < nsys; ++k) rec = std::max(rec, hs[k].resid / tol_scale);
      break;
    }
    if (all_ok || any_fatal || !std::isfinite(worst)) break;
    if (worst > AFEM_REFINE_PROGRESS * prev && outer > 0 && !fell_back) {  // no progress from a restart
      for (int k = 0; k < nsys; ++k)
        if (status[k] == AFEM_OK || status[k] == AFEM_EMAXITER) status[k] = status[k] == AFEM_OK ? AFEM_OK : AFEM_ESTAGNATION;
      break;
    }
    prev = worst;
    fell_back = false;
  }
  AFEM_CUDA(cudaEventRecord(e1, s));
  AFEM_CUDA(cudaEventSynchronize(e1));
  float ms = 0;
  cudaEventElapsedTime(&ms, e0, e1);
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  // keep solutions
  c->X.alloc(total);
  AFEM_CUDA(cudaMemcpyAsync(c->X.p, xacc.p, sizeof(double2) * total, cudaMemcpyDeviceToDevice, s));
  AFEM_CUDA(cudaStreamSynchronize(s));
  c->nsys = nsys;
  c->sol_packed = SEG;
  c->sol_freq.assign(freq, freq + nsys);
  int stat = AFEM_OK;
  for (int k = 0; k < nsys; ++k)
    if (status[k] != AFEM_OK) { stat = status[k]; break; }
  c->last_learned_its = learned_its;
  if (st) {
    st->iterations = it_total;
    st->refinements = refinements;
    st->resid_recursive = rec;
    st->resid_true = worst;
    st->seconds = ms * 1e-3;
    st->status = stat;
  }
  return stat;
}

}  // namespace

namespace {

// values of the colour-ordered split rows for the current assembly (FP64; the
// FP32 copies follow with the workspace)
void ensure_mc_values(afem_ctx* c) {
  if (c->mc_vals_gen != c->assemble_gen) {
    const long nl = (long)c->mc_lcol.n, nu = (long)c->mc_ucol.n;
    c->mc_lkm.alloc(nl);
    c->mc_ukm.alloc(nu);
    c->mc_dkm.alloc(c->nline);
    k_gather_entries<double2><<<c->num_sms * 8, 256, 0, c->stream>>>(c->km.p, c->mc_dsrc.p, (long)c->nline,
                                                                     c->mc_dkm.p);
    count_launch();
    if (nl) {
      k_gather_entries<double2><<<c->num_sms * 8, 256, 0, c->stream>>>(c->km.p, c->mc_lsrc.p, nl, c->mc_lkm.p);
      count_launch();
    }
    if (nu) {
      k_gather_entries<double2><<<c->num_sms * 8, 256, 0, c->stream>>>(c->km.p, c->mc_usrc.p, nu, c->mc_ukm.p);
      count_launch();
    }
    c->mc_vals_gen = c->assemble_gen;
    invalidate_work(c);
  }
}

}  // namespace

int solve_device(afem_ctx* c, int nsys, const double* freq, const int* src, const afem_solve_opts* o,
                 afem_solve_stats* st, const SolveExtra* ex) {
  AFEM_REQUIRE(c->assembled, AFEM_ESTATE, "solve: system not assembled");
  // the multicolour paths never read the natural-order level schedules
  const bool mc_only = o->precond == AFEM_PRECOND_HYBRID || o->precond == AFEM_PRECOND_SSOR_MC ||
                       (o->precond == AFEM_PRECOND_LEARNED && mpnn_base(c) == 1);
  {
    HostTimer ht(c, "host_setup_schedule");
    build_schedule(c, !mc_only);
  }
  {
    HostTimer ht(c, "host_setup_mc_values");
    ensure_mc_values(c);
  }
  if (o->precond == AFEM_PRECOND_HYBRID || (o->precond == AFEM_PRECOND_LEARNED && mpnn_base(c) == 1)) {
    HostTimer ht(c, "host_setup_hybrid");
    hybrid_prepare(c);
  }
  if (c->nseg > 0) {
    AFEM_REQUIRE(nsys == c->nseg, AFEM_EINVAL, "solve: a packed batch solves one system per mesh (nsys = nseg)");
    AFEM_REQUIRE(o->precond != AFEM_PRECOND_LEARNED, AFEM_EINVAL,
                 "solve: the learned preconditioner does not run on packed batches");
    AFEM_REQUIRE(!ex || (!ex->x0 && !ex->rhs), AFEM_EINVAL, "solve: packed batches take the assembled sources");
    return solve_ns<1, true>(c, freq, src, o, st, ex);
  }
  switch (nsys) {
    case 1: return solve_ns<1, false>(c, freq, src, o, st, ex);
    case 2: return solve_ns<2, false>(c, freq, src, o, st, ex);
    case 4: return solve_ns<4, false>(c, freq, src, o, st, ex);
    case 8: return solve_ns<8, false>(c, freq, src, o, st, ex);
    case 16: return solve_ns<16, false>(c, freq, src, o, st, ex);
    default: throw Error{AFEM_EINVAL, "solve: nsys must be 1, 2, 4, 8 or 16"};
  }
}

void precond_apply_device(afem_ctx* c, double omega, const double2* r, double2* z) {
  AFEM_REQUIRE(c->assembled, AFEM_ESTATE, "preconditioner: system not assembled");
  AFEM_REQUIRE(c->nseg == 0, AFEM_EINVAL, "preconditioner: packed batches are not supported here");
  build_schedule(c, false);
  ensure_mc_values(c);
  hybrid_prepare(c);
  SolverWork* w = ensure_work<1, false>(c, 1, false);
  cudaStream_t s = c->stream;
  const int n = c->nline;
  HybridState* h = c->hyb;
  // one system at omega, iteration 0: the sweeps leave x, p and q alone
  SysScal sc0;
  std::memset(&sc0, 0, sizeof sc0);
  sc0.omega = omega;
  sc0.active = 1;
  Ctrl ct;
  std::memset(&ct, 0, sizeof ct);
  ct.epoch = w->epoch_host;
  ct.maxit = 1;
  AFEM_CUDA(cudaMemcpyAsync(w->sc.p, &sc0, sizeof(SysScal), cudaMemcpyHostToDevice, s));
  AFEM_CUDA(cudaMemcpyAsync(w->ctrl.p, &ct, sizeof(Ctrl), cudaMemcpyHostToDevice, s));
  AFEM_CUDA(cudaMemcpyAsync(w->r.p, r, sizeof(double2) * n, cudaMemcpyDeviceToDevice, s));
  w->ht.alloc(h->node);
  w->hy.alloc(h->node);
  w->hdd.alloc(h->node);
  setup_dd<double, double, 1, false>(c, w, AFEM_PRECOND_HYBRID, 1.0);
  w->mc_blocks = std::min(std::min(coresident_blocks(k_fwd_mc<double, double, 1, false>, c->num_sms),
                                   coresident_blocks(k_bwd_mc<double, double, 1, false>, c->num_sms)), w->nblocks);
  w->nmc_blocks = std::min(coresident_blocks(k_nsweep_mc<double, 1, false>, c->num_sms), w->nblocks);
  launch_coop(k_fwd_mc<double, double, 1, false>, w->mc_blocks, s, (const int32_t*)c->mc_lptr.p,
              (const int32_t*)c->mc_lcol.p, (const double2*)c->mc_lkm.p, n, w->r.p, w->z.p, (const double2*)w->q.p,
              (const double2*)c->mc_dkm.p, 1.0, (const int32_t*)c->perm_mc.p, (const int32_t*)c->color_ptr.p,
              c->ncolors, w->sc.p, w->ctrl.p, w->part.p, (const uint8_t*)nullptr, (double2*)nullptr);
  launch_coop(k_bwd_mc<double, double, 1, false>, w->mc_blocks, s, (const int32_t*)c->mc_uptr.p,
              (const int32_t*)c->mc_ucol.p, (const double2*)c->mc_ukm.p, n, (const double2*)w->r.p, w->z.p,
              (const int32_t*)c->perm_mc.p, (const int32_t*)c->color_ptr.p, c->ncolors, w->sc.p, w->ctrl.p, w->part.p,
              (const uint8_t*)nullptr, (const double2*)c->mc_dkm.p, 1.0);
  k_grad_t<double, double, 1><<<c->num_sms * 8, 256, 0, s>>>(h->node, h->nptr.p, h->nlist.p, c->bc.p,
                                                              (const double2*)w->r.p, w->ht.p, w->ctrl.p);
  count_launch();
  for (int bwd = 0; bwd < 2; ++bwd)
    launch_coop(k_nsweep_mc<double, 1, false>, w->nmc_blocks, s, (const int32_t*)(bwd ? h->uptr.p : h->lptr.p),
                (const int32_t*)(bwd ? h->ucol.p : h->lcol.p), (const double2*)(bwd ? h->ukm.p : h->lkm.p),
                (const double2*)w->ht.p, w->hy.p, (const double2*)w->hdd.p, (const int32_t*)h->perm.p,
                (const int32_t*)h->cptr.p, h->ncolors, (const SysScal*)w->sc.p, (const Ctrl*)w->ctrl.p,
                (const uint8_t*)nullptr, bwd, (double*)nullptr);
  k_grad_add<double, double, 1, false><<<w->nblocks, 256, 0, s>>>(n, c->line.p, c->bc.p, (const double2*)w->hy.p,
                                                                  w->z.p, (const double2*)w->r.p, w->ctrl.p,
                                                                  w->part.p, (const uint8_t*)nullptr);
  count_launch();
  AFEM_CUDA(cudaMemcpyAsync(z, w->z.p, sizeof(double2) * n, cudaMemcpyDeviceToDevice, s));
  AFEM_CUDA(cudaStreamSynchronize(s));
}

void get_residual(afem_ctx* c, int k, double* r) {
  SolverWork* w = c->work;
  AFEM_REQUIRE(w && c->nsys > 0 && k >= 0 && k < c->nsys, AFEM_ESTATE, "get_residual: no such system");
  if (w->seg) {  // packed batch: the rows of mesh k
    const int r0 = c->seg_row_ptr[k], r1 = c->seg_row_ptr[k + 1];
    AFEM_CUDA(cudaMemcpyAsync(r, w->r64.p + r0, sizeof(double2) * (r1 - r0), cudaMemcpyDeviceToHost, c->stream));
    AFEM_CUDA(cudaStreamSynchronize(c->stream));
    return;
  }
  std::vector<double2> all((size_t)w->n * w->ns);
  w->r64.download(all.data(), all.size(), c->stream);
  AFEM_CUDA(cudaStreamSynchronize(c->stream));
  for (int i = 0; i < w->n; ++i) {
    r[2 * i] = all[(size_t)i * w->ns + k].x;
    r[2 * i + 1] = all[(size_t)i * w->ns + k].y;
  }
}

// New matrix values: the FP32 copies are stale.  The SpMV tuning stays (it
// depends on the pattern only), so repeated solves take the same reduction
// order and give the same bits.
void invalidate_work(afem_ctx* c) {
  if (c->work) c->work->kmf_valid = c->work->mcf_valid = false;
}

// A new pattern: also tune the SpMV again (ensure_work re-allocates when the
// size changes; buffers of the same size are kept).
void invalidate_pattern_work(afem_ctx* c) {
  c->spt_ready = false;
  if (c->work) {
    c->work->kmf_valid = c->work->mcf_valid = false;
    c->work->rpw64 = c->work->rpw32 = 0;
  }
  c->nsys = 0;  // the old solutions belong to the old pattern
}

void reset_spmv_tuning(afem_ctx* c) {
  if (c->work) c->work->rpw64 = c->work->rpw32 = 0;
}

void destroy_work(afem_ctx* c) {
  delete c->work;
  c->work = nullptr;
}

}  // namespace afem
