// Edge numbering (MKLINE_V2 / MKN6) and the CSR pattern, built on the device.
//
// Integer work only: every output is bit-identical to the reference's
// serial construction (tmtgem/common/m_line_type.f90:120-277 for the
// numbering, src/solver/m_iccg_var_takuto.f90:277-485 for the pattern).
#include <algorithm>
#include <vector>

#include <memory>

#include "afem_internal.h"

namespace afem {

namespace {

const int KL0[6] = {0, 1, 0, 0, 1, 2};  // kl(:,1)-1 (m_fem_edge_util.f90:5-11)
const int KL1[6] = {1, 2, 2, 3, 3, 3};  // kl(:,2)-1
__constant__ int c_kl0[6] = {0, 1, 0, 0, 1, 2};
__constant__ int c_kl1[6] = {1, 2, 2, 3, 3, 3};

// ---------------------------------------------------------------- exclusive scan
constexpr int SCAN_T = 1024;
constexpr int SCAN_PER = 4;
constexpr int SCAN_CHUNK = SCAN_T * SCAN_PER;

__global__ void k_scan_block(const int32_t* __restrict__ in, int32_t* __restrict__ out, int n,
                             int64_t* __restrict__ blocksum) {
  __shared__ int64_t s[SCAN_T];
  const int base = blockIdx.x * SCAN_CHUNK + threadIdx.x * SCAN_PER;
  int64_t v[SCAN_PER];
  int64_t t = 0;
#pragma unroll
  for (int k = 0; k < SCAN_PER; ++k) {
    v[k] = (base + k < n) ? in[base + k] : 0;
    t += v[k];
  }
  s[threadIdx.x] = t;
  __syncthreads();
  for (int off = 1; off < SCAN_T; off <<= 1) {
    int64_t a = (threadIdx.x >= off) ? s[threadIdx.x - off] : 0;
    __syncthreads();
    s[threadIdx.x] += a;
    __syncthreads();
  }
  int64_t run = s[threadIdx.x] - t;
#pragma unroll
  for (int k = 0; k < SCAN_PER; ++k) {
    if (base + k < n) out[base + k] = (int32_t)run;
    run += v[k];
  }
  if (threadIdx.x == SCAN_T - 1) blocksum[blockIdx.x] = s[SCAN_T - 1];
}

__global__ void k_scan_add(int32_t* __restrict__ out, int n, const int64_t* __restrict__ offs) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) out[i] += (int32_t)offs[i / SCAN_CHUNK];
}

__global__ void k_scan_sums(int64_t* __restrict__ sums, int nb, int64_t* __restrict__ total) {
  // single thread: nb is small (n / 4096)
  if (threadIdx.x == 0 && blockIdx.x == 0) {
    int64_t run = 0;
    for (int i = 0; i < nb; ++i) {
      int64_t v = sums[i];
      sums[i] = run;
      run += v;
    }
    *total = run;
  }
}

// ---------------------------------------------------------------- numbering
__global__ void k_count_node_tets(const int32_t* __restrict__ n4, int ntet, int32_t* __restrict__ cnt) {
  long i = blockIdx.x * (long)blockDim.x + threadIdx.x;
  if (i < 4L * ntet) atomicAdd(&cnt[n4[i] - 1], 1);
}

__global__ void k_fill_node_tets(const int32_t* __restrict__ n4, int ntet, const int32_t* __restrict__ ptr,
                                 int32_t* __restrict__ cursor, int32_t* __restrict__ list) {
  long i = blockIdx.x * (long)blockDim.x + threadIdx.x;
  if (i < 4L * ntet) {
    int nd = n4[i] - 1;
    int pos = atomicAdd(&cursor[nd], 1);
    list[ptr[nd] + pos] = (int32_t)(i / 4);
  }
}

// Sort each segment ascending (segments are short: insertion sort per thread).
__global__ void k_sort_segments(const int32_t* __restrict__ ptr, int nseg, int32_t* __restrict__ list, int maxlen,
                                DevStatus* st) {
  int s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= nseg) return;
  int a = ptr[s], b = ptr[s + 1];
  if (b - a > maxlen) raise_status(st, DEV_DEGREE, s);
  for (int i = a + 1; i < b; ++i) {
    int32_t v = list[i];
    int j = i - 1;
    while (j >= a && list[j] > v) {
      list[j + 1] = list[j];
      --j;
    }
    list[j + 1] = v;
  }
}

// MKLINE_V2 (m_line_type.f90:151-176): edges (n1, n2 > n1) in order of first
// encounter over the tetrahedra of n1 by ascending id and local nodes 1..4.
// Pass 0 counts, pass 1 writes line_item.
__global__ void k_mkline_group(const int32_t* __restrict__ n4, const int32_t* __restrict__ nptr,
                               const int32_t* __restrict__ nlist, int node, int32_t* __restrict__ cnt,
                               const int32_t* __restrict__ stack, int32_t* __restrict__ line, DevStatus* st) {
  int n1 = blockIdx.x * blockDim.x + threadIdx.x;  // 0-based
  if (n1 >= node) return;
  int32_t seen[NODE_NBR_MAX];
  int ns = 0;
  const int a = nptr[n1], b = nptr[n1 + 1];
  for (int q = a; q < b; ++q) {
    const int t = nlist[q];
    for (int k = 0; k < 4; ++k) {
      const int n2 = n4[4L * t + k];  // 1-based
      if (n2 <= n1 + 1) continue;
      bool found = false;
      for (int l = 0; l < ns; ++l)
        if (seen[l] == n2) { found = true; break; }
      if (found) continue;
      if (ns == NODE_NBR_MAX) { raise_status(st, DEV_DEGREE, n1); continue; }
      seen[ns++] = n2;
    }
  }
  if (line == nullptr) {
    cnt[n1] = ns;
  } else {
    const int base = stack[n1];
    for (int l = 0; l < ns; ++l) {
      line[2L * (base + l)] = n1 + 1;
      line[2L * (base + l) + 1] = seen[l];
    }
  }
}

// MKN6 (m_line_type.f90:224-277): signed edge id of each local edge.
__global__ void k_mkn6(const int32_t* __restrict__ n4, int ntet, const int32_t* __restrict__ stack,
                       const int32_t* __restrict__ line, int32_t* __restrict__ n6line, DevStatus* st) {
  long i = blockIdx.x * (long)blockDim.x + threadIdx.x;
  if (i >= 6L * ntet) return;
  const long t = i / 6;
  const int j = (int)(i % 6);
  int n11 = n4[4 * t + c_kl0[j]], n12 = n4[4 * t + c_kl1[j]], dir = 1;
  if (n11 > n12) { int tmp = n11; n11 = n12; n12 = tmp; dir = -1; }
  int id = -1;
  for (int k = stack[n11 - 1]; k < stack[n11]; ++k)
    if (line[2L * k + 1] == n12) { id = k + 1; break; }
  if (id < 0) { raise_status(st, DEV_NOTFOUND, (int)t); id = 1; }
  n6line[i] = dir * id;
}

// ---------------------------------------------------------------- pattern
__global__ void k_count_edge_tets(const int32_t* __restrict__ n6line, int ntet, int nline, int32_t* __restrict__ cnt,
                                  DevStatus* st) {
  long i = blockIdx.x * (long)blockDim.x + threadIdx.x;
  if (i < 6L * ntet) {
    int e = abs(n6line[i]) - 1;
    if (e < 0 || e >= nline) { raise_status(st, DEV_NOTFOUND, (int)(i / 6)); return; }
    atomicAdd(&cnt[e], 1);
  }
}

__global__ void k_fill_edge_tets(const int32_t* __restrict__ n6line, int ntet, int nline,
                                 const int32_t* __restrict__ ptr, int32_t* __restrict__ cursor,
                                 int32_t* __restrict__ list) {
  long i = blockIdx.x * (long)blockDim.x + threadIdx.x;
  if (i < 6L * ntet) {
    int e = abs(n6line[i]) - 1;
    if (e < 0 || e >= nline) return;
    int pos = atomicAdd(&cursor[e], 1);
    list[ptr[e] + pos] = (int32_t)((i / 6) * 8 + (i % 6));
  }
}

// One warp per row: the sorted unique set of edges of the tetrahedra around
// the row's edge (C_set_dof2's upper and lower lists plus the diagonal).
constexpr int PAT_WARPS = 8;
constexpr int PAT_CAND = 6 * EDGE_DEG_MAX;
__global__ void __launch_bounds__(PAT_WARPS * 32)
    k_row_pattern(const int32_t* __restrict__ n6line, const int32_t* __restrict__ etp, const int32_t* __restrict__ etl,
                  int nline, int32_t* __restrict__ rowlen, const int32_t* __restrict__ rowptr,
                  int32_t* __restrict__ col, int32_t* __restrict__ diagpos, DevStatus* st) {
  __shared__ int32_t cand[PAT_WARPS][PAT_CAND];
  const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int row = blockIdx.x * PAT_WARPS + w;
  if (row >= nline) return;
  const int a = etp[row], b = etp[row + 1];
  int deg = b - a;
  if (deg > EDGE_DEG_MAX) {
    if (lane == 0) raise_status(st, DEV_DEGREE, row);
    deg = EDGE_DEG_MAX;
  }
  const int c = 6 * deg;
  for (int k = lane; k < c; k += 32) {
    const int t = etl[a + k / 6] >> 3;
    cand[w][k] = abs(n6line[6L * t + (k % 6)]) - 1;
  }
  __syncwarp();
  // mark first occurrences (duplicates become -1), then rank = #distinct values below
  __shared__ int32_t uniq[PAT_WARPS][PAT_CAND];
  for (int k = lane; k < c; k += 32) {
    const int v = cand[w][k];
    bool first = true;
    for (int j = 0; j < k; ++j)
      if (cand[w][j] == v) { first = false; break; }
    uniq[w][k] = first ? v : -1;
  }
  __syncwarp();
  int count = 0;
  for (int k0 = 0; k0 < c; k0 += 32) {
    const int k = k0 + lane;
    const int v = (k < c) ? uniq[w][k] : -1;
    const bool first = v >= 0;
    int rank = 0;
    if (first)
      for (int j = 0; j < c; ++j) {
        const int u = uniq[w][j];
        rank += (u >= 0 && u < v);
      }
    const unsigned m = __ballot_sync(0xffffffffu, first);
    count += __popc(m);
    if (col != nullptr && first && rank < ROW_MAX) {
      col[rowptr[row] + rank] = v;
      if (v == row) diagpos[row] = rowptr[row] + rank;
    }
  }
  if (lane == 0 && col == nullptr) {
    if (count > ROW_MAX) raise_status(st, DEV_ROWLEN, row);
    rowlen[row] = count;
  }
}

inline unsigned nblk(long n, int t) { return (unsigned)((n + t - 1) / t); }

}  // namespace

void exclusive_scan(const int32_t* in, int32_t* out, int n, cudaStream_t s, long* total_host) {
  // out[0..n] with out[n] = total (out must hold n+1 values)
  const int nb = (n + SCAN_CHUNK - 1) / SCAN_CHUNK;
  DBuf<int64_t> sums;
  sums.alloc(nb + 1);
  if (n > 0) {
    k_scan_block<<<nb, SCAN_T, 0, s>>>(in, out, n, sums.p);
    count_launch();
    k_scan_sums<<<1, 1, 0, s>>>(sums.p, nb, sums.p + nb);
    count_launch();
    k_scan_add<<<nblk(n, 256), 256, 0, s>>>(out, n, sums.p);
    count_launch();
  } else {
    AFEM_CUDA(cudaMemsetAsync(sums.p, 0, sizeof(int64_t), s));
  }
  int64_t tot = 0;
  AFEM_CUDA(cudaMemcpyAsync(&tot, sums.p + nb, sizeof(int64_t), cudaMemcpyDeviceToHost, s));
  AFEM_CUDA(cudaStreamSynchronize(s));
  AFEM_REQUIRE(tot < (int64_t)INT32_MAX, AFEM_EINVAL, "scan total exceeds int32 range");
  int32_t t32 = (int32_t)tot;
  AFEM_CUDA(cudaMemcpyAsync(out + n, &t32, sizeof(int32_t), cudaMemcpyHostToDevice, s));
  AFEM_CUDA(cudaStreamSynchronize(s));
  if (total_host) *total_host = (long)tot;
}

void build_lines_device(afem_ctx* c) {
  cudaStream_t s = c->stream;
  const int node = c->node, ntet = c->ntet;
  DBuf<int32_t> cnt, nptr, cursor, nlist;
  cnt.alloc(node);
  cnt.zero(s);
  nptr.alloc(node + 1);
  k_count_node_tets<<<nblk(4L * ntet, 256), 256, 0, s>>>(c->n4.p, ntet, cnt.p);
  count_launch();
  exclusive_scan(cnt.p, nptr.p, node, s, nullptr);
  cursor.alloc(node);
  cursor.zero(s);
  nlist.alloc(4L * ntet);
  k_fill_node_tets<<<nblk(4L * ntet, 256), 256, 0, s>>>(c->n4.p, ntet, nptr.p, cursor.p, nlist.p);
  count_launch();
  k_sort_segments<<<nblk(node, 128), 128, 0, s>>>(nptr.p, node, nlist.p, NODE_DEG_MAX, c->status.p);
  count_launch();
  check_status(c, "edge numbering: node adjacency (more than 100 tetrahedra share a node)");
  k_mkline_group<<<nblk(node, 128), 128, 0, s>>>(c->n4.p, nptr.p, nlist.p, node, cnt.p, nullptr, nullptr,
                                                 c->status.p);
  count_launch();
  DBuf<int32_t> stack;
  stack.alloc(node + 1);
  long nline = 0;
  exclusive_scan(cnt.p, stack.p, node, s, &nline);
  check_status(c, "edge numbering: node degree");
  c->nline = (int)nline;
  c->line.alloc(2L * nline);
  k_mkline_group<<<nblk(node, 128), 128, 0, s>>>(c->n4.p, nptr.p, nlist.p, node, nullptr, stack.p, c->line.p,
                                                 c->status.p);
  count_launch();
  c->n6line.alloc(6L * ntet);
  k_mkn6<<<nblk(6L * ntet, 256), 256, 0, s>>>(c->n4.p, ntet, stack.p, c->line.p, c->n6line.p, c->status.p);
  count_launch();
  check_status(c, "edge numbering: MKN6");
  (void)KL0;
  (void)KL1;
}

void build_pattern_device(afem_ctx* c) {
  cudaStream_t s = c->stream;
  const int nline = c->nline, ntet = c->ntet;
  DBuf<int32_t> cnt, cursor;
  cnt.alloc(nline);
  cnt.zero(s);
  k_count_edge_tets<<<nblk(6L * ntet, 256), 256, 0, s>>>(c->n6line.p, ntet, nline, cnt.p, c->status.p);
  count_launch();
  check_status(c, "pattern: n6line holds an edge id outside 1..nline");
  c->etp.alloc(nline + 1);
  exclusive_scan(cnt.p, c->etp.p, nline, s, nullptr);
  cursor.alloc(nline);
  cursor.zero(s);
  c->etl.alloc(6L * ntet);
  k_fill_edge_tets<<<nblk(6L * ntet, 256), 256, 0, s>>>(c->n6line.p, ntet, nline, c->etp.p, cursor.p, c->etl.p);
  count_launch();
  k_sort_segments<<<nblk(nline, 128), 128, 0, s>>>(c->etp.p, nline, c->etl.p, EDGE_DEG_MAX, c->status.p);
  count_launch();
  check_status(c, "pattern: edge shared by too many tetrahedra");
  k_row_pattern<<<nblk(nline, PAT_WARPS), PAT_WARPS * 32, 0, s>>>(c->n6line.p, c->etp.p, c->etl.p, nline, cnt.p,
                                                                  nullptr, nullptr, nullptr, c->status.p);
  count_launch();
  check_status(c, "pattern: row length");
  c->rowptr.alloc(nline + 1);
  long nnz = 0;
  exclusive_scan(cnt.p, c->rowptr.p, nline, s, &nnz);
  c->nnz = nnz;
  c->col.alloc(nnz);
  c->diagpos.alloc(nline);
  k_row_pattern<<<nblk(nline, PAT_WARPS), PAT_WARPS * 32, 0, s>>>(c->n6line.p, c->etp.p, c->etl.p, nline, nullptr,
                                                                  c->rowptr.p, c->col.p, c->diagpos.p, c->status.p);
  count_launch();
  check_status(c, "pattern: fill");
  c->pattern_ready = true;
  c->schedule_ready = false;
  c->levels_ready = false;
}

// Dependency levels of the two triangular sweeps (computed once per pattern on
// the host: one pass over the strictly lower / upper parts) and the processing
// orders the sweep kernels walk: rows sorted by level.  Every row's formula is
// unchanged, only the order in which rows are visited; a row's dependencies
// always have a smaller level, so the order is topological.
void compute_schedule(int n, const int32_t* rp, const int32_t* dp, const int32_t* cl, int32_t* perm_f,
                      int32_t* perm_b, int* levels_f, int* levels_b) {
  std::vector<int32_t> lev(n);
  auto order = [&](bool forward, int32_t* perm, int* nlev) {
    int mx = 0;
    if (forward) {
      for (int i = 0; i < n; ++i) {
        int l = 0;
        for (int k = rp[i]; k < dp[i]; ++k) l = std::max(l, lev[cl[k]] + 1);
        lev[i] = l;
        mx = std::max(mx, l);
      }
    } else {
      for (int i = n - 1; i >= 0; --i) {
        int l = 0;
        for (int k = dp[i] + 1; k < rp[i + 1]; ++k) l = std::max(l, lev[cl[k]] + 1);
        lev[i] = l;
        mx = std::max(mx, l);
      }
    }
    *nlev = n > 0 ? mx + 1 : 0;
    std::vector<int32_t> cnt(mx + 2, 0);
    for (int i = 0; i < n; ++i) cnt[lev[i] + 1]++;
    for (int l = 0; l <= mx; ++l) cnt[l + 1] += cnt[l];
    if (forward) {
      for (int i = 0; i < n; ++i) perm[cnt[lev[i]]++] = i;
    } else {
      for (int i = n - 1; i >= 0; --i) perm[cnt[lev[i]]++] = i;
    }
  };
  order(true, perm_f, levels_f);
  order(false, perm_b, levels_b);
}

// Greedy distance-1 colouring of the matrix graph in row order (each row takes
// the smallest colour none of its already-coloured neighbours has), then the
// rows sorted by colour.  Rows of one colour share no nonzero, so a
// Gauss-Seidel pass can update all of them at once.
int compute_coloring(int n, const int32_t* rp, const int32_t* cl, uint8_t* color, int32_t* perm, int32_t* cptr,
                     int max_colors) {
  std::vector<int> mark(max_colors + 1, -1);
  int nc = 0;
  for (int i = 0; i < n; ++i) {
    for (int k = rp[i]; k < rp[i + 1]; ++k) {
      const int j = cl[k];
      if (j < i) mark[color[j]] = i;
    }
    int cidx = 0;
    while (cidx < max_colors && mark[cidx] == i) ++cidx;
    if (cidx >= max_colors) return -1;
    color[i] = (uint8_t)cidx;
    nc = std::max(nc, cidx + 1);
  }
  std::vector<int32_t> cnt(nc + 1, 0);
  for (int i = 0; i < n; ++i) cnt[color[i] + 1]++;
  for (int c = 0; c < nc; ++c) cnt[c + 1] += cnt[c];
  for (int c = 0; c <= nc; ++c) cptr[c] = cnt[c];
  for (int i = 0; i < n; ++i) perm[cnt[color[i]]++] = i;
  return nc;
}

namespace {

// Colour-ordered split rows on the device: position p holds row perm[p]; lcnt/ucnt count its
// entries of earlier / later colours, and the fill writes them in the row's CSR order.
__global__ void k_split_count(const int32_t* __restrict__ rp, const int32_t* __restrict__ cl,
                              const uint8_t* __restrict__ color, const int32_t* __restrict__ perm, int n,
                              int32_t* __restrict__ lcnt, int32_t* __restrict__ ucnt) {
  for (int p = blockIdx.x * blockDim.x + threadIdx.x; p < n; p += gridDim.x * blockDim.x) {
    const int i = perm[p];
    const int ci = color[i];
    int nl = 0, nu = 0;
    for (int k = rp[i]; k < rp[i + 1]; ++k) {
      const int cj = color[cl[k]];
      if (cj < ci) ++nl;
      else if (cj > ci) ++nu;
    }
    lcnt[p] = nl;
    ucnt[p] = nu;
  }
}

__global__ void k_split_fill(const int32_t* __restrict__ rp, const int32_t* __restrict__ cl,
                             const int32_t* __restrict__ dp, const uint8_t* __restrict__ color,
                             const int32_t* __restrict__ perm, int n, const int32_t* __restrict__ lptr,
                             const int32_t* __restrict__ uptr, int32_t* __restrict__ lcol, int32_t* __restrict__ lsrc,
                             int32_t* __restrict__ ucol, int32_t* __restrict__ usrc, int32_t* __restrict__ dsrc) {
  for (int p = blockIdx.x * blockDim.x + threadIdx.x; p < n; p += gridDim.x * blockDim.x) {
    const int i = perm[p];
    const int ci = color[i];
    int a = lptr[p], b = uptr[p];
    for (int k = rp[i]; k < rp[i + 1]; ++k) {
      const int j = cl[k];
      const int cj = color[j];
      if (cj < ci) { lcol[a] = j; lsrc[a++] = k; }
      else if (cj > ci) { ucol[b] = j; usrc[b++] = k; }
    }
    if (dsrc) dsrc[p] = dp[i];
  }
}

}  // namespace

void split_rows_device(afem_ctx* c, const int32_t* rp, const int32_t* cl, const int32_t* dp, const uint8_t* color,
                       const int32_t* perm, int n, DBuf<int32_t>& lptr, DBuf<int32_t>& lcol, DBuf<int32_t>& lsrc,
                       DBuf<int32_t>& uptr, DBuf<int32_t>& ucol, DBuf<int32_t>& usrc, DBuf<int32_t>* dsrc) {
  cudaStream_t s = c->stream;
  DBuf<int32_t> lcnt, ucnt;
  lcnt.alloc(n);
  ucnt.alloc(n);
  const int nb = c->num_sms * 8;
  k_split_count<<<nb, 256, 0, s>>>(rp, cl, color, perm, n, lcnt.p, ucnt.p);
  count_launch();
  lptr.alloc(n + 1);
  uptr.alloc(n + 1);
  long ltot = 0, utot = 0;
  exclusive_scan(lcnt.p, lptr.p, n, s, &ltot);
  exclusive_scan(ucnt.p, uptr.p, n, s, &utot);
  lcol.alloc(ltot);
  lsrc.alloc(ltot);
  ucol.alloc(utot);
  usrc.alloc(utot);
  int32_t* ds = nullptr;
  if (dsrc) {
    dsrc->alloc(n);
    ds = dsrc->p;
  }
  k_split_fill<<<nb, 256, 0, s>>>(rp, cl, dp, color, perm, n, lptr.p, uptr.p, lcol.p, lsrc.p, ucol.p, usrc.p, ds);
  count_launch();
}

void build_schedule(afem_ctx* c, bool levels) {
  if (c->schedule_ready && (!levels || c->levels_ready)) return;
  const int n = c->nline;
  cudaStream_t s = c->stream;
  // host copies of the pattern for the colouring (left uninitialised: filled by the copies)
  std::unique_ptr<int32_t[]> rp(new int32_t[n + 1]), cl(new int32_t[c->nnz]);
  c->rowptr.download(rp.get(), n + 1, s);
  c->col.download(cl.get(), c->nnz, s);
  AFEM_CUDA(cudaStreamSynchronize(s));
  if (levels && !c->levels_ready) {
    // the natural-order sweeps' dependency levels (IC, SSOR, DIAG, none)
    std::vector<int32_t> pf(n), pb(n), dp(n);
    c->diagpos.download(dp.data(), n, s);
    AFEM_CUDA(cudaStreamSynchronize(s));
    compute_schedule(n, rp.get(), dp.data(), cl.get(), pf.data(), pb.data(), &c->levels_f, &c->levels_b);
    c->perm_f.upload(pf.data(), n, s);
    c->perm_b.upload(pb.data(), n, s);
    AFEM_CUDA(cudaStreamSynchronize(s));
    c->levels_ready = true;
  }
  if (c->schedule_ready) return;
  std::vector<uint8_t> color(n);
  std::vector<int32_t> pm(n), cptr(256);
  const int nc = compute_coloring(n, rp.get(), cl.get(), color.data(), pm.data(), cptr.data(), 255);
  AFEM_REQUIRE(nc > 0, AFEM_EPATTERN, "colouring: more than 255 colours");
  c->ncolors = nc;
  c->color.upload(color.data(), n, s);
  c->perm_mc.upload(pm.data(), n, s);
  c->color_ptr.upload(cptr.data(), nc + 1, s);
  // colour-ordered split rows for the multicolour sweeps: position p holds row
  // perm[p]; its entries of earlier colours (the forward sweep's) and of later
  // colours (the backward sweep's), each with the index of the entry in the CSR;
  // built on the device from the colouring (counts, prefix sums, fill in CSR order)
  split_rows_device(c, c->rowptr.p, c->col.p, c->diagpos.p, c->color.p, c->perm_mc.p, n, c->mc_lptr, c->mc_lcol,
                    c->mc_lsrc, c->mc_uptr, c->mc_ucol, c->mc_usrc, &c->mc_dsrc);
  c->mc_vals_gen = -1;
  AFEM_CUDA(cudaStreamSynchronize(s));
  c->schedule_ready = true;
}

}  // namespace afem

// Host-only: greedy colouring of a CSR pattern (rows sorted by colour), for tests.
extern "C" int afem_coloring(int n, const int32_t* rowptr, const int32_t* col, uint8_t* color, int32_t* perm,
                             int32_t* cptr) {
  if (n < 0 || !rowptr || !col || !color || !perm || !cptr) return AFEM_EINVAL;
  return afem::compute_coloring(n, rowptr, col, color, perm, cptr, 255);
}

// Host-only: the sweep schedules of a CSR pattern (diagonal included, columns
// ascending, 0-based) for tests and tools.
extern "C" int afem_sweep_schedule(int n, const int32_t* rowptr, const int32_t* col, const int32_t* diagpos,
                                   int32_t* perm_f, int32_t* perm_b, int* levels_f, int* levels_b) {
  if (n < 0 || !rowptr || !col || !diagpos || !perm_f || !perm_b) return AFEM_EINVAL;
  afem::compute_schedule(n, rowptr, diagpos, col, perm_f, perm_b, levels_f, levels_b);
  return AFEM_OK;
}
