// Gradient-space (nodal) correction for COCG: the set-up half.
//
// The curl-curl operator vanishes on discrete gradients, so in the resistive
// air (sigma = 1e-8 S/m) the edge system has eigenvalues ~1e-12 of the rest
// along the gradients of nodal functions; SSOR on the edges does not reach
// them and COCG stagnates.  The hybrid preconditioner of Hiptmair (SIAM J.
// Numer. Anal. 36, 1998) adds a correction in that subspace:
//
//     z = SSOR_edge(r) + G SSOR_node(G^T r),   A_G = G^T A G,
//
// with G the edge-node incidence (G x)_e = x_n2(e) - x_n1(e) over the edges
// that are not Dirichlet.  A_G is formed here as a Galerkin product of the
// assembled edge matrix, split like A: A_G(omega) = K_G + i omega M_G, one
// (K_G, M_G) pair per nodal entry.  Its pattern is the node graph of the mesh
// (two nodes of one tetrahedron share an edge), so row a holds a and the far
// ends of a's edges.  The nodal SSOR runs multicoloured like the edge one.
#include <algorithm>

#include "afem_hybrid.h"

namespace afem {

namespace {

constexpr int NODE_EDGE_MAX = 128;  // edges meeting at one node

// node -> incident edges; entry = edge << 1 | 1 when the node is the tail
// line(1,e) (coefficient -1 in G), edge << 1 when it is the head (+1)
__global__ void k_count_node_edges(const int32_t* __restrict__ line, int nline, int* __restrict__ cnt) {
  const int e = blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= nline) return;
  atomicAdd(cnt + line[2 * e] - 1, 1);
  atomicAdd(cnt + line[2 * e + 1] - 1, 1);
}

__global__ void k_fill_node_edges(const int32_t* __restrict__ line, int nline, const int32_t* __restrict__ nptr,
                                  int* __restrict__ cursor, int32_t* __restrict__ nlist) {
  const int e = blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= nline) return;
  const int a = line[2 * e] - 1, b = line[2 * e + 1] - 1;
  nlist[nptr[a] + atomicAdd(cursor + a, 1)] = (e << 1) | 1;
  nlist[nptr[b] + atomicAdd(cursor + b, 1)] = e << 1;
}

// per node: sort the incident edges (the fill order is not deterministic), then
// write the nodal pattern row: the node and the far ends of its edges, ascending
__global__ void k_node_rows(const int32_t* __restrict__ line, int node, const int32_t* __restrict__ nptr,
                            int32_t* __restrict__ nlist, const int32_t* __restrict__ rowptr, int32_t* __restrict__ col,
                            int32_t* __restrict__ diagpos, DevStatus* st) {
  const int a = blockIdx.x * blockDim.x + threadIdx.x;
  if (a >= node) return;
  const int p0 = nptr[a], p1 = nptr[a + 1];
  if (p1 - p0 > NODE_EDGE_MAX) {
    raise_status(st, DEV_DEGREE, a);
    return;
  }
  for (int i = p0 + 1; i < p1; ++i) {
    const int32_t v = nlist[i];
    int j = i - 1;
    while (j >= p0 && nlist[j] > v) {
      nlist[j + 1] = nlist[j];
      --j;
    }
    nlist[j + 1] = v;
  }
  const int r0 = rowptr[a];
  int len = 0;
  col[r0 + len++] = a;
  for (int i = p0; i < p1; ++i) {
    const int e = nlist[i] >> 1;
    const int far = (nlist[i] & 1) ? line[2 * e + 1] - 1 : line[2 * e] - 1;
    // insertion keeps the row ascending (a mesh has no repeated edge)
    int j = len - 1;
    while (j >= 0 && col[r0 + j] > far) {
      col[r0 + j + 1] = col[r0 + j];
      --j;
    }
    col[r0 + j + 1] = far;
    ++len;
  }
  for (int k = 0; k < len; ++k)
    if (col[r0 + k] == a) diagpos[a] = r0 + k;
}

__global__ void k_node_row_len(const int32_t* __restrict__ nptr, int node, int32_t* __restrict__ len) {
  const int a = blockIdx.x * blockDim.x + threadIdx.x;
  if (a < node) len[a] = 1 + nptr[a + 1] - nptr[a];
}

// A_G = G^T P (K, M) P G, thread per nodal row (a fixed summation order)
__global__ void k_node_values(const int32_t* __restrict__ line, const uint8_t* __restrict__ bc, int node,
                              const int32_t* __restrict__ nptr, const int32_t* __restrict__ nlist,
                              const int32_t* __restrict__ erow, const int32_t* __restrict__ ecol,
                              const double2* __restrict__ ekm, const int32_t* __restrict__ rowptr,
                              const int32_t* __restrict__ col, double2* __restrict__ km, uint8_t* __restrict__ live) {
  const int a = blockIdx.x * blockDim.x + threadIdx.x;
  if (a >= node) return;
  const int r0 = rowptr[a], r1 = rowptr[a + 1];
  for (int k = r0; k < r1; ++k) km[k] = make_double2(0.0, 0.0);
  bool any = false;
  for (int i = nptr[a]; i < nptr[a + 1]; ++i) {
    const int e = nlist[i] >> 1;
    if (bc[e]) continue;
    any = true;
    const double ga = (nlist[i] & 1) ? -1.0 : 1.0;
    for (int k = erow[e]; k < erow[e + 1]; ++k) {
      const int f = ecol[k];
      if (bc[f]) continue;
      const double2 v = ekm[k];
      const int f1 = line[2 * f] - 1, f2 = line[2 * f + 1] - 1;
      for (int q = r0; q < r1; ++q) {
        const int b = col[q];
        if (b == f2) { km[q].x += ga * v.x; km[q].y += ga * v.y; }
        else if (b == f1) { km[q].x -= ga * v.x; km[q].y -= ga * v.y; }
      }
    }
  }
  live[a] = any ? 1 : 0;
}

__global__ void k_node_seg(const int32_t* __restrict__ ptr, int nseg, int node, uint8_t* __restrict__ seg) {
  const int a = blockIdx.x * blockDim.x + threadIdx.x;
  if (a >= node) return;
  int k = 0;
  while (k + 1 < nseg && a >= ptr[k + 1]) ++k;
  seg[a] = (uint8_t)k;
}

inline unsigned nblk(long n, int t) { return (unsigned)((n + t - 1) / t); }

}  // namespace

void hybrid_prepare(afem_ctx* c) {
  AFEM_REQUIRE(c->node > 0 && c->nline > 0 && c->line.p, AFEM_ESTATE,
               "hybrid preconditioner: needs the mesh (not available for a system loaded in split layout)");
  AFEM_REQUIRE(c->assembled, AFEM_ESTATE, "hybrid preconditioner: assemble first");
  if (!c->hyb) c->hyb = new HybridState();
  HybridState* h = c->hyb;
  cudaStream_t s = c->stream;
  const int node = c->node;
  if (h->node != node || h->nline != c->nline || !h->pattern_ready) {
    h->node = node;
    h->nline = c->nline;
    DBuf<int32_t> cnt, cursor, len;
    cnt.alloc(node);
    cnt.zero(s);
    k_count_node_edges<<<nblk(c->nline, 256), 256, 0, s>>>(c->line.p, c->nline, cnt.p);
    count_launch();
    h->nptr.alloc(node + 1);
    exclusive_scan(cnt.p, h->nptr.p, node, s, nullptr);
    h->nlist.alloc(2L * c->nline);
    cursor.alloc(node);
    cursor.zero(s);
    k_fill_node_edges<<<nblk(c->nline, 256), 256, 0, s>>>(c->line.p, c->nline, h->nptr.p, cursor.p, h->nlist.p);
    count_launch();
    len.alloc(node);
    k_node_row_len<<<nblk(node, 256), 256, 0, s>>>(h->nptr.p, node, len.p);
    count_launch();
    h->rowptr.alloc(node + 1);
    long nnz = 0;
    exclusive_scan(len.p, h->rowptr.p, node, s, &nnz);
    h->nnz = nnz;
    h->col.alloc(nnz);
    AFEM_CUDA(cudaMemsetAsync(h->col.p, 0xff, sizeof(int32_t) * nnz, s));  // -1: a row left unwritten shows
    h->diagpos.alloc(node);
    k_node_rows<<<nblk(node, 128), 128, 0, s>>>(c->line.p, node, h->nptr.p, h->nlist.p, h->rowptr.p, h->col.p,
                                                 h->diagpos.p, c->status.p);
    count_launch();
    check_status(c, "hybrid preconditioner: more than 128 edges meet at one node");
    std::vector<int32_t> rp(node + 1), cl(nnz), pm(node), cptr(256), dp(node);
    std::vector<uint8_t> color(node);
    h->rowptr.download(rp.data(), node + 1, s);
    h->col.download(cl.data(), nnz, s);
    AFEM_CUDA(cudaStreamSynchronize(s));
    // every row: ascending node ids within 0..node-1, holding its own node once
    for (int a = 0; a < node; ++a) {
      int d = -1;
      for (int k = rp[a]; k < rp[a + 1]; ++k) {
        AFEM_REQUIRE(cl[k] >= 0 && cl[k] < node && (k == rp[a] || cl[k] > cl[k - 1]), AFEM_EPATTERN,
                     "hybrid preconditioner: the node graph row of node " + std::to_string(a) + " is malformed");
        if (cl[k] == a) d = k;
      }
      AFEM_REQUIRE(d >= 0, AFEM_EPATTERN, "hybrid preconditioner: node " + std::to_string(a) + " misses its diagonal");
      dp[a] = d;
    }
    h->diagpos.upload(dp.data(), node, s);
    // multicolour order of the node graph (host greedy colouring, as for the edges)
    const int nc = compute_coloring(node, rp.data(), cl.data(), color.data(), pm.data(), cptr.data(), 255);
    AFEM_REQUIRE(nc > 0, AFEM_EPATTERN, "hybrid preconditioner: more than 255 colours in the node graph");
    h->ncolors = nc;
    h->color.upload(color.data(), node, s);
    h->perm.upload(pm.data(), node, s);
    h->cptr.upload(cptr.data(), nc + 1, s);
    h->km.alloc(nnz);
    h->live.alloc(node);
    h->pattern_ready = true;
    h->values_gen = -1;
  }
  if (h->values_gen != c->assemble_gen) {
    k_node_values<<<nblk(node, 128), 128, 0, s>>>(c->line.p, c->bc.p, node, h->nptr.p, h->nlist.p, c->rowptr.p,
                                                   c->col.p, c->km.p, h->rowptr.p, h->col.p, h->km.p, h->live.p);
    count_launch();
    h->values_gen = c->assemble_gen;
    h->kmf_valid = false;
  }
  if (c->nseg > 0 && (int)h->seg_nseg != c->nseg) {
    DBuf<int32_t> ptr;
    ptr.upload(c->seg_node_ptr.data(), c->nseg + 1, s);
    h->seg.alloc(node);
    k_node_seg<<<nblk(node, 256), 256, 0, s>>>(ptr.p, c->nseg, node, h->seg.p);
    count_launch();
    AFEM_CUDA(cudaStreamSynchronize(s));
    h->seg_nseg = c->nseg;
  }
  AFEM_CUDA(cudaStreamSynchronize(s));
}

void hybrid_invalidate(afem_ctx* c) {
  if (c->hyb) {
    c->hyb->pattern_ready = false;
    c->hyb->seg_nseg = 0;
  }
}

void hybrid_destroy(afem_ctx* c) {
  delete c->hyb;
  c->hyb = nullptr;
}

// Host only: the nodal matrix of the last preparation, for tests.
void hybrid_export(afem_ctx* c, int* node, long* nnz, int32_t* rowptr, int32_t* col, double* km) {
  hybrid_prepare(c);
  HybridState* h = c->hyb;
  if (node) *node = h->node;
  if (nnz) *nnz = h->nnz;
  cudaStream_t s = c->stream;
  if (rowptr) h->rowptr.download(rowptr, h->node + 1, s);
  if (col) h->col.download(col, h->nnz, s);
  if (km) h->km.download(reinterpret_cast<double2*>(km), h->nnz, s);
  AFEM_CUDA(cudaStreamSynchronize(s));
}

}  // namespace afem
