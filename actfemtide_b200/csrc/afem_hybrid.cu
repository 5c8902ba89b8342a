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

__global__ void k_gather_km(const double2* __restrict__ km, const int32_t* __restrict__ src, long cnt,
                            double2* __restrict__ out) {
  const long k = blockIdx.x * (long)blockDim.x + threadIdx.x;
  if (k < cnt) out[k] = km[src[k]];
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
    // The node graph, once per mesh, on the host: incident edges per node in
    // ascending edge order (edge << 1 | 1 at the tail line(1,e), edge << 1 at
    // the head), rows = the node and the far ends of its edges, ascending.
    const int nline = c->nline;
    std::vector<int32_t> ln(2L * nline);
    c->line.download(ln.data(), ln.size(), s);
    AFEM_CUDA(cudaStreamSynchronize(s));
    std::vector<int32_t> np(node + 1, 0);
    for (int e = 0; e < nline; ++e) {
      const int a = ln[2L * e] - 1, b = ln[2L * e + 1] - 1;
      AFEM_REQUIRE(a >= 0 && a < node && b >= 0 && b < node && a != b, AFEM_EINVAL,
                   "hybrid preconditioner: edge " + std::to_string(e + 1) + " has a bad node id");
      np[a + 1] += 1;
      np[b + 1] += 1;
    }
    for (int a = 0; a < node; ++a) {
      AFEM_REQUIRE(np[a + 1] <= NODE_EDGE_MAX, AFEM_EPATTERN,
                   "hybrid preconditioner: more than 128 edges meet at node " + std::to_string(a + 1));
      np[a + 1] += np[a];
    }
    std::vector<int32_t> nl(2L * nline), cur(np.begin(), np.end() - 1);
    for (int e = 0; e < nline; ++e) {
      nl[cur[ln[2L * e] - 1]++] = (e << 1) | 1;
      nl[cur[ln[2L * e + 1] - 1]++] = e << 1;
    }
    std::vector<int32_t> rp(node + 1, 0), dp(node);
    for (int a = 0; a < node; ++a) rp[a + 1] = rp[a] + 1 + (np[a + 1] - np[a]);
    const long nnz = rp[node];
    std::vector<int32_t> cl(nnz);
    for (int a = 0; a < node; ++a) {
      int32_t* row = cl.data() + rp[a];
      int len = 0;
      row[len++] = a;
      for (int q = np[a]; q < np[a + 1]; ++q) {
        const int e = nl[q] >> 1;
        row[len++] = (nl[q] & 1) ? ln[2L * e + 1] - 1 : ln[2L * e] - 1;
      }
      std::sort(row, row + len);
      for (int k = 0; k < len; ++k) {
        AFEM_REQUIRE(k == 0 || row[k] > row[k - 1], AFEM_EPATTERN,
                     "hybrid preconditioner: repeated edge at node " + std::to_string(a + 1));
        if (row[k] == a) dp[a] = rp[a] + k;
      }
    }
    h->nnz = nnz;
    h->nptr.upload(np.data(), np.size(), s);
    h->nlist.upload(nl.data(), nl.size(), s);
    h->rowptr.upload(rp.data(), rp.size(), s);
    h->col.upload(cl.data(), cl.size(), s);
    h->diagpos.upload(dp.data(), dp.size(), s);
    std::vector<int32_t> pm(node), cptr(256);
    std::vector<uint8_t> color(node);
    // multicolour order of the node graph (host greedy colouring, as for the edges)
    const int nc = compute_coloring(node, rp.data(), cl.data(), color.data(), pm.data(), cptr.data(), 255);
    AFEM_REQUIRE(nc > 0, AFEM_EPATTERN, "hybrid preconditioner: more than 255 colours in the node graph");
    h->ncolors = nc;
    h->color.upload(color.data(), node, s);
    h->perm.upload(pm.data(), node, s);
    h->cptr.upload(cptr.data(), nc + 1, s);
    // colour-ordered split rows of the node graph, built on the device like the edges'
    split_rows_device(c, h->rowptr.p, h->col.p, h->diagpos.p, h->color.p, h->perm.p, node, h->lptr, h->lcol, h->lsrc,
                      h->uptr, h->ucol, h->usrc, nullptr);
    h->lkm.alloc(h->lcol.n);
    h->ukm.alloc(h->ucol.n);
    h->km.alloc(nnz);
    h->live.alloc(node);
    h->pattern_ready = true;
    h->values_gen = -1;
  }
  if (h->values_gen != c->assemble_gen) {
    k_node_values<<<nblk(node, 128), 128, 0, s>>>(c->line.p, c->bc.p, node, h->nptr.p, h->nlist.p, c->rowptr.p,
                                                   c->col.p, c->km.p, h->rowptr.p, h->col.p, h->km.p, h->live.p);
    count_launch();
    if (h->lcol.n) {
      k_gather_km<<<nblk((long)h->lcol.n, 256), 256, 0, s>>>(h->km.p, h->lsrc.p, (long)h->lcol.n, h->lkm.p);
      count_launch();
    }
    if (h->ucol.n) {
      k_gather_km<<<nblk((long)h->ucol.n, 256), 256, 0, s>>>(h->km.p, h->usrc.p, (long)h->ucol.n, h->ukm.p);
      count_launch();
    }
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
