// Gradient-space (nodal) correction of the COCG preconditioner: device state.
#pragma once

#include "afem_internal.h"

namespace afem {

struct HybridState {
  int node = 0, nline = 0;
  long nnz = 0;
  bool pattern_ready = false;
  long values_gen = -1;         // assembly generation the values belong to
  DBuf<int32_t> nptr, nlist;    // node -> incident edges (edge << 1 | tail flag), ascending
  DBuf<int32_t> rowptr, col;    // nodal pattern (node graph), columns ascending
  DBuf<int32_t> diagpos;
  DBuf<double2> km;             // (K_G, M_G) per nodal entry
  DBuf<float2> kmf;             // FP32 copy for the mixed-precision inner solve
  bool kmf_valid = false;
  DBuf<uint8_t> live;           // 1 when the node has a non-Dirichlet edge
  DBuf<uint8_t> color;          // nodal multicolour order
  DBuf<int32_t> perm, cptr;
  int ncolors = 0;
  // rows in colour order, split into earlier-colour (l*) and later-colour (u*) parts;
  // *src = index of the entry in the nodal CSR, *km the values (FP64, FP32 copies)
  DBuf<int32_t> lptr, lcol, lsrc, uptr, ucol, usrc;
  DBuf<double2> lkm, ukm;
  DBuf<float2> lkmf, ukmf;
  DBuf<uint8_t> seg;            // packed batches: mesh of each node
  int seg_nseg = 0;
};

void hybrid_prepare(afem_ctx* c);     // pattern + colouring (once per mesh), values (once per assembly)
void hybrid_invalidate(afem_ctx* c);  // the mesh changed
void hybrid_destroy(afem_ctx* c);
void hybrid_export(afem_ctx* c, int* node, long* nnz, int32_t* rowptr, int32_t* col, double* km);

}  // namespace afem
