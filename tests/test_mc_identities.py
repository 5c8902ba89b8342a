"""Identities the multicolour COCG iteration rests on, checked on the CPU.

The device iteration of the gradient-corrected SSOR-COCG does not form the
textbook quantities where COCG13_single does (src/solver/COCG13_single.f90:
rho = r^T z after the preconditioner, x += alpha p beside r -= alpha q):

* the backward multicolour sweep takes rho = r^T M^-1 r as y^T D' y, where
  M = (D' + L) D'^-1 (D' + U) is SSOR in colour order, y = (D' + L)^-1 r is
  the forward sweep's output and D' the scaled diagonal.  That needs
  U = L^T in colour order, i.e. the assembled matrix (Dirichlet rows
  included) complex symmetric;
* the p update forms z + P G u on the fly and rho gets the nodal share
  r^T (P G u) = (G^T P r)^T u = t^T u from the backward nodal sweep.

Each identity is checked here on an oracle-assembled system, coloured by the
library's own host colouring (afem_coloring), to a relative 1e-12.
"""
import numpy as np
import scipy.sparse as sp
from scipy.sparse.linalg import spsolve_triangular

from actfemtide_b200 import synth
from actfemtide_b200.capi import ptr


def _system(oracle, gpulib):
    m = synth.tidal_box(6, 6, 6, seed=2, grf=True, block=False)
    of = oracle.OracleForward(m)
    A = of.assemble(m.freqs[0])
    S = A.to_scipy().tocsr()
    S.sort_indices()
    n = A.n
    # structural pattern (the assembled one, explicit zeros kept) for the colouring
    INU, IAU, INL, IAL = of.pat
    rows = np.concatenate([np.arange(n), np.repeat(np.arange(n), np.diff(INU)), np.repeat(np.arange(n), np.diff(INL))])
    cols = np.concatenate([np.arange(n), IAU - 1, IAL - 1])
    pat = sp.csr_matrix((np.ones(len(rows)), (rows, cols)), shape=(n, n))
    pat.sort_indices()
    rowptr = pat.indptr.astype(np.int32)
    col = pat.indices.astype(np.int32)
    color = np.zeros(n, np.uint8); perm = np.zeros(n, np.int32); cptr = np.zeros(256, np.int32)
    nc = gpulib.afem_coloring(n, ptr(rowptr), ptr(col), ptr(color), ptr(perm), ptr(cptr))
    assert nc > 1
    return m, of, A, S, color, perm


def _split(S, color):
    C = S.tocoo()
    lo = color[C.col] < color[C.row]
    up = color[C.col] > color[C.row]
    n = S.shape[0]
    L = sp.csr_matrix((C.data[lo], (C.row[lo], C.col[lo])), shape=(n, n))
    U = sp.csr_matrix((C.data[up], (C.row[up], C.col[up])), shape=(n, n))
    return L, U


def test_upper_part_is_the_transpose_in_colour_order(oracle, gpulib):
    _, _, A, S, color, _ = _system(oracle, gpulib)
    L, U = _split(S, color)
    diff = (U - L.T).tocsr()
    diff.eliminate_zeros()
    assert diff.nnz == 0  # COPY_UL and SET_BC keep the matrix exactly complex symmetric


def test_ssor_rho_equals_y_d_y(oracle, gpulib):
    _, _, A, S, color, perm = _system(oracle, gpulib)
    L, U = _split(S, color)
    n = A.n
    Dp = sp.diags(A.D)  # sd = 1, as in the solver's default
    P = sp.csr_matrix((np.ones(n), (np.arange(n), perm)), shape=(n, n))  # row k of P picks row perm[k]
    rng = np.random.default_rng(5)
    r = rng.standard_normal(n) + 1j * rng.standard_normal(n)
    # forward sweep y = (D' + L)^-1 r, backward z = (D' + U)^-1 D' y, both triangular in colour order
    Fl = (P @ (Dp + L) @ P.T).tocsr()
    y = P.T @ spsolve_triangular(Fl, P @ r, lower=True)
    Bu = (P @ (Dp + U) @ P.T).tocsr()
    z = P.T @ spsolve_triangular(Bu, P @ (A.D * y), lower=False)
    rho_textbook = np.sum(r * z)          # unconjugated, as COCG
    rho_diag = np.sum(A.D * y * y)        # what the backward sweep sums
    scale = np.sum(np.abs(r * z))
    assert abs(rho_textbook - rho_diag) <= 1e-12 * scale, (rho_textbook, rho_diag)


def test_nodal_share_of_rho(oracle, gpulib):
    m, of, A, S, color, _ = _system(oracle, gpulib)
    n = A.n
    line = of.line
    free = (A.bc == 0).astype(float)
    # (G u)_e = u_head(e) - u_tail(e), head = line(2, e), tail = line(1, e); P drops Dirichlet edges
    G = sp.csr_matrix((np.concatenate([np.ones(n), -np.ones(n)]),
                       (np.concatenate([np.arange(n)] * 2), np.concatenate([line[:, 1] - 1, line[:, 0] - 1]))),
                      shape=(n, m.node))
    PG = sp.diags(free) @ G
    rng = np.random.default_rng(6)
    r = rng.standard_normal(n) + 1j * rng.standard_normal(n)
    u = rng.standard_normal(m.node) + 1j * rng.standard_normal(m.node)
    t = PG.T @ r                          # k_grad_t
    lhs = np.sum(r * (PG @ u))            # r^T (z + P G u) - r^T z
    rhs = np.sum(t * u)                   # the backward nodal sweep's partial sums
    scale = np.sum(np.abs(r) * np.abs(PG) @ np.abs(u))
    assert abs(lhs - rhs) <= 1e-12 * scale
