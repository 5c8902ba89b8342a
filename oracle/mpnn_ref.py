"""CPU reference of the learned preconditioner network -- TEST INFRASTRUCTURE ONLY.

Message passing over the matrix graph of A = K + i*omega*M (unknowns = mesh
edges, graph edges = off-diagonal nonzeros).  The device kernels
(actfemtide_b200/csrc/afem_mpnn.cu) implement the same network; this module is
the checker for their forward values and gradients (FP64 here, with BF16
rounding of weights and activations emulated where the device rounds).

Network (width H = 48, L = 6 layers):
  s_i      = sqrt(|A_ii|)                       (Jacobi scale)
  rn       = r / rms(r)                           (scale normalisation)
  x_i      = [Re rn_i / s_i, Im rn_i / s_i, K_ii/|A_ii|, omega M_ii/|A_ii|, bc_i, 1, 0, 0]
  h^0      = x W_in                               (8 x H)
  X^l_i    = [h^l_i | sum_j a_ij h^l_j | sum_j b_ij h^l_j],  a_ij = K_ij/(s_i s_j), b_ij = omega M_ij/(s_i s_j)
  h^{l+1}  = h^l + relu(X^l W_l + c_l)            (3H x H)
  o        = h^L W_out                            (H x 2)
  z_i      = r_i / s_i^2 + rms(r) * (o_i0 + i o_i1) / s_i   (Jacobi term + learned correction)
Loss of one residual: ||A z - r||^2 / ||r||^2.
"""
from __future__ import annotations

import numpy as np

H = 48
L = 6
F_IN = 8


def bf16_round(a):
    """Round float values to bfloat16 (round to nearest even), returned as float64."""
    a = np.asarray(a, dtype=np.float32)
    u = a.view(np.uint32).astype(np.uint64)
    lsb = (u >> 16) & 1
    u = (u + 0x7FFF + lsb) & 0xFFFF0000
    return u.astype(np.uint32).view(np.float32).astype(np.float64)


class Graph:
    """Off-diagonal CSR of A with the normalised edge weights a_ij, b_ij and per-row features."""

    def __init__(self, rowptr, col, K, M, diagpos, omega, bc):
        n = len(rowptr) - 1
        self.n = n
        d = K[diagpos] + 1j * omega * M[diagpos]
        self.s = np.sqrt(np.abs(d))
        rows = np.repeat(np.arange(n), np.diff(rowptr))
        off = col != rows
        self.rows = rows[off]
        self.cols = col[off]
        ss = self.s[self.rows] * self.s[self.cols]
        self.a = K[off] / ss
        self.b = omega * M[off] / ss
        self.feat = np.stack([K[diagpos] / np.abs(d), omega * M[diagpos] / np.abs(d), bc.astype(np.float64),
                              np.ones(n)], axis=1)
        self.K, self.M, self.omega = K, M, omega
        self.rowptr, self.col = rowptr, col

    def agg(self, h, w):
        out = np.zeros_like(h)
        np.add.at(out, self.rows, w[:, None] * h[self.cols])
        return out

    def apply_A(self, z):
        rows = np.repeat(np.arange(self.n), np.diff(self.rowptr))
        Az = np.zeros(self.n, np.complex128)
        np.add.at(Az, rows, (self.K + 1j * self.omega * self.M) * z[self.col])
        return Az

    def apply_Aconj(self, z):
        rows = np.repeat(np.arange(self.n), np.diff(self.rowptr))
        Az = np.zeros(self.n, np.complex128)
        np.add.at(Az, rows, (self.K - 1j * self.omega * self.M) * z[self.col])
        return Az


def init_params(seed=0, scale=0.5):
    rng = np.random.default_rng(seed)
    P = {"W_in": rng.standard_normal((F_IN, H)) * scale / np.sqrt(F_IN)}
    for l in range(L):
        P[f"W{l}"] = rng.standard_normal((3 * H, H)) * scale / np.sqrt(3 * H)
        P[f"c{l}"] = np.zeros(H)
    P["W_out"] = rng.standard_normal((H, 2)) * scale / np.sqrt(H)
    return P


def inputs(g: Graph, r):
    rms = np.sqrt(np.mean(np.abs(r) ** 2))
    rn = r / rms
    x = np.zeros((g.n, F_IN))
    x[:, 0] = rn.real / g.s
    x[:, 1] = rn.imag / g.s
    x[:, 2:6] = g.feat
    return x, rms


def forward(P, g: Graph, r, bf16=False):
    rd = bf16_round if bf16 else (lambda v: v)
    x, rms = inputs(g, r)
    h = rd(x @ rd(P["W_in"]))
    cache = {"x": x, "rms": rms, "h": [h], "X": [], "Y": []}
    for l in range(L):
        X = np.concatenate([h, g.agg(h, g.a), g.agg(h, g.b)], axis=1)
        X = rd(X)
        Y = X @ rd(P[f"W{l}"]) + P[f"c{l}"]
        h = rd(h + np.maximum(Y, 0.0))
        cache["X"].append(X)
        cache["Y"].append(Y)
        cache["h"].append(h)
    o = h @ rd(P["W_out"])
    z = r / g.s ** 2 + rms * (o[:, 0] + 1j * o[:, 1]) / g.s
    cache["o"] = o
    return z, cache


def loss(P, g: Graph, r, bf16=False):
    z, cache = forward(P, g, r, bf16)
    res = g.apply_A(z) - r
    rn2 = np.sum(np.abs(r) ** 2)
    return float(np.sum(np.abs(res) ** 2) / rn2), (z, cache, res, rn2)


def grad(P, g: Graph, r, bf16=False):
    """Loss and gradients for every parameter (backpropagation, FP64)."""
    rd = bf16_round if bf16 else (lambda v: v)
    Lv, (z, cache, res, rn2) = loss(P, g, r, bf16)
    # dL/dz as a complex number gz = dL/dRe z + i dL/dIm z = 2 conj(A)^T res / ||r||^2 = 2 conj(A) res / ||r||^2
    gz = 2.0 * g.apply_Aconj(res) / rn2
    rms = cache["rms"]
    do = np.stack([(gz.real * rms / g.s), (gz.imag * rms / g.s)], axis=1)
    G = {}
    h = cache["h"][-1]
    G["W_out"] = h.T @ do
    dh = do @ rd(P["W_out"]).T
    for l in reversed(range(L)):
        X, Y = cache["X"][l], cache["Y"][l]
        dY = dh * (Y > 0)
        G[f"W{l}"] = X.T @ dY
        G[f"c{l}"] = dY.sum(axis=0)
        dX = dY @ rd(P[f"W{l}"]).T
        dh = dh + dX[:, :H] + g.agg(dX[:, H:2 * H], g.a) + g.agg(dX[:, 2 * H:], g.b)  # a, b symmetric
    G["W_in"] = cache["x"].T @ dh
    return Lv, G
