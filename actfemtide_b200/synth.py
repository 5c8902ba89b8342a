"""Seeded synthetic tidal-induction models on Kuhn-split box meshes.

The reference's own workflow builds its inputs offline (Gmsh meshes from
coastlines, OTPS tidal velocities, IGRF main field; ``Kikai/mesh/tetmeshgen.sh``,
``Kikai/fvxyz/mkfvxyz_mesh.sh``).  None of those inputs ship with it, so the
workloads here are generated: uniform hexahedral boxes, each hex split into six
tetrahedra along its main diagonal (the conforming Kuhn/Freudenthal split), with
the arrays laid out the way the reference's readers deliver them:

* ``xyz``  (node, 3) km, ``n4`` (ntet, 4) 1-based node ids, ``tag`` (ntet,)
  elementary volume tag (1 air, 2 ocean, >=3 land), as ``readmsh2`` fills
  ``h_mesh%xyz``, ``h_mesh%n4`` and ``h_mesh%n4flag(:,2)``
  (``src/common/m_mesh_type.f90:379-468``);
* ocean nodes are numbered first, so that ``readfxyz``/``readvxyz`` filling
  nodes ``1..nodes`` (``src/src_tide/m_readfvxyz.f90:7-62``) covers every node
  of every ocean tetrahedron;
* land tetrahedra (tag >= 3) come last, so ``sigma(iele - nphys1)`` indexes the
  per-land-element conductivity (``src/solver_mpi/forward_bxyz_mpi.f90:203``).

Every random quantity is drawn from ``numpy.random.default_rng(seed)``.
"""
from __future__ import annotations

import dataclasses
import math

import numpy as np

M2_PERIOD_S = 44714.0
# Tidal periods in hours used by the batched workload (M2, S2, N2, K2, K1, O1, P1, Q1).
BATCH_PERIODS_H = (12.4206, 12.0000, 12.6583, 11.9672, 23.9345, 25.8193, 24.0659, 26.8684)

SIGMA_AIR = 1e-8
SIGMA_SEA = 3.3
SIGMA_LAND = 0.01
SIGMA_BLOCK = 0.5
F_MAIN_NT = (30000.0, -3000.0, 35000.0)
SEA_DEPTH_KM = 5.0
SITE_DEPTH_KM = 0.001  # 1 m below the solid-earth surface


@dataclasses.dataclass
class TidalModel:
    """One forward problem: mesh, conductivity, tidal source, sites, bounds."""

    name: str
    xyz: np.ndarray          # (node, 3) float64 km
    n4: np.ndarray           # (ntet, 4) int32, 1-based
    tag: np.ndarray          # (ntet,) int32 elementary tag
    sigma_land: np.ndarray   # (nphys2,) float64 S/m, one per land tetrahedron (tag >= 3), in order
    nodes: int               # number of ocean-mesh nodes (source arrays cover 1..nodes)
    F: np.ndarray            # (nodes, 3) float64 nT
    v: np.ndarray            # (nodes, 3) complex128 m/s
    freqs: np.ndarray        # (nfreq,) Hz
    sites: np.ndarray        # (nobs, 3) km, already 1 m below the surface
    bounds: dict             # zmin, zmax, xout, yout for the Dirichlet boundary search
    sigma_air: float = SIGMA_AIR
    sigma_ocean: float = SIGMA_SEA
    seed: int = 0
    dims: tuple = (0, 0, 0)

    @property
    def node(self) -> int:
        return int(self.xyz.shape[0])

    @property
    def ntet(self) -> int:
        return int(self.n4.shape[0])

    @property
    def nphys1(self) -> int:
        return self.ntet - int(self.sigma_land.shape[0])

    def sigma_per_tet(self) -> np.ndarray:
        """Resolved conductivity per tetrahedron, as GENMAT selects it with a per-element file."""
        s = np.empty(self.ntet, dtype=np.float64)
        s[self.tag == 1] = self.sigma_air
        s[self.tag == 2] = self.sigma_ocean
        s[self.nphys1:] = self.sigma_land
        return s


def kuhn_box(nx: int, ny: int, nz: int, xb=(-50.0, 50.0), yb=(-50.0, 50.0), zb=(-50.0, 50.0)):
    """Nodes and Kuhn-split tetrahedra of an nx*ny*nz hex box.

    Returns (xyz, n4, hex_of_tet, centroid) with n4 0-based here; every
    tetrahedron is oriented so that the reference's signed volume
    ``volume(xx(:,1), xx(:,5), -xx(:,4))`` (``src/solver/m_fem_util.f90:22``)
    is positive.
    """
    xs = np.linspace(xb[0], xb[1], nx + 1)
    ys = np.linspace(yb[0], yb[1], ny + 1)
    zs = np.linspace(zb[0], zb[1], nz + 1)
    X, Y, Z = np.meshgrid(xs, ys, zs, indexing="ij")
    xyz = np.stack([X.ravel(order="F"), Y.ravel(order="F"), Z.ravel(order="F")], axis=1)

    def nid(i, j, k):
        return i + (nx + 1) * (j + (ny + 1) * k)

    I, J, K = np.meshgrid(np.arange(nx), np.arange(ny), np.arange(nz), indexing="ij")
    I = I.ravel(order="F"); J = J.ravel(order="F"); K = K.ravel(order="F")
    nhex = I.size
    e = np.eye(3, dtype=np.int64)
    perms = [(0, 1, 2), (0, 2, 1), (1, 0, 2), (1, 2, 0), (2, 0, 1), (2, 1, 0)]
    tets = np.empty((nhex, 6, 4), dtype=np.int64)
    base = np.stack([I, J, K], axis=1)
    for t, (a, b, _c) in enumerate(perms):
        p0 = base
        p1 = base + e[a]
        p2 = base + e[a] + e[b]
        p3 = base + 1
        for q, p in enumerate((p0, p1, p2, p3)):
            tets[:, t, q] = nid(p[:, 0], p[:, 1], p[:, 2])
    tets = tets.reshape(-1, 4)
    # orient: reference volume = 1/6 * ((p4-p3) x (p1-p3)) . (p2-p3)
    P = xyz[tets]
    vol = np.einsum("ij,ij->i", np.cross(P[:, 3] - P[:, 2], P[:, 0] - P[:, 2]), P[:, 1] - P[:, 2]) / 6.0
    neg = vol < 0
    tets[neg, 0], tets[neg, 1] = tets[neg, 1].copy(), tets[neg, 0].copy()
    hex_of_tet = np.repeat(np.arange(nhex), 6)
    centroid = xyz[tets].mean(axis=1)
    return xyz, tets, hex_of_tet, centroid


def gaussian_random_field(shape, spacing, corr_km: float, rng) -> np.ndarray:
    """Zero-mean unit-variance Gaussian random field with a Gaussian covariance of length corr_km."""
    noise = rng.standard_normal(shape)
    F = np.fft.rfftn(noise)
    ks = [np.fft.fftfreq(n, d=h) * 2 * np.pi for n, h in zip(shape[:-1], spacing[:-1])]
    ks.append(np.fft.rfftfreq(shape[-1], d=spacing[-1]) * 2 * np.pi)
    K2 = sum(np.meshgrid(*[k ** 2 for k in ks], indexing="ij"))
    F *= np.exp(-K2 * corr_km ** 2 / 4.0)
    f = np.fft.irfftn(F, s=shape)
    f -= f.mean()
    f /= f.std()
    return f


def _smooth_delta(x, y, rng, amp=0.1):
    """Smooth seeded perturbation with |delta| <= amp over the domain."""
    out = np.zeros_like(x)
    wsum = 0.0
    for _ in range(4):
        kx, ky = rng.uniform(-1, 1, size=2) * (2 * np.pi / 100.0) * 2
        ph = rng.uniform(0, 2 * np.pi)
        w = rng.uniform(0.5, 1.0)
        out += w * np.sin(kx * x + ky * y + ph)
        wsum += w
    return amp * out / wsum


def _velocity(xyz_nodes, seed: int):
    rng = np.random.default_rng(seed)
    theta = rng.uniform(0, 2 * np.pi)
    phi = rng.uniform(0, 2 * np.pi)
    delta = _smooth_delta(xyz_nodes[:, 0], xyz_nodes[:, 1], rng)
    amp = 0.05 * (1.0 + delta) * np.exp(1j * phi)
    v = np.zeros((xyz_nodes.shape[0], 3), dtype=np.complex128)
    v[:, 0] = amp * math.cos(theta)
    v[:, 1] = amp * math.sin(theta)
    return v


def surface_z(x, y):
    """Top of the solid earth: the seafloor (-5 km) where x < 0, the land surface (0) elsewhere."""
    return np.where(np.asarray(x) < 0.0, -SEA_DEPTH_KM, 0.0)


def tidal_box(nx: int, ny: int, nz: int, *, seed: int = 0, field_seed: int | None = None,
              grf: bool = False, block: bool = True, site_grid=None, freqs=None,
              vel_seed: int | None = None, name: str = "box", half_km: float = 50.0,
              zhalf_km: float | None = None) -> TidalModel:
    """Build one synthetic tidal-induction model on an nx*ny*nz Kuhn box over [-50,50]^3 km.

    Conductivity by tetrahedron centroid: air (z>0) 1e-8 S/m (tag 1); sea layer
    (-5<=z<=0, x<0) 3.3 S/m (tag 2); sea-layer land (x>=0) 0.01 S/m; subsurface
    0.01 S/m, or with ``grf`` a log10-normal Gaussian random field (mean -2,
    std 1, correlation 8 km, clipped to [-4, 0.5]); optional 0.5 S/m block at
    x in [5,15], y in [-5,5], z in [-15,-5].  Land tetrahedra carry tag 3
    (tag 4 inside the block).
    """
    zh = half_km if zhalf_km is None else zhalf_km
    xyz, tets, hex_of_tet, cen = kuhn_box(nx, ny, nz, (-half_km, half_km), (-half_km, half_km), (-zh, zh))
    cx, cy, cz = cen[:, 0], cen[:, 1], cen[:, 2]
    tag = np.full(tets.shape[0], 3, dtype=np.int32)
    tag[cz > 0.0] = 1
    ocean = (cz <= 0.0) & (cz >= -SEA_DEPTH_KM) & (cx < 0.0)
    tag[ocean] = 2
    sig = np.full(tets.shape[0], SIGMA_LAND)
    inblock = np.zeros(tets.shape[0], dtype=bool)
    if block:
        inblock = (cx >= 5) & (cx <= 15) & (cy >= -5) & (cy <= 5) & (cz >= -15) & (cz <= -5) & (tag == 3)
        tag[inblock] = 4
        sig[inblock] = SIGMA_BLOCK
    if grf:
        rng = np.random.default_rng(1 if field_seed is None else field_seed)
        g = gaussian_random_field((nx, ny, nz), (2 * half_km / nx, 2 * half_km / ny, 2 * zh / nz), 8.0, rng)
        logs = np.clip(-2.0 + 1.0 * g.ravel(order="F"), -4.0, 0.5)
        sub = (cz < -SEA_DEPTH_KM) & (tag >= 3) & ~inblock
        sig[sub] = 10.0 ** logs[hex_of_tet[sub]]

    # tetrahedra: air, ocean, land (stable within each group)
    order = np.concatenate([np.nonzero(tag == 1)[0], np.nonzero(tag == 2)[0], np.nonzero(tag >= 3)[0]])
    tets = tets[order]; tag = tag[order]; sig = sig[order]
    # nodes: those of ocean tetrahedra first, each group in grid order
    is_ocean_node = np.zeros(xyz.shape[0], dtype=bool)
    is_ocean_node[tets[tag == 2].ravel()] = True
    perm = np.concatenate([np.nonzero(is_ocean_node)[0], np.nonzero(~is_ocean_node)[0]])
    inv = np.empty_like(perm); inv[perm] = np.arange(perm.size)
    xyz = xyz[perm]
    tets = inv[tets]
    nodes = int(is_ocean_node.sum())

    F = np.tile(np.array(F_MAIN_NT), (nodes, 1))
    v = _velocity(xyz[:nodes], seed if vel_seed is None else vel_seed)
    if site_grid is None:
        site_grid = (-40.0, -20.0, 0.0, 20.0, 40.0)
    gx, gy = np.meshgrid(np.asarray(site_grid), np.asarray(site_grid), indexing="ij")
    sx = gx.ravel(); sy = gy.ravel()
    sites = np.stack([sx, sy, surface_z(sx, sy) - SITE_DEPTH_KM], axis=1)
    if freqs is None:
        freqs = np.array([1.0 / M2_PERIOD_S])
    land = tag >= 3
    return TidalModel(
        name=name, xyz=np.ascontiguousarray(xyz), n4=np.ascontiguousarray((tets + 1).astype(np.int32)),
        tag=tag.astype(np.int32), sigma_land=np.ascontiguousarray(sig[land]), nodes=nodes,
        F=np.ascontiguousarray(F), v=np.ascontiguousarray(v), freqs=np.asarray(freqs, dtype=np.float64),
        sites=np.ascontiguousarray(sites),
        bounds=dict(zmin=-zh, zmax=zh, xout=half_km, yout=half_km), seed=seed, dims=(nx, ny, nz))


def small_model(seed: int = 0) -> TidalModel:
    """20x20x20 hexes (48,000 tets, 59,660 edges): the CPU-runnable plain-method case."""
    return tidal_box(20, 20, 20, seed=seed, name="box20")


def large_model(seed: int = 0) -> TidalModel:
    """96x96x64 hexes (3,538,944 tets, 4,193,536 edges) with a log-normal subsurface, 400 sites."""
    grid = np.linspace(-47.5, 47.5, 20)
    return tidal_box(96, 96, 64, seed=seed, grf=True, block=False, site_grid=grid, name="box96x96x64")


def tiny_model(nx=2, ny=2, nz=4, seed: int = 0) -> TidalModel:
    """A few hexes over [-10,10]^3 km (5 km cells, so the sea layer holds whole cells)."""
    return tidal_box(nx, ny, nz, seed=seed, block=False, site_grid=(-5.0, 5.0), half_km=10.0,
                     name=f"box{nx}x{ny}x{nz}")
