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


def kuhn_box(nx: int, ny: int, nz: int, xb=(-50.0, 50.0), yb=(-50.0, 50.0), zb=(-50.0, 50.0), zs=None):
    """Nodes and Kuhn-split tetrahedra of an nx*ny*nz hex box.

    Returns (xyz, n4, hex_of_tet, centroid) with n4 0-based here; every
    tetrahedron is oriented so that the reference's signed volume
    ``volume(xx(:,1), xx(:,5), -xx(:,4))`` (``src/solver/m_fem_util.f90:22``)
    is positive.  ``zs`` (nz+1 ascending levels) replaces the uniform z spacing.
    """
    xs = np.linspace(xb[0], xb[1], nx + 1)
    ys = np.linspace(yb[0], yb[1], ny + 1)
    zs = np.linspace(zb[0], zb[1], nz + 1) if zs is None else np.asarray(zs, dtype=np.float64)
    assert zs.shape == (nz + 1,)
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
    f = np.fft.irfftn(F, s=shape, axes=tuple(range(len(shape))))
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


# ----------------------------------------------------------------------------- packed batches
@dataclasses.dataclass
class PackedModels:
    """Independent meshes packed into one union mesh (one system per mesh in one solve).

    Mesh k owns nodes ``node_ptr[k] .. node_ptr[k+1]-1`` (0-based) and its
    tetrahedra follow mesh k-1's; node ids, tetrahedra, tags and
    conductivities are the parts' own, offset.  The source arrays cover every
    union node (zero outside each part's ocean nodes), which gives each part
    exactly its own right-hand side.
    """

    parts: list
    xyz: np.ndarray
    n4: np.ndarray
    tag: np.ndarray
    sigma_tet: np.ndarray
    F: np.ndarray
    v: np.ndarray
    node_ptr: np.ndarray
    tet_ptr: np.ndarray
    bounds: dict

    @property
    def nseg(self) -> int:
        return len(self.parts)


def uneven_models(count: int = 24, seed: int = 0, nmin: int = 8, nmax: int = 32) -> list:
    """``count`` meshes of n x n x round(3n/4) cells over [-50,50]^3 km, n uniform in [nmin, nmax].

    Each mesh has its own seeded log-normal subsurface (``grf``), conductive
    block and velocity pattern; all share the M2 frequency and the 5x5 site grid.
    """
    rng = np.random.default_rng(seed)
    ns = rng.integers(nmin, nmax + 1, size=count)
    out = []
    for k, n in enumerate(ns):
        n = int(n)
        out.append(tidal_box(n, n, max(2, int(round(0.75 * n))), seed=seed * 1000 + k, field_seed=seed * 1000 + k + 1,
                             grf=True, name=f"uneven{k}_n{n}"))
    return out


def pack(models) -> PackedModels:
    """Union of independent meshes with the same Dirichlet bounds (see :class:`PackedModels`)."""
    b0 = models[0].bounds
    for m in models:
        if m.bounds != b0:
            raise ValueError("packed meshes must share the Dirichlet bounds")
    node_ptr = np.zeros(len(models) + 1, np.int32)
    tet_ptr = np.zeros(len(models) + 1, np.int32)
    for k, m in enumerate(models):
        node_ptr[k + 1] = node_ptr[k] + m.node
        tet_ptr[k + 1] = tet_ptr[k] + m.ntet
    total = int(node_ptr[-1])
    F = np.zeros((total, 3)); v = np.zeros((total, 3), np.complex128)
    for k, m in enumerate(models):
        F[node_ptr[k]:node_ptr[k] + m.nodes] = m.F
        v[node_ptr[k]:node_ptr[k] + m.nodes] = m.v
    return PackedModels(
        parts=list(models),
        xyz=np.ascontiguousarray(np.concatenate([m.xyz for m in models])),
        n4=np.ascontiguousarray(np.concatenate([m.n4 + node_ptr[k] for k, m in enumerate(models)]).astype(np.int32)),
        tag=np.ascontiguousarray(np.concatenate([m.tag for m in models]).astype(np.int32)),
        sigma_tet=np.ascontiguousarray(np.concatenate([m.sigma_per_tet() for m in models])),
        F=F, v=v, node_ptr=node_ptr, tet_ptr=tet_ptr, bounds=dict(b0))


# ----------------------------------------------------------------------------- reference file formats
def _write_msh(path, xyz, elems, etype):
    """Gmsh 2.2 ASCII as readmsh2 reads it (src/common/m_mesh_type.f90:379-468): two tags per element."""
    with open(path, "w") as f:
        f.write("$MeshFormat\n2.2 0 8\n$EndMeshFormat\n$Nodes\n")
        f.write(f"{xyz.shape[0]}\n")
        for i, p in enumerate(xyz):
            f.write(f"{i + 1} {float(p[0])!r} {float(p[1])!r} {float(p[2])!r}\n")
        f.write("$EndNodes\n$Elements\n")
        f.write(f"{len(elems)}\n")
        for k, (tag, nodes) in enumerate(elems):
            f.write(f"{k + 1} {etype} 2 {tag} {tag} " + " ".join(str(int(n)) for n in nodes) + "\n")
        f.write("$EndElements\n")


def write_reference_inputs(m: TidalModel, outdir: str, line=None, n6line=None, site_names=None,
                           plan_view=None, utm_sites=None, seafloor_view=None) -> str:
    """Write model m as the files the reference's tide forward reads; returns the ctl path.

    em3d.msh (tetrahedra, tags = elementary volume), polygonz.msh (top-of-earth
    triangles with z), ocean.msh (only its node count is used), lineinfo.dat
    (READLINE's layout; numbering from line/n6line when given), fxyz_mesh /
    vxyz_mesh (readfxyz / readvxyz records), cond_test.msh (READCOND: 11 header
    lines, nphys2, index and resistivity), tide_fwd.ctl (readparam's record
    order, labels in the first 20 columns, xyz sites given 1 m below the surface).
    utm_sites = (zone, lonorigin, latorigin, lonlat): sites given as longitude /
    latitude (lonlat: nobs x 2 degrees) in UTM zone `zone` (lonlatflag 1).
    plan_view = (xyfilehead, nx, ny, depth): the nx x ny plan view (ixyflag 1) at a
    constant depth (ixydepth 1), or 1 m below the seafloor when depth is None
    (ixydepth 2); seafloor_view = xyfilehead: the polygon_ki triangles' plan view
    (ixyflag 2).  The seafloor views also get polygon_ki.msh (the surface grid's
    triangles) and ki23dptr.dat (each of its nodes' 3-D surface node at z = 0 and
    seafloor node at the top of the solid earth; the mesh needs a node layer there).
    """
    import os
    os.makedirs(outdir, exist_ok=True)
    p = lambda name: os.path.join(outdir, name)  # noqa: E731
    _write_msh(p("em3d.msh"), m.xyz, [(int(t), nd) for t, nd in zip(m.tag, m.n4)], 4)
    # surface: nodes of the top grid with the solid-earth height
    nx, ny, _ = m.dims
    half = m.bounds["xout"]
    xs = np.linspace(-half, half, nx + 1)
    ys = np.linspace(-half, half, ny + 1)
    X, Y = np.meshgrid(xs, ys, indexing="ij")
    sxyz = np.stack([X.ravel(), Y.ravel(), surface_z(X.ravel(), Y.ravel())], axis=1)
    tris = []
    for i in range(nx):
        for j in range(ny):
            a = i * (ny + 1) + j + 1
            b = (i + 1) * (ny + 1) + j + 1
            tris.append((1, (a, b, b + 1)))
            tris.append((1, (a, b + 1, a + 1)))
    _write_msh(p("polygonz.msh"), sxyz, tris, 2)
    if seafloor_view is not None or (plan_view is not None and plan_view[3] is None):
        _write_msh(p("polygon_ki.msh"), np.stack([X.ravel(), Y.ravel(), np.zeros(X.size)], axis=1), tris, 2)
        key = {tuple(np.round(c, 6)): i + 1 for i, c in enumerate(m.xyz)}
        with open(p("ki23dptr.dat"), "w") as f:
            f.write(f"{sxyz.shape[0]}\n")
            for x, y, zs in sxyz:
                top = key[(round(float(x), 6), round(float(y), 6), 0.0)]
                bot = key[(round(float(x), 6), round(float(y), 6), round(float(zs), 6))]
                f.write(f"{top} {bot}\n")
    _write_msh(p("ocean.msh"), m.xyz[: m.nodes], [], 4)
    if line is not None:
        with open(p("lineinfo.dat"), "w") as f:
            f.write(f"{line.shape[0]:12d}\n")
            for a, b in line:
                f.write(f"{a:10d}{b:10d}\n")
            f.write(f"{n6line.shape[0]:12d}\n")
            for r in n6line:
                f.write("".join(f"{v:10d}" for v in r) + "\n")
    with open(p("fxyz_mesh"), "w") as f:
        for i in range(m.nodes):
            F = m.F[i]
            f.write(f"  0.0 0.0 {float(m.xyz[i, 2])!r} {float(F[0])!r} {float(F[1])!r} {float(F[2])!r} "
                    f"{float(np.linalg.norm(F))!r}\n")
    with open(p("vxyz_mesh"), "w") as f:
        for i in range(m.nodes):
            v = m.v[i]
            f.write(f"  0.0 0.0 {float(m.xyz[i, 2])!r} ({float(v[0].real)!r},{float(v[0].imag)!r}) "
                    f"({float(v[1].real)!r},{float(v[1].imag)!r}) {i + 1}\n")
    with open(p("cond_test.msh"), "w") as f:
        for k in range(11):
            f.write(f"# header line {k + 1}\n")
        f.write(f"{len(m.sigma_land)}\n")
        for k, s in enumerate(m.sigma_land):
            f.write(f"{m.nphys1 + k + 1} {float(1.0 / s)!r}\n")
    names = site_names or [f"S{k + 1:03d}" for k in range(m.sites.shape[0])]
    lab = lambda s: (s + " " * 20)[:20]  # noqa: E731
    rows = [lab("itopoflag") + "0",
            lab("mesh file") + p("em3d.msh"), lab("2d triangle z file") + p("polygonz.msh"),
            lab("local line file") + p("lineinfo.dat"), lab("Ocean mesh file.") + p("ocean.msh"),
            lab("mesh ctl file") + p("mesh.ctl"), lab("Vxyzfile") + p("vxyz_mesh"), lab("Fxyzfile") + p("fxyz_mesh"),
            lab("output folder") + outdir.rstrip("/") + "/", lab("header2d  (a50)") + "h2d", lab("header3d  (a50)") + "h3d",
            lab("# of frequency") + str(len(m.freqs))]
    rows += [lab("Frequency [Hz]") + repr(float(fr)) for fr in m.freqs]
    xb = float(half) - 10.0
    rows += [lab("west bound") + repr(-xb), lab("east bound") + repr(xb), lab("south bound") + repr(-xb),
             lab("north bound") + repr(xb), lab("lenout [km]") + "10.0", lab("upz in [km]  (>0)") + "5.0",
             lab("downz in [km](<0)") + "-5.0", lab("zmax   [km]") + repr(float(m.bounds["zmax"])),
             lab("zmin   [km]") + repr(float(m.bounds["zmin"]))]
    rows += [lab(k) + "0.1" for k in ("sizein [km]", "sizebo [km]", "sigma_obs [km]", "A_obs     [km]",
                                       "dlen_source [km]", "sigma_src [km]", "A_src     [km]")]
    if utm_sites is None:
        rows += [lab("# of observatory") + str(m.sites.shape[0]), lab("lonlat(1),xyz (2)") + "2",
                 lab("UTM ZONE") + "none", lab("lonlatorigin") + "0.0 0.0"]
        for nm, s in zip(names, m.sites):
            rows += [lab("Name") + nm, lab("xyz") + f"{float(s[0])!r} {float(s[1])!r} {-SITE_DEPTH_KM!r}"]
    else:
        zone, lon0, lat0, lonlat = utm_sites
        rows += [lab("# of observatory") + str(m.sites.shape[0]), lab("lonlat(1),xyz (2)") + "1",
                 lab("UTM ZONE") + f"{int(zone)}S", lab("lonlatorigin") + f"{float(lon0)!r} {float(lat0)!r}"]
        for nm, ll in zip(names, lonlat):
            rows += [lab("Name") + nm, lab("lonlatalt") + f"{float(ll[0])!r} {float(ll[1])!r} {-SITE_DEPTH_KM!r}"]
    if seafloor_view is not None:  # ixyflag 2: the polygon_ki triangles 1 m above the seafloor
        rows += [lab("0:no,1:nxny,2:ntrik") + "2", lab("xyfilehead") + seafloor_view,
                 lab("pokimsh") + p("polygon_ki.msh"), lab("ki23dfile") + p("ki23dptr.dat")]
    elif plan_view is None:
        rows += [lab("0:no,1:nxny,2:ntrik") + "0"]
    else:  # (xyfilehead, nx, ny, depth_xy): ixyflag 1, at depth_xy (ixydepth 1) or on the seafloor (2)
        head, pnx, pny, depth = plan_view
        rows += [lab("0:no,1:nxny,2:ntrik") + "1", lab("xyfilehead") + head, lab("nx ny") + f"{pnx} {pny}"]
        if depth is None:
            rows += [lab("ixydepth") + "2"]
        else:
            rows += [lab("ixydepth") + "1", lab("depth_xy [km]") + repr(float(depth))]
        rows += [lab("pokimsh") + p("polygon_ki.msh"), lab("ki23dfile") + p("ki23dptr.dat")]
    rows += [lab("# of sources") + "1", lab("Source Name") + "S1",
             lab("source start point") + "0.0 0.0 -0.001", lab("source end   point") + "0.1 0.0 -0.001",
             lab("Elcetric current[A]") + "0.0", lab("sigma_air    [S/m]") + repr(float(m.sigma_air)),
             lab("condflag 0:home,1:") + "1", lab("condfile") + p("cond_test.msh")]
    ctl = p("tide_fwd.ctl")
    with open(ctl, "w") as f:
        f.write("## forward control file written by actfemtide_b200.synth\n")
        f.write("\n".join(rows) + "\n")
    return ctl


# ----------------------------------------------------------------------------- magnetotelluric models
MT_FREQS_HZ = (0.1, 0.03, 0.01, 0.003)


def graded_levels(top: float, first: float, ratio: float, n: int) -> np.ndarray:
    """n cell boundaries below 0 down to -top (or above, for top < 0 reversed by the caller):
    first cell `first` km thick, each next one `ratio` times thicker, scaled to end at |top|."""
    d = first * ratio ** np.arange(n)
    d *= abs(top) / d.sum()
    return np.concatenate([[0.0], np.cumsum(d)])


def mt_box(nx: int, ny: int, n_air: int, n_earth: int, *, half_km: float = 50.0, air_km: float = 50.0,
           earth_km: float = 50.0, first_km: float = 1.0, ratio: float = 1.25, ratio_air: float | None = None,
           ratio_earth: float | None = None, sigma: float = 0.1,
           block_sigma: float | None = None, grf: bool = False, seed: int = 0, site_grid=None, freqs=None,
           name: str = "mt_box") -> TidalModel:
    """A magnetotelluric model on a Kuhn box over [-half_km, half_km]^2 with graded vertical cells
    (n_air above z = 0 up to air_km, n_earth below down to -earth_km, finest at the surface; each
    region's cells grow by its ratio, scaled to fill the region, so the ratio sets the first cell).

    Physical tags as the MT program reads them (``n4flag(:,1)``,
    ``src/src_3DMT/forward_3DMT.f90:240``): air (centroid z > 0) tag 1 with
    1e-8 S/m; earth tag 3 with a per-element conductivity (condflag 1): `sigma`,
    or with ``grf`` a log10-normal random field (mean log10(sigma), std 0.5,
    correlation 8 km), optionally a block of `block_sigma` at x in [5,15],
    y in [-5,5], z in [-15,-5] km (tag 4).  Earth tetrahedra come last, as
    ``sigma(iele - nphys1)`` expects.  Sites 1 m below the surface on
    `site_grid` (default 5x5 over +-30 km); no tidal source (``nodes`` = 0).
    """
    za = graded_levels(air_km, first_km, ratio if ratio_air is None else ratio_air, n_air)
    ze = graded_levels(earth_km, first_km, ratio if ratio_earth is None else ratio_earth, n_earth)
    zs = np.concatenate([0.0 - ze[::-1], za[1:]])
    xyz, tets, hex_of_tet, cen = kuhn_box(nx, ny, n_air + n_earth, (-half_km, half_km), (-half_km, half_km),
                                          zs=zs)
    cx, cy, cz = cen[:, 0], cen[:, 1], cen[:, 2]
    tag = np.where(cz > 0.0, 1, 3).astype(np.int32)
    sig = np.full(tets.shape[0], float(sigma))
    if grf:
        rng = np.random.default_rng(seed)
        hx = 2 * half_km / nx
        g = gaussian_random_field((nx, ny, n_air + n_earth), (hx, hx, hx), 8.0, rng)
        logs = np.clip(math.log10(sigma) + 0.5 * g.ravel(order="F"), -4.0, 0.5)
        sig = np.where(tag == 3, 10.0 ** logs[hex_of_tet], sig)
    if block_sigma is not None:
        inb = (cx >= 5) & (cx <= 15) & (cy >= -5) & (cy <= 5) & (cz >= -15) & (cz <= -5) & (tag == 3)
        tag[inb] = 4
        sig[inb] = block_sigma
    order = np.concatenate([np.nonzero(tag == 1)[0], np.nonzero(tag >= 3)[0]])
    tets = tets[order]; tag = tag[order]; sig = sig[order]
    if site_grid is None:
        site_grid = (-30.0, -15.0, 0.0, 15.0, 30.0)
    gx, gy = np.meshgrid(np.asarray(site_grid, dtype=np.float64), np.asarray(site_grid, dtype=np.float64),
                         indexing="ij")
    sites = np.stack([gx.ravel(), gy.ravel(), np.full(gx.size, -SITE_DEPTH_KM)], axis=1)
    land = tag >= 3
    return TidalModel(
        name=name, xyz=np.ascontiguousarray(xyz), n4=np.ascontiguousarray((tets + 1).astype(np.int32)),
        tag=tag, sigma_land=np.ascontiguousarray(sig[land]), nodes=0, F=np.zeros((0, 3)),
        v=np.zeros((0, 3), np.complex128),
        freqs=np.asarray(MT_FREQS_HZ if freqs is None else freqs, dtype=np.float64),
        sites=np.ascontiguousarray(sites),
        bounds=dict(zmin=float(zs[0]), zmax=float(zs[-1]), xout=half_km, yout=half_km), seed=seed,
        dims=(nx, ny, n_air + n_earth))
