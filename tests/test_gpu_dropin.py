"""Drop-in driver: the reference's ctl file and input files in, <site>_<src>.dat files out (GPU)."""
import os

import numpy as np
import pytest

from actfemtide_b200 import synth

pytestmark = pytest.mark.gpu


@pytest.fixture
def short_dir():
    """The reference reads file names into character(70) fields (m_param.f90:29-47): keep paths short."""
    import shutil
    import tempfile
    d = tempfile.mkdtemp(prefix="afem", dir="/tmp")
    yield d
    shutil.rmtree(d, ignore_errors=True)


def test_ctl_driver_matches_oracle(gpulib, oracle, short_dir):
    from actfemtide_b200.forward import Forward, amp_phase
    tmp_path = short_dir
    m = synth.tidal_box(4, 4, 6, seed=3, site_grid=(-6.0, 0.0, 6.0), half_km=12.0)
    m.freqs = np.array([1.0 / 44714.0, 1.0 / 43200.0])
    of = oracle.OracleForward(m)
    ctl = synth.write_reference_inputs(m, str(tmp_path), of.line, of.n6line)
    with Forward(0) as fw:
        fw.load_ctl(ctl)
        freqs, xyz = fw.ctl_info()
        assert np.allclose(freqs, m.freqs)
        # PREPZSRCOBS: z = interpolated surface height - 1 m
        assert np.allclose(xyz, m.sites, atol=1e-12)
        line, n6 = fw.lines()
        assert np.array_equal(line, of.line) and np.array_equal(n6, of.n6line)
        fw.run_ctl(precond="SSOR", tol=1e-10)
    # the ctl path uses GENMAT's ocean conductivity, the default-real literal 3.33
    m33 = synth.TidalModel(**{**m.__dict__, "sigma_ocean": float(np.float32(3.33)), "sites": xyz})
    of33 = oracle.OracleForward(m33, of.line, of.n6line)
    for fi, fr in enumerate(m.freqs):
        A = of33.assemble(fr)
        r = oracle.cocg13_single(A, precond="SSOR", resid=1e-11, maxit=100000)
        out, amp, ph = of33.sites(r["x"], fr)
        for s in range(xyz.shape[0]):
            path = os.path.join(str(tmp_path), f"S{s + 1:03d}_S1.dat")
            rows = [list(map(float, ln.split())) for ln in open(path).read().splitlines()]
            assert len(rows) == len(m.freqs) and all(len(rw) == 11 for rw in rows)
            vals = np.array(rows[fi][1:]).reshape(5, 2)
            assert abs(rows[fi][0] - fr) <= 1e-6 * fr
            np.testing.assert_allclose(vals[:, 0], amp[0, :, s], rtol=2e-6, atol=1e-6 * amp[0].max())
            big = amp[0, :, s] > 1e-3 * amp[0].max()
            dphi = (vals[big, 1] - ph[0, big, s] + 180.0) % 360.0 - 180.0
            assert np.all(np.abs(dphi) <= 1e-3)


def test_ctl_plan_view_matches_oracle(gpulib, oracle, short_dir):
    """ixyflag 1, ixydepth 1: PREPOBSCOEFF_XY points, FINDELEWITHGRID elements, OUTFREQFILES2 files."""
    from actfemtide_b200 import capi
    from actfemtide_b200.forward import Forward
    m = synth.tidal_box(4, 4, 6, seed=3, site_grid=(-6.0, 0.0, 6.0), half_km=12.0)
    m.freqs = np.array([1.0 / 44714.0])
    of = oracle.OracleForward(m)
    pnx, pny, depth = 5, 4, -5.5
    ctl = synth.write_reference_inputs(m, short_dir, of.line, of.n6line, plan_view=("xy", pnx, pny, depth))
    with Forward(0) as fw:
        fw.load_ctl(ctl)
        fw.run_ctl(precond="SSOR", tol=1e-10)
    xb = 12.0 - 10.0
    pts = capi.xy_points(-xb, xb, -xb, xb, pnx, pny, depth)
    m33 = synth.TidalModel(**{**m.__dict__, "sigma_ocean": float(np.float32(3.33))})
    of33 = oracle.OracleForward(m33, of.line, of.n6line)
    fr = m.freqs[0]
    A = of33.assemble(fr)
    r = oracle.cocg13_single(A, precond="SSOR", resid=1e-11, maxit=100000)
    item, ve, vf, _ = oracle.prepobscoeff_grid(m33, of.n6line, pts)
    _, amp, ph = oracle.calobsebcomp(r["x"][None, :], 2 * np.pi * fr, item, ve, vf)
    name = os.path.join(short_dir, "xy" + "0.22E-04" + "_S1.dat")
    rows = np.array([list(map(float, ln.split())) for ln in open(name).read().splitlines()])
    assert rows.shape == (pnx * pny, 13)
    np.testing.assert_allclose(rows[:, :3], pts, atol=5e-8)
    vals = rows[:, 3:].reshape(-1, 5, 2)
    np.testing.assert_allclose(vals[:, :, 0], amp[0].T, rtol=2e-6, atol=1e-6 * amp[0].max() + 5e-8)
    big = amp[0].T > 1e-3 * amp[0].max()
    dphi = (vals[:, :, 1][big] - ph[0].T[big] + 180.0) % 360.0 - 180.0
    assert np.all(np.abs(dphi) <= 1e-3)


def _lonlat_of(oracle, xy_km, zone, lon0, lat0):
    """Longitude/latitude whose UTMXY position is xy_km (Newton on the oracle's UTMXY)."""
    ll = np.array([lon0, lat0]) + np.array([xy_km[0] / 100.0, xy_km[1] / 111.0])
    for _ in range(20):
        f = oracle.utmxy(ll[0], ll[1], lon0, lat0, zone) - xy_km
        h = 1e-6
        J = np.stack([(oracle.utmxy(ll[0] + h, ll[1], lon0, lat0, zone) - oracle.utmxy(ll[0] - h, ll[1], lon0, lat0,
                                                                                         zone)) / (2 * h),
                      (oracle.utmxy(ll[0], ll[1] + h, lon0, lat0, zone) - oracle.utmxy(ll[0], ll[1] - h, lon0, lat0,
                                                                                         zone)) / (2 * h)], axis=1)
        ll = ll - np.linalg.solve(J, f)
    return ll


def test_ctl_utm_sites_match_xyz_sites(gpulib, oracle, short_dir):
    """lonlatflag 1: the same sites given as longitude/latitude in UTM zone 54 (UTMXY) land where the
    xyz sites are and give the same site files."""
    import shutil
    from actfemtide_b200.forward import Forward
    m = synth.tidal_box(4, 4, 6, seed=3, site_grid=(-6.0, 0.0, 6.0), half_km=12.0)
    m.freqs = np.array([1.0 / 44714.0])
    # sites strictly inside tetrahedra: on a shared face the fields of neighbouring elements differ
    # (B is constant per element), and the converted positions differ from the xyz ones in the last bits
    sx, sy = np.meshgrid([-4.37, 1.91, 3.23], [-2.71, 0.83, 4.57], indexing="ij")
    sx, sy = sx.ravel(), sy.ravel()
    m.sites = np.stack([sx, sy, synth.surface_z(sx, sy) - synth.SITE_DEPTH_KM], axis=1)
    of = oracle.OracleForward(m)
    zone, lon0, lat0 = 54, 139.8, 28.3
    lonlat = np.array([_lonlat_of(oracle, s[:2], zone, lon0, lat0) for s in m.sites])
    d_xyz = os.path.join(short_dir, "a")
    d_utm = os.path.join(short_dir, "b")
    ctl_a = synth.write_reference_inputs(m, d_xyz, of.line, of.n6line)
    ctl_b = synth.write_reference_inputs(m, d_utm, of.line, of.n6line, utm_sites=(zone, lon0, lat0, lonlat))
    with Forward(0) as fw:
        fw.load_ctl(ctl_b)
        _, xyz_b = fw.ctl_info()
        np.testing.assert_allclose(xyz_b[:, :2], m.sites[:, :2], atol=1e-9)
        for s, ll in zip(xyz_b, lonlat):
            np.testing.assert_allclose(s[:2], oracle.utmxy(ll[0], ll[1], lon0, lat0, zone), atol=1e-12)
        fw.run_ctl(precond="SSOR", tol=1e-10)
        fw.load_ctl(ctl_a)
        fw.run_ctl(precond="SSOR", tol=1e-10)
    for s in range(m.sites.shape[0]):
        a = np.loadtxt(os.path.join(d_xyz, f"S{s + 1:03d}_S1.dat"))
        b = np.loadtxt(os.path.join(d_utm, f"S{s + 1:03d}_S1.dat"))
        np.testing.assert_allclose(b, a, rtol=1e-5, atol=1e-6 * np.abs(a).max())
    shutil.rmtree(d_xyz, ignore_errors=True)


def _read_tri_msh(path):
    lines = open(path).read().split("\n")
    nn = int(lines[4])
    xyz = np.array([list(map(float, ln.split()[1:4])) for ln in lines[5:5 + nn]])
    ne = int(lines[7 + nn])
    n3 = np.array([list(map(int, ln.split()[5:8])) for ln in lines[8 + nn:8 + nn + ne]], np.int32)
    return xyz, n3


@pytest.mark.parametrize("view", ["ixydepth2", "ixyflag2"])
def test_ctl_seafloor_plan_views_match_oracle(gpulib, oracle, short_dir, view):
    """Seafloor plan views through the ctl driver: ixyflag 1 with ixydepth 2 (the nx x ny points moved 1 m
    below the seafloor by PREPZOBS over polygon_ki.msh and ki23dptr.dat) and ixyflag 2 (PREPOBSCOEFF_XYSBTM:
    the polygon_ki triangles 1 m above the seafloor, grid list 300 x 300 x 300), each writing the
    OUTFREQFILES2 file and IXYHOUT's ixyh_xy2D file; both checked against the oracle's restatement on the
    oracle's own solve."""
    from actfemtide_b200 import capi
    from actfemtide_b200.forward import Forward
    m = synth.tidal_box(8, 8, 8, seed=3, site_grid=(-6.0, 0.0, 6.0), half_km=20.0)
    m.freqs = np.array([1.0 / 44714.0])
    of = oracle.OracleForward(m)
    if view == "ixydepth2":
        pnx, pny = 5, 4
        ctl = synth.write_reference_inputs(m, short_dir, of.line, of.n6line, plan_view=("xy", pnx, pny, None))
        head = "xy"
    else:
        ctl = synth.write_reference_inputs(m, short_dir, of.line, of.n6line, seafloor_view="xyb")
        head = "xyb"
    with Forward(0) as fw:
        fw.load_ctl(ctl)
        fw.run_ctl(precond="SSOR", tol=1e-10)
    ki_xyz, ki_n3 = _read_tri_msh(os.path.join(short_dir, "polygon_ki.msh"))
    ki23 = np.loadtxt(os.path.join(short_dir, "ki23dptr.dat"), skiprows=1).astype(np.int32)
    if view == "ixydepth2":
        xb = 20.0 - 10.0
        pts0 = capi.xy_points(-xb, xb, -xb, xb, pnx, pny, 0.0)
        pts, items, vals = oracle.prepzobs(m.xyz, ki_xyz, ki_n3, ki23, pts0)
        nz = 50
    else:
        pts, items, vals = oracle.xysbtm_points(m.xyz, ki_n3, ki23)
        nz = 300
    m33 = synth.TidalModel(**{**m.__dict__, "sigma_ocean": float(np.float32(3.33))})
    of33 = oracle.OracleForward(m33, of.line, of.n6line)
    fr = m.freqs[0]
    A = of33.assemble(fr)
    r = oracle.cocg13_single(A, precond="SSOR", resid=1e-11, maxit=100000)
    item, ve, vf, _ = oracle.prepobscoeff_grid_nz(m33, of.n6line, pts, nz)
    fields, amp, ph = oracle.calobsebcomp(r["x"][None, :], 2 * np.pi * fr, item, ve, vf)
    # OUTFREQFILES2: x, y, z and (amp, phase) of bx..ey
    rows = np.loadtxt(os.path.join(short_dir, head + "0.22E-04_S1.dat"), ndmin=2)
    assert rows.shape == (pts.shape[0], 13)
    np.testing.assert_allclose(rows[:, :3], pts, atol=5e-8)
    vals_out = rows[:, 3:].reshape(-1, 5, 2)
    np.testing.assert_allclose(vals_out[:, :, 0], amp[0].T, rtol=2e-6, atol=1e-6 * amp[0].max() + 5e-8)
    big = amp[0].T > 1e-3 * amp[0].max()
    dphi = (vals_out[:, :, 1][big] - ph[0].T[big] + 180.0) % 360.0 - 180.0
    assert np.all(np.abs(dphi) <= 1e-3)
    # IXYHOUT: 26 columns per point
    F = np.zeros((m.node, 3)); F[:m.nodes] = m.F
    v = np.zeros((m.node, 3), np.complex128); v[:m.nodes] = m.v
    ref = oracle.ixyhout(pts, fields[0], F, v, items, vals)
    got = np.loadtxt(os.path.join(short_dir, "ixyh_xy2D0.22E-04.dat"), ndmin=2)
    assert got.shape == ref.shape == (pts.shape[0], 26)
    scale = np.abs(ref).max(axis=0) + 1e-30
    assert np.all(np.abs(got - ref) <= 2e-6 * scale + 1e-12), np.abs(got - ref).max(axis=0) / scale
    # the ocean points carry current: h > 0 and a nonzero sigma h (v x F) somewhere
    assert ref[:, 25].max() > 0.0 and np.abs(ref[:, 5:9]).max() > 0.0
