"""Packed batches of uneven meshes, host side: the union mesh and its edge numbering.

A packed batch solves independent meshes as one system per mesh in one
launch sequence.  The union's MKLINE_V2 numbering must be each part's own
numbering, offset, so that rows of one mesh are contiguous and the union
matrix is block diagonal; these checks run on the oracle's restatement of
MKLINE_V2/MKN6 and C_set_dof2 (no GPU).
"""
import numpy as np
import pytest

from actfemtide_b200 import synth


def small_parts(count=3, seed=4):
    return synth.uneven_models(count, seed=seed, nmin=2, nmax=5)


def test_uneven_models_shapes():
    ms = synth.uneven_models(24, seed=0, nmin=8, nmax=32)
    assert len(ms) == 24
    for m in ms:
        nx, ny, nz = m.dims
        assert nx == ny and 8 <= nx <= 32 and nz == max(2, int(round(0.75 * nx)))
        assert m.ntet == 6 * nx * ny * nz
    # seeded: the same draw twice
    again = synth.uneven_models(24, seed=0, nmin=8, nmax=32)
    assert [m.dims for m in ms] == [m.dims for m in again]


def test_pack_offsets_and_sources():
    parts = small_parts()
    pk = synth.pack(parts)
    assert pk.nseg == len(parts)
    assert pk.node_ptr[-1] == pk.xyz.shape[0] and pk.tet_ptr[-1] == pk.n4.shape[0]
    for k, m in enumerate(parts):
        a, b = pk.node_ptr[k], pk.node_ptr[k + 1]
        t0, t1 = pk.tet_ptr[k], pk.tet_ptr[k + 1]
        assert np.array_equal(pk.xyz[a:b], m.xyz)
        assert np.array_equal(pk.n4[t0:t1] - a, m.n4)
        assert np.array_equal(pk.sigma_tet[t0:t1], m.sigma_per_tet())
        assert np.array_equal(pk.F[a:a + m.nodes], m.F) and np.all(pk.F[a + m.nodes:b] == 0)
        assert np.array_equal(pk.v[a:a + m.nodes], m.v)


def test_pack_rejects_different_bounds():
    a = synth.tidal_box(2, 2, 2)
    b = synth.tidal_box(2, 2, 2, half_km=20.0)
    with pytest.raises(ValueError):
        synth.pack([a, b])


def test_union_numbering_is_the_parts_numbering_offset(oracle):
    parts = small_parts()
    pk = synth.pack(parts)
    line_u, n6_u = oracle.mkline(pk.xyz.shape[0], pk.n4)
    INU, IAU, INL, IAL = oracle.pattern(line_u.shape[0], n6_u)
    e_off = 0
    for k, m in enumerate(parts):
        line, n6 = oracle.mkline(m.node, m.n4)
        ne = line.shape[0]
        a = pk.node_ptr[k]
        t0, t1 = pk.tet_ptr[k], pk.tet_ptr[k + 1]
        assert np.array_equal(line_u[e_off:e_off + ne], line + a)
        assert np.array_equal(np.abs(n6_u[t0:t1]), np.abs(n6) + e_off)
        assert np.array_equal(np.sign(n6_u[t0:t1]), np.sign(n6))
        # block diagonal: every column of rows of mesh k lies in mesh k
        for i in range(e_off, e_off + ne):
            cols = np.concatenate([IAU[INU[i]:INU[i + 1]], IAL[INL[i]:INL[i + 1]]]) - 1
            assert np.all((cols >= e_off) & (cols < e_off + ne))
        e_off += ne
    assert e_off == line_u.shape[0]
