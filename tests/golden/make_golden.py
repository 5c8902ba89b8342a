"""Regenerate the golden fixtures of tests/golden from the CPU oracle.

The reference (Fortran + MKL) cannot be built in this environment and ships no
golden data for its forward path, so these fixtures are oracle outputs on
small seeded models: they pin the oracle against regressions and give the GPU
tests reference values that do not need the oracle at run time.

Usage: python tests/golden/make_golden.py
"""
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)

from actfemtide_b200 import synth  # noqa: E402
from oracle import oracle as O  # noqa: E402

HERE = os.path.dirname(os.path.abspath(__file__))


def make(m, name, ssor_tol=1e-12):
    of = O.OracleForward(m)
    A = of.assemble(m.freqs[0])
    r = O.cocg13_single(A, precond="SSOR", resid=ssor_tol, maxit=200000)
    r5 = O.cocg13_single(A, precond="IC", resid=1e-30, maxit=5)
    item, ve, vf, iele = O.prepobscoeff(m, of.n6line, m.sites)
    out, amp, ph = of.sites(r["x"], m.freqs[0])
    np.savez_compressed(
        os.path.join(HERE, name + ".npz"),
        xyz=m.xyz, n4=m.n4, tag=m.tag, sigma_land=m.sigma_land, nodes=m.nodes, F=m.F, v=m.v, sites=m.sites,
        freq=m.freqs[0], sigma_air=m.sigma_air, sigma_ocean=m.sigma_ocean,
        bounds=np.array([m.bounds["zmin"], m.bounds["zmax"], m.bounds["xout"], m.bounds["yout"]]),
        line=of.line, n6line=of.n6line, INU=A.INU, IAU=A.IAU, INL=A.INL, IAL=A.IAL, D=A.D, AU=A.AU, AL=A.AL, b=A.b,
        bc=A.bc, x_ssor=r["x"], iter_ssor=r["iter"], x_ic5=r5["x"], item=item, val_e=ve, val_f=vf, iele=iele,
        site_field=out, site_amp=amp, site_phase=ph)
    print(name, "nline", of.line.shape[0], "ssor iters", r["iter"])


if __name__ == "__main__":
    make(synth.tiny_model(), "tiny_2x2x4")
    make(synth.tidal_box(4, 4, 6, seed=3, site_grid=(-6.0, 0.0, 6.0), half_km=12.0, name="box4x4x6"), "box4x4x6")
