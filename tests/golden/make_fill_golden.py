"""Generates the force-grid-fill fixtures (tests/golden/fill/*.npz) from GALIC's
own C (oracle/_ref/libgalic_ref.so, built from the reference tree by
oracle/Makefile):  python tests/golden/make_fill_golden.py

Each fixture holds the mass particles that forcedensitygrid_calculate
(grid.c:621-757) samples for a seeded generator (halo, disk, bulge in the
reference's P order, with their P[].Mass) and the FG_DPotDR / FG_DPotDz /
FG_Pot it computes with its Barnes-Hut tree on one rank (gravity(),
gravtree.c:35-50), plus the fill parameters.
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
OUT = os.path.join(HERE, "fill")
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.dirname(HERE))

from galic_b200 import synth  # noqa: E402
import oracle_lib  # noqa: E402

# name: (components, FG_Nbin, Softening, ErrTolTheta, TopNodeFactor, MultipleDomains, N halo, disk, bulge, seed)
CASES = {
    "halo_disk": ("hd", 32, 0.3, 0.4, 4.0, 4, 2000, 500, 0, 777),
    "composite": ("hdb", 48, 0.3, 0.4, 4.0, 4, 3000, 1000, 400, 778),
    "fine_tree": ("hd", 24, 0.05, 0.25, 2.5, 8, 6000, 2000, 0, 779),
}


def case_params(kind, fg_nbin):
    Cc = synth.Component
    comps = [Cc("halo", 95.0, 30.0, 100), Cc("disk", 5.0, 3.5, 100, z0=0.7)]
    if "b" in kind:
        comps.append(Cc("bulge", 1.5, 1.0, 100))
    p, rmax, _ = synth.make_params(comps, level=5, fg_nbin=fg_nbin, outer_frac=0.49, inner_frac=1e-7)
    return p, rmax


def make(name):
    kind, fg, soft, theta, tnf, md, nh, nd, nb, seed = CASES[name]
    p, rmax = case_params(kind, fg)
    rf = oracle_lib.RefFillParams(soft, theta, tnf, 3.5, 0.7, rmax, md, nh, nd, nb, seed)
    pos, mass, dpotdr, dpotdz, pot = oracle_lib.run_reference(oracle_lib.reference_force_fill, p, rf)
    fill = np.array([p.FG_Rmin, p.FG_Fac, p.G, soft, theta, tnf], dtype=np.float64)
    np.savez_compressed(os.path.join(OUT, name + ".npz"), fg_nbin=np.array(fg), multiple_domains=np.array(md),
                        fill=fill, pos=pos, mass=mass, dpotdr=dpotdr, dpotdz=dpotdz, pot=pot)
    print(name, pos.shape, float(np.abs(dpotdr).max()))


if __name__ == "__main__":
    os.makedirs(OUT, exist_ok=True)
    for name in CASES:
        make(name)
