"""Tree force-grid fill through the C ABI (galic_force_grid_fill).

Replaces the tree part of GALIC's forcedensitygrid_calculate
(grid.c:621-750): the caller passes the sampled mass particles in the
reference's P order (halo, disk, bulge) and gets FG_DPotDR, FG_DPotDz and
FG_Pot as [FG_Nbin, FG_Nbin] arrays indexed [iz, iR].  There is no CPU
fallback.
"""
import ctypes as C

import numpy as np

from . import _ffi
from .context import _check


def fill_params(fg_nbin, fg_rmin, fg_fac, G, softening, theta=0.4, top_node_factor=4.0, multiple_domains=4):
    """galic_fill_params_t; ForceSoftening = 2.8 * Softening as init.c:83 sets it."""
    fp = _ffi.GalicFillParams()
    fp.FG_Nbin = int(fg_nbin)
    fp.MultipleDomains = int(multiple_domains)
    fp.FG_Rmin = float(fg_rmin)
    fp.FG_Fac = float(fg_fac)
    fp.G = float(G)
    fp.ForceSoftening = 2.8 * float(softening)
    fp.ErrTolTheta = float(theta)
    fp.TopNodeFactor = float(top_node_factor)
    return fp


def force_grid_fill(fp, pos, mass):
    """(FG_DPotDR, FG_DPotDz, FG_Pot, stats) for mass particles pos[n,3], mass[n];
    stats is a dict of galic_fill_stats_t."""
    lib = _ffi.load_library()
    pos = np.ascontiguousarray(pos, dtype=np.float64)
    mass = np.ascontiguousarray(mass, dtype=np.float64)
    n = mass.shape[0]
    if pos.shape != (n, 3):
        raise ValueError("pos must be [n, 3]")
    N = fp.FG_Nbin
    out = [np.empty((N, N)) for _ in range(3)]
    st = _ffi.GalicFillStats()
    _check(lib.galic_force_grid_fill(C.byref(fp), n, _ffi.dptr(pos), _ffi.dptr(mass), _ffi.dptr(out[0]),
                                     _ffi.dptr(out[1]), _ffi.dptr(out[2]), C.byref(st)), "galic_force_grid_fill")
    return out[0], out[1], out[2], {k: getattr(st, k) for k, _ in _ffi.GalicFillStats._fields_}


def peano_hilbert_key(x, y, z, bits):
    """peano_hilbert_key (peano.c:331-347) of one integer cell."""
    return int(_ffi.load_library().galic_peano_hilbert_key(int(x), int(y), int(z), int(bits)))
