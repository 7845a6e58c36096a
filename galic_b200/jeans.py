"""Jeans solvers through the C ABI (galic_calculate_dispfield).

Replaces GALIC's calculate_dispfield (disp_fields.c:502-1049): the spherical
Jeans equation (FG_Disp_r), the axisymmetric f(E, Lz) solution (FG_DispZ,
FG_DispPhi, FG_Vstream) and the tilted f(E, Lz, I3) method of lines
(FG_tilted_*) on the context's force grid.  The results also become the
context's streaming-velocity and Jeans tables.  There is no CPU fallback.
"""
import ctypes as C

import numpy as np

from . import _ffi
from .context import _check


def jeans_params(streaming=(0.0, 0.0, 0.0, 0.0), r_over_z=(0.0, 0.0, 0.0, 0.0)):
    """galic_jeans_params_t from All.{Halo,Disk,Bulge}StreamingVelocityParameter
    and All.{Halo,Disk,Bulge}DispersionRoverZratio (index = type, 0 unused)."""
    jp = _ffi.GalicJeansParams()
    for t in range(4):
        jp.StreamingVelocityParameter[t] = float(streaming[t])
        jp.DispersionRoverZratio[t] = float(r_over_z[t])
    return jp


def calculate_dispfield(ctx, sp, jp):
    """Runs the solvers; returns {type: {table name: [FG_Nbin, FG_Nbin] array}}
    for the types with particles (disp_r: its row 0 holds FG_Disp_r)."""
    N = ctx.params.FG_Nbin
    arrs = np.zeros((4, len(_ffi.JEANS_TABLES), N, N))
    out = (_ffi.GalicJeansTables * 4)()
    for t in (1, 2, 3):
        for w, name in enumerate(_ffi.JEANS_TABLES):
            setattr(out[t], name, _ffi.dptr(arrs[t, w]))
    _check(ctx.lib.galic_calculate_dispfield(ctx.h, C.byref(sp), C.byref(jp), out), "galic_calculate_dispfield")
    return {t: {name: arrs[t, w] for w, name in enumerate(_ffi.JEANS_TABLES)}
            for t in (1, 2, 3) if ctx.params.NType[t] > 0}
