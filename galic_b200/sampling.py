"""Set-up sampling through the C ABI (galic_sample_* in include/galic_gpu.h).

GALIC draws its target maps and the force-grid mass particles by Monte-Carlo
sampling from one sequential random stream:

* densitygrid_sample_targetresponse (grid.c:536-617) -> `sample_density_targets`
* calc_energy_grid_mass_maps (grid.c:941-1076)        -> `sample_energy_targets`
* {halo,disk,bulge}_get_fresh_coordinate
  (halo.c:17-40, disk.c:17-50, bulge.c:15-37)         -> `sample_positions`

The stream stand-in is a Philox4x32-10 stream (`Stream`): its k-th uniform
is computed directly, so the GPU replays the reference's sequential loops in
parallel and consumes exactly the draws the loop would.  There is no CPU
fallback.
"""
import ctypes as C

import numpy as np

from . import _ffi
from .context import _check


def sample_params(Rmax, Halo_A, HaloStretch=1.0, Disk_Z0=0.0, Disk_H=0.0, Bulge_A=0.0, BulgeStretch=1.0,
                  HaloBetaParameter=0.0, BulgeBetaParameter=0.0):
    """galic_sample_params_t from the All.* values of the same names."""
    sp = _ffi.GalicSampleParams()
    for k, v in dict(Rmax=Rmax, Halo_A=Halo_A, HaloStretch=HaloStretch, Disk_Z0=Disk_Z0, Disk_H=Disk_H,
                     Bulge_A=Bulge_A, BulgeStretch=BulgeStretch, HaloBetaParameter=HaloBetaParameter,
                     BulgeBetaParameter=BulgeBetaParameter).items():
        setattr(sp, k, float(v))
    return sp


class Stream:
    """A position in the Philox stream (seed, a, b) that stands in for GALIC's
    random_generator (gsl_rng_set(random_generator, 42 + ThisTask), init.c:27,
    is the stream (42 + ThisTask, 0, 0) at position 0)."""

    def __init__(self, seed=42, a=0, b=0, position=0):
        self.s = _ffi.GalicStream(int(seed), int(a), int(b), int(position))

    @property
    def position(self):
        return int(self.s.position)


def set_dispersion(ctx, ptype, disp_r=None, dispz=None, dispphi=None, tilted_vr2=None, tilted_vz2=None):
    """galic_set_dispersion: the type's Jeans tables, each [FG_Nbin, FG_Nbin] (or None where unread)."""
    arrs = [None if a is None else np.ascontiguousarray(a, dtype=np.float64).ravel()
            for a in (disp_r, dispz, dispphi, tilted_vr2, tilted_vz2)]
    _check(ctx.lib.galic_set_dispersion(ctx.h, int(ptype), *[_ffi.dptr(a) for a in arrs]), "galic_set_dispersion")


def sample_density_targets(ctx, sp, ntarget, stream, renormalize=False):
    """densitygrid_sample_targetresponse: DGs_MassTarget of every type with MType > 0."""
    _check(ctx.lib.galic_sample_density_targets(ctx.h, C.byref(sp), int(ntarget), C.byref(stream.s),
                                                1 if renormalize else 0), "galic_sample_density_targets")


def sample_energy_targets(ctx, sp, ntarget, stream):
    """calc_energy_grid_mass_maps: EGs_MassTarget and EGs_EgyTarget_{r,t,p,q} of every type with MType > 0."""
    _check(ctx.lib.galic_sample_energy_targets(ctx.h, C.byref(sp), int(ntarget), C.byref(stream.s)),
           "galic_sample_energy_targets")


def get_targets(ctx, ptype):
    """The type's six target stacks (DGs_MassTarget, EGs_MassTarget, EGs_EgyTarget_r/t/p/q)."""
    out = [np.zeros(ctx.nstack) for _ in range(6)]
    _check(ctx.lib.galic_get_targets(ctx.h, int(ptype), *[_ffi.dptr(a) for a in out]), "galic_get_targets")
    return out


def sample_positions(sp, ptype, n, stream):
    """n positions of the type's *_get_fresh_coordinate, as an [n, 3] array."""
    lib = _ffi.load_library()
    pos = np.zeros((int(n), 3))
    _check(lib.galic_sample_positions(C.byref(sp), int(ptype), int(n), C.byref(stream.s), _ffi.dptr(pos)),
           "galic_sample_positions")
    return pos
