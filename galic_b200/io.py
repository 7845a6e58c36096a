"""Output files through the C ABI: the Gadget snapshot (write_file,
io.c:906-1243, as output_particles calls it, io.c:460-540), forcefield.dat
(grid.c:789-823) and densfield_<type>_<num>.dat (output_density_field,
io.c:36-460), byte for byte the reference's files."""
import ctypes as C
import os

import numpy as np

from . import _ffi
from .context import _check


def _d(a):
    return None if a is None else np.ascontiguousarray(a, dtype=np.float64)


def write_file(fname, particles, snap_format=1, mass_table=None):
    """One snapshot file of SnapFormat 1 or 2 from the arrays
    initialize_particles returns (pos, vel, vel_theo, mass, id, type);
    mass_table: 6 masses, types with a non-zero entry get no MASS block."""
    lib = _ffi.load_library()
    pos, vel, vt, mass = (_d(particles[k]) for k in ("pos", "vel", "vel_theo", "mass"))
    pid = np.ascontiguousarray(particles["id"], dtype=np.int32)
    ptype = np.ascontiguousarray(particles["type"], dtype=np.int32)
    mt = _d(mass_table)
    _check(lib.galic_write_snapshot(os.fsencode(fname), int(snap_format), len(mass), _ffi.dptr(pos), _ffi.dptr(vel),
                                    _ffi.dptr(vt), _ffi.dptr(mass), _ffi.iptr(pid), _ffi.iptr(ptype),
                                    None if mt is None else _ffi.dptr(mt)), "galic_write_snapshot")


def output_particles(output_dir, output_file, num, particles, snap_format=1):
    """output_particles (io.c:460-540) with one file per snapshot: writes
    OutputDir + OutputFile + "_%03d" and returns the file name."""
    fname = f"{output_dir}{output_file}_{num:03d}"
    write_file(fname, particles, snap_format)
    return fname


def write_forcefield(fname, params, dpotdr, dpotdz, pot):
    """forcefield.dat from the force grid's derivatives and potential."""
    lib = _ffi.load_library()
    arrs = [_d(a) for a in (dpotdr, dpotdz, pot)]
    _check(lib.galic_write_forcefield(os.fsencode(fname), C.byref(params), *[_ffi.dptr(a) for a in arrs]),
           "galic_write_forcefield")


def output_density_field(ctx, output_dir, num):
    """output_density_field (io.c:36-460): densfield_<type>_<num>.dat for every
    type with particles, from the context's targets and committed grids."""
    _check(ctx.lib.galic_output_density_field(ctx.h, os.fsencode(str(output_dir)), int(num)),
           "galic_output_density_field")
