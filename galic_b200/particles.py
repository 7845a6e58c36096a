"""Particle initialisation through the C ABI (galic_initialize_particles).

Replaces GALIC's initialize_particles (set_particles.c:15-307): positions,
escape speeds, integration times, the halo's distribution-function
velocities (VelTheo), the Jeans dispersion targets, the Gaussian initial
velocities and the permutation, drawn exactly as the reference's sequential
loop draws them from the stream.  The particles become the context's.  There
is no CPU fallback.
"""
import ctypes as C

import numpy as np

from . import _ffi
from .context import _check

FIELDS = (("pos", 3, np.float64), ("vel", 3, np.float64), ("vel_theo", 3, np.float64), ("mass", 1, np.float64),
          ("vesc", 1, np.float64), ("tint", 1, np.float64), ("targets", 4, np.float64), ("type", 1, np.int32),
          ("id", 1, np.int32), ("permutation", 1, np.int32))


def _host_array(shape, dtype):
    """Page-locked host memory from torch's caching allocator (the device
    writes into it at full link speed, and repeated calls reuse the pages);
    plain memory where torch has no CUDA device."""
    try:
        import torch
        if torch.cuda.is_available():
            t = torch.empty(shape, dtype=torch.float64 if dtype == np.float64 else torch.int32, pin_memory=True)
            return t.numpy()
    except ImportError:
        pass
    return np.empty(shape, dtype=dtype)


def initialize_particles(ctx, sp, torbit_fac, stream):
    """Runs the initialisation; returns ({field: array}, low-dispersion counts [4, 4])."""
    n = sum(int(ctx.params.NType[t]) for t in (1, 2, 3))
    arrs = {k: _host_array((n, w) if w > 1 else (n,), dt) for k, w, dt in FIELDS}  # the call fills every one
    out = _ffi.GalicParticlesOut()
    for k, _, dt in FIELDS:
        setattr(out, k, _ffi.dptr(arrs[k]) if dt == np.float64 else _ffi.iptr(arrs[k]))
    _check(ctx.lib.galic_initialize_particles(ctx.h, C.byref(sp), float(torbit_fac), C.byref(stream.s), C.byref(out)),
           "galic_initialize_particles")
    ctx.n = n
    counts = np.array([[out.low_disp[t][k] for k in range(4)] for t in range(4)], dtype=np.int32)
    return arrs, counts
