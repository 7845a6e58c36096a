"""Ensembles of models advanced together (galic_ensemble_* in the C ABI).

`Ensemble(contexts)` groups up to 64 `Context`s on one device; each
`calc_all()` runs calc_all_response_fields + calc_global_fit for every member
in the FP32 form as one persistent orbit launch, replayed from a CUDA graph.
Results are read from the member contexts as usual.  There is no CPU
fallback.
"""
import ctypes as C

import numpy as np

from . import _ffi
from .context import GalicError, _check


class Ensemble:
    def __init__(self, contexts):
        self.lib = _ffi.load_library()
        self.members = list(contexts)
        arr = (C.c_void_p * len(self.members))(*[c.h.value for c in self.members])
        h = C.c_void_p()
        _check(self.lib.galic_ensemble_create(arr, len(self.members), C.byref(h)), "galic_ensemble_create")
        self.h = h

    def close(self):
        if getattr(self, "h", None):
            self.lib.galic_ensemble_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def calc_all(self):
        _check(self.lib.galic_ensemble_calc_all(self.h), "galic_ensemble_calc_all")

    @staticmethod
    def variants():
        lib = _ffi.load_library()
        b = (C.c_int * 64)()
        m = (C.c_int * 64)()
        n = lib.galic_ensemble_variants(b, m, 64)
        return [(b[i], m[i]) for i in range(n)]

    def set_variant(self, v):
        _check(self.lib.galic_ensemble_set_variant(self.h, int(v)), "galic_ensemble_set_variant")

    def autotune(self, sample_fraction=0.05):
        """Times every tile variant on a sample of the orbits; returns (best, ms per variant)."""
        n = len(self.variants())
        ms = np.zeros(n)
        best = C.c_int(0)
        _check(self.lib.galic_ensemble_autotune(self.h, float(sample_fraction), C.byref(best), _ffi.dptr(ms)),
               "galic_ensemble_autotune")
        return best.value, ms

    def last_timing(self):
        """(ms of the iteration, ms of the orbit kernel, orbit-steps, graph nodes)."""
        a, b = C.c_double(), C.c_double()
        st = C.c_longlong()
        nodes = C.c_int()
        _check(self.lib.galic_ensemble_last_timing(self.h, C.byref(a), C.byref(b), C.byref(st), C.byref(nodes)),
               "galic_ensemble_last_timing")
        return a.value, b.value, st.value, nodes.value


__all__ = ["Ensemble", "GalicError"]
