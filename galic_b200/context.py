"""Python view of a libgalic_cuda.so context.

`Context` owns one galic_ctx (include/galic_gpu.h) and exposes the entry
points under the names of the GALIC functions they replace:
produce_orbit_response_field_mod, calc_all_response_fields, optimize (one
repetition), calc_global_fit results, ...  Every call goes through the C ABI;
there is no Python or CPU fallback.
"""
import ctypes as C

import numpy as np

from . import _ffi


class GalicError(RuntimeError):
    def __init__(self, status, where):
        lib = _ffi.load_library()
        msg = lib.galic_status_string(status).decode()
        super().__init__(f"{where}: {_ffi.STATUS_NAMES.get(status, status)} ({msg})")
        self.status = status


def _check(st, where):
    if st != 0:
        raise GalicError(st, where)


class Context:
    def __init__(self, params):
        self.lib = _ffi.load_library()
        self.params = params.copy()
        h = C.c_void_p()
        _check(self.lib.galic_ctx_create(C.byref(self.params), C.byref(h)), "galic_ctx_create")
        self.h = h
        L = params.DG_MaxLevel
        self.ngrid = 1 << (2 * L)
        self.nstack = ((1 << (2 + 2 * L)) - 1) // 3
        self.n = 0

    def close(self):
        if getattr(self, "h", None):
            self.lib.galic_ctx_destroy(self.h)
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

    # ------------------------------------------------------------ uploads
    def load_model(self, m):
        """Uploads every table of a synth.Model (or any object with the same fields)."""
        L = self.lib
        _check(L.galic_set_force_grid(self.h, _ffi.dptr(m.pot), _ffi.dptr(m.dpotdr), _ffi.dptr(m.dpotdz)),
               "galic_set_force_grid")
        for t in (1, 2, 3):
            _check(L.galic_set_vstream(self.h, t, _ffi.dptr(np.ascontiguousarray(m.vstream[t], dtype=np.float64))),
                   "galic_set_vstream")
        _check(L.galic_set_density_geometry(self.h, _ffi.dptr(m.cellsize), _ffi.dptr(m.dgs_distance)),
               "galic_set_density_geometry")
        for t, tg in m.targets.items():
            _check(L.galic_set_targets(self.h, t, *[_ffi.dptr(np.ascontiguousarray(a)) for a in tg]),
                   "galic_set_targets")
        self.set_particles(m.pos, m.vel, m.mass, m.tint, m.vesc, m.ptype, m.ptargets)

    def set_particles(self, pos, vel, mass, tint, vesc, ptype, ptargets):
        n = len(mass)
        arrs = [np.ascontiguousarray(a, dtype=np.float64) for a in (pos, vel, mass, tint, vesc)]
        ty = np.ascontiguousarray(ptype, dtype=np.int32)
        tg = np.ascontiguousarray(ptargets, dtype=np.float64)
        _check(self.lib.galic_set_particles(self.h, n, *[_ffi.dptr(a) for a in arrs], _ffi.iptr(ty), _ffi.dptr(tg)),
               "galic_set_particles")
        self.n = n

    # ------------------------------------------------------------ drop-ins
    def produce_orbit_response_field_mod(self, pos, vel, mass, timespan, ptype):
        """orbit_response.c:155-491: returns (tall, orbits, m, r, t, q, p)."""
        g = [np.zeros(self.ngrid) for _ in range(5)]
        orbits = C.c_int(0)
        pos = np.ascontiguousarray(pos, dtype=np.float64)
        vel = np.ascontiguousarray(vel, dtype=np.float64)
        tall = self.lib.galic_produce_orbit_response_field_mod(
            self.h, _ffi.dptr(pos), _ffi.dptr(vel), 0, *[_ffi.dptr(a) for a in g], float(mass), float(timespan),
            C.byref(orbits), int(ptype))
        if tall < 0:
            raise GalicError(self.lib.galic_last_status(self.h), "galic_produce_orbit_response_field_mod")
        return (tall, orbits.value, *g)

    def produce_orbit_response_field(self, pos, vel, mass, timespan):
        """orbit_response.c:33-151: returns (tall, orbits, m)."""
        m = np.zeros(self.ngrid)
        orbits = C.c_int(0)
        pos = np.ascontiguousarray(pos, dtype=np.float64)
        vel = np.ascontiguousarray(vel, dtype=np.float64)
        tall = self.lib.galic_produce_orbit_response_field(self.h, _ffi.dptr(pos), _ffi.dptr(vel), 0, _ffi.dptr(m),
                                                           float(mass), float(timespan), C.byref(orbits))
        if tall < 0:
            raise GalicError(self.lib.galic_last_status(self.h), "galic_produce_orbit_response_field")
        return tall, orbits.value, m

    # ------------------------------------------------------------ batched path
    def calc_all_response_fields(self, form=_ffi.GALIC_FORM_FP64):
        _check(self.lib.galic_calc_all_response_fields(self.h, form), "galic_calc_all_response_fields")

    def calc_all_shard(self, form, rank, world):
        """This rank's part of a sharded calc_all (galic_calc_all_shard)."""
        _check(self.lib.galic_calc_all_shard(self.h, int(form), int(rank), int(world)), "galic_calc_all_shard")

    def calc_all_finish(self):
        _check(self.lib.galic_calc_all_finish(self.h), "galic_calc_all_finish")

    def optimize_rep(self, idx, seed, rep_serial, form=_ffi.GALIC_FORM_FP64):
        idx = np.ascontiguousarray(idx, dtype=np.int32)
        _check(self.lib.galic_optimize_rep(self.h, _ffi.iptr(idx), len(idx), int(seed), int(rep_serial), form),
               "galic_optimize_rep")

    def optimize_reps(self, idx, seed, rep_serial, form=_ffi.GALIC_FORM_FP64, window_bytes=0, fits=False):
        """idx: [reps, count] particle indices; repetition r draws its
        proposals from serial rep_serial + r (galic_optimize_reps).  With
        fits=True returns the [reps, 4, 7] fit after every repetition."""
        idx = np.ascontiguousarray(idx, dtype=np.int32)
        if idx.ndim != 2:
            raise ValueError("idx must be [reps, count]")
        out = np.zeros((idx.shape[0], 4, 7)) if fits else None
        _check(self.lib.galic_optimize_reps(self.h, _ffi.iptr(idx), idx.shape[1], idx.shape[0], int(seed),
                                            int(rep_serial), form, int(window_bytes),
                                            _ffi.dptr(out) if fits else None), "galic_optimize_reps")
        return out

    def fit(self):
        """4 x 7 array: per type S, Sdisp_r, Sdisp_t, Sdisp_p, Sdisp_q, Srelfac, Srelfac_count."""
        out = np.zeros(28)
        _check(self.lib.galic_get_fit(self.h, _ffi.dptr(out)), "galic_get_fit")
        return out.reshape(4, 7)

    def sall(self):
        """Sall = S + (Sdisp_r+t+p+q)/Srelfac_count per type (main.c:1270)."""
        f = self.fit()
        return f[:, 0] + (f[:, 1] + f[:, 2] + f[:, 3] + f[:, 4]) / np.where(f[:, 6] == 0, 1, f[:, 6])

    def counters(self):
        tr = np.zeros(4, dtype=np.int64)
        ch = np.zeros(4, dtype=np.int64)
        _check(self.lib.galic_get_counters(self.h, _ffi.llptr(tr), _ffi.llptr(ch)), "galic_get_counters")
        return tr, ch

    def response(self, ptype, which):
        out = np.zeros(self.ngrid)
        _check(self.lib.galic_get_response(self.h, int(ptype), int(which), _ffi.dptr(out)), "galic_get_response")
        return out

    def particles(self):
        vel = np.zeros((self.n, 3))
        orbits = np.zeros(self.n, dtype=np.int32)
        vdisp = np.zeros((self.n, 4))
        _check(self.lib.galic_get_particles(self.h, _ffi.dptr(vel), _ffi.iptr(orbits), _ffi.dptr(vdisp)),
               "galic_get_particles")
        return vel, orbits, vdisp

    def set_step_cap(self, cap):
        _check(self.lib.galic_set_step_cap(self.h, int(cap)), "galic_set_step_cap")

    def last_orbit_steps(self):
        return self.lib.galic_last_orbit_steps(self.h)

    def last_timing(self):
        """(ms of the whole last batched call, ms of its orbit kernel), CUDA events."""
        a, b = C.c_double(), C.c_double()
        _check(self.lib.galic_last_timing(self.h, C.byref(a), C.byref(b)), "galic_last_timing")
        return a.value, b.value

    def last_max_energy_error(self):
        return self.lib.galic_last_max_energy_error(self.h)

    def last_kernel_launches(self):
        return self.lib.galic_last_kernel_launches(self.h)
