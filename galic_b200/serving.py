"""Serving loop through the C ABI (galic_server_*).

`Server(budget_bytes, workers)` admits model-construction jobs by HBM budget
and runs them concurrently on the current device; `submit(model, ...)` queues
one synth.Model (or any object with the same fields) with an optimisation
schedule and returns a job id; `wait(id)` returns the job's result as a dict.
The model's arrays are kept alive by the Server until the job is done.
There is no CPU fallback.
"""
import ctypes as C

import numpy as np

from . import _ffi
from .context import _check


def _job(model, form, max_iterations, reps_per_iteration, fraction_per_rep, converge_rel, seed, permutation,
         want_velocities):
    keep = []

    def d(a):
        a = np.ascontiguousarray(a, dtype=np.float64)
        keep.append(a)
        return _ffi.dptr(a)

    j = _ffi.GalicJob()
    prm = model.params.copy()
    keep.append(prm)
    j.prm = C.pointer(prm)
    j.fg_pot, j.fg_dpotdr, j.fg_dpotdz = d(model.pot), d(model.dpotdr), d(model.dpotdz)
    for t in (1, 2, 3):
        j.vstream[t] = d(model.vstream[t])
    j.cellsize, j.dgs_distance = d(model.cellsize), d(model.dgs_distance)
    for t, tg in model.targets.items():
        for k, a in enumerate(tg):
            j.targets[t][k] = d(a)
    j.n = len(model.mass)
    j.pos, j.vel, j.mass, j.tint, j.vesc = (d(model.pos), d(model.vel), d(model.mass), d(model.tint),
                                            d(model.vesc))
    j.ptargets = d(model.ptargets)
    ty = np.ascontiguousarray(model.ptype, dtype=np.int32)
    keep.append(ty)
    j.type = _ffi.iptr(ty)
    j.form = int(form)
    j.max_iterations = int(max_iterations)
    j.reps_per_iteration = int(reps_per_iteration)
    j.fraction_per_rep = float(fraction_per_rep)
    j.converge_rel = float(converge_rel)
    j.seed = int(seed)
    if permutation is not None:
        perm = np.ascontiguousarray(permutation, dtype=np.int32)
        keep.append(perm)
        j.permutation = _ffi.iptr(perm)
    vel_out = None
    if want_velocities:
        vel_out = np.zeros((j.n, 3))
        keep.append(vel_out)
        j.vel_out = _ffi.dptr(vel_out)
    return j, keep, vel_out


class Server:
    def __init__(self, budget_bytes, workers=4):
        self.lib = _ffi.load_library()
        h = C.c_void_p()
        _check(self.lib.galic_server_create(int(budget_bytes), int(workers), C.byref(h)), "galic_server_create")
        self.h = h
        self._jobs = {}

    def close(self):
        if getattr(self, "h", None):
            self.lib.galic_server_destroy(self.h)
            self.h = None
            self._jobs.clear()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def submit(self, model, form=_ffi.GALIC_FORM_FP32, max_iterations=2, reps_per_iteration=4,
               fraction_per_rep=0.001, converge_rel=0.0, seed=1, permutation=None, want_velocities=False):
        job, keep, vel_out = _job(model, form, max_iterations, reps_per_iteration, fraction_per_rep, converge_rel,
                                  seed, permutation, want_velocities)
        jid = C.c_int()
        _check(self.lib.galic_server_submit(self.h, C.byref(job), C.byref(jid)), "galic_server_submit")
        self._jobs[jid.value] = (job, keep, vel_out)
        return jid.value

    @staticmethod
    def job_bytes(model, fraction_per_rep=0.001):
        job, keep, _ = _job(model, 0, 0, 0, fraction_per_rep, 0.0, 0, None, False)
        return int(_ffi.load_library().galic_job_device_bytes(C.byref(job)))

    def wait(self, job_id, timeout=600.0):
        r = _ffi.GalicJobResult()
        _check(self.lib.galic_server_wait(self.h, int(job_id), float(timeout), C.byref(r)), "galic_server_wait")
        out = {k: getattr(r, k) for k, _ in _ffi.GalicJobResult._fields_}
        out["fit"] = np.array(r.fit[:]).reshape(4, 7)
        vel_out = self._jobs.get(job_id, (None, None, None))[2]
        if vel_out is not None:
            out["vel"] = vel_out.copy()
        self._jobs.pop(job_id, None)
        return out

    def stats(self):
        pb = C.c_size_t()
        pr, q, r = C.c_int(), C.c_int(), C.c_int()
        _check(self.lib.galic_server_stats(self.h, C.byref(pb), C.byref(pr), C.byref(q), C.byref(r)),
               "galic_server_stats")
        return {"peak_bytes": pb.value, "peak_running": pr.value, "queued": q.value, "running": r.value}
