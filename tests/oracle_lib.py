"""ctypes access to the CPU oracle (test infrastructure only).

* `Oracle` drives oracle/liboracle.so, the C restatement of GALIC's hot path
  (oracle/galic_oracle.c), with either glibc's or the project's
  transcendental functions.
* `Reference` drives oracle/_ref/libgalic_ref.so, GALIC's own C compiled with
  the single-rank MPI / GSL stand-ins.  The reference keeps process-wide
  globals (and calls exit() on fatal errors), so `run_reference` executes each
  scenario in a fresh spawned process.
"""
import ctypes as C
import multiprocessing as mp
import os
import subprocess

import numpy as np

from galic_b200 import _ffi

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
ORACLE_SO = os.path.join(ROOT, "oracle", "liboracle.so")
REF_SO = os.path.join(ROOT, "oracle", "_ref", "libgalic_ref.so")
# GALIC's C with the reference's own optimisation flags (-O3 -march=native):
# the timed CPU baseline; the parity build above has FP contraction off
REF_FAST_SO = os.path.join(ROOT, "oracle", "_ref", "libgalic_ref_fast.so")
# GALIC's C (parity build) with log, atan2, sin, cos, acos from the project's
# gmath.h, the CUDA kernels' elementary functions (oracle/shim/gmath_libm.c)
REF_GMATH_SO = os.path.join(ROOT, "oracle", "_ref", "libgalic_ref_gmath.so")

dptr, iptr = _ffi.dptr, _ffi.iptr
PD, PI, VP = C.POINTER(C.c_double), C.POINTER(C.c_int), C.c_void_p
PP = C.POINTER(_ffi.GalicParams)
PSP = C.POINTER(_ffi.GalicSampleParams)
PST = C.POINTER(_ffi.GalicStream)
PJP = C.POINTER(_ffi.GalicJeansParams)


def build_oracle():
    """Compiles oracle/liboracle.so, and oracle/_ref when the reference tree
    is present (oracle/Makefile locates it: $GALIC_REF_SRC or its default)."""
    subprocess.run(["make", "-s", "-C", os.path.join(ROOT, "oracle"), "restatement"], check=True)
    subprocess.run(["make", "-s", "-j8", "-C", os.path.join(ROOT, "oracle"), "ref"], check=True)


def reference_available():
    return os.path.exists(REF_SO)


def reference_fast_available():
    return os.path.exists(REF_FAST_SO)


def reference_gmath_available():
    return os.path.exists(REF_GMATH_SO)


class OracleGeometry:
    """The restatement's set-up geometry under the names synth.use_geometry()
    expects (galic_grid_geometry, galic_density_geometry, galic_smooth_stack):
    lets a CPU-only process build the synthetic workloads without loading
    libgalic_cuda.so."""

    def __init__(self):
        L = oracle_lib()
        self.galic_grid_geometry = L.orc_grid_geometry
        self.galic_density_geometry = L.orc_density_geometry
        self.galic_smooth_stack = L.orc_smooth_stack


_olib = None


def oracle_lib():
    global _olib
    if _olib is None:
        if not os.path.exists(ORACLE_SO):
            build_oracle()
        L = C.CDLL(ORACLE_SO)
        sig = {
            "orc_create": (VP, [PP, C.c_int]),
            "orc_destroy": (None, [VP]),
            "orc_set_step_cap": (None, [VP, C.c_longlong]),
            "orc_set_force_grid": (None, [VP, PD, PD, PD]),
            "orc_set_vstream": (None, [VP, C.c_int, PD]),
            "orc_set_density_geometry": (None, [VP, PD, PD]),
            "orc_set_targets": (None, [VP, C.c_int, PD, PD, PD, PD, PD, PD]),
            "orc_set_particles": (None, [VP, C.c_int, PD, PD, PD, PD, PD, PI, PD]),
            "orc_get_particles": (None, [VP, PD, PI, PD]),
            "orc_forcegrid_acc": (None, [VP, PD, PD]),
            "orc_forcegrid_pot": (C.c_double, [VP, PD]),
            "orc_densitygrid_cell": (None, [VP, PD, PI, PI, PD, PD]),
            "orc_vstream": (C.c_double, [VP, PD, C.c_int]),
            "orc_orbit_mod": (C.c_double, [VP, PD, PD, PD, PD, PD, PD, PD, C.c_double, C.c_double, PI, C.c_int, PD]),
            "orc_orbit": (C.c_double, [VP, PD, PD, PD, C.c_double, C.c_double, PI, PD]),
            "orc_smooth_stack": (None, [PD, C.c_int]),
            "orc_stack_difference": (C.c_double, [VP, PD, PD, C.c_int, PD, PD, C.c_double, PD, C.c_int]),
            "orc_stack_difference_mod": (C.c_double, [VP, PD, PD, C.c_int, PD, PD, C.c_double, PD, C.c_int]),
            "orc_calc_all": (C.c_int, [VP]),
            "orc_optimize_rep": (C.c_int, [VP, PI, C.c_int, C.c_uint64, C.c_uint32]),
            "orc_get_fit": (None, [VP, PD]),
            "orc_get_counters": (None, [VP, C.POINTER(C.c_longlong), C.POINTER(C.c_longlong)]),
            "orc_get_response": (None, [VP, C.c_int, C.c_int, PD]),
            "orc_steps_total": (C.c_longlong, [VP]),
            "orc_grid_geometry": (C.c_int, [C.c_double, C.c_double, C.c_double, C.c_int, C.c_int, C.c_int, PD]),
            "orc_density_geometry": (C.c_int, [C.c_int, C.c_double, C.c_double, PD, PD, PD]),
            "orc_peano_key": (C.c_uint64, [C.c_int, C.c_int, C.c_int, C.c_int]),
            "orc_force_grid_fill": (C.c_int, [C.POINTER(_ffi.GalicFillParams), C.c_int, PD, PD, PD, PD, PD]),
            "orc_sample_positions": (None, [PSP, C.c_int, C.c_longlong, PST, C.c_int, PD]),
            "orc_calculate_dispfield": (C.c_int, [VP, PSP, PJP, PD]),
            "orc_initialize_particles": (C.c_int, [VP, PSP, C.c_double, C.POINTER(C.POINTER(PD)), PST, C.c_int,
                                                   PD, PD, PD, PD, PD, PD, PD, PI, PI, PI, PI]),
            "orc_sample_density": (None, [PP, PSP, C.c_int, C.c_longlong, PST, C.c_int, C.c_int, PD]),
            "orc_sample_energy": (None, [PP, PSP, C.c_int, C.c_longlong, PST, C.c_int, C.POINTER(PD), PD]),
        }
        for name, (res, args) in sig.items():
            f = getattr(L, name)
            f.restype = res
            f.argtypes = args
        _olib = L
    return _olib


class Oracle:
    """The C restatement; use_libm=True pins it to the reference, False matches the CUDA kernels."""

    def __init__(self, params, use_libm=False):
        self.L = oracle_lib()
        self.params = params.copy()
        self.h = self.L.orc_create(C.byref(self.params), 1 if use_libm else 0)
        Lv = params.DG_MaxLevel
        self.ngrid = 1 << (2 * Lv)
        self.nstack = ((1 << (2 + 2 * Lv)) - 1) // 3
        self.n = 0

    def __del__(self):
        if getattr(self, "h", None):
            self.L.orc_destroy(self.h)
            self.h = None

    def load_model(self, m, particles=True):
        self.L.orc_set_force_grid(self.h, dptr(m.pot), dptr(m.dpotdr), dptr(m.dpotdz))
        for t in (1, 2, 3):
            self.L.orc_set_vstream(self.h, t, dptr(np.ascontiguousarray(m.vstream[t], dtype=np.float64)))
        self.L.orc_set_density_geometry(self.h, dptr(m.cellsize), dptr(m.dgs_distance))
        for t, tg in m.targets.items():
            self.L.orc_set_targets(self.h, t, *[dptr(np.ascontiguousarray(a)) for a in tg])
        if particles:
            self.set_particles(m.pos, m.vel, m.mass, m.tint, m.vesc, m.ptype, m.ptargets)

    def set_particles(self, pos, vel, mass, tint, vesc, ptype, ptargets):
        arrs = [np.ascontiguousarray(a, dtype=np.float64) for a in (pos, vel, mass, tint, vesc)]
        self.L.orc_set_particles(self.h, len(mass), *[dptr(a) for a in arrs],
                                 iptr(np.ascontiguousarray(ptype, dtype=np.int32)),
                                 dptr(np.ascontiguousarray(ptargets, dtype=np.float64)))
        self.n = len(mass)

    def orbit_mod(self, pos, vel, mass, timespan, ptype):
        g = [np.zeros(self.ngrid) for _ in range(5)]
        orbits = C.c_int(0)
        info = np.zeros(2)
        tall = self.L.orc_orbit_mod(self.h, dptr(np.ascontiguousarray(pos, dtype=np.float64)),
                                    dptr(np.ascontiguousarray(vel, dtype=np.float64)), *[dptr(a) for a in g],
                                    float(mass), float(timespan), C.byref(orbits), int(ptype), dptr(info))
        return tall, orbits.value, g[0], g[1], g[2], g[3], g[4], info

    def orbit(self, pos, vel, mass, timespan):
        m = np.zeros(self.ngrid)
        orbits = C.c_int(0)
        info = np.zeros(2)
        tall = self.L.orc_orbit(self.h, dptr(np.ascontiguousarray(pos, dtype=np.float64)),
                                dptr(np.ascontiguousarray(vel, dtype=np.float64)), dptr(m), float(mass),
                                float(timespan), C.byref(orbits), dptr(info))
        return tall, orbits.value, m, info

    def calc_all(self):
        return self.L.orc_calc_all(self.h)

    def optimize_rep(self, idx, seed, rep_serial):
        idx = np.ascontiguousarray(idx, dtype=np.int32)
        return self.L.orc_optimize_rep(self.h, iptr(idx), len(idx), int(seed), int(rep_serial))

    def fit(self):
        out = np.zeros(28)
        self.L.orc_get_fit(self.h, dptr(out))
        return out.reshape(4, 7)

    def counters(self):
        tr = np.zeros(4, dtype=np.int64)
        ch = np.zeros(4, dtype=np.int64)
        self.L.orc_get_counters(self.h, _ffi.llptr(tr), _ffi.llptr(ch))
        return tr, ch

    def response(self, ptype, which):
        out = np.zeros(self.ngrid)
        self.L.orc_get_response(self.h, int(ptype), int(which), dptr(out))
        return out

    def particles(self):
        vel = np.zeros((self.n, 3))
        orbits = np.zeros(self.n, dtype=np.int32)
        vdisp = np.zeros((self.n, 4))
        self.L.orc_get_particles(self.h, dptr(vel), iptr(orbits), dptr(vdisp))
        return vel, orbits, vdisp

    def steps_total(self):
        return self.L.orc_steps_total(self.h)


# --------------------------------------------------------------- the reference


class RefFillParams(C.Structure):
    """ref_fill_params of oracle/ref_driver.c: the All.* members of the fill."""
    _fields_ = [("Softening", C.c_double), ("ErrTolTheta", C.c_double), ("TopNodeFactor", C.c_double),
                ("Disk_H", C.c_double), ("Disk_Z0", C.c_double), ("Rmax", C.c_double),
                ("MultipleDomains", C.c_int), ("SampleForceNhalo", C.c_int), ("SampleForceNdisk", C.c_int),
                ("SampleForceNbulge", C.c_int), ("seed", C.c_ulonglong)]


def oracle_force_grid_fill(fp, pos, mass):
    """orc_force_grid_fill: (status, FG_DPotDR, FG_DPotDz, FG_Pot) as [N, N] arrays."""
    L = oracle_lib()
    pos = np.ascontiguousarray(pos, dtype=np.float64)
    mass = np.ascontiguousarray(mass, dtype=np.float64)
    N = fp.FG_Nbin
    out = [np.zeros((N, N)) for _ in range(3)]
    st = L.orc_force_grid_fill(C.byref(fp), len(mass), dptr(pos), dptr(mass), *[dptr(a) for a in out])
    return st, out[0], out[1], out[2]


def fill_masses(params, nh, nd, nb):
    """P[].Mass of the sampled particles (grid.c:662-678)."""
    m = []
    if nh:
        m += [params.Halo_Mass / nh] * nh
    if nd:
        m += [params.Disk_Mass / nd] * nd
    if nb:
        m += [params.Bulge_Mass / nb] * nb
    return np.array(m, dtype=np.float64)


def reference_force_fill(params, rf, with_grid=True):
    """GALIC's own forcedensitygrid_calculate (one rank) for the model `params`
    and fill settings `rf` (RefFillParams); returns (pos[n,3], mass[n],
    FG_DPotDR, FG_DPotDz, FG_Pot).  Run it through run_reference()."""
    import tempfile
    L = _ref_lib()
    L.ref_setup(C.byref(params))
    n = rf.SampleForceNhalo + rf.SampleForceNdisk + rf.SampleForceNbulge
    pos = np.zeros((n, 3))
    L.ref_fill_positions(C.byref(rf), dptr(pos))
    mass = fill_masses(params, rf.SampleForceNhalo, rf.SampleForceNdisk, rf.SampleForceNbulge)
    N = params.FG_Nbin
    out = [np.zeros((N, N)) for _ in range(3)]
    if with_grid:
        with tempfile.TemporaryDirectory() as d:
            st = L.ref_force_fill(d.encode(), C.byref(rf), *[dptr(a) for a in out])
        if st != 0:
            raise RuntimeError(f"ref_force_fill status {st}")
    return pos, mass, out[0], out[1], out[2]


# ------------------------------------------------------------ set-up sampling
# stream = (seed, a, b, position); tables = {type: (disp_r, dispz, dispphi,
# tilted_vr2, tilted_vz2, vstream)} with None where a table is not read

def _stream(st):
    return _ffi.GalicStream(int(st[0]), int(st[1]), int(st[2]), int(st[3]))


def _stack_size(L):
    return ((1 << (2 + 2 * L)) - 1) // 3


def oracle_positions(sp, ptype, n, stream, use_libm):
    """orc_sample_positions: ([n, 3] positions, stream position after)."""
    s = _stream(stream)
    pos = np.zeros((n, 3))
    oracle_lib().orc_sample_positions(C.byref(sp), ptype, n, C.byref(s), 1 if use_libm else 0, dptr(pos))
    return pos, int(s.position)


def oracle_density(params, sp, ptype, ntarget, stream, use_libm, renorm=False):
    """orc_sample_density: (DGs_MassTarget stack, stream position after)."""
    s = _stream(stream)
    out = np.zeros(_stack_size(params.DG_MaxLevel))
    oracle_lib().orc_sample_density(C.byref(params), C.byref(sp), ptype, ntarget, C.byref(s), 1 if use_libm else 0,
                                    1 if renorm else 0, dptr(out))
    return out, int(s.position)


def oracle_energy(params, sp, ptype, ntarget, stream, use_libm, tab):
    """orc_sample_energy: ([5, Nstack] mass, r, t, p, q stacks, stream position after)."""
    s = _stream(stream)
    Ns = _stack_size(params.EG_MaxLevel)
    out = np.zeros((5, Ns))
    keep = [None if a is None else np.ascontiguousarray(a, dtype=np.float64).ravel() for a in tab]
    arr = (PD * 6)(*[dptr(a) if a is not None else PD() for a in keep])
    oracle_lib().orc_sample_energy(C.byref(params), C.byref(sp), ptype, ntarget, C.byref(s), 1 if use_libm else 0,
                                   arr, dptr(out))
    return out, int(s.position)


def reference_sampling(params, sp, ntarget, stream, kind, tables=None):
    """GALIC's own densitygrid_sample_targetresponse (kind "density") or
    calc_energy_grid_mass_maps (kind "energy") with one rank; returns
    ({type: six target stacks}, stream position after).  Run it through
    run_reference()."""
    L = _ref_lib()
    L.ref_setup(C.byref(params))
    L.ref_sample_setup(C.byref(sp), int(ntarget))
    keep = []
    for t, tab in (tables or {}).items():
        arrs = [None if a is None else np.ascontiguousarray(a, dtype=np.float64).ravel() for a in tab]
        keep.append(arrs)
        L.ref_set_dispersion(t, *[dptr(a) for a in arrs[:5]])
        if len(arrs) > 5 and arrs[5] is not None:
            L.ref_set_vstream(t, dptr(arrs[5]))
    L.ref_rng_stream(*[int(x) for x in stream])
    (L.ref_sample_density if kind == "density" else L.ref_sample_energy)()
    Ns = _stack_size(params.DG_MaxLevel)
    out = {}
    for t in (1, 2, 3):
        st = [np.zeros(Ns) for _ in range(6)]
        L.ref_get_targets(t, *[dptr(a) for a in st])
        out[t] = st
    return out, int(L.ref_rng_position())


def reference_positions(params, sp, ptype, n, stream):
    """n calls of GALIC's own *_get_fresh_coordinate: ([n, 3], stream position after)."""
    L = _ref_lib()
    L.ref_setup(C.byref(params))
    L.ref_sample_setup(C.byref(sp), 1)
    L.ref_rng_stream(*[int(x) for x in stream])
    pos = np.zeros((n, 3))
    L.ref_fresh_positions(int(ptype), int(n), dptr(pos))
    return pos, int(L.ref_rng_position())


def oracle_dispfield(m, sp, jp, use_libm):
    """orc_calculate_dispfield on the model's force grid: (status, [4, 8, N, N] tables)."""
    o = Oracle(m.params, use_libm=use_libm)
    o.load_model(m, particles=False)
    N = m.params.FG_Nbin
    out = np.zeros((4, 8, N, N))
    st = o.L.orc_calculate_dispfield(o.h, C.byref(sp), C.byref(jp), dptr(out))
    return st, out


def reference_dispfield(params, m_arrays, sp, jp):
    """GALIC's own calculate_dispfield (one rank) on the force grid
    m_arrays = (pot, dpotdr, dpotdz): [4, 8, N, N] tables of the types it
    computes.  Run it through run_reference()."""
    import tempfile
    L = _ref_lib()
    L.ref_setup(C.byref(params))
    pot, dpotdr, dpotdz = [np.ascontiguousarray(a, dtype=np.float64) for a in m_arrays]
    L.ref_set_force_grid(dptr(pot), dptr(dpotdr), dptr(dpotdz))
    with tempfile.TemporaryDirectory() as d:
        st = L.ref_calculate_dispfield(d.encode(), C.byref(sp), C.byref(jp))
    if st != 0:
        raise RuntimeError(f"ref_calculate_dispfield status {st}")
    N = params.FG_Nbin
    out = np.zeros((4, 8, N, N))
    for t in (1, 2, 3):
        L.ref_get_jeans(t, dptr(out[t]))
    return out


PARTICLE_FIELDS = (("pos", 3, np.float64), ("vel", 3, np.float64), ("vel_theo", 3, np.float64),
                   ("mass", 1, np.float64), ("vesc", 1, np.float64), ("tint", 1, np.float64),
                   ("targets", 4, np.float64), ("type", 1, np.int32), ("id", 1, np.int32), ("perm", 1, np.int32))


def _particle_arrays(n):
    return {k: np.zeros((n, w) if w > 1 else n, dtype=dt) for k, w, dt in PARTICLE_FIELDS}


def _ptr(a):
    return dptr(a) if a.dtype == np.float64 else iptr(a)


def oracle_particles(m, sp, torbit_fac, tables, stream, use_libm):
    """orc_initialize_particles on the model's force grid; tables = {type:
    (FG_Disp_r, FG_DispZ, FG_DispPhi, FG_tilted_vR2_prime, FG_tilted_vz2_prime,
    FG_Vstream)}.  Returns (status, {field: array}, low-dispersion counts [4, 4],
    stream position after)."""
    o = Oracle(m.params, use_libm=use_libm)
    o.load_model(m, particles=False)
    n = sum(m.params.NType[t] for t in (1, 2, 3))
    out = _particle_arrays(n)
    keep = {t: [np.ascontiguousarray(a, dtype=np.float64).ravel() for a in tab] for t, tab in tables.items()}
    rows = (C.POINTER(PD) * 4)()
    inner = {}
    for t in (1, 2, 3):
        if t in keep:
            inner[t] = (PD * 6)(*[dptr(a) for a in keep[t]])
            rows[t] = C.cast(inner[t], C.POINTER(PD))
    counts = np.zeros((4, 4), dtype=np.int32)
    s = _stream(stream)
    st = o.L.orc_initialize_particles(o.h, C.byref(sp), float(torbit_fac), rows, C.byref(s), 1 if use_libm else 0,
                                      *[_ptr(out[k]) for k, _, _ in PARTICLE_FIELDS], iptr(counts))
    return st, out, counts, int(s.position)


def reference_particles(params, grid, sp, torbit_fac, tables, stream):
    """GALIC's own initialize_particles (one rank) with the force grid
    grid = (pot, dpotdr, dpotdz) and tables as for oracle_particles: returns
    ({field: array}, stream position after).  Run it through run_reference()."""
    import tempfile
    L = _ref_lib()
    L.ref_setup(C.byref(params))
    pot, dpotdr, dpotdz = [np.ascontiguousarray(a, dtype=np.float64) for a in grid]
    L.ref_set_force_grid(dptr(pot), dptr(dpotdr), dptr(dpotdz))
    keep = []
    for t, tab in tables.items():
        arrs = [np.ascontiguousarray(a, dtype=np.float64).ravel() for a in tab]
        keep.append(arrs)
        L.ref_set_dispersion(t, dptr(arrs[0]), dptr(arrs[1]), dptr(arrs[2]), dptr(arrs[3]), dptr(arrs[4]))
        L.ref_set_vstream(t, dptr(arrs[5]))
    L.ref_rng_stream(*[int(x) for x in stream])
    with tempfile.TemporaryDirectory() as d:
        n = L.ref_initialize_particles(d.encode(), C.byref(sp), float(torbit_fac))
    out = _particle_arrays(n)
    L.ref_get_init_particles(*[_ptr(out[k]) for k, _, _ in PARTICLE_FIELDS])
    return out, int(L.ref_rng_position())


# ------------------------------------------------------------ output files

def reference_snapshot(params, grid, sp, torbit_fac, tables, stream, fmt):
    """GALIC's own initialize_particles, then output_particles with SnapFormat
    fmt: ({field: array} of the particles, the snapshot file's bytes).  Run it
    through run_reference()."""
    import tempfile
    L = _ref_lib()
    L.ref_setup(C.byref(params))
    pot, dpotdr, dpotdz = [np.ascontiguousarray(a, dtype=np.float64) for a in grid]
    L.ref_set_force_grid(dptr(pot), dptr(dpotdr), dptr(dpotdz))
    keep = []
    for t, tab in tables.items():
        arrs = [np.ascontiguousarray(a, dtype=np.float64).ravel() for a in tab]
        keep.append(arrs)
        L.ref_set_dispersion(t, dptr(arrs[0]), dptr(arrs[1]), dptr(arrs[2]), dptr(arrs[3]), dptr(arrs[4]))
        L.ref_set_vstream(t, dptr(arrs[5]))
    L.ref_rng_stream(*[int(x) for x in stream])
    with tempfile.TemporaryDirectory() as d:
        n = L.ref_initialize_particles(d.encode(), C.byref(sp), float(torbit_fac))
        out = _particle_arrays(n)
        L.ref_get_init_particles(*[_ptr(out[k]) for k, _, _ in PARTICLE_FIELDS])
        L.ref_output_particles((d + "/").encode(), int(fmt))
        with open(os.path.join(d, "snap_000"), "rb") as f:
            data = f.read()
    return out, data


def reference_density_field(m):
    """GALIC's own calc_all_response_fields on the model, then
    output_density_field: {type: (file bytes, six target stacks, the committed
    grids MASS_S, MASS_I, R_I, T_I, P_I, Q_I)}.  Run it through run_reference()."""
    import tempfile
    r = Reference(m.params)
    r.load_model(m)
    r.calc_all()
    res = {}
    with tempfile.TemporaryDirectory() as d:
        r.L.ref_output_density_field(d.encode())
        for t in (1, 2, 3):
            if m.params.NType[t] == 0:
                continue
            with open(os.path.join(d, f"densfield_{t}_000.dat"), "rb") as f:
                data = f.read()
            st = [np.zeros(r.nstack) for _ in range(6)]
            r.L.ref_get_targets(t, *[dptr(a) for a in st])
            locs = [r.response(t, w) for w in (_ffi.GRID_MASS_S, _ffi.GRID_MASS_I, _ffi.GRID_R_I, _ffi.GRID_T_I,
                                               _ffi.GRID_P_I, _ffi.GRID_Q_I)]
            res[t] = (data, st, locs)
    return res


def reference_forcefield(params, rf):
    """GALIC's own forcedensitygrid_calculate (one rank): (FG_DPotDR, FG_DPotDz,
    FG_Pot, the bytes of the forcefield.dat it writes).  Run it through
    run_reference()."""
    import tempfile
    L = _ref_lib()
    L.ref_setup(C.byref(params))
    N = params.FG_Nbin
    out = [np.zeros((N, N)) for _ in range(3)]
    with tempfile.TemporaryDirectory() as d:
        st = L.ref_force_fill(d.encode(), C.byref(rf), *[dptr(a) for a in out])
        if st != 0:
            raise RuntimeError(f"ref_force_fill status {st}")
        with open(os.path.join(d, "forcefield.dat"), "rb") as f:
            data = f.read()
    return out[0], out[1], out[2], data


def reference_peano_keys(xyz, bits):
    L = _ref_lib()
    return np.array([L.ref_peano_key(int(x), int(y), int(z), bits) for x, y, z in xyz], dtype=np.uint64)


def _ref_lib(fast=False, gmath=False):
    L = C.CDLL(REF_GMATH_SO if gmath else (REF_FAST_SO if fast else REF_SO))
    sig = {
        "ref_setup": (C.c_int, [PP]),
        "ref_set_force_grid": (None, [PD, PD, PD]),
        "ref_set_vstream": (None, [C.c_int, PD]),
        "ref_set_density_geometry": (None, [PD, PD]),
        "ref_set_targets": (None, [C.c_int, PD, PD, PD, PD, PD, PD]),
        "ref_set_particles": (None, [C.c_int, PD, PD, PD, PD, PD, PI, PD]),
        "ref_get_particles": (None, [PD, PI, PD]),
        "ref_orbit_mod": (C.c_double, [PD, PD, PD, PD, PD, PD, PD, C.c_double, C.c_double, PI, C.c_int]),
        "ref_orbit": (C.c_double, [PD, PD, PD, C.c_double, C.c_double, PI]),
        "ref_forcegrid_acc": (None, [PD, PD]),
        "ref_forcegrid_pot": (C.c_double, [PD]),
        "ref_densitygrid_cell": (None, [PD, PI, PI, PD, PD]),
        "ref_vstream": (C.c_double, [PD, C.c_int]),
        "ref_calc_all": (None, []),
        "ref_optimize_rep": (None, [PI, C.c_int, C.c_ulonglong, C.c_uint]),
        "ref_get_fit": (None, [PD]),
        "ref_get_counters": (None, [C.POINTER(C.c_longlong), C.POINTER(C.c_longlong)]),
        "ref_get_response": (None, [C.c_int, C.c_int, PD]),
        "ref_smooth_stack": (None, [PD, C.c_int]),
        "ref_stack_difference": (C.c_double, [PD, PD, C.c_int, PD, PD, C.c_double, PD, C.c_int]),
        "ref_stack_difference_mod": (C.c_double, [PD, PD, C.c_int, PD, PD, C.c_double, PD, C.c_int]),
        "ref_geometry": (C.c_int, [C.c_char_p, C.c_double, C.c_double, PD, PD, PD, PD]),
        "ref_fill_positions": (None, [C.POINTER(RefFillParams), PD]),
        "ref_force_fill": (C.c_int, [C.c_char_p, C.POINTER(RefFillParams), PD, PD, PD]),
        "ref_peano_key": (C.c_ulonglong, [C.c_int, C.c_int, C.c_int, C.c_int]),
        "ref_rng_stream": (None, [C.c_ulonglong, C.c_uint, C.c_uint, C.c_ulonglong]),
        "ref_rng_position": (C.c_ulonglong, []),
        "ref_sample_setup": (None, [PSP, C.c_longlong]),
        "ref_set_dispersion": (None, [C.c_int, PD, PD, PD, PD, PD]),
        "ref_sample_density": (None, []),
        "ref_sample_energy": (None, []),
        "ref_get_targets": (None, [C.c_int, PD, PD, PD, PD, PD, PD]),
        "ref_fresh_positions": (None, [C.c_int, C.c_longlong, PD]),
        "ref_calculate_dispfield": (C.c_int, [C.c_char_p, PSP, PJP]),
        "ref_get_jeans": (None, [C.c_int, PD]),
        "ref_initialize_particles": (C.c_int, [C.c_char_p, PSP, C.c_double]),
        "ref_output_particles": (None, [C.c_char_p, C.c_int]),
        "ref_output_density_field": (None, [C.c_char_p]),
        "ref_get_init_particles": (None, [PD, PD, PD, PD, PD, PD, PD, PI, PI, PI]),
    }
    for name, (res, args) in sig.items():
        f = getattr(L, name)
        f.restype = res
        f.argtypes = args
    return L


class Reference:
    """GALIC's own C (one model per process: the reference keeps globals).
    fast=True loads the build with the reference's own optimisation flags
    (the timed baseline) instead of the contraction-free parity build;
    gmath=True loads the parity build whose elementary functions are the
    CUDA kernels' (gmath.h)."""

    def __init__(self, params, fast=False, gmath=False):
        self.L = _ref_lib(fast, gmath)
        self.params = params.copy()
        self.L.ref_setup(C.byref(self.params))
        Lv = params.DG_MaxLevel
        self.ngrid = 1 << (2 * Lv)
        self.nstack = ((1 << (2 + 2 * Lv)) - 1) // 3
        self.n = 0

    def load_model(self, m, particles=True):
        self.L.ref_set_force_grid(dptr(m.pot), dptr(m.dpotdr), dptr(m.dpotdz))
        for t in (1, 2, 3):
            self.L.ref_set_vstream(t, dptr(np.ascontiguousarray(m.vstream[t], dtype=np.float64)))
        self.L.ref_set_density_geometry(dptr(m.cellsize), dptr(m.dgs_distance))
        for t, tg in m.targets.items():
            self.L.ref_set_targets(t, *[dptr(np.ascontiguousarray(a)) for a in tg])
        if not particles:
            return
        arrs = [np.ascontiguousarray(a, dtype=np.float64) for a in (m.pos, m.vel, m.mass, m.tint, m.vesc)]
        self.L.ref_set_particles(len(m.mass), *[dptr(a) for a in arrs],
                                 iptr(np.ascontiguousarray(m.ptype, dtype=np.int32)),
                                 dptr(np.ascontiguousarray(m.ptargets, dtype=np.float64)))
        self.n = len(m.mass)

    def orbit_mod(self, pos, vel, mass, timespan, ptype):
        g = [np.zeros(self.ngrid) for _ in range(5)]
        orbits = C.c_int(0)
        p = np.array(pos, dtype=np.float64)
        v = np.array(vel, dtype=np.float64)
        tall = self.L.ref_orbit_mod(dptr(p), dptr(v), *[dptr(a) for a in g], float(mass), float(timespan),
                                    C.byref(orbits), int(ptype))
        return tall, orbits.value, g[0], g[1], g[2], g[3], g[4]

    def orbit(self, pos, vel, mass, timespan):
        m = np.zeros(self.ngrid)
        orbits = C.c_int(0)
        p = np.array(pos, dtype=np.float64)
        v = np.array(vel, dtype=np.float64)
        tall = self.L.ref_orbit(dptr(p), dptr(v), dptr(m), float(mass), float(timespan), C.byref(orbits))
        return tall, orbits.value, m

    def calc_all(self):
        self.L.ref_calc_all()

    def optimize_rep(self, idx, seed, rep_serial):
        idx = np.ascontiguousarray(idx, dtype=np.int32)
        self.L.ref_optimize_rep(iptr(idx), len(idx), int(seed), int(rep_serial))

    def fit(self):
        out = np.zeros(28)
        self.L.ref_get_fit(dptr(out))
        return out.reshape(4, 7)

    def counters(self):
        tr = np.zeros(4, dtype=np.int64)
        ch = np.zeros(4, dtype=np.int64)
        self.L.ref_get_counters(_ffi.llptr(tr), _ffi.llptr(ch))
        return tr, ch

    def response(self, ptype, which):
        out = np.zeros(self.ngrid)
        self.L.ref_get_response(int(ptype), int(which), dptr(out))
        return out

    def particles(self):
        vel = np.zeros((self.n, 3))
        orbits = np.zeros(self.n, dtype=np.int32)
        vdisp = np.zeros((self.n, 4))
        self.L.ref_get_particles(dptr(vel), iptr(orbits), dptr(vdisp))
        return vel, orbits, vdisp


def reference_calc_all(arrays, gmath=False, orbits=()):
    """GALIC's own calc_all_response_fields (main.c:151-362, one rank) on a
    model given as tests/golden/make_golden.py arrays; returns ({type: [10,
    Ngrid] committed grids}, fit [4, 7], [orbit_mod results of the particles
    `orbits`]).  gmath=True: the build with the CUDA kernels' elementary
    functions.  Run it through run_reference()."""
    import sys

    sys.path.insert(0, os.path.join(ROOT, "tests", "golden"))
    from make_golden import model_from_arrays

    m = model_from_arrays(arrays)
    ref = Reference(m.params, gmath=gmath)
    ref.load_model(m)
    per_orbit = [ref.orbit_mod(m.pos[i], m.vel[i], m.mass[i], m.tint[i], m.ptype[i]) for i in orbits]
    ref.calc_all()
    grids = {t: np.stack([ref.response(t, w) for w in range(_ffi.GRID_COUNT)]) for t in (1, 2, 3)
             if m.params.NType[t]}
    return grids, ref.fit(), per_orbit


def _child(fn, args, q):
    try:
        q.put(("ok", fn(*args)))
    except BaseException as e:  # noqa: BLE001
        q.put(("err", repr(e)))


def run_reference(fn, *args, timeout=600):
    """Runs fn(*args) in a fresh spawned process (fn must be importable)."""
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    p = ctx.Process(target=_child, args=(fn, args, q))
    p.start()
    try:
        kind, val = q.get(timeout=timeout)
    finally:
        p.join(timeout=30)
        if p.is_alive():
            p.kill()
    if kind != "ok":
        raise RuntimeError(f"reference scenario failed: {val}")
    return val
