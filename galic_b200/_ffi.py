"""ctypes view of the C ABI in include/galic_gpu.h.

`GalicParams` mirrors `galic_params_t` field for field; `load_library()`
opens the in-tree libgalic_cuda.so and declares every entry point.  There is
no fallback: if the library is missing the import fails with the build
command to run.
"""
import ctypes as C
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libgalic_cuda.so")

GALIC_FORM_FP64 = 0
GALIC_FORM_FP32 = 1

# galic_grid_id
GRID_MASS_S, GRID_R_S, GRID_T_S, GRID_Q_S, GRID_P_S = 0, 1, 2, 3, 4
GRID_MASS_I, GRID_R_I, GRID_T_I, GRID_P_I, GRID_Q_I = 5, 6, 7, 8, 9
GRID_COUNT = 10

STATUS_NAMES = {
    0: "GALIC_OK", 1: "GALIC_ERR_INVALID_ARGUMENT", 2: "GALIC_ERR_STEP_CAP", 3: "GALIC_ERR_CUDA",
    4: "GALIC_ERR_NO_DEVICE", 5: "GALIC_ERR_BUDGET", 6: "GALIC_ERR_UNSUPPORTED",
    7: "GALIC_ERR_REJECTION_CAP", 8: "GALIC_ERR_OVERFLOW", 9: "GALIC_ERR_STATE",
}

D4 = C.c_double * 4
I4 = C.c_int * 4


class GalicParams(C.Structure):
    _fields_ = [
        ("V200", C.c_double), ("M200", C.c_double), ("R200", C.c_double), ("G", C.c_double),
        ("Halo_Mass", C.c_double), ("Halo_A", C.c_double), ("HaloStretch", C.c_double),
        ("Disk_Mass", C.c_double),
        ("Bulge_Mass", C.c_double), ("Bulge_A", C.c_double), ("BulgeStretch", C.c_double),
        ("TimeStepFactorOrbit", C.c_double), ("TimeStepFactorCellCross", C.c_double),
        ("LowerDispLimit", C.c_double), ("MaxVelInUnitsVesc", C.c_double),
        ("SampleForceNhalo", C.c_int), ("SampleForceNdisk", C.c_int), ("SampleForceNbulge", C.c_int),
        ("TypeOfVelocityStructure", I4),
        ("MinParticlesPerBinForDispersionMeasurement", C.c_int),
        ("MinParticlesPerBinForDensityMeasurement", C.c_int),
        ("MType", D4), ("NType", I4),
        ("fac_value_rs", D4), ("fac_value_ts", D4), ("fac_value_qs", D4), ("fac_value_ps", D4),
        ("FG_Nbin", C.c_int), ("DG_MaxLevel", C.c_int), ("EG_MaxLevel", C.c_int),
        ("FG_Rmin", C.c_double), ("FG_Fac", C.c_double), ("DG_Rmin", C.c_double),
        ("DG_Fac", C.c_double), ("EG_Rmin", C.c_double), ("EG_Fac", C.c_double),
    ]

    def copy(self):
        other = GalicParams()
        C.memmove(C.byref(other), C.byref(self), C.sizeof(GalicParams))
        return other


class GalicFillParams(C.Structure):
    """galic_fill_params_t: parameters of the tree force-grid fill."""
    _fields_ = [
        ("FG_Nbin", C.c_int), ("MultipleDomains", C.c_int),
        ("FG_Rmin", C.c_double), ("FG_Fac", C.c_double), ("G", C.c_double),
        ("ForceSoftening", C.c_double), ("ErrTolTheta", C.c_double), ("TopNodeFactor", C.c_double),
    ]


class GalicFillStats(C.Structure):
    """galic_fill_stats_t: diagnostics of one fill."""
    _fields_ = [("ms_walk", C.c_double), ("ms_total", C.c_double), ("tree_items", C.c_longlong),
                ("tree_nodes", C.c_longlong), ("interactions", C.c_longlong), ("node_tests", C.c_longlong)]


PD_ = C.POINTER(C.c_double)


class GalicJob(C.Structure):
    """galic_job_t: one model-construction job of the serving loop."""
    _fields_ = [
        ("prm", C.POINTER(GalicParams)),
        ("fg_pot", PD_), ("fg_dpotdr", PD_), ("fg_dpotdz", PD_),
        ("vstream", PD_ * 4),
        ("cellsize", PD_), ("dgs_distance", PD_),
        ("targets", (PD_ * 6) * 4),
        ("n", C.c_int),
        ("pos", PD_), ("vel", PD_), ("mass", PD_), ("tint", PD_), ("vesc", PD_), ("ptargets", PD_),
        ("type", C.POINTER(C.c_int)),
        ("form", C.c_int), ("max_iterations", C.c_int), ("reps_per_iteration", C.c_int),
        ("fraction_per_rep", C.c_double), ("converge_rel", C.c_double),
        ("seed", C.c_uint64),
        ("permutation", C.POINTER(C.c_int)),
        ("vel_out", PD_),
    ]


class GalicJobResult(C.Structure):
    """galic_job_result_t."""
    _fields_ = [
        ("status", C.c_int), ("iterations", C.c_int), ("reps", C.c_longlong), ("orbit_steps", C.c_longlong),
        ("sall_first", C.c_double), ("sall_last", C.c_double), ("fit", C.c_double * 28),
        ("t_submit", C.c_double), ("t_admit", C.c_double), ("t_first_response", C.c_double), ("t_done", C.c_double),
    ]


class GalicSampleParams(C.Structure):
    """galic_sample_params_t."""
    _fields_ = [(n, C.c_double) for n in ("Rmax", "Halo_A", "HaloStretch", "Disk_Z0", "Disk_H", "Bulge_A",
                                          "BulgeStretch", "HaloBetaParameter", "BulgeBetaParameter")]


class GalicStream(C.Structure):
    """galic_stream_t."""
    _fields_ = [("seed", C.c_uint64), ("a", C.c_uint32), ("b", C.c_uint32), ("position", C.c_uint64)]


class GalicJeansParams(C.Structure):
    """galic_jeans_params_t."""
    _fields_ = [("StreamingVelocityParameter", D4), ("DispersionRoverZratio", D4)]


class GalicJeansTables(C.Structure):
    """galic_jeans_tables_t (pointers to FG_Nbin^2 doubles)."""
    _fields_ = [(n, C.POINTER(C.c_double)) for n in ("disp_r", "dispz", "dispphi", "vstream", "tilted_vz2",
                                                      "tilted_vR2", "tilted_vz2_prime", "tilted_vR2_prime")]


class GalicParticlesOut(C.Structure):
    """galic_particles_out_t."""
    _fields_ = [(n, C.POINTER(C.c_double)) for n in ("pos", "vel", "vel_theo", "mass", "vesc", "tint", "targets")] + \
               [(n, C.POINTER(C.c_int)) for n in ("type", "id", "permutation")] + [("low_disp", I4 * 4)]


JEANS_TABLES = ("disp_r", "dispz", "dispphi", "vstream", "tilted_vz2", "tilted_vR2", "tilted_vz2_prime",
                "tilted_vR2_prime")


def dptr(a):
    """double* of a C-contiguous float64 numpy array (None passes NULL)."""
    if a is None:
        return None
    assert a.dtype == np.float64 and a.flags["C_CONTIGUOUS"], "need C-contiguous float64"
    return a.ctypes.data_as(C.POINTER(C.c_double))


def iptr(a):
    if a is None:
        return None
    assert a.dtype == np.int32 and a.flags["C_CONTIGUOUS"], "need C-contiguous int32"
    return a.ctypes.data_as(C.POINTER(C.c_int))


def llptr(a):
    assert a.dtype == np.int64 and a.flags["C_CONTIGUOUS"]
    return a.ctypes.data_as(C.POINTER(C.c_longlong))


PD = C.POINTER(C.c_double)
PI = C.POINTER(C.c_int)
PLL = C.POINTER(C.c_longlong)
VP = C.c_void_p

# (name, restype, argtypes) for every symbol of include/galic_gpu.h
SIGNATURES = [
    ("galic_ctx_create", C.c_int, [C.POINTER(GalicParams), C.POINTER(VP)]),
    ("galic_ctx_destroy", None, [VP]),
    ("galic_last_status", C.c_int, [VP]),
    ("galic_status_string", C.c_char_p, [C.c_int]),
    ("galic_set_force_grid", C.c_int, [VP, PD, PD, PD]),
    ("galic_set_vstream", C.c_int, [VP, C.c_int, PD]),
    ("galic_set_density_geometry", C.c_int, [VP, PD, PD]),
    ("galic_set_targets", C.c_int, [VP, C.c_int, PD, PD, PD, PD, PD, PD]),
    ("galic_set_particles", C.c_int, [VP, C.c_int, PD, PD, PD, PD, PD, PI, PD]),
    ("galic_get_particles", C.c_int, [VP, PD, PI, PD]),
    ("galic_produce_orbit_response_field_mod", C.c_double,
     [VP, PD, PD, C.c_int, PD, PD, PD, PD, PD, C.c_double, C.c_double, PI, C.c_int]),
    ("galic_produce_orbit_response_field", C.c_double, [VP, PD, PD, C.c_int, PD, C.c_double, C.c_double, PI]),
    ("galic_calc_all_response_fields", C.c_int, [VP, C.c_int]),
    ("galic_calc_all_shard", C.c_int, [VP, C.c_int, C.c_int, C.c_int]),
    ("galic_accumulators", C.c_int, [VP, C.POINTER(C.c_void_p), C.POINTER(C.c_size_t)]),
    ("galic_calc_all_finish", C.c_int, [VP]),
    ("galic_optimize_rep", C.c_int, [VP, PI, C.c_int, C.c_uint64, C.c_uint32, C.c_int]),
    ("galic_optimize_reps", C.c_int, [VP, PI, C.c_int, C.c_int, C.c_uint64, C.c_uint32, C.c_int, C.c_size_t, PD]),
    ("galic_get_fit", C.c_int, [VP, PD]),
    ("galic_get_counters", C.c_int, [VP, PLL, PLL]),
    ("galic_get_response", C.c_int, [VP, C.c_int, C.c_int, PD]),
    ("galic_set_step_cap", C.c_int, [VP, C.c_longlong]),
    ("galic_last_orbit_steps", C.c_longlong, [VP]),
    ("galic_last_timing", C.c_int, [VP, PD, PD]),
    ("galic_last_max_energy_error", C.c_double, [VP]),
    ("galic_last_kernel_launches", C.c_int, [VP]),
    ("galic_orbit_responses_noalloc", C.c_int,
     [C.POINTER(GalicParams), VP, VP, VP, VP, C.c_double, C.c_int, VP, VP, VP, VP, VP, VP, VP, VP]),
    ("galic_ensemble_create", C.c_int, [C.POINTER(VP), C.c_int, C.POINTER(VP)]),
    ("galic_ensemble_destroy", None, [VP]),
    ("galic_ensemble_last_status", C.c_int, [VP]),
    ("galic_ensemble_calc_all", C.c_int, [VP]),
    ("galic_ensemble_variants", C.c_int, [PI, PI, C.c_int]),
    ("galic_ensemble_set_variant", C.c_int, [VP, C.c_int]),
    ("galic_ensemble_autotune", C.c_int, [VP, C.c_double, PI, PD]),
    ("galic_ensemble_last_timing", C.c_int, [VP, PD, PD, PLL, PI]),
    ("galic_server_create", C.c_int, [C.c_size_t, C.c_int, C.POINTER(VP)]),
    ("galic_server_submit", C.c_int, [VP, C.POINTER(GalicJob), PI]),
    ("galic_server_wait", C.c_int, [VP, C.c_int, C.c_double, C.POINTER(GalicJobResult)]),
    ("galic_server_stats", C.c_int, [VP, C.POINTER(C.c_size_t), PI, PI, PI]),
    ("galic_server_destroy", None, [VP]),
    ("galic_job_device_bytes", C.c_size_t, [C.POINTER(GalicJob)]),
    ("galic_force_grid_fill", C.c_int,
     [C.POINTER(GalicFillParams), C.c_int, PD, PD, PD, PD, PD, C.POINTER(GalicFillStats)]),
    ("galic_peano_hilbert_key", C.c_uint64, [C.c_int, C.c_int, C.c_int, C.c_int]),
    ("galic_set_dispersion", C.c_int, [VP, C.c_int, PD, PD, PD, PD, PD]),
    ("galic_sample_density_targets", C.c_int,
     [VP, C.POINTER(GalicSampleParams), C.c_longlong, C.POINTER(GalicStream), C.c_int]),
    ("galic_sample_energy_targets", C.c_int, [VP, C.POINTER(GalicSampleParams), C.c_longlong, C.POINTER(GalicStream)]),
    ("galic_get_targets", C.c_int, [VP, C.c_int, PD, PD, PD, PD, PD, PD]),
    ("galic_calculate_dispfield", C.c_int,
     [VP, C.POINTER(GalicSampleParams), C.POINTER(GalicJeansParams), C.POINTER(GalicJeansTables)]),
    ("galic_initialize_particles", C.c_int,
     [VP, C.POINTER(GalicSampleParams), C.c_double, C.POINTER(GalicStream), C.POINTER(GalicParticlesOut)]),
    ("galic_get_params", C.c_int, [VP, C.POINTER(GalicParams)]),
    ("galic_write_snapshot", C.c_int, [C.c_char_p, C.c_int, C.c_int, PD, PD, PD, PD, PI, PI, PD]),
    ("galic_write_forcefield", C.c_int, [C.c_char_p, C.POINTER(GalicParams), PD, PD, PD]),
    ("galic_write_density_field", C.c_int, [C.c_char_p, C.POINTER(GalicParams), C.c_int, PD, PD, PD, PD]),
    ("galic_output_density_field", C.c_int, [VP, C.c_char_p, C.c_int]),
    ("galic_sample_positions", C.c_int,
     [C.POINTER(GalicSampleParams), C.c_int, C.c_longlong, C.POINTER(GalicStream), PD]),
    ("galic_grid_geometry", C.c_int, [C.c_double, C.c_double, C.c_double, C.c_int, C.c_int, C.c_int, PD]),
    ("galic_density_geometry", C.c_int, [C.c_int, C.c_double, C.c_double, PD, PD, PD]),
    ("galic_smooth_stack", None, [PD, C.c_int]),
]

_lib = None


def load_library(path=LIB_PATH):
    """Open libgalic_cuda.so and declare its entry points (no fallback)."""
    global _lib
    if _lib is not None and path == LIB_PATH:
        return _lib
    if not os.path.exists(path):
        raise RuntimeError(
            f"{path} is missing: build it with `python -c 'import __graft_entry__ as g; g.build()'` "
            "(there is no CPU fallback for the GALIC orbit-response path)")
    lib = C.CDLL(path)
    for name, res, args in SIGNATURES:
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    if path == LIB_PATH:
        _lib = lib
    return lib
