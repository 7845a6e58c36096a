"""libgalic_cuda.so loads on a CPU-only host, exports every symbol declared in
include/galic_gpu.h, and its host-side helpers match the oracle and GALIC's
own grid construction (grid.c:329-487, 830-850, 1247-1265)."""
import ctypes as C
import os
import re
import tempfile

import numpy as np
import pytest

from galic_b200 import _ffi, synth
import oracle_lib
from conftest import ROOT, cuda_available


def header_symbols():
    text = open(os.path.join(ROOT, "include", "galic_gpu.h")).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(galic_[a-z0-9_]+)\s*\(", text)))


def test_library_exports_every_declared_symbol():
    lib = C.CDLL(_ffi.LIB_PATH)
    syms = header_symbols()
    assert len(syms) >= 20
    for s in syms:
        assert hasattr(lib, s), s
    declared = {n for n, _, _ in _ffi.SIGNATURES}
    assert set(syms) == declared


def test_status_strings():
    lib = _ffi.load_library()
    assert lib.galic_status_string(0) == b"ok"
    assert lib.galic_status_string(2).startswith(b"an orbit exceeded")
    assert lib.galic_status_string(99) == b"unknown status"


def test_params_validation_before_device():
    lib = _ffi.load_library()
    p, _, _ = synth.make_params([synth.Component("halo", 100.0, 30.0, 100)], level=5, fg_nbin=64)
    h = C.c_void_p()
    bad = p.copy()
    bad.EG_MaxLevel = 4  # eval_fit_mod needs DG_MaxLevel == EG_MaxLevel (main.c:1056)
    assert lib.galic_ctx_create(C.byref(bad), C.byref(h)) == 6
    bad = p.copy()
    bad.TypeOfVelocityStructure[1] = 7
    assert lib.galic_ctx_create(C.byref(bad), C.byref(h)) == 1
    if not cuda_available():
        assert lib.galic_ctx_create(C.byref(p), C.byref(h)) == 4  # GALIC_ERR_NO_DEVICE


def test_noalloc_validation_before_device():
    """The allocation-free entry point rejects bad grid parameters before it
    touches a device, as galic_ctx_create does (the pointers are never read)."""
    lib = _ffi.load_library()
    p, _, _ = synth.make_params([synth.Component("halo", 100.0, 30.0, 100)], level=6, fg_nbin=64)
    dummy = (C.c_double * 8)()
    d = C.addressof(dummy)

    def call(prm):
        return lib.galic_orbit_responses_noalloc(C.byref(prm), d, d, d, d, 1.0, 0, None, None, None, None, None, d,
                                                 None, None)

    for field, value in (("FG_Rmin", 0.0), ("DG_Rmin", -1.0), ("EG_Rmin", float("nan")), ("FG_Fac", 1.0),
                         ("DG_Fac", 0.5), ("EG_Fac", 1.0)):
        bad = p.copy()
        setattr(bad, field, value)
        assert call(bad) == 1, field  # GALIC_ERR_INVALID_ARGUMENT
    bad = p.copy()
    bad.EG_MaxLevel = 5
    assert call(bad) == 1
    big = p.copy()
    big.DG_MaxLevel = big.EG_MaxLevel = 8
    assert call(big) == 5  # GALIC_ERR_BUDGET: beyond the fixed scratch array


@pytest.mark.parametrize("outer,inner,fg,L", [(0.980296, 9.80296e-5, 256, 6), (0.49, 1e-7, 256, 7),
                                              (0.999, 1e-7, 256, 7), (0.9, 1e-4, 64, 5)])
def test_grid_geometry_matches_oracle(outer, inner, fg, L):
    lib = _ffi.load_library()
    ol = oracle_lib.oracle_lib()
    a = np.zeros(8)
    b = np.zeros(8)
    assert lib.galic_grid_geometry(30.0, outer, inner, fg, L, L, _ffi.dptr(a)) == 0
    assert ol.orc_grid_geometry(30.0, outer, inner, fg, L, L, _ffi.dptr(b)) == 0
    assert np.array_equal(a, b)
    ns = ((1 << (2 + 2 * L)) - 1) // 3
    g = [np.zeros(ns), np.zeros(1 << 2 * L), np.zeros(1 << 2 * L)]
    h = [np.zeros(ns), np.zeros(1 << 2 * L), np.zeros(1 << 2 * L)]
    assert lib.galic_density_geometry(L, a[3], a[2], *[_ffi.dptr(x) for x in g]) == 0
    assert ol.orc_density_geometry(L, b[3], b[2], *[_ffi.dptr(x) for x in h]) == 0
    for x, y in zip(g, h):
        assert np.allclose(x, y, rtol=1e-14, atol=0)


def test_spurious_spacing_root_rejected():
    """grid.c:429-443 started at 1.02 converges to a root below 1 for 256 bins
    over a factor 233 (Rmax = 70 kpc, Rin = 0.3 kpc); the library refuses it."""
    lib = _ffi.load_library()
    a = np.zeros(8)
    assert lib.galic_grid_geometry(30.0, 0.49, 9.80296e-5, 256, 7, 7, _ffi.dptr(a)) == 1


def _ref_geometry(params, outer, inner):
    r = oracle_lib.Reference(params)
    L = params.DG_MaxLevel
    out = np.zeros(8)
    d = [np.zeros(((1 << (2 + 2 * L)) - 1) // 3), np.zeros(1 << 2 * L), np.zeros(1 << 2 * L)]
    with tempfile.TemporaryDirectory() as tmp:
        st = r.L.ref_geometry(tmp.encode(), outer, inner, _ffi.dptr(out), *[_ffi.dptr(x) for x in d])
    assert st == 0
    return out, d


@pytest.mark.skipif(not oracle_lib.reference_available(), reason="GALIC's C (oracle/_ref) not built here")
def test_grid_geometry_matches_reference():
    outer, inner = 0.980296, 9.80296e-5
    p, _, _ = synth.make_params([synth.Component("halo", 100.0, 30.0, 100)], level=6, fg_nbin=256,
                                outer_frac=outer, inner_frac=inner)
    p.SampleForceNhalo = 0
    out, (dist, cs, cv) = oracle_lib.run_reference(_ref_geometry, p, outer, inner)
    lib = _ffi.load_library()
    a = np.zeros(8)
    lib.galic_grid_geometry(p.Halo_A, outer, inner, 256, 6, 6, _ffi.dptr(a))
    assert np.array_equal(out, a)
    g = [np.zeros(len(dist)), np.zeros(len(cs)), np.zeros(len(cv))]
    lib.galic_density_geometry(6, a[3], a[2], *[_ffi.dptr(x) for x in g])
    assert np.allclose(g[0], dist, rtol=1e-14, atol=0)
    assert np.array_equal(g[1], cs)
    assert np.allclose(g[2], cv, rtol=1e-14, atol=0)


def test_smooth_stack_matches_oracle():
    lib = _ffi.load_library()
    ol = oracle_lib.oracle_lib()
    rng = np.random.default_rng(5)
    for L in (1, 3, 7):
        ns = ((1 << (2 + 2 * L)) - 1) // 3
        a = rng.random(ns)
        b = a.copy()
        lib.galic_smooth_stack(_ffi.dptr(a), L)
        ol.orc_smooth_stack(_ffi.dptr(b), L)
        assert np.array_equal(a, b)
        assert a[0] == pytest.approx(a[ns - (1 << 2 * L):].sum(), rel=1e-12)
