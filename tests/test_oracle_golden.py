"""The CPU restatement (oracle/galic_oracle.c) against fixtures produced by
GALIC's own C (tests/golden/make_golden.py).

With glibc's transcendental functions the restatement must reproduce the
reference bit for bit: orbits (orbit_response.c:33-491), the batched response
and fit (main.c:151-362) and an optimisation repetition (main.c:365-527,
808-874).  With the project's gmath.h functions (what the CUDA kernels use)
every value must stay within the stated tolerances."""
import os

import numpy as np
import pytest

import golden_lib
import oracle_lib
from oracle_lib import Oracle

# per-bin tolerance of the gmath form against the reference: relative to the
# largest bin of the same grid (ulp-level differences in log/atan2/sin/cos
# perturb the trajectory; bins of a regular orbit move by < 1e-10 of the peak)
BIN_TOL = 1e-9
# merit values: relative, with an absolute floor for types whose misfit is a
# pure rounding residual (e.g. a component whose whole stack is one leaf)
FIT_TOL = 1e-9
FIT_ATOL = 1e-14


@pytest.fixture(params=golden_lib.GOLDEN, ids=lambda p: os.path.basename(p)[:-4])
def golden(request):
    return golden_lib.load(request.param)


def test_fixtures_exist():
    assert len(golden_lib.GOLDEN) >= 3


def test_orbits_bit_exact_with_libm(golden):
    ins, outs = golden
    m = golden_lib.model(ins)
    o = Oracle(m.params, use_libm=True)
    o.load_model(m)
    for key in golden_lib.orbit_keys(outs):
        i = int(outs[f"{key}_idx"])
        tall, norbit, *g, info = o.orbit_mod(m.pos[i], m.vel[i], m.mass[i], m.tint[i], m.ptype[i])
        assert tall == outs[f"{key}_tall"]
        assert norbit == outs[f"{key}_norbit"]
        assert np.array_equal(np.stack(g), outs[f"{key}_grids"]), key
    for j in range(3):
        i = int(outs[f"orbit{j}_idx"])
        tall, norbit, mm, info = o.orbit(m.pos[i], m.vel[i], m.mass[i], m.tint[i])
        assert tall == outs[f"morbit{j}_tall"]
        assert norbit == outs[f"morbit{j}_norbit"]
        assert np.array_equal(mm, outs[f"morbit{j}_grid"])


def test_calc_all_and_rep_bit_exact_with_libm(golden):
    ins, outs = golden
    m = golden_lib.model(ins)
    o = Oracle(m.params, use_libm=True)
    o.load_model(m)
    assert o.calc_all() == 0
    present = [t for t in (1, 2, 3) if m.params.NType[t]]
    for t in present:
        got = np.stack([o.response(t, w) for w in range(10)])
        assert np.array_equal(got, outs[f"calc_resp{t}"]), t
    assert np.array_equal(o.fit()[present], outs["calc_fit"][present])
    vel, orbits, vdisp = o.particles()
    assert np.array_equal(orbits, outs["calc_orbits"])
    assert np.array_equal(vdisp, outs["calc_vdisp"])
    assert o.optimize_rep(outs["rep_idx"], 987654321, 7) == 0
    assert np.array_equal(o.fit()[present], outs["rep_fit"][present])
    tr, ch = o.counters()
    assert np.array_equal(tr, outs["rep_tries"]) and np.array_equal(ch, outs["rep_changes"])
    vel, orbits, vdisp = o.particles()
    assert np.array_equal(vel, outs["rep_vel"])
    assert np.array_equal(orbits, outs["rep_orbits"])
    assert np.array_equal(vdisp, outs["rep_vdisp"])
    for t in present:
        got = np.stack([o.response(t, w) for w in range(10)])
        assert np.array_equal(got, outs[f"rep_resp{t}"]), t


def rel_to_peak(a, b):
    den = np.max(np.abs(b), axis=-1, keepdims=True)
    den = np.where(den == 0, 1, den)
    return float(np.max(np.abs(a - b) / den))


def test_gmath_form_within_tolerance(golden):
    ins, outs = golden
    m = golden_lib.model(ins)
    o = Oracle(m.params, use_libm=False)
    o.load_model(m)
    for key in golden_lib.orbit_keys(outs):
        i = int(outs[f"{key}_idx"])
        tall, norbit, *g, info = o.orbit_mod(m.pos[i], m.vel[i], m.mass[i], m.tint[i], m.ptype[i])
        assert abs(tall - outs[f"{key}_tall"]) <= 1e-12 * tall
        assert rel_to_peak(np.stack(g), outs[f"{key}_grids"]) < BIN_TOL, key
    assert o.calc_all() == 0
    present = [t for t in (1, 2, 3) if m.params.NType[t]]
    for t in present:
        got = np.stack([o.response(t, w) for w in range(10)])
        assert rel_to_peak(got, outs[f"calc_resp{t}"]) < BIN_TOL
    f, g = o.fit()[present, :5], outs["calc_fit"][present, :5]
    assert np.all(np.abs(f - g) <= FIT_TOL * np.abs(g) + FIT_ATOL)


@pytest.mark.skipif(not oracle_lib.reference_gmath_available(), reason="GALIC's own C (oracle/_ref) is not built")
def test_reference_with_project_math_equals_restatement(golden):
    """GALIC's unmodified C linked with the project's elementary functions
    (oracle/shim/gmath_libm.c) and the restatement with the same functions
    (what the CUDA kernels evaluate) agree bit for bit: per orbit, the whole
    calc_all_response_fields and its fit."""
    import sys

    sys.path.insert(0, os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden"))
    from make_golden import model_arrays

    ins, outs = golden
    m = golden_lib.model(ins)
    idx = list(range(m.n))
    ref, ref_fit, per_orbit = oracle_lib.run_reference(oracle_lib.reference_calc_all, model_arrays(m), True, idx)
    o = Oracle(m.params, use_libm=False)
    o.load_model(m)
    for i, r in zip(idx, per_orbit):
        b = o.orbit_mod(m.pos[i], m.vel[i], m.mass[i], m.tint[i], m.ptype[i])
        assert r[0] == b[0] and r[1] == b[1], i
        for k in range(2, 7):
            assert np.array_equal(r[k], b[k]), (i, k)
    assert o.calc_all() == 0
    for t, g in ref.items():
        assert np.array_equal(np.stack([o.response(t, w) for w in range(10)]), g), t
    assert np.array_equal(o.fit(), ref_fit, equal_nan=True)  # absent types: NaN on both sides
