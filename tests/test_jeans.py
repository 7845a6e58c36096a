"""Jeans solvers: calculate_dispfield (disp_fields.c:502-1049).

CPU: the restatement (oracle/oracle_jeans.c) with glibc's functions gives
GALIC's own calculate_dispfield bit for bit (all eight tables of every type,
velocity structures 1-3, both forms of beta); with gmath.h's functions it
stays within 1e-9 of each table's peak.

GPU: galic_calculate_dispfield against the restatement with gmath.h's
functions: bit for bit."""
import ctypes as C

import numpy as np
import pytest

import oracle_lib
from galic_b200 import _ffi, synth

needs_ref = pytest.mark.skipif(not oracle_lib.reference_available(), reason="oracle/_ref not built")


def jeans_model(fg_nbin=48, tovs=(1, 3, 2), seed=5):
    comps = [synth.Component("halo", 93.5, 30.0, 400, beta=0.2, tovs=tovs[0]),
             synth.Component("disk", 5.0, 3.5, 200, z0=0.7, tovs=tovs[1]),
             synth.Component("bulge", 1.5, 1.0, 100, tovs=tovs[2])]
    return synth.build_model(comps, seed=seed, level=5, fg_nbin=fg_nbin)


def jeans_params(m, halo_beta=0.2, bulge_beta=0.0, k=(0.0, 0.6, 0.9, 0.3), f=(0.0, 1.4, 2.0, 1.2)):
    from galic_b200 import sampling
    sp = sampling.sample_params(Rmax=m.meta["rmax"], Halo_A=30.0, HaloStretch=m.params.HaloStretch, Disk_Z0=0.7,
                                Disk_H=3.5, Bulge_A=1.0, BulgeStretch=m.params.BulgeStretch,
                                HaloBetaParameter=halo_beta, BulgeBetaParameter=bulge_beta)
    jp = _ffi.GalicJeansParams()
    for t in range(4):
        jp.StreamingVelocityParameter[t] = k[t]
        jp.DispersionRoverZratio[t] = f[t]
    return sp, jp


def peak_rel(a, b):
    den = np.max(np.abs(b))
    return float(np.max(np.abs(a - b)) / (den if den > 0 else 1.0))


@needs_ref
@pytest.mark.parametrize("tovs,betas", [((1, 3, 2), (0.2, 0.0)), ((3, 2, 1), (1.0, 1.5)), ((0, 3, 3), (0.0, 0.0))])
def test_restatement_matches_reference(tovs, betas):
    m = jeans_model(tovs=tovs)
    sp, jp = jeans_params(m, *betas)
    ref = oracle_lib.run_reference(oracle_lib.reference_dispfield, m.params, (m.pot, m.dpotdr, m.dpotdz), sp, jp)
    st, out = oracle_lib.oracle_dispfield(m, sp, jp, use_libm=True)
    assert st == 0
    for t in (1, 2, 3):
        for w, name in enumerate(_ffi.JEANS_TABLES):
            a, b = out[t, w], ref[t, w]
            if name == "disp_r":
                a, b = a[0], b[0]  # only the first FG_Nbin entries are written
            assert np.array_equal(a, b), (t, name)
    assert np.any(out[1, 1]) and all(np.any(out[t, 4]) for t in (1, 2, 3) if tovs[t - 1] == 3)
    st, g = oracle_lib.oracle_dispfield(m, sp, jp, use_libm=False)
    for t in (1, 2, 3):
        for w in range(8):
            assert peak_rel(g[t, w], out[t, w]) < 1e-9, (t, w)


def test_restatement_refuses_zero_ratio():
    """Velocity structure 3 with DispersionRoverZratio = 0: the reference terminates."""
    m = jeans_model(tovs=(1, 3, 2))
    sp, jp = jeans_params(m, f=(0.0, 1.4, 0.0, 1.2))
    st, _ = oracle_lib.oracle_dispfield(m, sp, jp, use_libm=False)
    assert st == 6


def _gpu_dispfield(m, sp, jp):
    from galic_b200 import jeans
    from galic_b200.context import Context
    with Context(m.params) as ctx:
        ctx.load_model(m)
        res = jeans.calculate_dispfield(ctx, sp, jp)
        launches = ctx.lib.galic_last_kernel_launches(ctx.h)
    return res, launches


@pytest.mark.gpu
@pytest.mark.parametrize("tovs,betas", [((1, 3, 2), (0.2, 0.0)), ((3, 2, 1), (1.0, 1.5)), ((0, 3, 3), (0.0, 0.0))])
def test_gpu_bit_identical(tovs, betas):
    m = jeans_model(tovs=tovs)
    sp, jp = jeans_params(m, *betas)
    got, launches = _gpu_dispfield(m, sp, jp)
    st, ref = oracle_lib.oracle_dispfield(m, sp, jp, use_libm=False)
    assert st == 0 and launches > 0
    for t in (1, 2, 3):
        for w, name in enumerate(_ffi.JEANS_TABLES):
            a, b = got[t][name], ref[t, w]
            if name == "disp_r":
                a, b = a[0], b[0]
            assert np.array_equal(a, b), (t, name, peak_rel(a, b))


@pytest.mark.gpu
def test_gpu_workload_grid_bit_identical():
    """The 256^2 force grid of the halo + disk workload (disk: tilted case)."""
    comps = [synth.Component("halo", 95.0, 30.0, 400, tovs=0), synth.Component("disk", 5.0, 3.5, 200, z0=0.7, tovs=3)]
    m = synth.build_model(comps, seed=2, level=6, outer_frac=(70.0 / 100.0) ** 2, inner_frac=1e-7)
    sp, jp = jeans_params(m, 0.0, 0.0)
    got, _ = _gpu_dispfield(m, sp, jp)
    st, ref = oracle_lib.oracle_dispfield(m, sp, jp, use_libm=False)
    for t in (1, 2):
        for w, name in enumerate(_ffi.JEANS_TABLES):
            assert np.array_equal(got[t][name], ref[t, w]), (t, name)


@pytest.mark.gpu
def test_gpu_tables_feed_the_context():
    """The solved tables become the context's FG_Vstream and Jeans tables:
    the energy-target sampler runs on them without galic_set_dispersion."""
    from galic_b200 import jeans, sampling
    from galic_b200.context import Context, GalicError
    m = jeans_model(tovs=(1, 3, 2))
    sp, jp = jeans_params(m)
    with Context(m.params) as ctx:
        ctx.load_model(m)
        with pytest.raises(GalicError) as e:  # no Jeans tables yet
            sampling.sample_energy_targets(ctx, sp, 100, sampling.Stream(1))
        assert e.value.status == 9
        res = jeans.calculate_dispfield(ctx, sp, jp)
        sampling.sample_energy_targets(ctx, sp, 20000, sampling.Stream(1))
        tg = sampling.get_targets(ctx, 2)
    assert np.any(res[2]["vstream"]) and np.all(np.isfinite(tg[2]))
    bad = jeans_params(m, f=(0.0, 1.4, 0.0, 1.2))[1]
    with Context(m.params) as ctx:
        with pytest.raises(GalicError) as e:  # no force grid
            jeans.calculate_dispfield(ctx, sp, jp)
        assert e.value.status == 9
        ctx.load_model(m)
        with pytest.raises(GalicError) as e:  # the reference's terminate()
            jeans.calculate_dispfield(ctx, sp, bad)
        assert e.value.status == 6
