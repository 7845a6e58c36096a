"""Particle initialisation: initialize_particles (set_particles.c:15-307).

CPU: the restatement (oracle/oracle_particles.c) with glibc's functions
gives GALIC's own initialize_particles bit for bit: positions, velocities,
VelTheo, masses, escape speeds, integration times, dispersion targets, IDs,
the permutation and the stream position after the call.

GPU: galic_initialize_particles against the restatement with gmath.h's
functions: bit for bit."""
import numpy as np
import pytest

import oracle_lib
from galic_b200 import _ffi, synth

needs_ref = pytest.mark.skipif(not oracle_lib.reference_available(), reason="oracle/_ref not built")


def particle_model(tovs=(1, 3, 2), n=(400, 200, 100), fg_nbin=48, seed=5):
    comps = [synth.Component("halo", 93.5, 30.0, n[0], beta=0.2, tovs=tovs[0]),
             synth.Component("disk", 5.0, 3.5, n[1], z0=0.7, tovs=tovs[1]),
             synth.Component("bulge", 1.5, 1.0, n[2], tovs=tovs[2])]
    m = synth.build_model(comps, seed=seed, level=5, fg_nbin=fg_nbin)
    return m


def setup_inputs(m, halo_beta=0.2, bulge_beta=0.0, low=None, maxvel=None):
    """Sampler shapes, Jeans tables from the restatement (glibc), TorbitFac."""
    from galic_b200 import sampling
    import test_jeans as TJ
    sp, jp = TJ.jeans_params(m, halo_beta, bulge_beta)
    if low is not None:
        m.params.LowerDispLimit = low
    if maxvel is not None:
        m.params.MaxVelInUnitsVesc = maxvel
    st, J = oracle_lib.oracle_dispfield(m, sp, jp, use_libm=True)
    assert st == 0
    # get_disp_rtp reads FG_Disp_r, FG_DispZ, FG_DispPhi, FG_tilted_vR2_prime,
    # FG_tilted_vz2_prime; get_vstream reads FG_Vstream
    tables = {t: (J[t, 0], J[t, 1], J[t, 2], J[t, 7], J[t, 6], J[t, 3]) for t in (1, 2, 3)}
    return sp, jp, tables, 5.0


@needs_ref
@pytest.mark.parametrize("tovs", [(1, 3, 2), (0, 2, 1), (2, 3, 0)])
def test_restatement_matches_reference(tovs):
    m = particle_model(tovs=tovs)
    sp, _, tables, tf = setup_inputs(m)
    stream = (42, 0, 0, 7)
    ref, rpos = oracle_lib.run_reference(oracle_lib.reference_particles, m.params, (m.pot, m.dpotdr, m.dpotdz), sp,
                                         tf, tables, stream)
    st, out, counts, opos = oracle_lib.oracle_particles(m, sp, tf, tables, stream, use_libm=True)
    assert st == 0 and opos == rpos
    for k, _, _ in oracle_lib.PARTICLE_FIELDS:
        assert np.array_equal(out[k], ref[k]), k
    st, g, gcounts, gpos = oracle_lib.oracle_particles(m, sp, tf, tables, stream, use_libm=False)
    assert gpos == rpos and np.array_equal(g["perm"], out["perm"]) and np.array_equal(gcounts, counts)
    for k in ("pos", "vel", "vel_theo", "vesc", "tint", "targets"):
        assert np.max(np.abs(g[k] - out[k])) <= 1e-9 * np.max(np.abs(out[k])), k


def test_restatement_stops_on_low_dispersion():
    """More than 5 % of a type at LowerDispLimit: the reference's endrun().
    The limit is the median radial dispersion target of the halo, so about
    half of the halo is raised to it (a limit far above the dispersions would
    make the reference's escape-speed loop run for ever)."""
    m = particle_model()
    sp, _, tables, tf = setup_inputs(m)
    st, out, counts, _ = oracle_lib.oracle_particles(m, sp, tf, tables, (1, 0, 0, 0), use_libm=False)
    assert st == 0
    m.params.LowerDispLimit = float(np.median(out["targets"][out["type"] == 1, 0]))
    st, _, counts, _ = oracle_lib.oracle_particles(m, sp, tf, tables, (1, 0, 0, 0), use_libm=False)
    assert st == 6 and counts[1, 0] > 0.05 * m.params.NType[1]


def test_result_arrays_shape_and_type():
    """The wrapper's result arrays: page-locked where torch has a CUDA device,
    plain memory otherwise; shapes and types as initialize_particles fills them."""
    from galic_b200 import particles
    for k, w, dt in particles.FIELDS:
        a = particles._host_array((5, w) if w > 1 else (5,), dt)
        assert a.shape == ((5, w) if w > 1 else (5,)) and a.dtype == dt and a.flags["C_CONTIGUOUS"], k


def _gpu_particles(m, sp, tf, tables, stream, fit=True):
    from galic_b200 import particles, sampling
    from galic_b200.context import Context
    with Context(m.params) as ctx:
        ctx.load_model(m)
        for t, tab in tables.items():
            sampling.set_dispersion(ctx, t, *tab[:5])
            ctx.lib.galic_set_vstream(ctx.h, t, _ffi.dptr(np.ascontiguousarray(tab[5], dtype=np.float64).ravel()))
        s = sampling.Stream(*stream)
        out, counts = particles.initialize_particles(ctx, sp, tf, s)
        launches = ctx.lib.galic_last_kernel_launches(ctx.h)
        f = None
        if fit:
            ctx.calc_all_response_fields()  # the particles are the context's
            f = ctx.fit()
    return out, counts, s.position, launches, f


@pytest.mark.gpu
@pytest.mark.parametrize("tovs,n", [((1, 3, 2), (400, 200, 100)), ((0, 2, 1), (3000, 1000, 500)),
                                    ((2, 3, 0), (3000, 1000, 500)), ((1, 3, 2), (60000, 20000, 8000))])
def test_gpu_bit_identical(tovs, n):
    m = particle_model(tovs=tovs, n=n)
    sp, _, tables, tf = setup_inputs(m)
    stream = (42, 0, 0, 7)
    got, counts, gpos, launches, fit = _gpu_particles(m, sp, tf, tables, stream)
    st, ref, rcounts, rpos = oracle_lib.oracle_particles(m, sp, tf, tables, stream, use_libm=False)
    assert st == 0 and launches > 0
    assert gpos == rpos and np.array_equal(counts, rcounts)
    for k in ("pos", "vel", "vel_theo", "mass", "vesc", "tint", "targets", "type", "id"):
        assert np.array_equal(got[k], ref[k]), k
    assert np.array_equal(got["permutation"], ref["perm"])
    assert np.all(np.isfinite(fit))


@pytest.mark.gpu
def test_gpu_bit_identical_workload_size():
    """The halo + disk workload at full size (1.0e6 + 2.0e5 particles, ~9e7
    draws, 256^2 force grid): velocity loops of up to ~3e5 draw pairs are
    deferred and searched by the whole GPU, and the long resynchronisation
    walks go through windows of lengths evaluated ahead; every particle, the
    permutation and the stream position are still the restatement's."""
    m = synth.config_halo_disk()
    sp, _, tables, tf = setup_inputs(m, halo_beta=0.0)
    tables = {t: tab for t, tab in tables.items() if m.params.NType[t] > 0}
    stream = (42, 0, 0, 0)
    got, counts, gpos, _, _ = _gpu_particles(m, sp, tf, tables, stream, fit=False)
    st, ref, rcounts, rpos = oracle_lib.oracle_particles(m, sp, tf, tables, stream, use_libm=False)
    assert st == 0 and gpos == rpos and np.array_equal(counts, rcounts)
    for k in ("pos", "vel", "vel_theo", "mass", "vesc", "tint", "targets", "type", "id"):
        assert np.array_equal(got[k], ref[k]), k
    assert np.array_equal(got["permutation"], ref["perm"])


@pytest.mark.gpu
def test_gpu_installed_particles_match_upload():
    """The particles the initialisation leaves in the context (installed on
    the device, orbit order sorted there) give the same response fields,
    fit and per-particle results as the same arrays uploaded through
    galic_set_particles."""
    from galic_b200 import particles, sampling
    from galic_b200.context import Context
    m = particle_model(n=(3000, 1000, 500))
    sp, _, tables, tf = setup_inputs(m)
    res = []
    for upload in (False, True):
        with Context(m.params) as ctx:
            ctx.load_model(m)
            for t, tab in tables.items():
                sampling.set_dispersion(ctx, t, *tab[:5])
                ctx.lib.galic_set_vstream(ctx.h, t, _ffi.dptr(np.ascontiguousarray(tab[5], dtype=np.float64).ravel()))
            out, _ = particles.initialize_particles(ctx, sp, tf, sampling.Stream(42, 0, 0, 7))
            if upload:
                ctx.set_particles(out["pos"], out["vel"], out["mass"], out["tint"], out["vesc"], out["type"],
                                  out["targets"])
            ctx.calc_all_response_fields()
            grids = [ctx.response(t, w) for t in (1, 2, 3) for w in range(2)]
            res.append((grids, ctx.fit(), ctx.particles()))
    (g0, f0, p0), (g1, f1, p1) = res
    for a, b in zip(g0, g1):
        assert np.array_equal(a, b)
    assert np.array_equal(f0, f1)
    for a, b in zip(p0, p1):
        assert np.array_equal(a, b)


@pytest.mark.gpu
def test_gpu_refusals():
    """More than 5 % at LowerDispLimit: GALIC_ERR_UNSUPPORTED (the reference's
    endrun()), the stream not advanced; missing Jeans tables: GALIC_ERR_STATE."""
    from galic_b200 import particles, sampling
    from galic_b200.context import Context, GalicError
    m = particle_model()
    sp, _, tables, tf = setup_inputs(m)
    st, out, _, _ = oracle_lib.oracle_particles(m, sp, tf, tables, (1, 0, 0, 0), use_libm=False)
    m.params.LowerDispLimit = float(np.median(out["targets"][out["type"] == 1, 0]))
    with Context(m.params) as ctx:
        ctx.load_model(m)
        s = sampling.Stream(1)
        with pytest.raises(GalicError) as e:
            particles.initialize_particles(ctx, sp, tf, s)
        assert e.value.status == 9
        for t, tab in tables.items():
            sampling.set_dispersion(ctx, t, *tab[:5])
            ctx.lib.galic_set_vstream(ctx.h, t, _ffi.dptr(np.ascontiguousarray(tab[5], dtype=np.float64).ravel()))
        with pytest.raises(GalicError) as e:
            particles.initialize_particles(ctx, sp, tf, s)
        assert e.value.status == 6 and s.position == 0
