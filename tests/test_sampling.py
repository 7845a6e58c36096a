"""Set-up sampling: densitygrid_sample_targetresponse (grid.c:536-617),
calc_energy_grid_mass_maps (grid.c:941-1076) and the coordinate samplers
(halo.c:17-40, disk.c:17-50, bulge.c:15-37).

CPU: the restatement (oracle/oracle_sampling.c) with glibc's functions gives
GALIC's own functions' results bit for bit (positions, target stacks, stream
position after the call), and with gmath.h's functions the same stream
consumption and values within a few ulp.

GPU: galic_sample_* against the restatement with gmath.h's functions:
positions bit-identical, target stacks within 1e-12 of each grid's peak
(exact fixed-point sums against draw-order double sums), identical stream
positions, across window boundaries and the bulge's variable-length draws."""
import numpy as np
import pytest

import oracle_lib
from galic_b200 import synth
from galic_b200.context import Context, GalicError

needs_ref = pytest.mark.skipif(not oracle_lib.reference_available(), reason="oracle/_ref not built")


def composite(level=6, halo_tovs=1, disk_tovs=3, bulge_tovs=0):
    """Halo (a = 30), disk (h = 3.5, z0 = 0.7) and bulge (a = 1) of the composite configuration."""
    m = synth.config_composite(n_halo=2000, n_disk=1000, n_bulge=500, level=level, seed=4)
    p = m.params
    p.TypeOfVelocityStructure[1] = halo_tovs
    p.TypeOfVelocityStructure[2] = disk_tovs
    p.TypeOfVelocityStructure[3] = bulge_tovs
    return m


def shape(m, **kw):
    from galic_b200 import sampling
    d = dict(Rmax=m.meta["rmax"], Halo_A=30.0, HaloStretch=1.0, Disk_Z0=0.7, Disk_H=3.5, Bulge_A=1.0,
             BulgeStretch=1.0, HaloBetaParameter=0.2, BulgeBetaParameter=0.0)
    d.update(kw)
    return sampling.sample_params(**d)


def disp_tables(m, seed):
    """Smooth positive Jeans tables of every type (FG_Disp_r, FG_DispZ,
    FG_DispPhi, FG_tilted_vR2_prime, FG_tilted_vz2_prime) and FG_Vstream."""
    N = m.params.FG_Nbin
    rng = np.random.default_rng(seed)
    iR, iz = np.meshgrid(np.arange(N), np.arange(N))
    out = {}
    for t in (1, 2, 3):
        tabs = []
        for k in range(5):
            a, b, c = rng.uniform(1e3, 4e4), rng.uniform(10, 80), rng.uniform(10, 80)
            tabs.append(np.ascontiguousarray(a * np.exp(-iR / b - iz / c) + rng.uniform(10, 100)))
        out[t] = tabs + [np.ascontiguousarray(m.vstream[t], dtype=np.float64).reshape(N, N)]
    return out


def peak_rel(a, b):
    den = np.max(np.abs(b))
    return float(np.max(np.abs(a - b)) / (den if den > 0 else 1.0))


def _restatement_targets(m, sp, ntarget, stream, kind, use_libm, tables=None, renorm=False):
    """Chains the restatement over types 1..3 with MType > 0, as the reference's loop does."""
    out, pos = {}, stream[3]
    for t in (1, 2, 3):
        if not m.params.MType[t] > 0:
            continue
        st = (stream[0], stream[1], stream[2], pos)
        if kind == "density":
            out[t], pos = oracle_lib.oracle_density(m.params, sp, t, ntarget, st, use_libm, renorm)
        else:
            out[t], pos = oracle_lib.oracle_energy(m.params, sp, t, ntarget, st, use_libm, tables[t])
    return out, pos


# ------------------------------------------------------------------ CPU


@needs_ref
@pytest.mark.parametrize("ptype", [1, 2, 3])
def test_restatement_positions_match_reference(ptype):
    m = composite()
    sp = shape(m, Rmax=25.0, HaloStretch=1.3, BulgeStretch=0.8, Bulge_A=8.0)
    for stream in ((42, 0, 0, 0), (7, 3, 1, 12345)):
        ref, rpos = oracle_lib.run_reference(oracle_lib.reference_positions, m.params, sp, ptype, 3000, stream)
        pos, opos = oracle_lib.oracle_positions(sp, ptype, 3000, stream, use_libm=True)
        assert np.array_equal(pos, ref) and opos == rpos
        g, gpos = oracle_lib.oracle_positions(sp, ptype, 3000, stream, use_libm=False)
        assert gpos == rpos
        assert np.max(np.abs(g - ref)) <= 1e-12 * np.max(np.abs(ref))


@needs_ref
def test_restatement_density_targets_match_reference():
    m = composite()
    sp = shape(m, HaloStretch=1.2)
    stream = (42, 0, 0, 5)
    ref, rpos = oracle_lib.run_reference(oracle_lib.reference_sampling, m.params, sp, 20000, stream, "density")
    out, opos = _restatement_targets(m, sp, 20000, stream, "density", use_libm=True)
    assert opos == rpos
    for t in (1, 2, 3):
        assert np.array_equal(out[t], ref[t][0]), t
    g, gpos = _restatement_targets(m, sp, 20000, stream, "density", use_libm=False)
    assert gpos == rpos
    for t in (1, 2, 3):
        assert peak_rel(g[t], ref[t][0]) < 1e-12


@needs_ref
@pytest.mark.parametrize("tovs,betas", [((1, 3, 0), (0.2, 0.0)), ((1, 2, 1), (1.0, 1.5)), ((0, 2, 3), (0.0, 0.0))])
def test_restatement_energy_targets_match_reference(tovs, betas):
    m = composite(halo_tovs=tovs[0], disk_tovs=tovs[1], bulge_tovs=tovs[2])
    sp = shape(m, HaloBetaParameter=betas[0], BulgeBetaParameter=betas[1])
    tables = disp_tables(m, 3)
    stream = (11, 2, 0, 0)
    ref, rpos = oracle_lib.run_reference(oracle_lib.reference_sampling, m.params, sp, 10000, stream, "energy",
                                         tables)
    out, opos = _restatement_targets(m, sp, 10000, stream, "energy", use_libm=True, tables=tables)
    assert opos == rpos
    for t in (1, 2, 3):
        for k in range(5):
            assert np.array_equal(out[t][k], ref[t][k + 1]), (t, k)


def test_restatement_renormalisation():
    """grid.c:862-880: the finest level times MType / its draw-order sum; coarser levels untouched."""
    m = composite(level=5)
    sp = shape(m)
    a, pa = oracle_lib.oracle_density(m.params, sp, 1, 3000, (1, 0, 0, 0), False, renorm=False)
    b, pb = oracle_lib.oracle_density(m.params, sp, 1, 3000, (1, 0, 0, 0), False, renorm=True)
    L = m.params.DG_MaxLevel
    off = ((1 << (2 * L)) - 1) // 3
    msum = 0.0
    for v in a[off:]:
        msum += v
    assert pa == pb
    assert np.array_equal(b[:off], a[:off])
    assert np.array_equal(b[off:], a[off:] * (m.params.MType[1] / msum))


# ------------------------------------------------------------------ GPU


def _gpu_targets(m, sp, ntarget, stream, kind, tables=None, renorm=False, load=True):
    from galic_b200 import sampling
    with Context(m.params) as ctx:
        if load:
            ctx.load_model(m)
        if tables:
            for t, tab in tables.items():
                sampling.set_dispersion(ctx, t, *tab[:5])
        s = sampling.Stream(*stream)
        if kind == "density":
            sampling.sample_density_targets(ctx, sp, ntarget, s, renorm)
        else:
            sampling.sample_energy_targets(ctx, sp, ntarget, s)
        out = {t: sampling.get_targets(ctx, t) for t in (1, 2, 3)}
        launches = ctx.lib.galic_last_kernel_launches(ctx.h)
    return out, s.position, launches


@pytest.mark.gpu
@pytest.mark.parametrize("ptype", [1, 2, 3])
def test_gpu_positions_bit_identical(ptype):
    from galic_b200 import sampling
    m = composite()
    # Rmax well inside the halo: most halo and bulge draws are redrawn, so the
    # replay crosses several windows and the bulge's redraws shift the parse
    sp = shape(m, Rmax=12.0, HaloStretch=1.3, BulgeStretch=0.8, Bulge_A=6.0)
    for stream, n in (((42, 0, 0, 0), 60000), ((9, 1, 2, 777), 1), ((9, 1, 2, 778), 257)):
        s = sampling.Stream(*stream)
        got = sampling.sample_positions(sp, ptype, n, s)
        ref, rpos = oracle_lib.oracle_positions(sp, ptype, n, stream, use_libm=False)
        assert s.position == rpos
        assert np.array_equal(got, ref)


@pytest.mark.gpu
@pytest.mark.parametrize("rmax_frac", [1.0, 0.15])
def test_gpu_density_targets(rmax_frac):
    m = composite(level=7)
    sp = shape(m, Rmax=m.meta["rmax"] * rmax_frac, HaloStretch=1.2)
    stream = (42, 0, 0, 3)
    got, gpos, launches = _gpu_targets(m, sp, 200000, stream, "density")
    ref, rpos = _restatement_targets(m, sp, 200000, stream, "density", use_libm=False)
    assert gpos == rpos
    assert launches > 0
    for t in (1, 2, 3):
        err = peak_rel(got[t][0], ref[t])
        print(f"type {t}: DG target {err:.2e} of peak")
        assert err < 1e-12


@pytest.mark.gpu
@pytest.mark.parametrize("tovs,betas", [((1, 3, 0), (0.2, 0.0)), ((1, 2, 1), (1.0, 1.5)), ((0, 2, 3), (0.0, 0.0))])
def test_gpu_energy_targets(tovs, betas):
    m = composite(level=7, halo_tovs=tovs[0], disk_tovs=tovs[1], bulge_tovs=tovs[2])
    sp = shape(m, HaloBetaParameter=betas[0], BulgeBetaParameter=betas[1])
    tables = disp_tables(m, 5)
    stream = (11, 2, 0, 0)
    got, gpos, _ = _gpu_targets(m, sp, 100000, stream, "energy", tables)
    ref, rpos = _restatement_targets(m, sp, 100000, stream, "energy", use_libm=False, tables=tables)
    assert gpos == rpos
    for t in (1, 2, 3):
        for k in range(5):
            err = peak_rel(got[t][k + 1], ref[t][k])
            assert err < 1e-12, (t, k, err)


@pytest.mark.gpu
def test_gpu_renormalised_density_targets():
    m = composite(level=7)
    sp = shape(m)
    got, gpos, _ = _gpu_targets(m, sp, 50000, (3, 0, 0, 0), "density", renorm=True)
    ref, rpos = _restatement_targets(m, sp, 50000, (3, 0, 0, 0), "density", use_libm=False, renorm=True)
    assert gpos == rpos
    for t in (1, 2, 3):
        assert peak_rel(got[t][0], ref[t]) < 1e-12


@pytest.mark.gpu
def test_gpu_sampling_edge_cases():
    from galic_b200 import sampling
    m = composite(level=7)
    sp = shape(m)
    # one sample per type
    got, gpos, _ = _gpu_targets(m, sp, 1, (5, 0, 0, 0), "density")
    ref, rpos = _restatement_targets(m, sp, 1, (5, 0, 0, 0), "density", use_libm=False)
    assert gpos == rpos
    for t in (1, 2, 3):
        assert peak_rel(got[t][0], ref[t]) < 1e-12
    # a type without mass is skipped: it draws nothing and keeps its stack
    m.params.MType[2] = 0.0
    got, gpos, _ = _gpu_targets(m, sp, 5000, (5, 0, 0, 0), "density")
    ref, rpos = _restatement_targets(m, sp, 5000, (5, 0, 0, 0), "density", use_libm=False)
    assert gpos == rpos and np.array_equal(got[2][0], m.targets[2][0])
    for t in (1, 3):
        assert peak_rel(got[t][0], ref[t]) < 1e-12
    with Context(composite(level=7).params) as ctx:
        s = sampling.Stream(1)
        for bad in (0, -5):
            with pytest.raises(GalicError) as e:
                sampling.sample_density_targets(ctx, sp, bad, s)
            assert e.value.status == 1
        with pytest.raises(GalicError) as e:  # energy maps need the Jeans tables
            sampling.sample_energy_targets(ctx, sp, 10, s)
        assert e.value.status == 9
        with pytest.raises(GalicError) as e:  # nothing ever lands inside Rmax = 0
            sampling.sample_density_targets(ctx, shape(m, Rmax=0.0), 10, s)
        assert e.value.status == 7
        assert s.position == 0
    s = sampling.Stream(1, position=10)
    assert sampling.sample_positions(sp, 1, 0, s).shape == (0, 3) and s.position == 10


@pytest.mark.gpu
def test_gpu_sampled_targets_drive_calc_all():
    """Targets sampled on the device serve calc_all_response_fields directly."""
    from galic_b200 import sampling
    m = synth.config_halo_disk(n_halo=4000, n_disk=1000, level=6, seed=3)
    sp = shape(m)
    tables = disp_tables(m, 7)
    with Context(m.params) as ctx:
        ctx.load_model(m)
        for t in (1, 2):
            sampling.set_dispersion(ctx, t, *tables[t][:5])
        s = sampling.Stream(42)
        sampling.sample_density_targets(ctx, sp, 100000, s, renormalize=True)
        sampling.sample_energy_targets(ctx, sp, 100000, s)
        ctx.calc_all_response_fields()
        fit = ctx.fit()
        dg = sampling.get_targets(ctx, 1)[0]
    assert np.all(np.isfinite(fit)) and fit[1, 0] > 0
    L = m.params.DG_MaxLevel
    off = ((1 << (2 * L)) - 1) // 3
    assert abs(np.sum(dg[off:]) - m.params.MType[1]) < 1e-9 * m.params.MType[1]
