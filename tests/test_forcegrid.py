"""Tree force-grid fill (forcedensitygrid_calculate grid.c:621-750 with
gravity() gravtree.c:35-50).

CPU: the oracle restatement (oracle/oracle_forcegrid.c) is bit-identical to
GALIC's own fill in the committed fixtures (tests/golden/fill, made by
tests/golden/make_fill_golden.py) and to the live reference; Peano-Hilbert
keys of the oracle, the product's host function and the reference agree;
argument errors are caught before any device work.
GPU: galic_force_grid_fill is bit-identical to the fixtures and to the oracle
on larger seeded inputs, and reports the MAX_TREE_LEVEL case.
"""
import glob
import os

import numpy as np
import pytest

from galic_b200 import _ffi, forcegrid
import oracle_lib

HERE = os.path.dirname(os.path.abspath(__file__))
FIXTURES = sorted(glob.glob(os.path.join(HERE, "golden", "fill", "*.npz")))


def load_fixture(path):
    z = np.load(path)
    rmin, fac, G, soft, theta, tnf = z["fill"]
    fp = forcegrid.fill_params(int(z["fg_nbin"]), rmin, fac, G, soft, theta, tnf, int(z["multiple_domains"]))
    return fp, z["pos"], z["mass"], (z["dpotdr"], z["dpotdz"], z["pot"])


def seeded_particles(n_halo, n_disk, seed, halo_a=30.0, disk_h=3.5, disk_z0=0.7, rmax=500.0):
    """Hernquist halo (inverse CDF radii, isotropic) + exponential sech^2 disk."""
    rng = np.random.default_rng(seed)
    u = rng.uniform(0.0, 0.98, n_halo)
    r = halo_a * np.sqrt(u) / (1 - np.sqrt(u))
    r = np.minimum(r, rmax)
    cth = rng.uniform(-1, 1, n_halo)
    ph = rng.uniform(0, 2 * np.pi, n_halo)
    sth = np.sqrt(1 - cth ** 2)
    halo = np.stack([r * sth * np.cos(ph), r * sth * np.sin(ph), r * cth], axis=1)
    R = rng.gamma(2.0, disk_h, n_disk)
    z = disk_z0 / 2 * np.log(rng.uniform(1e-12, 1, n_disk) / rng.uniform(1e-12, 1, n_disk))
    phd = rng.uniform(0, 2 * np.pi, n_disk)
    disk = np.stack([R * np.cos(phd), R * np.sin(phd), z], axis=1)
    pos = np.concatenate([halo, disk])
    mass = np.concatenate([np.full(n_halo, 95.0 / max(n_halo, 1)), np.full(n_disk, 5.0 / max(n_disk, 1))])
    return pos, mass


# ------------------------------------------------------------------ CPU tests

def test_fixtures_present():
    assert len(FIXTURES) >= 3


@pytest.mark.parametrize("path", FIXTURES, ids=lambda p: os.path.basename(p)[:-4])
def test_oracle_fill_matches_reference_fixture(path):
    fp, pos, mass, want = load_fixture(path)
    st, *got = oracle_lib.oracle_force_grid_fill(fp, pos, mass)
    assert st == 0
    for g, w in zip(got, want):
        assert np.array_equal(g, w)


def test_oracle_fill_matches_live_reference():
    if not oracle_lib.reference_available():
        pytest.skip("GALIC's own C (oracle/_ref) is not built here")
    import sys
    sys.path.insert(0, os.path.join(HERE, "golden"))
    from make_fill_golden import case_params
    p, rmax = case_params("hdb", 20)
    rf = oracle_lib.RefFillParams(0.1, 0.5, 3.0, 3.5, 0.7, rmax, 2, 1500, 700, 300, 4242)
    pos, mass, *want = oracle_lib.run_reference(oracle_lib.reference_force_fill, p, rf)
    fp = forcegrid.fill_params(p.FG_Nbin, p.FG_Rmin, p.FG_Fac, p.G, rf.Softening, rf.ErrTolTheta,
                               rf.TopNodeFactor, rf.MultipleDomains)
    st, *got = oracle_lib.oracle_force_grid_fill(fp, pos, mass)
    assert st == 0
    for g, w in zip(got, want):
        assert np.array_equal(g, w)


def test_peano_keys_agree():
    rng = np.random.default_rng(5)
    ol = oracle_lib.oracle_lib()
    lib = _ffi.load_library()
    cases = []
    for bits in (1, 2, 3, 7, 13, 21):
        xyz = rng.integers(0, 1 << bits, size=(200, 3))
        cases.append((bits, xyz))
        for x, y, z in xyz:
            k = ol.orc_peano_key(int(x), int(y), int(z), bits)
            assert lib.galic_peano_hilbert_key(int(x), int(y), int(z), bits) == k
            assert k < (1 << (3 * bits))
    # a Peano-Hilbert curve visits neighbouring cells: keys k and k+1 are face neighbours
    bits = 4
    cells = {ol.orc_peano_key(x, y, z, bits): (x, y, z) for x in range(16) for y in range(16) for z in range(16)}
    assert sorted(cells) == list(range(16 ** 3))
    for k in range(16 ** 3 - 1):
        assert sum(abs(a - b) for a, b in zip(cells[k], cells[k + 1])) == 1
    if oracle_lib.reference_available():
        for bits, xyz in cases:
            ref = oracle_lib.run_reference(oracle_lib.reference_peano_keys, xyz, bits)
            mine = np.array([ol.orc_peano_key(int(x), int(y), int(z), bits) for x, y, z in xyz], dtype=np.uint64)
            assert np.array_equal(ref, mine)


def test_fill_argument_errors_before_device():
    lib = _ffi.load_library()
    fp, pos, mass, _ = load_fixture(FIXTURES[0])
    import ctypes as C
    out = [np.zeros(fp.FG_Nbin ** 2) for _ in range(3)]

    def call(f, n=len(mass)):
        return lib.galic_force_grid_fill(C.byref(f), n, _ffi.dptr(pos), _ffi.dptr(mass),
                                         *[_ffi.dptr(a) for a in out], None)
    for field, value in (("FG_Nbin", 1), ("FG_Fac", 1.0), ("FG_Rmin", 0.0), ("ErrTolTheta", 0.0),
                         ("ForceSoftening", -1.0), ("MultipleDomains", 0), ("TopNodeFactor", 0.0)):
        bad = _ffi.GalicFillParams()
        C.memmove(C.byref(bad), C.byref(fp), C.sizeof(bad))
        setattr(bad, field, value)
        assert call(bad) == 1, field
    assert call(fp, 0) == 1


def test_oracle_reports_coincident_particles():
    """Particles closer than DomainLen/2^30 reach the MAX_TREE_LEVEL slot shift
    of forcetree.c:400-416, which the fill does not reproduce."""
    fp, pos, mass, _ = load_fixture(FIXTURES[0])
    pos = pos.copy()
    pos[1] = pos[0]
    st, *_ = oracle_lib.oracle_force_grid_fill(fp, pos, mass)
    assert st == 6


# ------------------------------------------------------------------ GPU tests

@pytest.mark.gpu
@pytest.mark.parametrize("path", FIXTURES, ids=lambda p: os.path.basename(p)[:-4])
def test_gpu_fill_matches_reference_fixture(path):
    fp, pos, mass, want = load_fixture(path)
    got = forcegrid.force_grid_fill(fp, pos, mass)
    for g, w in zip(got[:3], want):
        assert np.array_equal(g, w)
    st = got[3]
    assert st["tree_items"] > len(mass) and st["tree_nodes"] == st["tree_items"] - len(mass)
    assert st["interactions"] > 0 and st["node_tests"] > 0 and st["ms_walk"] > 0


@pytest.mark.gpu
@pytest.mark.parametrize("nh,nd,fg,theta,soft,seed", [(60000, 20000, 64, 0.4, 0.3, 1),
                                                      (30000, 30000, 40, 0.7, 0.05, 2),
                                                      (5000, 0, 96, 0.2, 1.0, 3)])
def test_gpu_fill_matches_oracle(nh, nd, fg, theta, soft, seed):
    pos, mass = seeded_particles(nh, nd, seed)
    if seed == 2:
        mass[:100] = 0.0  # massless sampled particles (a component of zero mass)
    fp = forcegrid.fill_params(fg, 0.05, 1.06, 43007.1, soft, theta, 4.0, 4)
    st, *want = oracle_lib.oracle_force_grid_fill(fp, pos, mass)
    assert st == 0
    got = forcegrid.force_grid_fill(fp, pos, mass)
    for g, w in zip(got[:3], want):
        assert np.array_equal(g, w)


@pytest.mark.gpu
def test_gpu_fill_deterministic_and_coincident_rejected():
    fp, pos, mass, _ = load_fixture(FIXTURES[-1])
    a = forcegrid.force_grid_fill(fp, pos, mass)
    b = forcegrid.force_grid_fill(fp, pos, mass)
    for x, y in zip(a[:3], b[:3]):
        assert np.array_equal(x, y)
    pos = pos.copy()
    pos[1] = pos[0]
    with pytest.raises(Exception) as e:
        forcegrid.force_grid_fill(fp, pos, mass)
    assert getattr(e.value, "status", None) == 6
