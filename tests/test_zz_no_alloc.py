"""The allocation-free entry point galic_orbit_responses_noalloc.

Some callers cannot allocate device memory (a framework that owns every
device allocation, a fixed device budget), so this entry point works only on
caller-owned device buffers and a fixed file-scope scratch array.  These
tests call it through the C ABI with buffers the test allocates itself
(torch), twice in a row, and check its time-averaged response grids against
the context entry point (galic_calc_all_response_fields) within the batched
tolerance of the other GPU tests: a halo + disk model at DG level 6, and a
halo + disk + bulge model at level 7, the largest grid the scratch array
holds.  The file is named to be collected last."""
import ctypes as C

import numpy as np
import pytest

from galic_b200 import Context, _ffi, synth

pytestmark = pytest.mark.gpu

BATCH_TOL = 1e-12  # per grid, relative to the grid's peak bin (as in test_gpu_parity)


def _dev(torch, a, dtype):
    return torch.from_numpy(np.ascontiguousarray(a)).to(dtype=dtype, device="cuda")


class _Buffers:
    """Device copies of a model's tables and particles, owned by the test."""

    def __init__(self, torch, m):
        p = m.params
        self.acc2 = _dev(torch, np.stack([m.dpotdr, m.dpotdz], axis=1), torch.float64)
        self.pot = _dev(torch, m.pot, torch.float64)
        self.vstream = _dev(torch, np.concatenate([m.vstream[1], m.vstream[2], m.vstream[3]]), torch.float64)
        self.cellsize = _dev(torch, m.cellsize, torch.float64)
        self.pos, self.vel = _dev(torch, m.pos, torch.float64), _dev(torch, m.vel, torch.float64)
        self.mass, self.tint = _dev(torch, m.mass, torch.float64), _dev(torch, m.tint, torch.float64)
        self.ptype = _dev(torch, m.ptype, torch.int32)
        self.out = torch.empty((3, 5, 1 << (2 * p.DG_MaxLevel)), dtype=torch.float64, device="cuda")
        self.orbits = torch.empty(m.n, dtype=torch.int32, device="cuda")
        self.phi_bound = float(-min(m.pot.min(), 0.0))

    def call(self, lib, p, n):
        return lib.galic_orbit_responses_noalloc(
            C.byref(p), self.acc2.data_ptr(), self.pot.data_ptr(), self.vstream.data_ptr(),
            self.cellsize.data_ptr(), self.phi_bound, n, self.pos.data_ptr(), self.vel.data_ptr(),
            self.mass.data_ptr(), self.tint.data_ptr(), self.ptype.data_ptr(), self.out.data_ptr(),
            self.orbits.data_ptr(), None)


def _check_twice(m, types):
    import torch

    p = m.params
    with Context(p) as ctx:
        ctx.load_model(m)
        ctx.calc_all_response_fields()
        want = np.stack([np.stack([ctx.response(t, w) for w in range(5)]) for t in (1, 2, 3)])
        _, want_orbits, _ = ctx.particles()
    lib = _ffi.load_library()
    b = _Buffers(torch, m)
    torch.cuda.synchronize()
    results = []
    for _ in range(2):
        b.out.fill_(-1.0)
        b.orbits.fill_(-1)
        st = b.call(lib, p, m.n)
        assert st == 0, lib.galic_status_string(st)
        results.append(b.out.cpu().numpy().copy())
        assert np.array_equal(b.orbits.cpu().numpy(), want_orbits)
    for got in results:
        for t in range(3):
            if t + 1 in types:
                den = np.maximum(np.abs(want[t]).max(axis=1, keepdims=True), 1e-300)
                assert np.max(np.abs(got[t] - want[t]) / den) <= BATCH_TOL
                assert np.abs(got[t]).max() > 0
            else:
                assert np.all(got[t] == 0)
    assert np.array_equal(results[0], results[1])
    return b


def test_noalloc_matches_context_path_twice():
    m = synth.config_halo_disk(n_halo=3000, n_disk=1000, level=6, seed=21)
    _check_twice(m, (1, 2))


def test_noalloc_level7_with_bulge_matches_context_path_twice():
    m = synth.config_composite(n_halo=3000, n_disk=1000, n_bulge=800, level=7, seed=22)
    _check_twice(m, (1, 2, 3))


def test_noalloc_skips_and_reports_invalid_particles():
    """Particles with a type outside 1..3 or a non-positive Tint are skipped on
    the device (no deposit, orbit count 0) and the call reports
    GALIC_ERR_INVALID_ARGUMENT; the valid particles are binned as usual."""
    import torch

    m = synth.config_halo_disk(n_halo=300, n_disk=100, level=6, seed=23)
    lib = _ffi.load_library()
    b = _Buffers(torch, m)
    bad = [5, 17, 250]
    t = m.ptype.copy()
    t[5], t[17] = 0, 7
    tint = m.tint.copy()
    tint[250] = 0.0
    b.ptype.copy_(torch.from_numpy(t))
    b.tint.copy_(torch.from_numpy(tint))
    b.orbits.fill_(-1)
    assert b.call(lib, m.params, m.n) == 1  # GALIC_ERR_INVALID_ARGUMENT
    orb = b.orbits.cpu().numpy()
    assert np.all(orb[bad] == 0) and np.all(orb >= 0)


def test_noalloc_rejects_sizes_beyond_its_scratch():
    import torch

    lib = _ffi.load_library()
    p, _, _ = synth.make_params([synth.Component("halo", 100.0, 30.0, 100)], level=7, fg_nbin=64)
    big = p.copy()
    big.DG_MaxLevel = big.EG_MaxLevel = 8
    x = torch.zeros(8, dtype=torch.float64, device="cuda")
    st = lib.galic_orbit_responses_noalloc(C.byref(big), x.data_ptr(), x.data_ptr(), x.data_ptr(), x.data_ptr(),
                                           1.0, 0, None, None, None, None, None, x.data_ptr(), None, None)
    assert st == 5  # GALIC_ERR_BUDGET
