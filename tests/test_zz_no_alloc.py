"""The allocation-free entry point galic_orbit_responses_noalloc.

Some callers cannot allocate device memory (a framework that owns every
device allocation, work replayed from a captured CUDA graph, a fixed device
budget), so this entry point works only on caller-owned device buffers and a
fixed file-scope scratch array.  This test calls it through the C ABI with
buffers the test allocates itself (torch), twice in a row, and checks its
time-averaged response grids against the context entry point
(galic_calc_all_response_fields) within the batched tolerance of the other
GPU tests.  The file is named to be collected last."""
import ctypes as C

import numpy as np
import pytest

from galic_b200 import Context, _ffi, synth

pytestmark = pytest.mark.gpu

BATCH_TOL = 1e-12  # per grid, relative to the grid's peak bin (as in test_gpu_parity)


def _dev(torch, a, dtype):
    return torch.from_numpy(np.ascontiguousarray(a)).to(dtype=dtype, device="cuda")


def test_noalloc_matches_context_path_twice():
    import torch

    m = synth.config_halo_disk(n_halo=3000, n_disk=1000, level=6, seed=21)
    p = m.params
    with Context(p) as ctx:
        ctx.load_model(m)
        ctx.calc_all_response_fields()
        want = np.stack([np.stack([ctx.response(t, w) for w in range(5)]) for t in (1, 2, 3)])
    lib = _ffi.load_library()
    acc2 = _dev(torch, np.stack([m.dpotdr, m.dpotdz], axis=1), torch.float64)
    pot = _dev(torch, m.pot, torch.float64)
    vstream = _dev(torch, np.concatenate([m.vstream[1], m.vstream[2], m.vstream[3]]), torch.float64)
    cellsize = _dev(torch, m.cellsize, torch.float64)
    pos, vel = _dev(torch, m.pos, torch.float64), _dev(torch, m.vel, torch.float64)
    mass, tint = _dev(torch, m.mass, torch.float64), _dev(torch, m.tint, torch.float64)
    ptype = _dev(torch, m.ptype, torch.int32)
    out = torch.empty((3, 5, 1 << (2 * p.DG_MaxLevel)), dtype=torch.float64, device="cuda")
    orbits = torch.empty(m.n, dtype=torch.int32, device="cuda")
    phi_bound = float(-min(m.pot.min(), 0.0))
    torch.cuda.synchronize()
    results = []
    for _ in range(2):
        out.fill_(-1.0)
        st = lib.galic_orbit_responses_noalloc(
            C.byref(p), acc2.data_ptr(), pot.data_ptr(), vstream.data_ptr(), cellsize.data_ptr(), phi_bound, m.n,
            pos.data_ptr(), vel.data_ptr(), mass.data_ptr(), tint.data_ptr(), ptype.data_ptr(), out.data_ptr(),
            orbits.data_ptr(), None)
        assert st == 0, lib.galic_status_string(st)
        results.append(out.cpu().numpy().copy())
    for got in results:
        for t in range(2):  # halo and disk are present; the bulge grids stay zero
            den = np.maximum(np.abs(want[t]).max(axis=1, keepdims=True), 1e-300)
            assert np.max(np.abs(got[t] - want[t]) / den) <= BATCH_TOL
        assert np.all(got[2] == 0)
    assert np.array_equal(results[0], results[1])
    with Context(p) as ctx:
        ctx.load_model(m)
        ctx.calc_all_response_fields()
        _, want_orbits, _ = ctx.particles()
    assert np.array_equal(orbits.cpu().numpy(), want_orbits)


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
