"""Output files: the Gadget snapshot (write_file, io.c:906-1243), forcefield.dat
(grid.c:789-823) and densfield_<type>_<num>.dat (output_density_field,
io.c:36-460).

CPU: galic_write_snapshot, galic_write_forcefield and
galic_write_density_field, given the arrays GALIC's own code holds, write
files byte-identical to the ones GALIC's own writers produce.
GPU: galic_output_density_field writes the context's targets and committed
grids through the same writer."""
import ctypes as C
import os
import sys

import numpy as np
import pytest

import oracle_lib
from galic_b200 import _ffi, synth

HERE = os.path.dirname(os.path.abspath(__file__))
needs_ref = pytest.mark.skipif(not oracle_lib.reference_available(), reason="oracle/_ref not built")


@needs_ref
@pytest.mark.parametrize("fmt", [1, 2])
def test_snapshot_matches_reference(fmt, tmp_path):
    import test_particles as TP
    m = TP.particle_model(n=(300, 150, 60))
    sp, _, tables, tf = TP.setup_inputs(m)
    ref, data = oracle_lib.run_reference(oracle_lib.reference_snapshot, m.params, (m.pot, m.dpotdr, m.dpotdz), sp, tf,
                                         tables, (42, 0, 0, 3), fmt)
    from galic_b200 import io
    fn = io.output_particles(str(tmp_path) + "/", "snap", 0, ref, snap_format=fmt)
    assert fn.endswith("snap_000")
    got = open(fn, "rb").read()
    assert len(got) == len(data) and got == data


@needs_ref
def test_forcefield_matches_reference(tmp_path):
    sys.path.insert(0, os.path.join(HERE, "golden"))
    from make_fill_golden import case_params
    p, rmax = case_params("hdb", 20)
    rf = oracle_lib.RefFillParams(0.1, 0.5, 3.0, 3.5, 0.7, rmax, 2, 600, 300, 100, 77)
    dpotdr, dpotdz, pot, data = oracle_lib.run_reference(oracle_lib.reference_forcefield, p, rf)
    from galic_b200 import io
    fn = str(tmp_path / "forcefield.dat")
    io.write_forcefield(fn, p, dpotdr, dpotdz, pot)
    assert open(fn, "rb").read() == data


@needs_ref
def test_density_field_matches_reference(tmp_path):
    m = synth.config_composite(n_halo=600, n_disk=300, n_bulge=100, level=5, seed=3)
    ref = oracle_lib.run_reference(oracle_lib.reference_density_field, m)
    lib = _ffi.load_library()
    assert sorted(ref) == [1, 2, 3]
    for t, (data, st, locs) in ref.items():
        fn = str(tmp_path / f"densfield_{t}_000.dat")
        egs = np.ascontiguousarray(np.concatenate(st[1:]))
        loc = [np.ascontiguousarray(a) for a in locs]
        eg = np.ascontiguousarray(np.concatenate(loc[1:]))
        rc = lib.galic_write_density_field(fn.encode(), C.byref(m.params), t, _ffi.dptr(np.ascontiguousarray(st[0])),
                                           _ffi.dptr(egs), _ffi.dptr(loc[0]), _ffi.dptr(eg))
        assert rc == 0
        got = open(fn, "rb").read()
        assert len(got) == len(data) and got == data, t


def test_writers_reject_bad_arguments(tmp_path):
    lib = _ffi.load_library()
    z = np.zeros(3)
    i = np.zeros(1, dtype=np.int32)
    fn = str(tmp_path / "x").encode()
    assert lib.galic_write_snapshot(fn, 3, 1, *[_ffi.dptr(z)] * 4, _ffi.iptr(i), _ffi.iptr(i), None) == 1
    bad = np.array([7], dtype=np.int32)
    assert lib.galic_write_snapshot(fn, 1, 1, *[_ffi.dptr(z)] * 4, _ffi.iptr(i), _ffi.iptr(bad), None) == 1
    assert lib.galic_write_snapshot(str(tmp_path / "no" / "dir").encode(), 1, 0, None, None, None, None, None, None,
                                    None) == 1


@pytest.mark.gpu
def test_gpu_output_density_field(tmp_path):
    """The context's targets and committed grids through galic_write_density_field."""
    from galic_b200 import sampling
    from galic_b200.context import Context
    m = synth.config_halo_disk(n_halo=3000, n_disk=1000, level=6, seed=4)
    lib = _ffi.load_library()
    with Context(m.params) as ctx:
        ctx.load_model(m)
        ctx.calc_all_response_fields()
        from galic_b200 import io
        io.output_density_field(ctx, tmp_path, 7)
        for t in (1, 2):
            tg = sampling.get_targets(ctx, t)
            loc = [ctx.response(t, w) for w in (_ffi.GRID_MASS_S, _ffi.GRID_MASS_I, _ffi.GRID_R_I, _ffi.GRID_T_I,
                                               _ffi.GRID_P_I, _ffi.GRID_Q_I)]
            fn = str(tmp_path / f"check_{t}.dat")
            rc = lib.galic_write_density_field(fn.encode(), C.byref(m.params), t, _ffi.dptr(tg[0]),
                                               _ffi.dptr(np.ascontiguousarray(np.concatenate(tg[1:]))),
                                               _ffi.dptr(loc[0]), _ffi.dptr(np.ascontiguousarray(np.concatenate(loc[1:]))))
            assert rc == 0
            assert open(fn, "rb").read() == open(tmp_path / f"densfield_{t}_007.dat", "rb").read()
        assert not os.path.exists(tmp_path / "densfield_3_007.dat")
