"""Generates the golden fixtures from GALIC's own C (oracle/_ref/libgalic_ref.so).

Run in a checkout that has the reference tree (the library is built from it by
oracle/Makefile):  python tests/golden/make_golden.py

Each fixture holds the full input of a small seeded model (force grid with
FG_Nbin = 64, response grids of level 5) and the reference's outputs:
* per-orbit results of produce_orbit_response_field_mod / _field
  (orbit_response.c:33-491) for a list of particles, including edge cases
  (below the midplane, near the z axis, starting outside the grid);
* calc_all_response_fields (main.c:151-246): the committed per-type grids and
  the fit of calc_global_fit (main.c:251-362);
* one optimisation repetition (main.c:96-100) over a particle list with
  Philox proposal streams: fit, counters, velocities, orbit counts and the
  instantaneous projections afterwards.
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.dirname(HERE))

from galic_b200 import synth, _ffi  # noqa: E402
import oracle_lib  # noqa: E402

SEED = 20240611
REP_SEED = 987654321


def scenario_models():
    C = synth.Component
    out = {}
    m = synth.build_model([C("halo", 100.0, 30.0, 40, tovs=0)], seed=11, level=5, fg_nbin=64, torbit_fac=2.0)
    m.params.SampleForceNhalo = 0  # analytic halo force (grid.c:172-183)
    out["halo_analytic"] = m
    out["halo_disk"] = synth.build_model([C("halo", 95.0, 30.0, 30, tovs=0), C("disk", 5.0, 3.5, 20, z0=0.7, tovs=3)],
                                         seed=12, level=5, fg_nbin=64, torbit_fac=2.0, inner_frac=1e-7,
                                         outer_frac=0.49)
    out["composite"] = synth.build_model([C("halo", 93.5, 30.0, 30, beta=0.2, tovs=1),
                                          C("disk", 5.0, 3.5, 20, z0=0.7, tovs=2),
                                          C("bulge", 1.5, 1.0, 12, tovs=0)],
                                         seed=13, level=5, fg_nbin=64, torbit_fac=2.0)
    # halo from the force grid, bulge analytic (SampleForceNbulge = 0): the
    # bulge_get_acceleration / _potential branch of grid.c:185-196 and
    # grid.c:103-108 (bulge.c:64-85)
    m = synth.build_model([C("halo", 98.5, 30.0, 30, tovs=0), C("bulge", 1.5, 1.0, 20, tovs=0)],
                          seed=14, level=5, fg_nbin=64, torbit_fac=2.0)
    m.params.SampleForceNbulge = 0
    out["bulge_analytic"] = m
    for name, m in out.items():
        # edge cases: one particle mirrored below the midplane, one near the axis,
        # one outside the tabulated grid
        m.pos[1, 2] = -abs(m.pos[1, 2])
        m.pos[2, :2] *= 1e-6
        r = np.linalg.norm(m.pos[3])
        m.pos[3] *= 1.5 * m.meta["rmax"] / r
        m.vel[3] *= 0.2
        m.tint[3] = m.tint[0]
    return out


def model_arrays(m):
    d = {k: np.asarray(getattr(m, k)) for k in ("pot", "dpotdr", "dpotdz", "cellsize", "dgs_distance", "pos", "vel",
                                                 "mass", "tint", "vesc", "ptype", "ptargets")}
    for t in (1, 2, 3):
        d[f"vstream{t}"] = np.asarray(m.vstream[t])
    for t, tg in m.targets.items():
        for k, a in enumerate(tg):
            d[f"target{t}_{k}"] = a
    d["params"] = np.frombuffer(bytes(m.params), dtype=np.uint8).copy()
    return d


def run(name, arrays):
    """Runs one scenario through the reference (in its own process)."""
    m = model_from_arrays(arrays)
    ref = oracle_lib.Reference(m.params)
    ref.load_model(m)
    out = {}
    sel = list(range(0, 8)) + [m.n - 1]
    for j, i in enumerate(sel):
        tall, orbits, *g = ref.orbit_mod(m.pos[i], m.vel[i], m.mass[i], m.tint[i], m.ptype[i])
        out[f"orbit{j}_idx"] = np.array(i)
        out[f"orbit{j}_tall"] = np.array(tall)
        out[f"orbit{j}_norbit"] = np.array(orbits)
        out[f"orbit{j}_grids"] = np.stack(g)
    for j, i in enumerate(sel[:3]):
        tall, orbits, mm = ref.orbit(m.pos[i], m.vel[i], m.mass[i], m.tint[i])
        out[f"morbit{j}_tall"] = np.array(tall)
        out[f"morbit{j}_norbit"] = np.array(orbits)
        out[f"morbit{j}_grid"] = mm
    ref.calc_all()
    out["calc_fit"] = ref.fit()
    for t in (1, 2, 3):
        if m.params.NType[t]:
            out[f"calc_resp{t}"] = np.stack([ref.response(t, w) for w in range(_ffi.GRID_COUNT)])
    vel, orbits, vdisp = ref.particles()
    out["calc_orbits"] = orbits
    out["calc_vdisp"] = vdisp
    idx = np.random.default_rng(SEED).permutation(m.n)[:12].astype(np.int32)
    out["rep_idx"] = idx
    ref.optimize_rep(idx, REP_SEED, 7)
    out["rep_fit"] = ref.fit()
    tr, ch = ref.counters()
    out["rep_tries"] = tr
    out["rep_changes"] = ch
    vel, orbits, vdisp = ref.particles()
    out["rep_vel"] = vel
    out["rep_orbits"] = orbits
    out["rep_vdisp"] = vdisp
    for t in (1, 2, 3):
        if m.params.NType[t]:
            out[f"rep_resp{t}"] = np.stack([ref.response(t, w) for w in range(_ffi.GRID_COUNT)])
    return out


def model_from_arrays(a):
    p = _ffi.GalicParams.from_buffer_copy(a["params"].tobytes())
    targets = {}
    for t in (1, 2, 3):
        if f"target{t}_0" in a:
            targets[t] = tuple(np.ascontiguousarray(a[f"target{t}_{k}"]) for k in range(6))
    return synth.Model(params=p, pot=a["pot"], dpotdr=a["dpotdr"], dpotdz=a["dpotdz"],
                       vstream={t: a[f"vstream{t}"] for t in (1, 2, 3)}, cellsize=a["cellsize"],
                       dgs_distance=a["dgs_distance"], targets=targets, pos=np.ascontiguousarray(a["pos"]),
                       vel=np.ascontiguousarray(a["vel"]), mass=a["mass"], tint=a["tint"], vesc=a["vesc"],
                       ptype=np.ascontiguousarray(a["ptype"], dtype=np.int32), ptargets=a["ptargets"])


def main(names=None):
    """Writes every scenario's fixture, or only those named on the command line."""
    oracle_lib.build_oracle()
    assert oracle_lib.reference_available(), "oracle/_ref/libgalic_ref.so missing (needs the reference tree)"
    for name, m in scenario_models().items():
        if names and name not in names:
            continue
        arrays = model_arrays(m)
        out = oracle_lib.run_reference(run, name, arrays)
        path = os.path.join(HERE, f"{name}.npz")
        np.savez_compressed(path, **{f"in_{k}": v for k, v in arrays.items()}, **{f"out_{k}": v for k, v in out.items()})
        print(path, os.path.getsize(path))


if __name__ == "__main__":
    main(sys.argv[1:])
