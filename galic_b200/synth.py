"""Seeded synthetic GALIC models of the shapes the benchmark configurations name.

GALIC builds its inputs with set-up code that is not on the hot path: the
tree-filled force grid (grid.c:621-757), the Jeans dispersion tables
(disp_fields.c), the sampled target stacks (grid.c:536-617, 941-1076) and the
initial particles (set_particles.c:15-307).  This module produces inputs of
the same shapes and value ranges from closed forms, seeded, so that the hot
path can be exercised and timed without the set-up:

* force grid: Hernquist halo/bulge (halo.c:63-84) plus a Miyamoto-Nagai
  stand-in for the exponential disk, tabulated on the FG nodes
  R_j = FG_Rmin (FG_Fac^j - 1) (grid.c:199-202);
* streaming velocity: 0.7 v_c for disk particles, zero for spheroids;
* dispersion targets: Hernquist's isotropic closed form (halo.c:95-118) with
  the anisotropy beta (disp_fields.c:86-92), and pi G Sigma z0 for the disk;
* density targets: cell volume x density at the cell centre (grid.c:830-857),
  renormalised to the component mass (grid.c:864-878); the energy-grid
  targets use the same mass map times the dispersion at the cell centre;
* particles: inverse-CDF radii (halo.c:21-39), exponential/sech^2 disk,
  Gaussian velocities in the local frame with the escape-speed cut of
  set_particles.c:166-184, Tint = TorbitFac 2 pi r / sqrt(r |a|)
  (set_particles.c:87).

Units are GALIC's (kpc, km/s, 1e10 Msun): G and H follow init.c:46-63.
"""
from dataclasses import dataclass, field

import numpy as np

from . import _ffi

GRAVITY = 6.6738e-8
HUBBLE = 3.2407789e-18
UNIT_LENGTH = 3.085678e21
UNIT_MASS = 1.989e43
UNIT_VELOCITY = 1e5
UNIT_TIME = UNIT_LENGTH / UNIT_VELOCITY
G_INTERNAL = GRAVITY / UNIT_LENGTH ** 3 * UNIT_MASS * UNIT_TIME ** 2
H_INTERNAL = HUBBLE * UNIT_TIME

# Set-up geometry (grid spacing, cell sizes, stack smoothing): by default the
# host functions of libgalic_cuda.so (galic_grid_geometry,
# galic_density_geometry, galic_smooth_stack).  use_geometry() swaps in any
# object with the same three functions, so that a CPU-only process (the
# benchmark's timing of GALIC's own C) builds the same workload without
# loading the CUDA library.
_geometry = None


def use_geometry(provider):
    """Routes the set-up geometry to `provider` (None: libgalic_cuda.so)."""
    global _geometry
    _geometry = provider


def _geo():
    return _geometry if _geometry is not None else _ffi.load_library()


@dataclass
class Component:
    kind: str          # "halo", "disk", "bulge"
    mass: float
    scale: float       # a (Hernquist) or h (disk scale length)
    n: int
    z0: float = 0.0    # disk sech^2 height
    beta: float = 0.0  # spheroid anisotropy (TypeOfVelocityStructure 1)
    tovs: int = 0      # TypeOfVelocityStructure


@dataclass
class Model:
    params: _ffi.GalicParams
    pot: np.ndarray
    dpotdr: np.ndarray
    dpotdz: np.ndarray
    vstream: dict
    cellsize: np.ndarray
    dgs_distance: np.ndarray
    targets: dict       # type -> (dgs_mass, egs_mass, egs_r, egs_t, egs_p, egs_q)
    pos: np.ndarray
    vel: np.ndarray
    mass: np.ndarray
    tint: np.ndarray
    vesc: np.ndarray
    ptype: np.ndarray
    ptargets: np.ndarray
    meta: dict = field(default_factory=dict)

    @property
    def n(self):
        return len(self.mass)


TYPE_OF = {"halo": 1, "disk": 2, "bulge": 3}


def _hernquist_sigma2(r, mass, a):
    """Isotropic Hernquist dispersion (Hernquist 1990, as in halo.c:95-118)."""
    r = np.maximum(np.asarray(r, dtype=np.float64), 1e-8 * a)
    x = r / a
    with np.errstate(all="ignore"):
        s2 = G_INTERNAL * mass / (12.0 * a) * np.abs(
            12.0 * r * (r + a) ** 3 / a ** 4 * np.log((r + a) / r)
            - r / (r + a) * (25.0 + x * (52.0 + 42.0 * x + 12.0 * x * x)))
    # far out the closed form cancels catastrophically: use the large-r limit
    far = x > 300
    s2 = np.where(far, G_INTERNAL * mass / (5.0 * r), s2)
    return s2


class _Potential:
    """Analytic total potential/acceleration of the synthetic model."""

    def __init__(self, comps, md_a_fac=1.2):
        self.comps = comps
        self.md_a_fac = md_a_fac

    def evaluate(self, R, z):
        R = np.asarray(R, dtype=np.float64)
        z = np.asarray(z, dtype=np.float64)
        pot = np.zeros(np.broadcast(R, z).shape)
        aR = np.zeros_like(pot)
        az = np.zeros_like(pot)
        for c in self.comps:
            if c.kind in ("halo", "bulge"):
                a = c.scale
                r = np.sqrt(R * R + z * z)
                fac = G_INTERNAL * c.mass / ((r + 1e-6 * a) * (r + a) ** 2)
                aR += -fac * R
                az += -fac * z
                pot += -G_INTERNAL * c.mass / (r + a)
            else:
                ad = self.md_a_fac * c.scale
                b = max(c.z0, 1e-6)
                zeta = np.sqrt(z * z + b * b)
                D = np.sqrt(R * R + (ad + zeta) ** 2)
                pot += -G_INTERNAL * c.mass / D
                aR += -G_INTERNAL * c.mass * R / D ** 3
                az += -G_INTERNAL * c.mass * z * (ad + zeta) / (zeta * D ** 3)
        return pot, aR, az


def make_params(comps, v200=None, fg_nbin=256, level=6, outer_frac=0.980296, inner_frac=9.80296e-5,
                torbit_fac=5.0, f_orb=0.0314, f_cc=0.25, min_disp=100, min_dens=50):
    lib = _geo()
    m200 = sum(c.mass for c in comps)
    if v200 is None:
        v200 = (10.0 * G_INTERNAL * H_INTERNAL * m200) ** (1.0 / 3.0)  # structure.c:60
    halo = [c for c in comps if c.kind == "halo"][0]
    p = _ffi.GalicParams()
    p.V200 = v200
    p.M200 = m200
    p.R200 = v200 / (10.0 * H_INTERNAL)  # structure.c:63
    p.G = G_INTERNAL
    p.Halo_Mass = halo.mass
    p.Halo_A = halo.scale
    p.HaloStretch = 1.0
    p.BulgeStretch = 1.0
    for c in comps:
        if c.kind == "disk":
            p.Disk_Mass = c.mass
        if c.kind == "bulge":
            p.Bulge_Mass = c.mass
            p.Bulge_A = c.scale
    p.TimeStepFactorOrbit = f_orb
    p.TimeStepFactorCellCross = f_cc
    p.LowerDispLimit = (0.01 * v200) ** 2  # structure.c:65
    p.MaxVelInUnitsVesc = 0.99
    # force grid tabulated for every component (tree-filled in the reference)
    p.SampleForceNhalo = 1000000
    p.SampleForceNdisk = 1000000 if p.Disk_Mass > 0 else 0
    p.SampleForceNbulge = 1000000 if p.Bulge_Mass > 0 else 0
    p.MinParticlesPerBinForDispersionMeasurement = min_disp
    p.MinParticlesPerBinForDensityMeasurement = min_dens
    for c in comps:
        t = TYPE_OF[c.kind]
        p.TypeOfVelocityStructure[t] = c.tovs
        p.MType[t] = c.mass
        p.NType[t] = c.n
    for t in range(4):
        p.fac_value_rs[t] = p.fac_value_ts[t] = p.fac_value_qs[t] = p.fac_value_ps[t] = 1.0
    p.FG_Nbin = fg_nbin
    p.DG_MaxLevel = level
    p.EG_MaxLevel = level
    geo = np.zeros(8)
    st = lib.galic_grid_geometry(halo.scale, outer_frac, inner_frac, fg_nbin, level, level, _ffi.dptr(geo))
    if st:
        raise ValueError("grid geometry failed")
    p.DG_Fac, p.DG_Rmin, p.FG_Fac, p.FG_Rmin, p.EG_Fac, p.EG_Rmin = geo[2], geo[3], geo[4], geo[5], geo[6], geo[7]
    return p, float(geo[0]), torbit_fac


def _disp_rtp(comp, pot_obj, R, z, vstr):
    """(disp_r, disp_t, disp_p, disp_q) targets as get_disp_rtp (disp_fields.c:66-115) orders them."""
    r = np.sqrt(R * R + z * z)
    if comp.kind in ("halo", "bulge"):
        total = sum(c.mass for c in pot_obj.comps)
        a = comp.scale if comp.kind == "halo" else max(comp.scale, 1e-3)
        s2 = _hernquist_sigma2(r, total if comp.kind == "halo" else comp.mass + 0.1 * total, a)
        dr = s2
        dt = (1.0 - comp.beta) * dr
        if comp.tovs == 0:
            return dr, dr, dr, dr
        return dr, dt, dt, dt
    sigma_surf = comp.mass / (2 * np.pi * comp.scale ** 2) * np.exp(-R / comp.scale)
    sz2 = np.pi * G_INTERNAL * sigma_surf * comp.z0
    dr = sz2
    dt = sz2
    dp = 0.5 * sz2
    return dr, dt, dp, dp + vstr * vstr


def _density(comp, R, z):
    with np.errstate(over="ignore"):
        return _density_raw(comp, R, z)


def _density_raw(comp, R, z):
    r = np.sqrt(R * R + z * z)
    if comp.kind in ("halo", "bulge"):
        a = comp.scale
        return comp.mass / (2 * np.pi) * a / ((r + 1e-6 * a) * (r + a) ** 3)
    h, z0 = comp.scale, comp.z0
    return comp.mass / (4 * np.pi * h * h * z0) * np.exp(-R / h) * (2.0 / (np.exp(z / z0) + np.exp(-z / z0))) ** 2


def _stack_offset(l):
    return ((1 << (2 * l)) - 1) // 3


def _smooth(finest, level):
    lib = _geo()
    ns = ((1 << (2 + 2 * level)) - 1) // 3
    st = np.zeros(ns)
    st[_stack_offset(level):] = finest
    lib.galic_smooth_stack(_ffi.dptr(st), level)
    return st


def _sample_positions(comp, n, rng, rmax):
    out = np.zeros((n, 3))
    got = 0
    while got < n:
        m = 2 * (n - got) + 16
        if comp.kind in ("halo", "bulge"):
            q = rng.random(m)
            r = comp.scale * (q + np.sqrt(q)) / (1 - q)
            phi = rng.random(m) * 2 * np.pi
            th = np.arccos(rng.random(m) * 2 - 1)
            p = np.stack([r * np.sin(th) * np.cos(phi), r * np.sin(th) * np.sin(phi), r * np.cos(th)], axis=1)
        else:
            u = rng.random(m)
            # invert 1 - (1 + x) e^-x = u by Newton from x = -ln(1-u) + 1
            x = -np.log1p(-u) + 1.0
            for _ in range(30):
                f = 1 - (1 + x) * np.exp(-x) - u
                x = np.maximum(x - f / (x * np.exp(-x) + 1e-300), 1e-12)
            Rr = comp.scale * x
            zz = comp.z0 * np.arctanh(np.clip(2 * rng.random(m) - 1, -1 + 1e-15, 1 - 1e-15))
            phi = rng.random(m) * 2 * np.pi
            p = np.stack([Rr * np.cos(phi), Rr * np.sin(phi), zz], axis=1)
        rr = np.sqrt((p * p).sum(1))
        p = p[(rr < rmax) & (rr > 0)]
        k = min(len(p), n - got)
        out[got:got + k] = p[:k]
        got += k
    return out


def build_model(comps, seed=1, level=6, fg_nbin=256, outer_frac=0.980296, inner_frac=9.80296e-5,
                torbit_fac=5.0, f_orb=0.0314, f_cc=0.25, n_override=None):
    """Builds a synthetic model; `comps` are Components, N per component in comp.n."""
    rng = np.random.default_rng(seed)
    params, rmax, torbit_fac = make_params(comps, fg_nbin=fg_nbin, level=level, outer_frac=outer_frac,
                                           inner_frac=inner_frac, torbit_fac=torbit_fac, f_orb=f_orb, f_cc=f_cc)
    lib = _geo()
    potobj = _Potential(comps)
    N = params.FG_Nbin
    nodes = params.FG_Rmin * (params.FG_Fac ** np.arange(N) - 1.0)
    Zg, Rg = np.meshgrid(nodes, nodes, indexing="ij")  # [iz, iR]
    pot, aR, az = potobj.evaluate(Rg, Zg)
    pot = np.ascontiguousarray(pot.ravel())
    dpotdr = np.ascontiguousarray(aR.ravel())
    dpotdz = np.ascontiguousarray(az.ravel())
    # streaming velocity tables
    vc = np.sqrt(np.maximum(Rg * -aR, 0))
    vstream = {1: np.zeros(N * N), 2: np.zeros(N * N), 3: np.zeros(N * N)}
    for c in comps:
        if c.kind == "disk":
            vstream[2] = np.ascontiguousarray((0.7 * vc).ravel())
    # density geometry
    L = params.DG_MaxLevel
    nb = 1 << L
    ns = ((1 << (2 + 2 * L)) - 1) // 3
    dist = np.zeros(ns)
    cellsize = np.zeros(nb * nb)
    cellvol = np.zeros(nb * nb)
    lib.galic_density_geometry(L, params.DG_Rmin, params.DG_Fac, _ffi.dptr(dist), _ffi.dptr(cellsize),
                               _ffi.dptr(cellvol))
    edges = params.DG_Rmin * (params.DG_Fac ** np.arange(nb + 1) - 1.0)
    cen = 0.5 * (edges[:-1] + edges[1:])
    Zc, Rc = np.meshgrid(cen, cen, indexing="ij")
    targets = {}
    pc, aRc, azc = potobj.evaluate(Rc, Zc)
    vcc = np.sqrt(np.maximum(Rc * -aRc, 0))
    for c in comps:
        t = TYPE_OF[c.kind]
        mt = cellvol.reshape(nb, nb) * _density(c, Rc, Zc)
        mt *= c.mass / mt.sum()
        vs = 0.7 * vcc if c.kind == "disk" else np.zeros_like(Rc)
        d = _disp_rtp(c, potobj, Rc, Zc, vs)
        d = [np.maximum(x, params.LowerDispLimit) for x in d]
        dgs = _smooth(mt.ravel(), L)
        egs = _smooth(mt.ravel(), L)
        egr = _smooth((mt * d[0]).ravel(), L)
        egt = _smooth((mt * d[1]).ravel(), L)
        egp = _smooth((mt * d[2]).ravel(), L)
        egq = _smooth((mt * d[3]).ravel(), L)
        targets[t] = (dgs, egs, egr, egt, egp, egq)
    # particles
    P, V, Mm, T, VE, TY, TG = [], [], [], [], [], [], []
    for c in comps:
        t = TYPE_OF[c.kind]
        n = c.n if n_override is None else n_override.get(c.kind, c.n)
        x = _sample_positions(c, n, rng, rmax)
        R = np.sqrt(x[:, 0] ** 2 + x[:, 1] ** 2)
        z = x[:, 2]
        r = np.sqrt(R * R + z * z)
        ph, aRp, azp = potobj.evaluate(R, z)
        vesc = np.sqrt(-2.0 * ph)
        amag = np.sqrt(aRp ** 2 + azp ** 2)
        tint = torbit_fac * 2 * np.pi * r / np.sqrt(r * amag)
        vs = 0.7 * np.sqrt(np.maximum(R * -aRp, 0)) if c.kind == "disk" else np.zeros(n)
        d = _disp_rtp(c, potobj, R, z, vs)
        d = [np.maximum(np.broadcast_to(q, (n,)), params.LowerDispLimit) for q in d]
        s_r, s_t, s_p = np.sqrt(d[0]), np.sqrt(d[1]), np.sqrt(d[2])
        vel = np.zeros((n, 3))
        todo = np.arange(n)
        phi = np.arctan2(x[:, 1], x[:, 0])
        th = np.arccos(np.clip(z / r, -1, 1))
        for _ in range(200):
            if len(todo) == 0:
                break
            vr = rng.normal(0, 1, len(todo)) * s_r[todo]
            vt = rng.normal(0, 1, len(todo)) * s_t[todo]
            vp = rng.normal(0, 1, len(todo)) * s_p[todo] + vs[todo]
            st, ct, sp, cp = np.sin(th[todo]), np.cos(th[todo]), np.sin(phi[todo]), np.cos(phi[todo])
            v = (vr[:, None] * np.stack([st * cp, st * sp, ct], 1) +
                 vt[:, None] * np.stack([-ct * cp, -ct * sp, st], 1) +
                 vp[:, None] * np.stack([-sp, cp, np.zeros_like(sp)], 1))
            ok = np.sqrt((v * v).sum(1)) < params.MaxVelInUnitsVesc * vesc[todo]
            vel[todo[ok]] = v[ok]
            todo = todo[~ok]
        if len(todo):  # pathological: give the remainder a cold circular-ish start
            vel[todo] = 0.0
        P.append(x)
        V.append(vel)
        Mm.append(np.full(n, c.mass / n))
        T.append(tint)
        VE.append(vesc)
        TY.append(np.full(n, t, dtype=np.int32))
        TG.append(np.stack(d, 1))
        params.NType[t] = n
    model = Model(params=params, pot=pot, dpotdr=dpotdr, dpotdz=dpotdz, vstream=vstream, cellsize=cellsize,
                  dgs_distance=dist, targets=targets,
                  pos=np.ascontiguousarray(np.concatenate(P)), vel=np.ascontiguousarray(np.concatenate(V)),
                  mass=np.ascontiguousarray(np.concatenate(Mm)), tint=np.ascontiguousarray(np.concatenate(T)),
                  vesc=np.ascontiguousarray(np.concatenate(VE)),
                  ptype=np.ascontiguousarray(np.concatenate(TY)),
                  ptargets=np.ascontiguousarray(np.concatenate(TG)),
                  meta={"rmax": rmax, "seed": seed, "components": [c.__dict__ for c in comps]})
    return model


# ------------------------------------------------------------------ named configurations

def fill_sample(comps, counts, rmax, seed=7):
    """Mass particles of the tree force-grid fill (grid.c:662-678): counts[k]
    positions drawn from the density of comps[k], in the reference's P order
    (halo, disk, bulge), with P[].Mass = component mass / count.  Returns
    (pos[n, 3], mass[n])."""
    rng = np.random.default_rng(seed)
    order = sorted(range(len(comps)), key=lambda k: TYPE_OF[comps[k].kind])
    pos, mass = [], []
    for k in order:
        n = int(counts[k])
        if n <= 0:
            continue
        pos.append(_sample_positions(comps[k], n, rng, rmax))
        mass.append(np.full(n, comps[k].mass / n))
    return np.concatenate(pos), np.concatenate(mass)


def config_ensemble(count=64, seed=4, n_min=10000, n_max=1000000, level=6):
    """Batched ensemble: `count` Hernquist halos (M = 100) with N log-uniform in
    [n_min, n_max], scale a uniform in [10, 50] kpc and anisotropy beta uniform
    in [-0.5, 0.5] (TypeOfHaloVelocityStructure 1), each with its own 64x64
    response grid (DG level 6) and 256^2 force grid; all drawn from `seed`."""
    rng = np.random.default_rng(seed)
    n = np.exp(rng.uniform(np.log(n_min), np.log(n_max), count)).astype(int)
    a = rng.uniform(10.0, 50.0, count)
    beta = rng.uniform(-0.5, 0.5, count)
    return [build_model([Component("halo", 100.0, float(a[k]), int(n[k]), beta=float(beta[k]), tovs=1)],
                        seed=seed * 1000 + k, level=level) for k in range(count)]


def config_halo(n=100000, seed=1, level=6):
    """Plain method: Hernquist M=100, a=30 kpc, isotropic; 64x64 (R,|z|) response grid (DG level 6)
    from 0.01a to 100a; 256x256 force grid; TorbitFac 5, ~200 steps/orbit."""
    return build_model([Component("halo", 100.0, 30.0, n, tovs=0)], seed=seed, level=level)


def config_halo_disk(n_halo=1000000, n_disk=200000, seed=2, level=7):
    """Halo (M=95, a=30) + exponential disk (M=5, h=3.5, z0=0.7, sigma_R/sigma_z = 1);
    128x128 response grid (DG level 7) to R = 20 h = 70 kpc.  The inner edge uses
    InnermostBinEnclosedMassFraction = 1e-7 (Model_H1.param): with the 0.01 a edge the
    256-bin force-grid spacing iteration of grid.c:429-443 has no root above 1."""
    # outer enclosed-mass fraction of the Hernquist halo at R = 70 kpc (grid.c:334-336)
    f = (70.0 / (30.0 + 70.0)) ** 2
    return build_model([Component("halo", 95.0, 30.0, n_halo, tovs=0),
                        Component("disk", 5.0, 3.5, n_disk, z0=0.7, tovs=3)],
                       seed=seed, level=level, outer_frac=f, inner_frac=1e-7)


def config_composite(n_halo=3000000, n_disk=700000, n_bulge=300000, seed=3, level=7):
    """Halo (beta = 0.2) + disk (h=3.5, z0=0.7) + Hernquist bulge (M=1.5, a=1)."""
    return build_model([Component("halo", 93.5, 30.0, n_halo, beta=0.2, tovs=1),
                        Component("disk", 5.0, 3.5, n_disk, z0=0.7, tovs=3),
                        Component("bulge", 1.5, 1.0, n_bulge, tovs=0)],
                       seed=seed, level=level)
