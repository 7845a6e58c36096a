"""Benchmark of GALIC's orbit-response hot path on B200.

One step = one calc_all_response_fields pass (main.c:151-246 + calc_global_fit
main.c:251-362) over a whole seeded synthetic model of the halo + disk shape
(Hernquist halo M=95, a=30 kpc, N=1e6; exponential disk M=5, h=3.5 kpc,
z0=0.7 kpc, N=2e5; 128x128 response grid; 256x256 force grid): every
particle's orbit is integrated for Tint and binned into the per-type response
grids, then the merit function is evaluated.  The metric is orbit-steps/s
(one step = one iteration of orbit_response.c:211-458).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

Under torchrun every rank runs its own model (weak scaling: models are
independent), rank 0 prints one JSON line.  --impl reference times GALIC's
own C (oracle/_ref/libgalic_ref.so, else the C restatement) on the host cores.
"""
import argparse
import json
import multiprocessing as mp
import os
import statistics
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "orbit-steps/s (FP32 batched vs FP64 plain, same χ²); p50/p99 model latency"
FLOP_PER_STEP = 365  # algorithmic FP ops per orbit-step (orbit_response.c:211-458 and callees)
# DRAM bytes per orbit of the orbit kernels (ncu, one launch at 0.1 of the
# workload's particles; the count scales with the orbits: particle state in,
# orbit counts out, the grids and tables stay in L2)
KERNEL_DRAM_BYTES_PER_ORBIT = {"k_calc_all_fp64": (12.605952e6 + 0.0) / 120_000,
                               "k_calc_all_fp32": (16.947712e6 + 0.0) / 120_000}
REF_BUILD = "-O3 -march=native (its Makefile.template flags), one single-rank process per host core"
WORKLOAD = "halo+disk: Hernquist halo M=95 a=30 N=1e6 + exp disk M=5 h=3.5 z0=0.7 N=2e5, 128x128 DG/EG, 256^2 FG"


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=3)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--form", default="fp64", choices=["fp64", "fp32"],
                    help="form of the headline value (default: the FP64 drop-in, the reference's precision); "
                         "the other form is measured beside it")
    ap.add_argument("--scale", type=float, default=1.0, help="fraction of the workload's particle count")
    ap.add_argument("--cpu-seconds", type=float, default=12.0)
    ap.add_argument("--ensemble-models", type=int, default=64, help="models of the batched ensemble (0: skip)")
    ap.add_argument("--mode", default="replicas", choices=["replicas", "sharded"],
                    help="N>1: independent models per GPU (weak scaling) or one model sharded over the GPUs "
                         "with an exact int64 allreduce of the response accumulators (strong scaling)")
    ap.add_argument("--serve-requests", type=int, default=24,
                    help="requests of the serving stream measured (a prefix of its 500; 0: skip)")
    ap.add_argument("--serve-gap", type=float, default=0.5, help="mean Poisson gap between requests, s")
    ap.add_argument("--serve-scale", type=float, default=1.0, help="particle-count factor of the requests")
    ap.add_argument("--serve-workers", type=int, default=16, help="concurrent jobs of the serving loop")
    ap.add_argument("--serve-hbm-fraction", type=float, default=0.5,
                    help="share of the free HBM the serving loop may hold for its jobs")
    ap.add_argument("--construction", default="halo", choices=["halo", "composite", "none"],
                    help="full model construction measured in the bench line (calc_all + iterations x "
                         "repetitions, both forms); with --row construction it is the one measured")
    ap.add_argument("--construction-scale", type=float, default=1.0)
    ap.add_argument("--construction-window-gib", type=float, default=0.0,
                    help="byte budget of a window of repetitions (0: 32 GiB at level 7, 16 GiB below)")
    ap.add_argument("--row", default="all",
                    choices=["all", "calc_all", "construction", "serving", "fill", "sampling", "jeans", "particles"],
                    help="one secondary measurement alone on this workload (a diagnostic line for profiling, "
                         "not the bench line)")
    return ap.parse_args()


def build_workload(scale, seed):
    from galic_b200 import synth

    nh = max(int(1_000_000 * scale), 40)
    nd = max(int(200_000 * scale), 20)
    return synth.config_halo_disk(n_halo=nh, n_disk=nd, level=7, seed=seed)


# ------------------------------------------------------------------ CPU side


def _cpu_worker(args):
    """Integrates orbits of one chunk with GALIC's own C (or the restatement)."""
    arrays, idx, seconds, kind = args
    # GALIC's C prints its energy-drift warnings on stdout; this worker's copy
    # goes to /dev/null so that the bench's stdout stays one JSON line
    os.dup2(os.open(os.devnull, os.O_WRONLY), 1)
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    sys.path.insert(0, os.path.join(ROOT, "tests", "golden"))
    import oracle_lib
    from make_golden import model_from_arrays

    m = model_from_arrays(arrays)
    # the timed runner is GALIC's C with its own -O3 -march=native flags
    # (the parity build has contraction off and is slower)
    runner = (oracle_lib.Reference(m.params, fast=oracle_lib.reference_fast_available()) if kind == "reference"
              else oracle_lib.Oracle(m.params, use_libm=True))
    runner.load_model(m, particles=False)
    done = []
    t0 = time.perf_counter()
    for i in idx:
        runner.orbit_mod(m.pos[i], m.vel[i], m.mass[i], m.tint[i], m.ptype[i])
        done.append(i)
        if time.perf_counter() - t0 > seconds:
            break
    dt = time.perf_counter() - t0
    # step counts: the restatement with glibc math follows the parity build's
    # trajectory bit for bit and returns its step count (the -O3 build's
    # contracted arithmetic moves trajectories only in the last bits)
    counter = oracle_lib.Oracle(m.params, use_libm=True)
    counter.load_model(m, particles=False)
    steps = 0
    for i in done:
        steps += int(counter.orbit_mod(m.pos[i], m.vel[i], m.mass[i], m.tint[i], m.ptype[i])[7][0])
    return steps, dt, len(done)


def cpu_orbit_steps_per_s(model, seconds, cores=None):
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    sys.path.insert(0, os.path.join(ROOT, "tests", "golden"))
    import oracle_lib
    from make_golden import model_arrays

    kind = "reference" if oracle_lib.reference_available() else "port"
    cores = cores or os.cpu_count() or 1
    arrays = model_arrays(model)
    rng = np.random.default_rng(123)
    perm = rng.permutation(model.n)
    chunks = [perm[k::cores][:20000] for k in range(cores)]
    ctx = mp.get_context("spawn")
    with ctx.Pool(cores) as pool:
        res = pool.map(_cpu_worker, [(arrays, c, seconds, kind) for c in chunks])
    steps = sum(r[0] for r in res)
    wall = max(r[1] for r in res)
    orbits = sum(r[2] for r in res)
    return steps / wall, kind, cores, orbits, steps


FILL_FLOP_PER_INTERACTION = 19  # forcetree_walk.c:156-196: 3 sub, r2 (5), sqrt, 2 div, r2*r, 4 mul-add pairs
FILL_FLOP_PER_TEST = 11         # forcetree_walk.c:96-109: 3 sub, r2 (5), 2 mul by theta, float len*len


def fill_workload(model):
    """Mass particles of the tree force-grid fill for the workload (one per
    model particle, drawn from the same components) and the fill parameters:
    softening 0.01 a, opening angle 0.4, TopNodeFactor 4, MultipleDomains 4."""
    from galic_b200 import forcegrid, synth

    comps = [synth.Component(**c) for c in model.meta["components"]]
    pos, mass = synth.fill_sample(comps, [c.n for c in comps], model.meta["rmax"], seed=7)
    p = model.params
    halo_a = [c for c in comps if c.kind == "halo"][0].scale
    fp = forcegrid.fill_params(p.FG_Nbin, p.FG_Rmin, p.FG_Fac, p.G, 0.01 * halo_a, 0.4, 4.0, 4)
    return fp, pos, mass


def measure_fill(model, steps, cpu, fp64_peak):
    """galic_force_grid_fill through the C ABI with host buffers: per call the
    host->device copies, key sort, tree build, walk and read-back."""
    from galic_b200 import forcegrid

    fp, pos, mass = fill_workload(model)
    forcegrid.force_grid_fill(fp, pos, mass)
    walls, walks, hosts, stats = [], [], [], None
    for _ in range(max(steps, 1)):
        t = time.perf_counter()
        out = forcegrid.force_grid_fill(fp, pos, mass)
        walls.append(time.perf_counter() - t)
        stats = out[3]
        walks.append(stats["ms_walk"])
        hosts.append(stats["ms_total"])
    walk_ms = statistics.mean(walks)
    flop = stats["interactions"] * FILL_FLOP_PER_INTERACTION + stats["node_tests"] * FILL_FLOP_PER_TEST
    achieved = flop / (walk_ms * 1e-3) / 1e12
    res = {"probes": 8 * fp.FG_Nbin ** 2, "mass_particles": len(mass), "tree_items": stats["tree_items"],
           "interactions": stats["interactions"], "node_tests": stats["node_tests"],
           "ms_per_fill_e2e": statistics.mean(walls) * 1e3, "ms_in_call": statistics.mean(hosts), "ms_walk": walk_ms,
           "roofline_walk": {"bound": "fp64", "achieved": achieved, "peak": fp64_peak, "unit": "TFLOP/s",
                             "frac": achieved / fp64_peak,
                             "flop": f"{FILL_FLOP_PER_INTERACTION}/interaction + {FILL_FLOP_PER_TEST}/opening test"}}
    if cpu:
        sys.path.insert(0, os.path.join(ROOT, "tests"))
        import oracle_lib

        t = time.perf_counter()
        oracle_lib.oracle_force_grid_fill(fp, pos, mass)
        cpu_s = time.perf_counter() - t
        res["cpu_baseline"] = {"ms_per_fill": cpu_s * 1e3, "cores": 1, "kind": "port",
                               "sample": "the whole fill, single rank (the restatement is bit-identical to the "
                                         "reference's forcedensitygrid_calculate)"}
        res["speedup_e2e_vs_cpu"] = cpu_s / statistics.mean(walls)
    return res


SAMPLE_COUNT = 100_000_000  # SampleParticleCount of every Model_*.param


def sampling_inputs(model):
    """Sampler shapes of the workload's components and seeded smooth Jeans
    tables (the synthetic workload has no Jeans solution; the tables only set
    the values the energy maps deposit, not the work)."""
    from galic_b200 import sampling

    comps = {c["kind"]: c for c in model.meta["components"]}
    h, d = comps["halo"], comps.get("disk")
    sp = sampling.sample_params(Rmax=model.meta["rmax"], Halo_A=h["scale"], Disk_Z0=d["z0"] if d else 0.0,
                                Disk_H=d["scale"] if d else 0.0, HaloBetaParameter=h.get("beta", 0.0))
    N = model.params.FG_Nbin
    iR, iz = np.meshgrid(np.arange(N), np.arange(N))
    rng = np.random.default_rng(17)
    tables = {}
    for t in (1, 2, 3):
        if model.params.MType[t] > 0:
            tables[t] = [np.ascontiguousarray(rng.uniform(1e3, 4e4) * np.exp(-iR / 60.0 - iz / 40.0) + 50.0)
                         for _ in range(5)]
    return sp, tables


def _ref_sampling_timed(params, sp, ntarget, kind, tables):
    """GALIC's own sampling function (one rank) on the host; its progress
    output goes to /dev/null so that the bench's stdout stays one JSON line."""
    os.dup2(os.open(os.devnull, os.O_WRONLY), 1)
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    import oracle_lib

    t = time.perf_counter()
    oracle_lib.reference_sampling(params, sp, ntarget, (42, 0, 0, 0), kind, tables)
    return time.perf_counter() - t


def measure_sampling(model, ctx, steps, cpu):
    """densitygrid_sample_targetresponse and calc_energy_grid_mass_maps
    through the C ABI at SampleParticleCount = 1e8 (ntarget = 1e8 + 1 per
    type, one rank): per call the windows of draws, the exact fixed-point
    bins, the smoothing and the read-back of every target stack."""
    from galic_b200 import sampling

    sp, tables = sampling_inputs(model)
    for t, tab in tables.items():
        sampling.set_dispersion(ctx, t, *tab)
    types = sorted(tables)
    ntarget = SAMPLE_COUNT + 1
    res = {"sample_count": SAMPLE_COUNT, "types": types, "tables": "seeded smooth synthetic Jeans tables"}
    for kind, fn in (("density", sampling.sample_density_targets), ("energy", sampling.sample_energy_targets)):
        fn(ctx, sp, 10000, sampling.Stream(42))
        walls = []
        for _ in range(max(steps, 1)):
            s = sampling.Stream(42)
            t = time.perf_counter()
            fn(ctx, sp, ntarget, s)
            for ty in types:
                sampling.get_targets(ctx, ty)
            walls.append(time.perf_counter() - t)
        ms = statistics.mean(walls) * 1e3
        res[kind] = {"ms_per_call_e2e": ms, "samples_per_s": len(types) * ntarget / (ms * 1e-3),
                     "draws": s.position, "gpu_launches": ctx.last_kernel_launches()}
        if cpu:
            sys.path.insert(0, os.path.join(ROOT, "tests"))
            import oracle_lib

            n_cpu = 1_000_001
            sec = oracle_lib.run_reference(_ref_sampling_timed, model.params, sp, n_cpu, kind, tables)
            cps = len(types) * n_cpu / sec
            res[kind]["cpu_baseline"] = {"samples_per_s": cps, "cores": 1, "kind": "reference",
                                         "sample": f"GALIC's own function, {n_cpu} samples per type, one rank",
                                         "ms_per_call_extrapolated": len(types) * ntarget / cps * 1e3}
            res[kind]["speedup_e2e_vs_cpu"] = res[kind]["samples_per_s"] / cps
    return res


def jeans_inputs(model):
    """Jeans parameters of the workload: disk (velocity structure 3) with
    sigma_R / sigma_z = 1 (DispersionRoverZratio 1, as the halo + disk
    configuration fixes it) and streaming parameter 0.8; halo structure 0."""
    from galic_b200 import jeans

    sp, _ = sampling_inputs(model)
    jp = jeans.jeans_params(streaming=(0.0, 0.0, 0.8, 0.0), r_over_z=(0.0, 1.0, 1.0, 1.0))
    return sp, jp


def _ref_jeans_timed(params, grid, sp, jp):
    """GALIC's own calculate_dispfield (one rank) on the host, progress output to /dev/null."""
    os.dup2(os.open(os.devnull, os.O_WRONLY), 1)
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    import oracle_lib

    t = time.perf_counter()
    oracle_lib.reference_dispfield(params, grid, sp, jp)
    return time.perf_counter() - t


def measure_jeans(model, steps, cpu):
    """calculate_dispfield through the C ABI on the workload's 256^2 force
    grid (halo: spherical and f(E, Lz) tables; disk: also the tilted method
    of lines), host copies of every table included, in a context of its own."""
    from galic_b200 import Context, jeans

    sp, jp = jeans_inputs(model)
    with Context(model.params) as c:
        c.load_model(model)
        jeans.calculate_dispfield(c, sp, jp)
        walls = []
        for _ in range(max(steps, 1)):
            t = time.perf_counter()
            jeans.calculate_dispfield(c, sp, jp)
            walls.append(time.perf_counter() - t)
        launches = c.last_kernel_launches()
    ms = statistics.mean(walls) * 1e3
    res = {"ms_per_call_e2e": ms, "fg_nbin": model.params.FG_Nbin,
           "velocity_structures": {t: model.params.TypeOfVelocityStructure[t] for t in (1, 2, 3)
                                   if model.params.NType[t] > 0},
           "parameters": "synthetic: disk DispersionRoverZratio 1 (sigma_R/sigma_z = 1), "
                         "StreamingVelocityParameter 0.8",
           "gpu_launches": launches}
    if cpu:
        sys.path.insert(0, os.path.join(ROOT, "tests"))
        import oracle_lib

        sec = oracle_lib.run_reference(_ref_jeans_timed, model.params, (model.pot, model.dpotdr, model.dpotdz), sp, jp)
        res["cpu_baseline"] = {"ms_per_call": sec * 1e3, "cores": 1, "kind": "reference",
                               "sample": "GALIC's own calculate_dispfield, the whole call, one rank"}
        res["speedup_e2e_vs_cpu"] = sec * 1e3 / ms
    return res


TORBIT_FAC = 5.0  # TorbitFac of the synthetic workload (integration time in orbital periods)


def _ref_particles_timed(params, grid, sp, tables, nscale):
    """GALIC's own initialize_particles (one rank) on the host for NType x
    nscale particles, progress output to /dev/null; seconds per particle."""
    os.dup2(os.open(os.devnull, os.O_WRONLY), 1)
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    import oracle_lib

    p = params.copy()
    for t in (1, 2, 3):
        p.NType[t] = max(int(p.NType[t] * nscale), 1 if p.NType[t] else 0)
    t = time.perf_counter()
    oracle_lib.reference_particles(p, grid, sp, TORBIT_FAC, tables, (42, 0, 0, 0))
    return (time.perf_counter() - t) / sum(p.NType[t] for t in (1, 2, 3))


def measure_particles(model, steps, cpu):
    """initialize_particles through the C ABI for the workload's 1.2e6
    particles (Jeans tables from galic_calculate_dispfield), every particle
    array and the permutation copied out, in a context of its own."""
    from galic_b200 import Context, jeans, particles, sampling

    sp, jp = jeans_inputs(model)
    with Context(model.params) as c:
        c.load_model(model)
        J = jeans.calculate_dispfield(c, sp, jp)
        particles.initialize_particles(c, sp, TORBIT_FAC, sampling.Stream(42))
        walls = []
        for _ in range(max(steps, 1)):
            s = sampling.Stream(42)
            t = time.perf_counter()
            particles.initialize_particles(c, sp, TORBIT_FAC, s)
            walls.append(time.perf_counter() - t)
        launches = c.last_kernel_launches()
    n = sum(int(model.params.NType[t]) for t in (1, 2, 3))
    ms = statistics.mean(walls) * 1e3
    res = {"particles": n, "draws": s.position, "ms_per_call_e2e": ms, "particles_per_s": n / (ms * 1e-3),
           "gpu_launches": launches}
    if cpu:
        sys.path.insert(0, os.path.join(ROOT, "tests"))
        import oracle_lib

        tables = {t: (J[t]["disp_r"], J[t]["dispz"], J[t]["dispphi"], J[t]["tilted_vR2_prime"],
                      J[t]["tilted_vz2_prime"], J[t]["vstream"]) for t in J}
        per = oracle_lib.run_reference(_ref_particles_timed, model.params, (model.pot, model.dpotdr, model.dpotdz),
                                       sp, tables, 0.02)
        res["cpu_baseline"] = {"particles_per_s": 1.0 / per, "cores": 1, "kind": "reference",
                               "sample": "GALIC's own initialize_particles for 2 % of the particle counts, one rank",
                               "ms_per_call_extrapolated": per * n * 1e3}
        res["speedup_e2e_vs_cpu"] = per * n * 1e3 / ms
    return res


def measure_ensemble(count, steps):
    """Batched ensemble: `count` Hernquist halos of uneven N advanced per
    iteration by one persistent FP32 launch replayed from a CUDA graph, tile
    variant picked by the autotuner; beside it the same models one launch
    sequence per model (galic_calc_all_response_fields each)."""
    from galic_b200 import GALIC_FORM_FP32, Context, synth
    from galic_b200.ensemble import Ensemble

    models = synth.config_ensemble(count=count)
    ctxs = []
    for m in models:
        c = Context(m.params)
        c.load_model(m)
        ctxs.append(c)
    e = Ensemble(ctxs)
    best, tune_ms = e.autotune(0.05)
    e.calc_all()  # builds and runs the graph once
    tot, kern, st = [], [], []
    for _ in range(max(steps, 1)):
        e.calc_all()
        a, b, n, nodes = e.last_timing()
        tot.append(a)
        kern.append(b)
        st.append(n)
    seq_ms = 0.0
    for c in ctxs:
        c.calc_all_response_fields(GALIC_FORM_FP32)
        seq_ms += c.last_timing()[0]
    res = {"models": count, "particles": int(sum(m.n for m in models)),
           "n_range": [int(min(m.n for m in models)), int(max(m.n for m in models))],
           "orbit_steps_per_iteration": st[-1], "ms_per_iteration": statistics.mean(tot),
           "ms_orbit_kernel": statistics.mean(kern), "value": st[-1] / (statistics.mean(tot) * 1e-3),
           "unit": "orbit-steps/s", "variant": {"index": best, "block_min_blocks": Ensemble.variants()[best]},
           "autotune_ms": [round(float(x), 3) for x in tune_ms], "graph_nodes": nodes,
           "sequential_ms_per_iteration": seq_ms,
           "speedup_vs_sequential": seq_ms / statistics.mean(tot)}
    e.close()
    for c in ctxs:
        c.close()
    return res


# ------------------------------------------------------------ model construction

# main.c:83-110 with the optimisation settings every Model_*.param ships:
# FractionToOptimizeIndependendly 0.001, IndepenentOptimizationsPerStep 100
CONSTRUCTION = {
    "halo": {"desc": "plain method: Hernquist halo M=100 a=30 N=1e5, 64x64 DG/EG, 256^2 FG, TorbitFac 5, "
                     "MaximumNumberOfSteps 9 (10 iterations) x 100 repetitions, FractionToOptimizeIndependendly 0.001",
             "n": 100_000, "iterations": 10, "reps": 100, "fraction": 0.001},
    "composite": {"desc": "composite: beta=0.2 halo N=3e6 + disk N=7e5 (h=3.5, z0=0.7) + Hernquist bulge N=3e5 "
                          "(M=1.5, a=1), 128x128 DG/EG, 256^2 FG, 20 iterations x 100 repetitions, "
                          "FractionToOptimizeIndependendly 0.001",
                  "n": 4_000_000, "iterations": 20, "reps": 100, "fraction": 0.001},
}


def construction_model(name, scale):
    from galic_b200 import synth

    if name == "halo":
        return synth.config_halo(n=max(int(100_000 * scale), 200), level=6, seed=1)
    return synth.config_composite(n_halo=max(int(3_000_000 * scale), 300), n_disk=max(int(700_000 * scale), 70),
                                  n_bulge=max(int(300_000 * scale), 30), level=7, seed=3)


def construction_lists(perm, n_per, reps, it):
    """optimize_some_particles (main.c:120-146) on one rank: the next
    reps x n_per particles of the permutation, wrapping around."""
    pos = (it * reps * n_per + np.arange(reps * n_per)) % len(perm)
    return perm[pos].reshape(reps, n_per).astype(np.int32)


def _sall(fit, types):
    """Sall = S + (Sdisp_r + Sdisp_t + Sdisp_p + Sdisp_q) / Srelfac_count per type (main.c:1270)."""
    return [float(fit[t, 0] + (fit[t, 1] + fit[t, 2] + fit[t, 3] + fit[t, 4]) / (fit[t, 6] if fit[t, 6] else 1.0))
            for t in types]


def run_construction(model, form, iterations, reps, fraction, seed=11, window_bytes=0):
    """calc_all_response_fields, then `iterations` x `reps` repetitions
    (main.c:83-110) through the C ABI — the repetitions of the whole run in
    one galic_optimize_reps call, whose windows of repetitions overlap their
    orbits with the commits — wall clock with the device synchronised at both
    ends; Sall (main.c:1270) per type after every iteration, from the fits the
    call returns per repetition."""
    import torch

    from galic_b200 import Context

    n_per = 1 + int(fraction * model.n)  # main.c:128 with NTask = 1
    perm = np.random.default_rng(seed).permutation(model.n)
    types = [t for t in (1, 2, 3) if model.params.NType[t]]
    lists = np.concatenate([construction_lists(perm, n_per, reps, it) for it in range(iterations)])
    with Context(model.params) as ctx:
        ctx.load_model(model)
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        ctx.calc_all_response_fields(form)
        steps_calc = ctx.last_orbit_steps()
        sall = [_sall(ctx.fit(), types)]
        t_calc = time.perf_counter() - t0
        fits = ctx.optimize_reps(lists, seed, 0, form, window_bytes, fits=True)
        steps_rep = ctx.last_orbit_steps()
        torch.cuda.synchronize()
        wall = time.perf_counter() - t0
        tries, changes = ctx.counters()
    sall += [_sall(fits[(it + 1) * reps - 1], types) for it in range(iterations)]
    t_rep = wall - t_calc
    return {"wall_s": wall, "calc_all_s": t_calc, "repetition_phase_s": t_rep, "particles_per_rep": n_per,
            "orbit_steps": int(steps_calc + steps_rep), "repetition_orbit_steps": int(steps_rep),
            "orbit_steps_per_s": (steps_calc + steps_rep) / wall,
            "repetition_orbit_steps_per_s": steps_rep / t_rep if t_rep > 0 else None,
            "final_sall": dict(zip(map(str, types), sall[-1])), "sall_per_iteration": sall,
            "tries": int(tries.sum()), "changes": int(changes.sum())}


def _ref_reps_timed(arrays, n_per, k_reps, fast):
    """GALIC's own repetition (init_updates, optimize x n_per, commit_updates
    with its calc_global_fit) after its calc_all_response_fields, one rank:
    seconds per repetition over k_reps repetitions."""
    os.dup2(os.open(os.devnull, os.O_WRONLY), 1)
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    sys.path.insert(0, os.path.join(ROOT, "tests", "golden"))
    import oracle_lib
    from make_golden import model_from_arrays

    m = model_from_arrays(arrays)
    ref = oracle_lib.Reference(m.params, fast=fast)
    ref.load_model(m)
    ref.calc_all()
    perm = np.random.default_rng(5).permutation(m.n)
    t = time.perf_counter()
    for r in range(k_reps):
        ref.optimize_rep(perm[r * n_per:(r + 1) * n_per], 11, r)
    return (time.perf_counter() - t) / k_reps


def cpu_construction_estimate(name, model, steps_calc, ranks=16, seconds=4.0):
    """GALIC's own C at `ranks` single-rank processes (one per host core), as
    its MPI decomposition splits the run (set_particles.c:320-330,
    main.c:128): calc_all at the measured multi-process orbit-step rate; each
    repetition as one rank's share, 1 + Fraction N / ranks particles timed on
    a sample model of the same shape (its calc_global_fit runs on every rank;
    the MPI allreduce of the grids is not counted)."""
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    sys.path.insert(0, os.path.join(ROOT, "tests", "golden"))
    import oracle_lib
    from make_golden import model_arrays

    cfg = CONSTRUCTION[name]
    rate, kind, cores, _, _ = cpu_orbit_steps_per_s(model, seconds, cores=ranks)
    n_rank = 1 + int(cfg["fraction"] * cfg["n"] / ranks)
    sample = construction_model(name, 4000.0 / cfg["n"])
    k_reps = 10
    per_rep = oracle_lib.run_reference(_ref_reps_timed, model_arrays(sample), n_rank, k_reps,
                                       oracle_lib.reference_fast_available(), timeout=1800)
    reps_total = cfg["iterations"] * cfg["reps"]
    t = steps_calc / rate + reps_total * per_rep
    return {"seconds": t, "ranks": ranks, "kind": kind, "calc_all_orbit_steps_per_s": rate,
            "seconds_per_repetition": per_rep, "particles_per_rank_per_rep": n_rank,
            "sample": (f"calc_all: {ranks} processes on this model's orbits ({seconds:.0f} s each); repetitions: "
                       f"{k_reps} of GALIC's own, {n_rank} particles each, on a {sample.n}-particle model of the "
                       f"same shape, extrapolated to {reps_total} repetitions; MPI allreduce not counted")}


def measure_construction(name, scale, cpu, window_gib=0.0):
    """Both forms of a full model construction, and GALIC's own C estimate."""
    from galic_b200 import GALIC_FORM_FP32, GALIC_FORM_FP64

    cfg = CONSTRUCTION[name]
    model = construction_model(name, scale)
    # a window's orbit launch lasts as long as its longest orbit: large windows
    # (two are held at once) — level-7 grids are 640 KiB per orbit, 32 GiB
    # hold ~6 repetitions of config 3; 16 GiB hold ~500 of config 1
    window = (32 << 30) if model.params.DG_MaxLevel >= 7 else (16 << 30)
    if window_gib > 0:
        window = int(window_gib * (1 << 30))
    res = {"config": cfg["desc"], "particles": model.n, "scale": scale}
    # warm-up: one short run of each form loads every kernel of the path
    for form in (GALIC_FORM_FP64, GALIC_FORM_FP32):
        run_construction(model, form, 1, 2, cfg["fraction"], window_bytes=window)
    for label, form in (("fp64", GALIC_FORM_FP64), ("fp32", GALIC_FORM_FP32)):
        res[label] = run_construction(model, form, cfg["iterations"], cfg["reps"], cfg["fraction"],
                                      window_bytes=window)
    a, b = res["fp64"]["final_sall"], res["fp32"]["final_sall"]
    res["fp32_vs_fp64_final_sall_rel"] = {t: abs(b[t] - a[t]) / abs(a[t]) for t in a}
    target = {t: a[t] for t in a}
    reached = None
    for k, row in enumerate(res["fp32"]["sall_per_iteration"]):
        if all(v <= target[t] * (1 + 1e-12) for t, v in zip(a, row)):
            reached = k
            break
    res["fp32_iterations_to_fp64_final_sall"] = reached
    res["wall_fp32_over_fp64"] = res["fp64"]["wall_s"] / res["fp32"]["wall_s"]
    if cpu:
        steps_calc = res["fp64"]["orbit_steps"] - res["fp64"]["repetition_orbit_steps"]
        est = cpu_construction_estimate(name, model, steps_calc)
        res["cpu_reference"] = est
        res["speedup_fp64_vs_cpu"] = est["seconds"] / res["fp64"]["wall_s"]
    return res


def serving_requests(count, seed, scale):
    """The serving stream's requests: 70% halo-only (N log-uniform in
    [1e4, 1e6] x scale), 30% halo+disk+bulge (N log-uniform in [1e5, 2e6] x
    scale, masses and scale lengths of the composite shape times a seeded
    factor in [0.5, 2])."""
    from galic_b200 import synth

    rng = np.random.default_rng(seed)
    C_ = synth.Component
    out = []
    for k in range(count):
        if rng.random() < 0.7:
            n = int(np.exp(rng.uniform(np.log(1e4 * scale), np.log(1e6 * scale))))
            m = synth.build_model([C_("halo", 100.0, float(rng.uniform(10, 50)), max(n, 200), tovs=0)],
                                  seed=seed * 1000 + k, level=6)
        else:
            n = np.exp(rng.uniform(np.log(1e5 * scale), np.log(2e6 * scale)))
            f = float(rng.uniform(0.5, 2.0))
            nh, nd, nb = (max(int(n * w), 100) for w in (0.75, 0.175, 0.075))
            m = synth.build_model([C_("halo", 93.5 * f, 30.0 * f, nh, beta=0.2, tovs=1),
                                   C_("disk", 5.0 * f, 3.5 * f, nd, z0=0.7 * f, tovs=3),
                                   C_("bulge", 1.5 * f, 1.0 * f, nb, tovs=0)], seed=seed * 1000 + k, level=6)
        out.append(m)
    return out


SERVE_SCHEDULE = {"iterations_max": 20, "reps_per_iteration": 100, "fraction_per_rep": 0.001,
                  "converge_rel": 0.01}


def measure_serving(count, mean_gap, scale, torch, workers=16, hbm_fraction=0.5):
    """The serving stream's first `count` requests (Poisson arrivals, mean gap
    `mean_gap`) through the serving loop: admission by HBM budget, concurrent
    jobs on one GPU, each job calc_all plus iterations of 100 repetitions
    (FractionToOptimizeIndependendly 0.001, repetitions in windows) until an
    iteration lowers Sall by less than 1 % (at most 20 iterations); p50/p99
    time-to-convergence (submit to done)."""
    from galic_b200 import GALIC_FORM_FP32
    from galic_b200.serving import Server

    t_build = time.perf_counter()
    models = serving_requests(count, 5, scale)
    t_build = time.perf_counter() - t_build
    rng = np.random.default_rng(6)
    arrivals = np.cumsum(rng.exponential(mean_gap, count))
    free, total = torch.cuda.mem_get_info()
    budget = int(hbm_fraction * free)
    sch = SERVE_SCHEDULE
    schedule = dict(form=GALIC_FORM_FP32, max_iterations=sch["iterations_max"],
                    reps_per_iteration=sch["reps_per_iteration"], fraction_per_rep=sch["fraction_per_rep"],
                    converge_rel=sch["converge_rel"])
    with Server(budget, workers=workers) as srv:
        t0 = time.perf_counter()
        ids = []
        for k, m in enumerate(models):
            dt = arrivals[k] - (time.perf_counter() - t0)
            if dt > 0:
                time.sleep(dt)
            ids.append(srv.submit(m, seed=1000 + k, **schedule))
        res = [srv.wait(i, timeout=3600) for i in ids]
        makespan = time.perf_counter() - t0
        st = srv.stats()
    ok = [r for r in res if r["status"] == 0]
    lat = np.array([r["t_done"] - r["t_submit"] for r in ok])
    steps = sum(r["orbit_steps"] for r in ok)
    its = np.array([r["iterations"] for r in ok])
    return {"requests": count, "completed": len(ok), "mean_gap_s": mean_gap, "particles_scale": scale,
            "arrivals": f"first {count} requests of the 500-request stream (Poisson, mean gap {mean_gap} s)",
            "n_range": [int(min(m.n for m in models)), int(max(m.n for m in models))],
            "schedule": {"calc_all": "fp32", "reps": "fp32 orbits, fp64 merit, windows of repetitions", **sch},
            "iterations_to_convergence": {"median": float(np.median(its)), "max": int(its.max())},
            "p50_s": float(np.percentile(lat, 50)), "p99_s": float(np.percentile(lat, 99)),
            "makespan_s": makespan, "orbit_steps": int(steps), "orbit_steps_per_s": steps / makespan,
            "hbm_budget_bytes": budget, "peak_bytes": st["peak_bytes"], "peak_concurrent_jobs": st["peak_running"],
            "workers": workers, "host_build_s": t_build}


def cpu_model():
    try:
        for line in open("/proc/cpuinfo"):
            if line.startswith("model name"):
                return line.split(":", 1)[1].strip()
    except OSError:
        pass
    return "unknown"


# ------------------------------------------------------------------ clocks


class ClockSampler:
    QUERY = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device):
        self.device = device
        self.proc = None
        self.path = None

    def __enter__(self):
        fd, self.path = tempfile.mkstemp(suffix=".csv")
        os.close(fd)
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--query-gpu={self.QUERY}", "--format=csv,noheader,nounits",
                                          "-lms", "200", "-i", str(self.device)], stdout=open(self.path, "w"),
                                         stderr=subprocess.DEVNULL)
        except (OSError, FileNotFoundError):
            self.proc = None
        return self

    def __exit__(self, *a):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self):
        rows = []
        try:
            for line in open(self.path):
                f = [x.strip() for x in line.split(",")]
                if len(f) >= 9:
                    rows.append(f)
        except OSError:
            pass
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unavailable"], "samples": 0}
        sm = [float(r[1]) for r in rows if r[1].replace(".", "").isdigit()]
        reasons = set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for r in rows:
            for k, n in enumerate(names):
                if r[5 + k].lower().startswith("active"):
                    reasons.add(n)
        return {"sm_mhz": statistics.median(sm) if sm else None,
                "sm_max_mhz": float(rows[0][2]) if rows[0][2].replace(".", "").isdigit() else None,
                "reasons": sorted(reasons), "samples": len(rows)}


def measured_fp32_peak(torch):
    """FP32 (SIMT, no TF32) GEMM TFLOP/s, burst best of 5: the FP32 denominator."""
    prev = torch.backends.cuda.matmul.allow_tf32
    torch.backends.cuda.matmul.allow_tf32 = False
    n = 8192
    a = torch.randn(n, n, dtype=torch.float32, device="cuda")
    b = torch.randn(n, n, dtype=torch.float32, device="cuda")
    torch.matmul(a, b)
    torch.cuda.synchronize()
    best = 0.0
    for _ in range(5):
        s, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        s.record()
        torch.matmul(a, b)
        e.record()
        torch.cuda.synchronize()
        best = max(best, 2 * n ** 3 / (s.elapsed_time(e) * 1e-3) / 1e12)
    torch.backends.cuda.matmul.allow_tf32 = prev
    del a, b
    return best


def measured_fp64_peak(torch):
    """FP64 GEMM TFLOP/s (burst, best of 5) on this GPU: the FP64 denominator."""
    n = 4096
    a = torch.randn(n, n, dtype=torch.float64, device="cuda")
    b = torch.randn(n, n, dtype=torch.float64, device="cuda")
    for _ in range(2):
        torch.matmul(a, b)
    torch.cuda.synchronize()
    best = 0.0
    for _ in range(5):
        s, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        s.record()
        torch.matmul(a, b)
        e.record()
        torch.cuda.synchronize()
        best = max(best, 2 * n ** 3 / (s.elapsed_time(e) * 1e-3) / 1e12)
    del a, b
    return best


# ------------------------------------------------------------------ arms


def workload_config(model):
    """The `config` object both arms print (identical for the same workload)."""
    return {"workload": WORKLOAD, "particles": int(model.n)}


def reference_arm(args, rank, world):
    if rank != 0:
        return
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    import oracle_lib

    from galic_b200 import synth

    # the workload's set-up geometry from the C restatement: this arm never
    # loads libgalic_cuda.so
    synth.use_geometry(oracle_lib.OracleGeometry())
    model = build_workload(args.scale, seed=2)
    per_step = max(args.cpu_seconds / 3.0, 2.0)
    vals = []
    kind = cores = None
    for k in range(args.warmup + args.steps):
        v, kind, cores, orbits, steps = cpu_orbit_steps_per_s(model, per_step)
        if k >= args.warmup:
            vals.append(v)
    value = statistics.mean(vals)
    sample = (f"{orbits} orbits of the workload per step, {cores} processes x {per_step:.1f} s, "
              f"GALIC's C built {REF_BUILD}")
    line = {"impl": "reference", "metric": METRIC, "value": value, "unit": "orbit-steps/s", "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": per_step * 1e3, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": workload_config(model), "parallelism": f"{cores} host processes",
            "cpu_baseline": {"value": value, "unit": "orbit-steps/s", "cores": cores,
                             "kind": "reference" if kind == "reference" else "port", "sample": sample,
                             "cpu": cpu_model()},
            "e2e": {"value": value, "unit": "orbit-steps/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def _bin_errors(got, want, floors):
    """Peak-relative and per-bin relative errors of `got` against `want`
    ({(type, grid): array}), over the time-averaged grids."""
    from galic_b200 import _ffi

    peak_rel = 0.0
    per_bin = {f: [] for f in floors}
    for key, a in want.items():
        if key[1] >= _ffi.GRID_MASS_I:
            continue  # the instantaneous grids do not depend on the orbit form
        b = got[key]
        peak = np.abs(a).max()
        if peak <= 0:
            continue
        d = np.abs(b - a)
        peak_rel = max(peak_rel, float(d.max() / peak))
        for f in floors:
            sel = np.abs(a) >= f * peak
            per_bin[f].append(d[sel] / np.abs(a[sel]))
    res = {"peak_relative_max": peak_rel}
    for f in floors:
        r = np.concatenate(per_bin[f])
        res[f"per_bin_relative_bins_above_{f:g}_of_peak"] = {
            "bins": int(r.size), "max": float(r.max()), "median": float(np.median(r)),
            "p99": float(np.percentile(r, 99)), "frac_within_1e-4": float(np.mean(r <= 1e-4))}
    return res


def fp32_error(ctx, model):
    """Error of the FP32-integrate / FP64-accumulate form against the FP64
    drop-in on the same pass (same initial velocities): every time-averaged
    grid of every type, per bin relative to the FP64 bin (bins above a floor
    of the grid's peak) and relative to the grid's peak, and the merit
    values.  Beside it the orbits' own sensitivity: the FP64 form against
    itself with the initial velocities perturbed by 1e-7 (relative)."""
    from galic_b200 import GALIC_FORM_FP32, GALIC_FORM_FP64, _ffi

    types = [t for t in (1, 2, 3) if model.params.NType[t]]
    floors = (1e-1, 1e-2, 1e-3)

    def grids():
        return {(t, w): ctx.response(t, w) for t in types for w in range(_ffi.GRID_COUNT)}

    ctx.calc_all_response_fields(GALIC_FORM_FP64)
    g64, f64 = grids(), ctx.fit()
    ctx.calc_all_response_fields(GALIC_FORM_FP32)
    g32, f32 = grids(), ctx.fit()
    vel = model.vel * (1 + 1e-7 * np.random.default_rng(1).standard_normal(model.vel.shape))
    ctx.set_particles(model.pos, vel, model.mass, model.tint, model.vesc, model.ptype, model.ptargets)
    ctx.calc_all_response_fields(GALIC_FORM_FP64)
    gp = grids()
    ctx.set_particles(model.pos, model.vel, model.mass, model.tint, model.vesc, model.ptype, model.ptargets)
    res = {"vs": "FP64 drop-in form on the same pass", "grids": "DG_MassLoc, EG_EgyResponse{R,T,Q,P}LocS per type"}
    res.update(_bin_errors(g32, g64, floors))
    res["fp64_sensitivity_1e-7_velocity_perturbation"] = _bin_errors(gp, g64, floors)
    fit = {}
    for t in types:
        sall64 = f64[t, 0] + (f64[t, 1] + f64[t, 2] + f64[t, 3] + f64[t, 4]) / max(f64[t, 6], 1.0)
        sall32 = f32[t, 0] + (f32[t, 1] + f32[t, 2] + f32[t, 3] + f32[t, 4]) / max(f32[t, 6], 1.0)
        fit[str(t)] = {"S_rel": float(abs(f32[t, 0] - f64[t, 0]) / abs(f64[t, 0])),
                       "Sall_rel": float(abs(sall32 - sall64) / abs(sall64))}
    res["fit_relative"] = fit
    return res


def ours_arm(args, rank, world, local_rank):
    import torch

    from galic_b200 import GALIC_FORM_FP32, GALIC_FORM_FP64, Context
    from galic_b200 import _ffi

    torch.cuda.set_device(local_rank)
    dist = None
    if world > 1:
        import datetime

        import torch.distributed as dist

        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600))
    form = GALIC_FORM_FP64 if args.form == "fp64" else GALIC_FORM_FP32
    sharded = dist is not None and args.mode == "sharded"
    model = build_workload(args.scale, seed=2 if sharded else 2 + rank)
    ctx = Context(model.params)
    ctx.load_model(model)
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device="cuda")  # > 126 MB L2

    other = GALIC_FORM_FP32 if form == GALIC_FORM_FP64 else GALIC_FORM_FP64
    def one_pass():
        if sharded:
            from galic_b200.sharding import calc_all_sharded

            calc_all_sharded(ctx, form)
        else:
            ctx.calc_all_response_fields(form)

    for _ in range(args.warmup):
        one_pass()
    torch.cuda.synchronize()
    if dist:
        dist.barrier()

    dev_ms, kern_ms, steps, launches = [], [], [], 0
    with ClockSampler(local_rank) as clocks:
        t0 = time.perf_counter()
        for _ in range(args.steps):
            flush.fill_(1.0)
            torch.cuda.synchronize()
            if sharded:
                s_ev, e_ev = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                s_ev.record()
                one_pass()
                e_ev.record()
                torch.cuda.synchronize()
                tot = s_ev.elapsed_time(e_ev)
                kern = ctx.last_timing()[1]
            else:
                one_pass()
                tot, kern = ctx.last_timing()
            dev_ms.append(tot)
            kern_ms.append(kern)
            steps.append(ctx.last_orbit_steps())
            launches += ctx.last_kernel_launches()
        torch.cuda.synchronize()
        wall = time.perf_counter() - t0
    if dist:
        dist.barrier()
    # the other form on the same model (one warm-up, then K steps), for the
    # FP32-vs-FP64 comparison the metric names
    ctx.calc_all_response_fields(other)
    other_ms, other_kern, other_steps = [], [], []
    for _ in range(args.steps):
        flush.fill_(1.0)
        torch.cuda.synchronize()
        ctx.calc_all_response_fields(other)
        tot, kern = ctx.last_timing()
        other_ms.append(tot)
        other_kern.append(kern)
        other_steps.append(ctx.last_orbit_steps())
    total_ms = sum(dev_ms)
    total_steps = sum(steps)
    # whole job: steps of all ranks over the slowest rank's device time
    if dist:
        t = torch.tensor([total_ms, float(total_steps)], dtype=torch.float64, device="cuda")
        mx = t.clone()
        dist.all_reduce(mx[:1], op=dist.ReduceOp.MAX)
        dist.all_reduce(t[1:], op=dist.ReduceOp.SUM)
        total_ms, total_steps = float(mx[0]), float(t[1])
    value = total_steps / (total_ms * 1e-3)

    # end to end through the C ABI with host buffers: upload the particle state,
    # run the pass, read back the fit and every committed grid
    e2e_s = []
    h2d = sum(a.nbytes for a in (model.pos, model.vel, model.mass, model.tint, model.vesc, model.ptype,
                                 model.ptargets))
    types = [t for t in (1, 2, 3) if model.params.NType[t]]
    d2h = 28 * 8 + len(types) * _ffi.GRID_COUNT * ctx.ngrid * 8
    # the inputs of every step sit in page-locked host memory (filled once,
    # outside the timed region), as a serving host would stage them
    pinned = []
    for a in (model.pos, model.vel, model.mass, model.tint, model.vesc, model.ptype, model.ptargets):
        t = torch.empty(a.shape, dtype=torch.float64 if a.dtype == np.float64 else torch.int32, pin_memory=True)
        t.numpy()[...] = a
        pinned.append(t.numpy())
    for _ in range(max(1, min(args.steps, 2))):
        t1 = time.perf_counter()
        ctx.set_particles(*pinned)
        one_pass()
        ctx.fit()
        for t in types:
            for w in range(_ffi.GRID_COUNT):
                ctx.response(t, w)
        e2e_s.append(time.perf_counter() - t1)
    e2e_value = (total_steps / args.steps) / statistics.mean(e2e_s)  # whole-job steps of one pass

    other_value = sum(other_steps) / (sum(other_ms) * 1e-3)
    if rank == 0:
        peak = measured_fp64_peak(torch) if form == GALIC_FORM_FP64 else measured_fp32_peak(torch)
        kern_avg = sum(kern_ms) / len(kern_ms)
        fill = measure_fill(model, args.steps, world == 1 and args.cpu_seconds > 0,
                            peak if form == GALIC_FORM_FP64 else measured_fp64_peak(torch))
        target_sampling = measure_sampling(model, ctx, args.steps, world == 1 and args.cpu_seconds > 0)
        jeans_solve = measure_jeans(model, args.steps, world == 1 and args.cpu_seconds > 0)
        init_particles = measure_particles(model, args.steps, world == 1 and args.cpu_seconds > 0)
        ensemble = measure_ensemble(args.ensemble_models, args.steps) if args.ensemble_models > 0 else None
        construction = (measure_construction(args.construction, args.construction_scale,
                                             world == 1 and args.cpu_seconds > 0)
                        if args.construction != "none" else None)
        serving = (measure_serving(args.serve_requests, args.serve_gap, args.serve_scale, torch, args.serve_workers,
                                   args.serve_hbm_fraction)
                   if args.serve_requests > 0 else None)
        achieved = steps[-1] * FLOP_PER_STEP / (kern_avg * 1e-3) / 1e12
        fp32_err = fp32_error(ctx, model)
        cpu = None
        if world == 1 and args.cpu_seconds > 0:
            v, kind, cores, orbits, st = cpu_orbit_steps_per_s(model, args.cpu_seconds)
            cpu = {"value": v, "unit": "orbit-steps/s", "cores": cores, "kind": kind,
                   "sample": f"{orbits} orbits ({st} orbit-steps) of this workload, {cores} processes, "
                             f"~{args.cpu_seconds:.0f} s each", "cpu": cpu_model()}
        fp64_form = form == GALIC_FORM_FP64
        kern_name = "k_calc_all_fp64" if fp64_form else "k_calc_all_fp32"
        traffic = KERNEL_DRAM_BYTES_PER_ORBIT.get(kern_name)
        line = {"metric": METRIC, "value": value, "unit": "orbit-steps/s", "n_gpus": world, "steps": args.steps,
                "warmup": args.warmup, "ms_per_step": total_ms / args.steps, "higher_is_better": True,
                "scaling": "strong" if sharded else "weak", "vs_baseline": None,
                "dtype": "f64" if fp64_form else "f32",
                "data": "synthetic",
                "config": workload_config(model),
                "form": ("FP64 drop-in (bit-exact per orbit to the restatement of GALIC's C)" if fp64_form
                         else "FP32-integrate / FP64-accumulate"),
                "orbit_steps_per_step": steps[-1], "l2": "flushed (256 MiB write) between steps",
                "parallelism": (f"one model sharded over {world} GPUs (int64 allreduce)" if sharded
                                else f"{world} independent models (one per GPU)"),
                "roofline": {"bound": "fp64" if fp64_form else "fp32", "achieved": achieved,
                             "peak": peak, "unit": "TFLOP/s", "frac": achieved / peak,
                             "traffic": (traffic * model.n) if traffic else None,
                             "traffic_source": ("ncu dram__bytes_read.sum + dram__bytes_write.sum of one launch at "
                                                "0.1 of the workload's particles, scaled by the orbit count "
                                                f"(profiles/{kern_name}_halo_disk.md)") if traffic else None,
                             "peak_source": ("measured FP64 GEMM (torch.matmul float64 4096^3, burst)"
                                             if fp64_form else
                                             "measured FP32 SIMT GEMM (torch.matmul float32 8192^3, TF32 off, "
                                             "burst)") + "; MEASURED_PEAKS.json has no FP32/FP64 figure",
                             "flop_per_orbit_step": FLOP_PER_STEP,
                             "kernel": kern_name,
                             "kernel_ms": kern_avg},
                "forms": {args.form: value, ("fp64" if args.form == "fp32" else "fp32"): other_value,
                          "fp32_over_fp64": (value / other_value) if args.form == "fp32" else (other_value / value),
                          "unit": "orbit-steps/s"},
                "fp32_error": fp32_err,
                "cpu_baseline": cpu,
                "force_grid_fill": fill,
                "target_sampling": target_sampling,
                "jeans": jeans_solve,
                "particle_init": init_particles,
                "ensemble": ensemble,
                "construction": construction,
                "serving": serving,
                "e2e": {"value": e2e_value, "unit": "orbit-steps/s", "h2d_bytes_per_step": h2d,
                        "d2h_bytes_per_step": d2h},
                "gpu_launches": launches,
                "clocks": clocks.summary(),
                "wall_s": wall,
                "max_energy_error": ctx.last_max_energy_error()}
        print(json.dumps(line), flush=True)
    ctx.close()
    if dist:
        dist.barrier()
        dist.destroy_process_group()


def main():
    # every context drives two streams (galic_optimize_reps overlaps the next
    # window's orbits with the current window's commits) and the serving loop
    # runs up to 16 contexts: give the process 32 hardware work queues
    # instead of the default 8, so that a stream waiting on an event does not
    # hold up the streams that share its queue (read when CUDA starts)
    os.environ.setdefault("CUDA_DEVICE_MAX_CONNECTIONS", "32")
    args = parse()
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local_rank = int(os.environ.get("LOCAL_RANK", "0"))
    if args.impl == "reference":
        reference_arm(args, rank, world)
        return
    if args.row != "all":
        row_alone(args)
        return
    ours_arm(args, rank, world, local_rank)


def row_alone(args):
    """One secondary measurement on the workload, without its CPU baseline."""
    import torch

    from galic_b200 import Context

    torch.cuda.set_device(0)
    model = build_workload(args.scale, seed=2)
    if args.row == "calc_all":
        # the orbit pass alone in the --form form (the command the orbit
        # kernels' profile summaries run)
        from galic_b200 import GALIC_FORM_FP32, GALIC_FORM_FP64

        form = GALIC_FORM_FP64 if args.form == "fp64" else GALIC_FORM_FP32
        with Context(model.params) as ctx:
            ctx.load_model(model)
            for _ in range(args.warmup):
                ctx.calc_all_response_fields(form)
            ms = []
            for _ in range(args.steps):
                ctx.calc_all_response_fields(form)
                ms.append(ctx.last_timing()[1])
            res = {"form": args.form, "particles": model.n, "orbit_steps": ctx.last_orbit_steps(),
                   "kernel_ms": statistics.mean(ms),
                   "orbit_steps_per_s": ctx.last_orbit_steps() / (statistics.mean(ms) * 1e-3),
                   "max_energy_error": ctx.last_max_energy_error()}
    elif args.row == "serving":
        res = measure_serving(args.serve_requests, args.serve_gap, args.serve_scale, torch, args.serve_workers,
                              args.serve_hbm_fraction)
    elif args.row == "construction":
        res = measure_construction(args.construction, args.construction_scale, args.cpu_seconds > 0,
                                   args.construction_window_gib)
    elif args.row == "fill":
        res = measure_fill(model, args.steps, False, measured_fp64_peak(torch))
    elif args.row == "sampling":
        with Context(model.params) as ctx:
            ctx.load_model(model)
            res = measure_sampling(model, ctx, args.steps, False)
    elif args.row == "jeans":
        res = measure_jeans(model, args.steps, False)
    else:
        res = measure_particles(model, args.steps, False)
    print(json.dumps({"row": args.row, "steps": args.steps, **res}), flush=True)


if __name__ == "__main__":
    main()
