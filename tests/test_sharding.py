"""One model's calc_all sharded over ranks (galic_b200.sharding).

CPU, world size 2 over gloo: the exchange of a sharded pass (galic_b200.
sharding.sharded_pass) with every rank integrating its particles rank::world
through the oracle, rounding into the 64-bit fixed-point words the CUDA path
uses, and summing the words over the group: the result equals a one-rank
pass bit for bit and the oracle's sequential calc_all to 1e-12 of each grid's
peak.
GPU (one device): ranks emulated one after another with one context each;
their accumulators summed on the device equal a one-context pass bit for bit.
"""
import datetime
import multiprocessing as mp
import os
import socket

import numpy as np
import pytest

from galic_b200 import GALIC_FORM_FP32, GALIC_FORM_FP64, Context, _ffi, synth
from galic_b200.sharding import accumulator_tensor, sharded_pass
import oracle_lib


def small_model():
    C = synth.Component
    return synth.build_model([C("halo", 95.0, 30.0, 400, tovs=0), C("disk", 5.0, 3.5, 200, z0=0.7, tovs=3)],
                             seed=31, level=5, fg_nbin=64, torbit_fac=1.0, inner_frac=1e-7, outer_frac=0.49)


# ---- the fixed-point words of fixedpoint.cuh, restated in numpy

def fx_words(v, S):
    """(H, L) with round(v 2^S) = H 2^24 + L, 0 <= L < 2^24 (elementwise)."""
    t = np.ldexp(v, S - 24)
    fh = np.floor(t)
    fl = np.rint((t - fh) * 16777216.0)
    carry = fl == 16777216.0
    fh = fh + carry
    fl = np.where(carry, 0.0, fl)
    return fh.astype(np.int64), fl.astype(np.int64)


def fx_value(H, L, S):
    return np.ldexp(H.astype(np.float64), 24 - S) + np.ldexp(L.astype(np.float64), -S)


def shifts(m):
    """One shift per (type, field) from a bound on the field's total."""
    S = np.zeros((4, 5), dtype=np.int64)
    for t in (1, 2, 3):
        bound = max(m.params.MType[t], 1e-300) * 2.0 * 1e8
        for f in range(5):
            S[t, f] = 84 - int(np.ceil(np.log2(bound)))
    return S


def shard_words(m, rank, world):
    """This rank's particles (rank::world) through the oracle, as fixed-point words
    [type][field][H | L][Ngrid]."""
    orc = oracle_lib.Oracle(m.params, use_libm=False)
    orc.load_model(m, particles=False)
    S = shifts(m)
    G = orc.ngrid
    words = np.zeros((4, 5, 2, G), dtype=np.int64)
    for i in range(rank, m.n, world):
        out = orc.orbit_mod(m.pos[i], m.vel[i], m.mass[i], m.tint[i], m.ptype[i])
        t = int(m.ptype[i])
        for f in range(5):
            H, L = fx_words(out[2 + f], int(S[t, f]))
            words[t, f, 0] += H
            words[t, f, 1] += L
    return words


def values(m, words):
    S = shifts(m)
    return np.stack([[fx_value(words[t, f, 0], words[t, f, 1], int(S[t, f])) for f in range(5)]
                     for t in range(4)])


def _rank_main(rank, world, port, arrays, q):
    import torch
    import torch.distributed as dist
    import sys
    sys.path.insert(0, os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden"))
    from make_golden import model_from_arrays

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    try:
        dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
        m = model_from_arrays(arrays)
        state = {}

        def run(r, w):
            state["acc"] = torch.from_numpy(shard_words(m, r, w).reshape(-1))

        def finish():
            state["vals"] = values(m, state["acc"].numpy().reshape(4, 5, 2, -1))

        r, w = sharded_pass(run, lambda: state["acc"], finish)
        q.put((rank, r, w, state["vals"]))
        dist.barrier()
        dist.destroy_process_group()
    except BaseException as e:  # noqa: BLE001
        q.put((rank, "error", repr(e), None))


def free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def test_sharded_pass_gloo_world2_exact():
    sys_path = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
    import sys
    sys.path.insert(0, sys_path)
    from make_golden import model_arrays

    m = small_model()
    arrays = model_arrays(m)
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, 2, port, arrays, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = {}
    for _ in range(2):
        rank, r, w, vals = q.get(timeout=300)
        assert r != "error", w
        res[rank] = (r, w, vals)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert res[0][:2] == (0, 2) and res[1][:2] == (1, 2)
    # every rank holds the same grids, equal to the one-rank pass bit for bit
    one = values(m, shard_words(m, 0, 1))
    assert np.array_equal(res[0][2], res[1][2])
    assert np.array_equal(res[0][2], one)
    # and the oracle's sequential FP64 sums (main.c:214-223) to 1e-12 of the peak
    orc = oracle_lib.Oracle(m.params, use_libm=False)
    orc.load_model(m)
    assert orc.calc_all() == 0
    for t in (1, 2):
        for f in range(5):
            want = orc.response(t, f)
            peak = np.max(np.abs(want))
            assert np.max(np.abs(one[t, f] - want)) <= 1e-12 * peak


def test_shard_arguments_rejected():
    lib = _ffi.load_library()
    assert lib.galic_calc_all_shard(None, 0, 0, 1) == 1
    assert lib.galic_calc_all_finish(None) == 1


@pytest.mark.gpu
@pytest.mark.parametrize("form", [GALIC_FORM_FP64, GALIC_FORM_FP32])
@pytest.mark.parametrize("world", [2, 3])
def test_shards_sum_to_one_pass(form, world):
    import torch

    m = synth.config_halo_disk(n_halo=6000, n_disk=1500, level=6, seed=12)
    with Context(m.params) as full:
        full.load_model(m)
        full.calc_all_response_fields(form)
        want = [full.response(t, w) for t in (1, 2) for w in range(_ffi.GRID_COUNT)]
        want_fit = full.fit()
        want_steps = full.last_orbit_steps()
    ranks = []
    for r in range(world):
        c = Context(m.params)
        c.load_model(m)
        c.calc_all_shard(form, r, world)
        ranks.append(c)
    steps = sum(c.last_orbit_steps() for c in ranks)
    total = accumulator_tensor(ranks[0])
    for c in ranks[1:]:
        total += accumulator_tensor(c)
    torch.cuda.synchronize()
    ranks[0].calc_all_finish()
    got = [ranks[0].response(t, w) for t in (1, 2) for w in range(_ffi.GRID_COUNT)]
    for g, w in zip(got, want):
        assert np.array_equal(g, w)
    assert np.array_equal(ranks[0].fit(), want_fit)
    assert steps == want_steps
    for c in ranks:
        c.close()
