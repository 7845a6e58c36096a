"""Windows of optimisation repetitions (galic_optimize_reps): the loop body of
main.c:94-100 run `reps` times, with the old and trial orbits of a window of
repetitions integrated in one launch and the repetitions then evaluated,
accepted and committed in order.

* The result equals `reps` calls of galic_optimize_rep bit for bit, in both
  forms, whether the work runs as one window or many (window_bytes), and
  when the particle sequence wraps so that a particle is optimised twice
  (the window ends before the repeat).
* Against the restatement (oracle/galic_oracle.c) repeating its single
  repetition, main.c:120-146's cycling through a permutation: the same
  velocities, counters, orbit counts and merit values.
"""
import numpy as np
import pytest

from galic_b200 import GALIC_FORM_FP32, GALIC_FORM_FP64, Context, GalicError, synth
from oracle_lib import Oracle

pytestmark = pytest.mark.gpu

FIT_TOL = 1e-10
FIT_ATOL = 1e-14


def cycling_lists(n, count, reps, seed):
    """optimize_some_particles (main.c:120-146): count particles per repetition
    taken in permutation order, wrapping around at the end."""
    perm = np.random.default_rng(seed).permutation(n)
    pos = (np.arange(reps * count) % n)
    return perm[pos].reshape(reps, count).astype(np.int32)


def state(ctx, present):
    vel, orbits, vdisp = ctx.particles()
    resp = np.stack([ctx.response(t, w) for t in present for w in range(10)])
    return vel, orbits, vdisp, resp, ctx.fit(), ctx.counters()


@pytest.mark.parametrize("form", [GALIC_FORM_FP64, GALIC_FORM_FP32], ids=["fp64", "fp32"])
def test_windows_equal_sequential_repetitions(form):
    m = synth.config_halo_disk(n_halo=1500, n_disk=500, level=6, seed=51)
    present = (1, 2)
    lists = cycling_lists(m.n, 90, 30, 3)  # 2700 slots over 2000 particles: wraps once
    results = []
    for mode in ("sequential", "one_call", "small_windows"):
        with Context(m.params) as ctx:
            ctx.load_model(m)
            ctx.calc_all_response_fields(form)
            if mode == "sequential":
                for r in range(len(lists)):
                    ctx.optimize_rep(lists[r], 99, 1000 + r, form)
            elif mode == "one_call":
                ctx.optimize_reps(lists, 99, 1000, form)
            else:
                # about three repetitions per window
                ctx.optimize_reps(lists, 99, 1000, form, window_bytes=3 * 90 * 2 * 5 * 4096 * 8 + 1)
            results.append(state(ctx, present))
    a = results[0]
    assert a[5][1].sum() > 0  # some proposals accepted
    for b in results[1:]:
        for x, y in zip(a[:5], b[:5]):
            assert np.array_equal(x, y)
        assert np.array_equal(a[5][0], b[5][0]) and np.array_equal(a[5][1], b[5][1])


def test_windows_match_oracle_repetitions():
    m = synth.config_composite(n_halo=600, n_disk=300, n_bulge=200, level=5, seed=52)
    present = (1, 2, 3)
    lists = cycling_lists(m.n, 40, 40, 4)  # wraps once
    o = Oracle(m.params, use_libm=False)
    o.load_model(m)
    assert o.calc_all() == 0
    for r in range(len(lists)):
        assert o.optimize_rep(lists[r], 7, 50 + r) == 0
    with Context(m.params) as ctx:
        ctx.load_model(m)
        ctx.calc_all_response_fields()
        ctx.optimize_reps(lists, 7, 50)
        vel, orbits, vdisp = ctx.particles()
        ov, oo, od = o.particles()
        assert np.array_equal(vel, ov)
        assert np.array_equal(orbits, oo)
        assert np.array_equal(vdisp, od)
        tr, ch = ctx.counters()
        otr, och = o.counters()
        assert np.array_equal(tr, otr) and np.array_equal(ch, och)
        f, g = ctx.fit()[list(present), :5], o.fit()[list(present), :5]
        assert np.all(np.abs(f - g) <= FIT_TOL * np.abs(g) + FIT_ATOL)


def test_invalid_windows_rejected():
    m = synth.config_halo(n=64, level=5, seed=53)
    with Context(m.params) as ctx:
        ctx.load_model(m)
        with pytest.raises(GalicError) as e:
            ctx.optimize_reps(np.array([[1, 2]]), 1, 0)  # before any response
        assert e.value.status == 9
        ctx.calc_all_response_fields()
        for bad in ([[1, 1]], [[0, 1], [-1, 2]], [[0, 64]]):
            with pytest.raises(GalicError) as e:
                ctx.optimize_reps(np.array(bad), 1, 0)
            assert e.value.status == 1
        ctx.optimize_reps(np.zeros((3, 0), dtype=np.int32), 1, 0)


def test_windows_report_the_fit_after_every_repetition():
    """fits=True returns the galic_get_fit values after each repetition: the
    same as reading the fit after each galic_optimize_rep call."""
    m = synth.config_halo_disk(n_halo=800, n_disk=300, level=5, seed=54)
    lists = cycling_lists(m.n, 60, 25, 5)
    want = []
    with Context(m.params) as ctx:
        ctx.load_model(m)
        ctx.calc_all_response_fields()
        for r in range(len(lists)):
            ctx.optimize_rep(lists[r], 3, 10 + r)
            want.append(ctx.fit())
    with Context(m.params) as ctx:
        ctx.load_model(m)
        ctx.calc_all_response_fields()
        got = ctx.optimize_reps(lists, 3, 10, window_bytes=4 * 60 * 2 * 5 * 1024 * 8 + 1, fits=True)
    assert got.shape == (len(lists), 4, 7)
    assert np.array_equal(got, np.stack(want), equal_nan=True)
