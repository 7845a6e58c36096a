"""Serving loop (galic_server_*): jobs admitted by HBM budget, run
concurrently, each job's result identical alone and in the mix."""
import ctypes as C

import numpy as np
import pytest

from galic_b200 import GALIC_FORM_FP32, GALIC_FORM_FP64, _ffi, synth
from galic_b200.serving import Server

SCHEDULE = dict(max_iterations=2, reps_per_iteration=3, fraction_per_rep=0.003)


def small_models():
    ms = synth.config_ensemble(count=5, seed=21, n_min=2000, n_max=6000, level=5)
    C_ = synth.Component
    ms.append(synth.build_model([C_("halo", 93.5, 30.0, 3000, beta=0.2, tovs=1),
                                 C_("disk", 5.0, 3.5, 1500, z0=0.7, tovs=2),
                                 C_("bulge", 1.5, 1.0, 800, tovs=0)], seed=22, level=5))
    return ms


def test_job_bytes_grow_with_size():
    a = synth.config_ensemble(count=1, seed=1, n_min=1000, n_max=1001, level=5)[0]
    b = synth.config_ensemble(count=1, seed=1, n_min=50000, n_max=50001, level=5)[0]
    c = synth.config_ensemble(count=1, seed=1, n_min=50000, n_max=50001, level=6)[0]
    ba, bb, bc = Server.job_bytes(a), Server.job_bytes(b), Server.job_bytes(c)
    assert 0 < ba < bb < bc
    assert bb - ba >= (50000 - 1000) * 150  # particle state is resident


def test_server_argument_errors():
    lib = _ffi.load_library()
    h = C.c_void_p()
    assert lib.galic_server_create(0, 2, C.byref(h)) == 1
    assert lib.galic_server_create(1 << 30, 0, C.byref(h)) == 1
    assert lib.galic_server_submit(None, None, None) == 1


def run_all(models, workers, budget=64 << 30, seeds=None):
    with Server(budget, workers=workers) as s:
        ids = [s.submit(m, form=GALIC_FORM_FP32, seed=100 + k, want_velocities=True, **SCHEDULE)
               for k, m in enumerate(models)]
        res = [s.wait(i) for i in ids]
        st = s.stats()
    return res, st


@pytest.mark.gpu
def test_results_same_alone_and_in_the_mix():
    models = small_models()
    alone, st1 = run_all(models, workers=1)
    mixed, st4 = run_all(models, workers=4)
    assert st1["peak_running"] == 1
    assert st4["peak_running"] >= 2
    for a, b in zip(alone, mixed):
        assert a["status"] == 0 and b["status"] == 0
        assert a["iterations"] == b["iterations"] == SCHEDULE["max_iterations"]
        assert a["reps"] == b["reps"] == SCHEDULE["max_iterations"] * SCHEDULE["reps_per_iteration"]
        assert a["orbit_steps"] == b["orbit_steps"]
        assert np.array_equal(a["fit"], b["fit"])
        assert a["sall_first"] == b["sall_first"] and a["sall_last"] == b["sall_last"]
        assert np.array_equal(a["vel"], b["vel"])
        assert 0 <= b["t_submit"] <= b["t_admit"] <= b["t_first_response"] <= b["t_done"]


@pytest.mark.gpu
def test_admission_by_budget():
    models = small_models()
    biggest = max(Server.job_bytes(m, SCHEDULE["fraction_per_rep"]) for m in models)
    budget = int(2.5 * biggest)
    res, st = run_all(models, workers=6, budget=budget)
    assert all(r["status"] == 0 for r in res)
    assert st["peak_bytes"] <= budget
    assert 1 <= st["peak_running"] <= 2


@pytest.mark.gpu
def test_oversize_job_rejected_and_early_stop():
    models = small_models()[:2]
    need = Server.job_bytes(models[0], SCHEDULE["fraction_per_rep"])
    with Server(need - 1, workers=2) as s:
        r = s.wait(s.submit(models[0], **SCHEDULE))
        assert r["status"] == 5  # GALIC_ERR_BUDGET
    with Server(64 << 30, workers=2) as s:
        r = s.wait(s.submit(models[1], form=GALIC_FORM_FP64, max_iterations=5, reps_per_iteration=2,
                            fraction_per_rep=0.003, converge_rel=1.0))
        assert r["status"] == 0 and r["iterations"] == 1 and r["reps"] == 2
