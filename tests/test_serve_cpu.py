"""The serving loop's host logic (hartreefock_b200.serve) with a stand-in
runner: admission in arrival order against the HBM budget, at most `slots`
jobs at once, refusal of jobs above the whole budget, and the synthetic
request stream's mix."""
import threading
import time

import numpy as np
import pytest

from hartreefock_b200 import molecules, serve
from hartreefock_b200.engine import HfgError


class Recorder:
    """Runner that sleeps a little and records the device bytes in use."""

    def __init__(self, server_ref):
        self.server_ref = server_ref
        self.lock = threading.Lock()
        self.starts = []
        self.max_in_use = 0

    def __call__(self, job):
        s = self.server_ref[0]
        with self.lock:
            self.starts.append(job.id)
            self.max_in_use = max(self.max_in_use, s._in_use)
        time.sleep(0.02)
        return {"energy": -float(job.id), "converged": True}


def _water(k):
    Z, xyz = molecules.water_cluster(k, seed=k)
    return list(Z), xyz


def test_admission_respects_budget_slots_and_order():
    sizes = [serve.footprint_bytes(*_water(k), "6-31g") for k in (1, 2, 3)]
    budget = sizes[2] + sizes[1]  # the two largest fit together, not three
    ref = [None]
    rec = Recorder(ref)
    with serve.Server(slots=4, hbm_budget=budget, runner=rec) as s:
        ref[0] = s
        jobs = [s.submit(*_water(1 + i % 3), "6-31g") for i in range(12)]
        s.drain(timeout=30)
        assert all(j.wait() == {"energy": -float(j.id), "converged": True} for j in jobs)
    assert rec.starts == sorted(rec.starts)  # arrival order
    assert rec.max_in_use <= budget and s.peak_bytes <= budget
    assert 2 <= s.peak_running <= 4
    assert all(j.t_submit <= j.t_start <= j.t_end for j in jobs)


def test_slots_bound_concurrency():
    ref = [None]
    rec = Recorder(ref)
    with serve.Server(slots=3, hbm_budget=1 << 40, runner=rec) as s:
        ref[0] = s
        jobs = [s.submit(*_water(1), "sto-3g") for _ in range(10)]
        s.drain(timeout=30)
    assert s.peak_running == 3
    assert len(s.finished) == 10 and all(j.done for j in jobs)


def test_job_above_budget_is_refused():
    with serve.Server(slots=2, hbm_budget=1 << 20, runner=lambda j: {}) as s:
        j = s.submit(*_water(2), "6-31g*")
        with pytest.raises(HfgError) as e:
            j.wait(5)
        assert e.value.status == serve.HFG_OOM_BUDGET


def test_runner_errors_reach_the_caller_and_free_the_slot():
    def runner(job):
        if job.id == 0:
            raise RuntimeError("boom")
        return {"energy": 1.0}

    with serve.Server(slots=1, hbm_budget=1 << 40, runner=runner) as s:
        a = s.submit(*_water(1), "sto-3g")
        b = s.submit(*_water(1), "sto-3g")
        with pytest.raises(RuntimeError):
            a.wait(5)
        assert b.wait(5) == {"energy": 1.0}


def test_footprint_grows_with_size():
    a = serve.footprint_bytes(*_water(2), "6-31g")
    b = serve.footprint_bytes(*_water(8), "6-31g")
    c = serve.footprint_bytes(*_water(8), "6-31+g**")
    assert a < b < c


def test_request_stream_mix():
    jobs = serve.draw_jobs(200, seed=3)
    uhf = sum(j[3] for j in jobs)
    assert 20 <= uhf <= 60
    assert {j[2] for j in jobs} == set(serve.SERVE_BASES)
    from hartreefock_b200.basis_io import shell_table
    n = np.array([shell_table(Z, xyz, b).nbf for Z, xyz, b, u in jobs if not u])
    assert n.min() >= 5 and n.max() <= 700
    assert np.median(n) < 150  # log-uniform: most jobs are small


def test_poisson_stream_summary():
    with serve.Server(slots=4, hbm_budget=1 << 40, runner=lambda j: {"energy": 0.0}) as s:
        handles, summ = serve.poisson_stream(s, serve.draw_jobs(20, seed=1, nbf_range=(5, 60)), rate=200.0, seed=2)
    assert summ["jobs"] == 20 and summ["failed"] == 0
    assert summ["p50_ms"] <= summ["p99_ms"]
    assert summ["jobs_per_s"] > 0
