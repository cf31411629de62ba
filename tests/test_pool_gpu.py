"""The native serving pool (hfg_pool_*, C ABI) on the device: results the
same alone and in the mix, arrival-order admission against the budget,
refusal of a job above the whole budget, and cancellation / timeouts that
stop a job between SCF iterations (HartreeFockAlgorithm::terminate,
HartreeFockAlgorithm.cpp:142,159,187) without disturbing the others."""
import time

import pytest

from hartreefock_b200 import engine as E
from hartreefock_b200 import molecules, scf, serve

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("mixed,tol", [(True, 1e-6), (False, 1e-8)])
def test_native_results_same_alone_and_in_the_mix(mixed, tol):
    jobs = serve.draw_jobs(10, seed=11, nbf_range=(5, 80))
    with serve.NativeServer(slots=4, hbm_budget=8 << 30, mixed=mixed) as s:
        handles, summ = serve.poisson_stream(s, jobs, rate=0.0)
        assert summ["failed"] == 0 and summ["peak_running"] > 1
        for h, (Z, xyz, basis, uhf) in zip(handles, jobs):
            r = h.wait()
            assert r["converged"], (h.id, basis, uhf)
            kw = dict(s.defaults, **(serve.UHF_KW if uhf else serve.RHF_KW))
            alone = scf.run_scf(Z, xyz, basis, unrestricted=uhf, want_density=False, **kw)
            assert abs(r["energy"] - alone["energy"]) <= tol, (h.id, basis, uhf, r["energy"], alone["energy"])


def _long_job():
    # plain FP64 builds to the reference's thresholds: a few seconds of SCF
    Z, xyz = molecules.water_cluster(16, seed=0)
    return Z, xyz, "6-31g*"


def test_cancel_running_and_queued_jobs():
    Z, xyz, basis = _long_job()
    with serve.NativeServer(slots=1, hbm_budget=16 << 30, mixed=False,
                            scf_kwargs=dict(stop_at_precision_test=False, max_iterations=3000)) as s:
        a = s.submit(Z, xyz, basis, **serve.RHF_KW)
        b = s.submit(*molecules.water_cluster(1, seed=0), "6-31g", **serve.RHF_KW)
        deadline = time.time() + 120
        while a.poll() != serve.JOB_RUNNING and time.time() < deadline:
            time.sleep(0.01)
        assert a.poll() == serve.JOB_RUNNING
        assert b.poll() == serve.JOB_QUEUED  # one slot: b waits behind a
        b.cancel()
        assert b.poll() == serve.JOB_CANCELLED
        time.sleep(0.5)  # a few SCF iterations
        t0 = time.time()
        a.cancel()
        with pytest.raises(E.HfgError):
            a.wait(timeout=60)
        assert a.info.state == serve.JOB_CANCELLED and a.info.status == 6  # HFG_CANCELLED
        assert time.time() - t0 < 30  # stopped between iterations, not at the end
        assert not a.result["converged"]
        # the pool keeps serving after a cancellation
        c = s.submit(*molecules.water_cluster(1, seed=0), "6-31g", **serve.RHF_KW)
        assert c.wait(timeout=120)["converged"]


def test_timeout_ends_a_job():
    Z, xyz, basis = _long_job()
    with serve.NativeServer(slots=1, hbm_budget=16 << 30, mixed=False,
                            scf_kwargs=dict(stop_at_precision_test=False, max_iterations=3000)) as s:
        a = s.submit(Z, xyz, basis, timeout_s=0.5, **serve.RHF_KW)
        with pytest.raises(E.HfgError):
            a.wait(timeout=120)
        assert a.info.state == serve.JOB_TIMEOUT and a.info.status == 5  # HFG_TIMEOUT


def test_job_above_the_budget_is_refused():
    Z, xyz = molecules.water_cluster(8, seed=0)
    with serve.NativeServer(slots=2, hbm_budget=1 << 20) as s:
        with pytest.raises(E.HfgError) as ei:
            s.submit(Z, xyz, "6-31g*", **serve.RHF_KW)
        assert ei.value.status == 3  # HFG_OOM_BUDGET
