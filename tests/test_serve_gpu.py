"""Serving on the device: jobs that run concurrently in the request loop
(kernels of different jobs overlapping on their own streams) give the same
converged energies as the same jobs run alone, within 1e-6 Eh for the
precision form and 1e-8 Eh for plain FP64 builds."""
import pytest

from hartreefock_b200 import scf, serve

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("mixed,tol", [(True, 1e-6), (False, 1e-8)])
def test_results_same_alone_and_in_the_mix(mixed, tol):
    jobs = serve.draw_jobs(10, seed=11, nbf_range=(5, 80))
    with serve.Server(slots=4, hbm_budget=8 << 30, mixed=mixed) as s:
        handles, summ = serve.poisson_stream(s, jobs, rate=0.0)
    assert summ["failed"] == 0 and summ["peak_running"] > 1
    for h, (Z, xyz, basis, uhf) in zip(handles, jobs):
        r = h.wait()
        assert r["converged"], (h.id, basis, uhf)
        kw = dict(s.defaults, **(serve.UHF_KW if uhf else serve.RHF_KW))
        alone = scf.run_scf(Z, xyz, basis, unrestricted=uhf, want_density=False, **kw)
        assert abs(r["energy"] - alone["energy"]) <= tol, (h.id, basis, uhf, r["energy"], alone["energy"])


def test_small_jobs_share_batched_launches():
    """With the batch lane on, small jobs (<= 60 functions) that wait in the
    queue together (at least batch_min with the same settings) run as batched
    SCFs (one Fock launch per quartet class over all of them per iteration)
    while the slots keep taking the queue's head; every result converges to
    the energy of the same job run alone (the batched SCF stops on the
    reference's test, the driver's runs on the precision form's rule: they
    agree within 1e-6 Eh) and the batched jobs say so."""
    jobs = serve.draw_jobs(24, seed=3, nbf_range=(5, 120))
    with serve.Server(slots=2, hbm_budget=8 << 30, mixed=True, batch_nbf=60, batch_min=3) as s:
        handles, summ = serve.poisson_stream(s, jobs, rate=0.0)
        batches = list(s.batches)
    assert summ["failed"] == 0
    assert batches and min(batches) >= 3 and summ["batched_jobs"] == sum(batches)
    assert sum("batched" in h.result for h in handles) == sum(batches)
    for h, (Z, xyz, basis, uhf) in zip(handles, jobs):
        r = h.wait()
        assert r["converged"], (h.id, basis, uhf)
        assert "batched" not in r or h.nbf <= 60
        kw = dict(s.defaults, **(serve.UHF_KW if uhf else serve.RHF_KW))
        alone = scf.run_scf(Z, xyz, basis, unrestricted=uhf, want_density=False, **kw)
        assert abs(r["energy"] - alone["energy"]) <= 1e-6, (h.id, basis, uhf, r["energy"], alone["energy"])
