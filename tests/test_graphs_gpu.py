"""CUDA-graph replay of the plain direct build (hfg_set_graphs) and
concurrent class streams (hfg_set_streams): the second build with the same
buffers is captured, later ones replay it, and every result equals the
single-stream build without graphs -- also when the density changes in
place, when the buffers change and after a setter; SCF energies with both on
equal those without."""
import numpy as np
import pytest
import torch

from hartreefock_b200 import engine as E
from hartreefock_b200 import molecules, scf

pytestmark = pytest.mark.gpu


def _density(n, seed):
    rng = np.random.default_rng(seed)
    Q, _ = np.linalg.qr(rng.normal(size=(n, n // 4)))
    return 2.0 * Q @ Q.T


def test_graph_replay_matches_plain_builds():
    Z, xyz = molecules.water_cluster(3, seed=5)
    plain = E.Engine(Z, xyz, "6-31g*")
    graph = E.Engine(Z, xyz, "6-31g*")
    graph.set_graphs(True)
    graph.set_streams(True)
    n = plain.nbf
    dP = torch.zeros(n, n, dtype=torch.float64, device="cuda")
    dG = torch.zeros_like(dP)
    torch.cuda.synchronize()  # the builds run on the context's own stream
    # a created stream: the legacy default stream is not captured
    side = torch.cuda.Stream()
    with torch.cuda.stream(side):
        for k in range(5):  # build 1 plain, 2 captured, 3-5 replayed; density changes in place each time
            P = _density(n, k)
            dP.copy_(torch.from_numpy(P))
            torch.cuda.synchronize()
            graph.fock_rhf_tensor(dP, dG)
            torch.cuda.synchronize()
            want = plain.fock_rhf(P)
            got = dG.cpu().numpy()
            assert np.abs(got - want).max() < 1e-12 * max(1.0, np.abs(want).max()), k
        # new output buffer: built normally, then captured again
        dG2 = torch.zeros_like(dP)
        torch.cuda.synchronize()  # the builds run on the context's own stream
        for _ in range(3):
            graph.fock_rhf_tensor(dP, dG2)
        torch.cuda.synchronize()
        assert torch.allclose(dG2, dG, rtol=0, atol=1e-12 * float(dG.abs().max()))
        # a setter invalidates the graph; the result stays the same
        graph.autotune(dP)
        for _ in range(3):
            graph.fock_rhf_tensor(dP, dG2)
        torch.cuda.synchronize()
        assert torch.allclose(dG2, dG, rtol=0, atol=1e-12 * float(dG.abs().max()))
    assert graph.stats()["shell_quartets"] == plain.stats()["shell_quartets"]


def test_graph_replay_uhf():
    Z, xyz = molecules.hydroxyl()
    plain = E.Engine(Z, xyz, "6-31g*")
    graph = E.Engine(Z, xyz, "6-31g*")
    graph.set_graphs(True)
    graph.set_streams(True)
    n = plain.nbf
    Pa, Pb = _density(n, 1) * 0.5, _density(n, 2) * 0.5
    t = [torch.from_numpy(x).cuda() for x in (Pa, Pb)]
    Ga, Gb = torch.zeros_like(t[0]), torch.zeros_like(t[0])
    torch.cuda.synchronize()
    side = torch.cuda.Stream()
    with torch.cuda.stream(side):
        for _ in range(4):
            graph.fock_uhf_tensor(t[0], t[1], Ga, Gb)
    torch.cuda.synchronize()
    wa, wb = plain.fock_uhf(Pa, Pb)
    assert np.abs(Ga.cpu().numpy() - wa).max() < 1e-12 * max(1.0, np.abs(wa).max())
    assert np.abs(Gb.cpu().numpy() - wb).max() < 1e-12 * max(1.0, np.abs(wb).max())


@pytest.mark.parametrize("mixed", [False, True])
def test_scf_with_graphs_and_streams_matches(mixed):
    Z, xyz = molecules.water_cluster(3, seed=2)
    kw = dict(alpha=0.5, init_guess=0.0, post_diis=0, want_density=False)
    if mixed:
        kw["mixed_cutoff"] = 1e-4
    a = scf.run_scf(Z, xyz, "6-31g*", **kw)
    b = scf.run_scf(Z, xyz, "6-31g*", concurrent_classes=2, **kw)
    assert a["converged"] and b["converged"]
    assert abs(a["energy"] - b["energy"]) < (1e-6 if mixed else 1e-9)
