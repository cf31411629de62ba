"""The grid autotuner (hfg_autotune) picks one grid per fused class and the
builds after it give the same G as before."""
import numpy as np
import pytest
import torch

from hartreefock_b200 import engine as E
from hartreefock_b200 import molecules

pytestmark = pytest.mark.gpu


def _density(n, seed=3):
    rng = np.random.default_rng(seed)
    Q, _ = np.linalg.qr(rng.normal(size=(n, n // 4)))
    return 2.0 * Q @ Q.T


def test_autotune_keeps_the_build():
    Z, xyz = molecules.water_cluster(4, seed=1)
    eng = E.Engine(Z, xyz, "6-31g*")
    P = _density(eng.nbf)
    before = eng.fock_rhf(P)
    chosen = eng.autotune(P)
    assert chosen and set(chosen.values()) <= {1, 2, 4, 8, 16}
    after = eng.fock_rhf(P)
    assert np.abs(after - before).max() < 1e-11 * max(1.0, np.abs(before).max())


def test_autotune_on_a_batch():
    mols = []
    for k in (1, 2, 3):
        Z, xyz = molecules.water_cluster(k, seed=k)
        mols.append((list(Z), xyz, "6-31g"))
    be = E.BatchEngine(mols)
    flat = np.zeros(be.total)
    for i in range(len(mols)):
        n = int(be.nbf[i])
        flat[be.offset[i]: be.offset[i] + n * n] = _density(n, i).ravel()
    dP = torch.from_numpy(flat).cuda()
    G0 = torch.zeros_like(dP)
    be.fock_rhf(dP, G0)
    assert be.autotune(dP)
    G1 = torch.zeros_like(dP)
    be.fock_rhf(dP, G1)
    assert float((G1 - G0).abs().max()) < 1e-11 * max(1.0, float(G0.abs().max()))
