"""Batched contexts and the batched SCF: one launch per quartet class over
many molecules of uneven size gives every molecule the G (and the converged
energy) it gets alone."""
import numpy as np
import pytest
import torch

from conftest import load_golden
from hartreefock_b200 import batch
from hartreefock_b200 import engine as E
from hartreefock_b200 import molecules, scf

pytestmark = pytest.mark.gpu


def _mix():
    g = load_golden("h2o_sto3g")
    out = [dict(Z=list(g["Z"]), xyz=g["xyz"], basis="sto-3g")]
    for k, basis in ((1, "6-31g*"), (2, "6-31g"), (3, "sto-3g")):
        Z, xyz = molecules.water_cluster(k, seed=k)
        out.append(dict(Z=list(Z), xyz=xyz, basis=basis))
    for nc, basis in ((1, "sto-3g"), (3, "6-31g")):
        Z, xyz = molecules.alkane(nc)
        out.append(dict(Z=list(Z), xyz=xyz, basis=basis))
    return out


def _density(n, seed):
    rng = np.random.default_rng(seed)
    Q, _ = np.linalg.qr(rng.normal(size=(n, max(1, n // 4))))
    return 2.0 * Q @ Q.T


def test_batched_fock_equals_single_molecule_builds():
    mols = _mix()
    be = E.BatchEngine([(m["Z"], m["xyz"], m["basis"]) for m in mols])
    flatP = np.zeros(be.total)
    want = []
    for i, m in enumerate(mols):
        n = int(be.nbf[i])
        P = _density(n, i)
        flatP[be.offset[i]: be.offset[i] + n * n] = P.ravel()
        want.append(E.Engine(m["Z"], m["xyz"], m["basis"]).fock_rhf(P))
    dP = torch.from_numpy(flatP).cuda()
    dG = torch.full_like(dP, 7.0)
    active = np.ones(len(mols), dtype=np.uint8)
    active[2] = 0
    be.fock_rhf(dP, dG, active=active)
    G = dG.cpu().numpy()
    for i, w in enumerate(want):
        n = int(be.nbf[i])
        got = G[be.offset[i]: be.offset[i] + n * n].reshape(n, n)
        if i == 2:
            assert np.all(got == 7.0)  # inactive: left untouched
        else:
            assert np.abs(got - w).max() < 1e-11 * max(1.0, np.abs(w).max()), i


def test_batched_scf_matches_single_molecule_scf():
    mols = _mix()
    kw = dict(alpha=0.75, init_guess=0.75)
    bs = batch.BatchSCF(mols, **kw)
    energies = bs.run()
    assert bs.converged.all()
    for i, m in enumerate(mols):
        ref = scf.run_scf(m["Z"], m["xyz"], m["basis"], post_diis=0, **kw)
        assert abs(energies[i] - ref["energy"]) < 1e-8, (i, energies[i], ref["energy"])


def test_batched_uhf_scf_matches_single_molecule_scf():
    # planar CH3 (non-degenerate singly occupied orbital) at two C-H lengths;
    # OH is left out: its unpaired electron sits in a degenerate
    # pi level, so which pi orbital it occupies (and the state the SCF ends
    # in) is decided by rounding inside the eigensolver, alone or batched
    mols = []
    for basis in ("sto-3g", "6-31g"):
        Z, xyz = molecules.methyl_planar()
        mols.append(dict(Z=list(Z), xyz=xyz, basis=basis))
    Z, xyz = molecules.methyl_planar(r_ch=1.12)
    mols.append(dict(Z=list(Z), xyz=xyz, basis="6-31g"))
    kw = dict(alpha=0.5, init_guess=0.0)
    bs = batch.BatchSCF(mols, unrestricted=True, max_iter=3000, **kw)
    energies = bs.run()
    for i, m in enumerate(mols):
        ref = scf.run_scf(m["Z"], m["xyz"], m["basis"], unrestricted=True, post_diis=0, **kw)
        # the reference's UHF test (DIIS error < 1e-10) can stall for these
        # doublets near 1e-10 for thousands of steps, so which of the two runs
        # meets it first is not fixed; both get 3000 and their energies agree
        assert abs(energies[i] - ref["energy"]) < 1e-6, (i, energies[i], ref["energy"])


def test_async_batched_build_matches_host_masked_build():
    """The device-queue build (active mask in device memory, no host
    synchronisation) gives the host-masked build's G."""
    mols = _mix()
    be = E.BatchEngine([(m["Z"], m["xyz"], m["basis"]) for m in mols])
    flatP = np.zeros(be.total)
    for i in range(len(mols)):
        n = int(be.nbf[i])
        flatP[be.offset[i]: be.offset[i] + n * n] = _density(n, i).ravel()
    dP = torch.from_numpy(flatP).cuda()
    active = np.ones(len(mols), dtype=np.uint8)
    active[1] = active[4] = 0
    G1 = torch.full_like(dP, 3.0)
    be.fock_rhf(dP, G1, active=active)
    for _ in range(2):  # twice: the queue counters start over every build
        G2 = torch.full_like(dP, 3.0)
        be.fock_rhf_async(dP, G2, torch.from_numpy(active).cuda())
        torch.cuda.synchronize()
        assert torch.equal(G1 == 3.0, G2 == 3.0)
        assert float((G1 - G2).abs().max()) < 1e-11 * float(G1.abs().max())


def test_graph_captured_batched_scf_matches_eager():
    """Every iteration after the DIIS history fills is a replayed CUDA graph;
    energies agree with the host-driven loop and with single-molecule runs."""
    mols = _mix()
    kw = dict(alpha=0.75, init_guess=0.75)
    eager = batch.BatchSCF(mols, **kw).run()
    bs = batch.BatchSCF(mols, graphs=True, **kw)
    energies = bs.run()
    assert bs.graph_captures >= 1
    assert bs.converged.all()
    assert np.abs(energies - eager).max() < 1e-9
    for i, m in enumerate(mols):
        ref = scf.run_scf(m["Z"], m["xyz"], m["basis"], post_diis=0, **kw)
        assert abs(energies[i] - ref["energy"]) < 1e-8, (i, energies[i], ref["energy"])


def test_device_pulay_solve_matches_host():
    """hfg_pulay_solve_device against the host SCF's solve (the same
    column-pivoted QR), including a rank-deficient system."""
    rng = np.random.default_rng(3)
    B = rng.normal(size=(9, 7, 7))
    B = B + B.transpose(0, 2, 1)
    B[:, 6, :6] = B[:, :6, 6] = 1.0
    B[:, 6, 6] = 0.0
    B[0, 5, :] = B[0, 4, :]
    B[0, :, 5] = B[0, :, 4]
    got = E.pulay_solve_device(torch.from_numpy(B).cuda()).cpu().numpy()
    want = scf.pulay_solve(B)
    # the same QR in a different order of operations: agreement relative to
    # the solution's size (the rank-deficient system's entries reach 1e3)
    assert np.abs(got - want).max() < 1e-11 * max(1.0, np.abs(want).max())


@pytest.mark.parametrize("method", [0, 1])
def test_batched_uhf_doublets_with_both_eigensolvers(method):
    """The bench's UHF doublets (OH, planar CH3; STO-3G, 6-31G; alpha 0.5,
    initGuess 0.75) batched with the batched Jacobi solver (0, the default)
    and with one dsyevd per matrix (1) reach the single-molecule energies."""
    mols = []
    for basis in ("sto-3g", "6-31g"):
        for Z, xyz in (molecules.hydroxyl(), molecules.methyl_planar()):
            mols.append(dict(Z=list(Z), xyz=xyz, basis=basis))
    kw = dict(alpha=0.5, init_guess=0.75)
    bs = batch.BatchSCF(mols + mols, unrestricted=True, max_iter=1000, eigh_method=method, **kw)
    energies = bs.run()
    assert bs.converged.all()
    for i, m in enumerate(mols + mols):
        ref = scf.run_scf(m["Z"], m["xyz"], m["basis"], unrestricted=True, post_diis=0, want_density=False, **kw)
        assert abs(energies[i] - ref["energy"]) < 1e-9, (i, m["basis"], energies[i], ref["energy"])
