"""AO -> MO transform (hfg_mo_eri_ovov) and the RHF MP2 energy (hfg_mp2_rhf,
RestrictedHartreeFock::CalculateMp2Energy) against a numpy restatement of
RestrictedHartreeFock.cpp:251-288 over the oracle's packed ERI table."""
import numpy as np
import pytest
import torch

import oracle as O
from conftest import load_golden
from hartreefock_b200 import engine as E
from hartreefock_b200 import scf
from hartreefock_b200.basis_io import basis_path

pytestmark = pytest.mark.gpu


def full_eri(packed, n):
    idx = np.arange(n)
    ij = np.where(idx[:, None] >= idx[None, :], idx[:, None] * (idx[:, None] + 1) // 2 + idx[None, :],
                  idx[None, :] * (idx[None, :] + 1) // 2 + idx[:, None])
    a, b = ij[:, :, None, None], ij[None, None, :, :]
    return packed[np.where(a >= b, a * (a + 1) // 2 + b, b * (b + 1) // 2 + a)]


def mp2_numpy(eri, C, eps, nocc):
    Co, Cv = C[:, :nocc], C[:, nocc:]
    ovov = np.einsum("mnls,mi,na,lj,sb->iajb", eri, Co, Cv, Co, Cv, optimize=True)
    eo, ev = eps[:nocc], eps[nocc:]
    d = eo[:, None, None, None] - ev[None, :, None, None] + eo[None, None, :, None] - ev[None, None, None, :]
    return float(np.sum(ovov * (2 * ovov - ovov.transpose(0, 3, 2, 1)) / d)), ovov


def _setup(name="h2o_631gs"):
    g = load_golden(name)
    Z, xyz, basis = list(g["Z"]), g["xyz"], str(g["basis"])
    eng = E.Engine(Z, xyz, basis, schwarz_threshold=0.0)
    mol = O.Molecule(Z, xyz, basis_path(basis))
    return eng, full_eri(O.eri_packed(mol), mol.nbf), mol


def test_mo_block_and_mp2_on_random_orbitals():
    eng, eri, mol = _setup()
    n, nocc = mol.nbf, 5
    rng = np.random.default_rng(4)
    C, _ = np.linalg.qr(rng.normal(size=(n, n)))
    eps = np.concatenate([np.sort(rng.uniform(-20, -0.3, nocc)), np.sort(rng.uniform(0.2, 5, n - nocc))])
    want, ovov = mp2_numpy(eri, C, eps, nocc)
    got = eng.mp2_rhf(C, eps, nocc)
    assert abs(got - want) <= 1e-11 * max(1.0, abs(want))
    X = eng.mo_eri_ovov_tensor(torch.from_numpy(C).cuda(), 0, nocc, nocc, n - nocc).cpu().numpy()
    assert np.abs(X - ovov.reshape(nocc * (n - nocc), -1)).max() < 1e-11
    # twice in a row: no state carried between calls
    assert eng.mp2_rhf(C, eps, nocc) == pytest.approx(got, abs=1e-13)


def test_scf_mp2_matches_canonical_orbitals_of_the_converged_density():
    g = load_golden("h2o_sto3g")
    Z, xyz = list(g["Z"]), g["xyz"]
    r = scf.run_scf(Z, xyz, "sto-3g", alpha=0.5, init_guess=0.0, schwarz_threshold=0.0, mp2=True)
    mol = O.Molecule(Z, xyz, basis_path("sto-3g"))
    n, packed = mol.nbf, O.eri_packed(mol)
    S, T, V = O.one_electron(mol)
    F = T + V + O.g_rhf(n, packed, r["density"])
    s, U = np.linalg.eigh(S)
    X = U @ np.diag(s ** -0.5) @ U.T
    eps, Cp = np.linalg.eigh(X @ F @ X)
    want, _ = mp2_numpy(full_eri(packed, n), X @ Cp, eps, 5)
    assert want < 0
    assert abs(r["mp2_energy"] - want) < 1e-8, (r["mp2_energy"], want)


@pytest.mark.parametrize("nplus,nminus", [(5, 5), (5, 4), (4, 5), (5, 2), (2, 5), (7, 0)])
def test_uhf_mp2_cache_rule_on_random_orbitals(nplus, nminus):
    """hfg_mp2_uhf against the oracle's literal restatement of the reference's
    index-keyed MO cache (IntegralsRepository.h:190-291), unrelated C+ and C-
    so every mixed-spin block of the second sum shows, for both orders of the
    occupied counts."""
    g = load_golden("h2o_sto3g")
    Z, xyz = list(g["Z"]), g["xyz"]
    eng = E.Engine(Z, xyz, "sto-3g", schwarz_threshold=0.0)
    mol = O.Molecule(Z, xyz, basis_path("sto-3g"))
    n = mol.nbf
    rng = np.random.default_rng(10 * nplus + nminus)
    Cp, _ = np.linalg.qr(rng.normal(size=(n, n)))
    Cm, _ = np.linalg.qr(rng.normal(size=(n, n)))
    ep = np.concatenate([np.sort(rng.uniform(-20, -0.3, nplus)), np.sort(rng.uniform(0.2, 5, n - nplus))])
    em = np.concatenate([np.sort(rng.uniform(-20, -0.3, nminus)), np.sort(rng.uniform(0.2, 5, n - nminus))])
    want = O.mp2_uhf(full_eri(O.eri_packed(mol), n), Cp, ep, nplus, Cm, em, nminus)
    got = eng.mp2_uhf(Cp, ep, nplus, Cm, em, nminus)
    eng.close()
    assert abs(got - want) <= 1e-11 * max(1.0, abs(want)), (got, want)


MP2_TOL = 1e-8  # Eh: MP2 energies of SCF runs that match the reference's energies within 1e-9


@pytest.mark.parametrize("name,kind", [("h2o_sto3g", "rhf"), ("h2o_631gs", "rhf"), ("h2o2_631gs", "rhf"),
                                       ("h2o_sto3g", "uhf"), ("oh_631g", "uhf")])
def test_scf_mp2_matches_reference(name, kind):
    """CalculateMp2Energy after the SCF, RHF (RestrictedHartreeFock.cpp:251-288)
    and UHF (UnrestrictedHartreeFock.cpp:295-375, including its orbital-index
    cache), against the values the reference itself printed."""
    g = load_golden(name)
    r = scf.run_scf(list(g["Z"]), g["xyz"], str(g["basis"]), unrestricted=(kind == "uhf"),
                    alpha=float(g[f"{kind}_alpha"]), init_guess=float(g[f"{kind}_initguess"]),
                    schwarz_threshold=0.0, mp2=True)
    assert r["converged"]
    want = float(g[f"{kind}_mp2"][0])
    assert want < 0
    assert abs(r["mp2_energy"] - want) < MP2_TOL, (r["mp2_energy"], want)


def test_spin_orbital_tensor_matches_reference():
    """SpinOrbitalsElectronElectronIntegralsRepository::Compute over the
    reference's own converged C (README water, STO-3G), element by element."""
    g = load_golden("h2o_sto3g")
    eng = E.Engine(list(g["Z"]), g["xyz"], "sto-3g", schwarz_threshold=0.0)
    T = eng.spin_orbital_eri(g["rhf_C"])
    want = g["spin_orbital_eri"].reshape(T.shape)
    assert np.abs(T - want).max() < 1e-12
    # antisymmetry <pq||rs> = -<pq||sr> and the spin selection
    assert np.abs(T + T.transpose(0, 1, 3, 2)).max() < 1e-12
    assert np.abs(T[0, 1, 0, 1] - want[0, 1, 0, 1]) < 1e-12
    eng.close()
