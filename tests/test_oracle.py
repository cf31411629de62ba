"""The oracle restatement against the reference's own outputs (golden
fixtures written by the reference compiled headless), plus the Boys function
against its defining series.  CPU only."""
import math

import numpy as np
import pytest

import oracle as O
from conftest import load_golden
from hartreefock_b200.basis_io import basis_path

ALL = ["h2o_sto3g", "o2_631gs", "h2o_631gs", "oh_631g", "h2o_631ppgss"]


def mol_of(g):
    return O.Molecule(list(g["Z"]), g["xyz"], basis_path(str(g["basis"])))


@pytest.mark.parametrize("name", ALL)
def test_oracle_eri_matches_reference(name):
    g = load_golden(name)
    got = O.eri_packed(mol_of(g))
    ref = g["eri_packed"]
    # both sides compiled for x86-64-v3 with FMA contraction: agreement to
    # ~1e-13 (without matching contraction one oxygen (sp|sp) element of
    # o2_631gs moves by 1.85e-12)
    assert np.abs(got - ref).max() <= 1e-12


@pytest.mark.parametrize("name", ALL)
def test_oracle_core_hamiltonian_matches_reference(name):
    g = load_golden(name)
    S, T, V = O.one_electron(mol_of(g))
    assert np.abs(T + V - g["h"]).max() < 1e-11


def test_nuclear_repulsion_pins():
    # Test.cpp:623 (Crawford water geometry, Test.cpp:572-608) and Test.cpp:781 (methane)
    g = load_golden("h2o_sto3g")
    assert abs(O.Molecule(list(g["Z"]), g["xyz"], basis_path("sto-3g")).nuclear_repulsion() - float(g["enuc"][0])) < 1e-12


@pytest.mark.parametrize("name,kind", [("h2o_sto3g", "rhf"), ("h2o_sto3g", "uhf"), ("h2o_631gs", "rhf"),
                                       ("oh_631g", "uhf")])
def test_oracle_scf_energy_matches_reference(name, kind):
    g = load_golden(name)
    r = O.run_scf(mol_of(g), unrestricted=(kind == "uhf"), alpha=float(g[f"{kind}_alpha"]),
                  init_guess=float(g[f"{kind}_initguess"]), packed=g.get("eri_packed"))
    assert r["converged"]
    assert abs(r["energy"] - float(g[f"{kind}_energy"][0])) < 1e-9


@pytest.mark.parametrize("name", ["h2o_sto3g", "oh_631g"])
def test_oracle_uhf_mp2_matches_reference(name):
    """The literal restatement of the index-keyed MO cache
    (IntegralsRepository.h:190-291) on the canonical orbitals of the
    reference's converged UHF densities gives the MP2 energy the reference
    printed (UnrestrictedHartreeFock.cpp:295-375).  OH: Molecule::Init puts
    the odd electron in the minus spin (n+ = 4, n- = 5), so S- reads C+
    values cached by S+ for i, j < 4 and mixes spins for i or j = 4."""
    g = load_golden(name)
    mol = mol_of(g)
    n, packed = mol.nbf, g["eri_packed"]
    S, T, V = O.one_electron(mol)
    Pa, Pb = g["uhf_density_alpha"], g["uhf_density_beta"]
    Ga, Gb = O.g_uhf(n, packed, Pa, Pb)
    s, U = np.linalg.eigh(S)
    X = U @ np.diag(s ** -0.5) @ U.T
    ea, Ca = np.linalg.eigh(X @ (T + V + Ga) @ X)
    eb, Cb = np.linalg.eigh(X @ (T + V + Gb) @ X)
    na, nb = int(round(np.trace(Pa @ S))), int(round(np.trace(Pb @ S)))
    got = O.mp2_uhf(O.unpack_eri(packed, n), X @ Ca, ea, na, X @ Cb, eb, nb)
    assert abs(got - float(g["uhf_mp2"][0])) < 1e-10, (got, float(g["uhf_mp2"][0]))


@pytest.mark.parametrize("m,T", [(0, 0.0), (0, 1e-12), (3, 0.7), (8, 5.0), (8, 12.3), (4, 35.9), (8, 36.5),
                                 (2, 80.0), (9, 170.0)])
def test_boys_against_series(m, T):
    got = O.boys(m, T)
    for k in range(m + 1):
        # F_k(T) = e^-T sum_j (2T)^j / ((2k+1)(2k+3)...(2k+2j+1))
        term, s, j = 1.0 / (2 * k + 1), 0.0, 0
        while True:
            s += term
            j += 1
            term *= 2 * T / (2 * k + 2 * j + 1)
            if term < 1e-18 * s or j > 5000:
                break
        want = math.exp(-T) * s if T < 700 else 0.0
        if T > 100:  # the series loses everything to exp underflow; use the asymptote
            want = math.prod(range(2 * k - 1, 0, -2)) / 2 ** (k + 1) * math.sqrt(math.pi / T ** (2 * k + 1))
        # the reference clamps T below 1e-10 to 1e-10 for the top order
        # (BoysFunction.cpp:13-14), which moves F by O(1e-10 / (2m+3))
        tol = 1e-10 if T < 1e-10 else 1e-14 * max(1.0, abs(want)) + 1e-13 * abs(want)
        assert abs(got[k] - want) <= tol
