"""Device one-electron integrals (hfg_one_electron): S, T and V against the
oracle's restatement of QuantumMatrix / GaussianOverlap / GaussianKinetic /
GaussianNuclear, and h = T + V against the reference's own core Hamiltonian
(golden fixtures), over s, p and d shells, SP shells and diffuse sets."""
import numpy as np
import pytest

import oracle as O
from conftest import load_golden
from hartreefock_b200 import engine as E
from hartreefock_b200 import molecules, scf
from hartreefock_b200.basis_io import basis_path

pytestmark = pytest.mark.gpu

GOLDEN = ["h2o_sto3g", "h2o_631gs", "oh_631g", "o2_631gs", "h2o_631ppgss", "h2o2_631gs"]


@pytest.mark.parametrize("name", GOLDEN)
def test_core_hamiltonian_matches_reference(name):
    g = load_golden(name)
    S, h = scf.one_electron(list(g["Z"]), g["xyz"], str(g["basis"]))
    assert np.abs(h - g["h"]).max() < 1e-10
    assert np.abs(np.diag(S) - 1.0).max() < 1e-6  # contracted functions of these sets are near-normalised


@pytest.mark.parametrize("name", GOLDEN)
def test_s_t_v_match_oracle(name):
    g = load_golden(name)
    S, T, V = E.one_electron(list(g["Z"]), g["xyz"], str(g["basis"]))
    So, To, Vo = O.one_electron(O.Molecule(list(g["Z"]), g["xyz"], basis_path(str(g["basis"]))))
    for got, want in ((S, So), (T, To), (V, Vo)):
        assert np.abs(got - want).max() < 1e-11 * max(1.0, np.abs(want).max())


@pytest.mark.parametrize("kind,basis", [("alkane3", "6-31+g**"), ("water4", "6-31g*")])
def test_larger_molecules_match_oracle(kind, basis):
    Z, xyz = molecules.alkane(3) if kind == "alkane3" else molecules.water_cluster(4, seed=2)
    S, T, V = E.one_electron(Z, xyz, basis)
    So, To, Vo = O.one_electron(O.Molecule(list(Z), xyz, basis_path(basis)))
    for got, want in ((S, So), (T, To), (V, Vo)):
        assert np.abs(got - want).max() < 1e-11 * max(1.0, np.abs(want).max())
