"""Parity on the water-cluster workloads and the exact ERI convention.

- (H2O)_8 / 6-31G* (152 functions): the direct Fock build against the
  oracle's G from its full unscreened table, and the converged RHF energy of
  the C++ host SCF against the reference's own RHF (tests/golden/h2o8_631gs.npz,
  written by tests/golden/make_golden_large.py).
- (H2O)_16 / 6-31G* (304 functions, the benchmark workload and its density):
  rows of G against the oracle's rows, evaluated without a stored table.
- propane / 6-31G* under the exact electron-transfer convention (the serving
  stream's convention; d shells on bonded carbons): sampled packed ERIs, G and
  the converged energy against the oracle in exact mode.

G tolerances: the engine screens at Schwarz 1e-12 while the oracle evaluates
every quartet, so the comparison is relative to the largest element, 1e-10
(RestrictedHartreeFock.cpp:189-200 defines G).  Energies: 1e-9 Eh.
"""
import numpy as np
import pytest

from conftest import load_golden
from hartreefock_b200 import engine as E
from hartreefock_b200 import scf

pytestmark = pytest.mark.gpu

G_REL = 1e-10
E_TOL = 1e-9
ERI_ABS, ERI_REL = 1e-12, 2.5e-11


def rel_err(got, want):
    return float(np.abs(got - want).max() / np.abs(want).max())


def test_h2o8_fock_build_matches_oracle():
    g = load_golden("h2o8_631gs")
    eng = E.Engine(list(g["Z"]), g["xyz"], str(g["basis"]), schwarz_threshold=1e-12)
    assert eng.nbf == 152
    G = eng.fock_rhf(g["P"])
    err = rel_err(G, g["G"])
    eng.close()
    assert err < G_REL, err


def test_h2o8_rhf_energy_matches_reference():
    g = load_golden("h2o8_631gs")
    want = float(g["rhf_energy"]) if "rhf_energy" in g else float(g["oracle_energy"])
    r = scf.run_scf(list(g["Z"]), g["xyz"], str(g["basis"]), alpha=float(g["alpha"]),
                    init_guess=float(g["initguess"]), post_diis=int(g["post_diis"]))
    assert r["converged"]
    assert abs(r["energy"] - want) < E_TOL, r["energy"] - want
    dens = g["rhf_density"] if "rhf_density" in g else g["oracle_density"]
    assert np.abs(r["density"] - dens).max() < 1e-6


def test_h2o8_oracle_energy_matches_reference():
    """The oracle's SCF on the same cluster agrees with the reference's (the
    fixture's G comes from the oracle)."""
    g = load_golden("h2o8_631gs")
    if "rhf_energy" not in g:
        pytest.skip("fixture written without the reference run")
    assert abs(float(g["oracle_energy"]) - float(g["rhf_energy"])) < E_TOL


def test_h2o16_fock_rows_match_oracle():
    g = load_golden("h2o16_631gs_rows")
    eng = E.Engine(list(g["Z"]), g["xyz"], str(g["basis"]), schwarz_threshold=1e-12)
    assert eng.nbf == 304
    G = eng.fock_rhf(g["P"])
    err = rel_err(G[g["rows"]], g["G_rows"])
    eng.close()
    assert err < G_REL, err


def test_propane_exact_convention_matches_oracle():
    g = load_golden("propane_631gs_exact")
    eng = E.Engine(list(g["Z"]), g["xyz"], str(g["basis"]), schwarz_threshold=0.0, eri_convention=E.ERI_EXACT)
    packed = eng.eri_packed()
    got = packed[g["eri_index"]]
    want = g["eri_value"]
    tol = np.maximum(ERI_ABS, ERI_REL * np.abs(want))
    assert int((np.abs(got - want) > tol).sum()) == 0, float(np.abs(got - want).max())
    G = eng.fock_rhf(g["P"])
    assert rel_err(G, g["G"]) < G_REL
    eng.close()


def test_propane_exact_convention_scf_energy():
    g = load_golden("propane_631gs_exact")
    r = scf.run_scf(list(g["Z"]), g["xyz"], str(g["basis"]), alpha=float(g["alpha"]),
                    init_guess=float(g["initguess"]), post_diis=int(g["post_diis"]), eri_convention=E.ERI_EXACT)
    assert r["converged"]
    assert abs(r["energy"] - float(g["energy"])) < E_TOL, r["energy"] - float(g["energy"])
