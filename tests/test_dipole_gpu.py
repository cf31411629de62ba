"""Dipole moment matrices and the electric-field term of the core
Hamiltonian (HartreeFockAlgorithm.cpp:32,38; MomentMatrix,
QuantumMatrix.cpp:61-98; GetMoment, RestrictedHartreeFock.cpp:319-335),
against the reference's own Test::TestWaterDipoleMoment setup
(Test.cpp:627-733): the Crawford water in STO-3G, RHF without DIIS, alpha
0.5, initGuess 0.7.  The reference's test notes 0.603521 au for the
analytic dipole (Test.cpp:660-661); the fixture holds the reference's
GetMoment and its SCF energies in fields of +-0.001 au."""
import numpy as np
import pytest

from conftest import load_golden
from hartreefock_b200 import scf

pytestmark = pytest.mark.gpu


def _run(g, field=(0.0, 0.0, 0.0)):
    return scf.run_scf(list(g["Z"]), g["xyz"], str(g["basis"]), alpha=float(g["alpha"]),
                       init_guess=float(g["initguess"]), use_diis=bool(g["use_diis"]), schwarz_threshold=0.0,
                       electric_field=field)


def test_dipole_matches_reference():
    g = load_golden("h2o_crawford_sto3g")
    r = _run(g)
    assert r["converged"]
    assert abs(r["energy"] - float(g["rhf_energy"][0])) < 1e-9
    mu = np.array(r["dipole"])
    assert np.abs(mu - g["dipole"]).max() < 1e-8
    # the value the reference's test prints (Test.cpp:660-661), six digits
    assert abs(np.linalg.norm(mu) - 0.603521) < 5e-7


def test_field_energies_match_reference_and_finite_field_dipole():
    g = load_golden("h2o_crawford_sto3g")
    e = {}
    for Ex, Ey, Ez, E_ref in g["field_energies"]:
        r = _run(g, (Ex, Ey, Ez))
        assert r["converged"]
        assert abs(r["energy"] - E_ref) < 1e-9, (Ex, Ey, Ez, r["energy"], E_ref)
        e[(Ex, Ey, Ez)] = r["energy"]
    # mu = nuclear moment + (E(-d) - E(+d)) / 2d  (Test.cpp:722-724)
    Z, xyz = np.array(g["Z"], dtype=float), g["xyz"]
    nuclear = (Z[:, None] * xyz).sum(axis=0)
    d = 1e-3
    ff = []
    for axis in range(3):
        lo, hi = [0.0, 0.0, 0.0], [0.0, 0.0, 0.0]
        lo[axis], hi[axis] = -d, d
        ff.append(nuclear[axis] + (e[tuple(lo)] - e[tuple(hi)]) / (2 * d))
    assert np.abs(np.array(ff) - g["dipole"]).max() < 1e-5
