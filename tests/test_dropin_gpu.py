"""The engine dropped into the reference's own SCF (oracle/dropin_fock.cpp):
the reference's classes, compiled unmodified, with
IntegralsRepository::CalculateElectronElectronIntegrals taking the packed
table from the engine (ref_driver_gpu), or additionally InitFockMatrix /
InitFockMatrices taking G from the engine's direct builds
(ref_driver_gpu_direct).  The reference's DIIS, eigensolves and convergence
loop then reach the energies the unmodified reference reached, within
1e-9 Eh."""
import os
import tempfile

import pytest

import oracle as O
from conftest import load_golden
from hartreefock_b200.basis_io import basis_path

pytestmark = pytest.mark.gpu

E_TOL = 1e-9
DRIVERS = {"stored": os.path.join(O.REF_DIR, "ref_driver_gpu"),
           "direct": os.path.join(O.REF_DIR, "ref_driver_gpu_direct")}


@pytest.mark.parametrize("mode", ["stored", "direct"])
@pytest.mark.parametrize("name,kind", [("h2o_sto3g", "rhf"), ("h2o_sto3g", "uhf"), ("h2o_631gs", "rhf"),
                                       ("oh_631g", "uhf"), ("h2o2_631gs", "rhf")])
def test_reference_scf_on_engine_matches_reference(mode, name, kind):
    if not os.path.exists(DRIVERS[mode]):
        pytest.skip("drop-in build missing (make -C oracle dropin)")
    g = load_golden(name)
    mol = O.Molecule(list(g["Z"]), g["xyz"], basis_path(str(g["basis"])))
    with tempfile.TemporaryDirectory() as td:
        r = O.run_reference(mol, kind, os.path.join(td, "out.bin"), alpha=float(g[f"{kind}_alpha"]),
                            init_guess=float(g[f"{kind}_initguess"]), driver=DRIVERS[mode])
    assert r["converged"][0] == 1.0
    assert abs(float(r["energy"][0]) - float(g[f"{kind}_energy"][0])) < E_TOL
