"""Regenerate the golden fixtures from the reference itself.

Runs the reference's own IntegralsRepository / RestrictedHartreeFock /
UnrestrictedHartreeFock, compiled headless by oracle/Makefile into
oracle/_ref/ref_driver, on the fixture molecules and stores what it printed.
Only needed when fixtures change; needs the reference tree (REF_DIR).

    make -C oracle ref && python tests/golden/make_golden.py
"""
import os
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, os.path.join(ROOT, "oracle"))
sys.path.insert(0, ROOT)
import oracle as O  # noqa: E402
from hartreefock_b200 import molecules  # noqa: E402
from hartreefock_b200.basis_io import basis_path  # noqa: E402

REF_DIR = os.environ.get("REF_DIR", "/root/reference/HartreeFock")


def fixtures():
    h2o_Z, h2o_xyz = molecules.H2O_README
    return {
        # README.md water, STO-3G, initGuess 0, alpha 0.5
        "h2o_sto3g": dict(Z=h2o_Z, xyz=h2o_xyz, basis="sto-3g", ref_basis="sto3g.txt", eri=True,
                          scf=[("rhf", 0.5, 0.0), ("uhf", 0.5, 0.0)], spinorb=True),
        # two oxygens: exercises every class up to (dd|dd), two-centre bras included
        "o2_631gs": dict(Z=[8, 8], xyz=np.array([[0.0, 0.0, 0.0], [0.3, -0.2, 2.3]]), basis="6-31g*",
                         ref_basis="6-31g_st_.1.nw", eri=True, scf=[]),
        "h2o_631gs": dict(Z=h2o_Z, xyz=h2o_xyz, basis="6-31g*", ref_basis="6-31g_st_.1.nw", eri=True,
                          scf=[("rhf", 0.75, 0.75)]),
        "oh_631g": dict(Z=molecules.hydroxyl()[0], xyz=molecules.hydroxyl()[1], basis="6-31g", ref_basis="6-31g.1.nw",
                        eri=True, scf=[("uhf", 0.75, 0.75)]),
        "h2o2_631gs": dict(Z=molecules.water_cluster(2, seed=0)[0], xyz=molecules.water_cluster(2, seed=0)[1],
                           basis="6-31g*", ref_basis="6-31g_st_.1.nw", eri=False, scf=[("rhf", 0.75, 0.75)]),
        "h2o_631ppgss": dict(Z=h2o_Z, xyz=h2o_xyz, basis="6-31+g**", ref_basis="6-31+g_st__st_.1.nw", eri=True,
                             scf=[]),
    }


# Test::InitWaterMolecule (Test.cpp:572-608): O, H1, H2 in bohr
CRAWFORD_WATER = ([8, 1, 1], np.array([[0.0, -0.143225816552, 0.0], [1.638036840407, 1.136548822547, 0.0],
                                       [-1.638036840407, 1.136548822547, 0.0]]))


def dipole_fixture(td):
    """Test::TestWaterDipoleMoment (Test.cpp:627-733): the Crawford water in
    STO-3G, RHF without DIIS, alpha 0.5, initGuess 0.7; the analytic dipole
    (GetMoment) and the SCF energies in fields of +-0.001 au along each axis."""
    Z, xyz = CRAWFORD_WATER
    mol = O.Molecule(Z, xyz, os.path.join(REF_DIR, "sto3g.txt"))
    kw = dict(alpha=0.5, init_guess=0.7, use_diis=False)
    r = O.run_reference(mol, "rhf", os.path.join(td, "d.bin"), **kw)
    out = {"Z": np.array(Z), "xyz": xyz, "basis": np.array("sto-3g"), "alpha": np.array(0.5),
           "initguess": np.array(0.7), "use_diis": np.array(0), "rhf_energy": r["energy"], "dipole": r["dipole"],
           "enuc_test": np.array(8.002367061810450)}
    fields = []
    for axis in range(3):
        for sign in (-1, 1):
            f = [0.0, 0.0, 0.0]
            f[axis] = sign * 1e-3
            rf = O.run_reference(mol, "rhf", os.path.join(td, "f.bin"), extra="field %.17g %.17g %.17g" % tuple(f), **kw)
            fields.append(f + [float(rf["energy"][0])])
    out["field_energies"] = np.array(fields)  # rows: Ex, Ey, Ez, E
    np.savez_compressed(os.path.join(HERE, "h2o_crawford_sto3g.npz"), **out)
    print("h2o_crawford_sto3g", r["dipole"], np.linalg.norm(r["dipole"]))


def main():
    with tempfile.TemporaryDirectory() as td:
        dipole_fixture(td)
    for name, fx in fixtures().items():
        out = {"Z": np.array(fx["Z"]), "xyz": np.asarray(fx["xyz"]), "basis": np.array(fx["basis"])}
        mol = O.Molecule(fx["Z"], fx["xyz"], os.path.join(REF_DIR, fx["ref_basis"]))
        # the bundled subset must expand to the same basis as the reference file
        mol_b = O.Molecule(fx["Z"], fx["xyz"], basis_path(fx["basis"]))
        assert mol_b.nbf == mol.nbf
        with tempfile.TemporaryDirectory() as td:
            if fx["eri"]:
                r = O.run_reference(mol, "eri", os.path.join(td, "eri.bin"))
                out["eri_packed"] = r["eri_packed"]
                out["h"] = r["h"].reshape(mol.nbf, mol.nbf)
                out["enuc"] = r["enuc"]
            for kind, alpha, guess in fx["scf"]:
                so = kind == "rhf" and fx.get("spinorb", False)
                r = O.run_reference(mol, kind, os.path.join(td, kind + ".bin"), alpha=alpha, init_guess=guess,
                                    extra="mp2 1" + ("\nspinorb 1" if so else ""))
                if so:
                    # SpinOrbitalsElectronElectronIntegralsRepository over the converged C
                    out["rhf_C"] = r["C"].reshape(mol.nbf, mol.nbf)
                    out["spin_orbital_eri"] = r["spin_orbital_eri"]
                out[f"{kind}_energy"] = r["energy"]
                out[f"{kind}_mp2"] = r["mp2"]
                out[f"{kind}_alpha"] = np.array(alpha)
                out[f"{kind}_initguess"] = np.array(guess)
                if kind == "rhf":
                    out["rhf_density"] = r["density"].reshape(mol.nbf, mol.nbf)
                else:
                    out["uhf_density_alpha"] = r["density_alpha"].reshape(mol.nbf, mol.nbf)
                    out["uhf_density_beta"] = r["density_beta"].reshape(mol.nbf, mol.nbf)
                out["h"] = r["h"].reshape(mol.nbf, mol.nbf)
        np.savez_compressed(os.path.join(HERE, name + ".npz"), **out)
        print(name, mol.nbf, {k: (v.shape if hasattr(v, "shape") else v) for k, v in out.items()})


if __name__ == "__main__":
    main()
