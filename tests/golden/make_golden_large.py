"""Golden fixtures for the water-cluster workloads and the exact ERI convention.

    make -C oracle port ref && python tests/golden/make_golden_large.py [--no-reference]

Writes
  h2o8_631gs.npz        (H2O)_8 / 6-31G* (152 functions, cluster seed 0):
                        - the reference's own RHF (oracle/_ref/ref_driver, the
                          reference's classes compiled headless; initGuess 0.75,
                          alpha 0.75, DIIS, no post-DIIS iterations,
                          IntegralsRepository::SetUseLotsOfMemory(false) so the
                          build fits in host memory): energy, density, Init and
                          Calculate seconds;
                        - the oracle's G = sum_kl P_kl[(ij|kl) - 1/2 (il|kj)]
                          (RestrictedHartreeFock.cpp:189-200) for that density,
                          from the oracle's full unscreened packed table.
  h2o16_631gs_rows.npz  (H2O)_16 / 6-31G* (304 functions): rows of the oracle's
                        G for a fixed density (2 Q Q^T, Q orthonormal, seed 1),
                        evaluated from the contracted ERIs without a table.
  propane_631gs_exact.npz  C3H8 / 6-31G* (61 functions, d shells on three
                        bonded carbons): the exact electron-transfer convention
                        (every row of the recursion): oracle SCF energy and
                        density, G for that density, and a seeded sample of the
                        packed table.

The oracle (oracle/eri_oracle.c) is the plain-C restatement of the
reference's ERI path; it is pinned to the reference build on every table of
make_golden.py.  The reference run for (H2O)_8 takes of the order of an hour
on one core; --no-reference skips it (the fixture then carries the oracle's
SCF only).
"""
import argparse
import os
import sys
import tempfile
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, os.path.join(ROOT, "oracle"))
sys.path.insert(0, ROOT)
import oracle as O  # noqa: E402
from hartreefock_b200 import molecules  # noqa: E402
from hartreefock_b200.basis_io import basis_path  # noqa: E402


def orthonormal_density(n, seed):
    """2 Q Q^T for n/4 random orthonormal columns: a density of realistic
    magnitude that is not an SCF solution."""
    rng = np.random.default_rng(seed)
    Q, _ = np.linalg.qr(rng.normal(size=(n, max(1, n // 4))))
    return 2.0 * Q @ Q.T


def h2o8(with_reference: bool, reference_bin: str = ""):
    Z, xyz = molecules.water_cluster(8, seed=0)
    mol = O.Molecule(Z, xyz, basis_path("6-31g*"))
    n = mol.nbf
    out = {"Z": np.array(Z), "xyz": np.asarray(xyz), "basis": np.array("6-31g*"), "alpha": np.array(0.75),
           "initguess": np.array(0.75), "post_diis": np.array(0)}
    t = time.time()
    packed = O.eri_packed(mol)
    print(f"(H2O)8 oracle table {time.time() - t:.0f} s", flush=True)
    t = time.time()
    r = O.run_scf(mol, alpha=0.75, init_guess=0.75, post_diis=0, packed=packed)
    print(f"(H2O)8 oracle SCF {time.time() - t:.0f} s, E = {r['energy']:.12f}", flush=True)
    out["oracle_energy"] = np.array(r["energy"])
    out["oracle_density"] = r["density"]
    P = r["density"]
    if with_reference:
        if reference_bin:
            # output of an earlier ref_driver run with the same directives
            ref = O.read_records(reference_bin)
        else:
            with tempfile.TemporaryDirectory() as td:
                t = time.time()
                ref = O.run_reference(mol, "rhf", os.path.join(td, "rhf.bin"), alpha=0.75, init_guess=0.75,
                                      post_diis=0, extra="lowmem 1", timeout=6 * 3600)
                print(f"(H2O)8 reference RHF {time.time() - t:.0f} s", flush=True)
        print(f"(H2O)8 reference E = {float(ref['energy'][0]):.12f}", flush=True)
        out["rhf_energy"] = np.array(float(ref["energy"][0]))
        out["rhf_density"] = ref["density"].reshape(n, n)
        out["ref_init_seconds"] = np.array(float(ref["init_seconds"][0]))
        out["ref_scf_seconds"] = np.array(float(ref["scf_seconds"][0]))
        P = out["rhf_density"]
    out["P"] = P
    out["G"] = O.g_rhf(n, packed, P)
    np.savez_compressed(os.path.join(HERE, "h2o8_631gs.npz"), **out)


def h2o16_rows(rows=(0, 40, 301)):
    Z, xyz = molecules.water_cluster(16, seed=0)
    mol = O.Molecule(Z, xyz, basis_path("6-31g*"))
    P = orthonormal_density(mol.nbf, 1)
    t = time.time()
    G = O.g_rhf_rows(mol, P, list(rows))
    print(f"(H2O)16 oracle G rows {time.time() - t:.0f} s", flush=True)
    np.savez_compressed(os.path.join(HERE, "h2o16_631gs_rows.npz"), Z=np.array(Z), xyz=np.asarray(xyz),
                        basis=np.array("6-31g*"), P=P, rows=np.array(rows), G_rows=G)


def propane_exact(nsample=4000):
    Z, xyz = molecules.alkane(3)
    mol = O.Molecule(Z, xyz, basis_path("6-31g*"))
    n = mol.nbf
    packed = O.eri_packed(mol, exact_et=True)
    r = O.run_scf(mol, alpha=0.75, init_guess=0.75, post_diis=0, packed=packed, exact_et=True)
    print(f"propane exact SCF E = {r['energy']:.12f}", flush=True)
    P = r["density"]
    rng = np.random.default_rng(3)
    idx = np.sort(rng.choice(len(packed), size=nsample, replace=False))
    np.savez_compressed(os.path.join(HERE, "propane_631gs_exact.npz"), Z=np.array(Z), xyz=np.asarray(xyz),
                        basis=np.array("6-31g*"), alpha=np.array(0.75), initguess=np.array(0.75),
                        post_diis=np.array(0), energy=np.array(r["energy"]), P=P, G=O.g_rhf(n, packed, P),
                        eri_index=idx.astype(np.int64), eri_value=packed[idx])


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--no-reference", action="store_true")
    ap.add_argument("--only", choices=["h2o8", "h2o16", "propane"])
    ap.add_argument("--reference-bin", default="", help="(H2O)8: reuse this ref_driver rhf output")
    a = ap.parse_args()
    if a.only in (None, "propane"):
        propane_exact()
    if a.only in (None, "h2o16"):
        h2o16_rows()
    if a.only in (None, "h2o8"):
        h2o8(not a.no_reference, a.reference_bin)


if __name__ == "__main__":
    main()
