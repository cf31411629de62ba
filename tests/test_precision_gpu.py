"""The precision form of the direct Fock build (density screening, FP32
below the mixed cutoff, incremental builds from the density difference, an
all-FP64 finish) against the plain FP64 form of the same engine, which the
parity tests pin to the reference."""
import numpy as np
import pytest
import scipy.linalg

from hartreefock_b200 import engine as E
from hartreefock_b200 import molecules, scf

pytestmark = pytest.mark.gpu

BASIS = "6-31g*"


def _cluster(n, seed=0):
    Z, xyz = molecules.water_cluster(n, seed=seed)
    return list(Z), xyz


def _core_guess_density(Z, xyz, basis=BASIS):
    """Closed-shell density of the core-Hamiltonian guess (host one-electron
    code + scipy): a density with the structure of a real one."""
    S, h = scf.one_electron(Z, xyz, basis)
    _, C = scipy.linalg.eigh(h, S)
    nocc = sum(Z) // 2
    return 2.0 * C[:, :nocc] @ C[:, :nocc].T


def _perturbation(n, scale, seed):
    rng = np.random.default_rng(seed)
    A = rng.normal(size=(n, n)) * scale
    return A + A.T


@pytest.fixture(scope="module")
def water6():
    Z, xyz = _cluster(6)
    P = _core_guess_density(Z, xyz)
    plain = E.Engine(Z, xyz, BASIS)
    return Z, xyz, P, plain, plain.fock_rhf(P)


def test_density_screening_matches_plain(water6):
    Z, xyz, P, _, G0 = water6
    eng = E.Engine(Z, xyz, BASIS, density_screening=True)
    G = eng.fock_rhf(P)
    st = eng.stats()
    # every skipped quartet contributes below 1e-12 per element it touches
    assert np.abs(G - G0).max() < 1e-9
    assert st["fp32_shell_quartets"] == 0
    assert 0 < st["fp64_shell_quartets"] < st["shell_quartets"]


def test_incremental_build_matches_full_build(water6):
    Z, xyz, P, plain, _ = water6
    n = P.shape[0]
    P2 = P + _perturbation(n, 1e-3, 7)
    P3 = P2 + _perturbation(n, 1e-5, 8)
    eng = E.Engine(Z, xyz, BASIS, incremental=True)
    eng.fock_rhf(P)
    kept_full = eng.stats()["fp64_shell_quartets"]
    eng.fock_rhf(P2)
    G3 = eng.fock_rhf(P3)
    kept_small_step = eng.stats()["fp64_shell_quartets"]
    assert np.abs(G3 - plain.fock_rhf(P3)).max() < 1e-9
    # a small density change keeps fewer quartets than the full density
    assert kept_small_step < kept_full
    # after a reset the build starts again from the full density
    eng.fock_reset()
    assert np.abs(eng.fock_rhf(P2) - plain.fock_rhf(P2)).max() < 1e-9


def test_mixed_precision_error_is_fp32_sized(water6):
    Z, xyz, P, _, G0 = water6
    hi = E.Engine(Z, xyz, BASIS, density_screening=True)
    hi.fock_rhf(P)
    kept = hi.stats()["fp64_shell_quartets"]
    mix = E.Engine(Z, xyz, BASIS, density_screening=True, mixed_cutoff=1e-4)
    G = mix.fock_rhf(P)
    st = mix.stats()
    # the FP64 and FP32 kernels split the kept quartets between them
    assert st["fp32_shell_quartets"] > 0 and st["fp64_shell_quartets"] > 0
    assert st["fp32_shell_quartets"] + st["fp64_shell_quartets"] == kept
    err = np.abs(G - G0).max()
    # FP32 recursions on quartets bounded by 1e-4: errors of order
    # 1e-4 * 2^-24 per quartet, summed over the kept quartets
    assert 0 < err < 1e-6, err
    # the cutoff can be changed between builds: 0 returns to all-FP64
    mix.set_mixed_cutoff(0.0)
    assert np.abs(mix.fock_rhf(P) - G0).max() < 1e-9
    assert mix.stats()["fp32_shell_quartets"] == 0


def test_mixed_uhf_matches_plain():
    Z, xyz = _cluster(3, seed=2)
    Pt = _core_guess_density(Z, xyz)
    n = Pt.shape[0]
    Pa = 0.5 * Pt + _perturbation(n, 1e-3, 3)
    Pb = 0.5 * Pt - _perturbation(n, 1e-3, 3)
    ga0, gb0 = E.Engine(Z, xyz, BASIS).fock_uhf(Pa, Pb)
    eng = E.Engine(Z, xyz, BASIS, incremental=True, mixed_cutoff=1e-4)
    eng.fock_uhf(0.9 * Pa, 0.9 * Pb)
    ga, gb = eng.fock_uhf(Pa, Pb)
    assert np.abs(ga - ga0).max() < 1e-6 and np.abs(gb - gb0).max() < 1e-6
    assert eng.stats()["fp32_shell_quartets"] > 0


def test_mixed_scf_matches_plain_fp64():
    """(H2O)4 / 6-31G* RHF: the precision form (FP32 below 1e-4, incremental
    builds, two all-FP64 iterations at the end) lands within 1e-6 Eh of the
    plain FP64 SCF run to the reference's thresholds."""
    Z, xyz = _cluster(4, seed=1)
    kw = dict(alpha=0.75, init_guess=0.75, post_diis=0)
    ref = scf.run_scf(Z, xyz, BASIS, **kw)
    mix = scf.run_scf(Z, xyz, BASIS, mixed_cutoff=1e-4, **kw)
    assert ref["converged"] and mix["converged"]
    assert abs(mix["energy"] - ref["energy"]) < 1e-6
    assert np.abs(mix["density"] - ref["density"]).max() < 1e-4
    assert mix["mixed_steps"] > 0 and mix["fp32_quartets"] > 0
    assert mix["fock_builds"] == mix["mixed_steps"] + 2  # exactly two FP64 builds at the end
    assert mix["iterations"] < ref["iterations"]


def test_mixed_scf_converged_to_reference_thresholds():
    """With fp64_final_converge the FP64 phase runs on to the reference's own
    convergence test: the energy then agrees with the plain form to 1e-9."""
    Z, xyz = _cluster(3, seed=4)
    kw = dict(alpha=0.75, init_guess=0.75, post_diis=0)
    ref = scf.run_scf(Z, xyz, BASIS, **kw)
    mix = scf.run_scf(Z, xyz, BASIS, mixed_cutoff=1e-4, fp64_final_converge=True, **kw)
    assert ref["converged"] and mix["converged"]
    assert abs(mix["energy"] - ref["energy"]) < 1e-9
    assert np.abs(mix["density"] - ref["density"]).max() < 1e-6


def test_mixed_uhf_scf_matches_plain_fp64():
    Z, xyz = molecules.hydroxyl()
    kw = dict(unrestricted=True, alpha=0.5, init_guess=0.0, post_diis=0)
    ref = scf.run_scf(Z, xyz, "6-31g", **kw)
    mix = scf.run_scf(Z, xyz, "6-31g", mixed_cutoff=1e-4, **kw)
    assert ref["converged"] and mix["converged"]
    assert abs(mix["energy"] - ref["energy"]) < 1e-6
