"""CPU oracle for the ERI / Fock-build path -- TEST INFRASTRUCTURE ONLY.

Imported by tests/, ``__graft_entry__.smoke()`` and ``bench.py``'s
cpu_baseline / reference legs as the checker; the product package never
imports it.  Python glue over the plain-C restatement in ``eri_oracle.c``
plus a numpy restatement of the reference's SCF loop.  Every function cites
the reference file:line it follows (aromanro/HartreeFock, HartreeFock/).

Parity is pinned against the reference itself: ``oracle/_ref/ref_driver``
(the reference's own classes compiled headless by ``oracle/Makefile``) wrote
the fixtures in ``tests/golden/``; ``tests/test_oracle.py`` checks this
module against them.
"""
from __future__ import annotations

import ctypes
import math
import os
import re
import struct
import subprocess
from dataclasses import dataclass, field

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REF_DIR = os.path.join(HERE, "_ref")
LIB_PATH = os.path.join(REF_DIR, "liboracle.so")
DRIVER_PATH = os.path.join(REF_DIR, "ref_driver")

# ----------------------------------------------------------------------------
# basis sets: NWChem-format parser restating Chemistry::Basis::Load
# (Basis.cpp:15-84, LoadShell :118-158, GetNumberOfGaussiansInOrbital :87-115)
# ----------------------------------------------------------------------------
_ELEMENTS = ["H", "He", "Li", "Be", "B", "C", "N", "O", "F", "Ne", "Na", "Mg", "Al", "Si", "P", "S", "Cl", "Ar",
             "K", "Ca", "Sc", "Ti", "V", "Cr", "Mn", "Fe", "Co", "Ni", "Cu", "Zn", "Ga", "Ge", "As", "Se", "Br",
             "Kr", "Rb", "Sr", "Y", "Zr", "Nb", "Mo", "Tc", "Ru", "Rh", "Pd", "Ag", "Cd", "In", "Sn", "Sb", "Te",
             "I", "Xe", "Cs", "Ba", "La"]  # ChemUtils.cpp:8-15
_LETTER_L = {"s": 0, "p": 1, "d": 2, "f": 3, "g": 4, "h": 5}


def z_for_symbol(sym: str) -> int:
    return _ELEMENTS.index(sym) + 1 if sym in _ELEMENTS else 0


@dataclass
class Shell:
    """A basis-file shell line ('S', 'SP', 'D' ...) with its exponents and one
    coefficient column per letter (Basis.cpp:52-83)."""
    letters: str
    exponents: list = field(default_factory=list)
    coefs: list = field(default_factory=list)  # coefs[letter_index][primitive]


def load_basis(path: str) -> dict:
    """Return {Z: [Shell, ...]} in file order."""
    ignore = re.compile(r"^\s*(#|BASIS|END).*$|^\s*$")
    number = re.compile(r"[+-]?[0-9]*\.?[0-9]+((E|D)[+-][0-9]+)?")
    shell_re = re.compile(r"^(\w+)\s+(\w+)\s*$")
    atoms: dict = {}
    order: list = []
    cur = None
    with open(path) as fh:
        for line in fh:
            line = line.rstrip("\n").rstrip("\r")
            if ignore.match(line):
                continue
            m = shell_re.match(line)
            if m:
                z = z_for_symbol(m.group(1))
                if not order or order[-1] != z:
                    order.append(z)
                    atoms.setdefault(z, [])
                cur = Shell(m.group(2))
                cur.coefs = [[] for _ in cur.letters]
                atoms[z].append(cur)
                continue
            nums = [float(x.group(0).replace("D", "E")) for x in number.finditer(line)]
            if not nums or cur is None:
                continue
            cur.exponents.append(nums[0])
            for li, c in enumerate(nums[1:1 + len(cur.letters)]):
                cur.coefs[li].append(c)
    return atoms


def cartesian_components(L: int):
    """AddOrbitalsInCanonicalOrder (PrimitiveShell.cpp:232-244) with
    CanonicalIncrement (QuantumNumbers.h:60-80): xx, xy, xz, yy, yz, zz ..."""
    out = []
    l, m, n = L, 0, 0
    while True:
        out.append((l, m, n))
        if n == L:
            break
        if m > 0:
            m, n = m - 1, n + 1
        elif l > 0:
            l, m, n = l - 1, L - (l - 1), 0
    return out


def double_factorial(n: int) -> float:
    r = 1.0
    while n > 1:
        r *= n
        n -= 2
    return r


def primitive_norm(alpha: float, lmn) -> float:
    """GaussianOrbital::getNormalizationFactor (GaussianOrbital.cpp:25-30), with
    (2l-1)!! = 1 for l = 0 as on the reference's native (LLP64) platform."""
    l, m, n = lmn
    L = l + m + n
    return ((2 * alpha / math.pi) ** 0.75 * (4 * alpha) ** (L / 2.0)
            / math.sqrt(double_factorial(2 * l - 1) * double_factorial(2 * m - 1) * double_factorial(2 * n - 1)))


class OrcFunction(ctypes.Structure):
    _fields_ = [("center", ctypes.c_double * 3), ("l", ctypes.c_int), ("m", ctypes.c_int), ("n", ctypes.c_int),
                ("id", ctypes.c_int), ("shell_id", ctypes.c_int), ("prim_offset", ctypes.c_int),
                ("nprim", ctypes.c_int)]


class OrcPrimitive(ctypes.Structure):
    _fields_ = [("alpha", ctypes.c_double), ("coef", ctypes.c_double), ("norm", ctypes.c_double)]


@dataclass
class Molecule:
    """Atoms (Z, position in bohr) expanded against a basis the way
    Molecule::Init / SetIDs do (Molecule.cpp:41-72, 127-140)."""
    Z: list
    xyz: np.ndarray
    basis_path: str
    alpha_electrons: int = 0
    beta_electrons: int = 0

    def __post_init__(self):
        self.xyz = np.asarray(self.xyz, dtype=np.float64).reshape(-1, 3)
        basis = load_basis(self.basis_path)
        funcs, prims = [], []
        shell_id = 0
        self.max_l = 0
        for a, z in enumerate(self.Z):
            for sh in basis[z]:
                for li, letter in enumerate(sh.letters.lower()):
                    L = _LETTER_L[letter]
                    self.max_l = max(self.max_l, L)
                    for lmn in cartesian_components(L):
                        f = OrcFunction()
                        f.center[:] = self.xyz[a]
                        f.l, f.m, f.n = lmn
                        f.id = len(funcs)
                        f.shell_id = shell_id
                        f.prim_offset = len(prims)
                        f.nprim = len(sh.exponents)
                        for e, c in zip(sh.exponents, sh.coefs[li]):
                            prims.append((e, c, primitive_norm(e, lmn)))
                        funcs.append(f)
                shell_id += 1
        self.nbf = len(funcs)
        self.functions = (OrcFunction * len(funcs))(*funcs)
        self.primitives = (OrcPrimitive * len(prims))(*[OrcPrimitive(e, c, nf) for e, c, nf in prims])
        nel = int(sum(self.Z))
        if self.alpha_electrons == 0 and self.beta_electrons == 0:
            self.alpha_electrons = nel // 2
            self.beta_electrons = nel - nel // 2

    @property
    def max_boys_m(self) -> int:
        # IntegralsRepository::getBoysFunctions (IntegralsRepository.cpp:334-337)
        return 4 * self.max_l + 1

    def nuclear_repulsion(self) -> float:
        """Molecule::NuclearRepulsionEnergy (Molecule.cpp:75-85)."""
        e = 0.0
        for i in range(len(self.Z)):
            for j in range(i + 1, len(self.Z)):
                e += self.Z[i] * self.Z[j] / float(np.linalg.norm(self.xyz[i] - self.xyz[j]))
        return e


# ----------------------------------------------------------------------------
# C restatement bindings
# ----------------------------------------------------------------------------
_lib = None


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            subprocess.run(["make", "-C", HERE, "port"], check=True, capture_output=True)
        L = ctypes.CDLL(LIB_PATH)
        pd = ctypes.POINTER(ctypes.c_double)
        L.orc_boys_single.restype = ctypes.c_double
        L.orc_boys_single.argtypes = [ctypes.c_double, ctypes.c_double]
        L.orc_boys.argtypes = [ctypes.c_int, ctypes.c_double, pd]
        L.orc_eri.restype = ctypes.c_double
        L.orc_eri.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int, ctypes.c_int, ctypes.c_int,
                              ctypes.c_int, ctypes.c_int, ctypes.c_int]
        L.orc_packed_size.restype = ctypes.c_int64
        L.orc_packed_size.argtypes = [ctypes.c_int]
        L.orc_eri_packed.argtypes = [ctypes.c_int, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int, ctypes.c_int, pd]
        L.orc_g_rhf.argtypes = [ctypes.c_int, pd, pd, pd]
        L.orc_g_uhf.argtypes = [ctypes.c_int, pd, pd, pd, pd, pd]
        L.orc_eri_diagonal.argtypes = [ctypes.c_int, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int, ctypes.c_int, pd]
        L.orc_g_rhf_rows.argtypes = [ctypes.c_int, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int, ctypes.c_int, pd,
                                     ctypes.POINTER(ctypes.c_int), ctypes.c_int, pd]
        L.orc_one_electron.argtypes = [ctypes.c_int, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int, pd,
                                       ctypes.POINTER(ctypes.c_int), ctypes.c_int, pd, pd, pd]
        _lib = L
    return _lib


def _p(a: np.ndarray):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_double))


def boys(max_m: int, T: float) -> np.ndarray:
    out = np.zeros(max_m + 1)
    lib().orc_boys(max_m, T, _p(out))
    return out


def two_index(i, j):
    return j * (j + 1) // 2 + i if i < j else i * (i + 1) // 2 + j


def packed_index(i, j, k, l):
    """IntegralsRepository::GetElectronElectronIndex (IntegralsRepository.h:151-162)."""
    return two_index(two_index(i, j), two_index(k, l))


def eri(mol: Molecule, i, j, k, l, exact_et=False) -> float:
    return lib().orc_eri(ctypes.byref(mol.functions), ctypes.byref(mol.primitives), i, j, k, l, mol.max_boys_m,
                         int(exact_et))


def eri_packed(mol: Molecule, exact_et=False) -> np.ndarray:
    n = mol.nbf
    out = np.zeros(lib().orc_packed_size(n))
    lib().orc_eri_packed(n, ctypes.byref(mol.functions), ctypes.byref(mol.primitives), mol.max_boys_m,
                         int(exact_et), _p(out))
    return out


def g_rhf(n, packed, P):
    G = np.zeros((n, n))
    lib().orc_g_rhf(n, _p(packed), _p(np.ascontiguousarray(P)), _p(G))
    return G


def screened_quartets(mol: Molecule, threshold: float) -> dict:
    """Size of a direct Fock build under Schwarz screening: shells are the
    functions of one (shell ID, L) (the s and p parts of an SP shell are two
    shells), Q_ab = sqrt(max |(ij|ij)|) over the function pairs of the shell
    pair (exact electron transfer), and a shell quartet {ab, cd} is kept when
    Q_ab Q_cd >= threshold.  Returns the 8-fold unique function quartets kept
    and in total."""
    n = mol.nbf
    diag = np.zeros(n * (n + 1) // 2)
    lib().orc_eri_diagonal(n, ctypes.byref(mol.functions), ctypes.byref(mol.primitives), mol.max_boys_m, 1,
                           _p(diag))
    key = [(f.shell_id, f.l + f.m + f.n) for f in mol.functions]
    shells = []
    for i, k in enumerate(key):
        if i == 0 or k != key[i - 1]:
            shells.append([])
        shells[-1].append(i)
    Q, fcount = [], []
    for a in range(len(shells)):
        for b in range(a + 1):
            m = 0.0
            for i in shells[a]:
                for j in shells[b]:
                    m = max(m, abs(diag[two_index(i, j)]))
            Q.append(np.sqrt(m))
            na, nb = len(shells[a]), len(shells[b])
            fcount.append(na * (na + 1) // 2 if a == b else na * nb)
    Q, fcount = np.array(Q), np.array(fcount, dtype=np.float64)
    order = np.argsort(-Q)
    Q, fcount = Q[order], fcount[order]
    prefix = np.concatenate([[0.0], np.cumsum(fcount)])
    kept = 0.0
    for p_ in range(len(Q)):
        if Q[p_] <= 0:
            break
        # partners q < p_ (larger or equal bound) with Q_p Q_q >= threshold: all of them
        # when Q_p^2 >= threshold, else a prefix of the sorted list
        hi = int(np.searchsorted(-Q, -(threshold / Q[p_]), side="right"))
        m = min(hi, p_)
        kept += fcount[p_] * prefix[m]
        if Q[p_] * Q[p_] >= threshold:
            kept += fcount[p_] * (fcount[p_] + 1) / 2
    npair = n * (n + 1) // 2
    return {"kept": int(round(kept)), "total": npair * (npair + 1) // 2}


def g_rhf_rows(mol: Molecule, P, rows, exact_et=False) -> np.ndarray:
    """Rows of the RHF two-electron matrix G[P] straight from the contracted
    ERIs (no stored table): out[r] = G[rows[r], :]."""
    n = mol.nbf
    rows = np.ascontiguousarray(rows, dtype=np.int32)
    out = np.zeros((len(rows), n))
    lib().orc_g_rhf_rows(n, ctypes.byref(mol.functions), ctypes.byref(mol.primitives), mol.max_boys_m,
                         int(exact_et), _p(np.ascontiguousarray(P, dtype=np.float64)),
                         rows.ctypes.data_as(ctypes.POINTER(ctypes.c_int)), len(rows), _p(out))
    return out


def g_uhf(n, packed, Pa, Pb):
    Ga, Gb = np.zeros((n, n)), np.zeros((n, n))
    lib().orc_g_uhf(n, _p(packed), _p(np.ascontiguousarray(Pa)), _p(np.ascontiguousarray(Pb)), _p(Ga), _p(Gb))
    return Ga, Gb


def unpack_eri(packed, n):
    """full[m, n, l, s] = (mn|ls) from the 8-fold packed table
    (IntegralsRepository.h:151-162)."""
    idx = np.arange(n)
    ij = np.maximum(idx[:, None], idx[None, :])
    ij = ij * (ij + 1) // 2 + np.minimum(idx[:, None], idx[None, :])
    p, q = ij[:, :, None, None], ij[None, None, :, :]
    return np.asarray(packed)[np.maximum(p, q) * (np.maximum(p, q) + 1) // 2 + np.minimum(p, q)]


class MoCache:
    """MolecularOrbitalsIntegralsRepository (IntegralsRepository.h:190-291)
    restated literally: four quarter-transform levels, each cached in a dict
    keyed by the four orbital indices only -- not by the coefficient matrix
    the value was computed with.  ``eri`` is the full AO table, C column
    ``p`` the MO p (C[AO, MO])."""

    def __init__(self, eri):
        self.eri = eri
        self.levels = ({}, {}, {}, {})

    def _l1(self, o1, o2, o3, o4, C):  # IntegralsRepository.h:237-251
        key = (o1, o2, o3, o4)
        if key not in self.levels[0]:
            self.levels[0][key] = float(C[:, o4] @ self.eri[o1, o2, o3, :])
        return self.levels[0][key]

    def _l2(self, o1, o2, o3, o4, C):  # :253-268
        key = (o1, o2, o3, o4)
        if key not in self.levels[1]:
            self.levels[1][key] = sum(C[l, o3] * self._l1(o1, o2, l, o4, C) for l in range(C.shape[1]))
        return self.levels[1][key]

    def _l3(self, o1, o2, o3, o4, C):  # :270-284
        key = (o1, o2, o3, o4)
        if key not in self.levels[2]:
            self.levels[2][key] = sum(C[nu, o2] * self._l2(o1, nu, o3, o4, C) for nu in range(C.shape[1]))
        return self.levels[2][key]

    def get(self, o1, o2, o3, o4, C):  # :198-234
        key = (o1, o2, o3, o4)
        if key not in self.levels[3]:
            self.levels[3][key] = sum(C[mu, o1] * self._l3(mu, o2, o3, o4, C) for mu in range(C.shape[1]))
        return self.levels[3][key]


def mp2_uhf(eri, Cp, ep, nplus, Cm, em, nminus):
    """UnrestrictedHartreeFock::CalculateMp2Energy (UnrestrictedHartreeFock.cpp:295-375):
    0.25 (S+ + S-) through ONE MoCache, S+ first, so S- reuses what S+
    cached with C+.  Pure-Python loops: small cases only."""
    n = Cp.shape[0]
    repo = MoCache(eri)

    def spin_sum(C, e, nocc):  # CalculateMp2EnergyPlus :309-338 / Minus :340-369
        s = 0.0
        for i in range(nocc):
            for j in range(nocc):
                for a in range(nocc, n):
                    for b in range(nocc, n):
                        v = repo.get(i, a, j, b, C)
                        s += v * v / (e[i] + e[j] - e[a] - e[b])
        return s

    total = spin_sum(Cp, ep, nplus)
    total += spin_sum(Cm, em, nminus)
    return 0.25 * total


def one_electron(mol: Molecule):
    n = mol.nbf
    S, T, V = np.zeros((n, n)), np.zeros((n, n)), np.zeros((n, n))
    xyz = np.ascontiguousarray(mol.xyz)
    z = (ctypes.c_int * len(mol.Z))(*mol.Z)
    lib().orc_one_electron(n, ctypes.byref(mol.functions), ctypes.byref(mol.primitives), len(mol.Z), _p(xyz), z,
                           mol.max_boys_m, _p(S), _p(T), _p(V))
    return S, T, V


# ----------------------------------------------------------------------------
# SCF restatement (numpy): HartreeFockAlgorithm / RestrictedHartreeFock /
# UnrestrictedHartreeFock / DIIS, with the reference's conventions.
# ----------------------------------------------------------------------------
ENERGY_CONV_DIIS, ENERGY_CONV, RMSD_CONV, DIIS_CONV = 1e-11, 1e-13, 1e-10, 1e-10  # Constants.h:6-10


class _Diis:
    """DIIS.h:9-96: keep 6, first extrapolation with 5, B solved in least squares."""

    def __init__(self, keep=6, first=5):
        self.keep, self.first = keep, first
        self.errors, self.values = [], []

    def add(self, value, error):
        self.errors.append(error)
        self.values.append(value)
        if len(self.errors) > self.keep:
            self.errors.pop(0)
            self.values.pop(0)
        return len(self.errors) >= self.first

    def estimate(self):
        n = len(self.errors)
        B = np.zeros((n + 1, n + 1))
        last = 0.0
        for i in range(n):
            for j in range(i + 1):
                B[i, j] = B[j, i] = float(np.sum(self.errors[i] * self.errors[j]))
            if i in (n - 1, n - 2):
                last += B[i, i]
            B[n, i] = B[i, n] = 1.0
        rhs = np.zeros(n + 1)
        rhs[n] = 1.0
        c = np.linalg.lstsq(B, rhs, rcond=None)[0]
        return sum(c[i] * self.values[i] for i in range(n)), math.sqrt(last)


def _scf_rhf(S, h, enuc, fock_g, nocc, alpha, init_guess, use_diis, max_diis_iterations, post_diis,
             max_iterations):
    n = h.shape[0]
    s, U = np.linalg.eigh(S)
    V = U @ np.diag(1.0 / np.sqrt(s)) @ U.T
    V = 0.5 * (V + V.T)
    P = np.zeros((n, n))
    diis = _Diis()
    st = {"use_diis": use_diis, "last_err": 0.0, "energy": math.inf, "iters": 0}

    def step(it):
        nonlocal P
        if it == 0:  # RestrictedHartreeFock.cpp:175-186
            if init_guess > 0:
                d = np.diag(h)
                F = init_guess * S * (d[:, None] + d[None, :]) * 0.5
            else:
                F = h.copy()
        else:
            F = h + fock_g(P)
        F = 0.5 * (F + F.T)
        used = False
        if st["use_diis"] and it and it < max_diis_iterations:  # RestrictedHartreeFock.cpp:35-58
            err = S @ P @ F - F @ P @ S
            if diis.add(F, err):
                F, st["last_err"] = diis.estimate()
                used = True
        else:
            st["last_err"] = 0.0
        e, Cp = np.linalg.eigh(V.T @ F @ V)
        C = V @ Cp
        Pn = 2.0 * C[:, :nocc] @ C[:, :nocc].T
        # CalculateEnergy (RestrictedHartreeFock.cpp:209-249)
        st["energy"] = 0.5 * float(np.sum(Pn * h)) + float(np.sum(e[:nocc])) + enuc
        rms = math.sqrt(float(np.sum((Pn - P) ** 2)))
        P = Pn if used else alpha * Pn + (1 - alpha) * P
        st["iters"] += 1
        return rms

    converged = _drive(step, st, max_iterations, max_diis_iterations, post_diis)
    return {"energy": st["energy"], "density": P, "converged": converged, "iterations": st["iters"]}


def _scf_uhf(S, h, enuc, fock_g, na, nb, alpha, init_guess, use_diis, max_diis_iterations, post_diis,
             max_iterations, add_asymmetry, asymmetry):
    n = h.shape[0]
    s, U = np.linalg.eigh(S)
    V = U @ np.diag(1.0 / np.sqrt(s)) @ U.T
    V = 0.5 * (V + V.T)
    Pa, Pb = np.zeros((n, n)), np.zeros((n, n))
    da, db = _Diis(), _Diis()
    st = {"use_diis": use_diis, "last_err": 0.0, "energy": math.inf, "iters": 0}

    def step(it):
        nonlocal Pa, Pb
        if it == 0:  # UnrestrictedHartreeFock.cpp:199-222
            if init_guess > 0:
                d = np.diag(h)
                Fa = init_guess * S * (d[:, None] + d[None, :]) * 0.5
            else:
                Fa = h.copy()
            Fb = Fa.copy()
            if add_asymmetry and n > 1:
                Fa[0, 1] += asymmetry
                Fa[1, 0] = Fa[0, 1]
        else:
            Ga, Gb = fock_g(Pa, Pb)
            Fa, Fb = h + Ga, h + Gb
        used = False
        if st["use_diis"] and it and it < max_diis_iterations:  # UnrestrictedHartreeFock.cpp:62-84
            da.add(Fa, S @ Pa @ Fa - Fa @ Pa @ S)
            if db.add(Fb, S @ Pb @ Fb - Fb @ Pb @ S):
                Fb, e1 = db.estimate()
                Fa, e2 = da.estimate()
                st["last_err"] = e1 + e2
                used = True
        else:
            st["last_err"] = 0.0
        ea, Ca = np.linalg.eigh(V.T @ Fa @ V)
        eb, Cb = np.linalg.eigh(V.T @ Fb @ V)
        Ca, Cb = V @ Ca, V @ Cb
        Pan = Ca[:, :na] @ Ca[:, :na].T
        Pbn = Cb[:, :nb] @ Cb[:, :nb].T
        # CalculateEnergy (UnrestrictedHartreeFock.cpp:246-293)
        st["energy"] = 0.5 * (float(np.sum((Pan + Pbn) * h)) + float(np.sum(ea[:na])) + float(np.sum(eb[:nb]))) + enuc
        rms = math.sqrt(float(np.sum((Pan - Pa) ** 2)) + float(np.sum((Pbn - Pb) ** 2)))
        if used:
            Pa, Pb = Pan, Pbn
        else:
            Pa, Pb = alpha * Pan + (1 - alpha) * Pa, alpha * Pbn + (1 - alpha) * Pb
        st["iters"] += 1
        return rms

    converged = _drive(step, st, max_iterations, max_diis_iterations, post_diis)
    return {"energy": st["energy"], "density_alpha": Pa, "density_beta": Pb, "converged": converged,
            "iterations": st["iters"]}


def _drive(step, st, max_iterations, max_diis_iterations, post_diis):
    """FirstIterations / SelfConsistentIterations / NormalIterations
    (HartreeFockAlgorithm.cpp:129-192)."""
    prev = math.inf
    converged = False
    it = 0
    while it < max_iterations:
        rms = step(it)
        cur = st["energy"]
        if (abs(prev - cur) <= (ENERGY_CONV_DIIS if st["use_diis"] else ENERGY_CONV) and rms < RMSD_CONV
                and st["last_err"] < DIIS_CONV):
            converged = True
            break
        prev = cur
        it += 1
    if st["use_diis"] and it < max_diis_iterations and converged and post_diis:
        st["use_diis"] = False
        for i in range(post_diis):
            step(it + i)
            prev = st["energy"]
        it += post_diis
        st["use_diis"] = True
    if not converged:
        while it < max_iterations:
            rms = step(it)
            cur = st["energy"]
            if abs(prev - cur) <= ENERGY_CONV and rms < RMSD_CONV:
                converged = True
                break
            prev = cur
            it += 1
    return converged


def run_scf(mol: Molecule, unrestricted=False, alpha=0.75, init_guess=0.75, use_diis=True, post_diis=500,
            packed=None, exact_et=False):
    """Full oracle SCF: one-electron matrices, packed ERIs, then the loop."""
    S, T, V = one_electron(mol)
    h = T + V
    if packed is None:
        packed = eri_packed(mol, exact_et)
    n = mol.nbf
    enuc = mol.nuclear_repulsion()
    if unrestricted:
        na, nb = mol.beta_electrons, mol.alpha_electrons  # plus = total - floor(total/2)
        r = _scf_uhf(S, h, enuc, lambda a, b: g_uhf(n, packed, a, b), max(na, nb), min(na, nb), alpha,
                     init_guess, use_diis, 1000, post_diis, 3000, True, 0.1)
    else:
        r = _scf_rhf(S, h, enuc, lambda P: g_rhf(n, packed, P), (mol.alpha_electrons + mol.beta_electrons) // 2,
                     alpha, init_guess, use_diis, 1000, post_diis, 3000)
    r["h"], r["S"] = h, S
    return r


# ----------------------------------------------------------------------------
# reference driver (oracle/_ref/ref_driver) -- used to make / refresh fixtures
# ----------------------------------------------------------------------------
def read_records(path: str) -> dict:
    out = {}
    with open(path, "rb") as fh:
        buf = fh.read()
    o = 0
    while o < len(buf):
        (nlen,) = struct.unpack_from("<I", buf, o)
        o += 4
        name = buf[o:o + nlen].decode()
        o += nlen
        (cnt,) = struct.unpack_from("<Q", buf, o)
        o += 8
        out[name] = np.frombuffer(buf, dtype="<f8", count=cnt, offset=o).copy()
        o += 8 * cnt
    return out


def run_reference(mol: Molecule, mode: str, out_path: str, alpha=0.75, init_guess=0.75, use_diis=True,
                  post_diis=500, extra: str = "", timeout=3600, driver: str = "") -> dict:
    """Runs the reference's classes compiled headless (oracle/_ref/ref_driver,
    or `driver`: the drop-in builds ref_driver_gpu / ref_driver_gpu_direct)."""
    lines = [f"basis {mol.basis_path}"]
    for z, p in zip(mol.Z, mol.xyz):
        lines.append(f"atom {int(z)} {float(p[0]):.17g} {float(p[1]):.17g} {float(p[2]):.17g}")
    lines += [f"alpha {float(alpha):.17g}", f"initguess {float(init_guess):.17g}", f"diis {int(use_diis)}",
              f"postdiis {int(post_diis)}",
              f"mode {mode}", f"out {out_path}", extra]
    r = subprocess.run([driver or DRIVER_PATH], input="\n".join(lines) + "\n", capture_output=True, text=True,
                       timeout=timeout)
    if r.returncode != 0:
        raise RuntimeError(f"ref_driver failed: {r.stderr}")
    if mode == "bench":
        return {"stdout": r.stdout}
    return read_records(out_path)
