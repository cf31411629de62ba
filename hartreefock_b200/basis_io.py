"""NWChem-format basis files and molecule -> shell tables.

Reads the same format as Chemistry::Basis::Load (Basis.cpp:15-84): lines
`<Element> <letters>` open a shell ('S', 'P', 'SP', 'D' ...), the following
number lines hold an exponent and one contraction coefficient per letter;
'#', 'BASIS', 'END' and blank lines are skipped.  An SP line becomes two
engine shells (L = 0, then L = 1) sharing exponents, with the s function
ahead of px, py, pz in the AO order as in AddShell / AddOrbitals
(Atom.h:31-38, PrimitiveShell.cpp:181-244).
"""
from __future__ import annotations

import os
import re
from dataclasses import dataclass

import numpy as np

BASIS_DIR = os.path.join(os.path.dirname(os.path.abspath(__file__)), "basis")
BASIS_FILES = {"sto-3g": "sto-3g.nw", "6-31g": "6-31g.nw", "6-31g*": "6-31g_st.nw", "6-31+g**": "6-31+g_st_st.nw"}

ELEMENTS = ["H", "He", "Li", "Be", "B", "C", "N", "O", "F", "Ne"]
_L = {"s": 0, "p": 1, "d": 2, "f": 3, "g": 4, "h": 5}


def basis_path(name: str) -> str:
    """Path of a bundled basis by name ('sto-3g', '6-31g', '6-31g*', '6-31+g**'),
    or `name` itself if it is a file."""
    if os.path.isfile(name):
        return name
    key = name.lower()
    if key not in BASIS_FILES:
        raise KeyError(f"unknown basis {name!r}; bundled: {sorted(BASIS_FILES)}")
    return os.path.join(BASIS_DIR, BASIS_FILES[key])


@dataclass
class BasisShell:
    letters: str
    exponents: list
    coefs: list  # one list per letter


def read_basis(path: str) -> dict:
    """{Z: [BasisShell, ...]} in file order."""
    ignore = re.compile(r"^\s*(#|BASIS|END).*$|^\s*$")
    number = re.compile(r"[+-]?[0-9]*\.?[0-9]+((E|D)[+-][0-9]+)?")
    shell_re = re.compile(r"^(\w+)\s+(\w+)\s*$")
    out: dict = {}
    cur = None
    with open(path) as fh:
        for line in fh:
            line = line.rstrip("\r\n")
            if ignore.match(line):
                continue
            m = shell_re.match(line)
            if m:
                sym = m.group(1)
                if sym not in ELEMENTS:
                    raise ValueError(f"{path}: unknown element {sym!r}")
                z = ELEMENTS.index(sym) + 1
                cur = BasisShell(m.group(2), [], [[] for _ in m.group(2)])
                out.setdefault(z, []).append(cur)
                continue
            nums = [float(x.group(0).replace("D", "E")) for x in number.finditer(line)]
            if cur is None or not nums:
                continue
            cur.exponents.append(nums[0])
            for i, c in enumerate(nums[1:1 + len(cur.letters)]):
                cur.coefs[i].append(c)
    return out


@dataclass
class ShellTable:
    """Structure-of-arrays shell table in the engine's (hfg_shells) layout."""
    center: np.ndarray       # (nshells, 3) float64, bohr
    L: np.ndarray            # int32
    nprim: np.ndarray        # int32
    prim_offset: np.ndarray  # int32
    ao_offset: np.ndarray    # int32
    exponent: np.ndarray     # float64
    coefficient: np.ndarray  # float64
    nbf: int
    atom_of_shell: np.ndarray
    max_l: int


def shell_table(Z, xyz, basis: str) -> ShellTable:
    basis_data = read_basis(basis_path(basis))
    xyz = np.asarray(xyz, dtype=np.float64).reshape(-1, 3)
    center, L, nprim, poff, aoff, expo, coef, atom = [], [], [], [], [], [], [], []
    ao = 0
    for a, z in enumerate(Z):
        if z not in basis_data:
            raise KeyError(f"basis {basis!r} has no element Z={z}")
        for sh in basis_data[z]:
            for li, letter in enumerate(sh.letters.lower()):
                l = _L[letter]
                center.append(xyz[a])
                L.append(l)
                nprim.append(len(sh.exponents))
                poff.append(len(expo))
                aoff.append(ao)
                atom.append(a)
                expo.extend(sh.exponents)
                coef.extend(sh.coefs[li])
                ao += (l + 1) * (l + 2) // 2
    return ShellTable(np.array(center, dtype=np.float64).reshape(-1, 3), np.array(L, dtype=np.int32),
                      np.array(nprim, dtype=np.int32), np.array(poff, dtype=np.int32),
                      np.array(aoff, dtype=np.int32), np.array(expo, dtype=np.float64),
                      np.array(coef, dtype=np.float64), ao, np.array(atom, dtype=np.int32),
                      int(max(L)) if L else 0)


def nuclear_repulsion(Z, xyz) -> float:
    """Molecule::NuclearRepulsionEnergy (Molecule.cpp:75-85)."""
    xyz = np.asarray(xyz, dtype=np.float64).reshape(-1, 3)
    e = 0.0
    for i in range(len(Z)):
        for j in range(i + 1, len(Z)):
            e += Z[i] * Z[j] / float(np.linalg.norm(xyz[i] - xyz[j]))
    return e
