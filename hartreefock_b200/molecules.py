"""Seeded synthetic molecules for the engine's workloads.

The reference builds molecules by hand (README.md: H2O with H1, H2, O in
bohr) or reads XYZ files (Molecule::LoadXYZ, Molecule.cpp:143-199).  These
generators produce the benchmark systems: rigid water clusters at liquid
density, all-staggered linear alkanes, and the OH / planar CH3 radicals.
Every generator returns (Z list, positions in bohr as an (n, 3) array).
"""
from __future__ import annotations

import math

import numpy as np

BOHR = 0.529177210903  # Angstrom per bohr (Constants.h:4)
AVOGADRO = 6.02214076e23
WATER_MOLAR_MASS = 18.01528  # g/mol

# the README's water (bohr, atom order H1, H2, O)
H2O_README = ([1, 1, 8], np.array([[0.0, 1.43233673, -0.96104039],
                                   [0.0, -1.43233673, -0.96104039],
                                   [0.0, 0.0, 0.24026010]]))


def _rotation_from_quaternion(q: np.ndarray) -> np.ndarray:
    w, x, y, z = q / np.linalg.norm(q)
    return np.array([[1 - 2 * (y * y + z * z), 2 * (x * y - z * w), 2 * (x * z + y * w)],
                     [2 * (x * y + z * w), 1 - 2 * (x * x + z * z), 2 * (y * z - x * w)],
                     [2 * (x * z - y * w), 2 * (y * z + x * w), 1 - 2 * (x * x + y * y)]])


def water_monomer_angstrom(r_oh: float = 0.9572, angle_deg: float = 104.52) -> np.ndarray:
    """O at the origin, both H in the xz plane; rows O, H, H."""
    half = math.radians(angle_deg) / 2
    return np.array([[0.0, 0.0, 0.0],
                     [r_oh * math.sin(half), 0.0, r_oh * math.cos(half)],
                     [-r_oh * math.sin(half), 0.0, r_oh * math.cos(half)]])


def water_cluster_box_angstrom(n: int, density_g_cm3: float = 1.0) -> float:
    """Cube edge holding n waters at the given density: 6.209 A for n = 8."""
    volume_cm3 = n * WATER_MOLAR_MASS / (AVOGADRO * density_g_cm3)
    return volume_cm3 ** (1.0 / 3.0) * 1e8


def water_cluster(n: int, seed: int = 0, min_oo: float = 2.6, max_tries: int = 200000):
    """(H2O)_n: rigid monomers (O-H 0.9572 A, HOH 104.52 deg), orientation
    uniform on SO(3) (unit quaternion from 4 iid normals), O positions uniform
    in a cube sized for 1 g/cm^3, rejection-sampled so every O-O distance is
    at least `min_oo` A.  Atom order O, H, H per monomer."""
    rng = np.random.default_rng(seed)
    edge = water_cluster_box_angstrom(n)
    oxygens: list = []
    tries = 0
    while len(oxygens) < n:
        tries += 1
        if tries > max_tries:
            raise RuntimeError(f"water_cluster({n}): could not place oxygens after {max_tries} tries")
        p = rng.uniform(0.0, edge, size=3)
        if all(np.linalg.norm(p - o) >= min_oo for o in oxygens):
            oxygens.append(p)
    mono = water_monomer_angstrom()
    Z, xyz = [], []
    for o in oxygens:
        R = _rotation_from_quaternion(rng.normal(size=4))
        for z, r in zip((8, 1, 1), mono):
            Z.append(z)
            xyz.append(o + R @ r)
    return Z, np.array(xyz) / BOHR


def alkane(n_carbon: int, r_cc: float = 1.54, r_ch: float = 1.09):
    """Linear all-staggered C_nH_{2n+2} with tetrahedral angles: the carbon
    backbone is a planar zigzag, each carbon carries its hydrogens along the
    remaining tetrahedral directions."""
    tet = math.acos(-1.0 / 3.0)
    # zigzag in the xy plane: successive C-C bonds alternate about the x axis
    half = (math.pi - tet) / 2
    carbons = [np.zeros(3)]
    for i in range(1, n_carbon):
        s = 1 if i % 2 else -1
        carbons.append(carbons[-1] + r_cc * np.array([math.cos(half), s * math.sin(half), 0.0]))
    Z, xyz = [], []
    for i, c in enumerate(carbons):
        Z.append(6)
        xyz.append(c)
    for i, c in enumerate(carbons):
        bonds = []
        if i > 0:
            bonds.append((carbons[i - 1] - c) / np.linalg.norm(carbons[i - 1] - c))
        if i < n_carbon - 1:
            bonds.append((carbons[i + 1] - c) / np.linalg.norm(carbons[i + 1] - c))
        for d in _tetrahedral_completion(bonds, i):
            Z.append(1)
            xyz.append(c + r_ch * d)
    return Z, np.array(xyz) / BOHR


def _tetrahedral_completion(bonds, index):
    """Unit vectors completing a tetrahedron around a centre that already has
    the given bond directions (0, 1 or 2 of them)."""
    if not bonds:  # methane
        return [np.array(v) / math.sqrt(3) for v in ((1, 1, 1), (1, -1, -1), (-1, 1, -1), (-1, -1, 1))]
    if len(bonds) == 1:
        a = bonds[0]
        perp = np.cross(a, [0.0, 0.0, 1.0])
        if np.linalg.norm(perp) < 1e-8:
            perp = np.cross(a, [0.0, 1.0, 0.0])
        perp /= np.linalg.norm(perp)
        perp2 = np.cross(a, perp)
        cos_t = -1.0 / 3.0
        sin_t = math.sqrt(1 - cos_t * cos_t)
        out = []
        for k in range(3):
            phi = 2 * math.pi * k / 3 + (math.pi / 2 if index % 2 else -math.pi / 2)
            out.append(cos_t * a + sin_t * (math.cos(phi) * perp + math.sin(phi) * perp2))
        return out
    a, b = bonds
    bis = -(a + b)
    bis /= np.linalg.norm(bis)
    nrm = np.cross(a, b)
    nrm /= np.linalg.norm(nrm)
    # the two remaining tetrahedral directions lie in the plane of bis and nrm
    ang = math.acos(-1.0 / 3.0) / 2
    return [math.cos(ang) * bis + math.sin(ang) * nrm, math.cos(ang) * bis - math.sin(ang) * nrm]


def hydroxyl(r_oh: float = 1.0):
    """OH radical (doublet), O-H 1.0 A."""
    return [8, 1], np.array([[0.0, 0.0, 0.0], [0.0, 0.0, r_oh]]) / BOHR


def methyl_planar(r_ch: float = 1.08):
    """Planar CH3 radical (doublet), C-H 1.08 A at 120 degrees."""
    xyz = [[0.0, 0.0, 0.0]]
    for k in range(3):
        a = 2 * math.pi * k / 3
        xyz.append([r_ch * math.cos(a), r_ch * math.sin(a), 0.0])
    return [6, 1, 1, 1], np.array(xyz) / BOHR
