"""Algorithmic floating-point work of a quartet class, counted by walking the
reference's own recursion loops (aromanro/HartreeFock, GaussianTwoElectrons.cpp
and IntegralsRepository.cpp), independent of the engine's kernels.

Per primitive quartet (GaussianTwoElectrons::Reset, GaussianTwoElectrons.cpp:15-96):
  prefactor   the scalar set-up of Reset (exponent sums, P, Q, P - Q, the
              exponent, the 2 pi^(5/2) factor, T, Rpa, Rwp, Delta) and the
              (maxL + 1) products factor * F_m;
  Boys        F_maxL by the 7-term tabulated Taylor expansion, e^-T, and the
              downward recursion to F_0 (the method the engine uses; the
              reference's own series is a cache-backed incomplete gamma,
              BoysFunctions.cpp:10-25, whose cost is not an algorithmic figure);
  VRR         VerticalRecursion (:98-134): for every Cartesian component up to
              maxL and every order m it needs, 3 flops, 5 more when the
              two-back term exists;
  ET          ElectronTransfer (:137-188): for every ket component up to
              L3 + L4 and every bra component it sweeps, 3 flops, 3 more for
              each of the two optional terms;
  contraction IntegralsRepository::getElectronElectron (IntegralsRepository.cpp:
              396-421): the 8-factor product and one multiply-add per element
              of the cropped [e0|f0] block.
Per shell quartet: HorizontalRecursion1 (:198-272) and HorizontalRecursion2
(:278-359), 2 flops per element they write.

A flop is one add, multiply, divide or square root (an FMA counts 2, exp 1).
"""
from __future__ import annotations

from functools import lru_cache


def _components(L: int):
    """Cartesian components of total L in the reference's canonical order
    (QuantumNumbers::CanonicalIncrement, QuantumNumbers.h:60-80): l
    descending, then m descending."""
    return [(l, L - l - n, n) for l in range(L, -1, -1) for n in range(0, L - l + 1)]


def _direction(q) -> int:
    """The component the recursions step along: the first of l, m, n equal to
    the largest (GaussianTwoElectrons.h:40-73, 148-179)."""
    mx = max(q)
    return q.index(mx)


def ncart(L: int) -> int:
    return (L + 1) * (L + 2) // 2


def _n_components(lo: int, hi: int) -> int:
    return sum(ncart(L) for L in range(lo, hi + 1))


PREFACTOR = 87  # scalar operations of Reset before the Boys products (GaussianTwoElectrons.cpp:19-85)


def boys_flops(max_m: int) -> int:
    """Tabulated Taylor F_maxL (6 FMA + the offset), e^-T (8-term series times
    the tabulated value) and the downward recursion (one FMA and one multiply
    per order)."""
    return 14 + 17 + 3 * max_m


def vrr_flops(max_l: int) -> int:
    total = 0
    for L in range(1, max_l + 1):
        for q in _components(L):
            d = _direction(q)
            orders = max_l + 1 - L  # m = 0 .. size - L - 1
            total += orders * (3 + (5 if q[d] >= 2 else 0))
    return total


def et_flops(max_l: int, max_l34: int) -> int:
    total = 0
    for L2 in range(1, max_l34 + 1):
        for q2 in _components(L2):
            d = _direction(q2)
            prev_prev = q2[d] >= 2
            for L1 in range(L2 - 1, max_l - L2 + 1):
                for q1 in _components(L1):
                    total += 3 + (3 if q1[d] > 0 else 0) + (3 if prev_prev else 0)
    return total


def contraction_flops(l1: int, l2: int, l3: int, l4: int) -> int:
    return 7 + 2 * _n_components(l1, l1 + l2) * _n_components(l3, l3 + l4)


def hrr_flops(l1: int, l2: int, l3: int, l4: int) -> int:
    ind3 = _n_components(l3, l3 + l4)
    total = 0
    for k in range(1, l2 + 1):  # HorizontalRecursion1: QN2 of total k, QN1 of L1 .. L1 + L2 - k
        total += ncart(k) * _n_components(l1, l1 + l2 - k) * ind3 * 2
    for k in range(1, l4 + 1):  # HorizontalRecursion2: QN4 of total k, QN3 of L3 .. L3 + L4 - k
        total += ncart(k) * _n_components(l3, l3 + l4 - k) * ncart(l1) * ncart(l2) * 2
    return total


@lru_cache(maxsize=None)
def class_flops(l1: int, l2: int, l3: int, l4: int) -> tuple:
    """(flops per primitive quartet, flops per shell quartet) of the class
    (l1 l2 | l3 l4) in the reference's canonical orientation."""
    max_l = l1 + l2 + l3 + l4
    per_prim = (PREFACTOR + (max_l + 1) + boys_flops(max_l) + vrr_flops(max_l) + et_flops(max_l, l3 + l4)
                + contraction_flops(l1, l2, l3, l4))
    return per_prim, hrr_flops(l1, l2, l3, l4)


def build_flops(classes) -> float:
    """Algorithmic flops of a build from per-class (la, lb, lc, ld,
    primitive quartets, shell quartets) records."""
    total = 0.0
    for la, lb, lc, ld, prims, shells in classes:
        fp, fs = class_flops(la, lb, lc, ld)
        total += prims * fp + shells * fs
    return total
