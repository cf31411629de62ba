"""The algorithmic flop count of a quartet class: the reference's recursion
loops (GaussianTwoElectrons.cpp:98-359, IntegralsRepository.cpp:396-421)
walked on the host.  Hand counts for the small classes and the loop
structure's invariants.  CPU only."""
from hartreefock_b200 import flops as F


def test_small_classes_by_hand():
    # (ss|ss): prefactor + one Boys product + F_0 + the contraction of one element
    assert F.class_flops(0, 0, 0, 0) == (F.PREFACTOR + 1 + F.boys_flops(0) + 7 + 2, 0)
    # (ps|ss): three components of L = 1, one order each, 3 flops per VRR step
    per_prim, per_shell = F.class_flops(1, 0, 0, 0)
    assert per_prim == F.PREFACTOR + 2 + F.boys_flops(1) + 3 * 3 + 7 + 2 * 3
    assert per_shell == 0


def test_vrr_counts_two_back_terms():
    # L = 2 components xx, xy, xz, yy, yz, zz: xx, yy, zz step along a
    # component of 2 (two-back term, 5 more flops), xy, xz, yz do not
    assert F.vrr_flops(2) == 3 * 2 * 3 + 6 * 3 + 3 * 5


def test_hrr_only_with_angular_momentum_on_b_or_d():
    assert F.hrr_flops(2, 0, 2, 0) == 0
    # (pp|ss): QN2 of total 1 (3 components) x QN1 of total 1 (3) x one ket element x 2
    assert F.hrr_flops(1, 1, 0, 0) == 3 * 3 * 1 * 2
    # (ss|pp) side: QN4 of total 1 x QN3 of total 1 x one bra element x 2
    assert F.hrr_flops(0, 0, 1, 1) == 3 * 3 * 1 * 2


def test_work_grows_with_angular_momentum():
    classes = [(0, 0, 0, 0), (1, 0, 0, 0), (1, 0, 1, 0), (2, 0, 1, 0), (2, 1, 2, 0), (2, 2, 2, 1), (2, 2, 2, 2)]
    per_prim = [F.class_flops(*c)[0] for c in classes]
    assert per_prim == sorted(per_prim)
    assert F.build_flops([(1, 0, 0, 0, 10, 2), (2, 2, 2, 2, 1, 1)]) == 10 * per_prim[1] + sum(F.class_flops(2, 2, 2, 2))
