"""Sharded direct builds on one GPU: the partial G of shards 0..count-1 (built
one after another in this process, so no rank waits on another) sum to the
unsharded G, for RHF, UHF and the precision form."""
import numpy as np
import pytest

from hartreefock_b200 import engine as E
from hartreefock_b200 import molecules

pytestmark = pytest.mark.gpu

BASIS = "6-31g*"


def _density(n, seed):
    rng = np.random.default_rng(seed)
    Q, _ = np.linalg.qr(rng.normal(size=(n, n // 4)))
    return 2.0 * Q @ Q.T


@pytest.mark.parametrize("count", [2, 3])
def test_shard_partials_sum_to_full_rhf(count):
    Z, xyz = molecules.water_cluster(4, seed=3)
    eng = E.Engine(Z, xyz, BASIS)
    P = _density(eng.nbf, 1)
    full = eng.fock_rhf(P)
    q_full = eng.stats()["shell_quartets"]
    total = np.zeros_like(full)
    quartets = 0
    for r in range(count):
        eng.set_shard(r, count)
        total += eng.fock_rhf(P)
        quartets += eng.stats()["shell_quartets"]
    assert np.abs(total - full).max() < 1e-11 * max(1.0, np.abs(full).max())
    # each shard carries about its share of the work
    assert abs(quartets - q_full) <= count * 21


def test_shard_partials_sum_to_full_uhf_and_precision_form():
    Z, xyz = molecules.water_cluster(3, seed=5)
    plain = E.Engine(Z, xyz, BASIS)
    Pa, Pb = _density(plain.nbf, 2), _density(plain.nbf, 3)
    fa, fb = plain.fock_uhf(Pa, Pb)
    ga, gb = np.zeros_like(fa), np.zeros_like(fb)
    for r in range(2):
        plain.set_shard(r, 2)
        a, b = plain.fock_uhf(Pa, Pb)
        ga += a
        gb += b
    assert np.abs(ga - fa).max() < 1e-11 and np.abs(gb - fb).max() < 1e-11
    # incremental mixed-precision builds per shard: two builds each, summed
    shards = [E.Engine(Z, xyz, BASIS, incremental=True, mixed_cutoff=1e-4) for _ in range(2)]
    for r, e in enumerate(shards):
        e.set_shard(r, 2)
    P1 = 0.5 * (Pa + Pb)
    P2 = P1 + 1e-3 * np.eye(plain.nbf)
    for e in shards:
        e.fock_rhf(P1)
    total = sum(e.fock_rhf(P2) for e in shards)
    plain.set_shard(0, 1)
    assert np.abs(total - plain.fock_rhf(P2)).max() < 1e-6
