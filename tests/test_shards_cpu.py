"""The multi-GPU path's host logic (hartreefock_b200.shards) on CPU: two gloo
ranks, each holding a partial G from a stand-in engine whose shards sum to
the full matrix; after the all-reduce both ranks hold the full G."""
import os
import socket

import numpy as np
import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

from hartreefock_b200.shards import ShardedFock

N = 12


def _full_g(P):
    # any fixed linear map of P will do: G = A P A^T + P
    A = torch.arange(N * N, dtype=torch.float64).reshape(N, N).sin()
    return A @ P @ A.T + P


class FakeEngine:
    """Partial G of shard (rank, count): the rows i with i % count == rank."""

    def set_shard(self, rank, count):
        self.rank, self.count = rank, count

    def fock_rhf_tensor(self, P, G):
        full = _full_g(P)
        mask = (torch.arange(N) % self.count == self.rank).to(torch.float64)[:, None]
        G.copy_(full * mask)

    def fock_uhf_tensor(self, Pa, Pb, Ga, Gb):
        self.fock_rhf_tensor(Pa + Pb, Ga)
        self.fock_rhf_tensor(Pa - Pb, Gb)


def _worker(rank, world, port, out):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        torch.manual_seed(0)
        P = torch.randn(N, N, dtype=torch.float64)
        P = P + P.T
        sf = ShardedFock(FakeEngine())
        G = torch.empty_like(P)
        sf.fock_rhf(P, G)
        Ga, Gb = torch.empty_like(P), torch.empty_like(P)
        sf.fock_uhf(P, 0.5 * P, Ga, Gb)
        ok = (torch.allclose(G, _full_g(P)) and torch.allclose(Ga, _full_g(1.5 * P))
              and torch.allclose(Gb, _full_g(0.5 * P)) and sf.world == world)
        out[rank] = 1 if ok else 0
    finally:
        dist.destroy_process_group()


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


@pytest.mark.timeout(120)
def test_sharded_partials_all_reduce_to_full_g():
    world = 2
    out = mp.get_context("spawn").Array("i", world)
    mp.spawn(_worker, args=(world, _free_port(), out), nprocs=world, join=True)
    assert list(out) == [1] * world


# --- the engine's own shard partition (hfg_shard_range, host arithmetic) with
# the oracle's G of each shard's quartets, reduced over two gloo ranks

def _shard_tasks(n, width=8):
    """Tasks as the engine forms them: per bra pair ij (canonical order), its
    kets kl <= ij in runs of `width`; cost = kets x a per-bra weight."""
    tasks, cost = [], [0.0]
    for ij in range(n * (n + 1) // 2):
        for k0 in range(0, ij + 1, width):
            k1 = min(ij + 1, k0 + width)
            tasks.append((ij, k0, k1))
            cost.append(cost[-1] + (k1 - k0) * (1.0 + (ij % 5)))
    return tasks, np.array(cost)


def _oracle_worker(rank, world, port, out):
    import oracle as O
    from conftest import load_golden
    from hartreefock_b200 import engine as E
    from hartreefock_b200.basis_io import basis_path
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        g = load_golden("h2o_631gs")
        mol = O.Molecule(list(g["Z"]), g["xyz"], basis_path(str(g["basis"])))
        n, packed = mol.nbf, g["eri_packed"]
        rng = np.random.default_rng(2)
        A = rng.normal(size=(n, n))
        P = A + A.T
        tasks, prefix = _shard_tasks(n)
        first, count = E.shard_range(prefix, rank, world)
        # this shard's quartets (ij|kl) of the packed table; G is linear in it
        mask = np.zeros_like(packed)
        for ij, k0, k1 in tasks[first:first + count]:
            base = ij * (ij + 1) // 2
            mask[base + k0:base + k1] = 1.0
        G = torch.from_numpy(O.g_rhf(n, packed * mask, P))
        dist.all_reduce(G)
        cover = torch.tensor([count], dtype=torch.int64)
        dist.all_reduce(cover)
        ok = (np.abs(G.numpy() - O.g_rhf(n, packed, P)).max() < 1e-10 * np.abs(G.numpy()).max()
              and int(cover) == len(tasks) and count > 0)
        out[rank] = 1 if ok else 0
    finally:
        dist.destroy_process_group()


@pytest.mark.timeout(120)
def test_engine_shard_partition_with_oracle_partials_sums_to_full_g():
    world = 2
    out = mp.get_context("spawn").Array("i", world)
    mp.spawn(_oracle_worker, args=(world, _free_port(), out), nprocs=world, join=True)
    assert list(out) == [1] * world


def test_shard_ranges_tile_the_tasks_and_balance_cost():
    from hartreefock_b200 import engine as E
    rng = np.random.default_rng(3)
    cost = rng.pareto(1.5, size=5000) + 0.01  # heavy-tailed task costs
    prefix = np.concatenate([[0.0], np.cumsum(cost)])
    for count in (1, 2, 3, 8, 64):
        ranges = [E.shard_range(prefix, r, count) for r in range(count)]
        pos = 0
        for first, n in ranges:
            assert first == pos
            pos += n
        assert pos == len(cost)
        share = [prefix[f + n] - prefix[f] for f, n in ranges]
        # each shard within one task's cost of the even share
        assert max(abs(s - prefix[-1] / count) for s in share) <= cost.max() + 1e-9
    with pytest.raises(E.HfgError):
        E.shard_range(prefix, 2, 2)
