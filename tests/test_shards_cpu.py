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
