"""Sharded direct Fock build of one molecule over several GPUs.

One process per GPU (torch.distributed, NCCL).  Every rank holds the whole
molecule's context (shell pairs, Schwarz bounds, class task lists: a few
hundred MB at most) and the full density; `hfg_set_shard(rank, world)` makes
its builds evaluate the rank-th of `world` contiguous task ranges of equal
estimated cost in each quartet class, so each rank produces a partial G.  G is linear in the J/K sums, so one all-reduce (sum)
of the n x n partials gives every rank the full G (a few MB: latency-bound
over NVLink).  Nothing else crosses between ranks: the density every rank
feeds in is the same because every rank runs the same replicated SCF algebra.
"""
from __future__ import annotations


class ShardedFock:
    """`engine`: an object with set_shard(rank, count), fock_rhf_tensor(P, G)
    and fock_uhf_tensor(Pa, Pb, Ga, Gb) (hartreefock_b200.engine.Engine).
    Shards are ranges of each class's task list, so every rank's engine must
    hold the same task lists: the same molecule, options and lane-group
    targets (no per-rank Engine.autotune_tasks / set_prim_target choices)."""

    def __init__(self, engine, group=None):
        import torch.distributed as dist
        self._dist = dist
        self.group = group
        self.rank = dist.get_rank(group)
        self.world = dist.get_world_size(group)
        self.engine = engine
        engine.set_shard(self.rank, self.world)

    def fock_rhf(self, P, G):
        """G = full two-electron matrix of density P (both n x n float64
        tensors on this rank's device): partial build, then all-reduce."""
        self.engine.fock_rhf_tensor(P, G)
        if self.world > 1:
            self._dist.all_reduce(G, group=self.group)
        return G

    def fock_uhf(self, Pa, Pb, Ga, Gb):
        self.engine.fock_uhf_tensor(Pa, Pb, Ga, Gb)
        if self.world > 1:
            self._dist.all_reduce(Ga, group=self.group)
            self._dist.all_reduce(Gb, group=self.group)
        return Ga, Gb
