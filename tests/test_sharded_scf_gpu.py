"""Sharded SCF (HartreeFockAlgorithm::shardRank / shardCount / allReduce):
two processes on one GPU, each building its cost-balanced shard of every
Fock build, G summed over the gloo group on the host between builds (the
processes' kernels never wait on each other), reach the unsharded SCF's
energy.  The same code path runs one process per GPU with NCCL."""
import os
import socket

import pytest

pytestmark = pytest.mark.gpu


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, q):
    import datetime
    import torch.distributed as dist
    from hartreefock_b200 import molecules, scf
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=120))
    try:
        out = {}
        for uhf in (False, True):
            Z, xyz = molecules.water_cluster(2, seed=0) if not uhf else molecules.hydroxyl()
            basis = "6-31g*" if not uhf else "6-31g"
            r = scf.run_scf(Z, xyz, basis, unrestricted=uhf, post_diis=0, want_density=False,
                            shard=(rank, world), allreduce=scf.torch_allreduce())
            out[uhf] = (r["energy"], r["converged"])
        q.put((rank, out))
    finally:
        dist.destroy_process_group()


def test_two_shard_scf_matches_unsharded():
    import torch.multiprocessing as mp
    from hartreefock_b200 import molecules, scf
    want = {}
    for uhf in (False, True):
        Z, xyz = molecules.water_cluster(2, seed=0) if not uhf else molecules.hydroxyl()
        basis = "6-31g*" if not uhf else "6-31g"
        want[uhf] = scf.run_scf(Z, xyz, basis, unrestricted=uhf, post_diis=0, want_density=False)["energy"]
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    results = dict(q.get(timeout=600) for _ in procs)
    for p in procs:
        p.join(timeout=120)
        assert p.exitcode == 0
    for rank in (0, 1):
        for uhf in (False, True):
            e, conv = results[rank][uhf]
            assert conv
            assert abs(e - want[uhf]) < 1e-9, (rank, uhf, e, want[uhf])
