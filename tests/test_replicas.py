"""The multi-rank plumbing (marqov_b200.replicas) with two gloo ranks on CPU:
distinct replica ids, barriers, the slowest rank's time and aggregate sums, as
bench.py uses them for N-GPU weak scaling."""
import os
import socket

import pytest
import torch.multiprocessing as mp


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, out):
    os.environ.update(RANK=str(rank), WORLD_SIZE=str(world), LOCAL_RANK=str(rank),
                      MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    from marqov_b200.replicas import ReplicaGroup
    g = ReplicaGroup("gloo", timeout_s=60)
    g.barrier()
    t = 1.0 + 0.5 * rank              # this rank's time
    out[rank] = (g.replica_id(10), g.max(t), g.sum(100.0 * (rank + 1)))
    g.close()


def test_two_gloo_ranks():
    pytest.importorskip("torch.distributed")
    port = _free_port()
    world = 2
    with mp.Manager() as man:
        out = man.dict()
        mp.spawn(_rank_main, args=(world, port, out), nprocs=world, join=True)
        res = dict(out)
    ids = sorted(r[0] for r in res.values())
    assert ids == [10, 11]
    assert all(r[1] == 1.5 for r in res.values())    # max over ranks
    assert all(r[2] == 300.0 for r in res.values())  # aggregate
