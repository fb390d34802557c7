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


def _bench_rank(rank, world, port, out):
    os.environ.update(RANK=str(rank), WORLD_SIZE=str(world), LOCAL_RANK=str(rank),
                      MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    import bench
    from marqov_b200.replicas import ReplicaGroup
    g = ReplicaGroup("gloo", timeout_s=60)
    ws, r, local = bench.dist_env()
    # rank r "ran" 1e9 updates in (10 + 5 r) ms
    value, ms_max = bench.weak_scaling_value(g, 1.0e9, 10.0 + 5.0 * rank)
    out[rank] = (ws, r, local, g.replica_id(), value, ms_max)
    g.close()


def test_bench_rank_logic_two_gloo_ranks():
    """bench.py's multi-rank arithmetic: every rank sees WORLD_SIZE = 2, its
    own replica id, the slowest rank's time and the whole-job rate."""
    pytest.importorskip("torch.distributed")
    port = _free_port()
    with mp.Manager() as man:
        out = man.dict()
        mp.spawn(_bench_rank, args=(2, port, out), nprocs=2, join=True)
        res = dict(out)
    assert sorted(v[3] for v in res.values()) == [0, 1]
    for rank, (ws, r, local, rid, value, ms_max) in res.items():
        assert ws == 2 and r == rank and local == rank and rid == rank
        assert ms_max == 15.0
        assert abs(value - 2 * 1.0e9 / (15.0 * 1e6)) < 1e-9
