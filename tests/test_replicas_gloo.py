"""The multi-process path of bench.py on the CPU: two gloo ranks (the path
shards into independent replicas, so its only collectives are the barrier and
the max over ranks of the timed region)."""
import multiprocessing as mp
import os
import socket

from conftest import ROOT


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, ws, port, q):
    import sys
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(ws),
                      LOCAL_RANK=str(rank))
    sys.path.insert(0, ROOT)
    import bench
    import torch.distributed as dist
    n, r, _ = bench.dist_init("gloo")
    t_max = bench.max_over_ranks(1.5 + r, n)   # rank 1 is the slower one
    bench.barrier(n)
    q.put((r, n, t_max, bench.replica_seconds(t_max, 4, n)))
    dist.destroy_process_group()


def test_two_gloo_replicas_take_the_slowest_rank():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    out = sorted(q.get(timeout=180) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert [o[0] for o in out] == [0, 1] and all(o[1] == 2 for o in out)
    assert all(o[2] == 2.5 for o in out)            # max over ranks, seen by both
    assert all(o[3] == 2.5 / (4 * 2) for o in out)  # two designs finish per step


def test_replica_seconds_single_rank():
    import sys
    sys.path.insert(0, ROOT)
    import bench
    assert bench.replica_seconds(3.0, 6, 1) == 0.5
