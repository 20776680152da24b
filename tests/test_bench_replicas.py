"""The multi-GPU path of bench.py is replicas only: each rank steps its own dwarf and the
job throughput is all ranks' body-updates over the slowest rank's time.  Checked here with
two gloo ranks on the CPU (no GPU, no collective on any data path)."""
import os
import socket
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, out):
    os.environ.update(RANK=str(rank), WORLD_SIZE=str(world), LOCAL_RANK=str(rank),
                      MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    sys.path.insert(0, ROOT)
    import bench
    dist = bench.Dist(backend="gloo")
    try:
        dist.barrier()
        seconds = 2.0 if rank == 1 else 1.0          # rank 1 is the slow one
        value, t = bench.replica_throughput(dist, 1000, 10, seconds)
        total = dist.sum(rank + 1)
        out.put((rank, value, t, total))
    finally:
        dist.close()


def test_two_rank_replica_throughput_uses_the_slowest_rank():
    import torch.multiprocessing as mp
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    results = [q.get(timeout=120) for _ in procs]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    for rank, value, t, total in results:
        assert t == 2.0                               # max over ranks
        assert value == pytest.approx(2 * 1000 * 10 / 2.0)
        assert total == 3.0


def test_single_process_replica_throughput():
    sys.path.insert(0, ROOT)
    import bench
    d = bench.Dist()
    assert d.world == 1
    value, t = bench.replica_throughput(d, 1048576, 10, 0.5)
    assert t == 0.5 and value == pytest.approx(1048576 * 10 / 0.5)
