"""bench.py's multi-rank plumbing with two gloo ranks on CPU: the process group comes up
from torchrun-style environment variables, the reported time is the maximum over ranks,
the barrier holds every rank, and the job rate counts every replica's work."""
import os
import socket
import sys

import pytest

torch = pytest.importorskip("torch")
import torch.multiprocessing as mp  # noqa: E402

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, out):
    os.environ.update({"RANK": str(rank), "WORLD_SIZE": str(world), "LOCAL_RANK": str(rank),
                       "MASTER_ADDR": "127.0.0.1", "MASTER_PORT": str(port), "CFG_BENCH_BACKEND": "gloo"})
    sys.path.insert(0, ROOT)
    import bench
    r, w, local, pg = bench.dist_setup(world)
    assert (r, w, local) == (rank, world, rank) and pg is not None
    slowest = bench.allreduce_max(pg, local, 10.0 + 5.0 * rank)   # each rank's own seconds
    bench.barrier(pg)
    # rank 0 alone would pick 16384, rank 1 alone 65536: both take the best worst case
    times = {16384: 80.0 + 30.0 * rank, 32768: 95.0, 65536: 100.0 - 15.0 * rank}
    g, agreed = bench.agree_graph_count(pg, local, times)
    out.put((rank, slowest, bench.job_rate(w, 1000, 3, slowest), g))
    pg.destroy_process_group()


def test_two_gloo_ranks():
    world, port = 2, _free_port()
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    procs = [ctx.Process(target=_rank, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(120)
        assert p.exitcode == 0
    got = sorted(q.get(timeout=10) for _ in range(world))
    # both ranks see the slowest rank's time and the same job rate (2 replicas x 1000 units x
    # 3 steps / 15 s), and agree on the subgraph count with the best slowest time (32768: 95)
    assert got == [(0, 15.0, 400.0, 32768), (1, 15.0, 400.0, 32768)]


def test_single_process_needs_no_group():
    sys.path.insert(0, ROOT)
    import bench
    assert bench.allreduce_max(None, 0, 7.5) == 7.5
    assert bench.agree_graph_count(None, 0, {16384: 90.0, 65536: 80.0})[0] == 65536
    assert bench.job_rate(1, 1500, 2, 3.0) == 1000.0
