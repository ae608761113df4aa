"""bench.py's replica path (one process per GPU, no data-path collective) on CPU: two gloo ranks agree on the
slowest rank's time (max over ranks), meet at the barriers, and the reference arm's second rank exits without work."""
import os
import socket
import sys

import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank: int, world: int, port: int, out) -> None:
    os.environ.update(WORLD_SIZE=str(world), RANK=str(rank), LOCAL_RANK=str(rank), MASTER_ADDR="127.0.0.1",
                      MASTER_PORT=str(port))
    sys.path.insert(0, ROOT)
    import argparse

    import torch.distributed as dist

    import bench
    w, r, local = bench.dist_setup()
    assert (w, r, local) == (world, rank, rank) and dist.get_backend() == "gloo"
    slowest = bench.max_over_ranks(10.0 + 5.0 * rank, w)  # rank 1 took longer
    bench.barrier(w)
    skipped = bench.run_reference(argparse.Namespace(), w, r) if r != 0 else None
    bench.barrier(w)
    dist.destroy_process_group()
    out.put((rank, slowest, skipped))


def test_two_gloo_ranks():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=120)
        assert p.exitcode == 0
    got = sorted(q.get(timeout=10) for _ in range(2))
    assert [g[1] for g in got] == [15.0, 15.0], "both ranks see the slowest rank's time"
    assert got[1][2] is None, "the reference arm's second rank returns without work"
