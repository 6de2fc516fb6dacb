"""The benchmark's multi-rank plumbing (barrier, max over ranks of the step
time, rank-0-only output) on world_size 2 with the gloo backend, on CPU."""
import os
import socket
import sys
from pathlib import Path

import torch.multiprocessing as mp

ROOT = Path(__file__).resolve().parents[1]


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank: int, world: int, port: int, out):
    os.environ.update({"RANK": str(rank), "WORLD_SIZE": str(world), "LOCAL_RANK": str(rank),
                       "MASTER_ADDR": "127.0.0.1", "MASTER_PORT": str(port)})
    sys.path.insert(0, str(ROOT))
    import bench

    w, r, local, pg = bench.dist_setup(world, backend="gloo")
    assert (w, r, local) == (world, rank, rank)
    bench.barrier(pg, None)
    # each rank "timed" a different step; every rank must see the slowest
    t = bench.max_over_ranks(pg, 10.0 + 5.0 * rank, None)
    out.put((rank, t))
    pg.destroy_process_group()


def test_max_over_ranks_gloo():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(120)
        assert p.exitcode == 0
    got = sorted(q.get(timeout=10) for _ in range(2))
    assert got == [(0, 15.0), (1, 15.0)]
