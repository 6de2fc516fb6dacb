"""Host side of counting one graph on several GPUs (kcgpu_b200.sharding): the
128-bit limb arithmetic and the exact all-reduce of the shards' counts on
world_size 2 with the gloo backend, on CPU."""
import os
import socket
import sys
from pathlib import Path

import pytest
import torch.multiprocessing as mp

ROOT = Path(__file__).resolve().parents[1]
sys.path.insert(0, str(ROOT))

from kcgpu_b200 import sharding  # noqa: E402


@pytest.mark.parametrize("v", [0, 1, 2**32 - 1, 2**32, 2**64 - 1, 2**64, 2**127 + 12345, 2**128 - 1])
def test_limbs_round_trip(v):
    assert sharding.from_limb_sums(sharding.to_limbs(v)) == v


def test_limb_sums_carry():
    a, b = 2**128 - 2**40, 2**40 - 1
    sums = [x + y for x, y in zip(sharding.to_limbs(a), sharding.to_limbs(b))]
    assert sharding.from_limb_sums(sums) == 2**128 - 1
    with pytest.raises(ValueError):
        sharding.to_limbs(2**128)
    with pytest.raises(OverflowError):
        sharding.from_limb_sums([x + y for x, y in zip(sharding.to_limbs(2**128 - 1), sharding.to_limbs(1))])


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


CASES = [(2**128 - 1 - 987654321987654321, 987654321987654321), (2**64 - 1, 1), (0, 5), (2**96 + 7, 2**96 + 9)]


def _rank(rank: int, world: int, port: int, out):
    import datetime

    import torch.distributed as dist

    os.environ.update({"MASTER_ADDR": "127.0.0.1", "MASTER_PORT": str(port)})
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    sys.path.insert(0, str(ROOT))
    from kcgpu_b200 import sharding as sh

    got = [sh.sum_u128(c[rank]) for c in CASES]
    out.put((rank, got))
    dist.destroy_process_group()


def test_sum_u128_over_two_gloo_ranks():
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
    want = [a + b for a, b in CASES]
    assert got == [(0, want), (1, want)]


class _FakeGraph:
    """Stands in for kcgpu_b200.Graph: shard i of S counts the units j with
    j mod S == i of a fixed list of per-unit counts (as kc_count_shard deals
    out the units of a size class)."""

    UNITS = [3, 0, 7, 2**70, 5, 1, 9, 2**64 + 11, 4]

    def count(self, k, shard=None, **params):
        i, s = shard
        return sum(c for j, c in enumerate(self.UNITS) if j % s == i)


def _rank_sharded(rank: int, world: int, port: int, out):
    import datetime

    import torch.distributed as dist

    os.environ.update({"MASTER_ADDR": "127.0.0.1", "MASTER_PORT": str(port)})
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    sys.path.insert(0, str(ROOT))
    from kcgpu_b200 import sharding as sh

    out.put((rank, sh.count_sharded(_FakeGraph(), 5, mode="pivot")))
    dist.destroy_process_group()


@pytest.mark.parametrize("world", [2, 3])
def test_count_sharded_sums_every_unit_once(world):
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank_sharded, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(120)
        assert p.exitcode == 0
    got = sorted(q.get(timeout=10) for _ in range(world))
    assert got == [(r, sum(_FakeGraph.UNITS)) for r in range(world)]
