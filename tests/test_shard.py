"""Multi-rank plumbing on CPU: request and row sharding cover the work once,
and the max/sum over ranks run over a world-size-2 gloo process group."""
import os
import socket
import sys

import pytest
import torch.multiprocessing as mp

# Spawned ranks import this module afresh: make the package importable there too.
ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)
import __graft_entry__ as entry  # noqa: E402

entry.load_package()
from oxideav_render_b200 import shard  # noqa: E402


def test_shard_and_row_bands_partition_the_work():
    items = list(range(64))
    for world in (1, 2, 3, 8):
        parts = [shard.shard(items, r, world) for r in range(world)]
        assert sorted(sum(parts, [])) == items
        assert all(len(p) in (len(items) // world, len(items) // world + 1) for p in parts)
        for h in (1, 7, 1080):
            bands = [shard.row_bands(h, r, world) for r in range(world)]
            assert bands[0][0] == 0 and bands[-1][1] == h
            assert all(bands[i][1] == bands[i + 1][0] for i in range(world - 1))
            assert max(b - a for a, b in bands) - min(b - a for a, b in bands) <= 1
    with pytest.raises(ValueError):
        shard.shard(items, 2, 2)


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, out):
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        mine = shard.shard(list(range(10)), rank, world)
        out[rank] = (mine, shard.max_over_ranks(1.5 + rank), shard.sum_over_ranks(len(mine)))
    finally:
        dist.destroy_process_group()


def test_reductions_over_a_two_rank_gloo_group():
    world = 2
    mgr = mp.get_context("spawn").Manager()
    out = mgr.dict()
    ctx = mp.get_context("spawn")
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, world, port, out)) for r in range(world)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=120)
        assert p.exitcode == 0
    got = dict(out)
    mgr.shutdown()  # stop the manager process here, not at interpreter exit
    assert sorted(got[0][0] + got[1][0]) == list(range(10))
    assert got[0][1] == got[1][1] == 2.5
    assert got[0][2] == got[1][2] == 10.0
