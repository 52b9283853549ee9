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


def test_plan_requests_keeps_scenes_together_and_balances():
    keys = [3, 1, 3, 2, 1, 1, 7, 3, 2, 9]
    work = [10, 1, 10, 5, 1, 1, 4, 10, 5, 2]
    owners = shard.plan_requests(keys, work, 2)
    for k in set(keys):
        assert len({o for kk, o in zip(keys, owners) if kk == k}) == 1, k
    load = [sum(w for w, o in zip(work, owners) if o == r) for r in range(2)]
    per_scene = {k: sum(w for kk, w in zip(keys, work) if kk == k) for k in set(keys)}
    assert max(load) - min(load) <= max(per_scene.values())  # greedy bound: one scene's work
    assert shard.plan_requests(keys, work, 2) == owners  # deterministic
    assert shard.plan_requests(keys, work, 1) == [0] * len(keys)


def stub_render(req):
    """Stands in for a GPU render on CPU ranks: a pure function of the
    request, as a served image is of (scene, options, seed)."""
    import numpy as np
    key, seed, w, h = req
    return np.random.default_rng(seed * 1000 + key).random((h, w, 4)).astype("float32")


def _serve_rank(rank, world, port, reqs, out):
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        owners = shard.plan_requests([r[0] for r in reqs], [r[2] * r[3] for r in reqs], world)
        mine = {i: stub_render(r) for i, r in enumerate(reqs) if owners[i] == rank}
        ordered = shard.gather_ordered(mine, len(reqs), dst=0)
        total = shard.sum_over_ranks(len(mine))
        out[rank] = (sorted(mine), ordered, total)
    finally:
        dist.destroy_process_group()


def test_sharded_serving_gathers_results_in_request_order():
    import numpy as np
    reqs = [(k % 4, 100 + i, 8 + 4 * (i % 3), 6 + (i % 5)) for i, k in enumerate([0, 1, 2, 3, 1, 1, 0, 2, 3, 3, 0])]
    world = 2
    mgr = mp.get_context("spawn").Manager()
    out = mgr.dict()
    ctx = mp.get_context("spawn")
    port = _free_port()
    procs = [ctx.Process(target=_serve_rank, args=(r, world, port, reqs, out)) for r in range(world)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=120)
        assert p.exitcode == 0
    got = dict(out)
    mgr.shutdown()
    share0, ordered, total0 = got[0]
    share1, none1, total1 = got[1]
    assert none1 is None and total0 == total1 == len(reqs)
    assert sorted(share0 + share1) == list(range(len(reqs))) and not set(share0) & set(share1)
    assert share0 and share1  # both GPUs serve
    assert len(ordered) == len(reqs)
    for i, r in enumerate(reqs):
        assert np.array_equal(ordered[i], stub_render(r)), i


def test_gather_ordered_without_a_group_checks_coverage():
    assert shard.gather_ordered({1: "b", 0: "a"}, 2) == ["a", "b"]
    with pytest.raises(ValueError):
        shard.gather_ordered({0: "a"}, 2)
