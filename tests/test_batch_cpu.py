"""Host logic of the batched workload: instance draws, the LPT sharding over
ranks and the all-gather of per-instance results, run as two gloo ranks on CPU
(the solve itself is replaced by the CPU oracle, so no GPU is needed)."""
import importlib
import os
import socket

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _batch():
    return importlib.import_module("nested-parallelism_b200.batch")


def test_draws_follow_the_workload_definition():
    B = _batch()
    items = B.rmat_batch(64, seed=7, only=range(0, 64, 9))
    assert [it.index for it in items] == list(range(0, 64, 9))
    for it in items:
        assert 12 <= it.scale <= 18 and it.edge_factor in (4, 8, 16, 32)
        assert it.graph.n == 1 << it.scale and 0 <= it.source < it.graph.n
        assert it.graph.w.min() >= 1 and it.graph.w.max() <= 255
    again = B.rmat_batch(64, seed=7, only=[items[1].index])[0]
    assert again.source == items[1].source and np.array_equal(again.graph.col, items[1].graph.col)


@pytest.mark.parametrize("world", [1, 2, 3, 8])
def test_lpt_shards_cover_every_instance_once_and_balance(world):
    B = _batch()
    rng = np.random.default_rng(world)
    work = [int(x) for x in rng.integers(1, 10_000, 64)]
    parts = B.shard(work, world)
    assert len(parts) == world
    flat = sorted(i for p in parts for i in p)
    assert flat == list(range(64))
    loads = [sum(work[i] for i in p) for p in parts]
    assert max(loads) - min(loads) <= max(work)
    assert parts == B.shard(work, world)  # deterministic
    idx = [B.shard_indices(64, 7, world, r) for r in range(world)]
    assert sorted(i for p in idx for i in p) == list(range(64))


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _rank_main(rank, world, port, q):
    import sys
    sys.path.insert(0, ROOT)
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import torch.distributed as dist
    import oracle
    B = importlib.import_module("nested-parallelism_b200.batch")
    nps = importlib.import_module("nested-parallelism_b200")
    dist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port}", rank=rank, world_size=world,
                            timeout=__import__("datetime").timedelta(seconds=60))
    try:
        mine = B.shard_indices(16, 11, world, rank, scales=(6, 9))
        items = B.rmat_batch(16, seed=11, scales=(6, 9), only=mine)
        local = []
        for it in items:
            d = oracle.sssp_heap(it.graph.row_ptr, it.graph.col, it.graph.w, it.source)
            local.append({"index": it.index, "fnv1a": nps.fnv1a(d), "rank": rank})
        allr = B.gather_results(local)
        q.put((rank, allr))
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks_shard_and_gather():
    import multiprocessing as mp
    import oracle
    nps = importlib.import_module("nested-parallelism_b200")
    B = _batch()
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    got = dict(q.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    # every rank holds all 16 results, each solved by the rank its shard names
    want = {it.index: nps.fnv1a(oracle.sssp_heap(it.graph.row_ptr, it.graph.col, it.graph.w, it.source))
            for it in B.rmat_batch(16, seed=11, scales=(6, 9))}
    for rank in (0, 1):
        res = got[rank]
        assert [r["index"] for r in res] == list(range(16))
        assert {r["index"]: r["fnv1a"] for r in res} == want
        owner = {r["index"]: r["rank"] for r in res}
        for r in (0, 1):
            assert sorted(i for i, o in owner.items() if o == r) == B.shard_indices(16, 11, 2, r, scales=(6, 9))
