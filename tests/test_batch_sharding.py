"""Host logic of the multi-mock sharding (hitomi_b200/batch.py): the split over ranks and
the gather, with world-size-2 gloo process groups on CPU (no GPU)."""
import os
import socket

import numpy as np
import pytest


def test_shard_is_a_balanced_partition():
    from hitomi_b200.batch import shard
    rng = np.random.default_rng(1)
    sizes = rng.normal(2e6, 4e5, size=256).astype(int)
    for world in (1, 2, 3, 8):
        parts = shard(sizes, world)
        flat = sorted(i for p in parts for i in p)
        assert flat == list(range(len(sizes)))
        loads = [sizes[p].sum() for p in parts]
        assert max(loads) - min(loads) <= sizes.max()
        assert shard(sizes, world) == parts  # deterministic


def test_shard_more_ranks_than_mocks():
    from hitomi_b200.batch import shard
    parts = shard([5, 3], 4)
    assert sorted(i for p in parts for i in p) == [0, 1]
    assert sum(1 for p in parts if not p) == 2
    with pytest.raises(ValueError):
        shard([1], 0)


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _worker(rank, world, port, sizes, q):
    import datetime

    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        from hitomi_b200.batch import gather, run_rank
        local = run_rank(sizes, rank, world, lambda i: {"rank": rank, "value": float(i) * 2.0})
        allr = gather(local, world)
        import torch
        t = torch.tensor([float(len(local))])
        dist.all_reduce(t, op=dist.ReduceOp.MAX)  # the max-over-ranks reduction bench.py uses
        q.put((rank, sorted(local), {k: v["value"] for k, v in allr.items()}, float(t.item())))
    finally:
        dist.destroy_process_group()


def test_gather_over_two_gloo_ranks():
    import multiprocessing as mp
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    sizes = [10, 7, 7, 3, 12, 1, 9]
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, sizes, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = [q.get(timeout=120) for _ in procs]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    res.sort()
    (r0, own0, all0, mx0), (r1, own1, all1, mx1) = res
    assert sorted(own0 + own1) == list(range(len(sizes))) and not set(own0) & set(own1)
    assert all0 == all1 == {i: 2.0 * i for i in range(len(sizes))}
    assert mx0 == mx1 == max(len(own0), len(own1))


def test_run_pipelined_covers_every_mock_once_per_context():
    from hitomi_b200.batch import run_pipelined

    seen = []

    def measure_on(ctx, i):
        seen.append((ctx, i))
        return {"i": i, "ctx": ctx}

    out = run_pipelined(list(range(7)), ["a", "b"], measure_on)
    assert sorted(out) == list(range(7))
    assert sorted(i for _, i in seen) == list(range(7))
    # context c takes mocks c, c + 2, c + 4, ...
    assert all(out[i]["ctx"] == ("a" if i % 2 == 0 else "b") for i in range(7))


def test_run_pipelined_raises_a_worker_error():
    import pytest
    from hitomi_b200.batch import run_pipelined

    def measure_on(ctx, i):
        if i == 3:
            raise RuntimeError("mock 3 failed")
        return {}

    with pytest.raises(RuntimeError, match="mock 3 failed"):
        run_pipelined(list(range(6)), [0, 1, 2], measure_on)
