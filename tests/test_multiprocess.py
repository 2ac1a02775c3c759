"""The N > 1 path on CPU: two `gloo` ranks shard a candidate batch, compute
their slices independently (the CPU oracle stands in for the device, which
these tests do not need), gather the per-candidate outputs in candidate
order and take the max of the per-rank step times, as `bench.py` does under
torchrun."""
import datetime
import importlib
import os
import socket
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _batch():
    sys.path.insert(0, ROOT)
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    W = importlib.import_module("the-rule-and-compass_b200.workloads")
    trees, x, y = W.fit_workload(13, 300, seed=1)
    return trees, x, y


def _serial(trees, x, y, O):
    v, n = x.shape
    sse = np.array([O.score(t, x.reshape(-1), n, v, y, O.SQUARED) for t in trees])
    pred = np.stack([O.predict(t, x.reshape(-1), n, v)[:5] for t in trees])
    return sse, pred


def _worker(rank, world, port, q):
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=60))
    try:
        trees, x, y = _batch()
        import oracle as O
        S = importlib.import_module("the-rule-and-compass_b200.shard")
        s, e = S.shard_bounds(len(trees), rank, world)
        sse, pred = _serial(trees[s:e], x, y, O)
        full_sse = S.gather_candidates(sse, len(trees))
        full_pred = S.gather_candidates(pred, len(trees))
        tmax = S.max_over_ranks(10.0 + rank)
        q.put((rank, full_sse, full_pred, tmax))
    finally:
        dist.destroy_process_group()


def test_shard_bounds_partition():
    sys.path.insert(0, ROOT)
    S = importlib.import_module("the-rule-and-compass_b200.shard")
    for n in (0, 1, 7, 13, 4096):
        for world in (1, 2, 3, 8):
            b = [S.shard_bounds(n, r, world) for r in range(world)]
            assert b[0][0] == 0 and b[-1][1] == n
            assert all(b[i][1] == b[i + 1][0] for i in range(world - 1))
            sizes = [e - s for s, e in b]
            assert max(sizes) - min(sizes) <= 1
    with pytest.raises(ValueError):
        S.shard_bounds(5, 2, 2)


def test_single_rank_helpers_without_a_process_group():
    sys.path.insert(0, ROOT)
    S = importlib.import_module("the-rule-and-compass_b200.shard")
    a = np.arange(6.0).reshape(3, 2)
    assert np.array_equal(S.gather_candidates(a, 3), a)
    assert S.max_over_ranks(2.5) == 2.5


def test_two_gloo_ranks_reproduce_the_serial_batch():
    import torch.multiprocessing as mp
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    world = 2
    procs = [ctx.Process(target=_worker, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    got = {}
    try:
        for _ in range(world):
            rank, sse, pred, tmax = q.get(timeout=120)
            got[rank] = (sse, pred, tmax)
    finally:
        for p in procs:
            p.join(timeout=60)
            if p.is_alive():
                p.terminate()
    assert all(p.exitcode == 0 for p in procs)
    trees, x, y = _batch()
    import oracle as O
    O.lib()
    sse, pred = _serial(trees, x, y, O)
    for rank in range(world):
        r_sse, r_pred, tmax = got[rank]
        assert np.array_equal(r_sse.view(np.uint64), sse.view(np.uint64))
        assert np.array_equal(r_pred, pred)
        assert tmax == 11.0
