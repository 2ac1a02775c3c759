"""Several devices behind one C-ABI handle (rc_multi_*): candidate slices run
concurrently, one context per device, outputs gathered in place. Run here
with the one GPU named twice (two independent contexts; no kernel of one
waits on the other), a sharded batch must answer bit for bit what a single
context answers, for scoring and for the fused fit."""
import importlib

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def test_multi_handle_matches_one_context(pkg):
    W = importlib.import_module("the-rule-and-compass_b200.workloads")
    trees, x, y = W.scoring_workload(200, 30000, seed=12)
    prog, off = pkg.Population(trees).programs()
    ev = pkg.GpuEvaluator(x.reshape(-1), 30000, 5, y)
    want, wst, _ = ev.score_batch(prog, off, 0)
    ev.close()
    for devices in ([0], [0, 0], [0, 0, 0]):
        mv = pkg.MultiEvaluator(x.reshape(-1), 30000, 5, y, devices)
        got, st, ms = mv.score_batch(prog, off, 0)
        assert ms >= 0
        assert np.array_equal(st, wst), devices
        assert np.array_equal(got.view(np.uint64), want.view(np.uint64)), devices
        mv.close()

    ftrees, fx, fy = W.fit_workload(60, 8192, seed=3)
    v, n = fx.shape
    plans = [pkg.gpu_fit_plan(t) for t in ftrees]
    ev = pkg.GpuEvaluator(fx.astype(np.float32).reshape(-1), n, v, fy.astype(np.float32))
    ev.set_fit_data(fx.reshape(-1), fy)
    c1, l1, s1, _ = ev.fit_plans(plans, 20)
    ev.close()
    mv = pkg.MultiEvaluator(fx.astype(np.float32).reshape(-1), n, v, fy.astype(np.float32), [0, 0])
    mv.set_fit_data(fx.reshape(-1), fy)
    c2, l2, s2, ms = mv.fit_plans(plans, 20)
    mv.close()
    assert ms >= 0
    assert np.array_equal(s1, s2)
    assert np.array_equal(l1.view(np.uint64), l2.view(np.uint64))
    assert np.array_equal(c1.view(np.uint64), c2.view(np.uint64))


def test_contexts_on_one_device_with_different_shared_memory(pkg):
    """Two contexts on the same device fit slices whose programs need very
    different shared memory, concurrently and repeatedly: a kernel's shared
    memory limit is shared by both and only ever grows, so neither launch
    fails, and every answer equals the one-context answer."""
    W = importlib.import_module("the-rule-and-compass_b200.workloads")
    ftrees, fx, fy = W.fit_workload(80, 8192, seed=9)
    v, n = fx.shape
    plans = sorted((pkg.gpu_fit_plan(t) for t in ftrees), key=lambda p: len(p.words))
    ev = pkg.GpuEvaluator(fx.astype(np.float32).reshape(-1), n, v, fy.astype(np.float32))
    ev.set_fit_data(fx.reshape(-1), fy)
    c1, l1, s1, _ = ev.fit_plans(plans, 20)
    ev.close()
    mv = pkg.MultiEvaluator(fx.astype(np.float32).reshape(-1), n, v, fy.astype(np.float32), [0, 0])
    mv.set_fit_data(fx.reshape(-1), fy)
    for _ in range(3):
        c2, l2, s2, ms = mv.fit_plans(plans, 20)
        assert ms >= 0
        assert np.array_equal(s1, s2)
        assert np.array_equal(l1.view(np.uint64), l2.view(np.uint64))
        assert np.array_equal(c1.view(np.uint64), c2.view(np.uint64))
    mv.close()
