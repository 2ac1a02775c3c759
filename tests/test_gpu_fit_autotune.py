"""The fit autotuner (rc_fit_autotune): it chooses an assembly budget per
length bucket, caches it per (N, feature count) in its file and reuses it,
and a tuned context still fits a batch bit-identically alone and mixed, with
the same accuracy against the CPU LM."""
import importlib
import os

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def test_fit_autotune_chooses_caches_and_keeps_results_exact(pkg, O, tmp_path):
    W = importlib.import_module("the-rule-and-compass_b200.workloads")
    trees, x, y = W.fit_workload(96, 8192, seed=41)
    v, n = x.shape
    ev = pkg.GpuEvaluator(x.astype(np.float32).reshape(-1), n, v, y.astype(np.float32))
    ev.set_fit_data(x.reshape(-1), y)
    plans = [pkg.gpu_fit_plan(t) for t in trees]
    path = str(tmp_path / "fit_tune.txt")
    budgets = ev.fit_autotune(plans, 20, sample=16, path=path)
    buckets = {0 if len(p.words) // 4 <= 16 else 1 if len(p.words) // 4 <= 32 else
               2 if len(p.words) // 4 <= 64 else 3 for p in plans}
    for b in buckets:
        assert budgets[b] in (24, 32, 40, 56, 80), budgets
    lines = open(path).read().split("\n")
    assert sum(1 for ln in lines if ln.startswith(f"fit {n} {v} ")) == len(buckets)

    c, loss, status, _ = ev.fit_plans(plans, 20)
    # alone and in a different batch: the same bits
    for k in (0, 7, 50):
        c1, l1, s1, _ = ev.fit_plans([plans[k]], 20)
        assert l1[0].tobytes() == loss[k].tobytes() and s1[0] == status[k]
    ev.close()

    # a fresh context reads the table instead of timing again, and answers alike
    ev2 = pkg.GpuEvaluator(x.astype(np.float32).reshape(-1), n, v, y.astype(np.float32))
    ev2.set_fit_data(x.reshape(-1), y)
    assert ev2.fit_autotune(plans, 20, sample=16, path=path) == budgets
    c2, loss2, status2, _ = ev2.fit_plans(plans, 20)
    assert np.array_equal(loss2.view(np.uint64), loss.view(np.uint64))
    ev2.close()

    for k, (t, pl) in enumerate(zip(trees, plans)):
        if status[k] == 0:
            cpu, _ = O.fit(t, x.reshape(-1), n, v, y, 20)
            dev = O.flat_sse(pl.apply(t, c[k][: pl.nconst]), x.reshape(-1), n, v, y)
            assert dev <= cpu * (1 + 1e-3), (k, dev, cpu)
