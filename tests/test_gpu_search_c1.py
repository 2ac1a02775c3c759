"""The plain-method configuration through the build's own generation loop.

Seed 0, 10,000 rows (x ~ U(-5, 5), y = 2x + 1 + N(0, 0.1^2)), an 80/20
split, 4 islands x pop 200, squared error, 8 LM iterations, max complexity
30. The reference search cannot run here, so the candidates are the ones this
build's own loop (`GenerationLoop`: screen -> admit -> fit -> rescore ->
vary, all on the device) generates, and each device fit is held against the
CPU oracle's fit of the same candidate on the same training rows
(fit.rs:2534-2624 fit_lm, 8 iterations): the device's loss within 1e-6
relative of the CPU's or below it, and for a candidate whose device status is
0 and whose CPU fit also ran its course, the same constants to 1e-4.
"""
import concurrent.futures as cf
import importlib
import os

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def test_plain_method_generations_track_the_cpu_fit(pkg, O):
    W = importlib.import_module("the-rule-and-compass_b200.workloads")
    x, y, _, _ = W.line_workload(10000, seed=0)
    n = x.shape[1]
    ev = pkg.GpuEvaluator(x.astype(np.float32).reshape(-1), n, 1, y.astype(np.float32))
    ev.set_fit_data(x.reshape(-1), y)
    loop = pkg.GenerationLoop(ev, 4, 200, 1, max_complexity=30, fit_iters=8, seed=0)
    cols = np.ascontiguousarray(x.reshape(-1))
    records = []
    for g in range(12):
        recs, err = loop.generation()
        assert len(recs) > 0, g
        records += recs
    ev.close()

    def one(r):
        cpu, ctree, (stop, improved, start_ok) = O.fit_lm_traced(r.tree, cols, n, 1, y, 8)
        dev = O.flat_sse(r.fitted(), cols, n, 1, y)
        start = O.flat_sse(r.tree, cols, n, 1, y)
        same_c = None
        if r.status == 0 and stop == 0 and np.isfinite(cpu):
            a = np.asarray(r.fitted().constants())
            b = np.asarray(ctree.constants())
            same_c = bool(np.all(np.abs(a - b) <= 1e-4 * (1.0 + np.abs(b))))
        return cpu, dev, start, r.status, same_c

    with cf.ThreadPoolExecutor(max(1, min(32, os.cpu_count() or 1))) as ex:
        res = list(ex.map(one, records))
    cpu = np.array([q[0] for q in res])
    dev = np.array([q[1] for q in res])
    status = np.array([q[3] for q in res])
    usable = np.isin(status, [0, 4, 5, 6, 7, 8])
    fin = np.isfinite(cpu)
    ok = usable & fin
    within = dev[ok] <= cpu[ok] * (1.0 + 1e-6) + 1e-300
    same = [q[4] for q in res if q[4] is not None]
    print(f"\nC1: {len(records)} fitted candidates over 12 generations; usable "
          f"{int(usable.sum())}; device loss within 1e-6 of the CPU fit or below "
          f"{int(within.sum())}/{int(ok.sum())}; constants equal to 1e-4 "
          f"{sum(same)}/{len(same)}; status {np.bincount(status, minlength=9).tolist()}")
    assert usable.mean() >= 0.95
    assert within.mean() >= 0.95, np.sort((dev[ok] - cpu[ok]) / np.abs(cpu[ok]))[-10:]
    assert len(same) > 0 and np.mean(same) >= 0.9
    # the search finds the line: the best rescored training error is tiny
    assert np.nanmin(err) < 0.05
