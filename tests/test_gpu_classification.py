"""The classification score objectives (kinds 10-14: log-loss, Brier, the
sigmoid hinge, the ordinary and the squared hinge) on the device against the
oracle's restatement of metrics::score_native_weighted
(my-version/src/metrics.rs:705-763, :1534-1579), as the reference's
native-objective test does for the regression kinds (gpu.rs:3147-3212): the
device's value equals the CPU reducer on the device's own f32 predictions
widened to f64 (or, for a candidate its error bound sends to the f64 lane,
on the f64 predictions), unweighted and with row weights including zeros.
The label sign t = 2l - 1 is derived on the host from the target midpoint
(metrics.rs:1467-1532) and uploaded with rc_set_fit_sign."""
import importlib

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

KINDS = [10, 11, 12, 13, 14]


def _data(n, seed):
    rng = np.random.Generator(np.random.PCG64(seed))
    x = rng.standard_normal((3, n)).astype(np.float32)
    score = 1.3 * x[0] - 0.7 * x[1] * x[2] + rng.normal(0, 0.3, n)
    y = np.where(score > 0.0, 1.0, 0.0).astype(np.float32)
    return x, y


@pytest.mark.parametrize("weighted", [False, True])
def test_classification_objectives_match_the_cpu_reducer(pkg, O, weighted):
    W = importlib.import_module("the-rule-and-compass_b200.workloads")
    n, v = 6000, 3
    x, y = _data(n, 17)
    rng = np.random.Generator(np.random.PCG64(4))
    trees = [W.random_scoring_tree(rng, v) for _ in range(48)]
    y64 = y.astype(np.float64)
    w = None
    if weighted:
        w = rng.uniform(0.0, 2.0, n)
        w[rng.random(n) < 0.1] = 0.0
    labels = O.binary_labels(y64, w)
    ev = pkg.GpuEvaluator(x.reshape(-1), n, v, y)
    ev.set_fit_sign(2.0 * labels - 1.0)
    if weighted:
        ev.set_score_weights(w)
    prog, off = pkg.Population(trees).programs()
    preds = ev.predictions(prog, off).astype(np.float64)
    x64 = x.astype(np.float64).reshape(-1)
    checked = 0
    for kind in KINDS:
        vals, status, ms = ev.score_batch(prog, off, kind)
        assert ms >= 0
        for k, t in enumerate(trees):
            want32 = O.score_pred(preds[k], y64, kind, 0, w)
            t32 = t.clone()
            t32.set_constants([float(np.float32(c)) for c in t.constants()])
            want64 = O.score_pred(O.predict(t32, x64, n, v), y64, kind, 0, w)
            if not np.isfinite(want64):
                assert status[k] == 2 and np.isinf(vals[k]), (kind, k, status[k], vals[k])
                continue
            if status[k] != 0:
                # the f32 rows failed where f64 did not: only allowed when the
                # f32 predictions themselves are not finite
                assert not np.isfinite(want32), (kind, k, status[k])
                continue
            tol = 1e-12 * (1.0 + abs(want64))
            assert min(abs(vals[k] - want32), abs(vals[k] - want64)) <= tol, \
                (kind, k, vals[k], want32, want64)
            checked += 1
    assert checked >= len(KINDS) * 10, checked
    ev.close()


def test_classification_labels_and_extremes(pkg, O):
    """metrics.rs:1934-1944 on the device: log-loss of confident correct and
    wrong logits (0 and the margin), ln 2 at a zero logit."""
    n = 4
    x = np.array([[-1e6, 1e6, 0.0, 0.0]], np.float32)
    y = np.array([0.0, 1.0, 0.0, 1.0], np.float32)
    ev = pkg.GpuEvaluator(x.reshape(-1), n, 1, y)
    ev.set_fit_sign(2.0 * O.binary_labels(y.astype(np.float64)) - 1.0)
    VAR, NEG, HALT = 1, 17, 255
    prog = np.array([VAR, 0, HALT, VAR, 0, NEG, HALT], np.uint32)
    off = np.array([0, 3, 7], np.uint32)
    vals, status, _ = ev.score_batch(prog, off, 10)
    assert list(status) == [0, 0]
    want = [O.score_pred(x[0].astype(np.float64), y.astype(np.float64), 10),
            O.score_pred(-x[0].astype(np.float64), y.astype(np.float64), 10)]
    assert vals[0] == pytest.approx(want[0], rel=1e-9, abs=1e-12)
    assert vals[1] == pytest.approx(want[1], rel=1e-9)
    assert want[0] == pytest.approx(np.log(2.0) / 2.0, rel=1e-12)
    ev.close()
