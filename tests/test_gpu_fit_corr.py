"""The correlation fit arm on the device (metric codes 2 and 3,
my-version/src/cuda/eval.cu:1959-2440) against the recipes of the
reference's own tests (my-version/src/gpu.rs:5532-5660): the fitted
objective reaches the CPU optimum of 1 - |rho| (here the optimum of the
oracle's exact correlation metric over the free constant), the affine gauge
is renormalised to (sign, 0) and frozen, repeated fits are bit-identical, a
constant prediction scores exactly 1 with its constants kept, and a
non-finite start is labelled 7."""
import numpy as np
import pytest
from scipy.optimize import minimize_scalar

pytestmark = pytest.mark.gpu

CORR, CORR_SIGNED = 2, 3


def corr_fixture(n):
    x = -3.0 + 6.0 * np.arange(n) / (n - 1)
    noise = (((np.arange(n) * 29) % 13) - 6.0) * 1e-4
    y = 1.6 * np.sin(0.7 * x) + 0.35 * x + 0.2 + noise
    return x[None, :], y


def corr_model(E, a=0.8, f=1.1, b=0.25):
    return E.node(E.ADD, [E.node(E.MUL, [E.constant(a), E.node(E.SIN, [
        E.node(E.MUL, [E.constant(f), E.input(0)])])]), E.constant(b)])


def evaluator(pkg, x, y):
    v, n = x.shape
    ev = pkg.GpuEvaluator(x.astype(np.float32).reshape(-1), n, v, y.astype(np.float32))
    # the f64 rows are the f32 inputs widened, as the reference test uploads
    ev.set_fit_data(x.astype(np.float32).astype(np.float64).reshape(-1), y)
    return ev


def test_correlation_fit_reaches_the_cpu_optimum(pkg, E, O):
    n = 600
    x, y = corr_fixture(n)
    x64 = x.astype(np.float32).astype(np.float64)
    ev = evaluator(pkg, x, y)
    t = corr_model(E)
    plan = pkg.gpu_fit_plan(t)
    assert list(plan.gauge) == [0, 2]
    c, loss, status, _ = ev.fit_plans([plan], 8, metric=CORR)
    assert status[0] == 0
    assert c[0][0] in (1.0, -1.0) and c[0][2] == 0.0
    fitted = plan.apply(t, c[0][: plan.nconst])
    gpu_score = O.score(fitted, x64.reshape(-1), n, 1, y, O.CORRELATION)
    assert abs(loss[0] - gpu_score) <= 1e-6
    r = minimize_scalar(lambda f: O.score(corr_model(E, 1.0, f, 0.0), x64.reshape(-1), n, 1, y,
                                          O.CORRELATION),
                        bounds=(0.3, 1.5), method="bounded", options={"xatol": 1e-12})
    assert gpu_score <= r.fun + 1e-6, (gpu_score, r.fun)
    start = O.score(t, x64.reshape(-1), n, 1, y, O.CORRELATION)
    assert gpu_score < start
    again = ev.fit_plans([plan], 8, metric=CORR)
    assert np.array_equal(again[0].view(np.uint64), c.view(np.uint64))
    assert again[1][0] == loss[0]
    ev.close()


def test_signed_correlation_and_batch_independence(pkg, E, O):
    n = 900
    x, y = corr_fixture(n)
    x64 = x.astype(np.float32).astype(np.float64)
    ev = evaluator(pkg, x, y)
    trees = [corr_model(E), corr_model(E, -0.5, 0.9, 1.0),
             E.node(E.MUL, [E.constant(2.0), E.node(E.SIN, [E.node(E.MUL, [E.constant(0.8),
                                                                             E.input(0)])])])]
    plans = [pkg.gpu_fit_plan(tr) for tr in trees]
    c, loss, status, _ = ev.fit_plans(plans, 10, metric=CORR_SIGNED)
    for k, (tr, pl) in enumerate(zip(trees, plans)):
        assert status[k] in (0, 4, 5, 6)
        fitted = pl.apply(tr, c[k][: pl.nconst])
        s = O.score(fitted, x64.reshape(-1), n, 1, y, O.CORRELATION_SIGNED)
        assert abs(loss[k] - s) <= 1e-6
        assert s <= O.score(tr, x64.reshape(-1), n, 1, y, O.CORRELATION_SIGNED) + 1e-12
        one = ev.fit_plans([pl], 10, metric=CORR_SIGNED)
        assert one[1][0] == loss[k] and one[2][0] == status[k]
        assert np.array_equal(one[0][0][: pl.nconst], c[k][: pl.nconst])
    ev.close()


def test_degenerate_and_non_finite_correlation(pkg, E):
    n = 200
    x, y = corr_fixture(n)
    ev = evaluator(pkg, x, y)
    flat = E.node(E.ADD, [E.node(E.SIN, [E.node(E.MUL, [E.constant(0.0), E.input(0)])]),
                          E.constant(0.5)])
    plan = pkg.gpu_fit_plan(flat)
    c, loss, status, _ = ev.fit_plans([plan], 8, metric=CORR)
    assert status[0] == 0 and loss[0] == 1.0
    assert np.array_equal(c[0][: plan.nconst], np.asarray(plan.c0))
    ev.close()
    y2 = y.copy()
    y2[7] = np.nan
    ev = evaluator(pkg, x, y2)
    plan = pkg.gpu_fit_plan(corr_model(E))
    _, _, status, _ = ev.fit_plans([plan], 8, metric=CORR)
    assert status[0] == 7
    ev.close()
