"""The exact f64 finalist refit and the structure-of-arrays evaluator on the
host cores (host/refit.cpp, include/rcsr_refit.h), checked bit for bit
against the CPU oracle's row-at-a-time restatement of the reference's
`fit_lm` / IRLS / `expr::eval`, and against the reference's own refit tests
(my-version/src/fit/gpu.rs:806-824 and :870-900). Runs on the CPU."""
import importlib

import numpy as np
import pytest


def _W():
    return importlib.import_module("the-rule-and-compass_b200.workloads")


def _bits(a):
    return np.asarray(a, np.float64).view(np.uint64)


def _same(a, b):
    """Bit-identical, NaN payloads aside."""
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    both_nan = np.isnan(a) & np.isnan(b)
    return bool(np.all(both_nan | (_bits(a) == _bits(b))))


def _affine_sine(E):
    """c0 * sin(c1 * x0) + c2 at c = (1, 1, 0)."""
    return E.node(E.ADD, [
        E.node(E.MUL, [E.constant(1.0),
                       E.node(E.SIN, [E.node(E.MUL, [E.constant(1.0), E.input(0)])])]),
        E.constant(0.0)])


def test_finalist_refit_is_the_exact_lm_path(pkg, E, O):
    """fit/gpu.rs:806-824: the refit of a finalist is `fit_weighted` bit for
    bit (40 rows on [-2, 1.9], y = 1.5 sin(0.8 x) + 0.2, 40 iterations)."""
    x = np.array([-2.0 + 0.1 * i for i in range(40)])
    y = 1.5 * np.sin(0.8 * x) + 0.2
    t = _affine_sine(E)
    loss, out = pkg.host.refit_finalists_exact([t], x, y, 40, "squared")
    want, ref = O.fit(t, x, 40, 1, y, 40)
    assert _bits(loss[0]) == _bits(want)
    assert _same(out[0].constants(), ref.constants())
    assert loss[0] < 1e-12


def test_robust_finalist_refit_is_idempotent(pkg, E, O):
    """fit/gpu.rs:870-900: a log-squashed refit from its own endpoint changes
    nothing, and the value reported is the configured loss."""
    x = np.array([-1.5 + 0.05 * i for i in range(60)])
    y = 2.0 * np.sin(1.3 * x) + np.array([6.0 if i % 7 == 0 else 0.0 for i in range(60)])
    t = _affine_sine(E)
    first, once = pkg.host.refit_finalists_exact([t], x, y, 8, "log_squashed")
    second, twice = pkg.host.refit_finalists_exact(once, x, y, 8, "log_squashed")
    assert _bits(first[0]) == _bits(second[0])
    assert _same(once[0].constants(), twice[0].constants())
    want, ref = O.fit(t, x, 60, 1, y, 8, metric=2)
    assert _bits(first[0]) == _bits(want)
    assert _same(once[0].constants(), ref.constants())
    pred = pkg.host.soa_eval(once[0], x, 60)
    assert first[0] == pytest.approx(np.mean(np.log1p((pred - y) ** 2)), rel=1e-12)


@pytest.mark.parametrize("metric,code", [("squared", 0), ("aic", 7), ("absolute", 1),
                                         ("log_squashed", 2)])
@pytest.mark.parametrize("weighted", [False, True])
def test_benchmark_trees_refit_bit_identically(pkg, O, metric, code, weighted):
    """The fit benchmark's tree distribution (1-20 constants, 5-60 nodes) at
    a row count that is not a multiple of the block: losses and constants
    equal the oracle's row walk bit for bit, with and without weights (a
    tenth of them zero)."""
    trees, x, y = _W().fit_workload(12, 1000, seed=5 + code)
    v, n = x.shape
    w = None
    if weighted:
        rng = np.random.default_rng(3)
        w = rng.uniform(0.2, 2.0, n)
        w[rng.random(n) < 0.1] = 0.0
    xs = np.ascontiguousarray(x, np.float64).reshape(-1)
    loss, out = pkg.host.refit_finalists_exact(trees, xs, y, 6, metric, w=w, threads=4)
    for k, t in enumerate(trees):
        want, ref = O.fit(t, xs, n, v, y, 6, metric=code, w=w)
        assert _same(loss[k], want), (k, loss[k], want)
        assert _same(out[k].constants(), ref.constants()), k


def test_threads_do_not_change_the_result(pkg):
    trees, x, y = _W().fit_workload(10, 700, seed=2)
    xs = np.ascontiguousarray(x, np.float64).reshape(-1)
    a, ta = pkg.host.refit_finalists_exact(trees, xs, y, 5, "squared", threads=1)
    b, tb = pkg.host.refit_finalists_exact(trees, xs, y, 5, "squared", threads=0)
    assert _same(a, b)
    for p, q in zip(ta, tb):
        assert _same(p.constants(), q.constants())


def test_edge_cases(pkg, E, O):
    x = np.linspace(-1.0, 1.0, 300)
    y = 2.0 * x + 1.0
    # a constant-free tree, zero iterations, and the iterations-zero score
    free = E.node(E.MUL, [E.input(0), E.input(0)])
    loss, _ = pkg.host.refit_finalists_exact([free], x, y, 10, "squared")
    assert _bits(loss[0]) == _bits(O.fit(free, x, 300, 1, y, 10)[0])
    t = E.node(E.ADD, [E.node(E.MUL, [E.constant(0.5), E.input(0)]), E.constant(0.0)])
    for metric, code in (("squared", 0), ("absolute", 1)):
        loss, out = pkg.host.refit_finalists_exact([t], x, y, 0, metric)
        assert _bits(loss[0]) == _bits(O.fit(t, x, 300, 1, y, 0, metric=code)[0])
        assert out[0].constants() == t.constants()
    # a tree that is undefined everywhere keeps its constants
    bad = E.node(E.LOG, [E.node(E.SUB, [E.constant(-1.0), E.node(E.MUL, [E.input(0),
                                                                        E.input(0)])])])
    loss, out = pkg.host.refit_finalists_exact([bad], x, y, 5, "squared")
    assert loss[0] == np.inf and out[0].constants() == bad.constants()
    # no finalists, and a metric the refit does not cover
    loss, out = pkg.host.refit_finalists_exact([], x, y, 5, "squared")
    assert len(loss) == 0 and out == []
    with pytest.raises(ValueError):
        pkg.host.refit_finalists_exact([t], x, y, 5, "median")


def test_soa_evaluator_matches_the_tree_walk(pkg, O):
    """Predictions of the scoring benchmark's trees (every operator of its
    set, domain guards included) equal the oracle's tree walk bit for bit,
    NaN for NaN; and the SSE is the plain sum with +inf on a non-finite
    prediction (eval_soa.rs:522-540)."""
    W = _W()
    rng = np.random.default_rng(11)
    x = rng.normal(size=(5, 777))
    x[:, :5] = [[0.0, -0.0, 1e-13, -3.0, 700.5]] * 5
    y = rng.normal(size=777)
    xs = np.ascontiguousarray(x).reshape(-1)
    finite = 0
    for _ in range(60):
        t = W.random_scoring_tree(rng)
        got = pkg.host.soa_eval(t, xs, 777)
        want = O.predict(t, xs, 777, 5)
        assert _same(got, want), t
        sse = pkg.host.soa_sse(t, xs, y)
        if np.all(np.isfinite(want)):
            finite += 1
            acc = 0.0
            for e in want - y:  # sequential (sum() compensates on Python >= 3.12)
                acc += float(e) * float(e)
            assert _bits(sse) == _bits(acc)
        else:
            assert sse == np.inf
    assert finite >= 10


def test_soa_evaluator_covers_every_operator(pkg, E, O):
    """One tree per operator (codes 2..42 and the inverse hyperbolics) over
    inputs that hit each guard."""
    vals = np.array([-2.5, -1.0, -1e-13, 0.0, 1e-13, 0.5, 1.0, 1.5, 3.0, 701.0, np.nan, np.inf])
    xs = np.concatenate([vals, vals[::-1]])
    n = len(vals)
    for op in list(range(2, 43)) + [64, 65, 66]:
        ar = E.arity(op)
        kids = [E.input(0), E.input(1), E.input(0)][:ar]
        t = E.node(op, kids)
        assert _same(pkg.host.soa_eval(t, xs, n), O.predict(t, xs, n, 2)), op


@pytest.mark.parametrize("metric,code", [("squared", 0), ("absolute", 1)])
def test_a_refit_split_over_threads_is_bit_identical(pkg, O, metric, code):
    """Fewer finalists than threads and enough rows: each refit's passes are
    split by rows over a team of threads (two chunks of rows here), with the
    sums still taken in row order; the result equals the one-thread refit
    and the oracle's row walk bit for bit, zero weights included."""
    trees, x, y = _W().fit_workload(3, 70000, seed=21)
    v, n = x.shape
    rng = np.random.default_rng(8)
    w = rng.uniform(0.5, 1.5, n)
    w[rng.random(n) < 0.05] = 0.0
    xs = np.ascontiguousarray(x, np.float64).reshape(-1)
    one, t1 = pkg.host.refit_finalists_exact(trees, xs, y, 4, metric, w=w, threads=1)
    team, t6 = pkg.host.refit_finalists_exact(trees, xs, y, 4, metric, w=w, threads=6)
    assert _same(one, team)
    for k, t in enumerate(trees):
        assert _same(t1[k].constants(), t6[k].constants())
        want, ref = O.fit(t, xs, n, v, y, 4, metric=code, w=w)
        assert _same(team[k], want), (k, team[k], want)
        assert _same(t6[k].constants(), ref.constants())
