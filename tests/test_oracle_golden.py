"""Pin the CPU oracle to the reference's own known answers
(tests/golden/reference_known_answers.json, written by make_golden.py from
the reference's test sources) and to properties its tests assert."""
import json
import math
import os

import numpy as np
import pytest

GOLD = json.load(open(os.path.join(os.path.dirname(__file__), "golden",
                                   "reference_known_answers.json")))


def _f(v):
    return float(v)  # "-0.0", "nan", "inf" strings included


def test_centred_ranks_doubled(O):
    for case in GOLD["centred_ranks_doubled"]["cases"]:
        got = O.centred_ranks_doubled([_f(v) for v in case["v"]])
        assert list(got) == case["want"]


def test_rank_scores(O):
    g = GOLD["rank_score"]
    y = np.asarray(g["y"])
    for case in g["cases"]:
        pred = np.asarray([_f(v) for v in case["pred"]])
        metric = O.RANK_CORRELATION_SIGNED if case["signed"] else O.RANK_CORRELATION
        assert O.score_pred(pred, y, metric) == _f(case["want"])
    ct = g["constant_target"]
    assert O.score_pred(ct["pred"], ct["y"], O.RANK_CORRELATION) == ct["want"]
    one = g["one_row"]
    assert O.score_pred(one["pred"], one["y"], O.RANK_CORRELATION) == one["want"]


def test_rank_sums_are_integers_summing_to_zero(O):
    # metrics.rs:2181-2186
    rng = np.random.default_rng(7)
    for n in (1, 2, 3, 17, 1000):
        v = rng.uniform(0, 5, n)
        a = O.centred_ranks_doubled(v)
        assert int(a.sum()) == 0
        assert np.all(np.abs(a) < max(n, 2))


def test_rank_reflection(O):
    # gpu.rs:6364-6670: AB(-pred) = -AB(pred), AA and BB unchanged
    rng = np.random.default_rng(2)
    p = rng.normal(size=500)
    y = rng.normal(size=500)
    ab, aa, bb = O.rank_sums(p, y)
    ab2, aa2, bb2 = O.rank_sums(-p, y)
    assert ab2 == -ab and aa2 == aa and bb2 == bb


def test_recover_sin(E, O):
    g = GOLD["recover_sin"]
    xs = np.linspace(*g["grid"][:2], g["grid"][2])
    ys = np.sin(g["c"] * xs)
    t = E.node(E.SIN, [E.node(E.MUL, [E.constant(1.0), E.input(0)])])
    _, fitted = O.fit(t, xs, len(xs), 1, ys, g["iters"])
    pred = O.predict(fitted, xs, len(xs), 1)
    assert O.score_pred(pred, ys, O.SQUARED) < g["max_squared_error"]


def _circle(n):
    th = 2 * np.pi * np.arange(n) / n
    return np.concatenate([np.cos(th), np.sin(th)])


def test_implicit_circle(E, O):
    g = GOLD["implicit_circle"]
    n = g["points"]
    cols = _circle(n)
    f = E.node(E.SUB, [E.node(E.ADD, [E.node(E.SQUARE, [E.input(0)]),
                                      E.node(E.SQUARE, [E.input(1)])]), E.constant(1.0)])
    assert O.implicit_score(f, cols, n, 2) < g["on_circle_tol"]
    scaled = E.node(E.MUL, [E.constant(7.0), f])
    for i in range(n):
        one = np.asarray([cols[i], cols[n + i]])
        a = O.implicit_score(f, one, 1, 2)
        b = O.implicit_score(scaled, one, 1, 2)
        assert np.float64(a).tobytes() == np.float64(b).tobytes()
    assert O.implicit_score(E.constant(0.0), cols, n, 2) == math.inf
    assert O.implicit_score(E.constant(3.0), cols, n, 2) == math.inf
    f4 = E.node(E.SUB, [E.node(E.ADD, [E.node(E.SQUARE, [E.input(0)]),
                                       E.node(E.SQUARE, [E.input(1)])]), E.constant(4.0)])
    _, fitted = O.implicit_fit(f4, cols, n, 2, g["iters"])
    c = -O.predict(fitted, np.zeros(2), 1, 2)[0]
    assert abs(c - 1.0) < g["radius_tol"]


def test_erf(O):
    g = GOLD["erf"]
    for x, e, ec in g["cases"]:
        assert abs(O.erf(x) - e) <= g["tol"]
        assert abs(O.erfc(x) - ec) <= g["tol"] * max(1.0, abs(ec))
    assert O.erf(float("inf")) == 1.0 and O.erf(float("-inf")) == -1.0
    assert np.float64(O.erf(-0.0)).tobytes() == np.float64(0.0).tobytes()
    assert math.isnan(O.erf(float("nan")))


def test_aic_family(O):
    for case in GOLD["aic"]["cases"]:
        n, rss, k = case["n"], case["rss"], case["k"]
        # a residual vector with the given RSS
        r = np.zeros(n)
        r[0] = math.sqrt(rss)
        y = np.zeros(n)
        assert O.score_pred(r, y, O.AIC, k) == pytest.approx(case["aic"], rel=1e-14)
        assert O.score_pred(r, y, O.BIC, k) == pytest.approx(case["bic"], rel=1e-14)
        assert O.score_pred(r, y, O.AICC, k) == pytest.approx(case["aicc"], rel=1e-14)


def test_cpu_adjoint_matches_central_differences(E, O):
    # fit.rs:1453-1671 against a finite-difference derivative
    t = E.node(E.ADD, [E.node(E.MUL, [E.constant(1.3), E.node(E.SIN, [E.input(0)])]),
                       E.node(E.DIV, [E.constant(0.7), E.node(E.ADD, [E.input(1),
                                                                      E.constant(3.0)])])])
    row = np.asarray([0.4, -0.2])
    v, cg, ig = O.row_grad(t, row)
    cs = np.asarray(t.constants())
    for j in range(len(cs)):
        h = 1e-6
        tp, tm = t.clone(), t.clone()
        a, b = cs.copy(), cs.copy()
        a[j] += h
        b[j] -= h
        tp.set_constants(a)
        tm.set_constants(b)
        fd = (O.row_grad(tp, row)[0] - O.row_grad(tm, row)[0]) / (2 * h)
        assert abs(cg[j] - fd) < 1e-8
    assert abs(ig[0] - 1.3 * math.cos(0.4)) < 1e-14
    assert abs(ig[1] + 0.7 / (2.8 ** 2)) < 1e-14


def test_linear_lm_reaches_the_least_squares_optimum(E, O):
    # the p=1..20 design of gpu.rs:4388-4417 is linear, so the CPU LM must land
    # on numpy's least-squares solution
    n, p = 800, 7
    t = 2 * np.pi * np.arange(n) / (n - 1)
    x = np.stack([np.sin((k + 1) * t) for k in range(p)])
    y = (np.asarray([1.0 + 0.31 * k for k in range(p)])[:, None] * x).sum(0) + \
        (((np.arange(n) * 37) % 11) - 5.0) * 2e-4
    terms = [E.node(E.MUL, [E.constant(0.25 + 0.07 * k), E.input(k)]) for k in range(p)]
    tree = terms.pop()
    while terms:
        tree = E.node(E.ADD, [terms.pop(), tree])
    sse, fitted = O.fit(tree, x.reshape(-1), n, p, y, 8)
    coef, res, *_ = np.linalg.lstsq(x.T, y, rcond=None)
    assert np.allclose(fitted.constants(), coef, rtol=1e-7, atol=1e-9)
    assert abs(sse - float(res[0])) / float(res[0]) < 1e-6
