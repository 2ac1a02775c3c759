"""The exactness gate of the CPU oracle against the reference's own gate tests.

`oracle.fit_verified` restates `fit_batch_verified` / `verify_proposal`
(my-version/src/fit/gpu.rs:176-317): a device proposal replaces the starting
constants only when it is finite, of the right length and no worse on the
configured objective; otherwise the exact CPU fit runs from the start. The
cases restate my-version/src/fit/gpu.rs:758-805 (squared) and :831-872,
:1488-1538 (a robust proposal judged by its own metric, not by SSE).
"""
import numpy as np


def _model(E):
    # fit/gpu.rs:705-710: 0.7 x + 0.1
    return E.node(E.ADD, [E.node(E.MUL, [E.constant(0.7), E.input(0)]), E.constant(0.1)])


def _line(n=20):
    x = np.arange(n, dtype=np.float64)
    return x, 2.0 * x + 3.0


def _outlier_rows():
    # fit/gpu.rs:833-838: an affine trend with 5 % gross outliers
    x = np.arange(40, dtype=np.float64) / 4.0
    y = 1.0 + 0.5 * x
    y[3::8] += 40.0
    return x, y


def test_a_good_proposal_is_accepted(E, O):
    x, y = _line()
    score, tree, state = O.fit_verified(_model(E), x, len(x), 1, y, 8, [2.0, 3.0])
    assert state == 0
    assert score < 1e-20
    c = O.flat_constants(tree)
    assert abs(c[0] - 2.0) < 1e-12 and abs(c[1] - 3.0) < 1e-12


def test_non_finite_wrong_length_and_missing_proposals_fall_back_exactly(E, O):
    x, y = _line()
    ref, cpu = O.fit(_model(E), x, len(x), 1, y, 8)
    for proposal, want_state in (([np.nan, 3.0], 1), ([2.0], 1), (None, 2)):
        score, tree, state = O.fit_verified(_model(E), x, len(x), 1, y, 8, proposal)
        assert state == want_state
        assert np.float64(score).view(np.uint64) == np.float64(ref).view(np.uint64)
        assert np.array_equal(O.flat_constants(tree).view(np.uint64),
                              O.flat_constants(cpu).view(np.uint64))


def test_a_worse_proposal_never_replaces_the_cpu_fit(E, O):
    x, y = _line()
    ref, _ = O.fit(_model(E), x, len(x), 1, y, 8)
    score, _, state = O.fit_verified(_model(E), x, len(x), 1, y, 8, [0.0, 0.0])
    assert state != 0
    assert np.float64(score).view(np.uint64) == np.float64(ref).view(np.uint64)


def test_a_robust_proposal_is_judged_by_its_own_metric(E, O):
    x, y = _outlier_rows()
    n = len(x)
    for metric in (O.LOG_SQUASHED, O.ABSOLUTE):
        robust, reference = O.fit(_model(E), x, n, 1, y, 8, metric)
        proposal = O.flat_constants(reference)
        start = O.flat_sse(_model(E), x, n, 1, y)
        assert O.flat_sse(reference, x, n, 1, y) > start, "the fixture must cost SSE"
        score, tree, state = O.fit_verified(_model(E), x, n, 1, y, 8, proposal, metric)
        assert state == 0, metric
        assert np.float64(score).view(np.uint64) == np.float64(robust).view(np.uint64)
        assert np.array_equal(O.flat_constants(tree).view(np.uint64), proposal.view(np.uint64))


def test_the_traced_lm_is_fit_lm_bit_for_bit(E, O):
    """fit_lm_traced is fit_lm plus a record of how its loop ended."""
    x = np.linspace(-2, 2, 200)
    y = 1.5 * np.sin(0.8 * x) + 0.2
    t = E.node(E.ADD, [E.node(E.MUL, [E.constant(1.0), E.node(E.SIN, [
        E.node(E.MUL, [E.constant(1.0), E.input(0)])])]), E.constant(0.0)])
    a, ta = O.fit(t, x, len(x), 1, y, 20)
    b, tb, (stop, improved, start_ok) = O.fit_lm_traced(t, x, len(x), 1, y, 20)
    assert np.float64(a).view(np.uint64) == np.float64(b).view(np.uint64)
    assert np.array_equal(O.flat_constants(ta), O.flat_constants(tb))
    assert stop == 0 and improved == 1 and start_ok == 1
    # exp(c x) with c = 800 overflows f64 at x > 0.89: not finite from the start
    bad = E.node(E.MUL, [E.constant(1.0), E.node(E.EXP, [
        E.node(E.MUL, [E.constant(800.0), E.input(0)])])])
    _, _, (stop, improved, start_ok) = O.fit_lm_traced(bad, x, len(x), 1, y, 20)
    assert start_ok == 0 and stop == 2 and improved == 0
    assert not O.normal_equations_ok(bad, x, len(x), 1, y)
