"""The oracle's classification objectives (score kinds 10-14) against the
reference's own known answers (my-version/src/metrics.rs:1873-2140):
the three hinge forms, the stable log-loss at extreme logits, the constant
model optima of log-loss and Brier, weighted rows as duplicated rows, and
zero-weight rows that stay invisible."""
import math

import numpy as np
import pytest

KINDS = [10, 11, 12, 13, 14]


def sp(O, p, y, kind, w=None):
    return O.score_pred(np.asarray(p, float), np.asarray(y, float), kind, 0,
                        None if w is None else np.asarray(w, float))


def test_hinge_forms_are_distinct(O):
    # metrics.rs:1894-1930
    y = [0.0, 1.0]
    assert sp(O, [0.0, 0.0], y, O.HINGE_SIGMOID) == pytest.approx(1.0, abs=1e-12)
    assert sp(O, [0.0, 0.0], y, O.HINGE_ORDINARY) == pytest.approx(1.0, abs=1e-12)
    assert sp(O, [0.0, 0.0], y, O.HINGE_SQUARED) == pytest.approx(1.0, abs=1e-12)
    good = [-30.0, 30.0]
    assert sp(O, good, y, O.HINGE_SIGMOID) > 0.0
    assert sp(O, good, y, O.HINGE_ORDINARY) == pytest.approx(0.0, abs=1e-12)
    assert sp(O, good, y, O.HINGE_SQUARED) == pytest.approx(0.0, abs=1e-12)
    half = [-0.5, 0.5]
    assert sp(O, half, y, O.HINGE_ORDINARY) == pytest.approx(0.5, abs=1e-12)
    assert sp(O, half, y, O.HINGE_SQUARED) == pytest.approx(0.25, abs=1e-12)
    kink = [-1.0, 1.0]
    assert sp(O, kink, y, O.HINGE_ORDINARY) == pytest.approx(0.0, abs=1e-12)
    assert sp(O, kink, y, O.HINGE_SQUARED) == pytest.approx(0.0, abs=1e-12)


def test_log_loss_is_the_stable_softplus(O):
    # metrics.rs:1934-1944
    y = [0.0, 1.0]
    assert sp(O, [-1e6, 1e6], y, O.LOG_LOSS) == 0.0
    assert sp(O, [1e6, -1e6], y, O.LOG_LOSS) == pytest.approx(1e6, rel=1e-6)
    assert sp(O, [0.0, 0.0], y, O.LOG_LOSS) == pytest.approx(math.log(2.0), abs=1e-15)


def test_constant_model_optima(O):
    # metrics.rs:1947-1977
    y = [1.0, 1.0, 1.0, 0.0]
    b = math.log(3.0)
    best = sp(O, [b] * 4, y, O.LOG_LOSS)
    best_brier = sp(O, [b] * 4, y, O.BRIER)
    for d in (-0.25, -0.01, 0.01, 0.25):
        assert sp(O, [b + d] * 4, y, O.LOG_LOSS) >= best - 1e-15
        assert sp(O, [b + d] * 4, y, O.BRIER) >= best_brier - 1e-15
    assert best_brier == pytest.approx(0.75 * 0.25, abs=1e-12)
    assert math.isfinite(sp(O, [0.0, 0.0], [0.0, 0.0], O.BRIER))


def test_weighted_rows_are_duplicated_rows(O):
    # metrics.rs:2064-2101
    y = [0.0, 1.0, 1.0, 0.0, 1.0, 0.0]
    p = [-1.5, 0.3, 2.2, -0.4, 0.8, 0.1]
    w = [1.0, 2.0, 1.0, 3.0, 1.0, 1.0]
    dp, dy = [], []
    for pi, yi, wi in zip(p, y, w):
        dp += [pi] * int(wi)
        dy += [yi] * int(wi)
    for kind in KINDS:
        assert sp(O, p, y, kind, w) == pytest.approx(sp(O, dp, dy, kind), abs=1e-12)
    for kind in (10, 11, 12):
        assert sp(O, p, y, kind, w) == pytest.approx(sp(O, p, y, kind, np.asarray(w) * 7.5),
                                                     abs=1e-12)


def test_zero_weight_rows_are_invisible(O):
    # metrics.rs:2105-2137
    y = [0.0, 1.0, 0.0, 1.0]
    p = [0.2, -0.4, 0.9, 1.3]
    w = [1.0, 1.0, 0.0, 1.0]
    for kind in KINDS:
        base = sp(O, p, y, kind, w)
        for pp, yy in (([0.2, -0.4, math.nan, 1.3], y), (p, [0.0, 1.0, math.nan, 1.0]),
                       (p, [0.0, 1.0, math.inf, 1.0])):
            assert np.float64(sp(O, pp, yy, kind, w)).tobytes() == np.float64(base).tobytes()
    wb = [1.0] * 4
    assert sp(O, p, [0.0, 1.0, math.nan, 1.0], O.LOG_LOSS, wb) == math.inf
    assert sp(O, [0.2, math.nan, 0.9, 1.3], y, O.BRIER, wb) == math.inf


def test_labels_from_the_target_midpoint(O):
    # metrics.rs:1467-1475: l = [y > (min + max) / 2]
    assert list(O.binary_labels([-1.0, 0.0, 1.0, 0.2])) == [0.0, 0.0, 1.0, 1.0]
    assert list(O.binary_labels([3.0, 5.0, 5.0], [1.0, 0.0, 1.0])) == [0.0, 0.0, 1.0]
