"""The `gpu.fit` run-record (my-version/src/main.rs:995-1010) and its
accounting (my-version/src/search.rs:2040-2120, :2939-2959): restated from
the reference's own ledger test (main.rs:9676-9704) and its cause rules.
Runs on the CPU."""
import importlib

import numpy as np


def _host():
    return importlib.import_module("the-rule-and-compass_b200.host")


def test_ledger_json_matches_the_reference_layout():
    H = _host()
    L = H.FitLedger()
    L.screened, L.attempts, L.gpu, L.fallback = 100, 40, 37, 3
    L.fallback_by_cause = {"non_finite": 1, "ill_conditioned": 2}
    L.status_by_label = {"rank_deficient": 4}
    L.refits = 5
    L.seconds, L.host_seconds, L.fallback_seconds = 0.25, 0.5, 0.125
    L.fallback_bounded, L.fallback_workers, L.fallback_max = 0, 8, 4096
    assert L.to_json() == (
        '"fit":{"strategy":"gpu","screened":100,"attempts":40,"gpu":37,"fallback":3,'
        '"fallback_by_cause":{"ill_conditioned":2,"non_finite":1},'
        '"status_by_label":{"rank_deficient":4},"refits":5,"seconds":0.25,'
        '"host_seconds":0.5,"fallback_seconds":0.125,"fallback_bounded":0,'
        '"fallback_workers":8,"fallback_max":4096}')


def test_status_rules():
    H = _host()
    assert [H.fit_status_usable(s) for s in range(9)] == [True, False, False, False, True,
                                                          True, True, True, True]
    assert H.status_fallback_cause(1) == "ill_conditioned"
    assert H.status_fallback_cause(2) == "non_finite"
    assert H.status_fallback_cause(3) == "rank_declined"
    assert H.status_fallback_cause(9) == "unsupported_plan"


def test_batch_accounting(E):
    H = _host()
    x = E.input(0)
    fit = E.node(E.ADD, [E.node(E.MUL, [E.constant(1.5), x]), E.constant(0.5)])
    no_const = E.node(E.SIN, [x])
    many = E.constant(1.0)
    for k in range(24):
        many = E.node(E.ADD, [many, E.node(E.MUL, [E.constant(float(k)), x])])
    L = H.FitLedger()
    trees = [fit, no_const, many, fit, fit, fit, fit]
    # planned, in order: fit x5
    c = np.zeros((5, 2))
    c[4, 0] = np.nan
    L.record_batch(trees, c, [0, 4, 1, 2, 0], 12.5)
    assert L.attempts == 6                       # the constant-free tree is not offered
    assert L.gpu == 2 and L.status_by_label == {"rank_deficient": 1}
    assert L.fallback_by_cause == {"too_many_constants": 1, "ill_conditioned": 1,
                                   "non_finite": 2}
    assert L.fallback == 4 and abs(L.seconds - 0.0125) < 1e-15
    L.record_batch([fit, fit], np.zeros((2, 2)), [0, 0], -1.0)
    assert L.fallback_by_cause["launch"] == 2 and L.attempts == 8
