"""Exact statistics on the device against the CPU oracle: rank-correlation
sums (my-version/src/gpu.rs:6364-6670 recipes: target ranks, bit-identical
sums for linear / tied / flat models, ties and constant predictions),
order statistics of |r| and the maximum-error scan."""
import importlib

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _evaluator(pkg, cols, y):
    v, n = cols.shape
    ev = pkg.GpuEvaluator(cols.astype(np.float32).reshape(-1), n, v, y.astype(np.float32))
    ev.set_fit_data(cols.reshape(-1), y)
    return ev


def _fixture(n, seed=0, tied_y=True):
    """Integer-valued x0 (many ties), continuous x1, and a target with
    repeated values and a signed zero."""
    rng = np.random.Generator(np.random.PCG64(seed))
    x0 = rng.integers(-6, 7, n).astype(np.float64)
    x1 = rng.uniform(-2.0, 2.0, n)
    x2 = rng.normal(0.0, 1.0, n)
    y = 0.5 * x0 + np.sin(x1) + 0.1 * x2
    if tied_y:
        y = np.round(y, 1)
        y[::97] = -0.0
        y[1::97] = 0.0
    return np.stack([x0, x1, x2]), y


def _models(E):
    linear = E.node(E.ADD, [E.node(E.MUL, [E.constant(2.0), E.input(1)]), E.constant(1.0)])
    tied = E.node(E.ADD, [E.node(E.MUL, [E.constant(0.5), E.input(0)]), E.constant(-1.0)])
    flat = E.node(E.MUL, [E.constant(0.0), E.input(0)])
    return {"linear": linear, "tied": tied, "flat": flat}


def _pack(pkg, trees):
    plans = [pkg.gpu_fit_plan(t, allow_no_constants=True) for t in trees]
    prog, off, pcount, c0, gauge, kmax = pkg.pack_plans(plans)
    return plans, prog, off, pcount, c0, kmax


def _oracle_pred(O, t, cols):
    v, n = cols.shape
    return np.asarray(O.predict(t, cols.reshape(-1), n, v), np.float64)


def test_target_ranks_match_the_oracle(pkg, O):
    cols, y = _fixture(10007)
    ev = _evaluator(pkg, cols, y)
    b = ev.rank_target()
    want = O.centred_ranks_doubled(y)
    assert np.array_equal(b, want)
    ev.close()


@pytest.mark.parametrize("n", [5, 4096, 4097, 10007, 70001])
def test_rank_sums_are_bit_identical(pkg, E, O, n):
    cols, y = _fixture(n, seed=n)
    ev = _evaluator(pkg, cols, y)
    models = _models(E)
    trees = list(models.values())
    plans, prog, off, pcount, c0, kmax = _pack(pkg, trees)
    sums, status, bb, _ = ev.rank_sums(prog, off, pcount, c0, kmax)
    for k, t in enumerate(trees):
        ab, aa, bb_cpu = O.rank_sums(_oracle_pred(O, t, cols), y)
        assert status[k] == 0
        assert sums[k] == (ab, aa), (list(models)[k], sums[k], (ab, aa))
        assert bb == bb_cpu
    # the flat model: one run, A = 0 everywhere
    assert sums[2] == (0, 0)
    ev.close()


@pytest.mark.parametrize("n", [500, 5000])
def test_rank_sums_of_keys_that_agree_in_their_upper_halves(pkg, E, O, n):
    """Predictions whose f64 bit patterns share their upper 32 bits in long
    groups and differ below: integer x0 plus a 1e-9 x1 perturbation puts
    about n / 13 distinct keys in each group, and 1 + 1e-12 x2 puts all of
    them in one; the lower digit passes alone order them. Mixed in one batch
    with models whose keys spread over every digit, the sums must equal the
    CPU's exactly."""
    cols, y = _fixture(n, seed=17)
    ev = _evaluator(pkg, cols, y)
    clustered = E.node(E.ADD, [E.node(E.MUL, [E.constant(0.5), E.input(0)]),
                               E.node(E.MUL, [E.constant(1e-9), E.input(1)])])
    near = E.node(E.ADD, [E.constant(1.0), E.node(E.MUL, [E.constant(1e-12), E.input(2)])])
    models = _models(E)
    trees = [models["linear"], clustered, near, models["tied"]]
    plans, prog, off, pcount, c0, kmax = _pack(pkg, trees)
    sums, status, bb, _ = ev.rank_sums(prog, off, pcount, c0, kmax)
    for k, t in enumerate(trees):
        ab, aa, bb_cpu = O.rank_sums(_oracle_pred(O, t, cols), y)
        assert status[k] == 0
        assert sums[k] == (ab, aa), (k, sums[k], (ab, aa))
        assert bb == bb_cpu
    ev.close()


def test_rank_sums_of_random_models_and_trials(pkg, E, O):
    W = importlib.import_module("the-rule-and-compass_b200.workloads")
    trees, x, _ = W.fit_workload(24, 9000, seed=3, nvars=3)
    cols, y = _fixture(9000, seed=5)
    cols[1] = x[1]
    cols[2] = x[2]
    ev = _evaluator(pkg, cols, y)
    plans, prog, off, pcount, c0, kmax = _pack(pkg, trees)
    ntrials = 3
    rng = np.random.Generator(np.random.PCG64(11))
    c = np.repeat(c0[:, None, :], ntrials, axis=1)
    c[:, 1:, :] += rng.uniform(-0.5, 0.5, c[:, 1:, :].shape)
    sums, status, bb, _ = ev.rank_sums(prog, off, pcount, c.reshape(-1), kmax, ntrials)
    checked = 0
    for i, t in enumerate(trees):
        for k in range(ntrials):
            tk = plans[i].apply(t, c[i, k, : plans[i].nconst])
            pred = _oracle_pred(O, tk, cols)
            want = O.rank_sums(pred, y)
            s = i * ntrials + k
            if want is None:
                assert status[s] == 2
                continue
            if status[s] != 0:
                # the device's f64 libm may overflow where the CPU's does not;
                # never the other way round for these inputs
                assert not np.all(np.isfinite(pred)) or np.max(np.abs(pred)) > 1e300
                continue
            assert sums[s] == want[:2], (i, k)
            checked += 1
    assert checked >= 40
    ev.close()


def test_non_finite_predictions_are_flagged(pkg, E, O):
    cols, y = _fixture(5000)
    ev = _evaluator(pkg, cols, y)
    bad = E.node(E.LOG, [E.node(E.SUB, [E.input(1), E.constant(1.0)])])
    good = _models(E)["linear"]
    plans, prog, off, pcount, c0, kmax = _pack(pkg, [bad, good])
    sums, status, _, _ = ev.rank_sums(prog, off, pcount, c0, kmax)
    assert list(status) == [2, 0]
    assert sums[0] is None
    ev.close()


def test_order_statistics_match_the_oracle(pkg, E, O):
    for n in (3, 4, 7, 4096, 10007):
        cols, y = _fixture(n, seed=n, tied_y=False)
        ev = _evaluator(pkg, cols, y)
        trees = [_models(E)["linear"], _models(E)["tied"]]
        plans, prog, off, pcount, c0, kmax = _pack(pkg, trees)
        med, st0, _ = ev.order_stat(prog, off, pcount, c0, kmax, 0)
        iqm, st1, _ = ev.order_stat(prog, off, pcount, c0, kmax, 1)
        for k, t in enumerate(trees):
            pred = _oracle_pred(O, t, cols)
            assert st0[k] == 0 and st1[k] == 0
            # the models are exact in f64, so the median is bit-identical
            assert med[k] == O.score_pred(pred, y, O.MEDIAN), (n, k)
            want = O.score_pred(pred, y, O.INTERQUARTILE)
            assert abs(iqm[k] - want) <= 1e-14 * abs(want), (n, k, iqm[k], want)
        ev.close()


def test_max_scan_and_level_intervals(pkg, E, O):
    cols, y = _fixture(10007, seed=2, tied_y=False)
    ev = _evaluator(pkg, cols, y)
    lin = _models(E)["linear"]
    bad = E.node(E.LOG, [E.node(E.SUB, [E.input(1), E.constant(1.0)])])
    plans, prog, off, pcount, c0, kmax = _pack(pkg, [lin, bad])
    # coordinate 0 of the linear model at a level above its max error, one at
    # a level below (vetoed or a narrow interval), and the bad model
    pred = _oracle_pred(O, lin, cols)
    r = pred - y
    vmax = np.max(np.abs(r))
    row = int(np.flatnonzero(np.abs(r) == vmax)[0])
    out, _ = ev.max_scan(prog, off, pcount, c0, kmax)
    assert out[0][0] == vmax and out[0][1] == row and out[0][4] == 0
    assert out[1][4] == 2 and out[1][1] == -1
    # dr/dc for the slot that multiplies x1
    slot = None
    for j in range(plans[0].nconst):
        c = c0[0].copy()
        c[j] += 1.0
        d = _oracle_pred(O, plans[0].apply(lin, c[: plans[0].nconst]), cols) - pred
        if not np.allclose(d, 1.0):
            slot = j
            b = cols[1]
    assert slot is not None
    for level in (vmax * 1.5, vmax * 0.999):
        outs, _ = ev.max_scan(prog[: off[1]], off[:2], pcount[:1], c0[:1], kmax,
                              coords=np.array([slot]), levels=np.array([level]))
        o = outs[0]
        with np.errstate(divide="ignore"):
            e1 = (-level - r) / b
            e2 = (level - r) / b
        nz = b != 0.0
        if np.any(np.abs(r[~nz]) > level):
            assert o[2] == np.inf and o[3] == -np.inf
        else:
            assert o[2] == np.max(np.minimum(e1[nz], e2[nz]))
            assert o[3] == np.min(np.maximum(e1[nz], e2[nz]))
    ev.close()


def _bucket_models(E):
    """Keys of every shape the bucketed sums meet: distinct (linear), few
    values with many ties (integer x0), 2,001 values with ties (x1 rounded
    to 1/500, column 3), one value (flat), long groups sharing their upper
    bits (clustered, near-constant) and a heavy tail whose last buckets span
    many binades (exp)."""
    m = _models(E)
    clustered = E.node(E.ADD, [E.node(E.MUL, [E.constant(0.5), E.input(0)]),
                               E.node(E.MUL, [E.constant(1e-9), E.input(1)])])
    near = E.node(E.ADD, [E.constant(1.0), E.node(E.MUL, [E.constant(1e-12), E.input(2)])])
    step = E.node(E.MUL, [E.constant(1.5), E.input(3)])
    tail = E.node(E.EXP, [E.node(E.MUL, [E.constant(3.0), E.input(2)])])
    return [m["linear"], m["tied"], m["flat"], clustered, near, step, tail]


def _fixture4(n, seed):
    cols, y = _fixture(n, seed=seed)
    return np.concatenate([cols, np.round(cols[1:2] * 500.0) / 500.0]), y


def _check_sums(O, trees, cols, y, sums, status):
    for k, t in enumerate(trees):
        ab, aa, _ = O.rank_sums(_oracle_pred(O, t, cols), y)
        assert status[k] == 0
        assert sums[k] == (ab, aa), (k, sums[k], (ab, aa))


@pytest.mark.parametrize("n", [8192, 8193, 300007])
def test_bucketed_rank_sums_match_the_oracle(pkg, E, O, n):
    """One range bucket (8,192 rows), the smallest multi-bucket size and 147
    buckets: the sums equal the CPU's exactly, and no segment needs the
    radix sort."""
    cols, y = _fixture4(n, seed=n % 1000)
    ev = _evaluator(pkg, cols, y)
    trees = _bucket_models(E)
    plans, prog, off, pcount, c0, kmax = _pack(pkg, trees)
    sums, status, _, _ = ev.rank_sums(prog, off, pcount, c0, kmax)
    _check_sums(O, trees, cols, y, sums, status)
    assert ev.rank_fallbacks() == 0
    ev.close()


@pytest.mark.parametrize("cap,gmax", [(64, 0), (0, 1), (-1, 0)])
def test_rank_sums_on_the_radix_fallback(pkg, E, O, cap, gmax):
    """Buckets of 64 slots overflow (those segments go to the radix sort one
    at a time), a comparison bound of one sorts every bucket holding two
    distinct keys with one digit, and -1 turns the buckets off (the radix
    sort for all): the same sums each way."""
    n = 100003
    cols, y = _fixture4(n, seed=7)
    ev = _evaluator(pkg, cols, y)
    trees = _bucket_models(E)
    plans, prog, off, pcount, c0, kmax = _pack(pkg, trees)
    ev.rank_tuning(cap, gmax)
    sums, status, _, _ = ev.rank_sums(prog, off, pcount, c0, kmax)
    _check_sums(O, trees, cols, y, sums, status)
    fb = ev.rank_fallbacks()
    if cap < 0:
        assert fb == len(trees)
    elif cap > 0:
        assert 1 <= fb < len(trees)  # the flat model's one value never overflows
    else:
        assert fb == 0
    ev.rank_tuning(0, 0)
    sums2, _, _, _ = ev.rank_sums(prog, off, pcount, c0, kmax)
    assert sums2 == sums
    ev.close()


@pytest.mark.parametrize("n,bucketed", [(4194304, True), (4194305, False)])
def test_rank_sums_at_the_bucket_row_limit(pkg, E, n, bucketed):
    """4,194,304 rows is the largest segment the buckets take (2,048 range
    buckets, 16,384 samples); one row more goes to the radix sort for every
    segment. Either way the sums equal the radix sort's bit for bit."""
    cols, y = _fixture4(n, seed=3)
    ev = _evaluator(pkg, cols, y)
    trees = _bucket_models(E)
    plans, prog, off, pcount, c0, kmax = _pack(pkg, trees)
    sums, status, _, _ = ev.rank_sums(prog, off, pcount, c0, kmax)
    assert list(status) == [0] * len(trees)
    assert ev.rank_fallbacks() == (0 if bucketed else len(trees))
    ev.rank_tuning(-1, 0)
    sums_r, _, _, _ = ev.rank_sums(prog, off, pcount, c0, kmax)
    assert ev.rank_fallbacks() == len(trees)
    assert sums == sums_r
    ev.close()
