"""The fit plan of a postfix program built straight from its words
(`gpu_fit_plan_words`, the generation loop's path) must equal the plan of
the tree the words decode to (`gpu_fit_plan(from_postfix(words))`, the
reference's fit.rs:985-1056 through the tree), rejection labels included,
and a program that is not one expression must be "malformed" on both."""
import importlib

import numpy as np
import pytest


def _both(pkg, E, words):
    H = pkg.host
    try:
        t = E.from_postfix(words)
    except ValueError:
        t = None
    try:
        got = H.gpu_fit_plan_words(words)
    except H.GpuFitReject as e:
        got = e.label
    if t is None:
        want = "malformed"
    else:
        try:
            want = H.gpu_fit_plan(t)
        except H.GpuFitReject as e:
            want = e.label
    return got, want


def _same(got, want):
    if isinstance(want, str) or isinstance(got, str):
        return got == want
    return (np.array_equal(got.words, want.words) and got.nconst == want.nconst
            and np.array_equal(got.c0.view(np.uint64), want.c0.view(np.uint64))
            and np.array_equal(got.gauge, want.gauge))


def _padded(words, width=64):
    w = np.full(max(width, len(words)), 255, np.uint32)
    w[: len(words)] = words
    return w


def test_plans_of_compiled_trees_match_the_tree_path(pkg, E):
    W = importlib.import_module("the-rule-and-compass_b200.workloads")
    trees, _, _ = W.fit_workload(120, 16, seed=5, nvars=3)
    rng = np.random.Generator(np.random.PCG64(9))
    trees += [W.random_scoring_tree(rng, 3) for _ in range(120)]
    labels = set()
    for t in trees:
        words, _ = pkg.compile_program(t)
        got, want = _both(pkg, E, _padded(words))
        assert _same(got, want), (got, want)
        labels.add(got if isinstance(got, str) else "ok")
    assert "ok" in labels and "no_constants" in labels


def test_rejections_and_malformed_programs(pkg, E):
    c = int(np.float32(1.5).view(np.uint32))
    cases = [
        [E.CONST, c, E.VAR, 0, E.IF, 255],                  # too few operands
        [E.CONST, c, E.VAR, 0, 255],                        # two values left
        [E.CONST, c, E.VAR, 0, E.ADD],                      # no HALT
        [E.CONST],                                          # truncated operand
        [E.CONST, c, 200, 255],                             # unknown operator
        [E.VAR, 0, E.VAR, 1, E.ADD, 255],                   # no constants
        [E.CONST, c, E.VAR, 0, E.ADD, E.STEP, 255],         # unsupported operator
        [255],                                              # empty program
    ]
    many = []
    for _ in range(21):
        many += [E.CONST, c]
    many += [E.ADD] * 20 + [255]
    cases.append(many)                                      # too many constants
    seen = set()
    for words in cases:
        got, want = _both(pkg, E, np.asarray(words, np.uint32))
        assert _same(got, want), (words, got, want)
        seen.add(got if isinstance(got, str) else "ok")
    assert {"malformed", "no_constants", "too_many_constants"} <= seen


@pytest.mark.parametrize("seed", [0, 1, 2])
def test_random_word_soup(pkg, E, seed):
    """Arbitrary word sequences over the opcodes, operands and HALT."""
    rng = np.random.Generator(np.random.PCG64(seed))
    alphabet = np.array([E.CONST, E.VAR, E.ADD, E.MUL, E.SIN, E.EXP, E.IF, E.NEG, 255, 0, 1,
                         int(np.float32(0.5).view(np.uint32))], np.uint32)
    for _ in range(400):
        words = rng.choice(alphabet, size=int(rng.integers(1, 24)))
        got, want = _both(pkg, E, words)
        assert _same(got, want), (list(words), got, want)


def test_batched_plans_match_one_at_a_time(pkg, E):
    H = pkg.host
    W = importlib.import_module("the-rule-and-compass_b200.workloads")
    trees, _, _ = W.fit_workload(60, 16, seed=8, nvars=3)
    rows = [_padded(pkg.compile_program(t)[0][:63].tolist() + [255]) for t in trees]
    rows.append(_padded([E.CONST]))                     # malformed
    rows.append(_padded([E.VAR, 0, 255]))               # no constants
    batch = H.gpu_fit_plans_words(np.stack(rows))
    assert len(batch) == len(rows)
    for w, b in zip(rows, batch):
        try:
            one = H.gpu_fit_plan_words(w)
        except H.GpuFitReject as e:
            one = e.label
        assert _same(b, one), (b, one)
    assert H.gpu_fit_plans_words(np.zeros((0, 64), np.uint32)) == []


def test_constants_written_into_words_match_the_compiled_fitted_tree(pkg, E):
    """The generation loop writes a fit's constants straight into the pool
    words; compiling the fitted tree and storing it in the slot (the tree
    path) must give the same words, HALT padding included."""
    H = pkg.host
    W = importlib.import_module("the-rule-and-compass_b200.workloads")
    trees, _, _ = W.fit_workload(150, 16, seed=11, nvars=3)
    rng = np.random.Generator(np.random.PCG64(4))
    width = 64
    rows, want, cs, ks = [], [], [], []
    for t in trees:
        words, _ = pkg.compile_program(t)
        if len(words) > width:
            continue
        slot = np.full(width, 255, np.uint32)
        slot[: len(words)] = words
        slot[len(words):] = rng.integers(0, 300, width - len(words))  # junk after HALT
        try:
            plan = H.gpu_fit_plan(E.from_postfix(slot))
        except H.GpuFitReject:
            continue
        c = rng.normal(0.0, 3.0, plan.nconst) * 10.0 ** rng.integers(-8, 8, plan.nconst)
        w2, _ = pkg.compile_program(plan.apply(E.from_postfix(slot), c))
        ref = np.full(width, 255, np.uint32)
        ref[: len(w2)] = w2
        rows.append(slot)
        want.append(ref)
        cs.append(np.pad(c, (0, 20 - len(c))))
        ks.append(plan.nconst)
    assert len(rows) > 50
    pool = np.ascontiguousarray(np.stack(rows))
    st = H.set_postfix_constants(pool, np.arange(len(rows)), np.stack(cs), ks)
    assert np.all(st >= np.asarray(ks))
    assert np.array_equal(pool, np.stack(want))
    # a malformed row and one with too few constants are left as they were
    bad = np.ascontiguousarray(np.stack([np.full(width, E.ADD, np.uint32), rows[0].copy()]))
    keep = bad.copy()
    st = H.set_postfix_constants(bad, [0, 1], np.zeros((2, 25)), [0, 25])
    assert list(st) == [-4, -3]
    assert np.array_equal(bad, keep)
