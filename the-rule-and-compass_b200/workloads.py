"""Seeded synthetic workloads with the shapes of the benchmark configurations.

Every generator uses numpy's PCG64 with an explicit seed, so a workload is a
pure function of its arguments:

- `scoring_workload`: random expression trees (depth <= 6, ops
  {+,-,*,/,exp,log,sin,cos,sqrt,pow,neg}, 0-8 constants ~U(-3,3), postfix
  length 3-64 skewed short) over N rows x 5 features ~N(0,1),
  y = x0*x1 + sin(x2) + N(0, 0.05^2);
- `fit_workload`: candidates with 1-20 constants ~U(-2,2) and 5-60 nodes over
  N rows x 8 features ~U(-2,2),
  y = 1.7 exp(-0.5 x0^2) cos(2.3 x1) + 0.4 x2 + N(0, 0.02^2);
- `implicit_workload`: noisy unit circle (x, y) plus 2 distractors ~N(0,1);
- `heavy_tail_workload`: 6 N(0,1) + 4 Student-t(3) features,
  y = 0.8 x0/(1+x1^2) + log(1+|x3|) + 0.1 t3 noise.
"""
from __future__ import annotations

import numpy as np

from . import expr as E

SCORE_UNARY = [E.EXP, E.LOG, E.SIN, E.COS, E.SQRT, E.NEG]
SCORE_BINARY = [E.ADD, E.SUB, E.MUL, E.DIV, E.POW]
FIT_UNARY = [E.SIN, E.COS, E.EXP, E.TANH, E.SIG, E.SQUARE, E.GAUSS, E.NEG]
FIT_BINARY = [E.ADD, E.SUB, E.MUL, E.DIV]


def _grow(rng, size, depth, max_depth, nvars, unary, binary, leaf):
    """A tree of about `size` nodes; `leaf()` makes a terminal."""
    if size <= 1 or depth >= max_depth:
        return leaf()
    if size == 2 or (rng.random() < 0.3 and size < 6):
        return E.node(int(rng.choice(unary)), [_grow(rng, size - 1, depth + 1, max_depth, nvars,
                                                     unary, binary, leaf)])
    left = int(rng.integers(1, size - 1))
    right = size - 1 - left
    return E.node(int(rng.choice(binary)), [
        _grow(rng, left, depth + 1, max_depth, nvars, unary, binary, leaf),
        _grow(rng, max(right, 1), depth + 1, max_depth, nvars, unary, binary, leaf)])


def random_scoring_tree(rng, nvars=5, max_depth=6):
    # postfix op count 3..64, geometric-skewed towards short (mean ~12)
    size = int(min(64, 3 + rng.geometric(1.0 / 9.0)))
    budget = [int(rng.integers(0, 9))]

    def leaf():
        if budget[0] > 0 and rng.random() < 0.35:
            budget[0] -= 1
            return E.constant(float(rng.uniform(-3.0, 3.0)))
        return E.input(int(rng.integers(0, nvars)))
    return _grow(rng, size, 0, max_depth, nvars, SCORE_UNARY, SCORE_BINARY, leaf)


def scoring_data(n, seed=0, nvars=5):
    rng = np.random.Generator(np.random.PCG64(seed))
    x = rng.standard_normal((nvars, n)).astype(np.float32)
    noise = rng.normal(0.0, 0.05, n)
    y = (x[0].astype(np.float64) * x[1] + np.sin(x[2].astype(np.float64)) + noise)
    return x, y.astype(np.float32)


def scoring_workload(P, n, seed=0, nvars=5):
    """(trees, cols f32 [V][N], y f32 [N])."""
    rng = np.random.Generator(np.random.PCG64(seed + 1000))
    trees = [random_scoring_tree(rng, nvars) for _ in range(P)]
    x, y = scoring_data(n, seed, nvars)
    return trees, x, y


def _fit_tree(rng, nconst, nodes, nvars):
    """A tree with exactly `nconst` constants (leaves) and about `nodes` nodes."""
    min_nodes = 2 * nconst + 1
    nodes = max(nodes, min_nodes)
    leaves = (nodes + 1) // 2
    kinds = [True] * nconst + [False] * max(leaves - nconst, 1)
    rng.shuffle(kinds)
    it = iter(kinds)

    def leaf():
        try:
            k = next(it)
        except StopIteration:
            k = False
        if k:
            return E.constant(float(rng.uniform(-2.0, 2.0)))
        return E.input(int(rng.integers(0, nvars)))

    t = _grow(rng, nodes, 0, 12, nvars, FIT_UNARY, FIT_BINARY, leaf)
    # top up constants that the depth limit cut off: c * t + c ...
    have = len(t.constants())
    while have < nconst:
        t = E.node(E.ADD, [E.node(E.MUL, [E.constant(float(rng.uniform(-2, 2))), t]),
                           E.constant(float(rng.uniform(-2, 2)))]) if nconst - have >= 2 else \
            E.node(E.MUL, [E.constant(float(rng.uniform(-2, 2))), t])
        have = len(t.constants())
    return t


def fit_data(n, seed=0, nvars=8):
    rng = np.random.Generator(np.random.PCG64(seed))
    x = rng.uniform(-2.0, 2.0, (nvars, n))
    y = 1.7 * np.exp(-0.5 * x[0] ** 2) * np.cos(2.3 * x[1]) + 0.4 * x[2] + \
        rng.normal(0.0, 0.02, n)
    return x, y


def fit_workload(P, n, seed=0, nvars=8, max_const=20):
    """(trees, cols64 [V][N], y64 [N]); constants per candidate uniform in
    1..max_const, node counts 5..60."""
    rng = np.random.Generator(np.random.PCG64(seed + 2000))
    trees = []
    for _ in range(P):
        k = int(rng.integers(1, max_const + 1))
        nodes = int(rng.integers(max(5, 2 * k + 1), 61))
        trees.append(_fit_tree(rng, k, nodes, nvars))
    x, y = fit_data(n, seed, nvars)
    return trees, x, y


def implicit_data(n, seed=0):
    rng = np.random.Generator(np.random.PCG64(seed))
    th = rng.uniform(0.0, 2 * np.pi, n)
    r = 1.0 + rng.normal(0.0, 0.01, n)
    cols = np.stack([r * np.cos(th), r * np.sin(th), rng.standard_normal(n),
                     rng.standard_normal(n)])
    return cols


def implicit_workload(P, n, seed=0):
    """Candidates of f(x, y, d1, d2): length 3-40, 0-6 constants. Returns
    (trees, cols64 [4][N]). The first candidates include the circle
    x^2 + y^2 - c."""
    rng = np.random.Generator(np.random.PCG64(seed + 3000))
    trees = [E.node(E.SUB, [E.node(E.ADD, [E.node(E.SQUARE, [E.input(0)]),
                                           E.node(E.SQUARE, [E.input(1)])]),
                            E.constant(1.5)])]
    while len(trees) < P:
        k = int(rng.integers(0, 7))
        nodes = int(rng.integers(max(3, 2 * k + 1), 41))
        if k == 0:
            budget = [0]

            def leaf():
                return E.input(int(rng.integers(0, 4)))
            trees.append(_grow(rng, nodes, 0, 10, 4, FIT_UNARY, FIT_BINARY, leaf))
            del budget
        else:
            trees.append(_fit_tree(rng, k, nodes, 4))
    return trees[:P], implicit_data(n, seed)


def heavy_tail_data(n, seed=0):
    rng = np.random.Generator(np.random.PCG64(seed))
    g = rng.standard_normal((6, n))
    t = rng.standard_t(3.0, (4, n))
    x = np.concatenate([g, t])
    y = 0.8 * x[0] / (1.0 + x[1] ** 2) + np.log1p(np.abs(x[3])) + 0.1 * rng.standard_t(3.0, n)
    return x, y


def line_workload(n=10000, seed=0, test_frac=0.2):
    """The plain-method configuration: one feature x ~ U(-5, 5),
    y = 2x + 1 + N(0, 0.1^2), split into training and test rows by a seeded
    permutation (the last `test_frac` of it held out). Returns
    (x_train [1][n_train] f64, y_train, x_test [1][n_test], y_test)."""
    rng = np.random.Generator(np.random.PCG64(seed))
    x = rng.uniform(-5.0, 5.0, n)
    y = 2.0 * x + 1.0 + rng.normal(0.0, 0.1, n)
    perm = rng.permutation(n)
    n_test = int(round(n * test_frac))
    tr, te = perm[: n - n_test], perm[n - n_test:]
    return x[tr][None, :], y[tr], x[te][None, :], y[te]
