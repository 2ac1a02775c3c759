"""ctypes wrapper of the CPU f64 oracle (`oracle/oracle.cpp`).

TEST INFRASTRUCTURE ONLY: the checker for the device path and the timed CPU
baseline. Only `tests/`, `__graft_entry__.smoke()` and `bench.py`'s CPU-baseline
leg load it. Trees are passed as pre-order `(op, val)` arrays (any object with
a `prefix()` method works, e.g. the package's `expr.Node`).
"""
from __future__ import annotations

import ctypes
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "liboracle.so")

# Metric codes of the oracle (regression block equals the device score codes).
SQUARED, ABSOLUTE, LOG_SQUASHED, SIGNED, MAXIMUM = 0, 1, 2, 3, 4
CORRELATION, CORRELATION_SIGNED, AIC, AICC, BIC = 5, 6, 7, 8, 9
MEDIAN, INTERQUARTILE = 15, 16
LOG_LOSS, BRIER, HINGE_SIGMOID, HINGE_ORDINARY, HINGE_SQUARED = 10, 11, 12, 13, 14
RANK_CORRELATION, RANK_CORRELATION_SIGNED = 20, 21

_lib = None


def build() -> str:
    subprocess.run(["make", "-C", HERE, "-s"], check=True)
    return LIB_PATH


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH) or any(
                os.path.getmtime(LIB_PATH) < os.path.getmtime(os.path.join(HERE, f))
                for f in ("oracle.cpp", "variation.cpp")):
            build()
        L = ctypes.CDLL(LIB_PATH)
        P = ctypes.POINTER
        i32p, f64p, f32p, u64p, i64p = (P(ctypes.c_int32), P(ctypes.c_double), P(ctypes.c_float),
                                        P(ctypes.c_uint64), P(ctypes.c_int64))
        ci, cd = ctypes.c_int, ctypes.c_double
        u32, u32p = ctypes.c_uint32, P(ctypes.c_uint32)
        u8p, u16p = P(ctypes.c_uint8), P(ctypes.c_uint16)
        sig = {
            "or_tree_ok": (ci, [i32p, f64p, ci]),
            "or_predict": (ci, [i32p, f64p, ci, f64p, ci, ci, f64p]),
            "or_cpu_sse": (cd, [i32p, f64p, ci, f32p, ci, ci, f32p]),
            "or_score": (cd, [i32p, f64p, ci, f64p, ci, ci, f64p, f64p, ci]),
            "or_score_pred": (cd, [f64p, f64p, f64p, ci, ci, ci]),
            "or_fit": (cd, [i32p, f64p, ci, f64p, ci, ci, f64p, f64p, ci, ci]),
            "or_flat_sse": (cd, [i32p, f64p, ci, f64p, ci, ci, f64p, f64p]),
            "or_row_grad": (ci, [i32p, f64p, ci, f64p, ci, f64p, f64p, f64p]),
            "or_implicit_score": (cd, [i32p, f64p, ci, f64p, ci, ci, f64p]),
            "or_implicit_fit": (cd, [i32p, f64p, ci, f64p, ci, ci, f64p, ci]),
            "or_rank_sums": (ci, [f64p, f64p, ci, u64p]),
            "or_centred_ranks_doubled": (ci, [f64p, ci, i64p]),
            "or_erf": (cd, [cd]),
            "or_fit_lm_traced": (cd, [i32p, f64p, ci, f64p, ci, ci, f64p, f64p, ci, i32p]),
            "or_flat_constants": (ci, [i32p, f64p, ci, f64p]),
            "or_binary_labels": (ci, [f64p, f64p, ci, f64p]),
            "or_normal_equations_ok": (ci, [i32p, f64p, ci, f64p, ci, ci, f64p, f64p]),
            "or_verify_proposal": (ci, [i32p, f64p, ci, f64p, ci, ci, f64p, f64p, ci, f64p, ci,
                                        f64p]),
            "or_fit_verified": (cd, [i32p, f64p, ci, f64p, ci, ci, f64p, f64p, ci, ci, f64p, ci,
                                     i32p]),
            "orv_philox": (None, [u32, u32, u32, u32, u32, ci, u32p]),
            "orv_hash": (ctypes.c_uint64, [u32p, ci]),
            "orv_spans": (ci, [u32p, ci]),
            "orv_random_arena": (None, [ci, ci, ci, u32, ci, u32p, ci, u32, ci, ci, u32p]),
            "orv_next_generation": (ci, [ci, ci, ci, u32, ci, ci, u32p, ci, ci, ci, u32p, f64p,
                                         u32, u8p, u32p, u32p, ci, cd, u32p, u16p, u16p, u64p,
                                         f64p]),
            "or_erfc": (cd, [cd]),
        }
        for name, (res, args) in sig.items():
            fn = getattr(L, name)
            fn.restype = res
            fn.argtypes = args
        _lib = L
    return _lib


def _ptr(a, ct):
    if a is None:
        return None
    return a.ctypes.data_as(ctypes.POINTER(ct))


def _tree(t):
    ops, vals = t.prefix()
    return np.ascontiguousarray(ops, np.int32), np.ascontiguousarray(vals, np.float64)


def _cols(cols):
    c = np.ascontiguousarray(cols, np.float64)
    return c


def predict(t, cols, n, v):
    ops, vals = _tree(t)
    c = _cols(cols)
    out = np.empty(n, np.float64)
    rc = lib().or_predict(_ptr(ops, ctypes.c_int32), _ptr(vals, ctypes.c_double), len(ops),
                          _ptr(c, ctypes.c_double), n, v, _ptr(out, ctypes.c_double))
    assert rc == 0
    return out


def cpu_sse(t, cols32, n, v, y32):
    ops, vals = _tree(t)
    c = np.ascontiguousarray(cols32, np.float32)
    y = np.ascontiguousarray(y32, np.float32)
    return lib().or_cpu_sse(_ptr(ops, ctypes.c_int32), _ptr(vals, ctypes.c_double), len(ops),
                            _ptr(c, ctypes.c_float), n, v, _ptr(y, ctypes.c_float))


def score(t, cols, n, v, y, metric, w=None):
    ops, vals = _tree(t)
    c = _cols(cols)
    y = np.ascontiguousarray(y, np.float64)
    w = None if w is None else np.ascontiguousarray(w, np.float64)
    return lib().or_score(_ptr(ops, ctypes.c_int32), _ptr(vals, ctypes.c_double), len(ops),
                          _ptr(c, ctypes.c_double), n, v, _ptr(y, ctypes.c_double),
                          _ptr(w, ctypes.c_double), metric)


def score_pred(pred, y, metric, k=0, w=None):
    p = np.ascontiguousarray(pred, np.float64)
    y = np.ascontiguousarray(y, np.float64)
    w = None if w is None else np.ascontiguousarray(w, np.float64)
    return lib().or_score_pred(_ptr(p, ctypes.c_double), _ptr(y, ctypes.c_double),
                               _ptr(w, ctypes.c_double), len(p), metric, k)


def fit(t, cols, n, v, y, iters, metric=SQUARED, w=None):
    """fit::fit_weighted_metric; returns (objective, fitted tree)."""
    ops, vals = _tree(t)
    c = _cols(cols)
    y = np.ascontiguousarray(y, np.float64)
    w = None if w is None else np.ascontiguousarray(w, np.float64)
    r = lib().or_fit(_ptr(ops, ctypes.c_int32), _ptr(vals, ctypes.c_double), len(ops),
                     _ptr(c, ctypes.c_double), n, v, _ptr(y, ctypes.c_double),
                     _ptr(w, ctypes.c_double), iters, metric)
    out = t.clone()
    out.set_prefix_values(vals)
    return r, out


def fit_lm_traced(t, cols, n, v, y, iters, w=None):
    """fit::fit_lm with how its loop ended; returns (sse, fitted tree,
    (stop, improved, start_ok)), stop 0 = ran out of iterations / lambda /
    loss, 1 = a damped solve failed, 2 = the normal equations were not
    finite."""
    ops, vals = _tree(t)
    c = _cols(cols)
    y = np.ascontiguousarray(y, np.float64)
    w = None if w is None else np.ascontiguousarray(w, np.float64)
    lab = np.zeros(3, np.int32)
    r = lib().or_fit_lm_traced(_ptr(ops, ctypes.c_int32), _ptr(vals, ctypes.c_double), len(ops),
                               _ptr(c, ctypes.c_double), n, v, _ptr(y, ctypes.c_double),
                               _ptr(w, ctypes.c_double), iters, _ptr(lab, ctypes.c_int32))
    out = t.clone()
    out.set_prefix_values(vals)
    return r, out, tuple(int(q) for q in lab)


def binary_labels(y, w=None):
    """metrics::binary_labels(_weighted): l = [y > (min + max) / 2]."""
    y = np.ascontiguousarray(y, np.float64)
    w = None if w is None else np.ascontiguousarray(w, np.float64)
    out = np.zeros(len(y), np.float64)
    rc = lib().or_binary_labels(_ptr(y, ctypes.c_double), _ptr(w, ctypes.c_double), len(y),
                                _ptr(out, ctypes.c_double))
    return None if rc != 0 else out


def flat_constants(t):
    """The tree's constants in the flat evaluator's slot order."""
    ops, vals = _tree(t)
    out = np.zeros(max(len(ops), 1), np.float64)
    k = lib().or_flat_constants(_ptr(ops, ctypes.c_int32), _ptr(vals, ctypes.c_double), len(ops),
                                _ptr(out, ctypes.c_double))
    assert k >= 0
    return out[:k].copy()


def normal_equations_ok(t, cols, n, v, y, w=None):
    """Whether fit.rs `normal_equations` are finite at the tree's constants."""
    ops, vals = _tree(t)
    c = _cols(cols)
    y = np.ascontiguousarray(y, np.float64)
    w = None if w is None else np.ascontiguousarray(w, np.float64)
    return lib().or_normal_equations_ok(_ptr(ops, ctypes.c_int32), _ptr(vals, ctypes.c_double),
                                        len(ops), _ptr(c, ctypes.c_double), n, v,
                                        _ptr(y, ctypes.c_double), _ptr(w, ctypes.c_double)) == 1


def fit_verified(t, cols, n, v, y, iters, proposal, metric=SQUARED, w=None):
    """fit::gpu::fit_batch_verified for one tree: `proposal` (constants in
    flat slot order, or None when the device gave no usable answer) goes
    through verify_proposal; a rejected or missing one falls back on the CPU
    fit. Returns (score, tree, state) with state 0 = device answer accepted,
    1 = rejected, 2 = no proposal."""
    ops, vals = _tree(t)
    c = _cols(cols)
    y = np.ascontiguousarray(y, np.float64)
    w = None if w is None else np.ascontiguousarray(w, np.float64)
    if proposal is None:
        prop, npr = None, -1
    else:
        prop = np.ascontiguousarray(proposal, np.float64)
        npr = len(prop)
    st = np.zeros(1, np.int32)
    r = lib().or_fit_verified(_ptr(ops, ctypes.c_int32), _ptr(vals, ctypes.c_double), len(ops),
                              _ptr(c, ctypes.c_double), n, v, _ptr(y, ctypes.c_double),
                              _ptr(w, ctypes.c_double), iters, metric,
                              _ptr(prop, ctypes.c_double), npr, _ptr(st, ctypes.c_int32))
    out = t.clone()
    out.set_prefix_values(vals)
    return r, out, int(st[0])


def flat_sse(t, cols, n, v, y, w=None):
    ops, vals = _tree(t)
    c = _cols(cols)
    y = np.ascontiguousarray(y, np.float64)
    w = None if w is None else np.ascontiguousarray(w, np.float64)
    return lib().or_flat_sse(_ptr(ops, ctypes.c_int32), _ptr(vals, ctypes.c_double), len(ops),
                             _ptr(c, ctypes.c_double), n, v, _ptr(y, ctypes.c_double),
                             _ptr(w, ctypes.c_double))


def row_grad(t, row):
    """(value, d/dconstants, d/dinputs) of one row via backward_impl."""
    ops, vals = _tree(t)
    r = np.ascontiguousarray(row, np.float64)
    nconst = len(t.constants())
    val = ctypes.c_double(0.0)
    cg = np.zeros(max(nconst, 1), np.float64)
    ig = np.zeros(len(r), np.float64)
    k = lib().or_row_grad(_ptr(ops, ctypes.c_int32), _ptr(vals, ctypes.c_double), len(ops),
                          _ptr(r, ctypes.c_double), len(r), ctypes.byref(val),
                          _ptr(cg, ctypes.c_double), _ptr(ig, ctypes.c_double))
    assert k == nconst
    return val.value, cg[:nconst], ig


def implicit_score(t, cols, n, v, w=None):
    ops, vals = _tree(t)
    c = _cols(cols)
    w = None if w is None else np.ascontiguousarray(w, np.float64)
    return lib().or_implicit_score(_ptr(ops, ctypes.c_int32), _ptr(vals, ctypes.c_double),
                                   len(ops), _ptr(c, ctypes.c_double), n, v,
                                   _ptr(w, ctypes.c_double))


def implicit_fit(t, cols, n, v, iters, w=None):
    ops, vals = _tree(t)
    c = _cols(cols)
    w = None if w is None else np.ascontiguousarray(w, np.float64)
    r = lib().or_implicit_fit(_ptr(ops, ctypes.c_int32), _ptr(vals, ctypes.c_double), len(ops),
                              _ptr(c, ctypes.c_double), n, v, _ptr(w, ctypes.c_double), iters)
    out = t.clone()
    out.set_prefix_values(vals)
    return r, out


def _i128(hi, lo):
    v = (int(hi) << 64) | int(lo)
    if v >= 1 << 127:
        v -= 1 << 128
    return v


def rank_sums(pred, y):
    """(ab, aa, bb) as Python ints, or None when a value is not finite."""
    p = np.ascontiguousarray(pred, np.float64)
    yy = np.ascontiguousarray(y, np.float64)
    out = np.zeros(6, np.uint64)
    rc = lib().or_rank_sums(_ptr(p, ctypes.c_double), _ptr(yy, ctypes.c_double), len(p),
                            _ptr(out, ctypes.c_uint64))
    if rc != 0:
        return None
    return _i128(out[0], out[1]), _i128(out[2], out[3]), _i128(out[4], out[5])


def centred_ranks_doubled(v):
    a = np.ascontiguousarray(v, np.float64)
    out = np.zeros(len(a), np.int64)
    rc = lib().or_centred_ranks_doubled(_ptr(a, ctypes.c_double), len(a),
                                        _ptr(out, ctypes.c_int64))
    return None if rc != 0 else out


def erf(x):
    return lib().or_erf(float(x))


def erfc(x):
    return lib().or_erfc(float(x))


# ---- flat postfix variation (oracle/variation.cpp) --------------------------

def philox(seed, island, gen, slot, n=1, draw=0):
    """The first n Philox4x32-10 outputs at (seed, island, gen, slot, draw)."""
    out = np.zeros(4 * n, np.uint32)
    lib().orv_philox(seed, island, gen, slot, draw, n, _ptr(out, ctypes.c_uint32))
    return out.reshape(n, 4)


def postfix_hash(words):
    w = np.ascontiguousarray(words, np.uint32)
    return int(lib().orv_hash(_ptr(w, ctypes.c_uint32), len(w)))


def spans_count(words):
    """Node count of the strict postfix parse, or -1 when malformed."""
    w = np.ascontiguousarray(words, np.uint32)
    return int(lib().orv_spans(_ptr(w, ctypes.c_uint32), len(w)))


def _ops(ops):
    return np.ascontiguousarray(np.asarray(ops, np.uint32).reshape(-1, 2))


def random_arena(width, nvars, max_complexity, ops, rng_seed, depth, count):
    """Parents as the reference's tests draw them: consecutive random
    programs from the generator at (rng_seed, 0, 0, 0); [count, width]."""
    o = _ops(ops)
    out = np.zeros(count * width, np.uint32)
    lib().orv_random_arena(width, nvars, max_complexity, 0, 3, _ptr(o, ctypes.c_uint32), len(o),
                           rng_seed, depth, count, _ptr(out, ctypes.c_uint32))
    return out.reshape(count, width)


def next_generation(words, err, islands, pop, width, nvars, max_complexity, seed, gen, ops,
                    init_depth=3, dedup=True, restart=None, front=None, front_p=0.0):
    """Variation::next_generation_with_front on the CPU. Returns
    (words [islands*pop, width], len, cost, hash, err)."""
    o = _ops(ops)
    w = np.ascontiguousarray(words, np.uint32).reshape(-1)
    e = np.ascontiguousarray(err, np.float64)
    r = None if restart is None else np.ascontiguousarray(restart, np.uint8)
    fw, fo, nf = None, None, 0
    if front:
        fo = np.zeros(len(front) + 1, np.uint32)
        fo[1:] = np.cumsum([len(f) for f in front])
        fw = np.ascontiguousarray(np.concatenate([np.asarray(f, np.uint32) for f in front]))
        nf = len(front)
    n = islands * pop
    ow = np.zeros(n * width, np.uint32)
    ol = np.zeros(n, np.uint16)
    oc = np.zeros(n, np.uint16)
    oh = np.zeros(n, np.uint64)
    oe = np.zeros(n, np.float64)
    rc = lib().orv_next_generation(width, nvars, max_complexity, seed, init_depth, int(dedup),
                                   _ptr(o, ctypes.c_uint32), len(o), islands, pop,
                                   _ptr(w, ctypes.c_uint32), _ptr(e, ctypes.c_double), gen,
                                   _ptr(r, ctypes.c_uint8), _ptr(fw, ctypes.c_uint32),
                                   _ptr(fo, ctypes.c_uint32), nf, front_p,
                                   _ptr(ow, ctypes.c_uint32), _ptr(ol, ctypes.c_uint16),
                                   _ptr(oc, ctypes.c_uint16), _ptr(oh, ctypes.c_uint64),
                                   _ptr(oe, ctypes.c_double))
    assert rc == 0, "parents are not valid postfix programs"
    return ow.reshape(n, width), ol, oc, oh, oe
