"""Tree -> device program, through the C++ host compiler (`librcsr_host.so`).

Mirrors the reference's host API for this path:
`compile_program` (my-version/src/gpu.rs:198-219), `Population`
(my-version/src/gpu.rs:972-1068, the packed `prog` + `off[P+1]` batch) and
`gpu_fit_plan_reason` / `GpuFitPlan` (my-version/src/fit.rs:929-1056).
"""
from __future__ import annotations

import ctypes
import os

import numpy as np

from . import expr as E

_HERE = os.path.dirname(os.path.abspath(__file__))
HOST_LIB = os.path.join(_HERE, "librcsr_host.so")
_lib = None

HOST_MAX_STACK = 56
GPU_FIT_MAX_CONSTANTS = 20
GPU_FIT_MAX_NODES = 96


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(HOST_LIB):
            raise ImportError(f"{HOST_LIB} is not built: run the package's build.py")
        L = ctypes.CDLL(HOST_LIB)
        P = ctypes.POINTER
        L.rch_compile_program.restype = ctypes.c_int
        L.rch_compile_program.argtypes = [P(ctypes.c_int32), P(ctypes.c_double), ctypes.c_int,
                                          P(ctypes.c_uint32), ctypes.c_int, P(ctypes.c_int)]
        L.rch_peak_stack.restype = ctypes.c_int
        L.rch_peak_stack.argtypes = [P(ctypes.c_int32), P(ctypes.c_double), ctypes.c_int]
        L.rch_fit_plan.restype = ctypes.c_int
        L.rch_fit_plan.argtypes = [P(ctypes.c_int32), P(ctypes.c_double), ctypes.c_int,
                                   P(ctypes.c_uint32), ctypes.c_int, P(ctypes.c_double),
                                   ctypes.c_int, P(ctypes.c_int32), P(ctypes.c_int),
                                   ctypes.c_int]
        L.rch_fit_plan_postfix.restype = ctypes.c_int
        L.rch_fit_plan_postfix.argtypes = [P(ctypes.c_uint32), ctypes.c_int, P(ctypes.c_uint32),
                                           ctypes.c_int, P(ctypes.c_double), ctypes.c_int,
                                           P(ctypes.c_int32), P(ctypes.c_int), ctypes.c_int]
        L.rch_fit_plans_postfix.restype = ctypes.c_int
        L.rch_fit_plans_postfix.argtypes = [ctypes.c_int, P(ctypes.c_uint32), ctypes.c_int,
                                            P(ctypes.c_uint32), P(ctypes.c_double),
                                            P(ctypes.c_int32), P(ctypes.c_int32),
                                            P(ctypes.c_int32), ctypes.c_int]
        L.rch_set_postfix_constants_rows.restype = ctypes.c_int
        L.rch_set_postfix_constants_rows.argtypes = [ctypes.c_int, P(ctypes.c_uint32),
                                                     ctypes.c_int, P(ctypes.c_int32),
                                                     P(ctypes.c_double), ctypes.c_int,
                                                     P(ctypes.c_int32), P(ctypes.c_int32)]
        L.rch_admission_count.restype = ctypes.c_int
        L.rch_admission_count.argtypes = [ctypes.c_int, ctypes.c_longlong]
        L.rch_select_promoted.restype = ctypes.c_int
        L.rch_select_promoted.argtypes = [ctypes.c_int, P(ctypes.c_int32), ctypes.c_int,
                                          P(ctypes.c_int32), P(ctypes.c_int32),
                                          P(ctypes.c_double), P(ctypes.c_double),
                                          P(ctypes.c_uint8), ctypes.c_longlong,
                                          P(ctypes.c_int32), P(ctypes.c_int32), ctypes.c_int]
        L.rch_refit_finalists.restype = ctypes.c_int
        L.rch_refit_finalists.argtypes = [P(ctypes.c_int32), P(ctypes.c_double), P(ctypes.c_int32),
                                          ctypes.c_int, P(ctypes.c_double), ctypes.c_int64,
                                          ctypes.c_int, P(ctypes.c_double), P(ctypes.c_double),
                                          ctypes.c_int, ctypes.c_int, ctypes.c_int,
                                          P(ctypes.c_double)]
        L.rch_soa_eval.restype = ctypes.c_int
        L.rch_soa_eval.argtypes = [P(ctypes.c_int32), P(ctypes.c_double), ctypes.c_int,
                                   P(ctypes.c_double), ctypes.c_int64, ctypes.c_int,
                                   P(ctypes.c_double)]
        L.rch_soa_sse.restype = ctypes.c_double
        L.rch_soa_sse.argtypes = [P(ctypes.c_int32), P(ctypes.c_double), ctypes.c_int,
                                  P(ctypes.c_double), ctypes.c_int64, ctypes.c_int,
                                  P(ctypes.c_double)]
        _lib = L
    return _lib


def _p(a, ct):
    return a.ctypes.data_as(ctypes.POINTER(ct))


class CompileError(Exception):
    """Why a tree cannot run on the scoring kernel (gpu.rs:131-158)."""


def compile_program(tree: E.Node):
    """Postfix words (HALT-terminated) and whether `lower` rewrote the tree."""
    ops, vals = tree.prefix()
    cap = 4 * len(ops) * 16 + 64
    words = np.zeros(cap, np.uint32)
    lowered = ctypes.c_int(0)
    n = lib().rch_compile_program(_p(ops, ctypes.c_int32), _p(vals, ctypes.c_double), len(ops),
                                  _p(words, ctypes.c_uint32), cap, ctypes.byref(lowered))
    if n == -1:
        raise CompileError("unsupported operator")
    if n == -2:
        raise CompileError(f"postfix program needs more than {HOST_MAX_STACK} stack slots")
    if n < 0:
        raise CompileError(f"malformed tree ({n})")
    return words[:n].copy(), bool(lowered.value)


def peak_stack(tree: E.Node) -> int:
    ops, vals = tree.prefix()
    return lib().rch_peak_stack(_p(ops, ctypes.c_int32), _p(vals, ctypes.c_double), len(ops))


class Population:
    """Packed postfix batch `(prog, off)`; unsupported trees are counted and
    skipped (gpu.rs:972-1068)."""

    def __init__(self, trees=()):
        self._words = []
        self.offsets = [0]
        self.unsupported = 0
        self.lowered = 0
        self.index = []
        for i, t in enumerate(trees):
            if self.add(t):
                self.index.append(i)

    def add(self, tree) -> bool:
        try:
            w, low = compile_program(tree)
        except CompileError:
            self.unsupported += 1
            return False
        self._words.append(w)
        self.offsets.append(self.offsets[-1] + len(w))
        self.lowered += int(low)
        return True

    def __len__(self):
        return len(self.offsets) - 1

    def programs(self):
        prog = np.concatenate(self._words).astype(np.uint32) if self._words else \
            np.zeros(0, np.uint32)
        return prog, np.asarray(self.offsets, np.uint32)


REJECT = {-1: "too_many_constants", -2: "too_many_nodes", -3: "no_constants",
          -5: "unsupported_op", -4: "malformed", -6: "capacity"}


class GpuFitPlan:
    """One candidate flattened for the fit kernel (fit.rs:929-950)."""

    def __init__(self, words, c0, gauge, nconst):
        self.words = words
        self.c0 = c0
        self.gauge = gauge
        self.nconst = nconst

    @property
    def nodes(self):
        return len(self.words) // 4

    def apply(self, tree: E.Node, c) -> E.Node:
        """Write fitted constants back into a copy of `tree` (slot order is the
        tree's pre-order constant order)."""
        t = tree.clone()
        t.set_constants(list(c)[: self.nconst])
        return t


class GpuFitReject(Exception):
    def __init__(self, code):
        super().__init__(REJECT.get(code, str(code)))
        self.label = REJECT.get(code, str(code))


def gpu_fit_plan(tree: E.Node, allow_no_constants=False) -> GpuFitPlan:
    ops, vals = tree.prefix()
    cap = 4 * max(len(ops), 1)
    words = np.zeros(cap, np.uint32)
    c0 = np.zeros(max(len(ops), 1), np.float64)
    gauge = np.full(2, -1, np.int32)
    nconst = ctypes.c_int(0)
    m = lib().rch_fit_plan(_p(ops, ctypes.c_int32), _p(vals, ctypes.c_double), len(ops),
                           _p(words, ctypes.c_uint32), cap, _p(c0, ctypes.c_double), len(c0),
                           _p(gauge, ctypes.c_int32), ctypes.byref(nconst),
                           1 if allow_no_constants else 0)
    if m < 0:
        raise GpuFitReject(m)
    k = nconst.value
    return GpuFitPlan(words[: 4 * m].copy(), c0[:k].copy(), gauge.copy(), k)


def gpu_fit_plan_words(words, allow_no_constants=False) -> GpuFitPlan:
    """gpu_fit_plan of a postfix program (its words up to HALT, as the pool
    holds them) without building the tree: the same plan, the same
    rejections, and "malformed" for a program that is not one expression."""
    w = np.ascontiguousarray(words, np.uint32).reshape(-1)
    cap = 4 * max(len(w), 1)
    out = np.zeros(cap, np.uint32)
    c0 = np.zeros(max(len(w), 1), np.float64)
    gauge = np.full(2, -1, np.int32)
    nconst = ctypes.c_int(0)
    m = lib().rch_fit_plan_postfix(_p(w, ctypes.c_uint32), len(w), _p(out, ctypes.c_uint32), cap,
                                   _p(c0, ctypes.c_double), len(c0), _p(gauge, ctypes.c_int32),
                                   ctypes.byref(nconst), 1 if allow_no_constants else 0)
    if m < 0:
        raise GpuFitReject(m)
    k = nconst.value
    return GpuFitPlan(out[: 4 * m].copy(), c0[:k].copy(), gauge.copy(), k)


def gpu_fit_plans_words(words, allow_no_constants=False):
    """gpu_fit_plan_words of every row of a [programs, width] word array in
    one native call: a list with, per row, its GpuFitPlan or the rejection
    label."""
    w = np.ascontiguousarray(words, np.uint32)
    n, width = w.shape
    if n == 0:
        return []
    out = np.zeros((n, 4 * width), np.uint32)
    c0 = np.zeros((n, width), np.float64)
    gauge = np.full((n, 2), -1, np.int32)
    nconst = np.zeros(n, np.int32)
    status = np.zeros(n, np.int32)
    if lib().rch_fit_plans_postfix(n, _p(w, ctypes.c_uint32), width, _p(out, ctypes.c_uint32),
                                   _p(c0, ctypes.c_double), _p(gauge, ctypes.c_int32),
                                   _p(nconst, ctypes.c_int32), _p(status, ctypes.c_int32),
                                   1 if allow_no_constants else 0) < 0:
        raise RuntimeError("rch_fit_plans_postfix failed")
    res = []
    for i in range(n):
        m = int(status[i])
        if m < 0:
            res.append(REJECT.get(m, str(m)))
        else:
            k = int(nconst[i])
            res.append(GpuFitPlan(out[i, : 4 * m].copy(), c0[i, :k].copy(), gauge[i].copy(), k))
    return res


def set_postfix_constants(words, rows, c, k):
    """Write fitted constants into pool programs in place: row rows[r] of the
    [programs, width] uint32 array `words` gets c[r, :k[r]] (f32-rounded) in
    its constant operands, in the tree's pre-order slot order, and HALT after
    its end, as compile_program of the fitted tree would emit it. Returns
    each row's status (its constant count, or -4 malformed, -2 stack beyond
    the host limit, -3 fewer constants than k: that row is left as it was)."""
    assert words.dtype == np.uint32 and words.flags.c_contiguous
    rows = np.ascontiguousarray(rows, np.int32)
    n = len(rows)
    c = np.ascontiguousarray(c, np.float64).reshape(n, -1) if n else np.zeros((0, 1))
    k = np.ascontiguousarray(k, np.int32)
    status = np.zeros(n, np.int32)
    if n == 0:
        return status
    if lib().rch_set_postfix_constants_rows(n, _p(words, ctypes.c_uint32), words.shape[1],
                                            _p(rows, ctypes.c_int32), _p(c, ctypes.c_double),
                                            c.shape[1], _p(k, ctypes.c_int32),
                                            _p(status, ctypes.c_int32)) < 0:
        raise RuntimeError("rch_set_postfix_constants_rows failed")
    return status


def pack_plans(plans, kmax=None):
    """Concatenate fit plans into the rc_fit_batch inputs:
    (prog, off, pcount, c0[P*kmax], gauge[2P], kmax)."""
    if kmax is None:
        kmax = max([p.nconst for p in plans] + [1])
    prog = np.concatenate([p.words for p in plans]).astype(np.uint32)
    off = np.zeros(len(plans) + 1, np.uint32)
    off[1:] = np.cumsum([len(p.words) for p in plans])
    pcount = np.asarray([p.nconst for p in plans], np.int32)
    c0 = np.zeros((len(plans), kmax), np.float64)
    for i, p in enumerate(plans):
        c0[i, : p.nconst] = p.c0
    gauge = np.concatenate([p.gauge for p in plans]).astype(np.int32)
    return prog, off, pcount, c0, gauge, kmax


def admission_count(island_pop, train_rows):
    """Offspring of one island admitted to the fitted batch
    (my-version/src/search.rs:3006-3031)."""
    return lib().rch_admission_count(int(island_pop), int(train_rows))


def select_promoted(island_pop, pending, error, complexity, has_constants, train_rows):
    """The (island, index) pairs promoted to the fitted batch
    (my-version/src/search.rs:3033-3074). `pending` is a list of (island,
    index); `error`, `complexity` and `has_constants` are aligned with it."""
    isl = np.asarray([p[0] for p in pending], np.int32)
    idx = np.asarray([p[1] for p in pending], np.int32)
    pops = np.asarray(island_pop, np.int32)
    err = np.ascontiguousarray(error, np.float64)
    cx = np.ascontiguousarray(complexity, np.float64)
    hc = np.ascontiguousarray(has_constants, np.uint8)
    oi = np.zeros(max(len(pending), 1), np.int32)
    oj = np.zeros(max(len(pending), 1), np.int32)
    k = lib().rch_select_promoted(len(pops), _p(pops, ctypes.c_int32), len(pending),
                                  _p(isl, ctypes.c_int32), _p(idx, ctypes.c_int32),
                                  _p(err, ctypes.c_double), _p(cx, ctypes.c_double),
                                  _p(hc, ctypes.c_uint8), int(train_rows),
                                  _p(oi, ctypes.c_int32), _p(oj, ctypes.c_int32), len(oi))
    if k < 0:
        raise RuntimeError("rch_select_promoted failed")
    return list(zip(oi[:k].tolist(), oj[:k].tolist()))


# Op::default_set() (my-version/src/expr.rs:392-398) through postfix_opcode
# (my-version/src/gpu.rs:447-494): the variation engine's (opcode, arity)
# table, in table order.
DEFAULT_VARIATION_OPS = ((17, 1), (9, 1), (10, 1), (12, 1), (11, 1), (6, 1), (7, 1), (8, 1),
                         (21, 1), (22, 1), (13, 1), (14, 1), (18, 1), (15, 1), (16, 1),
                         (2, 2), (3, 2), (4, 2), (5, 2), (20, 2), (32, 3))


def width_for(max_complexity):
    """Fixed slot width for a maximum complexity (genome.rs:35-37)."""
    return max(2 * max_complexity + 4, 8)


# ---- the run-level fit ledger ------------------------------------------------

# Labels of the finite device answers (my-version/src/search.rs:2939-2948).
STATUS_LABELS = {4: "rank_deficient", 5: "recovered", 6: "no_improvement", 7: "start_unusable",
                 8: "recovered_skipped"}


def fit_status_usable(status):
    """Statuses that carry a finite answer the search may keep
    (my-version/src/fit/gpu.rs:103-105)."""
    return int(status) in (0, 4, 5, 6, 7, 8)


def status_fallback_cause(status):
    """The CPU-fallback cause of a device status (search.rs:2952-2959)."""
    return {1: "ill_conditioned", 2: "non_finite", 3: "rank_declined"}.get(int(status),
                                                                         "unsupported_plan")


def _jnum(v):
    """A number as the reference's ledger prints it (Rust's shortest
    round-trip decimal, no exponent; null when not finite)."""
    v = float(v)
    if not np.isfinite(v):
        return "null"
    return np.format_float_positional(v, unique=True, trim="-")


def _jmap(d):
    return ",".join('"%s":%d' % (k, d[k]) for k in sorted(d))


class FitLedger:
    """The `gpu.fit` run-record of the reference's `--json` output
    (my-version/src/main.rs:995-1010) and its accounting
    (search.rs:2040-2120): candidates screened, offered to the fit arm,
    answered on the device, sent to the exact CPU arm by cause, device
    answers by status label, finalist refits, and the fit stage's times."""

    def __init__(self, strategy="gpu"):
        self.strategy = strategy
        self.screened = self.attempts = self.gpu = self.fallback = self.refits = 0
        self.fallback_by_cause = {}
        self.status_by_label = {}
        self.seconds = self.host_seconds = self.fallback_seconds = 0.0
        self.fallback_bounded = self.fallback_workers = self.fallback_max = 0

    def note_fallback(self, cause):
        self.fallback += 1
        self.fallback_by_cause[cause] = self.fallback_by_cause.get(cause, 0) + 1

    def record_batch(self, trees, constants, status, ms):
        """One fit batch of `trees` with the device's `constants` [P][kmax],
        `status` [P] and kernel `ms` (negative: the launch failed). A tree
        without constants is not offered; a tree the plan rejects falls back
        as `too_many_constants` or `unsupported_plan`; a planned tree is a
        device answer when its status is usable and its constants finite,
        else a fallback by its status (`non_finite` for a non-finite
        constant). Trees that were planned are in `constants` order."""
        planned = []
        for t in trees:
            try:
                gpu_fit_plan(t)
                planned.append(t)
                self.attempts += 1
            except GpuFitReject as r:
                if r.label == "no_constants":
                    continue
                self.attempts += 1
                self.note_fallback("too_many_constants" if r.label == "too_many_constants"
                                   else "unsupported_plan")
        if ms < 0:
            for _ in planned:
                self.note_fallback("launch")
            return
        self.seconds += ms / 1e3
        for k in range(len(planned)):
            s = int(status[k])
            finite = bool(np.all(np.isfinite(constants[k])))
            if fit_status_usable(s) and finite:
                self.gpu += 1
                if s in STATUS_LABELS:
                    lab = STATUS_LABELS[s]
                    self.status_by_label[lab] = self.status_by_label.get(lab, 0) + 1
            else:
                self.note_fallback("non_finite" if not finite else status_fallback_cause(s))

    def to_json(self):
        return ('"fit":{"strategy":"%s","screened":%d,"attempts":%d,"gpu":%d,"fallback":%d,'
                '"fallback_by_cause":{%s},"status_by_label":{%s},"refits":%d,"seconds":%s,'
                '"host_seconds":%s,"fallback_seconds":%s,"fallback_bounded":%d,'
                '"fallback_workers":%d,"fallback_max":%d}' % (
                    self.strategy, self.screened, self.attempts, self.gpu, self.fallback,
                    _jmap(self.fallback_by_cause), _jmap(self.status_by_label), self.refits,
                    _jnum(self.seconds), _jnum(self.host_seconds), _jnum(self.fallback_seconds),
                    self.fallback_bounded, self.fallback_workers, self.fallback_max))


# ---- the exact f64 finalist refit (host/refit.cpp) ---------------------------

REFIT_METRICS = {"squared": 0, "absolute": 1, "log_squashed": 2, "aic": 7, "aicc": 8, "bic": 9}


def _cols64(cols, n):
    c = np.ascontiguousarray(cols, np.float64)
    nvars = c.size // n if n else 0
    return c, nvars


def refit_finalists_exact(trees, cols, y, iters, metric="squared", w=None, threads=0):
    """`refit_finalists_exact` (fit/gpu.rs:666-687) for the least-squares
    family (`fit_lm`) and the absolute / log-squashed IRLS arms, on the host
    cores. `cols` is column-major f64 [nvars][n]. Returns (objective per
    finalist, refit trees); the inputs are not modified. Raises ValueError for
    a metric this refit does not cover."""
    code = REFIT_METRICS.get(metric, metric)
    y = np.ascontiguousarray(y, np.float64)
    n = len(y)
    c, nvars = _cols64(cols, n)
    wv = None if w is None else np.ascontiguousarray(w, np.float64)
    ops, vals, off = [], [], [0]
    for t in trees:
        o, v = t.prefix()
        ops.append(np.asarray(o, np.int32))
        vals.append(np.asarray(v, np.float64))
        off.append(off[-1] + len(o))
    ops = np.ascontiguousarray(np.concatenate(ops) if ops else np.zeros(1, np.int32), np.int32)
    vals = np.ascontiguousarray(np.concatenate(vals) if vals else np.zeros(1), np.float64)
    off = np.asarray(off, np.int32)
    loss = np.zeros(max(len(trees), 1), np.float64)
    rc = lib().rch_refit_finalists(_p(ops, ctypes.c_int32), _p(vals, ctypes.c_double),
                                   _p(off, ctypes.c_int32), len(trees), _p(c, ctypes.c_double),
                                   n, nvars, _p(y, ctypes.c_double),
                                   None if wv is None else _p(wv, ctypes.c_double), int(iters),
                                   int(code), int(threads), _p(loss, ctypes.c_double))
    if rc == -2:
        raise ValueError(f"the exact refit does not cover metric {metric!r}")
    if rc != 0:
        raise ValueError(f"rch_refit_finalists rejected its arguments ({rc})")
    out = []
    for i, t in enumerate(trees):
        u = t.clone()
        u.set_prefix_values(vals[off[i]:off[i + 1]])
        out.append(u)
    return loss[:len(trees)], out


def soa_eval(tree, cols, n):
    """Predictions of `tree` over n rows (`eval_soa::eval_batch`)."""
    o, v = tree.prefix()
    o = np.ascontiguousarray(o, np.int32)
    v = np.ascontiguousarray(v, np.float64)
    c, nvars = _cols64(cols, n)
    out = np.empty(max(n, 1), np.float64)
    rc = lib().rch_soa_eval(_p(o, ctypes.c_int32), _p(v, ctypes.c_double), len(o),
                            _p(c, ctypes.c_double), n, nvars, _p(out, ctypes.c_double))
    if rc != 0:
        raise ValueError("malformed tree")
    return out[:n]


def soa_sse(tree, cols, y):
    """The raw SSE of `tree` (`eval_soa::sse`)."""
    o, v = tree.prefix()
    o = np.ascontiguousarray(o, np.int32)
    v = np.ascontiguousarray(v, np.float64)
    y = np.ascontiguousarray(y, np.float64)
    c, nvars = _cols64(cols, len(y))
    return lib().rch_soa_sse(_p(o, ctypes.c_int32), _p(v, ctypes.c_double), len(o),
                             _p(c, ctypes.c_double), len(y), nvars, _p(y, ctypes.c_double))


# ---- the checkpoint's backend identity ---------------------------------------
#
# A run on this library is a `gpu` run: its checkpoint records `backend gpu`
# and `error_kind f32_proxy` (the saved errors are the f32 device scores), and
# a resume onto the other backend is refused unless explicitly allowed
# (checkpoint.rs:89-160, :525-550, :1133-1175; provenance.rs:13-85). The
# device name is the library's own `rc_device_name`.

BACKENDS = ("cpu", "gpu", "unknown")


class CheckpointMismatch(Exception):
    """A resume the reference refuses (exit code 3, input error)."""


def parse_backend(s: str) -> str:
    """`Backend::parse` (checkpoint.rs:108-117)."""
    if s not in BACKENDS:
        raise ValueError(f"backend must be 'cpu', 'gpu' or 'unknown', got '{s}'")
    return s


def error_kind_for_backend(backend: str) -> str:
    """`ErrorKind::for_backend` (checkpoint.rs:153-160): what the saved
    errors are."""
    return {"gpu": "f32_proxy", "cpu": "f64", "unknown": "unknown"}[parse_backend(backend)]


def check_backend(saved: str, current: str, allow_change: bool = False) -> None:
    """`Checkpoint::check_backend` (checkpoint.rs:1133-1151): a checkpoint
    from before the record (`unknown`) is not checked."""
    if saved == "unknown":
        return
    if saved != current and not allow_change:
        raise CheckpointMismatch(
            f"checkpoint backend mismatch: saved run used '{saved}', this run uses "
            f"'{current}'; pass --allow-backend-change to resume across backends (the "
            f"trajectory and reported errors will differ)")


def backend_change_note(saved: str, current: str):
    """The stderr line of an allowed backend change (main.rs:4196-4206), or
    None when there is no change to report."""
    if saved == "unknown" or saved == current:
        return None
    return f"# checkpoint: backend changed {saved} -> {current} (allowed by --allow-backend-change)"


class BuildIdentity:
    """`provenance::BuildIdentity` (provenance.rs:13-85): what produced a
    saved state. For a `gpu` run `device` is `rc_device_name()` and `driver`
    the driver version; a CPU run records `cpu` / `n/a`."""

    FIELDS = ("version", "commit", "binary_sha256", "device", "driver", "threads")

    def __init__(self, version, commit, binary_sha256, device, driver, threads):
        self.version, self.commit, self.binary_sha256 = version, commit, binary_sha256
        self.device, self.driver, self.threads = device, driver, int(threads)

    @classmethod
    def current(cls, gpu: bool, version="unknown", commit="unknown", binary_sha256="unknown"):
        device, driver = device_identity(gpu)
        return cls(version, commit, binary_sha256, device, driver, os.cpu_count() or 1)

    def differences(self, now: "BuildIdentity"):
        """Every differing field as `name: saved A -> current B`; device and
        driver only when both runs used the GPU."""
        out = []

        def cmp(name, a, b):
            if a != b:
                out.append(f"{name}: saved {a} -> current {b}")
        cmp("version", self.version, now.version)
        cmp("commit", self.commit, now.commit)
        cmp("binary_sha256", self.binary_sha256, now.binary_sha256)
        if self.device != "cpu" and now.device != "cpu":
            cmp("device", self.device, now.device)
            cmp("driver", self.driver, now.driver)
        cmp("threads", str(self.threads), str(now.threads))
        return out

    def records(self):
        """The `build ...` lines of a checkpoint (checkpoint.rs:543-550)."""
        return [f"build {k} {getattr(self, k)}" for k in self.FIELDS]


def check_identity(saved, current: BuildIdentity, allow_change: bool = False) -> None:
    """`Checkpoint::check_identity` (checkpoint.rs:1156-1175); `saved` None
    is a checkpoint written before the identity existed."""
    if saved is None:
        return
    diff = saved.differences(current)
    if not diff or allow_change:
        return
    raise CheckpointMismatch(
        f"checkpoint build identity mismatch ({'; '.join(diff)}); pass "
        f"--allow-build-change to resume under a different binary, device or thread count "
        f"(the trajectory may differ)")


def device_identity(gpu: bool):
    """`manifest::device_info` (manifest.rs:358-389) without the CUDA
    version: (device, driver)."""
    if not gpu:
        return "cpu", "n/a"
    from . import device as _device
    name = _device.device_name()
    driver = "unknown"
    try:
        import subprocess
        r = subprocess.run(["nvidia-smi"], capture_output=True, text=True, timeout=30)
        if r.returncode == 0:
            for line in r.stdout.splitlines():
                if "Driver Version:" in line:
                    driver = line.split("Driver Version:")[1].split()[0]
                    break
    except (OSError, subprocess.SubprocessError):
        pass
    return name, driver


def checkpoint_backend_records(identity: BuildIdentity = None):
    """The identity lines a checkpoint of a run on this library carries:
    `backend gpu`, `error_kind f32_proxy` and, with an identity, its
    `build ...` lines (checkpoint.rs:533, :542-550)."""
    lines = ["backend gpu", f"error_kind {error_kind_for_backend('gpu')}"]
    if identity is not None:
        lines += identity.records()
    return lines
