"""ctypes binding of the C ABI (`librcsr_b200.so`) and the host evaluator.

`GpuEvaluator` mirrors the reference's `GpuEvaluator` (my-version/src/gpu.rs:
1182-2896): it owns one device context over a resident dataset and offers the
batched scorer, raw predictions, the batched fit, the implicit score and the
per-row gradients. There is no CPU fallback: if the CUDA library is missing
or a device call fails, the call raises.
"""
from __future__ import annotations

import ctypes
import os

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
CUDA_LIB = os.path.join(_HERE, "librcsr_b200.so")
_lib = None

P = ctypes.POINTER
u32p, i32p, f32p, f64p, u64p, i64p = (P(ctypes.c_uint32), P(ctypes.c_int32), P(ctypes.c_float),
                                      P(ctypes.c_double), P(ctypes.c_uint64), P(ctypes.c_int64))
ci, cf, cvp = ctypes.c_int, ctypes.c_float, ctypes.c_void_p


class RcStats(ctypes.Structure):
    _fields_ = [("kernel_ms", ctypes.c_double), ("launch_ms", ctypes.c_double),
                ("sync_ms", ctypes.c_double), ("alloc_ms", ctypes.c_double),
                ("h2d_ms", ctypes.c_double), ("d2h_ms", ctypes.c_double),
                ("wall_ms", ctypes.c_double), ("h2d_bytes", ctypes.c_ulonglong),
                ("d2h_bytes", ctypes.c_ulonglong), ("batch", ctypes.c_int),
                ("failed", ctypes.c_int)]


class RcArenaReport(ctypes.Structure):
    _fields_ = [("async_copy", ctypes.c_int), ("reason", ctypes.c_char * 96),
                ("pinned_bytes", ctypes.c_ulonglong), ("alloc_calls", ctypes.c_ulonglong),
                ("steady_alloc_calls", ctypes.c_ulonglong),
                ("overlapped_uploads", ctypes.c_ulonglong), ("batches", ctypes.c_ulonglong),
                ("fs_alloc_calls", ctypes.c_ulonglong), ("fs_growths", ctypes.c_ulonglong),
                ("fs_steady_alloc_calls", ctypes.c_ulonglong),
                ("fs_batches", ctypes.c_ulonglong), ("fs_dev_bytes", ctypes.c_ulonglong),
                ("fs_pinned_bytes", ctypes.c_ulonglong)]


class RcMaxOut(ctypes.Structure):
    _fields_ = [("vmax", ctypes.c_double), ("lo", ctypes.c_double), ("hi", ctypes.c_double),
                ("row", ctypes.c_int), ("status", ctypes.c_int)]


# name -> (restype, argtypes): every symbol include/rcsr_b200.h declares.
SIGNATURES = {
    "rc_create": (cvp, [f32p, ci, ci, f32p]),
    "rc_destroy": (None, [cvp]),
    "rc_set_fit_data": (ci, [cvp, f64p, f64p, f64p]),
    "rc_set_score_weights": (ci, [cvp, f64p]),
    "rc_set_fit_sign": (ci, [cvp, f64p]),
    "rc_set_programs": (ci, [cvp, u32p, u32p, ci]),
    "rc_eval": (cf, [cvp, f32p, ci]),
    "rc_eval_submit": (ci, [cvp, ci]),
    "rc_eval_collect": (cf, [cvp, f32p]),
    "rc_score_batch": (cf, [cvp, u32p, u32p, ci, ci, i32p, f64p, i32p]),
    "rc_pool_reserve": (ci, [cvp, ci, ci]),
    "rc_pool_upload": (ci, [cvp, ci, u32p, ci]),
    "rc_pool_eval": (cf, [cvp, ci, ci, ci, f32p, ci]),
    "rc_pool_score": (cf, [cvp, ci, ci, ci, ci, i32p, f64p, i32p]),
    "rc_pool_hash": (ci, [cvp, ci, ci, ci, u64p]),
    "rc_pool_vary": (cf, [cvp, ci, ci, ci, ci, f64p, ci, ci, ctypes.c_uint, ctypes.c_uint, ci, ci,
                          u32p, ci, P(ctypes.c_uint8), u32p, u32p, ci, ctypes.c_double,
                          P(ctypes.c_uint16), P(ctypes.c_uint16), u64p, f64p, u32p]),
    "rc_predict": (ci, [cvp, u32p, u32p, ci, f32p]),
    "rc_fit_batch": (cf, [cvp, u32p, u32p, i32p, ci, ci, f64p, i32p, ci, ci, f64p, f64p, i32p]),
    "rc_fit_kernel_info": (ci, [ci, i32p, i32p, i32p]),
    "rc_rank_score_batch": (cf, [cvp, u32p, u32p, i32p, ci, ci, ci, f64p, u64p, i32p, u64p]),
    "rc_rank_debug_b": (ci, [cvp, i64p]),
    "rc_launch_count": (ci, [cvp, u64p]),
    "rc_rank_tuning": (ci, [cvp, ci, ci]),
    "rc_rank_last_fallbacks": (ci, [cvp]),
    "rc_last_fit_sweeps": (ci, [cvp, ci, ctypes.POINTER(ctypes.c_int32)]),
    "rc_multi_create": (cvp, [f32p, ci, ci, f32p, ci, i32p]),
    "rc_multi_destroy": (None, [cvp]),
    "rc_multi_set_fit_data": (ci, [cvp, f64p, f64p, f64p]),
    "rc_multi_score_batch": (cf, [cvp, u32p, u32p, ci, ci, i32p, f64p, i32p]),
    "rc_multi_fit_batch": (cf, [cvp, u32p, u32p, i32p, ci, ci, f64p, i32p, ci, ci, ci, f64p,
                                f64p, i32p]),
    "rc_multi_devices": (ci, [cvp, ctypes.POINTER(cvp)]),
    "rc_fit_autotune": (ci, [cvp, u32p, u32p, i32p, ci, ci, f64p, i32p, ci, ci, ci,
                             ctypes.c_char_p]),
    "rc_fit_budgets": (ci, [cvp, i32p]),
    "rc_last_score_profile": (ci, [cvp, ctypes.POINTER(ctypes.c_float),
                                   ctypes.POINTER(ctypes.c_float), u64p, u64p, u64p, u64p]),
    "rc_order_stat_score_batch": (cf, [cvp, u32p, u32p, i32p, ci, ci, ci, f64p, ci, f64p,
                                       i32p]),
    "rc_max_scan_batch": (cf, [cvp, u32p, u32p, i32p, ci, ci, ci, f64p, i32p, f64p,
                               P(RcMaxOut)]),
    "rc_stats_begin": (None, [cvp]),
    "rc_last_stats": (ci, [cvp, P(RcStats)]),
    "rc_arena_report": (ci, [cvp, P(RcArenaReport)]),
    "rc_arena_force_sync": (ci, [cvp, ci]),
    "rc_device_count": (ci, []),
    "rc_device_name": (ctypes.c_char_p, []),
    "rc_unified": (ci, []),
    "rc_fit_batch_fused": (cf, [cvp, u32p, u32p, i32p, ci, ci, f64p, i32p, ci, ci, ci, f64p,
                                f64p, i32p]),
    "rc_fit_batch_plain": (cf, [cvp, u32p, u32p, i32p, ci, ci, f64p, i32p, ci, ci, f64p, f64p,
                                i32p]),
    "rc_grad_batch": (ci, [cvp, u32p, u32p, i32p, ci, ci, f64p, ci, ci, ci, f32p, f32p]),
    "rc_implicit_score_batch": (cf, [cvp, u32p, u32p, i32p, ci, ci, f64p, f64p, i32p]),
    "rc_autotune": (ci, [cvp, u32p, u32p, ci, ctypes.c_char_p]),
    "rc_score_batch_noalloc": (ci, [cvp, cvp, ci, ci, ci, cvp, cvp, ci, ci, cvp, cvp, cvp]),
}


def lib():
    """Load the CUDA library. Raises when it is not built: the device path has
    no fallback."""
    global _lib
    if _lib is None:
        if not os.path.exists(CUDA_LIB):
            raise ImportError(f"{CUDA_LIB} is not built: run the package's build.py")
        L = ctypes.CDLL(CUDA_LIB)
        for name, (res, args) in SIGNATURES.items():
            fn = getattr(L, name)
            fn.restype = res
            fn.argtypes = args
        _lib = L
    return _lib


def _p(a, ct):
    if a is None:
        return None
    return a.ctypes.data_as(ctypes.POINTER(ct))


def _c(a, dt):
    return None if a is None else np.ascontiguousarray(a, dtype=dt)


def _i128(hi, lo):
    """Two's-complement 128-bit value from its (hi, lo) u64 halves."""
    v = (int(hi) << 64) | int(lo)
    return v - (1 << 128) if v >= 1 << 127 else v


# Score objective codes (RC_SCORE_*, my-version/src/cuda/eval.cu:609-640).
SCORE_SQUARED, SCORE_ABSOLUTE, SCORE_LOG_SQUASHED, SCORE_SIGNED, SCORE_MAXIMUM = 0, 1, 2, 3, 4
SCORE_CORRELATION, SCORE_CORRELATION_SIGNED, SCORE_AIC, SCORE_AICC, SCORE_BIC = 5, 6, 7, 8, 9
SCORE_LOG_LOSS, SCORE_BRIER, SCORE_HINGE_SIGMOID = 10, 11, 12
SCORE_HINGE_ORDINARY, SCORE_HINGE_SQUARED = 13, 14
# Fit metric codes (RC_LOSS_*, eval.cu:589-604) plus the additive implicit arm.
LOSS_SQUARED, LOSS_LOG_SQUASHED, LOSS_CORRELATION, LOSS_CORRELATION_SIGNED = 0, 1, 2, 3
LOSS_ABSOLUTE, LOSS_LOGISTIC, LOSS_IMPLICIT = 4, 5, 6
# Fit statuses usable by the caller (my-version/src/fit/gpu.rs:103-105).
FIT_STATUS_USABLE = {0, 4, 5, 6, 7, 8}


class DeviceError(RuntimeError):
    pass


class GpuEvaluator:
    """One device context over a resident dataset (f32 column-major)."""

    def __init__(self, cols, n, v, y):
        L = lib()
        self.n, self.v = int(n), int(v)
        self._cols = _c(cols, np.float32)
        self._y = _c(y, np.float32)
        self.ctx = L.rc_create(_p(self._cols, ctypes.c_float), self.n, self.v,
                               _p(self._y, ctypes.c_float))
        if not self.ctx:
            raise DeviceError("rc_create failed (no usable CUDA device?)")

    def close(self):
        if self.ctx:
            lib().rc_destroy(self.ctx)
            self.ctx = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    # -- data ----------------------------------------------------------
    def set_fit_data(self, cols64, y64, w=None):
        c, y = _c(cols64, np.float64), _c(y64, np.float64)
        w = _c(w, np.float64) if w is not None and len(w) else None
        rc = lib().rc_set_fit_data(self.ctx, _p(c, ctypes.c_double), _p(y, ctypes.c_double),
                                   _p(w, ctypes.c_double))
        if rc != 0:
            raise DeviceError("rc_set_fit_data failed")

    def set_score_weights(self, w):
        w = _c(w, np.float64)
        if lib().rc_set_score_weights(self.ctx, _p(w, ctypes.c_double)) != 0:
            raise DeviceError("rc_set_score_weights failed")

    def set_fit_sign(self, sign):
        s = _c(sign, np.float64)
        if lib().rc_set_fit_sign(self.ctx, _p(s, ctypes.c_double)) != 0:
            raise DeviceError("rc_set_fit_sign failed")

    # -- scoring -------------------------------------------------------
    def score_batch(self, prog, off, kind, pcount=None):
        prog, off = _c(prog, np.uint32), _c(off, np.uint32)
        P_ = len(off) - 1
        pc = _c(pcount if pcount is not None else np.zeros(P_), np.int32)
        out = np.zeros(P_, np.float64)
        status = np.zeros(P_, np.int32)
        ms = lib().rc_score_batch(self.ctx, _p(prog, ctypes.c_uint32), _p(off, ctypes.c_uint32),
                                  P_, kind, _p(pc, ctypes.c_int32), _p(out, ctypes.c_double),
                                  _p(status, ctypes.c_int32))
        if ms < 0:
            raise DeviceError(f"rc_score_batch failed ({ms})")
        return out, status, ms

    def eval_batch(self, prog, off, loss=0):
        prog, off = _c(prog, np.uint32), _c(off, np.uint32)
        P_ = len(off) - 1
        L = lib()
        if L.rc_set_programs(self.ctx, _p(prog, ctypes.c_uint32), _p(off, ctypes.c_uint32),
                             P_) != 0:
            raise DeviceError("rc_set_programs failed")
        out = np.zeros(P_, np.float32)
        ms = L.rc_eval(self.ctx, _p(out, ctypes.c_float), loss)
        if ms < 0:
            raise DeviceError("rc_eval failed")
        return out, ms

    def predictions(self, prog, off):
        prog, off = _c(prog, np.uint32), _c(off, np.uint32)
        P_ = len(off) - 1
        out = np.zeros((P_, self.n), np.float32)
        if lib().rc_predict(self.ctx, _p(prog, ctypes.c_uint32), _p(off, ctypes.c_uint32), P_,
                            _p(out, ctypes.c_float)) != 0:
            raise DeviceError("rc_predict failed")
        return out

    # -- fitting -------------------------------------------------------
    def _fit(self, fn, prog, off, pcount, c0, gauge, kmax, iters, metric, flags=None):
        prog, off = _c(prog, np.uint32), _c(off, np.uint32)
        pcount, gauge = _c(pcount, np.int32), _c(gauge, np.int32)
        c0 = _c(c0, np.float64)
        P_ = len(off) - 1
        outc = np.zeros((P_, kmax), np.float64)
        outsse = np.zeros(P_, np.float64)
        status = np.zeros(P_, np.int32)
        args = [self.ctx, _p(prog, ctypes.c_uint32), _p(off, ctypes.c_uint32),
                _p(pcount, ctypes.c_int32), P_, kmax, _p(c0, ctypes.c_double),
                _p(gauge, ctypes.c_int32), iters, metric]
        if flags is not None:
            args.append(flags)
        args += [_p(outc, ctypes.c_double), _p(outsse, ctypes.c_double),
                 _p(status, ctypes.c_int32)]
        ms = fn(*args)
        if ms < 0:
            raise DeviceError(f"fit launch failed ({ms})")
        return outc, outsse, status, ms

    def fit_batch(self, prog, off, pcount, c0, gauge, kmax, iters, metric=LOSS_SQUARED):
        return self._fit(lib().rc_fit_batch, prog, off, pcount, c0, gauge, kmax, iters, metric)

    def fit_batch_fused(self, prog, off, pcount, c0, gauge, kmax, iters, metric=LOSS_SQUARED,
                        flags=0):
        return self._fit(lib().rc_fit_batch_fused, prog, off, pcount, c0, gauge, kmax, iters,
                         metric, flags)

    def fit_batch_plain(self, prog, off, pcount, c0, gauge, kmax, iters, metric=LOSS_SQUARED):
        return self._fit(lib().rc_fit_batch_plain, prog, off, pcount, c0, gauge, kmax, iters,
                         metric)

    def fit_plans(self, plans, iters, metric=LOSS_SQUARED, fused=True, flags=0):
        """Fit a list of `host.GpuFitPlan`; returns (c[P][kmax], loss[P],
        status[P], ms)."""
        from .host import pack_plans
        prog, off, pcount, c0, gauge, kmax = pack_plans(plans)
        if fused:
            return self.fit_batch_fused(prog, off, pcount, c0, gauge, kmax, iters, metric, flags)
        return self.fit_batch(prog, off, pcount, c0, gauge, kmax, iters, metric)

    # -- gradients / implicit -------------------------------------------
    def grad_batch(self, prog, off, pcount, c, kmax, want, row0, nrows):
        prog, off, pcount = _c(prog, np.uint32), _c(off, np.uint32), _c(pcount, np.int32)
        c = _c(c, np.float64)
        P_ = len(off) - 1
        width = kmax if want == 1 else self.v
        value = np.zeros((P_, nrows), np.float32)
        out = np.zeros((P_, nrows, width), np.float32)
        rc = lib().rc_grad_batch(self.ctx, _p(prog, ctypes.c_uint32), _p(off, ctypes.c_uint32),
                                 _p(pcount, ctypes.c_int32), P_, kmax, _p(c, ctypes.c_double),
                                 want, row0, nrows, _p(value, ctypes.c_float),
                                 _p(out, ctypes.c_float))
        if rc != 0:
            raise DeviceError("rc_grad_batch failed")
        return value, out

    def implicit_score(self, prog, off, pcount, c, kmax):
        prog, off, pcount = _c(prog, np.uint32), _c(off, np.uint32), _c(pcount, np.int32)
        c = _c(c, np.float64)
        P_ = len(off) - 1
        out = np.zeros(P_, np.float64)
        status = np.zeros(P_, np.int32)
        ms = lib().rc_implicit_score_batch(self.ctx, _p(prog, ctypes.c_uint32),
                                           _p(off, ctypes.c_uint32), _p(pcount, ctypes.c_int32),
                                           P_, kmax, _p(c, ctypes.c_double),
                                           _p(out, ctypes.c_double), _p(status, ctypes.c_int32))
        if ms < 0:
            raise DeviceError("rc_implicit_score_batch failed")
        return out, status, ms

    # -- exact statistics (my-version/src/gpu.rs:1986-2075, :2628-2838) ----
    @staticmethod
    def _segments(prog, off, pcount, c0, kmax, ntrials):
        prog, off, pcount = _c(prog, np.uint32), _c(off, np.uint32), _c(pcount, np.int32)
        nsets = len(off) - 1
        c0 = _c(c0, np.float64).reshape(-1)
        if c0.size != nsets * ntrials * kmax:
            raise ValueError("c0 must hold nsets * ntrials * kmax constants")
        return prog, off, pcount, c0, nsets

    def rank_sums(self, prog, off, pcount, c0, kmax, ntrials=1):
        """Exact rank sums per (set, trial) segment: a list of (ab, aa) Python
        ints (None where status != 0), the statuses, sum B^2 and the ms."""
        prog, off, pcount, c0, nsets = self._segments(prog, off, pcount, c0, kmax, ntrials)
        nseg = nsets * ntrials
        out = np.zeros(4 * nseg, np.uint64)
        status = np.zeros(nseg, np.int32)
        bb = np.zeros(2, np.uint64)
        ms = lib().rc_rank_score_batch(self.ctx, _p(prog, ctypes.c_uint32),
                                       _p(off, ctypes.c_uint32), _p(pcount, ctypes.c_int32),
                                       nsets, ntrials, kmax, _p(c0, ctypes.c_double),
                                       _p(out, ctypes.c_uint64), _p(status, ctypes.c_int32),
                                       _p(bb, ctypes.c_uint64))
        if ms < 0:
            raise DeviceError("rc_rank_score_batch failed")
        sums = []
        for s in range(nseg):
            if status[s] != 0:
                sums.append(None)
            else:
                sums.append((_i128(out[4 * s], out[4 * s + 1]), _i128(out[4 * s + 2], out[4 * s + 3])))
        return sums, status, _i128(bb[0], bb[1]), ms

    def rank_tuning(self, bucket_cap=0, group_max=0):
        """Rank-sum method: bucket capacity (0 built in, -1 radix sort only)
        and the largest group of distinct keys ranked by comparison."""
        if lib().rc_rank_tuning(self.ctx, int(bucket_cap), int(group_max)) != 0:
            raise ValueError("rc_rank_tuning refused its arguments")

    def rank_fallbacks(self):
        """Segments of the last rank_sums call that the radix sort summed."""
        return int(lib().rc_rank_last_fallbacks(self.ctx))

    def rank_target(self):
        out = np.zeros(self.n, np.int64)
        if lib().rc_rank_debug_b(self.ctx, _p(out, ctypes.c_int64)) != 0:
            raise DeviceError("rc_rank_debug_b failed")
        return out

    def order_stat(self, prog, off, pcount, c0, kmax, what, ntrials=1):
        """Exact median (what 0) or interquartile mean (what 1) of |r| per
        segment, with statuses and the ms."""
        prog, off, pcount, c0, nsets = self._segments(prog, off, pcount, c0, kmax, ntrials)
        nseg = nsets * ntrials
        val = np.zeros(nseg, np.float64)
        status = np.zeros(nseg, np.int32)
        ms = lib().rc_order_stat_score_batch(self.ctx, _p(prog, ctypes.c_uint32),
                                             _p(off, ctypes.c_uint32), _p(pcount, ctypes.c_int32),
                                             nsets, ntrials, kmax, _p(c0, ctypes.c_double), what,
                                             _p(val, ctypes.c_double), _p(status, ctypes.c_int32))
        if ms < 0:
            raise DeviceError("rc_order_stat_score_batch failed")
        return val, status, ms

    def max_scan(self, prog, off, pcount, c0, kmax, ntrials=1, coords=None, levels=None):
        """Exact max |r|, its lowest row and the level intervals per segment."""
        prog, off, pcount, c0, nsets = self._segments(prog, off, pcount, c0, kmax, ntrials)
        nseg = nsets * ntrials
        out = (RcMaxOut * nseg)()
        coords = _c(coords, np.int32)
        levels = _c(levels, np.float64)
        ms = lib().rc_max_scan_batch(self.ctx, _p(prog, ctypes.c_uint32), _p(off, ctypes.c_uint32),
                                     _p(pcount, ctypes.c_int32), nsets, ntrials, kmax,
                                     _p(c0, ctypes.c_double), _p(coords, ctypes.c_int32),
                                     _p(levels, ctypes.c_double), out)
        if ms < 0:
            raise DeviceError("rc_max_scan_batch failed")
        return [(o.vmax, o.row, o.lo, o.hi, o.status) for o in out], ms

    # -- telemetry -----------------------------------------------------
    def stats_begin(self):
        lib().rc_stats_begin(self.ctx)

    def last_stats(self):
        s = RcStats()
        lib().rc_last_stats(self.ctx, ctypes.byref(s))
        return s

    def autotune(self, prog, off, path=None):
        """Time the scorer's candidates-per-item choice per length bucket on
        this batch; returns the number of cached entries."""
        prog, off = _c(prog, np.uint32), _c(off, np.uint32)
        p = path.encode() if path else None
        k = lib().rc_autotune(self.ctx, _p(prog, ctypes.c_uint32), _p(off, ctypes.c_uint32),
                              len(off) - 1, p)
        if k < 0:
            raise DeviceError("rc_autotune failed")
        return k

    def launch_count(self):
        """Kernels launched on this context so far."""
        out = np.zeros(1, np.uint64)
        if lib().rc_launch_count(self.ctx, _p(out, ctypes.c_uint64)) != 0:
            raise DeviceError("rc_launch_count failed")
        return int(out[0])

    def fit_autotune(self, plans, iters=20, metric=LOSS_SQUARED, sample=0, path=None):
        """Tune the fit's assembly budget per length bucket on these plans
        (rc_fit_autotune; sample 0: a GPU-filling tuning batch); returns the
        budgets in KB per bucket."""
        from .host import pack_plans
        prog, off, pcount, c0, gauge, kmax = pack_plans(plans)
        prog, off = _c(prog, np.uint32), _c(off, np.uint32)
        pcount, gauge, c0 = _c(pcount, np.int32), _c(gauge, np.int32), _c(c0, np.float64)
        rc = lib().rc_fit_autotune(self.ctx, _p(prog, ctypes.c_uint32), _p(off, ctypes.c_uint32),
                                   _p(pcount, ctypes.c_int32), len(off) - 1, kmax,
                                   _p(c0, ctypes.c_double), _p(gauge, ctypes.c_int32), iters,
                                   metric, sample, None if path is None else path.encode())
        if rc < 0:
            raise DeviceError("rc_fit_autotune failed")
        return self.fit_budgets()

    def fit_budgets(self):
        out = np.zeros(4, np.int32)
        if lib().rc_fit_budgets(self.ctx, _p(out, ctypes.c_int32)) != 0:
            raise DeviceError("rc_fit_budgets failed")
        return out.tolist()

    def fit_sweeps(self, nprog):
        """Sweeps per candidate of the last fit: int32 [P][4] (f32 assembly,
        f32 objective, f64 assembly, f64 objective)."""
        out = np.zeros((nprog, 4), np.int32)
        if lib().rc_last_fit_sweeps(self.ctx, nprog, _p(out, ctypes.c_int32)) != 0:
            raise DeviceError("rc_last_fit_sweeps failed")
        return out

    def score_profile(self):
        """Profile of the last scoring call: dict with the device ms of the
        f32 scoring kernels (`ms_f32`) and of the rest (`ms_rest`), the rows
        the f32 interpreter and the f64 lane evaluated (`rows_f32`,
        `rows_f64`) and those rows x (postfix ops + 2) (`ops_f32`,
        `ops_f64`)."""
        ms = np.zeros(2, np.float32)
        q = np.zeros(4, np.uint64)
        if lib().rc_last_score_profile(self.ctx, _p(ms[0:1], ctypes.c_float),
                                       _p(ms[1:2], ctypes.c_float), _p(q[0:1], ctypes.c_uint64),
                                       _p(q[1:2], ctypes.c_uint64), _p(q[2:3], ctypes.c_uint64),
                                       _p(q[3:4], ctypes.c_uint64)) != 0:
            raise DeviceError("rc_last_score_profile failed")
        return {"ms_f32": float(ms[0]), "ms_rest": float(ms[1]), "rows_f32": int(q[0]),
                "rows_f64": int(q[1]), "ops_f32": int(q[2]), "ops_f64": int(q[3])}

    def arena_report(self):
        r = RcArenaReport()
        lib().rc_arena_report(self.ctx, ctypes.byref(r))
        return r


def device_count() -> int:
    return lib().rc_device_count()


def device_name() -> str:
    return lib().rc_device_name().decode()


class GenomePool:
    """The device's double-buffered fixed-width program pool (`rc_pool_*`,
    eval.cu:3514-3874) of islands x pop slots, with the next generation built
    on the device (`rc_pool_vary`, postfix.rs:511-567)."""

    def __init__(self, ev, islands, pop, width):
        self.ev, self.islands, self.pop, self.width = ev, islands, pop, width
        if lib().rc_pool_reserve(ev.ctx, islands * pop, width) != 0:
            raise DeviceError("rc_pool_reserve failed")

    def upload(self, which, words):
        w = np.ascontiguousarray(words, np.uint32).reshape(-1)
        assert w.size == self.islands * self.pop * self.width
        if lib().rc_pool_upload(self.ev.ctx, which, _p(w, ctypes.c_uint32),
                                self.islands * self.pop) != 0:
            raise DeviceError("rc_pool_upload failed")

    def score(self, which, kind=0, pcount=None):
        """Score every slot of pool `which` (rc_pool_score): (values f64,
        status i32, ms)."""
        n = self.islands * self.pop
        pc = _c(pcount if pcount is not None else np.zeros(n), np.int32)
        out = np.zeros(n, np.float64)
        st = np.zeros(n, np.int32)
        ms = lib().rc_pool_score(self.ev.ctx, which, n, self.width, kind, _p(pc, ctypes.c_int32),
                                 _p(out, ctypes.c_double), _p(st, ctypes.c_int32))
        if ms < 0:
            raise DeviceError("rc_pool_score failed")
        return out, st, ms

    def hash(self, which):
        out = np.zeros(self.islands * self.pop, np.uint64)
        if lib().rc_pool_hash(self.ev.ctx, which, self.islands * self.pop, self.width,
                              _p(out, ctypes.c_uint64)) != 0:
            raise DeviceError("rc_pool_hash failed")
        return out

    def vary(self, which, err, gen, nvars, max_complexity, seed, ops, init_depth=3, dedup=True,
             restart=None, front=None, front_p=0.0, words=True, out=None):
        """Children of pool `which` into pool `which ^ 1`. Returns
        (words [islands*pop, width] or None, len, cost, hash, err, ms).
        `out` may hold caller-owned result arrays (words or None, len u16,
        cost u16, hash u64, err f64, each C-contiguous with islands*pop rows),
        for example in pinned memory reused across generations; they are
        filled and returned in place of fresh ones."""
        n = self.islands * self.pop
        e = np.ascontiguousarray(err, np.float64)
        o = np.ascontiguousarray(np.asarray(ops, np.uint32).reshape(-1))
        r = None if restart is None else np.ascontiguousarray(restart, np.uint8)
        fw = fo = None
        nf = 0
        if front:
            fo = np.zeros(len(front) + 1, np.uint32)
            fo[1:] = np.cumsum([len(f) for f in front])
            fw = np.ascontiguousarray(np.concatenate([np.asarray(f, np.uint32) for f in front]))
            nf = len(front)
        if out is not None:
            ow, ol, oc, oh, oe = out
            for a, dt, m in ((ol, np.uint16, n), (oc, np.uint16, n), (oh, np.uint64, n),
                             (oe, np.float64, n), (ow, np.uint32, n * self.width)):
                if a is None and dt is np.uint32:
                    continue
                if a.dtype != dt or a.size != m or not a.flags.c_contiguous:
                    raise ValueError("vary: out arrays must be C-contiguous words u32 "
                                     "[n*width], len u16, cost u16, hash u64, err f64 [n]")
            ow = None if ow is None else ow.reshape(-1)
        else:
            ol = np.zeros(n, np.uint16)
            oc = np.zeros(n, np.uint16)
            oh = np.zeros(n, np.uint64)
            oe = np.zeros(n, np.float64)
            ow = np.zeros(n * self.width, np.uint32) if words else None
        ms = lib().rc_pool_vary(self.ev.ctx, which, self.islands, self.pop, self.width,
                                _p(e, ctypes.c_double), nvars, max_complexity, seed, gen,
                                init_depth, int(dedup), _p(o, ctypes.c_uint32), len(o) // 2,
                                _p(r, ctypes.c_uint8), _p(fw, ctypes.c_uint32),
                                _p(fo, ctypes.c_uint32), nf, front_p, _p(ol, ctypes.c_uint16),
                                _p(oc, ctypes.c_uint16), _p(oh, ctypes.c_uint64),
                                _p(oe, ctypes.c_double), _p(ow, ctypes.c_uint32))
        if ms < 0:
            raise DeviceError("rc_pool_vary failed")
        return (None if ow is None else ow.reshape(n, self.width)), ol, oc, oh, oe, ms


class MultiEvaluator:
    """Several GPUs behind one handle (`rc_multi_*`): one context per device,
    each holding the rows; batches are split into contiguous candidate slices
    run concurrently, and the outputs gathered in place."""

    def __init__(self, cols, n, v, y, devices):
        c, yy = _c(cols, np.float32), _c(y, np.float32)
        d = np.ascontiguousarray(devices, np.int32)
        self.n, self.v, self.ndev = n, v, len(d)
        self.h = lib().rc_multi_create(_p(c, ctypes.c_float), n, v, _p(yy, ctypes.c_float),
                                       len(d), _p(d, ctypes.c_int32))
        if not self.h:
            raise DeviceError("rc_multi_create failed")

    def close(self):
        if self.h:
            lib().rc_multi_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def set_fit_data(self, cols64, y64, w=None):
        c, y = _c(cols64, np.float64), _c(y64, np.float64)
        w = _c(w, np.float64) if w is not None else None
        if lib().rc_multi_set_fit_data(self.h, _p(c, ctypes.c_double), _p(y, ctypes.c_double),
                                       _p(w, ctypes.c_double)) != 0:
            raise DeviceError("rc_multi_set_fit_data failed")

    def score_batch(self, prog, off, kind, pcount=None):
        prog, off = _c(prog, np.uint32), _c(off, np.uint32)
        P_ = len(off) - 1
        pc = _c(pcount if pcount is not None else np.zeros(P_), np.int32)
        out = np.zeros(P_, np.float64)
        st = np.zeros(P_, np.int32)
        ms = lib().rc_multi_score_batch(self.h, _p(prog, ctypes.c_uint32),
                                        _p(off, ctypes.c_uint32), P_, kind,
                                        _p(pc, ctypes.c_int32), _p(out, ctypes.c_double),
                                        _p(st, ctypes.c_int32))
        if ms < 0:
            raise DeviceError("rc_multi_score_batch failed")
        return out, st, ms

    def fit_plans(self, plans, iters, metric=LOSS_SQUARED, flags=0):
        from .host import pack_plans
        prog, off, pcount, c0, gauge, kmax = pack_plans(plans)
        prog, off = _c(prog, np.uint32), _c(off, np.uint32)
        pcount, gauge, c0 = _c(pcount, np.int32), _c(gauge, np.int32), _c(c0, np.float64)
        P_ = len(off) - 1
        outc = np.zeros((P_, kmax), np.float64)
        outsse = np.zeros(P_, np.float64)
        st = np.zeros(P_, np.int32)
        ms = lib().rc_multi_fit_batch(self.h, _p(prog, ctypes.c_uint32), _p(off, ctypes.c_uint32),
                                      _p(pcount, ctypes.c_int32), P_, kmax,
                                      _p(c0, ctypes.c_double), _p(gauge, ctypes.c_int32), iters,
                                      metric, flags, _p(outc, ctypes.c_double),
                                      _p(outsse, ctypes.c_double), _p(st, ctypes.c_int32))
        if ms < 0:
            raise DeviceError("rc_multi_fit_batch failed")
        return outc, outsse, st, ms
