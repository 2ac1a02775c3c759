"""Benchmark of the rcsr device hot path on B200.

Default workload (`--workload score`): batched evaluation + squared-error
scoring of P = 4096 random expression programs over N = 1,048,576 rows x 5
features (the batched-scoring configuration), metric expr*row evals/s. On one
GPU the same line also carries the other configurations:
  fit:      batched LM fit of P = 2048 candidates (1-20 constants, 5-60
            nodes, 20 iterations) over N = 262,144 rows x 8 features, fitted
            candidates/s, for the fused graph-replayed batch and for the plain
            one-candidate-per-launch form of the same steps (on a seeded
            random sample of the batch);
  fit_1m:   the same fit distribution at N = 1,048,576 rows;
  implicit: |f|/||grad f|| scoring of P = 1024 candidates of f(x, y, d1, d2)
            over N = 1,048,576 rows through the fused input adjoint, and the
            LM fit of those with constants;
  c5:       one island's generation (P = 1000) over N = 4,194,304 rows x 10
            heavy-tailed features: the L1 IRLS fit and the exact
            rank-correlation sums;
  vary:     the next generation of a 16 x 1000 program pool built on the
            device (tournament, crossover, mutation, hashing, dedup),
            children/s beside the CPU restatement of the reference engine.
`--workload fit|implicit|c5|rank|vary` makes one of them the primary line;
`--workload refit` times the exact f64 finalist refit on the host cores alone.

One step is one pass of the hot path over the whole batch. `value` is
device-timed with CUDA events on the library's stream (inputs resident in
HBM, L2 flushed between steps); `e2e` is the same metric through the public
C-ABI call with host buffers (program upload, decode, launches, result
download inside the timed region). The CPU baseline times the f64 oracle (a
restatement of the reference's CPU path) on a bounded sample on the host's
cores.

Multi-GPU: candidates shard across ranks with no data-path collective
(weak scaling); every rank scores its own P-candidate batch.
"""
from __future__ import annotations

import argparse
import concurrent.futures as cf
import importlib
import json
import os
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)
PKG = "the-rule-and-compass_b200"


def load_peaks():
    try:
        return json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json")))
    except Exception:
        return {"hbm_gbs": 6650.0, "sm_max_mhz": 1965.0, "fallback": True}


class ClockSampler:
    """nvidia-smi clocks and throttle reasons during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index):
        self.gpu = gpu_index
        self.proc = None
        self.lines = []

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.gpu), "--query-gpu=" + self.FIELDS,
                 "--format=csv,noheader,nounits", "-lms", "25"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except Exception:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def __exit__(self, *a):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()

    def summary(self):
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            parts = [p.strip() for p in ln.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                mx = float(parts[2])
            except ValueError:
                continue
            for nm, val in zip(names, parts[5:9]):
                if val.lower() == "active":
                    reasons.add(nm)
        if not sm:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        return {"sm_mhz": float(np.median(sm)), "sm_max_mhz": mx, "reasons": sorted(reasons),
                "samples": len(sm)}


# The scoring CPU sample (the oracle's timed baseline and the parity check):
# the first programs and rows of the timed workload.
SCORE_SAMPLE_PROGS, SCORE_SAMPLE_ROWS = 64, 1 << 16
# DRAM bytes (read + write) of one launch of the f32 scoring kernel on the
# P = 4096, N = 1,048,576 workload, from ncu (profiles/rc_score_kernel_P4096_N1M.md).
SCORE_TRAFFIC = 25.69e6
# DRAM bytes per candidate*row of one f32 assembly sweep of the fit (ncu on
# the first assembly of P = 256 at N = 1,048,576: 1.90 GB and 2.05 GB for the
# two active-thread classes of 128 candidates each; mostly the constant-free
# subtree cache columns), profiles/ft_sweep4_classes_fit_P256_N1M.md.
FIT_ASM_TRAFFIC = {"bytes_per_candidate_row_f32_assembly": 15.0,
                   "source": "profiles/ft_sweep4_classes_fit_P256_N1M.md"}
# DRAM bytes per candidate*row of the whole rank stage, from the per-kernel
# ncu launch list of profiles/rank_buckets_P16_N1M_P100_N4M.md (bucketed
# sums): 2,847 MB over 3 calls of 16 x 1,048,576 rows -- the key kernel's
# column reads and key writes (19.2 B), the bucket scatter (24.1 B), the
# local ranking pass (12.1 B), sampling and splitters (1.1 B).
RANK_TRAFFIC = {"bytes_per_candidate_row": 56.6, "algorithmic": 32.0,
                "source": "profiles/rank_buckets_P16_N1M_P100_N4M.md"}


def flush_l2(buf):
    """Write a buffer larger than the 126 MB L2 between timed steps."""
    if buf is not None:
        buf.zero_()


def postfix_ops(prog, off):
    """Per program: bytecode ops excluding HALT (const/var count one op)."""
    out = []
    for i in range(len(off) - 1):
        w = prog[off[i]:off[i + 1]]
        k, ops = 0, 0
        while k < len(w):
            if w[k] in (0, 1):
                k += 2
            elif w[k] == 255:
                break
            else:
                k += 1
            ops += 1
        out.append(ops)
    return np.asarray(out)


# ---------------------------------------------------------------------------
# CPU baseline: the oracle on a bounded sample, parallel over candidates.
# ---------------------------------------------------------------------------

def cpu_model():
    """The host CPU's model name (Linux /proc/cpuinfo), or None."""
    try:
        for line in open("/proc/cpuinfo"):
            if line.startswith("model name"):
                return line.split(":", 1)[1].strip()
    except OSError:
        pass
    return None


def f32_constants(t):
    """The tree with its constants rounded to f32, as the device's postfix
    words carry them (gpu.rs:354)."""
    t32 = t.clone()
    t32.set_constants([float(np.float32(c)) for c in t.constants()])
    return t32


def cpu_score_baseline(trees, x, y, n_rows, n_cand, threads, want_values=False):
    """The oracle's squared-error score (metrics::score_weighted over
    expr::eval) of the first `n_cand` programs (constants as the device sees
    them) on the first `n_rows` rows, parallel over candidates; returns
    (expr*row/s, seconds[, values])."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle as O
    O.lib()
    x64 = np.ascontiguousarray(x[:, :n_rows].astype(np.float64)).reshape(-1)
    y64 = y[:n_rows].astype(np.float64)
    sample = [f32_constants(t) for t in trees[:n_cand]]
    t0 = time.perf_counter()
    with cf.ThreadPoolExecutor(max_workers=threads) as ex:
        vals = list(ex.map(lambda t: O.score(t, x64, n_rows, x.shape[0], y64, O.SQUARED),
                           sample))
    dt = time.perf_counter() - t0
    if want_values:
        return n_cand * n_rows / dt, dt, np.asarray(vals)
    return n_cand * n_rows / dt, dt


def score_parity(pkg, trees, x, y, n_rows, oracle_vals):
    """Device scores of the oracle's sample (the first len(oracle_vals)
    programs on the first n_rows rows of the timed workload) against the
    oracle: the largest relative error over candidates finite in both, and
    how many candidates differ in their non-finite classification (device
    status != 0 against a non-finite oracle value)."""
    k = len(oracle_vals)
    xs = np.ascontiguousarray(x[:, :n_rows])
    ev = pkg.GpuEvaluator(xs.reshape(-1), n_rows, x.shape[0], np.ascontiguousarray(y[:n_rows]))
    prog, off = pkg.Population(trees[:k]).programs()
    vals, status, _ = ev.score_batch(prog, off, 0)
    ev.close()
    fin_cpu = np.isfinite(oracle_vals)
    fin_dev = np.asarray(status) == 0
    both = fin_cpu & fin_dev
    rel = np.abs(vals[both] - oracle_vals[both]) / np.maximum(np.abs(oracle_vals[both]), 1e-300)
    return {"checked": int(k), "rows": int(n_rows), "finite": int(both.sum()),
            "max_rel_err": float(rel.max()) if rel.size else 0.0,
            "nonfinite_mismatch": int((fin_cpu != fin_dev).sum()),
            "bar": "relative error <= 1e-4 (gpu.rs:3349-3369), identical non-finite class",
            "oracle": "f64 CPU restatement of expr::eval + metrics::score_weighted"}


def cpu_fit_sample(trees, x, y, N, n_rows, n_cand, threads, metric=0, kind="fit", iters=20):
    """The oracle's CPU fit (fit_weighted_metric: fit_lm, or irls_fit for the
    absolute metric; implicit::fit for kind="implicit") of the first `n_cand`
    candidates on the first `n_rows` rows, parallel over candidates; the rate
    in candidates/s is scaled linearly in rows to the full N."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle as O
    O.lib()
    v = x.shape[0]
    x64 = np.ascontiguousarray(np.asarray(x, np.float64)[:, :n_rows]).reshape(-1)
    y64 = None if y is None else np.ascontiguousarray(np.asarray(y, np.float64)[:n_rows])
    sample = trees[:n_cand]
    if kind == "implicit":
        fn = lambda t: O.implicit_fit(t, x64, n_rows, v, iters)  # noqa: E731
    else:
        om = {0: O.SQUARED, 4: O.ABSOLUTE, 1: O.LOG_SQUASHED}[metric]
        fn = lambda t: O.fit(t, x64, n_rows, v, y64, iters, om)  # noqa: E731
    t0 = time.perf_counter()
    with cf.ThreadPoolExecutor(max_workers=threads) as ex:
        list(ex.map(fn, sample))
    dt = time.perf_counter() - t0
    return {"value": n_cand / dt * n_rows / N, "unit": "candidates/s", "cores": threads,
            "kind": "port", "cpu_model": cpu_model(),
            "sample": f"the first {n_cand} candidates x the first {n_rows} rows, {iters} "
                      f"iterations, f64 oracle, rate scaled linearly in rows to N={N}"}


def cpu_fit_baseline(trees, x, y, n_rows, n_cand, iters, threads):
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle as O
    O.lib()
    x64 = np.ascontiguousarray(x[:, :n_rows]).reshape(-1)
    y64 = y[:n_rows]
    sample = trees[:n_cand]
    t0 = time.perf_counter()
    with cf.ThreadPoolExecutor(max_workers=threads) as ex:
        list(ex.map(lambda t: O.fit(t, x64, n_rows, x.shape[0], y64, iters), sample))
    dt = time.perf_counter() - t0
    # per-candidate cost grows linearly in rows: scale to the full row count
    return n_cand / dt, dt


def bench_refit(pkg, W, P=16, N=1 << 18, iters=20, port_sample=2):
    """The exact f64 finalist refit on the host cores (host/refit.cpp): P
    finalists of the fit workload's tree distribution at N rows x 8 features,
    `iters` LM iterations, squared error, all host threads; beside it the
    oracle's row-at-a-time restatement of the reference's refit (the port),
    single-threaded on the first `port_sample` finalists, with the product's
    own single-thread time on the same sample and a bit-for-bit comparison of
    the two on it."""
    trees, x, y = W.fit_workload(P, N, seed=7)
    v = x.shape[0]
    x64 = np.ascontiguousarray(x, np.float64).reshape(-1)
    y64 = np.ascontiguousarray(y, np.float64)
    threads = os.cpu_count() or 1
    warm = np.ascontiguousarray(x64.reshape(v, N)[:, :4096]).reshape(-1)
    pkg.refit_finalists_exact(trees[:1], warm, y64[:4096], 2)
    t0 = time.perf_counter()
    loss, _ = pkg.refit_finalists_exact(trees, x64, y64, iters, "squared", threads=threads)
    dt = time.perf_counter() - t0
    sample = trees[:port_sample]
    t0 = time.perf_counter()
    own, _ = pkg.refit_finalists_exact(sample, x64, y64, iters, "squared", threads=1)
    dt1 = time.perf_counter() - t0
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle as O
    O.lib()
    t0 = time.perf_counter()
    port = [O.fit(t, x64, N, v, y64, iters)[0] for t in sample]
    dtp = time.perf_counter() - t0
    same = bool(np.array_equal(np.asarray(port, np.float64).view(np.uint64),
                               own.view(np.uint64)))
    return {"metric": "refit_finalists_per_s", "value": P / dt, "unit": "finalists/s",
            "threads": threads, "s": dt, "value_1_thread": port_sample / dt1,
            "config": {"workload": f"exact f64 finalist refit, {P} finalists of the fit "
                                   f"workload's trees, N={N} rows x {v} features, {iters} LM "
                                   f"iterations, squared error"},
            "cpu_baseline": {"value": port_sample / dtp, "unit": "finalists/s", "cores": 1,
                             "kind": "port", "cpu_model": cpu_model(),
                             "sample": f"the first {port_sample} finalists, row-at-a-time "
                                       f"f64 oracle, one thread"},
            "same_bits_as_port": same}


# ---------------------------------------------------------------------------

def run_reference(args, rank, world):
    """The reference arm: the reference's CPU path (its f64 restatement; the
    Rust reference cannot be built here) on all host threads, on a bounded
    sample of this arm's workload per step."""
    if rank != 0:
        return
    W = importlib.import_module(PKG + ".workloads")
    threads = os.cpu_count() or 1
    if args.workload == "score":
        # the repo arm's workload (seed 0): its first programs and rows
        P, N = args.P or 4096, args.N or (1 << 20)
        trees, x, y = W.scoring_workload(P, N, seed=0)
        n_rows, n_cand = SCORE_SAMPLE_ROWS, SCORE_SAMPLE_PROGS
        metric, unit = "expr_row_evals_per_s", "expr*row/s"
        fn = lambda: cpu_score_baseline(trees, x, y, n_rows, n_cand, threads)  # noqa: E731
        sample = (f"the first {n_cand} programs x the first {n_rows} rows of the P={P}, N={N} "
                  f"workload per step")
        cfg = {"workload": f"batched scoring, P={P} programs, N={N} rows x 5 features, "
                           f"squared error", "l2": "flushed between steps"}
    else:
        P, N = args.P or 2048, args.N or 262144
        trees, x, y = W.fit_workload(P, N, seed=0)
        n_rows, n_cand = 1 << 14, 16
        metric, unit = "fitted_candidates_per_s", "candidates/s"

        def fn():
            v, dt = cpu_fit_baseline(trees, x, y, n_rows, n_cand, 20, threads)
            return v * n_rows / float(N), dt
        sample = (f"the first {n_cand} candidates x the first {n_rows} rows x 20 LM iterations "
                  f"per step, scaled linearly to N={N}")
        cfg = {"workload": f"batched LM fit (squared), P={P}, N={N} rows x 8 features, 20 "
                           f"iters, fused adjoint", "l2": "flushed between steps"}
    for _ in range(args.warmup):
        fn()
    vals, total = [], 0.0
    for _ in range(args.steps):
        v, dt = fn()
        vals.append(v)
        total += dt
    value = float(np.mean(vals))
    line = {"impl": "reference", "metric": metric, "value": value, "unit": unit,
            "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": 1e3 * total / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": cfg,
            "cpu_baseline": {"value": value, "unit": unit, "cores": threads, "kind": "port",
                             "cpu_model": cpu_model(), "sample": sample},
            "e2e": {"value": value, "unit": unit, "h2d_bytes_per_step": 0,
                    "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def bench_score(args, rank, world, dev, pkg, W, flushbuf):
    P, N, V = args.P or 4096, args.N or (1 << 20), 5
    trees, x, y = W.scoring_workload(P, N, seed=rank)
    ev = pkg.GpuEvaluator(x.reshape(-1), N, V, y)
    pop = pkg.Population(trees)
    prog, off = pop.programs()
    assert len(pop) == P
    ops = postfix_ops(prog, off)
    alg_ops = float(N) * float((ops + 2).sum())      # lane-ops per launch
    pcount = np.zeros(P, np.int32)
    # the scorer's autotuner (candidates per work item, per length bucket)
    # on this batch, before and outside the timed steps; a candidate's score
    # does not depend on the choice
    ev.autotune(prog, off)
    # warm-up
    for _ in range(args.warmup):
        ev.score_batch(prog, off, 0, pcount)
    dev_ms, wall, prof = [], [], []
    import torch
    torch.cuda.synchronize()
    n0 = ev.launch_count()
    with ClockSampler(int(os.environ.get("LOCAL_RANK", 0))) as clk:
        for _ in range(args.steps):
            flush_l2(flushbuf)
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            vals, status, ms = ev.score_batch(prog, off, 0, pcount)
            wall.append(time.perf_counter() - t0)
            dev_ms.append(ms)
            prof.append(ev.score_profile())
    launches = ev.launch_count() - n0
    stats = ev.last_stats()
    clocks = clk.summary()
    extra = score_plain_and_absolute(ev, prog, off, pcount, vals, N, flushbuf, seed=rank)
    ev.close()
    h2d = int(prog.nbytes + off.nbytes + pcount.nbytes)
    d2h = int(P * (8 + 4))
    finite = np.asarray(status) == 0
    return dict(P=P, N=N, dev_ms=dev_ms, wall=wall, alg_ops=alg_ops, clocks=clocks,
                h2d=h2d, d2h=d2h, trees=trees, x=x, y=y, stats=stats, prof=prof,
                launches=launches, unit_count=float(P) * N,
                finite=int(finite.sum()), alg_ops_finite=float(N) * float((ops[finite] + 2).sum()),
                **extra)


def score_plain_and_absolute(ev, prog, off, pcount, vals, N, flushbuf, seed, sample=64,
                             abs_steps=3):
    """Outside the timed region, the two other forms the scoring
    configuration names: the plain form, one program per scoring call (one
    launch sequence each) on a seeded random sample of the batch, whose
    scores must equal the batched ones; and the batched form under absolute
    error (L2 flushed before each call)."""
    import torch
    P = len(off) - 1
    rng = np.random.Generator(np.random.PCG64(seed + 77))
    pick = np.sort(rng.choice(P, size=min(sample, P), replace=False))
    ms_plain, same = 0.0, True
    for i in pick:
        one = np.ascontiguousarray(prog[off[i]:off[i + 1]])
        o1 = np.array([0, len(one)], np.uint32)
        ev.score_batch(one, o1, 0, pcount[i:i + 1])  # its own warm-up
        flush_l2(flushbuf)
        torch.cuda.synchronize()
        v1, _, ms = ev.score_batch(one, o1, 0, pcount[i:i + 1])
        ms_plain += ms
        same = same and bool(np.array_equal(np.asarray(v1).view(np.uint64),
                                            np.asarray(vals)[i:i + 1].view(np.uint64)))
    plain = float(len(pick)) * N / (ms_plain / 1e3)
    ev.score_batch(prog, off, 1, pcount)
    ms_abs = []
    for _ in range(abs_steps):
        flush_l2(flushbuf)
        torch.cuda.synchronize()
        ms_abs.append(ev.score_batch(prog, off, 1, pcount)[2])
    absolute = float(P) * N / (float(np.mean(ms_abs)) / 1e3)
    return {"plain": {"value": plain, "unit": "expr*row/s", "same_scores": same,
                      "sample": f"{len(pick)} programs drawn at random (seeded) from the batch, "
                                "one scoring call each"},
            "absolute": {"value": absolute, "unit": "expr*row/s", "steps": abs_steps,
                         "config": "the same batch and rows, absolute error"}}


def fit_lane_ops(plans, sweeps, N, metric):
    """Algorithmic work of one fit in FP32-lane-op equivalents, from the
    sweeps each candidate actually ran (the device's per-candidate counts):
    per row, an f32 assembly is the forward (L) and reverse (2.5 L) sweeps
    plus G = p(p+1)/2 + p + 1 f64 FMAs of the Gram fold (each counted twice:
    FP64 issues at half the FP32 rate), an f32 objective sweep L + 2, and the
    f64 sweeps the same work at twice the cost; the implicit Jacobian is four
    passes (7 L) plus G, its cost sweep the forward and input adjoint (3.5 L)
    plus the norm and the division. L = the candidate's records."""
    tot = 0.0
    for pl, sw in zip(plans, sweeps):
        L = len(pl.words) / 4.0
        p = pl.nconst
        G = p * (p + 1) / 2.0 + p + 1 + (2 if metric in (2, 3) else 0) * (p + 2)
        a32, l32, a64, l64 = (float(q) for q in sw)
        if metric == 6:
            per = 2.0 * a64 * (7.0 * L + G) + 2.0 * l64 * (3.5 * L + 6.0)
        else:
            per = (a32 * (3.5 * L + 2.0 * G) + l32 * (L + 2.0) +
                   2.0 * a64 * (3.5 * L + G) + 2.0 * l64 * (L + 2.0))
        tot += per
    return tot * N


def fit_setup(pkg, W, case, P, N, seed):
    """The evaluator, fit plans and label of one fit configuration:
      c3:  1-20 constants, 5-60 nodes over N rows x 8 features ~U(-2,2),
           y = 1.7 exp(-x0^2/2) cos(2.3 x1) + 0.4 x2 + noise; squared error;
      c5:  1-20 constants over N rows x 10 heavy-tailed features,
           y = 0.8 x0/(1+x1^2) + log(1+|x3|) + 0.1 t3 noise; absolute error
           (L1 IRLS with true-MAE acceptance)."""
    if case == "c3":
        trees, x, y = W.fit_workload(P, N, seed=seed)
        metric, what = 0, f"batched LM fit (squared), P={P}, N={N} rows x 8 features, 20 iters"
    else:
        x, y = W.heavy_tail_data(N, seed=seed)
        trees, _, _ = W.fit_workload(P, 16, seed=7 + seed, nvars=10)
        metric = 4
        what = (f"batched L1 IRLS fit (absolute), P={P}, N={N} rows x 10 heavy-tailed "
                f"features, 20 iters")
    ev = pkg.GpuEvaluator(x.astype(np.float32).reshape(-1), N, x.shape[0], y.astype(np.float32))
    ev.set_fit_data(x.reshape(-1), y)
    plans = [pkg.gpu_fit_plan(t) for t in trees]
    return ev, plans, trees, x, y, metric, what


def time_fit(pkg, ev, plans, metric, N, steps, warmup, flushbuf, plain_n, seed, tune=True):
    """Fused fits of the whole batch (graph-replayed), timed per step on the
    device and end to end; then the plain one-candidate-per-launch form on a
    seeded random sample of the same candidates (its cost is linear in the
    candidate count), whose losses must equal the fused ones bit for bit.
    With `tune`, before timing (and outside it), the library's fit autotuner
    chooses the assembly budget per length bucket on this batch
    (`rc_fit_autotune`, which keeps the built-in budgets unless the whole
    batch is faster with its choice); both arms then run with that table."""
    import torch
    iters = 20
    P = len(plans)
    # sample 0: a tuning batch of about 16,384 (candidate, tile) items per bucket
    budgets = ev.fit_autotune(plans, iters, metric, sample=0) if tune else None
    prog, off, pcount, c0, gauge, kmax = pkg.pack_plans(plans)
    for _ in range(warmup):
        ev.fit_batch_fused(prog, off, pcount, c0, gauge, kmax, iters, metric)
    dev_ms, wall = [], []
    n0 = ev.launch_count()
    with ClockSampler(int(os.environ.get("LOCAL_RANK", 0))) as clk:
        for _ in range(steps):
            flush_l2(flushbuf)
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            _, loss, st, ms = ev.fit_batch_fused(prog, off, pcount, c0, gauge, kmax, iters,
                                                 metric)
            wall.append(time.perf_counter() - t0)
            dev_ms.append(ms)
    launches = ev.launch_count() - n0
    sweeps = ev.fit_sweeps(P)
    out = dict(P=P, N=N, dev_ms=dev_ms, wall=wall, clocks=clk.summary(), launches=launches,
               unit_count=float(P), status=np.bincount(st, minlength=9).tolist(),
               h2d=int(prog.nbytes + off.nbytes + pcount.nbytes + c0.nbytes + gauge.nbytes),
               d2h=int(P * (kmax * 8 + 8 + 4)), loss=loss, status_list=st,
               sweeps_mean=sweeps.mean(0).tolist(), fit_budgets_kb=budgets,
               lane_ops=fit_lane_ops(plans, sweeps, N, metric))
    if plain_n:
        rng = np.random.Generator(np.random.PCG64(seed + 77))
        idx = np.sort(rng.choice(P, size=min(plain_n, P), replace=False))
        sp, so, spc, sc0, sg, _ = pkg.pack_plans([plans[i] for i in idx], kmax)
        w = pkg.pack_plans([plans[i] for i in idx[:2]], kmax)
        ev.fit_batch_plain(w[0], w[1], w[2], w[3], w[4], kmax, iters, metric)
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        _, ploss, pst, pms = ev.fit_batch_plain(sp, so, spc, sc0, sg, kmax, iters, metric)
        pwall = time.perf_counter() - t0
        out["plain"] = {"value": len(idx) / (pms / 1e3), "unit": "candidates/s",
                        "sample": f"{len(idx)} candidates drawn at random (seeded) from the "
                                  f"batch, one launch sequence each",
                        "e2e": len(idx) / pwall,
                        "same_losses": bool(np.array_equal(ploss.view(np.uint64),
                                                           loss[idx].view(np.uint64)))}
    return out


def fit_summary(r, peaks, what):
    """The fit block of a JSON line."""
    fv = r["unit_count"] * len(r["dev_ms"]) / (sum(r["dev_ms"]) / 1e3)
    d = {"metric": "fitted_candidates_per_s", "value": fv, "unit": "candidates/s",
         "e2e": r["unit_count"] * len(r["wall"]) / sum(r["wall"]),
         "ms_per_step": float(np.mean(r["dev_ms"])), "steps": len(r["dev_ms"]),
         "config": what, "gpu_launches": r["launches"], "status_histogram": r["status"],
         "sweeps_per_candidate": r["sweeps_mean"], "fit_budgets_kb": r.get("fit_budgets_kb"),
         "clocks": r["clocks"]}
    for k in ("status_histogram_reference_mode", "status57_classified", "cpu_baseline"):
        if k in r:
            d[k] = r[k]
    if "plain" in r:
        d["plain"] = r["plain"]
        d["fused_over_plain"] = fv / r["plain"]["value"]
    d["roofline"] = fit_roofline(r, peaks)
    return d


def fit_reference_mode(pkg, ev, plans, metric, trees, x, y, r, threads):
    """The same batch once more with the f64 rescue off (flags bit 1: the
    reference kernel's behaviour, stopping at an f32-only failure), untimed;
    every status 5 / 7 of either run is classified on the CPU: `f32_only` when
    the oracle's f64 normal equations (fit.rs:1774-1827) are finite at the
    returned constants, `genuine` otherwise."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle as O
    O.lib()
    prog, off, pcount, c0, gauge, kmax = pkg.pack_plans(plans)
    c_ref, _, st_ref, _ = ev.fit_batch_fused(prog, off, pcount, c0, gauge, kmax, 20, metric, 2)
    c_res, _, st_res, _ = ev.fit_batch_fused(prog, off, pcount, c0, gauge, kmax, 20, metric, 0)
    v, n = x.shape
    cols = np.ascontiguousarray(x, np.float64).reshape(-1)
    y64 = np.ascontiguousarray(y, np.float64)

    def classify(args):
        k, cc = args
        at = plans[k].apply(trees[k], cc[k][: plans[k].nconst])
        return "f32_only" if O.normal_equations_ok(at, cols, n, v, y64) else "genuine"

    out = {}
    for tag, cc, st in (("rescue_on", c_res, st_res), ("reference_mode", c_ref, st_ref)):
        ks = [k for k in range(len(plans)) if st[k] in (5, 7)]
        with cf.ThreadPoolExecutor(threads) as ex:
            cls = list(ex.map(classify, [(k, cc) for k in ks]))
        out[tag] = {"f32_only": cls.count("f32_only"), "genuine": cls.count("genuine")}
    r["status_histogram_reference_mode"] = np.bincount(st_ref, minlength=9).tolist()
    r["status57_classified"] = out
    return out


def bench_fit(args, rank, world, dev, pkg, W, flushbuf, steps=None, warmup=None, plain=True,
              N=None, classify=False, cpu=False, tune=True):
    P = args.P if args.workload == "fit" and args.P else 2048
    N = N or (args.N if args.workload == "fit" and args.N else 262144)
    steps = args.steps if steps is None else steps
    warmup = args.warmup if warmup is None else warmup
    ev, plans, trees, x, y, metric, what = fit_setup(pkg, W, "c3", P, N, rank)
    out = time_fit(pkg, ev, plans, metric, N, steps, warmup, flushbuf, 64 if plain else 0, rank,
                   tune=tune and not args.no_tune)
    threads = os.cpu_count() or 1
    if classify:
        fit_reference_mode(pkg, ev, plans, metric, trees, x, y, out, threads)
    ev.close()
    if cpu and not args.no_cpu_baseline:
        out["cpu_baseline"] = cpu_fit_sample(trees, x, y, N, 1 << 14, 16, threads)
    out.update(trees=trees, x=x, y=y, what=what)
    return out


def bench_implicit(args, rank, pkg, W, flushbuf, steps, warmup, fit_steps, fit_warmup):
    """The implicit metric (P = 1024 candidates of f(x, y, d1, d2) on a noisy
    unit circle with two distractors, length 3-40, 0-6 constants;
    N = 1,048,576 rows): scoring |f|/||grad f|| through the fused input
    adjoint (candidate*rows/s), and the LM fit of the candidates that hold
    constants."""
    import torch
    P = args.P if args.workload == "implicit" and args.P else 1024
    N = args.N if args.workload == "implicit" and args.N else 1 << 20
    trees, cols = W.implicit_workload(P, N, seed=rank)
    ev = pkg.GpuEvaluator(cols.astype(np.float32).reshape(-1), N, 4, np.zeros(N, np.float32))
    ev.set_fit_data(cols.reshape(-1), np.zeros(N))
    splans = [pkg.gpu_fit_plan(t, allow_no_constants=True) for t in trees]
    prog, off, pcount, c0, gauge, kmax = pkg.pack_plans(splans)
    for _ in range(warmup):
        ev.implicit_score(prog, off, pcount, c0, kmax)
    dev_ms, wall = [], []
    n0 = ev.launch_count()
    for _ in range(steps):
        flush_l2(flushbuf)
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        vals, status, ms = ev.implicit_score(prog, off, pcount, c0, kmax)
        wall.append(time.perf_counter() - t0)
        dev_ms.append(ms)
    rows = float(P) * N
    peaks = load_peaks()
    peak = 148 * 128 * peaks.get("sm_max_mhz", 1965.0) * 1e6 / 1e9
    fin = np.asarray(status) == 0
    # U_grad per candidate*row: forward L, input adjoint 2.5 L, the norm of
    # the 4-input gradient and the division
    ugrad = float(N) * sum(3.5 * len(pl.words) / 4.0 + 4.0 + 2.0
                           for pl, f in zip(splans, fin) if f)
    per = float(np.mean(dev_ms)) / 1e3
    score = {"metric": "implicit_score_candidate_rows_per_s",
             "value": rows * steps / (sum(dev_ms) / 1e3), "unit": "candidate*row/s",
             "e2e": rows * steps / sum(wall), "ms_per_step": float(np.mean(dev_ms)),
             "gpu_launches": ev.launch_count() - n0,
             "finite_candidates": int(fin.sum()),
             "roofline": {"bound": "fp32_issue", "achieved": ugrad / per / 1e9, "peak": peak,
                          "unit": "Glane-op/s", "frac": ugrad / per / 1e9 / peak,
                          "traffic": None,
                          "note": "finite candidates x N x (3.5 L + 4 + 2) lane-ops (forward, "
                                  "input adjoint, gradient norm, division; L = records) / "
                                  "event time of the scoring call; infeasible candidates stop "
                                  "at their first bad row and are not counted"},
             "config": f"implicit |f|/||grad f|| scoring, P={P}, N={N} rows x 4 inputs"}
    fplans = [pkg.gpu_fit_plan(t) for t in trees if t.constants()]
    ftrees = [t for t in trees if t.constants()]
    # the implicit sweeps' shapes do not depend on the assembly budget
    fit = time_fit(pkg, ev, fplans, 6, N, fit_steps, fit_warmup, flushbuf, 16, rank, tune=False)
    ev.close()
    if not args.no_cpu_baseline:
        threads = os.cpu_count() or 1
        sys.path.insert(0, os.path.join(ROOT, "oracle"))
        import oracle as O
        O.lib()
        nr, nc = 1 << 16, 64
        c64 = np.ascontiguousarray(cols[:, :nr]).reshape(-1)
        t0 = time.perf_counter()
        with cf.ThreadPoolExecutor(threads) as ex:
            list(ex.map(lambda t: O.implicit_score(t, c64, nr, 4), trees[:nc]))
        dt = time.perf_counter() - t0
        score["cpu_baseline"] = {"value": nc * nr / dt, "unit": "candidate*row/s",
                                 "cores": threads, "kind": "port", "cpu_model": cpu_model(),
                                 "sample": f"the first {nc} candidates x the first {nr} rows, "
                                           f"implicit::score restated in f64"}
        fit["cpu_baseline"] = cpu_fit_sample(ftrees, cols, None, N, 1 << 14, 16, threads,
                                             kind="implicit")
    what = (f"implicit |f|/||grad f|| LM fit (exact Jacobian from the input adjoint), the "
            f"{fit['P']} of P={P} candidates with constants, N={N} rows, 20 iters")
    return score, fit, what


def rank_stage(pkg, ev, plans, N, flushbuf, steps, warmup):
    """Exact rank sums of every plan's predictions against the resident
    target: candidate*rows/s and the HBM roofline of 32 algorithmic bytes per
    candidate*row."""
    import torch
    P = len(plans)
    # one call holds at most 2^31 - 1 candidate*rows (the ABI's limit, as in
    # the reference); larger batches go in chunks, as its binding does
    per_call = max(1, 0x7FFFFFFF // N)
    chunks = [pkg.pack_plans(plans[s:s + per_call]) for s in range(0, P, per_call)]

    fb = [0]

    def run():
        ms, st = 0.0, []
        fb[0] = 0
        for cp, co, cc, c0_, _, km in chunks:
            _, s, _, m = ev.rank_sums(cp, co, cc, c0_, km)
            ms += m
            st.append(s)
            fb[0] += ev.rank_fallbacks()
        return np.concatenate(st), ms

    ev.rank_target()
    for _ in range(warmup):
        run()
    dev_ms, wall = [], []
    n0 = ev.launch_count()
    for _ in range(steps):
        flush_l2(flushbuf)
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        status, ms = run()
        wall.append(time.perf_counter() - t0)
        dev_ms.append(ms)
    launches = ev.launch_count() - n0
    fallbacks = fb[0]
    # the same calls through the eight-pass radix sort (the bucketed sums'
    # fallback), timed beside them; the sums must be the same bits
    sums_b = [sm for cp, co, cc, c0_, _, km in chunks[:1]
              for sm in ev.rank_sums(cp, co, cc, c0_, km)[0]]
    ev.rank_tuning(-1, 0)
    radix_ms = []
    for k in range(2):
        flush_l2(flushbuf)
        torch.cuda.synchronize()
        radix_ms.append(run()[1])
    sums_r = [sm for cp, co, cc, c0_, _, km in chunks[:1]
              for sm in ev.rank_sums(cp, co, cc, c0_, km)[0]]
    ev.rank_tuning(0, 0)
    rows = float(P) * N
    per = float(np.mean(dev_ms)) / 1e3
    achieved = 32.0 * rows / per / 1e9
    peak = load_peaks().get("hbm_gbs", 6650.0)
    return {"metric": "rank_candidate_rows_per_s", "value": rows / per, "unit": "candidate*row/s",
            "e2e": rows * steps / sum(wall), "ms_per_step": 1e3 * per, "launches": launches,
            "h2d": int(sum(c[0].nbytes + c[1].nbytes + c[2].nbytes + c[3].nbytes
                           for c in chunks)),
            "d2h": int(P * (4 * 8 + 4) + 16 * len(chunks)), "calls_per_step": len(chunks),
            "finite_segments": int((status == 0).sum()),
            "method": "bucketed sums (sample splitters, one scatter, per-bucket ranking)",
            "radix_fallback_segments": fallbacks,
            "radix_sort_ms_per_step": float(np.median(radix_ms)),
            "bucketed_over_radix": float(np.median(radix_ms)) / (1e3 * per),
            "same_sums_as_radix": sums_b == sums_r,
            "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                         "frac": achieved / peak, "traffic": RANK_TRAFFIC,
                         "note": "algorithmic 32 B per candidate*row (f64 eval, 8 B key, 4 B "
                                 "row, read back, 8 B gathered target rank) / event time; "
                                 "peak = measured copy bandwidth (MEASURED_PEAKS.json)"}}


def bench_rank(args, rank, pkg, W, flushbuf, steps, warmup):
    """Exact rank sums of P fit-style candidates (default 64) over N rows
    (default 1,048,576) x 10 heavy-tailed features."""
    P = args.P if args.workload == "rank" and args.P else 64
    N = args.N if args.workload == "rank" and args.N else 1 << 20
    x, y = W.heavy_tail_data(N, seed=rank)
    trees, _, _ = W.fit_workload(P, 16, seed=100 + rank, nvars=10)
    ev = pkg.GpuEvaluator(x.astype(np.float32).reshape(-1), N, 10, y.astype(np.float32))
    ev.set_fit_data(x.reshape(-1), y)
    r = rank_stage(pkg, ev, [pkg.gpu_fit_plan(t) for t in trees], N, flushbuf, steps, warmup)
    ev.close()
    r["config"] = f"exact rank sums, P={P} candidates x 1 trial, N={N} rows x 10 features"
    return r


def bench_c5(args, rank, pkg, W, flushbuf, steps, warmup, fit_steps, fit_warmup):
    """The heavy-tailed configuration (N = 4,194,304 rows x 10 features, one
    island's generation of P = 1000 candidates): the L1 IRLS fit and the exact
    rank-correlation sums of the same candidates."""
    P = args.P if args.workload == "c5" and args.P else 1000
    N = args.N if args.workload == "c5" and args.N else 1 << 22
    ev, plans, trees, x, y, metric, what = fit_setup(pkg, W, "c5", P, N, rank)
    # tuning at 4M rows takes minutes of whole-batch checks: built-in budgets here
    fit = time_fit(pkg, ev, plans, metric, N, fit_steps, fit_warmup, flushbuf, 16, rank,
                   tune=False)
    rk = rank_stage(pkg, ev, plans, N, flushbuf, steps, warmup)
    rk["config"] = (f"exact rank-correlation sums, P={P} candidates x 1 trial, N={N} rows x "
                    f"10 heavy-tailed features")
    ev.close()
    if not args.no_cpu_baseline:
        threads = os.cpu_count() or 1
        fit["cpu_baseline"] = cpu_fit_sample(trees, x, y, N, 1 << 14, 16, threads, metric=4)
        rk["cpu_baseline"] = cpu_rank_sample(trees, x, y, 4, threads)
    return fit, what, rk


def cpu_rank_sample(trees, x, y, n_cand, threads):
    """The oracle's exact rank sums (expr::eval predictions, then
    RankTarget::sums: sort, average ranks, i128 sums) of the first `n_cand`
    candidates over all rows, parallel over candidates: candidate*rows/s."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle as O
    O.lib()
    v, n = x.shape
    cols = np.ascontiguousarray(x, np.float64).reshape(-1)
    y64 = np.ascontiguousarray(y, np.float64)
    t0 = time.perf_counter()
    with cf.ThreadPoolExecutor(threads) as ex:
        list(ex.map(lambda t: O.rank_sums(O.predict(t, cols, n, v), y64), trees[:n_cand]))
    dt = time.perf_counter() - t0
    return {"value": n_cand * float(n) / dt, "unit": "candidate*row/s", "cores": threads,
            "kind": "port", "cpu_model": cpu_model(),
            "sample": f"the first {n_cand} candidates over all {n} rows, f64 oracle "
                      f"(expr::eval + RankTarget::sums)"}


def bench_vary(args, rank, pkg, flushbuf, steps, warmup):
    """One generation of the device variation (rc_pool_vary): 16 islands x
    1000 slots of width 64 (max complexity 30, 10 inputs, the default
    operator set), parents drawn as the reference's tests draw them, seeded
    errors. children/s from the library's events around the call, e2e from
    the wall clock of the call with host buffers (errors in; lengths, node
    counts, hashes, errors and the child programs out; pinned and reused
    across generations, as a generation loop would keep them), beside the
    CPU restatement of the reference engine on one thread."""
    islands = args.P if args.workload == "vary" and args.P else 16
    pop, width, nvars, mc = 1000, 64, 10, 30
    n = islands * pop
    ops = pkg.DEFAULT_VARIATION_OPS
    err = np.array([((i * 7919) % 10007) / 10007.0 for i in range(n)])
    x = np.linspace(-1.0, 1.0, 64, dtype=np.float32)
    ev = pkg.GpuEvaluator(np.stack([x, x]).reshape(-1), 64, 2, x)
    pool = pkg.GenomePool(ev, islands, pop, width)
    # parents: a restarted (random) population built by the device into pool 1
    seed_words = np.full((n, width), 255, np.uint32)
    seed_words[:, 0], seed_words[:, 1] = 1, 0
    pool.upload(0, seed_words)
    words = pool.vary(0, err, 0, nvars, mc, 5 + rank, ops, restart=[1] * islands)[0]
    import torch

    def pinned(count, dt):
        b = torch.empty(count * np.dtype(dt).itemsize, dtype=torch.uint8, pin_memory=True)
        return b.numpy().view(dt)

    err_h = pinned(n, np.float64)
    err_h[:] = err
    outbuf = (pinned(n * width, np.uint32), pinned(n, np.uint16), pinned(n, np.uint16),
              pinned(n, np.uint64), pinned(n, np.float64))
    for g in range(warmup):
        pool.vary(1, err_h, 1 + g, nvars, mc, 77, ops, out=outbuf)
    dev_ms, wall = [], []
    n0 = ev.launch_count()
    for g in range(steps):
        flush_l2(flushbuf)
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        out = pool.vary(1, err_h, 1 + g, nvars, mc, 77, ops, out=outbuf)
        wall.append(time.perf_counter() - t0)
        dev_ms.append(out[5])
    launches = ev.launch_count() - n0
    # the CPU baseline and checker: the reference engine restated on the CPU
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle as O
    t0 = time.perf_counter()
    ref = O.next_generation(words, err, islands, pop, width, nvars, mc, 77, steps, ops)
    cpu_s = time.perf_counter() - t0
    same = bool(np.array_equal(out[0], ref[0]) and np.array_equal(out[3], ref[3]))
    ev.close()
    n = float(n)
    per = float(np.mean(dev_ms)) / 1e3
    return {"metric": "children_per_s", "value": n / per, "unit": "children/s",
            "e2e": n * steps / sum(wall), "ms_per_step": 1e3 * per, "launches": launches,
            "h2d": int(err.nbytes), "d2h": int(n * (2 + 2 + 8 + 8 + 4 * width)),
            "same_as_cpu": same,
            "cpu_baseline": {"value": n / cpu_s, "unit": "children/s", "cores": 1,
                             "kind": "port",
                             "sample": "the last timed generation, CPU restatement of the "
                                       "reference engine (sequential, as the reference)"},
            "config": f"device variation, {islands} islands x {pop} slots, width {width}, "
                      f"max complexity {mc}, {nvars} inputs, default operator set, dedup on"}


def oracle_fit_agreement(records, cols, n, v, y, iters, threads, metric=0, refit=False):
    """The device answers of a generation loop's fitted candidates against the
    oracle's CPU fit of the same candidates on the same rows: the share whose
    device loss (the oracle's exact objective at the device's constants) is
    within 1e-6 relative of the CPU fit's or below it; with `refit`, also the
    share after the caller's path (the device answer through the exactness
    gate, fit::gpu::fit_batch_verified, then the CPU finalist refit from the
    gated constants)."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle as O
    O.lib()
    om = {0: O.SQUARED, 4: O.ABSOLUTE}[metric]

    def one(r):
        cpu, _ = O.fit(r.tree, cols, n, v, y, iters, om)
        dev = (O.flat_sse(r.fitted(), cols, n, v, y) if metric == 0
               else O.score(r.fitted(), cols, n, v, y, om))
        final = np.nan
        if refit:
            usable = r.status in (0, 4, 5, 6, 7, 8) and np.all(np.isfinite(r.c[: r.plan.nconst]))
            proposal = O.flat_constants(r.fitted()) if usable else None
            _, gtree, _ = O.fit_verified(r.tree, cols, n, v, y, iters, proposal, om)
            final, _ = O.fit(gtree, cols, n, v, y, iters, om)
        return cpu, dev, r.status, final

    with cf.ThreadPoolExecutor(threads) as ex:
        res = list(ex.map(one, records))
    cpu = np.array([q[0] for q in res])
    dev = np.array([q[1] for q in res])
    st = np.array([q[2] for q in res], np.int64)
    ok = np.isin(st, [0, 4, 5, 6, 7, 8]) & np.isfinite(cpu)
    within = dev[ok] <= cpu[ok] * (1.0 + 1e-6) + 1e-300
    out = {"checked": int(len(res)), "usable_finite": int(ok.sum()),
           "within_1e-6_or_better": float(within.mean()) if ok.any() else None,
           "status_histogram": np.bincount(st, minlength=9).tolist()}
    if refit:
        final = np.array([q[3] for q in res])
        fin = np.isfinite(cpu)
        after = final[fin] <= cpu[fin] * (1.0 + 1e-6) + 1e-300
        out["within_1e-6_after_gate_and_refit"] = float(after.mean()) if fin.any() else None
    return out


def bench_c1(pkg, W, gens=200, sample_every=20):
    """The plain-method configuration through the build's own generation loop
    (seed 0, 10,000 rows, 80/20 split, 4 islands x 200, squared error, 8 LM
    iterations, max complexity 30): generations/s and fitted candidates/s end
    to end (device steps and the host bookkeeping between them), the device
    time of each step, and every `sample_every`-th generation's fitted
    candidates against the oracle's CPU fit."""
    x, y, _, _ = W.line_workload(10000, seed=0)
    n = x.shape[1]
    ev = pkg.GpuEvaluator(x.astype(np.float32).reshape(-1), n, 1, y.astype(np.float32))
    ev.set_fit_data(x.reshape(-1), y)
    loop = pkg.GenerationLoop(ev, 4, 200, 1, max_complexity=30, fit_iters=8, seed=0)
    sample, nfit = [], 0
    t0 = time.perf_counter()
    for g in range(gens):
        recs, err = loop.generation()
        nfit += len(recs)
        if g % sample_every == 0:
            sample += recs
    wall = time.perf_counter() - t0
    ev.close()
    agree = oracle_fit_agreement(sample, np.ascontiguousarray(x.reshape(-1)), n, 1, y, 8,
                                 os.cpu_count() or 1, refit=True)
    return {"generations_per_s": gens / wall, "fitted_candidates_per_s": nfit / wall,
            "generations": gens, "fitted_candidates": nfit, "wall_s": wall,
            "device_ms": loop.device_ms, "step_ms": loop.timing,
            "best_train_mse": float(np.nanmin(err)), "agreement": agree,
            "config": "plain-method search: seed 0, N=10000 (8000 train rows), x ~ U(-5,5), "
                      "y = 2x + 1 + N(0, 0.1^2), 4 islands x pop 200, 200 generations, squared "
                      "error, 8 LM iterations, max complexity 30"}


def bench_c5gen(args, pkg, W, agree=16):
    """One generation of the heavy-tailed configuration at its stated size:
    16 islands x pop 1000 over N = 4,194,304 rows x 10 features, absolute
    error (screen and rescore with the absolute score, L1 IRLS fit with up to
    20 constants, 20 iterations). At >= 2^20 rows every offspring with
    constants is admitted. Reports the device time of each step (screen, fit,
    rescore, vary) and the host time between them, the plain
    one-candidate-per-launch fit of 16 of the admitted candidates, and (with
    `agree`) a seeded sample of the fitted candidates against the oracle's
    CPU IRLS fit of the same candidates on the same rows."""
    islands = args.P or 16
    N = args.N or (1 << 22)
    x, y = W.heavy_tail_data(N, seed=0)
    ev = pkg.GpuEvaluator(x.astype(np.float32).reshape(-1), N, 10, y.astype(np.float32))
    ev.set_fit_data(x.reshape(-1), y)
    loop = pkg.GenerationLoop(ev, islands, 1000, 10, max_complexity=30, fit_iters=20, seed=5,
                              fit_metric=4, score_kind=1)
    t0 = time.perf_counter()
    recs, err = loop.generation()
    wall = time.perf_counter() - t0
    plans = [r.plan for r in recs[:16]]
    prog, off, pcount, c0, gauge, kmax = pkg.pack_plans(plans)
    _, _, _, pms = ev.fit_batch_plain(prog, off, pcount, c0, gauge, kmax, 20, 4)
    ev.close()
    fused = len(recs) / (loop.timing["fit"] / 1e3)
    plain = len(plans) / (pms / 1e3)
    out = {}
    if agree and recs:
        rng = np.random.Generator(np.random.PCG64(23))
        pick = [recs[i] for i in np.sort(rng.choice(len(recs), min(agree, len(recs)),
                                                     replace=False))]
        out["agreement"] = oracle_fit_agreement(pick, np.ascontiguousarray(x.reshape(-1)), N,
                                                10, y, 20, os.cpu_count() or 1, metric=4)
    return {"generation_s": wall, "admitted": len(recs), "step_ms": loop.timing, **out,
            "fit_fused": fused, "fit_plain": plain, "fused_over_plain": fused / plain,
            "status_histogram": np.bincount([r.status for r in recs], minlength=9).tolist(),
            "config": f"one generation, {islands} islands x pop 1000, N={N} rows x 10 "
                      f"heavy-tailed features, absolute error, L1 IRLS, 20 iterations"}


def fit_roofline(r, peaks):
    per = float(np.mean(r["dev_ms"])) / 1e3
    achieved = r["lane_ops"] / per / 1e9
    peak = 148 * 128 * peaks.get("sm_max_mhz", 1965.0) * 1e6 / 1e9
    return {"bound": "fp32_issue", "achieved": achieved, "peak": peak, "unit": "Glane-op/s",
            "frac": achieved / peak, "traffic": FIT_ASM_TRAFFIC,
            "note": "the sweeps each candidate ran (device counts) x N x their per-row "
                    "FP32-lane-op equivalents (f32 assembly 3.5 L + 2 G, f32 objective L + 2, "
                    "f64 sweeps twice the f32 cost; G = p(p+1)/2 + p + 1 FMAs of the Gram "
                    "fold), L = records, / CUDA-event time of the whole fused fit (the graph "
                    "of all its kernels); peak = 148 SMs x 128 FP32 lanes x sm_max_mhz "
                    "(MEASURED_PEAKS.json)"}


def _cpu(block):
    cb = block.get("cpu_baseline")
    return None if cb is None else cb["value"]


def secondary(args, rank, world, local, pkg, W, flushbuf, peaks, line):
    """The other configurations on the default line: nested blocks with the
    detail, and their headline numbers as top-level keys (so a record that
    keeps only top-level scalars still has them)."""
    f = bench_fit(args, rank, world, local, pkg, W, flushbuf, steps=3, warmup=3, classify=True,
                  cpu=True)
    fs = line["fit"] = fit_summary(f, peaks, f["what"])
    cls = fs.get("status57_classified", {})
    line.update(fit_fused=fs["value"], fit_fused_e2e=fs["e2e"],
                fit_plain=fs["plain"]["value"], fused_over_plain=fs["fused_over_plain"],
                fit_same_losses=fs["plain"]["same_losses"],
                fit_roofline_frac=fs["roofline"]["frac"], fit_cpu_baseline=_cpu(fs),
                fit_status_histogram=fs["status_histogram"],
                fit_status_histogram_reference_mode=fs.get("status_histogram_reference_mode"),
                fit_f32_only_failures=cls.get("rescue_on", {}).get("f32_only"),
                fit_f32_only_failures_reference_mode=cls.get("reference_mode", {}).get("f32_only"))
    f = bench_fit(args, rank, world, local, pkg, W, flushbuf, steps=2, warmup=3, N=1 << 20,
                  cpu=True, tune=False)
    fs = line["fit_1m"] = fit_summary(f, peaks, f["what"])
    line.update(fit_1m_fused=fs["value"], fit_1m_fused_e2e=fs["e2e"],
                fit_1m_plain=fs["plain"]["value"], fused_over_plain_1m=fs["fused_over_plain"],
                fit_1m_same_losses=fs["plain"]["same_losses"],
                fit_1m_roofline_frac=fs["roofline"]["frac"], fit_1m_cpu_baseline=_cpu(fs),
                fit_1m_status_histogram=fs["status_histogram"])
    del f
    score, fit, what = bench_implicit(args, rank, pkg, W, flushbuf, 3, 3, 1, 1)
    fs = fit_summary(fit, peaks, what)
    line["implicit"] = {"score": score, "fit": fs}
    line.update(implicit_score=score["value"], implicit_score_e2e=score["e2e"],
                implicit_score_roofline_frac=score["roofline"]["frac"],
                implicit_score_cpu_baseline=_cpu(score),
                implicit_fit_fused=fs["value"], implicit_fit_plain=fs["plain"]["value"],
                implicit_fused_over_plain=fs["fused_over_plain"],
                implicit_fit_roofline_frac=fs["roofline"]["frac"],
                implicit_fit_cpu_baseline=_cpu(fs))
    fit, what, rk = bench_c5(args, rank, pkg, W, flushbuf, 3, 3, 1, 1)
    fs = fit_summary(fit, peaks, what)
    line["c5"] = {"absolute_fit": fs, "rank": rk}
    line.update(c5_fit_fused=fs["value"], c5_fit_plain=fs["plain"]["value"],
                c5_fused_over_plain=fs["fused_over_plain"],
                c5_fit_roofline_frac=fs["roofline"]["frac"], c5_fit_cpu_baseline=_cpu(fs),
                c5_rank=rk["value"], c5_rank_e2e=rk["e2e"],
                c5_rank_roofline_frac=rk["roofline"]["frac"], c5_rank_cpu_baseline=_cpu(rk),
                c5_rank_bucketed_over_radix=rk["bucketed_over_radix"],
                c5_rank_same_sums_as_radix=rk["same_sums_as_radix"])
    c1 = line["c1"] = bench_c1(pkg, W)
    line.update(c1_generations_per_s=c1["generations_per_s"],
                c1_fitted_candidates_per_s=c1["fitted_candidates_per_s"],
                c1_agreement=c1["agreement"]["within_1e-6_or_better"],
                c1_agreement_after_refit=c1["agreement"].get("within_1e-6_after_gate_and_refit"))
    g5 = line["c5_generation"] = bench_c5gen(argparse.Namespace(P=0, N=0), pkg, W)
    line.update(c5gen_generation_s=g5["generation_s"], c5gen_fit_fused=g5["fit_fused"],
                c5gen_fused_over_plain=g5["fused_over_plain"],
                c5gen_agreement=g5.get("agreement", {}).get("within_1e-6_or_better"))
    vy = line["vary"] = bench_vary(args, rank, pkg, flushbuf, 5, 3)
    line.update(vary_children=vy["value"], vary_children_e2e=vy["e2e"],
                vary_same_as_cpu=vy["same_as_cpu"], vary_cpu_baseline=_cpu(vy))
    if not args.no_cpu_baseline:
        rf = line["refit"] = bench_refit(pkg, W)
        line.update(refit_finalists=rf["value"], refit_cpu_baseline=_cpu(rf),
                    refit_same_bits=rf["same_bits_as_port"])


def single_gpu_line(args, world, r, metric, unit, what, extra):
    """The JSON line of a one-GPU workload whose numbers come from a fit or
    rank block."""
    line = {"metric": metric, "value": r["value"], "unit": unit, "n_gpus": world,
            "steps": r.get("steps", args.steps), "warmup": args.warmup,
            "ms_per_step": r["ms_per_step"], "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32 rows, f64 sums", "data": "synthetic",
            "config": {"workload": what, "l2": "flushed between steps"},
            "roofline": r.get("roofline"), "clocks": r.get("clocks"),
            "e2e": {"value": r["e2e"], "unit": unit, "h2d_bytes_per_step": r.get("h2d"),
                    "d2h_bytes_per_step": r.get("d2h")},
            "gpu_launches": r.get("gpu_launches", r.get("launches"))}
    line.update(extra)
    return line


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="score",
                    choices=["score", "fit", "rank", "implicit", "c5", "vary", "refit", "c1",
                             "c5gen"])
    ap.add_argument("--P", type=int, default=0)
    ap.add_argument("--N", type=int, default=0)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-tune", action="store_true",
                    help="fit with the built-in assembly budgets instead of tuning them first")
    ap.add_argument("--no-secondary", action="store_true",
                    help="skip the fit, implicit and heavy-tailed measurements of the "
                         "default line")
    args = ap.parse_args()

    rank = int(os.environ.get("RANK", 0))
    world = int(os.environ.get("WORLD_SIZE", 1))
    if args.impl == "reference":
        return run_reference(args, rank, world)
    if args.workload == "refit":
        # host cores only: no device work
        if rank == 0:
            r = bench_refit(importlib.import_module(PKG),
                            importlib.import_module(PKG + ".workloads"),
                            P=args.P or 16, N=args.N or (1 << 18))
            print(json.dumps(r), flush=True)
        return

    import torch
    import torch.distributed as dist
    local = int(os.environ.get("LOCAL_RANK", 0))
    torch.cuda.set_device(local)
    if world > 1:
        import datetime
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    pkg = importlib.import_module(PKG)
    W = importlib.import_module(PKG + ".workloads")
    flushbuf = torch.empty(256 << 20, dtype=torch.uint8, device="cuda")
    peaks = load_peaks()

    if world > 1:
        dist.barrier()
    torch.cuda.synchronize()
    if args.workload in ("c1", "c5gen"):
        # the generation loop: one GPU, rank 0 reports
        r = bench_c1(pkg, W) if args.workload == "c1" else bench_c5gen(args, pkg, W)
        if rank == 0:
            print(json.dumps({"metric": "generation", "workload": args.workload, **r},
                             default=float), flush=True)
        if world > 1:
            dist.barrier()
            dist.destroy_process_group()
        return
    if args.workload in ("rank", "implicit", "c5", "vary"):
        # one-GPU stages: each rank measures its own copy; rank 0 reports
        if args.workload == "vary":
            r = bench_vary(args, rank, pkg, flushbuf, args.steps, args.warmup)
            line = single_gpu_line(args, world, r, r["metric"], r["unit"], r.pop("config"),
                                   {"dtype": "u32 words, integer", "cpu_baseline": r["cpu_baseline"],
                                    "same_as_cpu": r["same_as_cpu"]})
        elif args.workload == "rank":
            r = bench_rank(args, rank, pkg, W, flushbuf, args.steps, args.warmup)
            line = single_gpu_line(args, world, r, r["metric"], r["unit"], r.pop("config"),
                                   {"dtype": "f64 eval, integer sums"})
        elif args.workload == "implicit":
            score, fit, what = bench_implicit(args, rank, pkg, W, flushbuf, args.steps,
                                              args.warmup, args.steps, args.warmup)
            fs = fit_summary(fit, peaks, what)
            line = single_gpu_line(args, world, fs, fs["metric"], fs["unit"], what,
                                   {"dtype": "f64", "implicit_score": score,
                                    "plain": fs.get("plain"),
                                    "fused_over_plain": fs.get("fused_over_plain"),
                                    "fit_status_histogram": fs["status_histogram"]})
            line["h2d"] = fit["h2d"]
        else:
            fit, what, rk = bench_c5(args, rank, pkg, W, flushbuf, args.steps, args.warmup,
                                     args.steps, args.warmup)
            fs = fit_summary(fit, peaks, what)
            fs["h2d"], fs["d2h"] = fit["h2d"], fit["d2h"]
            line = single_gpu_line(args, world, fs, fs["metric"], fs["unit"], what,
                                   {"plain": fs.get("plain"),
                                    "fused_over_plain": fs.get("fused_over_plain"),
                                    "fit_status_histogram": fs["status_histogram"],
                                    "rank": rk})
        if rank == 0:
            print(json.dumps(line), flush=True)
        if world > 1:
            dist.barrier()
            dist.destroy_process_group()
        return
    if args.workload == "score":
        r = bench_score(args, rank, world, local, pkg, W, flushbuf)
    else:
        r = bench_fit(args, rank, world, local, pkg, W, flushbuf, plain=not args.no_secondary)
    torch.cuda.synchronize()

    dev_s = sum(r["dev_ms"]) / 1e3
    wall_s = sum(r["wall"])
    if world > 1:
        t = torch.tensor([dev_s, wall_s], dtype=torch.float64, device="cuda")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        dev_s, wall_s = float(t[0]), float(t[1])
        dist.barrier()
    units = r["unit_count"] * args.steps * world
    value = units / dev_s
    e2e = units / wall_s
    if rank == 0:
        if args.workload == "score":
            metric, unit = "expr_row_evals_per_s", "expr*row/s"
            pr = r["prof"]
            ms_f32 = float(np.mean([q["ms_f32"] for q in pr]))
            ops_f32 = float(np.mean([q["ops_f32"] for q in pr]))
            rows_f32 = float(np.mean([q["rows_f32"] for q in pr]))
            rows_f64 = float(np.mean([q["rows_f64"] for q in pr]))
            peak = 148 * 128 * peaks.get("sm_max_mhz", 1965.0) * 1e6 / 1e9
            achieved = ops_f32 / (ms_f32 / 1e3) / 1e9
            achieved_all = r["alg_ops"] / (ms_f32 / 1e3) / 1e9
            roof = {"bound": "fp32_issue", "achieved": achieved, "peak": peak,
                    "unit": "Glane-op/s", "frac": achieved / peak, "traffic": SCORE_TRAFFIC,
                    "kernel": "rc_score_kernel<256,true> (the f32 scoring launches)",
                    "kernel_ms": ms_f32,
                    "rest_ms": float(np.mean([q["ms_rest"] for q in pr])),
                    "achieved_if_all_rows": achieved_all, "frac_if_all_rows": achieved_all / peak,
                    "finite_candidates": r["finite"],
                    "note": "lane-ops the interpreter actually ran (rows it evaluated x (postfix "
                            "ops + residual + loss) of their candidate, counted by the kernel) / "
                            "CUDA-event time of the f32 scoring launches on the library's "
                            "stream; *_if_all_rows charges every candidate all N rows; peak = "
                            "148 SMs x 128 FP32 lanes x sm_max_mhz (MEASURED_PEAKS.json); "
                            "traffic = dram read+write bytes of one scoring-kernel launch (ncu, "
                            "profiles/rc_score_kernel_P4096_N1M.md)"}
            cfg = {"workload": f"batched scoring, P={r['P']} programs, N={r['N']} rows x 5 "
                               f"features, squared error", "l2": "flushed between steps"}
        else:
            metric, unit = "fitted_candidates_per_s", "candidates/s"
            roof = fit_roofline(r, peaks)
            cfg = {"workload": r["what"] + ", fused adjoint", "l2": "flushed between steps"}
        line = {"metric": metric, "value": value, "unit": unit, "n_gpus": world,
                "steps": args.steps, "warmup": args.warmup,
                "ms_per_step": 1e3 * dev_s / args.steps, "higher_is_better": True,
                "scaling": "weak", "vs_baseline": None, "dtype": "f32 rows, f64 sums",
                "data": "synthetic", "config": cfg, "roofline": roof,
                "clocks": r["clocks"],
                "e2e": {"value": e2e, "unit": unit, "h2d_bytes_per_step": r["h2d"],
                        "d2h_bytes_per_step": r["d2h"]},
                "gpu_launches": r["launches"]}
        if args.workload == "score":
            # work actually done: a candidate stops at its first hard failure
            line["value_evaluated"] = rows_f32 * world * args.steps / dev_s
            line["rows_evaluated_per_step"] = rows_f32
            line["rows_f64_rescored_per_step"] = rows_f64
            line["candidates_finite"] = r["finite"]
            line["scorer_tuning"] = ("candidates per work item chosen per length bucket by "
                                     "rc_autotune on the batch, before the warm-up")
            line["plain"] = r["plain"]
            line["batched_over_plain"] = value / r["plain"]["value"]
            line["absolute_error_value"] = r["absolute"]["value"]
        if args.workload == "fit" and "plain" in r:
            line["plain"] = r["plain"]
            line["fused_over_plain"] = value / r["plain"]["value"]
            line["fit_status_histogram"] = r["status"]
        if not args.no_cpu_baseline and world == 1:
            threads = os.cpu_count() or 1
            if args.workload == "score":
                v, dt, ovals = cpu_score_baseline(r["trees"], r["x"], r["y"], SCORE_SAMPLE_ROWS,
                                                  SCORE_SAMPLE_PROGS, threads, want_values=True)
                v1, _ = cpu_score_baseline(r["trees"], r["x"], r["y"], SCORE_SAMPLE_ROWS, 8, 1)
                line["cpu_baseline"] = {"value": v, "unit": unit, "cores": threads,
                                        "kind": "port", "cpu_model": cpu_model(),
                                        "value_1_thread": v1,
                                        "sample": f"the first {SCORE_SAMPLE_PROGS} programs x "
                                                  f"the first {SCORE_SAMPLE_ROWS} rows of the "
                                                  f"timed workload, f64 oracle (single thread: "
                                                  f"8 programs)"}
                line["parity"] = score_parity(pkg, r["trees"], r["x"], r["y"],
                                              SCORE_SAMPLE_ROWS, ovals)
            else:
                v, dt = cpu_fit_baseline(r["trees"], r["x"], r["y"], 1 << 14, 16, 20, threads)
                line["cpu_baseline"] = {"value": v * (1 << 14) / r["N"], "unit": unit,
                                        "cores": threads, "kind": "port",
                                        "cpu_model": cpu_model(),
                                        "sample": "16 candidates x 16384 rows x 20 iters, "
                                                  "scaled linearly in rows"}
        if args.workload == "score" and "parity" in line:
            line["parity_max_rel_err"] = line["parity"]["max_rel_err"]
            line["parity_nonfinite_mismatch"] = line["parity"]["nonfinite_mismatch"]
        if args.workload == "score" and world == 1 and not args.no_secondary:
            secondary(args, rank, world, local, pkg, W, flushbuf, peaks, line)
        print(json.dumps(line), flush=True)
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
