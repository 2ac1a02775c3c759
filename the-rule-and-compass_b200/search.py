"""A generation loop over the device path.

The island search of the reference (my-version/src/search.rs:5607, the
generation loop, and :1075-1120, `GpuSearch::score`) runs each generation as
screen -> admit -> fit -> rescore -> vary. Here every step runs on the
device behind the library's C ABI, and only the bookkeeping between them is
host code:

  screen   rc_pool_score of every slot of the current pool (the configured
           score kind, squared error by default, with the programs' own
           constants);
  admit    rch_select_promoted (search.rs:3033-3074): per island, the best
           screened offspring that have constants, as many as
           rch_admission_count allows (everyone with constants at >= 2^20
           rows);
  fit      the admitted programs flattened into fit plans straight from
           their words (only the accepted ones are decoded into trees),
           through rc_fit_batch_fused (the fused adjoint LM);
  rescore  the fitted constants written back into their slots' words (a
           usable, finite answer only: fit/gpu.rs:103-105; the words the
           compiled fitted tree would be), the pool re-uploaded and rescored,
           so selection sees the fitted constants;
  vary     rc_pool_vary builds the next generation from the scores
           (tournament, crossover, mutation, dedup: postfix.rs:511-567).

`GenerationLoop.generation()` returns what the fit step saw and answered, so
a caller (or a test) can hold every device answer against the exact CPU
fit of the same candidate.
"""
from __future__ import annotations

import time

import numpy as np

from . import expr as E
from .device import GenomePool
from .host import (DEFAULT_VARIATION_OPS, fit_status_usable, gpu_fit_plans_words,
                   select_promoted, set_postfix_constants, width_for)


class FitRecord:
    """One admitted candidate of one generation: its slot, the program words
    it was fitted from (and their tree, decoded when first asked for), its
    plan, and the device's answer."""

    __slots__ = ("slot", "words", "_tree", "plan", "c", "loss", "status")

    def __init__(self, slot, words, plan, c, loss, status):
        self.slot, self.words, self._tree, self.plan = slot, words, None, plan
        self.c, self.loss, self.status = c, loss, status

    @property
    def tree(self):
        if self._tree is None:
            self._tree = E.from_postfix(self.words)
        return self._tree

    def fitted(self):
        return self.plan.apply(self.tree, self.c[: self.plan.nconst])


class GenerationLoop:
    """Island-model generations of `islands` x `pop` fixed-width programs
    over the evaluator's resident rows (the training rows)."""

    def __init__(self, ev, islands, pop, nvars, max_complexity=30, fit_iters=8, seed=0,
                 ops=DEFAULT_VARIATION_OPS, init_depth=3, fit_metric=0, score_kind=0):
        self.ev = ev
        self.islands, self.pop = islands, pop
        self.nvars, self.max_complexity = nvars, max_complexity
        self.fit_iters, self.fit_metric = fit_iters, fit_metric
        self.score_kind = score_kind
        self.timing = {"screen": 0.0, "host": 0.0, "fit": 0.0, "rescore": 0.0, "vary": 0.0}
        self.seed, self.ops, self.init_depth = seed, ops, init_depth
        self.width = width_for(max_complexity)
        self.train_rows = ev.n
        self.pool = GenomePool(ev, islands, pop, self.width)
        n = islands * pop
        # generation 0: random programs built on the device (every island
        # restarts from an all-x0 pool)
        words = np.full((n, self.width), E.HALT, np.uint32)
        words[:, 0], words[:, 1] = E.VAR, 0
        self.pool.upload(0, words)
        out = self.pool.vary(0, np.zeros(n), 0, nvars, max_complexity, seed, ops,
                             init_depth=init_depth, restart=[1] * islands)
        self.words = out[0].copy()
        self.cost = out[2].astype(np.float64)
        self.cur = 1
        self.gen = 0
        self.device_ms = 0.0

    @staticmethod
    def _has_constant(w):
        """Whether a postfix program pushes a constant (a CONST opcode word,
        not an operand word)."""
        i, n = 0, len(w)
        while i < n:
            op = w[i]
            if op == E.HALT:
                return False
            if op == E.CONST:
                return True
            i += 2 if op == E.VAR else 1
        return False

    def generation(self):
        """Run one generation; returns (records, errors after the rescore).
        `timing` accumulates the device ms of the screen, fit, rescore and
        vary calls and the host ms of the steps between them."""
        n = self.islands * self.pop
        err, _, ms = self.pool.score(self.cur, self.score_kind)
        self.device_ms += ms
        self.timing["screen"] += ms
        t0 = time.perf_counter()
        # admission ranks by the screened error and the complexity the
        # variation engine reports; the admitted programs' fit plans are built
        # straight from their words (a record decodes its tree when asked)
        wl = self.words.tolist()
        hasc = np.array([self._has_constant(w) for w in wl], np.uint8)
        pending = [(i // self.pop, i % self.pop) for i in range(n)]
        admitted = select_promoted([self.pop] * self.islands, pending, err, self.cost, hasc,
                                   self.train_rows)
        slots, plans = [], []
        adm = [isl * self.pop + j for isl, j in admitted]
        for s, plan in zip(adm, gpu_fit_plans_words(self.words[adm])):
            if not isinstance(plan, str):
                plans.append(plan)
                slots.append(s)
        records = []
        self.timing["host"] += 1e3 * (time.perf_counter() - t0)
        if plans:
            c, loss, status, ms = self.ev.fit_plans(plans, self.fit_iters, self.fit_metric)
            self.device_ms += ms
            self.timing["fit"] += ms
            t0 = time.perf_counter()
            back, kc = [], []
            for k, (s, pl) in enumerate(zip(slots, plans)):
                rec = FitRecord(s, self.words[s].copy(), pl, c[k].copy(), float(loss[k]),
                                int(status[k]))
                records.append(rec)
                if fit_status_usable(rec.status) and np.all(np.isfinite(rec.c[: pl.nconst])):
                    back.append(k)
                    kc.append(pl.nconst)
            set_postfix_constants(self.words, np.asarray(slots, np.int32)[back], c[back], kc)
            self.pool.upload(self.cur, self.words)
            self.timing["host"] += 1e3 * (time.perf_counter() - t0)
            err, _, ms = self.pool.score(self.cur, self.score_kind)
            self.device_ms += ms
            self.timing["rescore"] += ms
        self.gen += 1
        out = self.pool.vary(self.cur, err, self.gen, self.nvars, self.max_complexity, self.seed,
                             self.ops, init_depth=self.init_depth)
        self.device_ms += out[5]
        self.timing["vary"] += out[5]
        self.words = out[0].copy()
        self.cost = out[2].astype(np.float64)
        self.cur ^= 1
        return records, err
