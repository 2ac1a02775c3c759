/*
 * rcsr_refit.h -- the exact f64 finalist refit and the structure-of-arrays
 * evaluator on the host cores (librcsr_host.so).
 *
 * After a device fit the caller refits every reported finalist exactly in f64
 * on the CPU; these entry points replace that CPU code with a blocked,
 * multi-threaded restatement whose results are bit-identical to it.
 *
 * Trees are pre-order (op, val) arrays: `ops[i]` the operator code (the
 * device opcodes 0..42 of rcsr_b200.h, 64..66 for asinh / acosh / atanh),
 * `vals[i]` a constant's value or an input's column index (unused otherwise).
 * Inputs are column-major f64, `cols[var * n + row]`. `w` may be null (every
 * row weighs 1).
 */
#ifndef RCSR_REFIT_H
#define RCSR_REFIT_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Refit `ntrees` finalists exactly. Tree t is ops/vals[tree_off[t] ..
   tree_off[t + 1]); its constants are refit in place in `vals` and its
   objective is written to loss[t] (NaN for a malformed tree).
   metric: 0 squared, 7 aic, 8 aicc, 9 bic (the LM arm: the weighted SSE is
   returned), 1 absolute, 2 log_squashed (the IRLS arm: the configured
   objective is returned). `threads` <= 0 uses every hardware thread; the
   result does not depend on it.
   Returns 0, -1 on bad arguments, -2 for a metric outside that list.
   Replaces `refit_finalists_exact` (my-version/src/fit/gpu.rs:666-687) for
   those metrics, i.e. `fit_lm` (my-version/src/fit.rs:2534-2624) and the
   IRLS arms of `fit_weighted_metric` (my-version/src/fit.rs:2937-2974,
   :3092-3170). */
int rch_refit_finalists(const int32_t *ops, double *vals, const int32_t *tree_off, int ntrees,
                        const double *cols, int64_t n, int nvars, const double *y, const double *w,
                        int iters, int metric, int threads, double *loss);

/* Predictions of one tree over n rows with the tree evaluator's domain
   rules. Returns 0, or -1 for a malformed tree or bad arguments.
   Replaces `eval_soa::compile` + `eval_soa::eval_batch`
   (my-version/src/eval_soa.rs:211-271, :481-503); unlike `compile`, every
   operator is supported, so no caller-side fallback is needed. */
int rch_soa_eval(const int32_t *ops, const double *vals, int nn, const double *cols, int64_t n,
                 int nvars, double *out);

/* The raw sum of squared residuals of one tree; +inf when any prediction is
   not finite, NaN for a malformed tree. Replaces `eval_soa::sse`
   (my-version/src/eval_soa.rs:522-540). */
double rch_soa_sse(const int32_t *ops, const double *vals, int nn, const double *cols, int64_t n,
                   int nvars, const double *y);

#ifdef __cplusplus
}
#endif

#endif /* RCSR_REFIT_H */
