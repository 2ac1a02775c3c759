/*
 * rcsr_b200.h -- the C ABI of the B200-native device library for rcsr's
 * per-generation hot path (batched bytecode evaluation, loss scoring,
 * batched LM/IRLS constant fitting, exact rank sums, input gradients).
 *
 * The first block is a drop-in for the reference's device library: every
 * symbol, argument order, struct layout and return convention matches the
 * definitions in my-version/src/cuda/eval.cu and the binding block in
 * my-version/src/gpu.rs:668-824 (cited per entry point below). Linking the
 * reference's Rust crate against librcsr_b200.so instead of its own build.rs
 * object changes no Rust code.
 *
 * Conventions (the reference's):
 *   - float-returning calls return kernel milliseconds >= 0 on success and a
 *     negative value when every output must be discarded;
 *   - int-returning calls return 0 on success and -1 on failure;
 *   - host buffers are caller-owned and only borrowed for the call; device
 *     memory is owned by the context and grows at the high-water mark;
 *   - every call completes before it returns, except rc_eval_submit /
 *     rc_eval_collect;
 *   - a context is used by one host thread at a time.
 *
 * Program formats:
 *   - "postfix words" (scoring): [OP_CONST, f32 bits] | [OP_VAR, column] |
 *     operator word ... OP_HALT, packed with off[nprog + 1] word offsets
 *     (my-version/src/gpu.rs:349-438);
 *   - "fit records" (fitting, ranks, gradients): post-order 4-word records
 *     [op, kid0, kid1, slot] with constants in c0[cand * kmax + slot]
 *     (my-version/src/fit.rs:985-1056).
 */
#ifndef RCSR_B200_H
#define RCSR_B200_H

#ifdef __cplusplus
extern "C" {
#endif

/* Host-side ledger of one batch, in milliseconds (eval.cu:95-107). */
typedef struct RcStats {
    double kernel_ms;
    double launch_ms;
    double sync_ms;
    double alloc_ms;
    double h2d_ms;
    double d2h_ms;
    double wall_ms;
    unsigned long long h2d_bytes;
    unsigned long long d2h_bytes;
    int batch;
    int failed;
} RcStats;

/* Arena / copy-mode snapshot (eval.cu:116-135). */
typedef struct RcArenaReport {
    int async_copy;
    char reason[96];
    unsigned long long pinned_bytes;
    unsigned long long alloc_calls;
    unsigned long long steady_alloc_calls;
    unsigned long long overlapped_uploads;
    unsigned long long batches;
    unsigned long long fs_alloc_calls;
    unsigned long long fs_growths;
    unsigned long long fs_steady_alloc_calls;
    unsigned long long fs_batches;
    unsigned long long fs_dev_bytes;
    unsigned long long fs_pinned_bytes;
} RcArenaReport;

/* Exact maximum-error scan output per segment (eval.cu:4529-4535). */
typedef struct RcMaxOut {
    double vmax;
    double lo;
    double hi;
    int row;
    int status;
} RcMaxOut;

/* ---- context -------------------------------------------------------- */

/* eval.cu:3137 rc_create: copies f32 column-major cols[v*n + row] and y[n];
   NULL on failure. Reads RCSR_GPU_SYNC. */
void *rc_create(const float *cols, int n, int v, const float *y);
/* eval.cu:3221 rc_destroy. */
void rc_destroy(void *ctx);
/* eval.cu:3882 rc_set_fit_data: f64 twins of the rows (+ optional base row
   weights) used by the f64 polish, the rank keys and the order statistics. */
int rc_set_fit_data(void *ctx, const double *cols, const double *y, const double *w);
/* eval.cu:3935 rc_set_score_weights: NULL clears (every row weighs 1). */
int rc_set_score_weights(void *ctx, const double *w);
/* eval.cu:3955 rc_set_fit_sign: label sign t = 2l-1 per row; NULL clears. */
int rc_set_fit_sign(void *ctx, const double *sign);

/* ---- scoring -------------------------------------------------------- */

/* eval.cu:3268 rc_set_programs: stage a packed postfix batch. */
int rc_set_programs(void *ctx, const unsigned int *prog, const unsigned int *off, int nprog);
/* eval.cu:3429 rc_eval: f32 sum of the row loss (0 squared, 1 log-squashed,
   4 absolute) per staged program; a non-finite or |pred| > 1e30 row adds 1e30. */
float rc_eval(void *ctx, float *out, int loss);
/* eval.cu:3344 / :3395 split submit/collect of rc_eval. */
int rc_eval_submit(void *ctx, int loss);
float rc_eval_collect(void *ctx, float *out);
/* eval.cu:3803 rc_score_batch: native objectives (RC_SCORE_* codes 0..14);
   out[P] f64, status[P] (0 ok, 2 non-finite, 4 all-zero weight). pcount is
   read only by the AIC family. */
float rc_score_batch(void *ctx, const unsigned int *prog, const unsigned int *off, int nprog,
                     int kind, const int *pcount, double *out, int *status);
/* eval.cu:3514 / :3550 / :3565: fixed-stride, double-buffered program pool. */
int rc_pool_reserve(void *ctx, int nprog, int width);
int rc_pool_upload(void *ctx, int which, const unsigned int *prog, int nprog);
float rc_pool_eval(void *ctx, int which, int nprog, int width, float *out, int loss);
/* eval.cu:3823 rc_pool_score. */
float rc_pool_score(void *ctx, int which, int nprog, int width, int kind, const int *pcount,
                    double *out, int *status);
/* eval.cu:3864 rc_pool_hash: FNV-1a of each slot up to and including HALT. */
int rc_pool_hash(void *ctx, int which, int nprog, int width, unsigned long long *out);
/* The next generation of the fixed-width pool, on the device
   (postfix.rs:511-567 Variation::next_generation_with_front with the engine
   of postfix.rs:438-973 and genome.rs:43-302; the reference runs this on the
   host). Parents: pool `which`, islands*pop slots of `width` (<= 128) words
   with their errors err[islands*pop] (host). Children go to pool which ^ 1.
   ops: nops (opcode, arity) pairs in the engine's table order; restart:
   [islands] or NULL; front: nfront programs packed by front_off[nfront+1]
   (words, each 2..width long), drawn with probability front_p. Outputs (host, each nullable):
   len/cost [islands*pop] u16, hash u64, err f64 (the island's elite keeps its
   parent's error, every other slot NaN), words [islands*pop*width]. Returns
   kernel ms >= 0, or -1 (bad arguments, a parent slot that is not a valid
   program, or no pool of this width reserved). */
float rc_pool_vary(void *ctx, int which, int islands, int pop, int width, const double *err,
                   int nvars, int max_complexity, unsigned int seed, unsigned int gen,
                   int init_depth, int dedup, const unsigned int *ops, int nops,
                   const unsigned char *restart, const unsigned int *front,
                   const unsigned int *front_off, int nfront, double front_p,
                   unsigned short *out_len, unsigned short *out_cost,
                   unsigned long long *out_hash, double *out_err, unsigned int *out_words);
/* eval.cu:3438 rc_predict: raw P x N predictions, row-major, no 1e30 rule. */
int rc_predict(void *ctx, const unsigned int *prog, const unsigned int *off, int nprog,
               float *out);

/* ---- fitting -------------------------------------------------------- */

/* eval.cu:4001 rc_fit_batch: batched LM/IRLS over fit records. metric:
   0 squared, 1 log-squashed, 2 correlation, 3 correlation_signed,
   4 absolute, 5 logistic. outc[P*kmax], outsse[P] (the configured objective),
   outstatus[P] (0 ok, 1 no finite step, 2 no finite iterate, 4 rank
   deficient, 5 recovered, 6 no improvement, 7 start unusable, 8 recovered
   with skipped rows). kmax > 20 is refused. */
float rc_fit_batch(void *ctx, const unsigned int *prog, const unsigned int *off,
                   const int *pcount, int nprog, int kmax, const double *c0, const int *gauge,
                   int iters, int metric, double *outc, double *outsse, int *outstatus);
/* eval.cu:4084 rc_fit_kernel_info: block width, dynamic shared bytes and the
   constant cap of the launch shape a batch with kmax constants uses. */
int rc_fit_kernel_info(int kmax, int *threads, int *smem_bytes, int *max_constants);

/* ---- exact statistics ----------------------------------------------- */

/* eval.cu:4270 rc_rank_score_batch: exact 128-bit rank sums per segment
   (seg = set * ntrials + trial): out[4*seg] = (ab_hi, ab_lo, aa_hi, aa_lo);
   out_bb = (hi, lo) of the target's sum B^2. */
float rc_rank_score_batch(void *ctx, const unsigned int *prog, const unsigned int *off,
                          const int *pcount, int nsets, int ntrials, int kmax, const double *c0,
                          unsigned long long *out, int *out_status, unsigned long long *out_bb);
/* eval.cu:4852 rc_rank_debug_b: the cached target ranks B per row. */
int rc_rank_debug_b(void *ctx, long long *out);
/* eval.cu:4743 rc_order_stat_score_batch: exact median (what=0) or
   interquartile mean (what=1) of |r| per segment. */
float rc_order_stat_score_batch(void *ctx, const unsigned int *prog, const unsigned int *off,
                                const int *pcount, int nsets, int ntrials, int kmax,
                                const double *c0, int what, double *out_value, int *out_status);
/* eval.cu:4651 rc_max_scan_batch: exact max |r| per segment. */
float rc_max_scan_batch(void *ctx, const unsigned int *prog, const unsigned int *off,
                        const int *pcount, int nsets, int ntrials, int kmax, const double *c0,
                        const int *coords, const double *levels, RcMaxOut *out);

/* ---- telemetry / probe ---------------------------------------------- */

/* eval.cu:3836 / :3855. */
void rc_stats_begin(void *ctx);
int rc_last_stats(void *ctx, RcStats *out);
/* eval.cu:3469 / :3494. */
int rc_arena_report(void *ctx, RcArenaReport *out);
int rc_arena_force_sync(void *ctx, int sync);
/* eval.cu:4886 / :4872 / :4863. */
int rc_device_count(void);
const char *rc_device_name(void);
int rc_unified(void);

/* ---- additive entry points (no counterpart in the reference ABI) ----- */

/* Batched LM with the fused forward+adjoint sweep: every LM iteration of
   every candidate runs on the device as a fixed sequence of steps (persistent
   sweeps over (candidate, 2,048-row tile) work items, then a control kernel
   that reduces, solves and queues each candidate's next sweep), captured once
   as a CUDA graph per batch shape and replayed. Arguments, outputs and status
   codes are rc_fit_batch's; metric adds 6 = implicit (minimises
   sum w (f/|grad_x f|)^2 with an exact forward-over-reverse constant
   Jacobian). flags: bit 0 skips the f64 re-baseline and polish; bit 1 turns
   off the f64 rescue (by default a candidate whose f32 assembly meets a
   non-finite row is re-assembled in f64 at the same constants and, when that
   is finite, continues its LM in f64, as the CPU fit would; with the bit set
   it stops there as the reference kernel does). rc_fit_batch and
   rc_fit_batch_plain run with flags 0. */
float rc_fit_batch_fused(void *ctx, const unsigned int *prog, const unsigned int *off,
                         const int *pcount, int nprog, int kmax, const double *c0,
                         const int *gauge, int iters, int metric, int flags, double *outc,
                         double *outsse, int *outstatus);
/* The plain comparison arm: the same LM, one candidate per launch, each
   launch a single block, candidates run back to back. Same arguments and
   outputs as rc_fit_batch. */
float rc_fit_batch_plain(void *ctx, const unsigned int *prog, const unsigned int *off,
                         const int *pcount, int nprog, int kmax, const double *c0,
                         const int *gauge, int iters, int metric, double *outc,
                         double *outsse, int *outstatus);
/* Fit autotuner: per length bucket of the batch (fit programs of <= 16,
   <= 32, <= 64 and more records) the assembly region budget that sets each
   candidate's active threads, chosen by timing the fused fit of a tuning
   batch of the bucket's candidates at budgets of 24-80 KB (`sample`
   candidates, or with sample <= 0 as many as make about 16,384 (candidate,
   tile) work items, so that the tuning batch fills the GPU like a real one;
   the bucket's first candidates repeated when it has fewer); a budget
   replaces the default only when at least 3 % faster, and the new table
   only when the caller's whole batch fits at least 3 % faster with it than
   with the defaults. Kept in the context
   for its (N, feature count) and, with a path, cached in that text file
   ("fit n v bucket budget_kb" lines; a cached bucket is not re-timed). The other arguments are rc_fit_batch_fused's. Returns the
   number of buckets with a budget, or -1. No counterpart in the reference
   ABI (its kernel shape is fixed at build time). */
int rc_fit_autotune(void *ctx, const unsigned int *prog, const unsigned int *off,
                    const int *pcount, int nprog, int kmax, const double *c0, const int *gauge,
                    int iters, int metric, int sample, const char *path);
/* The context's fit budgets in KB per length bucket (out_kb[4], 0 = the
   built-in default). Returns 0, or -1. */
int rc_fit_budgets(void *ctx, int *out_kb);
/* Sweeps each candidate of the context's last fit ran (valid until the next
   call on the context), out[4 * cand + k]: k = 0 f32 assembly sweeps, 1 f32
   objective sweeps, 2 f64 assembly sweeps (implicit: Jacobian sweeps), 3 f64
   objective sweeps (implicit: cost sweeps); the correlation arm's assembly
   and trial sweeps count as 0 and 1. Returns 0, or -1 when the last call was
   not a fit of nprog candidates. No counterpart in the reference ABI. */
int rc_last_fit_sweeps(void *ctx, int nprog, int *out);
/* Per-row gradients of fit-record programs from the fused adjoint sweep, over
   rows [row0, row0 + nrows): want = 1 writes d f / d c_j (f32,
   out[(cand * nrows + r) * kmax + j]); want = 2 writes d f / d x_k
   (out[(cand * nrows + r) * v + k]). value[cand * nrows + r] receives f. */
int rc_grad_batch(void *ctx, const unsigned int *prog, const unsigned int *off,
                  const int *pcount, int nprog, int kmax, const double *c, int want, int row0,
                  int nrows, float *value, float *out);
/* The implicit metric mean_w |f| / ||grad_x f|| per candidate from the fused
   input-adjoint sweep; status 2 (+inf) when any positive-weight row has a
   non-finite value, a non-finite gradient or a zero gradient norm. */
float rc_implicit_score_batch(void *ctx, const unsigned int *prog, const unsigned int *off,
                              const int *pcount, int nprog, int kmax, const double *c,
                              double *out, int *status);
/* Rank-sum method of rc_rank_score_batch on this context. By default a
   segment's keys are cut into buckets by splitters from a sample of them and
   each bucket is ranked on its own (a bucket holding a group of more than
   group_max distinct keys that one digit cannot tell apart is sorted whole);
   a segment with a bucket over capacity (bucket_cap keys, at most 8192) is
   redone by the radix sort. 0 keeps the built-in value; bucket_cap -1 uses
   the radix sort for every segment. The sums are the same bits either way. No counterpart in
   the reference ABI. Returns 0, or -1 for a bad argument. */
int rc_rank_tuning(void *ctx, int bucket_cap, int group_max);
/* Segments of the context's last rc_rank_score_batch that the radix sort
   summed (all of them when the buckets were off or n is past 4,194,304
   rows), or -1 on a null context. No counterpart in the reference ABI. */
int rc_rank_last_fallbacks(void *ctx);
/* Kernels this context has launched so far (a replayed fit graph counts its
   kernel nodes). No counterpart in the reference: telemetry for callers that
   check the device path really ran. Returns 0, or -1 on a null argument. */
int rc_launch_count(void *ctx, unsigned long long *out);
/* Autotune the scoring launch shape (candidates per work item, rows per work
   item) for this context's (N, feature count) and the length buckets of the
   staged program batch; the choice is cached per (N, V, bucket) and, when
   path is non-NULL, persisted to / loaded from that file. Returns the number
   of cached entries, or -1. */
int rc_autotune(void *ctx, const unsigned int *prog, const unsigned int *off, int nprog,
                const char *path);

/* Profile of the context's last scoring call (rc_score_batch, rc_eval,
   rc_pool_score, ...): device ms of the f32 scoring kernels and of the rest
   (finalize, the f64 rescore lane), the rows each interpreter actually
   evaluated (a candidate stops at its first hard failure), and the same rows
   weighted by their program's postfix ops + 2 (algorithmic lane-ops). Any
   pointer may be NULL. Returns 0, or -1 before the first scoring call. No
   counterpart in the reference ABI. */
int rc_last_score_profile(void *ctx, float *ms_f32, float *ms_rest,
                          unsigned long long *rows_f32, unsigned long long *rows_f64,
                          unsigned long long *ops_f32, unsigned long long *ops_f64);

/* ---- several GPUs behind one handle (no counterpart in the reference) -- */

/* One context per device in devices[ndev] (a device may be named twice),
   each holding the rows. The batch calls split the candidates into
   contiguous slices balanced by program words, run each slice on its device
   from its own host thread, and write every candidate's outputs at its place
   in the caller's arrays; a candidate answers exactly what a single context
   would. They return the slowest slice's kernel ms, or a negative value when
   any slice failed (then every output is to be discarded). NULL / -1 on
   failure. */
void *rc_multi_create(const float *cols, int n, int v, const float *y, int ndev,
                      const int *devices);
void rc_multi_destroy(void *multi);
int rc_multi_set_fit_data(void *multi, const double *cols, const double *y, const double *w);
float rc_multi_score_batch(void *multi, const unsigned int *prog, const unsigned int *off,
                           int nprog, int kind, const int *pcount, double *out, int *status);
float rc_multi_fit_batch(void *multi, const unsigned int *prog, const unsigned int *off,
                         const int *pcount, int nprog, int kmax, const double *c0,
                         const int *gauge, int iters, int metric, int flags, double *outc,
                         double *outsse, int *outstatus);
/* The number of devices; with ctx_out[ndev], each device's context (make that
   device current before passing it to a single-device call). */
int rc_multi_devices(void *multi, void **ctx_out);

/* Scoring for callers that cannot allocate device memory. No counterpart in
   the reference: it exists for host applications whose device memory is
   owned by another allocator, and for pipelined callers on their own streams
   for whom cudaMalloc/cudaFree (which synchronise the device) are not
   acceptable. It calls no allocator at all; its scratch is a static
   16 MiB device array that every GPU loading this library holds until exit.

   Every buffer is a caller-owned device pointer: cols is column-major with
   leading dimension ld (ld % 4 == 0, ld >= n rounded up to 1024 rows, those
   padding rows readable), y has ld readable entries, cols and y are 16-byte
   aligned, prog/off are the packed postfix batch (off[nprog + 1]), out/status
   receive nprog results. kind is 0..4 (squared, absolute, log-squashed,
   signed, maximum) with rc_score_batch's values and statuses; a program
   needing more than 16 stack entries gets status 3 and NaN. The work is
   enqueued on `stream` (a cudaStream_t, NULL = legacy default stream) and
   the call returns without waiting. Returns 0; -2 when the batch needs more
   scratch than the static maximum; -3 for an invalid argument or layout;
   -1 for a CUDA error. The first call on a device looks up the scratch
   address and sets kernel attributes, so make it before any stream capture.
   All calls share the one scratch array: calls that overlap on the GPU race
   and must be serialised by the caller. */
int rc_score_batch_noalloc(const float *cols, const float *y, int n, int v, int ld,
                           const unsigned int *prog, const unsigned int *off, int nprog, int kind,
                           double *out, int *status, void *stream);

#ifdef __cplusplus
}
#endif

#endif /* RCSR_B200_H */
