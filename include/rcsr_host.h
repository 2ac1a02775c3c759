/*
 * rcsr_host.h -- the host side of the device path (librcsr_host.so): the
 * expression compiler, the fit-plan builder, fit admission and the
 * write-back of fitted constants into pool programs.
 *
 * The reference keeps this code in its Rust host (my-version/src/gpu.rs,
 * fit.rs, search.rs); these entry points restate it for a C or C++ caller
 * that drives the device library (rcsr_b200.h) without that host, producing
 * the same bytes. Trees are pre-order (op, val) arrays as in rcsr_refit.h;
 * postfix programs are the word streams the device consumes:
 * [CONST, f32 bits], [VAR, column], operator words, HALT.
 */
#ifndef RCSR_HOST_H
#define RCSR_HOST_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* compile_program (my-version/src/gpu.rs:198-219: `lower`, the peak_stack
   guard of 56, `emit`): the postfix words of a tree into words[cap]. Returns
   the word count (HALT included), -1 for an unsupported operator, -2 for a
   stack beyond 56, -3 when `cap` is too small, -4 for a malformed tree.
   `lowered` (may be null) receives 1 when `lower` rewrote the tree. */
int rch_compile_program(const int *ops, const double *vals, int nn, uint32_t *words, int cap,
                        int *lowered);

/* The peak stack depth of the lowered tree (gpu.rs:952-969), or -4. */
int rch_peak_stack(const int *ops, const double *vals, int nn);

/* gpu_fit_plan_reason (my-version/src/fit.rs:985-1196 with `flatten`, the
   correlation gauge of fit/correlation.rs:83-128): 4 words per node into
   words[cap], the constants in slot order into c0[cap_c], the gauge
   (scale, offset; -1 when absent) into gauge[2], the constant count into
   *nconst. Returns the node count, or -1 too many constants (> 20), -2 too
   many nodes (> 96), -3 no constants (unless allow_no_constants), -4 a
   malformed tree, -5 an unsupported operator, -6 capacity. */
int rch_fit_plan(const int *ops, const double *vals, int nn, uint32_t *words, int cap,
                 double *c0, int cap_c, int *gauge, int *nconst, int allow_no_constants);

/* rch_fit_plan of a postfix program (its `len` words, up to HALT) instead of
   a tree: the same plan and rejections, -4 for a program that is not one
   expression. */
int rch_fit_plan_postfix(const uint32_t *prog, int len, uint32_t *words, int cap, double *c0,
                         int cap_c, int *gauge, int *nconst, int allow_no_constants);

/* rch_fit_plan_postfix of `nprog` programs, row i of prog[nprog][width]:
   status[i] its node count or rejection, its plan at words + 4 * width * i
   (4 * width words), c0 + width * i, gauge + 2 * i and nconst[i]. Returns the
   number of accepted programs, or -1 for a bad argument. */
int rch_fit_plans_postfix(int nprog, const uint32_t *prog, int width, uint32_t *words,
                          double *c0, int *gauge, int *nconst, int *status,
                          int allow_no_constants);

/* Writes c[0..k) into the constant operands of a postfix program in place,
   in the tree's pre-order slot order (f32-rounded), and HALT after its end:
   the words compiling the tree with those constants would give. Returns the
   program's constant count, -4 for a malformed program, -2 for a stack
   beyond 56, -3 for fewer than k constants (the words are then unchanged). */
int rch_set_postfix_constants(uint32_t *w, int len, const double *c, int k);

/* rch_set_postfix_constants on rows[r] of words[][width] with c + kmax * r
   and k[r] constants for r < nrec; status[r] gets each answer. Returns the
   number of rows written, or -1 for a bad argument. */
int rch_set_postfix_constants_rows(int nrec, uint32_t *words, int width, const int *rows,
                                   const double *c, int kmax, const int *k, int *status);

/* admission_count (my-version/src/search.rs:3006-3031): how many of an
   island's offspring enter the fitted batch. */
int rch_admission_count(int island_pop, long long train_rows);

/* select_promoted (my-version/src/search.rs:3033-3074): per island, the
   pending offspring with constants ranked by screened error, complexity and
   index, the best admission_count of each promoted; the (island, index)
   pairs in ascending order into out_island / out_index. Returns their count,
   or -1 when `cap` is too small. */
int rch_select_promoted(int nislands, const int *island_pop, int npending, const int *pend_island,
                        const int *pend_index, const double *error, const double *complexity,
                        const unsigned char *has_constants, long long train_rows, int *out_island,
                        int *out_index, int cap);

#ifdef __cplusplus
}
#endif

#endif /* RCSR_HOST_H */
