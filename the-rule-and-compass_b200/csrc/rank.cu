/*
 * Exact statistics: rank sums, order statistics, maximum scan, autotune.
 */
#include <cstring>

#include "rc_internal.h"
#include "rc_ops.cuh"

extern "C" {

float rc_rank_score_batch(void *ctx, const unsigned int *prog, const unsigned int *off,
                          const int *pcount, int nsets, int ntrials, int kmax, const double *c0,
                          unsigned long long *out, int *out_status, unsigned long long *out_bb)
{
    (void)ctx; (void)prog; (void)off; (void)pcount; (void)nsets; (void)ntrials; (void)kmax;
    (void)c0; (void)out; (void)out_status; (void)out_bb;
    return -1.0f;
}

int rc_rank_debug_b(void *ctx, long long *out)
{
    (void)ctx; (void)out;
    return -1;
}

float rc_order_stat_score_batch(void *ctx, const unsigned int *prog, const unsigned int *off,
                                const int *pcount, int nsets, int ntrials, int kmax,
                                const double *c0, int what, double *out_value, int *out_status)
{
    (void)ctx; (void)prog; (void)off; (void)pcount; (void)nsets; (void)ntrials; (void)kmax;
    (void)c0; (void)what; (void)out_value; (void)out_status;
    return -1.0f;
}

float rc_max_scan_batch(void *ctx, const unsigned int *prog, const unsigned int *off,
                        const int *pcount, int nsets, int ntrials, int kmax, const double *c0,
                        const int *coords, const double *levels, RcMaxOut *out)
{
    (void)ctx; (void)prog; (void)off; (void)pcount; (void)nsets; (void)ntrials; (void)kmax;
    (void)c0; (void)coords; (void)levels; (void)out;
    return -1.0f;
}

int rc_autotune(void *ctx, const unsigned int *prog, const unsigned int *off, int nprog,
                const char *path)
{
    (void)ctx; (void)prog; (void)off; (void)nprog; (void)path;
    return -1;
}

}  // extern "C"
