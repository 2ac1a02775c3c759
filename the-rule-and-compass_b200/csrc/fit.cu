/*
 * Batched Levenberg-Marquardt / IRLS constant fitting with a fused
 * forward + reverse-mode adjoint sweep.
 *
 * Semantics follow the reference's batched fit (my-version/src/cuda/eval.cu:
 * 1106-2606: the LM/IRLS control flow of `fit_kernel`, the per-row weights of
 * `ft_assemble` / `ft_assemble_d`, the objective sweeps `ft_loss` /
 * `ft_loss_d`, the Jacobi-equilibrated damped Cholesky with the ln-det gate
 * `ft_solve`, and the status labels 0-8) and the CPU fitter it stands in for
 * (my-version/src/fit.rs:2534-2624 `fit_lm`, :3092-3170 `irls_fit`). The
 * implicit arm follows my-version/src/implicit.rs:277-409.
 *
 * B200 design:
 *  - one block owns one candidate for its whole LM; blocks are persistent and
 *    pull candidates from a queue ordered by decreasing cost, one launch per
 *    node-count bucket so each bucket gets the shared memory it needs;
 *  - the per-row tape lives in shared memory, [node][thread]. The forward
 *    sweep writes values; the reverse sweep overwrites a child's value with
 *    its adjoint once its (single) parent has been processed, so one array
 *    serves both sweeps (a fit record program is a tree);
 *  - each chunk of rows deposits its scaled Jacobian rows and residuals in a
 *    shared f64 row buffer; J^T J and J^T r are accumulated by a 4x4
 *    register-blocked f64 SYRK (one block of the augmented Gram per thread,
 *    rows split across thread groups), then reduced across groups in a fixed
 *    order: deterministic, no atomics;
 *  - rows are f32 in the LM phase and f64 in the polish (as in the
 *    reference); the damped solve and accept/reject are f64.
 */
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "rc_internal.h"
#include "rc_ops.cuh"

#define FT_MAX_CONST 20
#define FT_MAX_NODES_ABI 96   /* the reference's plan cap (fit.rs:854) */
#define FT_MAX_NODES 255      /* what this kernel accepts */
#define FT_THREADS 128
#define FT_L1_EPS 1e-6
#define FT_LN_DET_FLOOR (-27.631021115928547)

enum {
    FM_SQUARED = 0, FM_LOG_SQUASHED = 1, FM_CORRELATION = 2, FM_CORRELATION_SIGNED = 3,
    FM_ABSOLUTE = 4, FM_LOGISTIC = 5, FM_IMPLICIT = 6
};

struct FitArgs {
    const float *cols;
    const float *y;
    const float *tsign;
    const double *cols64;
    const double *y64;
    const double *tsign64;
    const double *w;
    int n, npad, v;
    const uint4 *rec;      /* fit records, 16 bytes per node */
    const int *node_off;   /* [P+1] node offsets */
    const int *pcount;
    int kmax;
    const double *c0;
    const int *valid;      /* host-validated: 1 = a well-formed tree */
    int iters;
    int metric;
    int flags;
    const int *order;      /* candidates of this bucket, costliest first */
    int ncand;
    int *counter;
    int mmax;              /* largest node count in the bucket */
    int W;                 /* padded augmented width, multiple of 4, >= p + 1 */
    double *outc;
    double *outsse;
    int *outstatus;
};

/* ---- shared-memory layout ------------------------------------------- */

struct FitLayout {
    size_t o_rec, o_tape, o_rows, o_gram, o_jtj, o_jtr, o_L, o_c, o_cf, o_trial, o_delta, o_red,
        o_base, total;
};

__host__ __device__ inline size_t ft_align(size_t x) { return (x + 15) & ~(size_t)15; }

__host__ __device__ inline FitLayout ft_layout(int mmax, int W, int T)
{
    FitLayout L;
    size_t cur = 0;
    auto take = [&](size_t bytes) {
        size_t o = cur;
        cur = ft_align(cur + bytes);
        return o;
    };
    L.o_rec = take(sizeof(uint4) * (size_t)mmax);
    /* f32 tape [m][T] in the LM phase; f64 tape [m][T/2] in the polish. */
    L.o_tape = take(sizeof(float) * (size_t)mmax * T);
    /* Jacobian rows [T][W] f64; reused for the SYRK partials [T][16] f64. */
    size_t rows = sizeof(double) * (size_t)T * W;
    size_t part = sizeof(double) * (size_t)T * 16;
    L.o_rows = take(rows > part ? rows : part);
    L.o_gram = take(sizeof(double) * (size_t)W * W);
    L.o_jtj = take(sizeof(double) * (FT_MAX_CONST * (FT_MAX_CONST + 1) / 2));
    L.o_jtr = take(sizeof(double) * FT_MAX_CONST);
    L.o_L = take(sizeof(double) * FT_MAX_CONST * (FT_MAX_CONST + 1));
    L.o_c = take(sizeof(double) * FT_MAX_CONST);
    L.o_cf = take(sizeof(float) * FT_MAX_CONST);
    L.o_trial = take(sizeof(double) * FT_MAX_CONST);
    L.o_delta = take(sizeof(double) * FT_MAX_CONST);
    L.o_red = take(sizeof(double) * T);
    L.o_base = take(sizeof(double) * FT_MAX_CONST);
    L.total = cur;
    return L;
}

struct FitCtx {
    uint4 *rec;
    float *tape;
    double *tape64;
    double *rows;
    double *gram;
    double *jtj;
    double *jtr;
    double *L;
    double *c;
    float *cf;
    double *trial;
    double *delta;
    double *red;
    double *base;
};

__device__ inline FitCtx ft_bind(unsigned char *smem, const FitLayout &L)
{
    FitCtx f;
    f.rec = reinterpret_cast<uint4 *>(smem + L.o_rec);
    f.tape = reinterpret_cast<float *>(smem + L.o_tape);
    f.tape64 = reinterpret_cast<double *>(smem + L.o_tape);
    f.rows = reinterpret_cast<double *>(smem + L.o_rows);
    f.gram = reinterpret_cast<double *>(smem + L.o_gram);
    f.jtj = reinterpret_cast<double *>(smem + L.o_jtj);
    f.jtr = reinterpret_cast<double *>(smem + L.o_jtr);
    f.L = reinterpret_cast<double *>(smem + L.o_L);
    f.c = reinterpret_cast<double *>(smem + L.o_c);
    f.cf = reinterpret_cast<float *>(smem + L.o_cf);
    f.trial = reinterpret_cast<double *>(smem + L.o_trial);
    f.delta = reinterpret_cast<double *>(smem + L.o_delta);
    f.red = reinterpret_cast<double *>(smem + L.o_red);
    f.base = reinterpret_cast<double *>(smem + L.o_base);
    return f;
}

/* ---- per-row sweeps ---------------------------------------------------- */

/* f32 forward sweep of one row; `tp` is this thread's tape column (stride T). */
template <int T>
__device__ __forceinline__ float ft_fwd_f(const uint4 *rec, int m, const float *cols, int npad,
                                          int row, const float *cf, float *tp)
{
    float val = 0.0f;
    for (int i = 0; i < m; ++i) {
        const uint4 r = rec[i];
        if (r.x == OP_CONST) val = cf[r.w];
        else if (r.x == OP_VAR) val = __ldg(cols + (size_t)r.w * npad + row);
        else {
            const float a = tp[r.y * T];
            const float b = ft_op_binary(r.x) ? tp[r.z * T] : 0.0f;
            val = ft_value_f(r.x, a, b);
        }
        tp[i * T] = val;
    }
    return val;
}

/* f64 forward sweep; `tp` has stride TS. */
template <int TS>
__device__ __forceinline__ double ft_fwd_d(const uint4 *rec, int m, const double *cols, int npad,
                                           int row, const double *c, double *tp)
{
    double val = 0.0;
    for (int i = 0; i < m; ++i) {
        const uint4 r = rec[i];
        if (r.x == OP_CONST) val = c[r.w];
        else if (r.x == OP_VAR) val = __ldg(cols + (size_t)r.w * npad + row);
        else {
            const double a = tp[r.y * TS];
            const double b = ft_op_binary(r.x) ? tp[r.z * TS] : 0.0;
            val = ft_value_d(r.x, a, b);
        }
        tp[i * TS] = val;
    }
    return val;
}

/* f64 forward with the row's inputs given explicitly (implicit metric). */
template <int TS>
__device__ __forceinline__ double ft_fwd_d_x(const uint4 *rec, int m, const double *x,
                                             const double *c, double *tp)
{
    double val = 0.0;
    for (int i = 0; i < m; ++i) {
        const uint4 r = rec[i];
        if (r.x == OP_CONST) val = c[r.w];
        else if (r.x == OP_VAR) val = x[r.w];
        else {
            const double a = tp[r.y * TS];
            const double b = ft_op_binary(r.x) ? tp[r.z * TS] : 0.0;
            val = ft_value_d(r.x, a, b);
        }
        tp[i * TS] = val;
    }
    return val;
}

/* Reverse sweep in place (f32). Adjoints of constants are written to
   g[slot * gs] (f64), of inputs accumulated into ig[col * is] when ig != 0.
   Every node of a fit-record tree has one parent, so a child's tape entry
   switches from value to adjoint exactly when its parent is processed.
   Mirrors eval.cu:1236-1317 (an adjoint of zero passes nothing). */
template <int T>
__device__ __forceinline__ void ft_bwd_f(const uint4 *rec, int m, float *tp, double *g, int gs,
                                         float *ig, int is)
{
    tp[(m - 1) * T] = 1.0f;
    for (int i = m - 1; i >= 0; --i) {
        const uint4 r = rec[i];
        const float a = tp[i * T];
        if (r.x == OP_CONST) {
            if (g) g[r.w * gs] += (double)a;
            continue;
        }
        if (r.x == OP_VAR) {
            if (ig) ig[r.w * is] += a;
            continue;
        }
        const bool bin = ft_op_binary(r.x);
        const float x = tp[r.y * T];
        const float yv = bin ? tp[r.z * T] : 0.0f;
        float c0 = 0.0f, c1 = 0.0f;
        if (a != 0.0f && !(r.x == OP_POW && !(x > 0.0f))) {
            float d0, d1;
            ft_partials_f(r.x, x, yv, d0, d1);
            c0 = a * d0;
            c1 = a * d1;
        }
        tp[r.y * T] = c0;
        if (bin) tp[r.z * T] = c1;
    }
}

template <int TS>
__device__ __forceinline__ void ft_bwd_d(const uint4 *rec, int m, double *tp, double *g, int gs,
                                         double *ig, int is)
{
    tp[(m - 1) * TS] = 1.0;
    for (int i = m - 1; i >= 0; --i) {
        const uint4 r = rec[i];
        const double a = tp[i * TS];
        if (r.x == OP_CONST) {
            if (g) g[r.w * gs] += a;
            continue;
        }
        if (r.x == OP_VAR) {
            if (ig) ig[r.w * is] += a;
            continue;
        }
        const bool bin = ft_op_binary(r.x);
        const double x = tp[r.y * TS];
        const double yv = bin ? tp[r.z * TS] : 0.0;
        double c0 = 0.0, c1 = 0.0;
        if (a != 0.0 && !(r.x == OP_POW && !(x > 0.0))) {
            double d0, d1;
            ft_partials_d(r.x, x, yv, d0, d1);
            c0 = a * d0;
            c1 = a * d1;
        }
        tp[r.y * TS] = c0;
        if (bin) tp[r.z * TS] = c1;
    }
}

/* ---- objective pieces (eval.cu:638-693, 1492-1855) ------------------- */

__device__ __forceinline__ float ft_row_loss_f(float r, int metric)
{
    if (metric == FM_LOG_SQUASHED) {
        const float rr = r * r;
        return isfinite(rr) ? log1pf(rr) : 2.0f * logf(fabsf(r));
    }
    if (metric == FM_ABSOLUTE) return fabsf(r);
    return r * r;
}

__device__ __forceinline__ double ft_row_weight(double base, double r, int metric)
{
    if (metric == FM_LOG_SQUASHED) return base * 2.0 / (1.0 + r * r);
    if (metric == FM_ABSOLUTE) return base / fmax(fabs(r), FT_L1_EPS);
    return base;
}

__device__ __forceinline__ double ft_logistic_q(double u)
{
    double q;
    if (u >= 0.0) q = 1.0 / (1.0 + exp(-u));
    else {
        const double e = exp(u);
        q = e / (1.0 + e);
    }
    return fmin(1.0 - 1e-9, fmax(1e-9, q));
}

__device__ __forceinline__ double ft_softplus_neg(double u)
{
    const double a = fabs(u);
    return (u < 0.0 ? -u : 0.0) + log1p(exp(-a));
}

/* ---- block reductions -------------------------------------------------- */

template <int T>
__device__ __forceinline__ double ft_block_sum(double v, double *red)
{
    const int tid = threadIdx.x;
    red[tid] = v;
    __syncthreads();
    for (int st = T / 2; st > 0; st >>= 1) {
        if (tid < st) red[tid] += red[tid + st];
        __syncthreads();
    }
    const double total = red[0];
    __syncthreads();
    return total;
}

/* SYRK block assignment: the (W/4)x(W/4) block lower triangle of the
   augmented Gram [J | r]^T [J | r] is split into nblk 4x4 blocks; thread t
   owns block t % nblk and rows r == t / nblk (mod RG). */
struct Syrk {
    int nblk, RG, blk, rg, bi, bj;
};

template <int T>
__device__ __forceinline__ Syrk ft_syrk_setup(int W)
{
    Syrk s;
    const int nb = W / 4;
    s.nblk = nb * (nb + 1) / 2;
    s.RG = T / s.nblk;
    if (s.RG < 1) s.RG = 1;
    s.blk = threadIdx.x % s.nblk;
    s.rg = threadIdx.x / s.nblk;
    int b = s.blk, i = 0;
    while (b > i) {
        b -= i + 1;
        ++i;
    }
    s.bi = i;
    s.bj = b;
    return s;
}

/* Accumulate rows [0, R) of the row buffer into this thread's block. */
__device__ __forceinline__ void ft_syrk_chunk(const Syrk &s, const double *rows, int W, int R,
                                              double acc[16])
{
    if (s.rg >= s.RG) return;
    for (int r = s.rg; r < R; r += s.RG) {
        const double *row = rows + (size_t)r * W;
        const double2 a01 = *reinterpret_cast<const double2 *>(row + 4 * s.bi);
        const double2 a23 = *reinterpret_cast<const double2 *>(row + 4 * s.bi + 2);
        const double2 b01 = *reinterpret_cast<const double2 *>(row + 4 * s.bj);
        const double2 b23 = *reinterpret_cast<const double2 *>(row + 4 * s.bj + 2);
        const double av[4] = {a01.x, a01.y, a23.x, a23.y};
        const double bv[4] = {b01.x, b01.y, b23.x, b23.y};
#pragma unroll
        for (int i = 0; i < 4; ++i)
#pragma unroll
            for (int j = 0; j < 4; ++j) acc[i * 4 + j] = fma(av[i], bv[j], acc[i * 4 + j]);
    }
}

/* Reduce the per-group partial blocks in ascending group order and unpack the
   packed lower triangle J^T J (p(p+1)/2) and J^T r (p). */
template <int T>
__device__ __forceinline__ void ft_syrk_finish(const Syrk &s, double acc[16], double *part,
                                               double *gram, int W, int p, double *jtj,
                                               double *jtr)
{
    const int tid = threadIdx.x;
    if (s.rg < s.RG) {
#pragma unroll
        for (int e = 0; e < 16; ++e) part[(s.rg * s.nblk + s.blk) * 16 + e] = acc[e];
    }
    __syncthreads();
    for (int q = tid; q < s.nblk * 16; q += T) {
        const int blk = q / 16, e = q % 16;
        double sum = 0.0;
        for (int g = 0; g < s.RG; ++g) sum += part[(g * s.nblk + blk) * 16 + e];
        int b = blk, bi = 0;
        while (b > bi) {
            b -= bi + 1;
            ++bi;
        }
        const int i = 4 * bi + e / 4, j = 4 * b + e % 4;
        gram[i * W + j] = sum;
    }
    __syncthreads();
    for (int q = tid; q < p * (p + 1) / 2 + p; q += T) {
        if (q < p * (p + 1) / 2) {
            int i = 0, k = q;
            while (k > i) {
                k -= i + 1;
                ++i;
            }
            jtj[q] = gram[i * W + k];
        } else {
            const int j = q - p * (p + 1) / 2;
            jtr[j] = gram[p * W + j];
        }
    }
    __syncthreads();
}

/* ---- the damped solve (eval.cu:1873-1949 `ft_solve`) ----------------- */

__device__ int ft_solve(const double *jtj, const double *jtr, double lambda, int p, double *delta,
                        double *L)
{
    double dscale[FT_MAX_CONST];
    for (int i = 0; i < p; ++i) {
        const double aii = jtj[i * (i + 1) / 2 + i];
        if (!(aii > 0.0) || !isfinite(aii)) return 1;
        dscale[i] = sqrt(aii);
    }
    int rank_deficient = 0;
    double sum_ln_L = 0.0;
    int ok = 1;
    for (int i = 0; i < p && ok; ++i) {
        for (int j = 0; j <= i; ++j) {
            double s = jtj[i * (i + 1) / 2 + j] / (dscale[i] * dscale[j]);
            if (!isfinite(s)) return 1;
            for (int k = 0; k < j; ++k) s -= L[i * p + k] * L[j * p + k];
            if (i == j) {
                if (!(s > 0.0) || !isfinite(s)) {
                    ok = 0;
                    break;
                }
                L[i * p + i] = sqrt(s);
                sum_ln_L += 0.5 * log(s);
            } else {
                L[i * p + j] = s / L[j * p + j];
            }
        }
    }
    if (!ok) rank_deficient = 1;
    else {
        const double ln_det = 2.0 * sum_ln_L;
        if (!isfinite(ln_det) || ln_det < FT_LN_DET_FLOOR) rank_deficient = 1;
    }
    for (int i = 0; i < p; ++i) {
        for (int j = 0; j <= i; ++j) {
            double s = jtj[i * (i + 1) / 2 + j] / (dscale[i] * dscale[j]);
            if (i == j) s = s * (1.0 + lambda) + 1e-12;
            for (int k = 0; k < j; ++k) s -= L[i * p + k] * L[j * p + k];
            if (i == j) {
                if (!(s > 1e-18) || !isfinite(s)) return 1;
                L[i * p + i] = sqrt(s);
            } else {
                L[i * p + j] = s / L[j * p + j];
            }
        }
    }
    double rhs[FT_MAX_CONST];
    for (int i = 0; i < p; ++i) rhs[i] = -jtr[i] / dscale[i];
    for (int i = 0; i < p; ++i) {
        double s = rhs[i];
        for (int k = 0; k < i; ++k) s -= L[i * p + k] * rhs[k];
        rhs[i] = s / L[i * p + i];
    }
    for (int i = p - 1; i >= 0; --i) {
        double s = rhs[i];
        for (int k = i + 1; k < p; ++k) s -= L[k * p + i] * delta[k];
        delta[i] = s / L[i * p + i];
    }
    for (int i = 0; i < p; ++i) delta[i] /= dscale[i];
    return rank_deficient ? 4 : 0;
}

/* Gaussian elimination with partial pivoting on (A + lambda diag A + 1e-12 I)
   (implicit.rs:215-253). `M` is p x (p+1) scratch. Returns 0 or 1 (singular). */
__device__ int ft_gauss_solve(const double *jtj, const double *jtr, double lambda, int p,
                              double *delta, double *M)
{
    const int w = p + 1;
    for (int i = 0; i < p; ++i) {
        for (int j = 0; j < p; ++j) {
            const int a = i > j ? i : j, b = i > j ? j : i;
            M[i * w + j] = jtj[a * (a + 1) / 2 + b];
        }
        M[i * w + i] = M[i * w + i] * (1.0 + lambda) + 1e-12;
        M[i * w + p] = -jtr[i];
    }
    for (int col = 0; col < p; ++col) {
        int piv = col;
        for (int r = col + 1; r < p; ++r)
            if (fabs(M[r * w + col]) > fabs(M[piv * w + col])) piv = r;
        if (fabs(M[piv * w + col]) < 1e-300) return 1;
        if (piv != col)
            for (int c = 0; c <= p; ++c) {
                const double t = M[col * w + c];
                M[col * w + c] = M[piv * w + c];
                M[piv * w + c] = t;
            }
        for (int r = col + 1; r < p; ++r) {
            const double f = M[r * w + col] / M[col * w + col];
            if (f != 0.0)
                for (int c = col; c <= p; ++c) M[r * w + c] -= f * M[col * w + c];
        }
    }
    for (int i = p - 1; i >= 0; --i) {
        double s = M[i * w + p];
        for (int j = i + 1; j < p; ++j) s -= M[i * w + j] * delta[j];
        delta[i] = s / M[i * w + i];
    }
    return 0;
}

/* ---- sweeps over all rows -------------------------------------------- */

struct SweepOut {
    double loss;
    int bad;
    int skipped;
};

/* f32 assembly at f.c (eval.cu:1692-1804): J^T J, J^T r and the objective. */
template <int T>
__device__ SweepOut ft_assemble_f(const FitArgs &a, const FitCtx &f, int m, int p, int W,
                                  const Syrk &sy)
{
    const int tid = threadIdx.x;
    double acc[16];
#pragma unroll
    for (int e = 0; e < 16; ++e) acc[e] = 0.0;
    double loss = 0.0;
    int bad = 0;
    float *tp = f.tape + tid;
    double *myrow = f.rows + (size_t)tid * W;
    for (int base = 0; base < a.n; base += T) {
        const int row = base + tid;
        for (int j = 0; j < W; ++j) myrow[j] = 0.0;
        const double wr = (row < a.n && a.w) ? a.w[row] : 1.0;
        if (row < a.n && wr > 0.0) {
            const float pred = ft_fwd_f<T>(f.rec, m, a.cols, a.npad, row, f.cf, tp);
            const float r = pred - a.y[row];
            bool ok = isfinite(pred) && fabsf(pred) <= 1e30f && isfinite(r);
            ft_bwd_f<T>(f.rec, m, tp, myrow, 1, nullptr, 0);
            double sw, resp = (double)r, rowloss;
            if (a.metric == FM_LOGISTIC) {
                const double tt = a.tsign ? (double)a.tsign[row] : 0.0;
                const double u = tt * (double)pred;
                if (!a.tsign || !isfinite(tt)) ok = false;
                const double q = ft_logistic_q(u);
                sw = wr * q * (1.0 - q);
                resp = -tt / q;
                rowloss = wr * ft_softplus_neg(u);
            } else {
                sw = ft_row_weight(wr, (double)r, a.metric);
                rowloss = wr * (double)ft_row_loss_f(r, a.metric);
            }
            const float s = sqrtf((float)sw);
            for (int j = 0; j < p; ++j)
                if (!isfinite((float)myrow[j])) ok = false;
            for (int j = 0; j < p; ++j) myrow[j] = ok ? (double)(s * (float)myrow[j]) : 0.0;
            myrow[p] = ok ? (double)(float)(s * resp) : 0.0;
            if (ok) loss += rowloss;
            else bad = 1;
        }
        __syncthreads();
        ft_syrk_chunk(sy, f.rows, W, T, acc);
        __syncthreads();
    }
    SweepOut o;
    o.bad = __syncthreads_or(bad);
    o.loss = ft_block_sum<T>(loss, f.red);
    o.skipped = 0;
    ft_syrk_finish<T>(sy, acc, f.rows, f.gram, W, p, f.jtj, f.jtr);
    return o;
}

/* f64 assembly for the polish (eval.cu:1492-1630), T/2 rows per chunk. */
template <int T>
__device__ SweepOut ft_assemble_d(const FitArgs &a, const FitCtx &f, int m, int p, int W,
                                  const Syrk &sy)
{
    constexpr int TS = T / 2;
    const int tid = threadIdx.x;
    double acc[16];
#pragma unroll
    for (int e = 0; e < 16; ++e) acc[e] = 0.0;
    double loss = 0.0;
    int bad = 0, skipped = 0;
    double *tp = f.tape64 + tid;
    double *myrow = f.rows + (size_t)tid * W;
    for (int base = 0; base < a.n; base += TS) {
        const int row = base + tid;
        if (tid < TS) {
            for (int j = 0; j < W; ++j) myrow[j] = 0.0;
            const double wr = (row < a.n && a.w) ? a.w[row] : 1.0;
            if (row < a.n && wr > 0.0) {
                const double pred = ft_fwd_d<TS>(f.rec, m, a.cols64, a.npad, row, f.c, tp);
                const double r = pred - a.y64[row];
                bool ok = isfinite(pred) && isfinite(r);
                ft_bwd_d<TS>(f.rec, m, tp, myrow, 1, nullptr, 0);
                bool grad_ok = true;
                for (int j = 0; j < p; ++j)
                    if (!isfinite(myrow[j])) grad_ok = false;
                double sw, resp = r, rho;
                if (a.metric == FM_LOGISTIC) {
                    const double tt = a.tsign64 ? a.tsign64[row] : 0.0;
                    const double u = tt * pred;
                    if (!a.tsign64 || !isfinite(tt)) ok = false;
                    const double q = ft_logistic_q(u);
                    sw = wr * q * (1.0 - q);
                    resp = -tt / q;
                    rho = ft_softplus_neg(u);
                } else {
                    sw = ft_row_weight(wr, r, a.metric);
                    if (a.metric == FM_SQUARED) rho = r * r;
                    else if (a.metric == FM_ABSOLUTE) rho = fabs(r);
                    else rho = log1p(r * r);
                }
                const double s = sqrt(sw);
                const bool use = ok && grad_ok;
                for (int j = 0; j < p; ++j) myrow[j] = use ? s * myrow[j] : 0.0;
                myrow[p] = use ? s * resp : 0.0;
                if (ok) loss += wr * rho;
                else bad = 1;
                if (ok && !grad_ok) skipped = 1;
            }
        } else if (tid < T) {
            /* rows [TS, T) of the buffer stay unused in the polish */
        }
        __syncthreads();
        ft_syrk_chunk(sy, f.rows, W, TS, acc);
        __syncthreads();
    }
    SweepOut o;
    o.bad = __syncthreads_or(bad);
    o.skipped = __syncthreads_or(skipped);
    o.loss = ft_block_sum<T>(loss, f.red);
    ft_syrk_finish<T>(sy, acc, f.rows, f.gram, W, p, f.jtj, f.jtr);
    return o;
}

/* f32 objective at constants `cf` (eval.cu:1808-1855). */
template <int T>
__device__ double ft_loss_f(const FitArgs &a, const FitCtx &f, int m, const float *cf)
{
    const int tid = threadIdx.x;
    double local = 0.0;
    float *tp = f.tape + tid;
    for (int row = tid; row < a.n; row += T) {
        const double wr = a.w ? a.w[row] : 1.0;
        if (wr <= 0.0) continue;
        const float pred = ft_fwd_f<T>(f.rec, m, a.cols, a.npad, row, cf, tp);
        const float r = pred - a.y[row];
        if (!isfinite(pred) || fabsf(pred) > 1e30f || !isfinite(r)) local += 1e30;
        else if (a.metric == FM_LOGISTIC) {
            const double tt = a.tsign ? (double)a.tsign[row] : 0.0;
            local += isfinite(tt) ? wr * ft_softplus_neg(tt * (double)pred) : 1e30;
        } else if (a.metric == FM_SQUARED) local += wr * (double)r * (double)r;
        else local += wr * (double)ft_row_loss_f(r, a.metric);
    }
    return ft_block_sum<T>(local, f.red);
}

/* f64 objective at constants `c` (eval.cu:1634-1682), T/2 rows at a time. */
template <int T>
__device__ double ft_loss_d(const FitArgs &a, const FitCtx &f, int m, const double *c)
{
    constexpr int TS = T / 2;
    const int tid = threadIdx.x;
    double local = 0.0;
    if (tid < TS) {
        double *tp = f.tape64 + tid;
        for (int row = tid; row < a.n; row += TS) {
            const double wr = a.w ? a.w[row] : 1.0;
            if (wr <= 0.0) continue;
            const double pred = ft_fwd_d<TS>(f.rec, m, a.cols64, a.npad, row, c, tp);
            const double r = pred - a.y64[row];
            if (!isfinite(pred) || !isfinite(r)) local += 1e30;
            else if (a.metric == FM_LOGISTIC) {
                const double tt = a.tsign64 ? a.tsign64[row] : 0.0;
                local += isfinite(tt) ? wr * ft_softplus_neg(tt * pred) : 1e30;
            } else if (a.metric == FM_SQUARED) local += wr * r * r;
            else if (a.metric == FM_ABSOLUTE) local += wr * fabs(r);
            else local += wr * log1p(r * r);
        }
    }
    return ft_block_sum<T>(local, f.red);
}

/* ---- the implicit metric (implicit.rs:68-409) ---------------------------
 * Per row: d = f / ||grad_x f|| (f64 forward + input adjoint); a row with a
 * non-finite value or gradient, or a zero gradient norm, makes the whole
 * evaluation undefined. The LM's Jacobian is central differences of d with
 * h = 1e-6 (1 + |c_j|), exactly as the reference CPU arm. */

#define FT_IMPLICIT_MAXV 16

template <int TS>
__device__ __forceinline__ bool ft_implicit_d(const uint4 *rec, int m, const double *x, int v,
                                              const double *c, double *tp, double &d)
{
    const double fv = ft_fwd_d_x<TS>(rec, m, x, c, tp);
    if (!isfinite(fv)) return false;
    double ig[FT_IMPLICIT_MAXV];
    for (int k = 0; k < FT_IMPLICIT_MAXV; ++k) ig[k] = 0.0;
    /* input adjoint accumulated in registers: columns are < FT_IMPLICIT_MAXV */
    tp[(m - 1) * TS] = 1.0;
    for (int i = m - 1; i >= 0; --i) {
        const uint4 r = rec[i];
        const double a = tp[i * TS];
        if (r.x == OP_CONST) continue;
        if (r.x == OP_VAR) {
#pragma unroll
            for (int k = 0; k < FT_IMPLICIT_MAXV; ++k)
                if ((int)r.w == k) ig[k] += a;
            continue;
        }
        const bool bin = ft_op_binary(r.x);
        const double xx = tp[r.y * TS];
        const double yy = bin ? tp[r.z * TS] : 0.0;
        double c0 = 0.0, c1 = 0.0;
        if (a != 0.0 && !(r.x == OP_POW && !(xx > 0.0))) {
            double d0, d1;
            ft_partials_d(r.x, xx, yy, d0, d1);
            c0 = a * d0;
            c1 = a * d1;
        }
        tp[r.y * TS] = c0;
        if (bin) tp[r.z * TS] = c1;
    }
    double nsq = 0.0;
    for (int k = 0; k < FT_IMPLICIT_MAXV; ++k) {
        if (k >= v) break;
        if (!isfinite(ig[k])) return false;
        nsq += ig[k] * ig[k];
    }
    const double norm = sqrt(nsq);
    if (!(isfinite(norm) && norm > 0.0)) return false;
    d = fv / norm;
    return isfinite(d);
}

/* One implicit sweep at f.c: when `jac`, also the central-difference Jacobian
   rows and the J^T J / J^T r assembly; returns the cost sum w d^2, or +inf
   when any positive-weight row is undefined (at c or at a perturbation). */
template <int T>
__device__ double ft_implicit_sweep(const FitArgs &a, const FitCtx &f, int m, int p, int W,
                                    const Syrk &sy, const double *c, bool jac, int *undefined)
{
    constexpr int TS = T / 2;
    const int tid = threadIdx.x;
    double acc[16];
#pragma unroll
    for (int e = 0; e < 16; ++e) acc[e] = 0.0;
    double cost = 0.0;
    int bad = 0;
    double *tp = f.tape64 + tid;
    double *myrow = f.rows + (size_t)tid * W;
    double x[FT_IMPLICIT_MAXV];
    double cp[FT_MAX_CONST];
    for (int base = 0; base < a.n; base += TS) {
        const int row = base + tid;
        if (tid < TS) {
            if (jac)
                for (int j = 0; j < W; ++j) myrow[j] = 0.0;
            const double wr = (row < a.n && a.w) ? a.w[row] : 1.0;
            if (row < a.n && wr > 0.0 && isfinite(wr)) {
                for (int k = 0; k < FT_IMPLICIT_MAXV; ++k)
                    x[k] = k < a.v ? a.cols64[(size_t)k * a.npad + row] : 0.0;
                double d;
                if (!ft_implicit_d<TS>(f.rec, m, x, a.v, c, tp, d)) bad = 1;
                else {
                    const double sw = sqrt(wr);
                    const double r = sw * d;
                    cost += r * r;
                    if (jac) {
                        for (int j = 0; j < p; ++j) cp[j] = c[j];
                        for (int j = 0; j < p && !bad; ++j) {
                            const double h = 1e-6 * (1.0 + fabs(c[j]));
                            double dp, dm;
                            cp[j] = c[j] + h;
                            const bool okp = ft_implicit_d<TS>(f.rec, m, x, a.v, cp, tp, dp);
                            cp[j] = c[j] - h;
                            const bool okm = ft_implicit_d<TS>(f.rec, m, x, a.v, cp, tp, dm);
                            cp[j] = c[j];
                            if (!okp || !okm) {
                                bad = 1;
                                break;
                            }
                            myrow[j] = (sw * dp - sw * dm) / (2.0 * h);
                            if (!isfinite(myrow[j])) bad = 1;
                        }
                        myrow[p] = r;
                    }
                }
            } else if (row < a.n && !(wr >= 0.0 && isfinite(wr))) {
                bad = 1;
            }
        }
        if (jac) {
            __syncthreads();
            ft_syrk_chunk(sy, f.rows, W, TS, acc);
            __syncthreads();
        }
    }
    *undefined = __syncthreads_or(bad);
    const double total = ft_block_sum<T>(cost, f.red);
    if (jac) ft_syrk_finish<T>(sy, acc, f.rows, f.gram, W, p, f.jtj, f.jtr);
    return *undefined ? INFINITY : total;
}

/* ---- the LM driver, one candidate per block ----------------------------- */

__device__ __forceinline__ void ft_set_c(const FitCtx &f, int p, const double *src)
{
    const int tid = threadIdx.x;
    if (tid < p) {
        f.c[tid] = src[tid];
        f.cf[tid] = (float)src[tid];
    }
    __syncthreads();
}

template <int T>
__device__ void ft_lm_standard(const FitArgs &a, const FitCtx &f, int m, int p, int W,
                               const Syrk &sy, double &best_out, int &status_out)
{
    const int tid = threadIdx.x;
    __shared__ double s_best, s_lambda, s_tsse;
    __shared__ int s_flag, s_rank, s_improved, s_start, s_skip;
    const int irls = (a.metric == FM_ABSOLUTE);
    const int iters = a.iters;
    const int rounds = irls ? (iters < 1 ? 1 : (iters < 4 ? iters : 4)) : 1;
    const int inner = irls ? (iters / rounds < 1 ? 1 : iters / rounds) : iters;
    int status = 0;
    double best = 0.0;
    if (tid == 0) {
        s_rank = 0;
        s_improved = 0;
        s_start = 0;
        s_skip = 0;
        s_lambda = 1e-3;
    }
    __syncthreads();
    if (iters > 0) {
        SweepOut o = ft_assemble_f<T>(a, f, m, p, W, sy);
        int assembled = 1;
        best = o.loss;
        if (tid == 0) s_start = o.bad ? 0 : 1;
        if (o.bad) status = 2;
        for (int round = 0; round < rounds && status == 0 && best != 0.0; ++round) {
            if (irls && round > 0) assembled = 0;
            for (int it = 0; it < inner && status == 0; ++it) {
                if (!assembled) {
                    o = ft_assemble_f<T>(a, f, m, p, W, sy);
                    assembled = 1;
                    if (o.bad) {
                        status = 2;
                        break;
                    }
                }
                if (tid == 0) {
                    const int sv = ft_solve(f.jtj, f.jtr, s_lambda, p, f.delta, f.L);
                    s_flag = sv != 1;
                    if (sv == 4) s_rank = 1;
                    if (s_flag)
                        for (int j = 0; j < p; ++j) {
                            const double t = f.c[j] + f.delta[j];
                            f.trial[j] = fmin(1e6, fmax(-1e6, t));
                        }
                }
                __syncthreads();
                if (!s_flag) {
                    status = 1;
                    break;
                }
                /* f32 copy of the trial constants lives in `base` (as floats) */
                float *tcf = reinterpret_cast<float *>(f.base);
                if (tid < p) tcf[tid] = (float)f.trial[tid];
                __syncthreads();
                double tsse = ft_loss_f<T>(a, f, m, tcf);
                /* True-metric Armijo for L1: two halvings (eval.cu:2486-2497). */
                for (int half = 0; half < (irls ? 2 : 0) && !(tsse < best); ++half) {
                    if (tid < p) {
                        f.trial[tid] = f.c[tid] + 0.5 * (f.trial[tid] - f.c[tid]);
                        tcf[tid] = (float)f.trial[tid];
                    }
                    __syncthreads();
                    tsse = ft_loss_f<T>(a, f, m, tcf);
                }
                if (tsse < best) {
                    ft_set_c(f, p, f.trial);
                    best = tsse;
                    if (tid == 0) {
                        s_lambda = fmax(s_lambda / 8.0, 1e-12);
                        s_improved = 1;
                    }
                    __syncthreads();
                    assembled = 0;
                    if (best == 0.0) break;
                } else {
                    if (tid == 0) s_lambda *= 6.0;
                    __syncthreads();
                    if (s_lambda > 1e9) break;
                }
            }
        }
        /* Re-baseline in f64, then the undamped Gauss-Newton polish in f64
           (eval.cu:2537-2580). */
        if (status == 0 && !(a.flags & 1)) {
            const double exact = ft_loss_d<T>(a, f, m, f.c);
            if (isfinite(exact)) best = exact;
            for (int it = 0; it < 4 && status == 0 && best != 0.0; ++it) {
                SweepOut od = ft_assemble_d<T>(a, f, m, p, W, sy);
                if (tid == 0 && od.skipped) s_skip = 1;
                if (od.bad) {
                    status = 2;
                    break;
                }
                if (tid == 0) {
                    const int sv = ft_solve(f.jtj, f.jtr, 0.0, p, f.delta, f.L);
                    s_flag = sv != 1;
                    if (sv == 4) s_rank = 1;
                    if (s_flag)
                        for (int j = 0; j < p; ++j) {
                            const double t = f.c[j] + f.delta[j];
                            f.trial[j] = fmin(1e6, fmax(-1e6, t));
                        }
                }
                __syncthreads();
                if (!s_flag) break;
                double tsse = ft_loss_d<T>(a, f, m, f.trial);
                if (irls && !(tsse < best)) {
                    if (tid < p) f.trial[tid] = f.c[tid] + 0.5 * (f.trial[tid] - f.c[tid]);
                    __syncthreads();
                    tsse = ft_loss_d<T>(a, f, m, f.trial);
                }
                if (tsse < best) {
                    ft_set_c(f, p, f.trial);
                    best = tsse;
                    if (tid == 0) s_improved = 1;
                    __syncthreads();
                } else {
                    break;
                }
            }
        }
    }
    __syncthreads();
    /* Status labels (eval.cu:2583-2600). */
    if (status == 1 || status == 2) {
        if (!s_start) status = 7;
        else if (s_improved) status = 5;
        else status = 6;
    } else if (status == 0) {
        if (s_skip) status = 8;
        else if (s_rank) status = 4;
        else if (!s_improved && iters > 0) status = 6;
    }
    best_out = best;
    status_out = status;
    (void)s_tsse;
    (void)s_best;
}

/* implicit.rs:277-409: LM on the signed geometric residual. */
template <int T>
__device__ void ft_lm_implicit(const FitArgs &a, const FitCtx &f, int m, int p, int W,
                               const Syrk &sy, double &best_out, int &status_out)
{
    const int tid = threadIdx.x;
    __shared__ double s_lambda;
    __shared__ int s_flag, s_improved;
    int undefined = 0;
    if (tid == 0) {
        s_lambda = 1e-3;
        s_improved = 0;
    }
    __syncthreads();
    /* the starting constants stay in f.base for the final comparison */
    if (tid < p) f.base[tid] = f.c[tid];
    __syncthreads();
    double best = ft_implicit_sweep<T>(a, f, m, p, W, sy, f.c, false, &undefined);
    if (undefined) {
        best_out = INFINITY;
        status_out = 7;
        return;
    }
    const double start = best;
    if (p > 0 && a.iters > 0) {
        const int outer = a.iters < 1 ? 1 : a.iters;
        for (int it = 0; it < outer; ++it) {
            ft_implicit_sweep<T>(a, f, m, p, W, sy, f.c, true, &undefined);
            if (undefined) break;
            if (tid == 0) {
                const int sv = ft_gauss_solve(f.jtj, f.jtr, s_lambda, p, f.delta, f.L);
                s_flag = sv == 0;
                if (s_flag)
                    for (int j = 0; j < p; ++j)
                        f.trial[j] = fmin(1e6, fmax(-1e6, f.c[j] + f.delta[j]));
            }
            __syncthreads();
            if (!s_flag) {
                if (tid == 0) s_lambda *= 6.0;
                __syncthreads();
                if (s_lambda > 1e9) break;
                continue;
            }
            int und2 = 0;
            const double s = ft_implicit_sweep<T>(a, f, m, p, W, sy, f.trial, false, &und2);
            if (!und2 && s < best) {
                best = s;
                ft_set_c(f, p, f.trial);
                if (tid == 0) {
                    s_lambda = fmax(s_lambda / 8.0, 1e-12);
                    s_improved = 1;
                }
                __syncthreads();
                if (best == 0.0) break;
            } else {
                if (tid == 0) s_lambda *= 6.0;
                __syncthreads();
                if (s_lambda > 1e9) break;
            }
        }
    }
    /* The reference writes constants back only when they beat the start. */
    if (!(best < start)) ft_set_c(f, p, f.base);
    best_out = best;
    status_out = s_improved ? 0 : 6;
}

template <int T>
__global__ void __launch_bounds__(T) ft_kernel(FitArgs a)
{
    extern __shared__ __align__(16) unsigned char ft_smem[];
    const FitLayout Lo = ft_layout(a.mmax, a.W, T);
    const FitCtx f = ft_bind(ft_smem, Lo);
    const int tid = threadIdx.x;
    __shared__ int s_item;
    for (;;) {
        if (tid == 0) s_item = atomicAdd(a.counter, 1);
        __syncthreads();
        const int item = s_item;
        __syncthreads();
        if (item >= a.ncand) break;
        const int cand = a.order[item];
        const int nb = a.node_off[cand];
        const int m = a.node_off[cand + 1] - nb;
        const int p = a.pcount[cand];
        for (int i = tid; i < m; i += T) f.rec[i] = a.rec[nb + i];
        if (tid < p) {
            const double c0 = a.c0[(size_t)cand * a.kmax + tid];
            f.c[tid] = c0;
            f.cf[tid] = (float)c0;
        }
        __syncthreads();
        double best = 0.0;
        int status = 1;
        if (a.valid[cand]) {
            int W = 4 * ((p + 1 + 3) / 4);
            const Syrk sy = ft_syrk_setup<T>(W);
            if (a.metric == FM_IMPLICIT) ft_lm_implicit<T>(a, f, m, p, W, sy, best, status);
            else ft_lm_standard<T>(a, f, m, p, W, sy, best, status);
        } else {
            best = INFINITY;
        }
        if (tid == 0) {
            for (int j = 0; j < p; ++j) a.outc[(size_t)cand * a.kmax + j] = f.c[j];
            a.outsse[cand] = best;
            a.outstatus[cand] = status;
        }
        __syncthreads();
    }
}

/* ---- gradients and the implicit score ------------------------------ */

/* One block per (candidate, 128-row tile): per-row value and gradients. */
template <int T>
__global__ void __launch_bounds__(T) ft_grad_kernel(FitArgs a, int want, int row0, int nrows,
                                                    int ntiles, float *value, float *out)
{
    extern __shared__ __align__(16) unsigned char smem[];
    const int cand = blockIdx.x / ntiles;
    const int tile = blockIdx.x % ntiles;
    const int tid = threadIdx.x;
    uint4 *rec = reinterpret_cast<uint4 *>(smem);
    float *cf = reinterpret_cast<float *>(rec + a.mmax);
    float *tape = cf + FT_MAX_CONST;
    double *g = reinterpret_cast<double *>(tape + (size_t)a.mmax * T);
    float *ig = reinterpret_cast<float *>(g + (size_t)FT_MAX_CONST * T);
    const int nb = a.node_off[cand];
    const int m = a.node_off[cand + 1] - nb;
    const int p = a.pcount[cand];
    for (int i = tid; i < m; i += T) rec[i] = a.rec[nb + i];
    if (tid < p) cf[tid] = (float)a.c0[(size_t)cand * a.kmax + tid];
    __syncthreads();
    if (!a.valid[cand]) return;
    const int r = tile * T + tid;
    if (r >= nrows) return;
    const int row = row0 + r;
    if (row >= a.n) return;
    const float val = ft_fwd_f<T>(rec, m, a.cols, a.npad, row, cf, tape + tid);
    for (int j = 0; j < FT_MAX_CONST; ++j) g[j * T + tid] = 0.0;
    for (int k = 0; k < a.v; ++k) ig[k * T + tid] = 0.0f;
    ft_bwd_f<T>(rec, m, tape + tid, g + tid, T, ig + tid, T);
    const size_t o = (size_t)cand * nrows + r;
    value[o] = val;
    if (want == 1) {
        for (int j = 0; j < a.kmax; ++j) out[o * a.kmax + j] = j < p ? (float)g[j * T + tid] : 0.0f;
    } else {
        for (int k = 0; k < a.v; ++k) out[o * a.v + k] = ig[k * T + tid];
    }
}

/* Implicit score per (candidate, tile of rows): partial sums of w * d and w. */
template <int T>
__global__ void __launch_bounds__(T) ft_implicit_score_kernel(FitArgs a, int ntiles,
                                                               int rows_per_tile,
                                                               double *partial, int *bad)
{
    extern __shared__ __align__(16) unsigned char smem[];
    const int cand = blockIdx.x / ntiles;
    const int tile = blockIdx.x % ntiles;
    const int tid = threadIdx.x;
    uint4 *rec = reinterpret_cast<uint4 *>(smem);
    float *cf = reinterpret_cast<float *>(rec + a.mmax);
    float *tape = cf + FT_MAX_CONST;
    float *ig = tape + (size_t)a.mmax * T;
    double *red = reinterpret_cast<double *>(ig + (size_t)a.v * T);
    const int nb = a.node_off[cand];
    const int m = a.node_off[cand + 1] - nb;
    const int p = a.pcount[cand];
    for (int i = tid; i < m; i += T) rec[i] = a.rec[nb + i];
    if (tid < p) cf[tid] = (float)a.c0[(size_t)cand * a.kmax + tid];
    __syncthreads();
    double sum = 0.0, wsum = 0.0;
    int isbad = !a.valid[cand];
    const int r0 = tile * rows_per_tile;
    const int r1 = min(a.n, r0 + rows_per_tile);
    if (!isbad) {
        for (int row = r0 + tid; row < r1; row += T) {
            const double wr = a.w ? a.w[row] : 1.0;
            if (!isfinite(wr) || wr < 0.0) {
                isbad = 1;
                continue;
            }
            if (wr == 0.0) continue;
            const float fv = ft_fwd_f<T>(rec, m, a.cols, a.npad, row, cf, tape + tid);
            for (int k = 0; k < a.v; ++k) ig[k * T + tid] = 0.0f;
            ft_bwd_f<T>(rec, m, tape + tid, nullptr, 0, ig + tid, T);
            double nsq = 0.0;
            bool ok = isfinite(fv);
            for (int k = 0; k < a.v; ++k) {
                const double gk = (double)ig[k * T + tid];
                if (!isfinite(gk)) ok = false;
                nsq += gk * gk;
            }
            const double norm = sqrt(nsq);
            if (!(isfinite(norm) && norm > 0.0)) ok = false;
            const double d = ok ? fabs((double)fv) / norm : 0.0;
            if (!ok || !isfinite(d)) {
                isbad = 1;
                continue;
            }
            sum += wr * d;
            wsum += wr;
        }
    }
    const int anybad = __syncthreads_or(isbad);
    red[tid] = sum;
    __syncthreads();
    for (int st = T / 2; st > 0; st >>= 1) {
        if (tid < st) red[tid] += red[tid + st];
        __syncthreads();
    }
    const double s = red[0];
    __syncthreads();
    red[tid] = wsum;
    __syncthreads();
    for (int st = T / 2; st > 0; st >>= 1) {
        if (tid < st) red[tid] += red[tid + st];
        __syncthreads();
    }
    if (tid == 0) {
        partial[2 * ((size_t)cand * ntiles + tile)] = s;
        partial[2 * ((size_t)cand * ntiles + tile) + 1] = red[0];
        if (anybad) atomicOr(&bad[cand], 1);
    }
}

__global__ void ft_implicit_finalize(int nprog, int ntiles, const double *partial, const int *bad,
                                     double *out, int *status)
{
    const int cand = blockIdx.x * blockDim.x + threadIdx.x;
    if (cand >= nprog) return;
    double s = 0.0, w = 0.0;
    for (int t = 0; t < ntiles; ++t) {
        s += partial[2 * ((size_t)cand * ntiles + t)];
        w += partial[2 * ((size_t)cand * ntiles + t) + 1];
    }
    if (bad[cand] || !(isfinite(w) && w > 0.0)) {
        out[cand] = INFINITY;
        status[cand] = 2;
    } else {
        out[cand] = s / w;
        status[cand] = 0;
    }
}

/* ---- host side -------------------------------------------------------- */

namespace {

/* A fit-record program is accepted when every record is an analytic operator,
   children precede parents, every node except the root has exactly one
   parent (a tree), constant slots are < p and input columns are < v. */
bool validate_records(const uint32_t *rec, int m, int p, int v)
{
    if (m <= 0 || m > FT_MAX_NODES) return false;
    std::vector<int> parents(m, 0);
    for (int i = 0; i < m; ++i) {
        const uint32_t op = rec[4 * i], k0 = rec[4 * i + 1], k1 = rec[4 * i + 2],
                       slot = rec[4 * i + 3];
        if (!ft_op_supported(op)) return false;
        if (op == OP_CONST) {
            if ((int)slot >= p || slot >= FT_MAX_CONST) return false;
        } else if (op == OP_VAR) {
            if ((int64_t)slot >= (int64_t)v) return false;
        } else {
            if ((int)k0 >= i) return false;
            parents[k0]++;
            if (ft_op_binary(op)) {
                if ((int)k1 >= i) return false;
                parents[k1]++;
            }
        }
    }
    for (int i = 0; i < m - 1; ++i)
        if (parents[i] != 1) return false;
    return parents[m - 1] == 0;
}

struct FitBatchPrep {
    std::vector<int> node_off, valid, order[4];
    int mmax[4] = {1, 1, 1, 1};
    int pmax[4] = {0, 0, 0, 0};
};

int bucket_of(int m)
{
    if (m <= 16) return 0;
    if (m <= 32) return 1;
    if (m <= 64) return 2;
    return 3;
}

void prep_batch(const unsigned int *off, const unsigned int *prog, const int *pcount, int nprog,
                int v, FitBatchPrep &b)
{
    b.node_off.resize(nprog + 1);
    b.valid.resize(nprog);
    std::vector<double> cost(nprog);
    for (int i = 0; i <= nprog; ++i) b.node_off[i] = (int)(off[i] / 4);
    for (int i = 0; i < nprog; ++i) {
        const int m = b.node_off[i + 1] - b.node_off[i];
        const int p = pcount[i];
        const bool ok = (off[i] % 4 == 0) && p >= 0 && p <= FT_MAX_CONST &&
                        validate_records(prog + off[i], m, p, v);
        b.valid[i] = ok ? 1 : 0;
        const int bk = bucket_of(m < 1 ? 1 : m);
        b.order[bk].push_back(i);
        b.mmax[bk] = std::max(b.mmax[bk], std::max(m, 1));
        b.pmax[bk] = std::max(b.pmax[bk], std::max(p, 0));
        cost[i] = (double)m * (1.0 + 0.05 * p);
    }
    for (int k = 0; k < 4; ++k)
        std::stable_sort(b.order[k].begin(), b.order[k].end(),
                         [&](int x, int y) { return cost[x] > cost[y]; });
}

int fit_occupancy(size_t smem)
{
    int blocks = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&blocks, ft_kernel<FT_THREADS>, FT_THREADS,
                                                      smem) != cudaSuccess) {
        cudaGetLastError();
        return 1;
    }
    return blocks < 1 ? 1 : blocks;
}

/* Launches the bucketed persistent fit on the context stream. `one_by_one`
   launches one single-block kernel per candidate (the plain arm). */
int launch_fit(RcCtx *c, FitArgs base, const FitBatchPrep &b, int *d_order, int *d_counters,
               int nprog, bool one_by_one)
{
    int obase = 0;
    for (int k = 0; k < 4; ++k) {
        const int nb = (int)b.order[k].size();
        if (nb == 0) continue;
        FitArgs a = base;
        a.mmax = b.mmax[k];
        a.W = 4 * ((b.pmax[k] + 1 + 3) / 4);
        const size_t smem = ft_layout(a.mmax, a.W, FT_THREADS).total;
        if (cudaFuncSetAttribute(ft_kernel<FT_THREADS>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 (int)smem) != cudaSuccess) {
            cudaGetLastError();
            return -1;
        }
        if (one_by_one) {
            for (int i = 0; i < nb; ++i) {
                a.order = d_order + obase + i;
                a.ncand = 1;
                a.counter = d_counters + 8 + obase + i;
                ft_kernel<FT_THREADS><<<1, FT_THREADS, smem, c->s>>>(a);
            }
        } else {
            a.order = d_order + obase;
            a.ncand = nb;
            a.counter = d_counters + k;
            int grid = c->sm_count * fit_occupancy(smem);
            if (grid > nb) grid = nb;
            ft_kernel<FT_THREADS><<<grid, FT_THREADS, smem, c->s>>>(a);
        }
        obase += nb;
    }
    (void)nprog;
    return cudaGetLastError() == cudaSuccess ? 0 : -1;
}

float fit_run(RcCtx *c, const unsigned int *prog, const unsigned int *off, const int *pcount,
              int nprog, int kmax, const double *c0, const int *gauge, int iters, int metric,
              int flags, double *outc, double *outsse, int *outstatus, int mode)
{
    (void)gauge;
    if (!c || !prog || !off || !pcount || !c0 || !outc || !outsse || !outstatus) return -1.0f;
    if (nprog <= 0 || kmax <= 0 || kmax > FT_MAX_CONST) return -1.0f;
    if (metric == FM_LOGISTIC && !c->has_tsign) return -1.0f;
    if (metric != FM_SQUARED && metric != FM_LOG_SQUASHED && metric != FM_ABSOLUTE &&
        metric != FM_LOGISTIC && metric != FM_IMPLICIT)
        return -1.0f;
    if (metric == FM_IMPLICIT && c->v > FT_IMPLICIT_MAXV) return -1.0f;
    for (int i = 0; i < nprog; ++i)
        if (pcount[i] < 0 || pcount[i] > kmax) return -1.0f;
    RcStats *st = &c->stats;
    double t = rc_now_ms();
    if (rc_ensure_f64(c) != 0) return -1.0f;
    FitBatchPrep b;
    prep_batch(off, prog, pcount, nprog, c->v, b);
    std::vector<int> order;
    order.reserve(nprog);
    for (int k = 0; k < 4; ++k) order.insert(order.end(), b.order[k].begin(), b.order[k].end());
    const size_t words = off[nprog];
    size_t cur = 0;
    const size_t o_rec = rc_take(&cur, sizeof(uint32_t) * words);
    const size_t o_noff = rc_take(&cur, sizeof(int) * (nprog + 1));
    const size_t o_p = rc_take(&cur, sizeof(int) * nprog);
    const size_t o_c0 = rc_take(&cur, sizeof(double) * (size_t)nprog * kmax);
    const size_t o_valid = rc_take(&cur, sizeof(int) * nprog);
    const size_t o_order = rc_take(&cur, sizeof(int) * nprog);
    const size_t in_end = rc_take(&cur, 0);
    const size_t o_c = rc_take(&cur, sizeof(double) * (size_t)nprog * kmax);
    const size_t o_sse = rc_take(&cur, sizeof(double) * nprog);
    const size_t o_status = rc_take(&cur, sizeof(int) * nprog);
    const size_t io_end = rc_take(&cur, 0);
    const size_t o_cnt = rc_take(&cur, sizeof(int) * (8 + nprog));
    const size_t dev_end = rc_take(&cur, 0);
    if (rc_reserve(c, dev_end, io_end) != 0) return -1.0f;
    st->alloc_ms += rc_now_ms() - t;
    unsigned char *dev = c->dev, *host = c->host;
    t = rc_now_ms();
    memcpy(host + o_rec, prog, sizeof(uint32_t) * words);
    memcpy(host + o_noff, b.node_off.data(), sizeof(int) * (nprog + 1));
    memcpy(host + o_p, pcount, sizeof(int) * nprog);
    memcpy(host + o_c0, c0, sizeof(double) * (size_t)nprog * kmax);
    memcpy(host + o_valid, b.valid.data(), sizeof(int) * nprog);
    memcpy(host + o_order, order.data(), sizeof(int) * nprog);
    /* outputs start as the inputs so untouched slots echo c0 */
    memcpy(host + o_c, c0, sizeof(double) * (size_t)nprog * kmax);
    cudaMemcpyAsync(dev, host, io_end, cudaMemcpyHostToDevice, c->s);
    cudaMemsetAsync(dev + o_cnt, 0, sizeof(int) * (8 + nprog), c->s);
    st->h2d_ms += rc_now_ms() - t;
    st->h2d_bytes += io_end;

    FitArgs a;
    memset(&a, 0, sizeof(a));
    a.cols = c->d_cols;
    a.y = c->d_y;
    a.tsign = c->d_tsign;
    a.cols64 = c->d_cols64;
    a.y64 = c->d_y64;
    a.tsign64 = c->d_tsign64;
    a.w = c->d_w64;
    a.n = c->n;
    a.npad = c->npad;
    a.v = c->v;
    a.rec = reinterpret_cast<const uint4 *>(dev + o_rec);
    a.node_off = reinterpret_cast<const int *>(dev + o_noff);
    a.pcount = reinterpret_cast<const int *>(dev + o_p);
    a.kmax = kmax;
    a.c0 = reinterpret_cast<const double *>(dev + o_c0);
    a.valid = reinterpret_cast<const int *>(dev + o_valid);
    a.iters = iters;
    a.metric = metric;
    a.flags = flags;
    a.outc = reinterpret_cast<double *>(dev + o_c);
    a.outsse = reinterpret_cast<double *>(dev + o_sse);
    a.outstatus = reinterpret_cast<int *>(dev + o_status);
    t = rc_now_ms();
    cudaEventRecord(c->t0, c->s);
    const int rc = launch_fit(c, a, b, reinterpret_cast<int *>(dev + o_order),
                              reinterpret_cast<int *>(dev + o_cnt), nprog, mode == 1);
    cudaEventRecord(c->t1, c->s);
    st->launch_ms += rc_now_ms() - t;
    if (rc != 0) {
        cudaStreamSynchronize(c->s);
        cudaGetLastError();
        return -1.0f;
    }
    t = rc_now_ms();
    cudaMemcpyAsync(host + in_end, dev + in_end, io_end - in_end, cudaMemcpyDeviceToHost, c->s);
    if (rc_finish(c) != 0) return -1.0f;
    st->sync_ms += rc_now_ms() - t;
    memcpy(outc, host + o_c, sizeof(double) * (size_t)nprog * kmax);
    memcpy(outsse, host + o_sse, sizeof(double) * nprog);
    memcpy(outstatus, host + o_status, sizeof(int) * nprog);
    st->d2h_bytes += io_end - in_end;
    float ms = 0.0f;
    cudaEventElapsedTime(&ms, c->t0, c->t1);
    st->kernel_ms = ms;
    st->batch = nprog;
    c->warm = 1;
    c->batches++;
    return ms;
}

}  // namespace

extern "C" {

float rc_fit_batch(void *ctx, const unsigned int *prog, const unsigned int *off, const int *pcount,
                   int nprog, int kmax, const double *c0, const int *gauge, int iters, int metric,
                   double *outc, double *outsse, int *outstatus)
{
    if (metric == FM_IMPLICIT) return -1.0f; /* additive code: rc_fit_batch_fused only */
    return fit_run((RcCtx *)ctx, prog, off, pcount, nprog, kmax, c0, gauge, iters, metric, 0, outc,
                   outsse, outstatus, 0);
}

float rc_fit_batch_fused(void *ctx, const unsigned int *prog, const unsigned int *off,
                         const int *pcount, int nprog, int kmax, const double *c0,
                         const int *gauge, int iters, int metric, int flags, double *outc,
                         double *outsse, int *outstatus)
{
    return fit_run((RcCtx *)ctx, prog, off, pcount, nprog, kmax, c0, gauge, iters, metric, flags,
                   outc, outsse, outstatus, 0);
}

float rc_fit_batch_plain(void *ctx, const unsigned int *prog, const unsigned int *off,
                         const int *pcount, int nprog, int kmax, const double *c0,
                         const int *gauge, int iters, int metric, double *outc, double *outsse,
                         int *outstatus)
{
    return fit_run((RcCtx *)ctx, prog, off, pcount, nprog, kmax, c0, gauge, iters, metric, 0, outc,
                   outsse, outstatus, 1);
}

int rc_fit_kernel_info(int kmax, int *threads, int *smem_bytes, int *max_constants)
{
    if (!threads || !smem_bytes || !max_constants) return -1;
    if (kmax > FT_MAX_CONST || kmax < 0) return -1;
    const int W = 4 * ((kmax + 1 + 3) / 4);
    *threads = FT_THREADS;
    *smem_bytes = (int)ft_layout(FT_MAX_NODES_ABI, W, FT_THREADS).total;
    *max_constants = FT_MAX_CONST;
    return 0;
}

int rc_grad_batch(void *ctx, const unsigned int *prog, const unsigned int *off, const int *pcount,
                  int nprog, int kmax, const double *c, int want, int row0, int nrows, float *value,
                  float *out)
{
    RcCtx *rc = (RcCtx *)ctx;
    if (!rc || !prog || !off || !pcount || !c || !value || !out) return -1;
    if (nprog <= 0 || kmax <= 0 || kmax > FT_MAX_CONST || (want != 1 && want != 2)) return -1;
    if (row0 < 0 || nrows <= 0 || row0 + nrows > rc->n) return -1;
    FitBatchPrep b;
    prep_batch(off, prog, pcount, nprog, rc->v, b);
    int mmax = 1;
    for (int k = 0; k < 4; ++k) mmax = std::max(mmax, b.mmax[k]);
    const int width = want == 1 ? kmax : rc->v;
    const size_t words = off[nprog];
    size_t cur = 0;
    const size_t o_rec = rc_take(&cur, sizeof(uint32_t) * words);
    const size_t o_noff = rc_take(&cur, sizeof(int) * (nprog + 1));
    const size_t o_p = rc_take(&cur, sizeof(int) * nprog);
    const size_t o_c = rc_take(&cur, sizeof(double) * (size_t)nprog * kmax);
    const size_t o_valid = rc_take(&cur, sizeof(int) * nprog);
    const size_t in_end = rc_take(&cur, 0);
    const size_t o_val = rc_take(&cur, sizeof(float) * (size_t)nprog * nrows);
    const size_t o_out = rc_take(&cur, sizeof(float) * (size_t)nprog * nrows * width);
    const size_t io_end = rc_take(&cur, 0);
    if (rc_reserve(rc, io_end, io_end) != 0) return -1;
    unsigned char *dev = rc->dev, *host = rc->host;
    memcpy(host + o_rec, prog, sizeof(uint32_t) * words);
    memcpy(host + o_noff, b.node_off.data(), sizeof(int) * (nprog + 1));
    memcpy(host + o_p, pcount, sizeof(int) * nprog);
    memcpy(host + o_c, c, sizeof(double) * (size_t)nprog * kmax);
    memcpy(host + o_valid, b.valid.data(), sizeof(int) * nprog);
    cudaMemcpyAsync(dev, host, in_end, cudaMemcpyHostToDevice, rc->s);
    cudaMemsetAsync(dev + in_end, 0, io_end - in_end, rc->s);
    FitArgs a;
    memset(&a, 0, sizeof(a));
    a.cols = rc->d_cols;
    a.n = rc->n;
    a.npad = rc->npad;
    a.v = rc->v;
    a.rec = reinterpret_cast<const uint4 *>(dev + o_rec);
    a.node_off = reinterpret_cast<const int *>(dev + o_noff);
    a.pcount = reinterpret_cast<const int *>(dev + o_p);
    a.kmax = kmax;
    a.c0 = reinterpret_cast<const double *>(dev + o_c);
    a.valid = reinterpret_cast<const int *>(dev + o_valid);
    a.mmax = mmax;
    const int T = 128;
    const int ntiles = (nrows + T - 1) / T;
    const size_t smem = sizeof(uint4) * mmax + sizeof(float) * FT_MAX_CONST +
                        sizeof(float) * (size_t)mmax * T + sizeof(double) * FT_MAX_CONST * T +
                        sizeof(float) * (size_t)rc->v * T + 64;
    if (cudaFuncSetAttribute(ft_grad_kernel<128>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)smem) != cudaSuccess) {
        cudaGetLastError();
        return -1;
    }
    ft_grad_kernel<128><<<nprog * ntiles, T, smem, rc->s>>>(
        a, want, row0, nrows, ntiles, reinterpret_cast<float *>(dev + o_val),
        reinterpret_cast<float *>(dev + o_out));
    cudaMemcpyAsync(host + in_end, dev + in_end, io_end - in_end, cudaMemcpyDeviceToHost, rc->s);
    if (rc_finish(rc) != 0) return -1;
    memcpy(value, host + o_val, sizeof(float) * (size_t)nprog * nrows);
    memcpy(out, host + o_out, sizeof(float) * (size_t)nprog * nrows * width);
    return 0;
}

float rc_implicit_score_batch(void *ctx, const unsigned int *prog, const unsigned int *off,
                              const int *pcount, int nprog, int kmax, const double *c, double *out,
                              int *status)
{
    RcCtx *rc = (RcCtx *)ctx;
    if (!rc || !prog || !off || !pcount || !c || !out || !status) return -1.0f;
    if (nprog <= 0 || kmax <= 0 || kmax > FT_MAX_CONST || rc->n <= 0) return -1.0f;
    RcStats *st = &rc->stats;
    FitBatchPrep b;
    prep_batch(off, prog, pcount, nprog, rc->v, b);
    int mmax = 1;
    for (int k = 0; k < 4; ++k) mmax = std::max(mmax, b.mmax[k]);
    const int T = 128;
    const int rows_per_tile = 16384;
    const int ntiles = (rc->n + rows_per_tile - 1) / rows_per_tile;
    const size_t words = off[nprog];
    size_t cur = 0;
    const size_t o_rec = rc_take(&cur, sizeof(uint32_t) * words);
    const size_t o_noff = rc_take(&cur, sizeof(int) * (nprog + 1));
    const size_t o_p = rc_take(&cur, sizeof(int) * nprog);
    const size_t o_c = rc_take(&cur, sizeof(double) * (size_t)nprog * kmax);
    const size_t o_valid = rc_take(&cur, sizeof(int) * nprog);
    const size_t in_end = rc_take(&cur, 0);
    const size_t o_out = rc_take(&cur, sizeof(double) * nprog);
    const size_t o_status = rc_take(&cur, sizeof(int) * nprog);
    const size_t io_end = rc_take(&cur, 0);
    const size_t o_part = rc_take(&cur, sizeof(double) * 2 * (size_t)nprog * ntiles);
    const size_t o_bad = rc_take(&cur, sizeof(int) * nprog);
    const size_t dev_end = rc_take(&cur, 0);
    if (rc_reserve(rc, dev_end, io_end) != 0) return -1.0f;
    unsigned char *dev = rc->dev, *host = rc->host;
    double t = rc_now_ms();
    memcpy(host + o_rec, prog, sizeof(uint32_t) * words);
    memcpy(host + o_noff, b.node_off.data(), sizeof(int) * (nprog + 1));
    memcpy(host + o_p, pcount, sizeof(int) * nprog);
    memcpy(host + o_c, c, sizeof(double) * (size_t)nprog * kmax);
    memcpy(host + o_valid, b.valid.data(), sizeof(int) * nprog);
    cudaMemcpyAsync(dev, host, in_end, cudaMemcpyHostToDevice, rc->s);
    cudaMemsetAsync(dev + o_bad, 0, sizeof(int) * nprog, rc->s);
    st->h2d_ms += rc_now_ms() - t;
    FitArgs a;
    memset(&a, 0, sizeof(a));
    a.cols = rc->d_cols;
    a.w = rc->d_w64;
    a.n = rc->n;
    a.npad = rc->npad;
    a.v = rc->v;
    a.rec = reinterpret_cast<const uint4 *>(dev + o_rec);
    a.node_off = reinterpret_cast<const int *>(dev + o_noff);
    a.pcount = reinterpret_cast<const int *>(dev + o_p);
    a.kmax = kmax;
    a.c0 = reinterpret_cast<const double *>(dev + o_c);
    a.valid = reinterpret_cast<const int *>(dev + o_valid);
    a.mmax = mmax;
    const size_t smem = sizeof(uint4) * mmax + sizeof(float) * FT_MAX_CONST +
                        sizeof(float) * (size_t)mmax * T + sizeof(float) * (size_t)rc->v * T +
                        sizeof(double) * T + 64;
    if (cudaFuncSetAttribute(ft_implicit_score_kernel<128>,
                             cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) != cudaSuccess) {
        cudaGetLastError();
        return -1.0f;
    }
    cudaEventRecord(rc->t0, rc->s);
    ft_implicit_score_kernel<128><<<nprog * ntiles, T, smem, rc->s>>>(
        a, ntiles, rows_per_tile, reinterpret_cast<double *>(dev + o_part),
        reinterpret_cast<int *>(dev + o_bad));
    ft_implicit_finalize<<<(nprog + 127) / 128, 128, 0, rc->s>>>(
        nprog, ntiles, reinterpret_cast<const double *>(dev + o_part),
        reinterpret_cast<const int *>(dev + o_bad), reinterpret_cast<double *>(dev + o_out),
        reinterpret_cast<int *>(dev + o_status));
    cudaEventRecord(rc->t1, rc->s);
    if (cudaGetLastError() != cudaSuccess) {
        cudaStreamSynchronize(rc->s);
        return -1.0f;
    }
    cudaMemcpyAsync(host + in_end, dev + in_end, io_end - in_end, cudaMemcpyDeviceToHost, rc->s);
    if (rc_finish(rc) != 0) return -1.0f;
    memcpy(out, host + o_out, sizeof(double) * nprog);
    memcpy(status, host + o_status, sizeof(int) * nprog);
    float ms = 0.0f;
    cudaEventElapsedTime(&ms, rc->t0, rc->t1);
    st->kernel_ms = ms;
    return ms;
}

}  // extern "C"
