#pragma once
/*
 * Device building blocks of the batched fit: per-row forward and reverse
 * sweeps over fit records (f32 and f64), the per-row objective pieces, the
 * block reductions, the 4x4 register-blocked SYRK of the augmented Gram, the
 * damped solves (a warp-cooperative Cholesky and the implicit arm's Gaussian
 * elimination), and the implicit-metric residual.
 *
 * Semantics follow the reference's batched fit (my-version/src/cuda/eval.cu:
 * 1106-2606) and the CPU fitter it stands in for (my-version/src/fit.rs:
 * 1453-1827, :2534-2624, :3092-3170; my-version/src/implicit.rs:68-409).
 */
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
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

/* ---- the damped solve on one warp --------------------------------------

   The step of one LM iteration solves (S + lambda diag S + 1e-12 I) u = -D^-1 g
   for the Jacobi-equilibrated normal matrix S = D^-1 (J^T J) D^-1,
   D = sqrt(diag J^T J), and returns delta = D^-1 u. The labels are the
   reference kernel's (eval.cu:1873-1949): 1 when a diagonal entry of J^T J is
   negative or not finite, a scaled entry is not finite, or the damped factor
   breaks down (pivot <= 1e-18); 4 (rank deficient, the step is still
   returned) when the undamped factor of S breaks down or ln det S <
   ln 1e-12; else 0. One case follows the CPU fit instead (fit.rs:1686-1727):
   a constant whose Jacobian column is exactly zero (a zero diagonal; its
   gradient is then zero too) is held where it is, as the CPU's unscaled solve
   does through its 1e-12 ridge, and the others' step is solved without it
   (label 4). The reference kernel gives up the whole step there (label 1),
   and in f32 such columns are common (a saturated logistic or tanh, an exp
   that underflows), so its LM stopped where the CPU's went on.

   Layout: lane i (< p) keeps row i of both Cholesky factors of S, the
   undamped one (for the rank label) and the damped one (for the step), in
   registers. Column k of both factors is one step: each lane at or below the
   diagonal finishes its entry (i, k) from the k entries of its own row and
   lane k's row, which arrive by shuffles; the pivot is then broadcast from
   lane k. The triangular solves are columns too: lane k finishes its unknown
   and broadcasts it; the forward pass updates the lanes below with their own
   row entry, the backward pass with lane k's row entry. Every lane of the
   warp calls this with the same arguments; lanes >= p follow the same
   uniform branches. */

#define FT_FULL_MASK 0xffffffffu

__device__ __forceinline__ int ft_solve_warp(const double *jtj, const double *jtr, double lambda,
                                             int p, double *delta)
{
    const int lane = threadIdx.x & 31;
    const bool mine = lane < p;
    const double aii = mine ? jtj[lane * (lane + 1) / 2 + lane] : 1.0;
    if (__any_sync(FT_FULL_MASK, aii < 0.0 || !isfinite(aii))) return 1;
    /* a zero column: its row and column of S become the unit row and its
       right-hand side zero, so its step is zero */
    const bool held = mine && aii == 0.0;
    const bool any_held = __any_sync(FT_FULL_MASK, held);
    const double di = held ? 1.0 : sqrt(aii);

    double u[FT_MAX_CONST], l[FT_MAX_CONST];
    bool nonfinite = false;
#pragma unroll
    for (int j = 0; j < FT_MAX_CONST; ++j) {
        const double dj = __shfl_sync(FT_FULL_MASK, di, j);
        const bool hj = __shfl_sync(FT_FULL_MASK, held ? 1 : 0, j) != 0;
        double sij = 0.0;
        if (mine && j <= lane) {
            if (held || hj) sij = (j == lane) ? 1.0 : 0.0;
            else sij = jtj[lane * (lane + 1) / 2 + j] / (di * dj);
            nonfinite = nonfinite || !isfinite(sij);
        }
        u[j] = sij;
        l[j] = sij;
    }
    if (__any_sync(FT_FULL_MASK, nonfinite)) return 1;

    bool broke = false; /* the undamped factor broke down */
    double lndet = 0.0; /* ln det S from the undamped pivots, summed on every lane */
#pragma unroll
    for (int k = 0; k < FT_MAX_CONST; ++k) {
        if (k >= p) break;
        double su = u[k], sd = l[k];
        if (lane == k) sd = sd * (1.0 + lambda) + 1e-12;
#pragma unroll
        for (int m = 0; m < k; ++m) {
            su -= u[m] * __shfl_sync(FT_FULL_MASK, u[m], k);
            sd -= l[m] * __shfl_sync(FT_FULL_MASK, l[m], k);
        }
        const double pu = __shfl_sync(FT_FULL_MASK, su, k);
        const double pd = __shfl_sync(FT_FULL_MASK, sd, k);
        if (!(pd > 1e-18) || !isfinite(pd)) return 1;
        if (!broke && (!(pu > 0.0) || !isfinite(pu))) broke = true;
        if (!broke) lndet += log(pu);
        const double ru = broke ? 1.0 : sqrt(pu), rd = sqrt(pd);
        if (lane == k) {
            u[k] = ru;
            l[k] = rd;
        } else if (lane > k) {
            u[k] = su / ru;
            l[k] = sd / rd;
        }
    }
    const int label =
        (any_held || broke || !isfinite(lndet) || lndet < FT_LN_DET_FLOOR) ? 4 : 0;

    /* forward: L y = -D^-1 g */
    double yv = (mine && !held) ? -jtr[lane] / di : 0.0;
#pragma unroll
    for (int k = 0; k < FT_MAX_CONST; ++k) {
        if (k >= p) break;
        if (lane == k) yv = yv / l[k];
        const double yk = __shfl_sync(FT_FULL_MASK, yv, k);
        if (lane > k) yv -= l[k] * yk;
    }
    /* backward: L^T x = y; lane k's row holds column k of L^T */
#pragma unroll
    for (int k = FT_MAX_CONST - 1; k >= 0; --k) {
        if (k >= p) continue;
        if (lane == k) yv = yv / l[k];
        const double xk = __shfl_sync(FT_FULL_MASK, yv, k);
#pragma unroll
        for (int j = 0; j < k; ++j) {
            const double lkj = __shfl_sync(FT_FULL_MASK, l[j], k);
            if (lane == j) yv -= lkj * xk;
        }
    }
    if (mine) delta[lane] = yv / di;
    __syncwarp();
    return label;
}

/* Gaussian elimination with partial pivoting on (A + lambda diag A + 1e-12 I)
   (implicit.rs:215-253). `M` is p x (p+1) scratch. Returns 0 or 1 (singular). */
__device__ inline int ft_gauss_solve(const double *jtj, const double *jtr, double lambda, int p,
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

/* First and second local partials of one node (f64): d0, d1 as
   ft_partials_d, and d00 = d2 node / da2, d01 = d2 node / da db,
   d11 = d2 node / db2. A `pow` with a non-positive base passes nothing. */
__device__ __forceinline__ void ft_partials2_d(unsigned op, double x, double y, double &d0,
                                               double &d1, double &d00, double &d01,
                                               double &d11)
{
    d0 = d1 = d00 = d01 = d11 = 0.0;
    switch (op) {
        case OP_NEG: d0 = -1.0; break;
        case OP_EXP: d0 = exp(x); d00 = d0; break;
        case OP_LOG: d0 = 1.0 / x; d00 = -d0 * d0; break;
        case OP_ABS: d0 = x >= 0.0 ? 1.0 : -1.0; break;
        case OP_SQRT: {
            const double s = sqrt(x);
            d0 = 1.0 / (2.0 * s);
            d00 = -d0 / (2.0 * x);
        } break;
        case OP_SIN: {
            double s, c;
            sincos(x, &s, &c);
            d0 = c;
            d00 = -s;
        } break;
        case OP_COS: {
            double s, c;
            sincos(x, &s, &c);
            d0 = -s;
            d00 = -c;
        } break;
        case OP_TAN: {
            double s, c;
            sincos(x, &s, &c);
            d0 = 1.0 / (c * c);
            d00 = 2.0 * s / (c * c * c);
        } break;
        case OP_SINH: d0 = cosh(x); d00 = sinh(x); break;
        case OP_COSH: d0 = sinh(x); d00 = cosh(x); break;
        case OP_TANH: {
            const double t = tanh(x);
            d0 = 1.0 - t * t;
            d00 = -2.0 * t * d0;
        } break;
        case OP_SIG: {
            const double s = 1.0 / (1.0 + exp(-x));
            d0 = s * (1.0 - s);
            d00 = d0 * (1.0 - 2.0 * s);
        } break;
        case OP_GAUSS: {
            const double e = exp(-x * x);
            d0 = (-2.0 * x) * e;
            d00 = (4.0 * x * x - 2.0) * e;
        } break;
        case OP_SQUARE: d0 = 2.0 * x; d00 = 2.0; break;
        case OP_CUBE: d0 = 3.0 * x * x; d00 = 6.0 * x; break;
        case OP_ERF: d0 = 1.1283791670955126 * exp(-x * x); d00 = -2.0 * x * d0; break;
        case OP_ERFC: d0 = -1.1283791670955126 * exp(-x * x); d00 = -2.0 * x * d0; break;
        case OP_ADD: d0 = 1.0; d1 = 1.0; break;
        case OP_SUB: d0 = 1.0; d1 = -1.0; break;
        case OP_MUL: d0 = y; d1 = x; d01 = 1.0; break;
        case OP_DIV: {
            const double iy = 1.0 / y;
            d0 = iy;
            d1 = -x / (y * y);
            d01 = -iy * iy;
            d11 = 2.0 * x * iy * iy * iy;
        } break;
        case OP_POW:
            if (x > 0.0) {
                const double lx = log(x), pm1 = pow(x, y - 1.0), pw = pow(x, y);
                d0 = y * pm1;
                d1 = pw * lx;
                d00 = y * (y - 1.0) * pow(x, y - 2.0);
                d01 = pm1 * (1.0 + y * lx);
                d11 = pw * lx * lx;
            }
            break;
        default: break;
    }
}

/* a * d with a zero factor passing nothing (an adjoint or tangent of zero
   does not meet an infinite partial). */
__device__ __forceinline__ double ft_mul0(double a, double d) { return a == 0.0 ? 0.0 : a * d; }

/* ---- the implicit metric (implicit.rs:68-409) ---------------------------
 * Per row: d = f / ||grad_x f|| (f64 forward + input adjoint); a row with a
 * non-finite value or gradient, or a zero gradient norm, makes the whole
 * evaluation undefined. The LM's Jacobian is exact (below) where the
 * reference CPU arm takes central differences of d with h = 1e-6 (1 +
 * |c_j|). */

#define FT_IMPLICIT_MAXV 16

/* Child references of the compact records the Jacobian sweep runs over:
   an internal node's tape slot, or a tagged leaf (an input column or a
   constant slot) whose value and tangent are read from the row's inputs,
   the constants and the input gradient instead of being taped. */
#define IJ_LEAF 0x80000000u
#define IJ_CONST 0x40000000u
#define IJ_INDEX 0x0000ffffu

/* Compact a candidate's fit records in place for the Jacobian sweep: the
   internal nodes only, in post-order (record k is tape slot k), each child
   a tape slot or a tagged leaf; `ref` is scratch for m entries. Run by one
   thread. Returns the number of internal records (0 for a lone leaf). */
__device__ __forceinline__ int ij_compact(uint4 *rec, int m, unsigned *ref)
{
    int k = 0;
    for (int i = 0; i < m; ++i) {
        const uint4 r = rec[i];
        if (r.x == OP_CONST) {
            ref[i] = IJ_LEAF | IJ_CONST | r.w;
        } else if (r.x == OP_VAR) {
            ref[i] = IJ_LEAF | r.w;
        } else {
            rec[k] = make_uint4(r.x, ref[r.y], ft_op_binary(r.x) ? ref[r.z] : 0u, 0u);
            ref[i] = (unsigned)k++;
        }
    }
    return k;
}

template <int TS>
__device__ __forceinline__ double ij_val(unsigned ref, const double *vt, const double *x,
                                         const double *c)
{
    if (ref & IJ_LEAF) return (ref & IJ_CONST) ? c[ref & IJ_INDEX] : x[ref & IJ_INDEX];
    return vt[ref * TS];
}

/* A leaf's tangent along x' = g: g[col] for an input, 0 for a constant. */
template <int TS>
__device__ __forceinline__ double ij_tan(unsigned ref, const double *tt,
                                         const double (&ig)[FT_IMPLICIT_MAXV])
{
    if (!(ref & IJ_LEAF)) return tt[ref * TS];
    if (ref & IJ_CONST) return 0.0;
    double t = 0.0;
#pragma unroll
    for (int k = 0; k < FT_IMPLICIT_MAXV; ++k)
        if ((int)(ref & IJ_INDEX) == k) t = ig[k];
    return t;
}

/* Hand a first-order adjoint to a child: an internal child's tape slot, a
   constant's Jacobian entry, an input's gradient. */
template <int TS>
__device__ __forceinline__ void ij_put(unsigned ref, double v, double *tt, double *jrow,
                                       double (&ig)[FT_IMPLICIT_MAXV])
{
    if (!(ref & IJ_LEAF)) {
        tt[ref * TS] = v;
    } else if (ref & IJ_CONST) {
        jrow[ref & IJ_INDEX] += v;
    } else {
#pragma unroll
        for (int k = 0; k < FT_IMPLICIT_MAXV; ++k)
            if ((int)(ref & IJ_INDEX) == k) ig[k] += v;
    }
}

/* The implicit residual of one row and its exact Jacobian row (f64):
   d = f / ||g||, g = grad_x f, and for each constant
     dd/dc_j = (df/dc_j) / ||g|| - f (g . dg/dc_j) / ||g||^3,
   where g . dg/dc_j = d/dc_j (grad_x f . v) at v = g held fixed, a
   Hessian-vector product of f. Four sweeps over the records:
   1. forward values (tape `vt`);
   2. reverse: the input adjoint g and df/dc (into jrow), each node's
      adjoint in `tt` (the values in `vt` stay); once a unary node's
      adjoint is consumed, its slot keeps the node's partial;
   3. forward tangents along x' = g over the stored values (into `tt`);
   4. reverse of the tangent: each node's slots switch from (value,
      tangent) to (adjoint u, second-order adjoint w) when its parent is
      processed; a constant's w is g . dg/dc_j.
   jrow[j] receives sqrt(w_row) dd/dc_j for j < p. Returns false when the
   row is undefined (non-finite value, gradient or Jacobian entry, or a
   zero gradient): the rows the cost sweep rejects, plus a non-finite
   Jacobian entry. The sweeps run over the compact records of ij_compact:
   only internal nodes own tape slots (about half of a tree's nodes), so
   both tapes take half the shared memory; a leaf's adjoint is applied to
   its gradient entry when its parent is processed (for an input shared by
   several leaves that changes the order of its gradient's additions, not
   the sum's meaning). */
template <int TS>
__device__ bool ft_implicit_jac(const uint4 *ir, int ni, const double *x, int v, const double *c,
                                int p, double sw, double *vt, double *tt, double &d, double *jrow)
{
    /* a lone constant has no gradient; a lone input holds no constant */
    if (ni == 0) return false;
    /* 1: values of the internal nodes */
    double fv = 0.0;
    for (int k = 0; k < ni; ++k) {
        const uint4 r = ir[k];
        const double a = ij_val<TS>(r.y, vt, x, c);
        const double b = ft_op_binary(r.x) ? ij_val<TS>(r.z, vt, x, c) : 0.0;
        fv = ft_value_d(r.x, a, b);
        vt[k * TS] = fv;
    }
    if (!isfinite(fv)) return false;
    for (int j = 0; j < p; ++j) jrow[j] = 0.0;
    double ig[FT_IMPLICIT_MAXV];
#pragma unroll
    for (int k = 0; k < FT_IMPLICIT_MAXV; ++k) ig[k] = 0.0;
    /* 2: reverse; a leaf's adjoint goes straight to its gradient entry */
    tt[(ni - 1) * TS] = 1.0;
    for (int k = ni - 1; k >= 0; --k) {
        const uint4 r = ir[k];
        const double a = tt[k * TS];
        const double xx = ij_val<TS>(r.y, vt, x, c);
        if (!ft_op_binary(r.x)) {
            /* a unary node's own partial goes to its (now consumed) slot for
               the tangent pass */
            double d0, d1;
            ft_partials_d(r.x, xx, 0.0, d0, d1);
            ij_put<TS>(r.y, a != 0.0 ? a * d0 : 0.0, tt, jrow, ig);
            tt[k * TS] = d0;
            continue;
        }
        const double yy = ij_val<TS>(r.z, vt, x, c);
        double c0 = 0.0, c1 = 0.0;
        if (a != 0.0 && !(r.x == OP_POW && !(xx > 0.0))) {
            double d0, d1;
            ft_partials_d(r.x, xx, yy, d0, d1);
            c0 = a * d0;
            c1 = a * d1;
        }
        ij_put<TS>(r.y, c0, tt, jrow, ig);
        ij_put<TS>(r.z, c1, tt, jrow, ig);
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
    if (!isfinite(d)) return false;
    /* 3: tangents along x' = g over the stored values (a node's adjoint in
       tt is replaced by its tangent; its children's are tangents already) */
    for (int k = 0; k < ni; ++k) {
        const uint4 r = ir[k];
        double tan = 0.0;
        if (!ft_op_binary(r.x)) {
            const double ta = ij_tan<TS>(r.y, tt, ig);
            if (ta != 0.0) tan = ft_mul0(ta, tt[k * TS]) + 0.0;
        } else {
            const double a = ij_val<TS>(r.y, vt, x, c), ta = ij_tan<TS>(r.y, tt, ig);
            const double b = ij_val<TS>(r.z, vt, x, c), tb = ij_tan<TS>(r.z, tt, ig);
            if (!(r.x == OP_POW && !(a > 0.0)) && (ta != 0.0 || tb != 0.0)) {
                double d0, d1;
                ft_partials_d(r.x, a, b, d0, d1);
                tan = ft_mul0(ta, d0) + ft_mul0(tb, d1);
            }
        }
        tt[k * TS] = tan;
    }
    /* 4: reverse of the tangent; u = first-order adjoint, w = second; a
       constant's w is g . dg/dc_j */
    const double s1 = sw / norm, s3 = sw * fv / (norm * norm * norm);
    for (int j = 0; j < p; ++j) jrow[j] *= s1;
    vt[(ni - 1) * TS] = 1.0;
    tt[(ni - 1) * TS] = 0.0;
    for (int k = ni - 1; k >= 0; --k) {
        const uint4 r = ir[k];
        const double u = vt[k * TS], w = tt[k * TS];
        const bool bin = ft_op_binary(r.x);
        const double a = ij_val<TS>(r.y, vt, x, c), ta = ij_tan<TS>(r.y, tt, ig);
        const double b = bin ? ij_val<TS>(r.z, vt, x, c) : 0.0;
        const double tb = bin ? ij_tan<TS>(r.z, tt, ig) : 0.0;
        double u0 = 0.0, u1 = 0.0, w0 = 0.0, w1 = 0.0;
        if ((u != 0.0 || w != 0.0) && !(r.x == OP_POW && !(a > 0.0))) {
            double d0, d1, d00, d01, d11;
            ft_partials2_d(r.x, a, b, d0, d1, d00, d01, d11);
            if (u != 0.0) {
                u0 = u * d0;
                u1 = u * d1;
            }
            const double h0 = ft_mul0(ta, d00) + ft_mul0(tb, d01);
            const double h1 = ft_mul0(ta, d01) + ft_mul0(tb, d11);
            w0 = ft_mul0(w, d0) + ft_mul0(u, h0);
            w1 = ft_mul0(w, d1) + ft_mul0(u, h1);
        }
        if (!(r.y & IJ_LEAF)) {
            vt[r.y * TS] = u0;
            tt[r.y * TS] = w0;
        } else if (r.y & IJ_CONST) {
            jrow[r.y & IJ_INDEX] -= ft_mul0(w0, s3);
        }
        if (bin) {
            if (!(r.z & IJ_LEAF)) {
                vt[r.z * TS] = u1;
                tt[r.z * TS] = w1;
            } else if (r.z & IJ_CONST) {
                jrow[r.z & IJ_INDEX] -= ft_mul0(w1, s3);
            }
        }
    }
    for (int j = 0; j < p; ++j)
        if (!isfinite(jrow[j])) return false;
    return true;
}


