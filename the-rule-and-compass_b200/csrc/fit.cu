/*
 * Batched Levenberg-Marquardt / IRLS constant fitting with a fused
 * forward + reverse-mode adjoint sweep, driven as a fixed sequence of device
 * steps captured once in a CUDA graph.
 *
 * Semantics follow the reference's batched fit (my-version/src/cuda/eval.cu:
 * 2264-2606 `fit_kernel`: the LM/IRLS control flow, lambda law, Armijo
 * halvings, f64 re-baseline and polish, status labels 0-8) and the CPU fitter
 * it stands in for (my-version/src/fit.rs:2534-2624 `fit_lm`, :3092-3170
 * `irls_fit`); the implicit arm follows my-version/src/implicit.rs:277-409.
 *
 * B200 design. The reference runs one block per candidate for the whole LM,
 * so a candidate's 262,144 rows are swept by 128 threads while most of the
 * GPU waits for the slowest candidate. Here every sweep is spread over
 * (candidate x 2,048-row tile) work items for all active candidates at once:
 *
 *   step s:  sweep kernels, one per kind (f32 assembly, f64 assembly, f32
 *            objective, f64 objective; implicit Jacobian / cost), each a
 *            persistent grid over the (candidate, tile) items whose candidate
 *            requested that kind -> per-tile partials (packed J^T J / J^T r
 *            blocks, objective, flags);
 *            control kernel: per candidate that had a sweep, reduce its tile
 *            partials in ascending tile order, run the reference's LM state
 *            machine (damped Jacobi-equilibrated Cholesky in f64, trial
 *            clamp, accept / reject, lambda, IRLS rounds, polish) until it
 *            needs the next sweep, and queue it for step s+1.
 *
 * The number of steps any candidate can need is bounded (two sweeps per LM
 * iteration, four with L1 halvings, plus the polish), so the whole fit is a
 * fixed graph of kernels replayed per batch; candidates that finish early
 * simply stop queueing work. Every statistic is a fixed-order sum (per row
 * chunk, SYRK row groups, tiles), so a candidate's result does not depend on
 * the batch it is fitted in.
 */
#include <algorithm>
#include <cmath>
#include <cstddef>
#include <cstdio>
#include <cstring>
#include <fstream>
#include <string>
#include <type_traits>
#include <vector>

#include "fit_common.cuh"
#include "fit_interp.cuh"
#include "fit_prep.h"

#define FT_TILE_ROWS 2048
#define FT_NBLK_MAX 21                     /* 4x4 blocks of a 24-wide augmented Gram */
#define FT_PART_LOSS (FT_NBLK_MAX * 16)
#define FT_PART_BAD (FT_PART_LOSS + 1)
#define FT_PART_SKIP (FT_PART_LOSS + 2)
#define FT_PART_STRIDE (FT_PART_LOSS + 4)
#define FT_NTRI (FT_MAX_CONST * (FT_MAX_CONST + 1) / 2)

enum {
    FOP_NONE = 0, FOP_ASM32 = 1, FOP_ASM64 = 2, FOP_LOSS32 = 3, FOP_LOSS64 = 4,
    FOP_IJAC = 5, FOP_ICOST = 6, FOP_CASM = 7, FOP_CSCORE = 8, FOP_IJACS = 9,
    /* the assembly queues of the other launch classes (ft_cls_*): their
       sweeps run in blocks of the class's threads, sized for the class */
    FOP_ASM32_64 = 10, FOP_ASM32_32 = 11, FOP_ASM64_64 = 12, FOP_ASM64_32 = 13,
    FOP_ASM32_64A = 14, FOP_ASM32_64B = 15, FOP_ASM64_64A = 16, FOP_ASM64_64B = 17,
    FOP_ASM32_128L = 18, FOP_ASM64_128L = 19,
    FOP_COUNT = 20
};

/* Launch classes of the assemblies. A candidate's active threads A and its
   shared region decide it: 0: A = 128 with a region of at most 41 KB; 5:
   A = 128 with a larger one (a length bucket the autotuner gave a bigger
   budget); 1, 2, 3: A = 64 with a region of at most 21 KB, at most 30 KB, or
   more; 4: A = 32. A class's launch uses blocks of A threads and the largest
   region of its candidates, so the small-region classes fit more blocks on
   an SM (10, 7 and 5 of 64 threads at 21, 30 and 40 KB), and a large region
   never shrinks the launch of the others. Which launch runs a candidate does
   not change its arithmetic (that depends on A alone). */
#define FT_NCLS 6
__host__ __device__ constexpr int ft_cls_threads(int cls)
{
    return (cls == 0 || cls == 5) ? 128 : (cls == 4 ? 32 : 64);
}

inline int ft_cls_of(int A, size_t region)
{
    if (A >= 128) return region <= 41 * 1024 ? 0 : 5;
    if (A <= 32) return 4;
    return region <= 21 * 1024 ? 1 : (region <= 30 * 1024 ? 2 : 3);
}

/* The kind a queue's sweep performs (a class queue performs its base kind). */
__host__ __device__ constexpr int ft_base_kind(int k)
{
    return (k == FOP_ASM32_64 || k == FOP_ASM32_32 || k == FOP_ASM32_64A || k == FOP_ASM32_64B ||
            k == FOP_ASM32_128L)
               ? FOP_ASM32
           : (k == FOP_ASM64_64 || k == FOP_ASM64_32 || k == FOP_ASM64_64A ||
              k == FOP_ASM64_64B || k == FOP_ASM64_128L)
               ? FOP_ASM64
               : k;
}

/* The launch class of an assembly queue kind (0 for the base kinds). */
__host__ __device__ constexpr int ft_kind_cls(int k)
{
    return (k == FOP_ASM32_64A || k == FOP_ASM64_64A)   ? 1
           : (k == FOP_ASM32_64B || k == FOP_ASM64_64B) ? 2
           : (k == FOP_ASM32_64 || k == FOP_ASM64_64)   ? 3
           : (k == FOP_ASM32_32 || k == FOP_ASM64_32)   ? 4
           : (k == FOP_ASM32_128L || k == FOP_ASM64_128L) ? 5
                                                        : 0;
}

/* The queue of a sweep request: f32 / f64 assemblies go to the queue of the
   candidate's launch class. */
__host__ __device__ inline int ft_queue_kind(int op, int cls)
{
    static constexpr int k32[FT_NCLS] = {FOP_ASM32, FOP_ASM32_64A, FOP_ASM32_64B, FOP_ASM32_64,
                                         FOP_ASM32_32, FOP_ASM32_128L};
    static constexpr int k64[FT_NCLS] = {FOP_ASM64, FOP_ASM64_64A, FOP_ASM64_64B, FOP_ASM64_64,
                                         FOP_ASM64_32, FOP_ASM64_128L};
    if (op == FOP_ASM32) return k32[cls];
    if (op == FOP_ASM64) return k64[cls];
    return op;
}

enum {
    PC_INIT = 0, PC_AFTER_FIRST_ASM, PC_ROUND, PC_ITER, PC_AFTER_ASM, PC_SOLVE,
    PC_AFTER_TRIAL, PC_REBASE, PC_AFTER_REBASE, PC_POLISH, PC_AFTER_PASM, PC_AFTER_PTRIAL,
    PC_END, PC_I_INIT, PC_I_AFTER_BASE, PC_I_ITER, PC_I_AFTER_JAC, PC_I_SOLVE, PC_I_AFTER_TRIAL,
    PC_I_END,
    PC_C_INIT, PC_C_SCORE_ONLY, PC_C_AFTER_FIRST, PC_C_ITER, PC_C_AFTER_ASM, PC_C_SOLVE,
    PC_C_AFTER_TRIAL, PC_C_POLISH, PC_C_AFTER_PASM, PC_C_AFTER_PTRIAL, PC_C_END, PC_DONE
};

/* Per-candidate LM state, resident in device memory between steps. */
struct FitState {
    double c[FT_MAX_CONST];
    double trial[FT_MAX_CONST];
    double start_c[FT_MAX_CONST];
    double jtj[FT_NTRI];
    double jtr[FT_MAX_CONST];
    double lambda, best, start_best;
    double rho, svar, syy; /* correlation arm: moments of the last assembly */
    double req_lambda;     /* damping of the requested solve */
    int pc, op, sel;
    int status, round, it, half, pit;
    int assembled, improved, rank, skip, start;
    int req, sv;           /* solve request (FT_REQ_*) and the answered label */
    int f64;               /* 0: f32 sweeps; 1: switched to f64 sweeps after an f32-only
                              failure, loss not yet re-baselined; 2: f64, re-baselined */
    int nsw[4];            /* sweeps run: f32 assembly, f32 objective, f64 assembly, f64
                              objective (correlation and implicit kinds count in their
                              class: CASM / CSCORE as f32, IJAC / ICOST as f64) */
};

/* Fit flags of rc_fit_batch_fused. */
#define FT_FLAG_NO_POLISH 1 /* skip the f64 re-baseline and polish */
#define FT_FLAG_NO_RESCUE 2 /* keep the reference kernel's f32-only failures */

/* The controller's thread 0 runs the state machine; a damped solve is
   handed to warp 0 (ft_solve_warp) by a request in the state, and the state
   machine resumes at the same state with the answer. */
enum { FT_REQ_NONE = 0, FT_REQ_SOLVE = 1, FT_REQ_DONE = 2 };

__device__ __forceinline__ void ft_request_solve(FitState &st, double lambda)
{
    st.req = FT_REQ_SOLVE;
    st.req_lambda = lambda;
    st.op = FOP_NONE;
}

/* The answer to the last request (and clears it). */
__device__ __forceinline__ int ft_take_solve(FitState &st)
{
    st.req = FT_REQ_NONE;
    return st.sv;
}

/* The f64 rescue of an f32 assembly that failed. The f32 sweep marks a row
   bad when its prediction, residual or Jacobian entry is not finite (or the
   prediction exceeds 1e30) in f32, where the CPU fit's f64 arithmetic may
   well be finite (an exp beyond 88, a square of a denominator below 1e-19).
   Instead of stopping there (status 2, reported 5 or 7, as the reference
   kernel does), the candidate's assembly is re-run in f64 at the same
   constants, and from then on every sweep of its LM runs in f64: it stops
   only where the CPU fit's normal equations would stop too (a non-finite
   f64 residual or Jacobian entry). Returns true when the f64 assembly was
   queued (the state is re-entered with its outputs). */
__device__ __forceinline__ bool ft_rescue(int flags, FitState &st, int rb)
{
    if (!rb || st.f64 || (flags & FT_FLAG_NO_RESCUE)) return false;
    st.f64 = 1;
    st.op = FOP_ASM64;
    st.sel = 0;
    return true;
}

struct FitArgs {
    const float *cols;
    const float *y;
    const float *tsign;
    const double *cols64;
    const double *y64;
    const double *tsign64;
    const double *w;
    int n, npad, v;
    const uint4 *rec;
    const int *node_off;
    const int *pcount;
    int kmax;
    const double *c0;
    const int *gauge;      /* [2P] correlation gauge pair (scale, offset), -1 = none */
    const int *valid;
    const FIns *fins;      /* stack-machine translation of the records */
    const int *fins_off;   /* [P+1] start of [forward | reverse] */
    const int4 *finfo;     /* [P] forward count, reverse count, active threads | launch
                              class << 16,
                              spill slots | tape slots << 16 */
    int fslots;            /* spill slots needed by the batch */
    int ftape;             /* partial-tape slots needed by the batch */
    int fmaxins;           /* longest forward + reverse list */
    size_t asm_region;     /* assembly region of a 128-thread launch over every class */
    size_t asm_reg[6];     /* assembly region of each launch class (ft_cls_of) */
    const int2 *fcinfo;    /* [P] cached forward count (after the reverse list),
                              first cache column */
    float *cache;          /* [columns][npad] values of constant-free subtrees */
    double *cache64;       /* the same columns in f64 for the polish, or null */
    const FIns *sub_fins;  /* forward lists of the cached subtrees */
    const int *sub_off;    /* [nsub + 1] */
    const int *sub_col;    /* [nsub] */
    int nsub;
    int sub_slots, sub_maxins;
    const FIns *xfins;     /* implicit metric: input-mode lists [forward | reverse] */
    const int *xfins_off;  /* [P + 1] */
    const int4 *xinfo;     /* forward count, reverse count, spill slots, tape slots */
    int xmaxins, xslots, xtape;
    int iters, metric, flags;
    int ntiles;
    int mmax;
    int ijac_small;        /* implicit: programs of at most this many records take the
                              short Jacobian launch (FOP_IJACS); 0: one launch */
    int ijac_tape;         /* internal-node tape slots of the Jacobian launch */
    int ijac_tape_small;   /* ... and of the short one */
    int Wmax;
    int nprog;
    FitState *state;
    double *part;      /* [P][ntiles][FT_PART_STRIDE] */
    int *lists;        /* [2][FOP_COUNT][P] */
    int *counts;       /* [2][FOP_COUNT] candidates queued per kind */
    int *work;         /* [2][FOP_COUNT] persistent-grid work counters */
    double *outc;
    double *outsse;
    int *outstatus;
};

/* ---- sweep kernels ------------------------------------------------------ */

__host__ __device__ inline bool ft_op_assembles(int opk)
{
    opk = ft_base_kind(opk);
    return opk == FOP_ASM32 || opk == FOP_ASM64 || opk == FOP_IJAC || opk == FOP_CASM ||
           opk == FOP_IJACS;
}

__host__ __device__ inline bool ft_op_ijac(int opk) { return opk == FOP_IJAC || opk == FOP_IJACS; }

/* Columns of a sweep's augmented Gram: the Jacobian and the residual, or for
   the correlation assembly the Jacobian and the weighted 1, f and y
   (eval.cu:1959-2063 moments). */
__host__ __device__ inline int ft_gram_cols(int opk, int p)
{
    return p + (opk == FOP_CASM ? 3 : 1);
}

__host__ __device__ inline size_t ft_rows_bytes(int Wmax, int T)
{
    const size_t rows = sizeof(double) * (size_t)T * Wmax;
    const size_t part = sizeof(double) * (size_t)T * 16;
    return rows > part ? rows : part;
}

/* Threads of the implicit sweeps: every thread carries one row. */
#define FT_ITHREADS 64

/* Dynamic shared memory of an exact-Jacobian sweep: the compact records
   and their reference scratch for `mrec` records, the constants, the two
   f64 tapes ([slot][T], `tcap` internal-node slots each), the Jacobian row
   buffer and a reduction buffer. */
__host__ __device__ inline size_t ft_ijac_smem(int mrec, int tcap, int Wmax, int T)
{
    return 16 * (size_t)mrec + 16 * (size_t)((mrec + 3) / 4) + 8 * (size_t)FT_MAX_CONST +
           16 * (size_t)tcap * T + ft_rows_bytes(Wmax, T) + 8 * (size_t)T;
}

/* Fixed-order reduction of the per-thread SYRK blocks over the row groups,
   written packed ([block][16]) to the tile's partial. */
template <int T>
__device__ __forceinline__ void ft_tile_gram_out(const Syrk &sy, const double acc[16],
                                                 double *buf, double *pt)
{
    const int tid = threadIdx.x;
    if (sy.rg < sy.RG) {
#pragma unroll
        for (int e = 0; e < 16; ++e) buf[(sy.rg * sy.nblk + sy.blk) * 16 + e] = acc[e];
    }
    __syncthreads();
    for (int q = tid; q < sy.nblk * 16; q += T) {
        const int blk = q >> 4, e = q & 15;
        double s = 0.0;
        for (int g = 0; g < sy.RG; ++g) s += buf[(g * sy.nblk + blk) * 16 + e];
        pt[q] = s;
    }
    __syncthreads();
}

/* Implicit metric of one tile (implicit.rs:156-174, :302-333): the cost
   sum w d^2 at `cd`, the Jacobian rows of sqrt(w) d (exact,
   forward-over-reverse, where the reference takes central differences
   with h = 1e-6 (1 + |c_j|)) and their J^T J / J^T r. An undefined row
   marks the tile bad. `rec` holds the ni compact records of ij_compact;
   `tape64` and `tan64` are the two f64 tapes. */
template <int T>
__device__ void ft_tile_implicit(const FitArgs &a, const uint4 *rec, int ni, int p,
                                 const double *cd, double *tape64, double *tan64, double *rows,
                                 double *red, int r0, int r1, double *pt)
{
    constexpr int TS = T;
    const int tid = threadIdx.x;
    const int W = 4 * ((p + 1 + 3) / 4);
    const Syrk sy = ft_syrk_setup<T>(W);
    double acc[16];
#pragma unroll
    for (int e = 0; e < 16; ++e) acc[e] = 0.0;
    double cost = 0.0;
    int bad = 0;
    double *tp = tape64 + tid;
    double *myrow = rows + (size_t)tid * W;
    double x[FT_IMPLICIT_MAXV];
    for (int base = r0; base < r1; base += TS) {
        const int row = base + tid;
        if (tid < TS) {
            for (int j = 0; j < W; ++j) myrow[j] = 0.0;
            const double wr = (row < r1 && a.w) ? a.w[row] : 1.0;
            if (row < r1 && !(isfinite(wr) && wr >= 0.0)) bad = 1;
            else if (row < r1 && wr > 0.0) {
                for (int k = 0; k < FT_IMPLICIT_MAXV; ++k)
                    x[k] = k < a.v ? a.cols64[(size_t)k * a.npad + row] : 0.0;
                double d;
                const double sw = sqrt(wr);
                const bool ok =
                    ft_implicit_jac<TS>(rec, ni, x, a.v, cd, p, sw, tp, tan64 + tid, d, myrow);
                if (!ok) {
                    bad = 1;
                    for (int j = 0; j < p; ++j) myrow[j] = 0.0;
                } else {
                    const double r = sw * d;
                    cost += r * r;
                    myrow[p] = r;
                }
            }
        }
        __syncthreads();
        ft_syrk_chunk(sy, rows, W, TS, acc);
        __syncthreads();
    }
    bad = __syncthreads_or(bad);
    cost = ft_block_sum<T>(cost, red);
    ft_tile_gram_out<T>(sy, acc, rows, pt);
    if (tid == 0) {
        pt[FT_PART_LOSS] = cost;
        pt[FT_PART_BAD] = bad ? 1.0 : 0.0;
        pt[FT_PART_SKIP] = 0.0;
    }
}

/* The implicit cost of one tile, sum w d^2 with d = f / ||grad_x f||
   (implicit.rs:156-174), on the stack machine: f64, one row per thread, the
   forward sweep keeping partials on input paths and the input-adjoint
   reverse sweep (fi_reverse_x). A row with a non-finite value or input
   gradient, or a zero gradient norm, marks the tile undefined
   (implicit.rs:156-174). */
template <int T>
__device__ void ft_tile_icost_x(const FitArgs &a, const FIns *fwd, int nf, int nr,
                                const double *cd, FiV<double, 1>::V4 *stk,
                                FiV<double, 1>::V4 *tape, FiV<double, 1>::V4 *ig, double *red,
                                int r0, int r1, double *pt)
{
    const int tid = threadIdx.x;
    double cost = 0.0;
    int bad = 0;
    for (int base = r0; base < r1; base += T) {
        const int row = base + tid;
        double fv;
        fi_forward<double, 1, true>(fwd, cd, a.cols64, a.npad, row, stk, tape, T, tid, &fv);
        if (row >= r1) continue;
        const double wr = a.w ? a.w[row] : 1.0;
        if (!(isfinite(wr) && wr >= 0.0)) {
            bad = 1;
            continue;
        }
        if (wr == 0.0) continue;
        if (!isfinite(fv)) {
            bad = 1;
            continue;
        }
        for (int k = 0; k < a.v; ++k) ig[k * T + tid].v[0] = 0.0;
        double seed = 1.0;
        fi_reverse_x<double, 1>(fwd + nf, nr, stk, tape, T, tid, ig, &seed);
        double nsq = 0.0;
        bool ok = true;
        for (int k = 0; k < a.v; ++k) {
            const double g = ig[k * T + tid].v[0];
            if (!isfinite(g)) ok = false;
            nsq += g * g;
        }
        const double norm = sqrt(nsq);
        if (!ok || !(isfinite(norm) && norm > 0.0)) {
            bad = 1;
            continue;
        }
        const double d = fv / norm;
        if (!isfinite(d)) {
            bad = 1;
            continue;
        }
        const double r = sqrt(wr) * d;
        cost += r * r;
    }
    bad = __syncthreads_or(bad);
    cost = ft_block_sum<T>(cost, red);
    if (tid == 0) {
        pt[FT_PART_LOSS] = cost;
        pt[FT_PART_BAD] = bad ? 1.0 : 0.0;
        pt[FT_PART_SKIP] = 0.0;
    }
}

/* The implicit cost sweep over every queued (candidate, tile) item of step
   parity q. */
template <int OPK, int T>
__global__ void __launch_bounds__(T) ft_sweep(FitArgs a, int q)
{
    extern __shared__ __align__(16) unsigned char sm[];
    static_assert(OPK == FOP_ICOST, "ft_sweep runs the cost kind");
    {
        /* [instructions | constants | spill slots | tape | input gradients | reduction] */
        using V4 = FiV<double, 1>::V4;
        FIns *ins = reinterpret_cast<FIns *>(sm);
        double *cd = reinterpret_cast<double *>(sm + 8 * (size_t)((a.xmaxins + 1) & ~1));
        V4 *stk = reinterpret_cast<V4 *>(cd + FT_MAX_CONST);
        V4 *tape = stk + (size_t)a.xslots * T;
        V4 *ig = tape + (size_t)a.xtape * T;
        double *red = reinterpret_cast<double *>(ig + (size_t)a.v * T);
        __shared__ int s_item;
        const int tid = threadIdx.x;
        const int *list = a.lists + ((size_t)q * FOP_COUNT + OPK) * a.nprog;
        const int total = a.counts[q * FOP_COUNT + OPK] * a.ntiles;
        int *work = a.work + q * FOP_COUNT + OPK;
        for (;;) {
            if (tid == 0) s_item = atomicAdd(work, 1);
            __syncthreads();
            const int item = s_item;
            __syncthreads();
            if (item >= total) break;
            const int cand = list[item / a.ntiles];
            const int tile = item % a.ntiles;
            const FitState *st = a.state + cand;
            const int4 info = a.xinfo[cand];
            const int ib = a.xfins_off[cand];
            const int p = a.pcount[cand];
            const int sel = st->sel;
            for (int i = tid; i < info.x + info.y; i += T) ins[i] = a.xfins[ib + i];
            if (tid < p) cd[tid] = sel ? st->trial[tid] : st->c[tid];
            __syncthreads();
            const int r0 = tile * FT_TILE_ROWS;
            const int r1 = min(a.n, r0 + FT_TILE_ROWS);
            double *pt = a.part + ((size_t)cand * a.ntiles + tile) * FT_PART_STRIDE;
            ft_tile_icost_x<T>(a, ins, info.x, info.y, cd, stk, tape, ig, red, r0, r1, pt);
            __syncthreads();
        }
    }
}

/* The exact-Jacobian sweep (FOP_IJAC, or FOP_IJACS for the short programs)
   over every queued (candidate, tile) item of step parity q: eight 64-thread
   blocks per SM fit beside the compact tapes, so registers are held to
   that. The short launch is laid out for its own record and tape bounds. */
template <int OPK, int T>
__global__ void __launch_bounds__(T, 8) ft_jac_sweep(FitArgs a, int q)
{
    extern __shared__ __align__(16) unsigned char sm[];
    const int mcap = OPK == FOP_IJACS ? a.ijac_small : a.mmax;
    const int tcap = OPK == FOP_IJACS ? a.ijac_tape_small : a.ijac_tape;
    uint4 *rec = reinterpret_cast<uint4 *>(sm);
    unsigned *refs = reinterpret_cast<unsigned *>(sm + 16 * (size_t)mcap);
    double *cd = reinterpret_cast<double *>(sm + 16 * (size_t)mcap + 16 * (size_t)((mcap + 3) / 4));
    double *tape64 = cd + FT_MAX_CONST;
    double *tan64 = tape64 + (size_t)tcap * T;
    double *rows = tan64 + (size_t)tcap * T;
    double *red = rows + ft_rows_bytes(a.Wmax, T) / 8;
    __shared__ int s_item, s_ni;
    const int tid = threadIdx.x;
    const int *list = a.lists + ((size_t)q * FOP_COUNT + OPK) * a.nprog;
    const int total = a.counts[q * FOP_COUNT + OPK] * a.ntiles;
    int *work = a.work + q * FOP_COUNT + OPK;
    for (;;) {
        if (tid == 0) s_item = atomicAdd(work, 1);
        __syncthreads();
        const int item = s_item;
        __syncthreads();
        if (item >= total) break;
        const int cand = list[item / a.ntiles];
        const int tile = item % a.ntiles;
        const FitState *st = a.state + cand;
        const int nb = a.node_off[cand];
        const int m = a.node_off[cand + 1] - nb;
        const int p = a.pcount[cand];
        const int sel = st->sel;
        for (int i = tid; i < m; i += T) rec[i] = a.rec[nb + i];
        if (tid < p) cd[tid] = sel ? st->trial[tid] : st->c[tid];
        __syncthreads();
        if (tid == 0) s_ni = ij_compact(rec, m, refs);
        __syncthreads();
        const int r0 = tile * FT_TILE_ROWS;
        const int r1 = min(a.n, r0 + FT_TILE_ROWS);
        double *pt = a.part + ((size_t)cand * a.ntiles + tile) * FT_PART_STRIDE;
        ft_tile_implicit<T>(a, rec, s_ni, p, cd, tape64, tan64, rows, red, r0, r1, pt);
        __syncthreads();
    }
}

/* ---- four-rows-per-thread sweeps ------------------------------------- */

#define FT_ASM_T 128
#ifndef FT_ASM_BUDGET
#define FT_ASM_BUDGET (40 * 1024)
#endif

/* Rows per thread of each sweep: the assemblies carry 8 bytes of rows per
   thread (two f32 or one f64 row) to fit more threads beside their tapes;
   the objective sweeps, which keep no tape, carry 16 (four f32 or two f64
   rows). */
#define FT_ASM32_NR 2
#define FT_ASM64_NR 1
#define FT_LOSS32_NR 4
#define FT_LOSS64_NR 2

/* Per-candidate shared region of an assembly sweep at A active threads:
   spill slots and partial tape ([slot][A] 8-byte row vectors), then the
   Jacobian rows column-major ([W8][NR * A + 4], W8 = p + 1 rounded up to 8).
   A column stride of 4 mod 32 words (f32) or 4 mod 16 doubles (f64) keeps
   both the per-thread stores of the reverse sweep and the tensor-core
   fragment loads bank-conflict free. The size is that of the f64 layout,
   the larger of the two. */
__host__ __device__ inline size_t ft_asm_region(int A, int slots, int tape, int W8)
{
    return 8 * (size_t)A * (size_t)(slots + tape) + 8 * (size_t)W8 * ((size_t)A + 4);
}

/* Active threads of a candidate: the most (128, 64 or 32) whose region fits
   the budget of its length bucket (FT_ASM_BUDGET unless the context's fit
   autotuner chose another). It depends on the candidate and the context's
   table alone, so its summation order does not depend on the batch. */
inline int ft_asm_threads(int slots, int tape, int ncols, size_t budget)
{
    const int W8 = 8 * ((ncols + 7) / 8);
    int A = FT_ASM_T;
    while (A > 32 && ft_asm_region(A, slots, tape, W8) > budget) A /= 2;
    return A;
}

/* Length bucket of a fit program of m records (the autotuner's key). */
inline int ft_length_bucket(int m) { return m <= 16 ? 0 : (m <= 32 ? 1 : (m <= 64 ? 2 : 3)); }

__host__ __device__ inline bool ft_op_f64(int opk)
{
    return ft_base_kind(opk) == FOP_ASM64 || opk == FOP_LOSS64;
}

/* Shared memory of a four-row sweep: forward and reverse instructions,
   constants, the assembly region (or the spill slots of an objective sweep),
   a reduction buffer. */
__host__ __device__ inline size_t ft_sweep4_smem(int opk, int maxins, int slots, size_t region,
                                                 int T)
{
    size_t s = 8 * (size_t)((maxins + 1) & ~1) + 8 * FT_MAX_CONST;
    s += ft_op_assembles(opk) ? region : 16 * (size_t)(slots > 0 ? slots : 1) * T;
    return s + 8 * (size_t)T;
}

/* One row's place in an assembly, from its prediction (eval.cu:1692-1804
   for f32, :1492-1630 for f64): whether it counts, whether it is usable, the
   adjoint seed (its square-root IRLS/GN weight), the weighted residual and
   its objective term. */
struct FtRow {
    bool use, ok;
    float s_zero;
    double seed, res, loss;
    double c1, c2; /* correlation: the weighted prediction and target columns */
};

/* A row of the correlation assembly (eval.cu:2031-2047): the reverse sweep
   is seeded with sqrt(w), and the extra columns carry sqrt(w), sqrt(w) f and
   sqrt(w) y, so the augmented Gram holds every weighted moment the objective
   needs. A row whose prediction or target is not finite fails the
   assembly. */
__device__ __forceinline__ FtRow ft_row_corr(const FitArgs &a, int rr, int r1, float pred)
{
    FtRow o;
    const double wr = (rr < r1 && a.w) ? a.w[rr] : 1.0;
    o.use = rr < r1 && wr > 0.0;
    o.ok = false;
    o.s_zero = 0.0f;
    o.seed = o.res = o.loss = o.c1 = o.c2 = 0.0;
    if (!o.use) return o;
    const float t = a.y[rr];
    if (!(isfinite(pred) && fabsf(pred) <= 1e30f && isfinite(t))) return o;
    const float s = sqrtf((float)wr);
    o.ok = true;
    o.seed = s;
    o.c1 = s * pred;
    o.c2 = s * t;
    return o;
}

__device__ __forceinline__ FtRow ft_row_f32(const FitArgs &a, int rr, int r1, float pred)
{
    FtRow o;
    const double wr = (rr < r1 && a.w) ? a.w[rr] : 1.0;
    o.use = rr < r1 && wr > 0.0;
    o.ok = false;
    o.s_zero = 0.0f;
    o.seed = 0.0;
    o.res = 0.0;
    o.loss = 0.0;
    if (!o.use) return o;
    const float r = pred - a.y[rr];
    bool good = isfinite(pred) && fabsf(pred) <= 1e30f && isfinite(r);
    double sw, resp = (double)r;
    if (a.metric == FM_LOGISTIC) {
        const double tt = a.tsign ? (double)a.tsign[rr] : 0.0;
        const double u = tt * (double)pred;
        if (!a.tsign || !isfinite(tt)) good = false;
        const double qq = ft_logistic_q(u);
        sw = wr * qq * (1.0 - qq);
        resp = -tt / qq;
        o.loss = wr * ft_softplus_neg(u);
    } else {
        sw = ft_row_weight(wr, (double)r, a.metric);
        o.loss = wr * (double)ft_row_loss_f(r, a.metric);
    }
    const float s = sqrtf((float)sw);
    o.ok = good;
    if (good) {
        o.seed = s > 0.0f ? s : 1.0f;
        o.s_zero = s > 0.0f ? 0.0f : 1.0f;
        o.res = (float)(s * resp);
    }
    return o;
}

__device__ __forceinline__ FtRow ft_row_f64(const FitArgs &a, int rr, int r1, double pred)
{
    FtRow o;
    const double wr = (rr < r1 && a.w) ? a.w[rr] : 1.0;
    o.use = rr < r1 && wr > 0.0;
    o.ok = false;
    o.s_zero = 0.0f;
    o.seed = 0.0;
    o.res = 0.0;
    o.loss = 0.0;
    if (!o.use) return o;
    const double r = pred - a.y64[rr];
    bool good = isfinite(pred) && isfinite(r);
    double sw, resp = r, rho;
    if (a.metric == FM_LOGISTIC) {
        const double tt = a.tsign64 ? a.tsign64[rr] : 0.0;
        const double u = tt * pred;
        if (!a.tsign64 || !isfinite(tt)) good = false;
        const double qq = ft_logistic_q(u);
        sw = wr * qq * (1.0 - qq);
        resp = -tt / qq;
        rho = ft_softplus_neg(u);
    } else {
        sw = ft_row_weight(wr, r, a.metric);
        if (a.metric == FM_SQUARED) rho = r * r;
        else if (a.metric == FM_ABSOLUTE) rho = fabs(r);
        else rho = log1p(r * r);
    }
    const double s = sqrt(sw);
    o.ok = good;
    o.loss = wr * rho;
    if (good) {
        o.seed = s > 0.0 ? s : 1.0;
        o.s_zero = s > 0.0 ? 0.0f : 1.0f;
        o.res = s * resp;
    }
    return o;
}

/* Fold the warp's NR * 32 rows of the column-major Jacobian into its
   J^T J | J^T r blocks with f64 tensor-core MMAs (f32 values widen
   exactly, so products are exact and sums f64). */
template <int NB, typename V, int NR>
__device__ __forceinline__ void ft_fold(const V *g, int R, int A, int w, int gid, int tig,
                                        double (*acc)[2])
{
#pragma unroll 4
    for (int s = 0; s < 8 * NR; ++s) {
        const int q = 4 * s + tig;
        const int local = (q >> 5) * A + 32 * w + (q & 31);
        double x[NB];
#pragma unroll
        for (int I = 0; I < NB; ++I) x[I] = (double)g[(8 * I + gid) * R + local];
        int b = 0;
#pragma unroll
        for (int I = 0; I < NB; ++I)
#pragma unroll
            for (int J = 0; J <= I; ++J, ++b) fi_dmma(acc[b][0], acc[b][1], x[I], x[J]);
    }
}

/* Assembly of one tile in f32 or f64: the forward sweep of the thread's
   rows, the reverse sweep seeded with each row's square-root weight (so it
   yields the weighted Jacobian row), the weighted residual as column p, and
   the warp's rows folded into the augmented Gram matrix. Warps work
   independently over their own rows; the tile's sum is a fixed-order sum
   over warps, written in the packed 4x4-block layout the controller reads. */
template <typename V, int NR, int T, bool CORR>
__device__ void ft_tile_asm(const FitArgs &a, const FIns *fwd, const FIns *rev, int nr, int p,
                            int A, int slots, int ntape, const V *cv, unsigned char *region,
                            double *red, int r0, int r1, double *pt, const V *ccols)
{
    using F = FiV<V, NR>;
    using V4 = typename F::V4;
    constexpr bool F64 = sizeof(V) == 8;
    const int tid = threadIdx.x;
    const int lane = tid & 31, w = tid >> 5, gid = lane >> 2, tig = lane & 3;
    const int ncols = p + (CORR ? 3 : 1);
    const int NB = (ncols + 7) / 8;
    const int W8 = 8 * NB, R = NR * A + 4;
    V4 *stk = reinterpret_cast<V4 *>(region);
    V4 *tape = stk + slots * A;
    V *g = reinterpret_cast<V *>(tape + ntape * A);
    const V *cols = F64 ? reinterpret_cast<const V *>(a.cols64) : reinterpret_cast<const V *>(a.cols);
    for (int i = tid; i < W8 * R; i += T) g[i] = V(0);
    __syncthreads();
    double acc[6][2];
#pragma unroll
    for (int b = 0; b < 6; ++b) acc[b][0] = acc[b][1] = 0.0;
    double loss = 0.0;
    int bad = 0, skipped = 0;
    if (tid < A) {
        V *gt = g + tid;
        for (int base = r0; base < r1; base += NR * A) {
            const int row = base + NR * tid;
            V pr[NR];
            fi_forward<V, NR, true>(fwd, cv, cols, a.npad, row, stk, tape, A, tid, pr, ccols);
            FtRow rw[NR];
            V seed[NR];
            bool special = false;
#pragma unroll
            for (int i = 0; i < NR; ++i) {
                rw[i] = CORR  ? ft_row_corr(a, row + i, r1, (float)pr[i])
                        : F64 ? ft_row_f64(a, row + i, r1, (double)pr[i])
                              : ft_row_f32(a, row + i, r1, (float)pr[i]);
                seed[i] = (V)rw[i].seed;
                special = special || rw[i].s_zero != 0.0f;
            }
            const bool fin = fi_reverse<V, NR>(rev, nr, stk, tape, A, tid, gt, R, A, seed);
            if (!fin || special) {
                /* rare rows: a non-finite Jacobian entry (the row is dropped
                   from the Jacobian; in f32 it counts as failed), or a zero
                   weight (its entries are zero) */
#pragma unroll
                for (int i = 0; i < NR; ++i) {
                    if (!rw[i].ok) continue;
                    V *gi = gt + i * A;
                    bool rf = true;
                    if (!fin)
                        for (int j = 0; j < p; ++j) rf = rf && isfinite(gi[j * R]);
                    if (!rf || rw[i].s_zero != 0.0f)
                        for (int j = 0; j < p; ++j) gi[j * R] = V(0);
                    if (!rf) {
                        if (F64 && !CORR) {
                            skipped = 1;
                            rw[i].res = 0.0;
                            rw[i].seed = 0.0; /* marks the row's residual column zero */
                        } else {
                            rw[i].ok = false;
                        }
                    }
                }
            }
#pragma unroll
            for (int i = 0; i < NR; ++i) {
                if (CORR) {
                    const bool ok = rw[i].ok;
                    gt[p * R + i * A] = ok ? (V)rw[i].seed : V(0);
                    gt[(p + 1) * R + i * A] = ok ? (V)rw[i].c1 : V(0);
                    gt[(p + 2) * R + i * A] = ok ? (V)rw[i].c2 : V(0);
                } else {
                    const bool jac = rw[i].ok && rw[i].seed != 0.0;
                    gt[p * R + i * A] = jac ? (V)rw[i].res : V(0);
                }
                if (rw[i].ok) loss += rw[i].loss;
                else if (rw[i].use) bad = 1;
            }
            __syncwarp();
            if (NB <= 1) ft_fold<1, V, NR>(g, R, A, w, gid, tig, acc);
            else if (NB == 2) ft_fold<2, V, NR>(g, R, A, w, gid, tig, acc);
            else ft_fold<3, V, NR>(g, R, A, w, gid, tig, acc);
            __syncwarp();
        }
    }
    __syncthreads();
    const int NBLK = NB * (NB + 1) / 2;
    double *gb = reinterpret_cast<double *>(region);
    if (tid < A) {
#pragma unroll
        for (int b = 0; b < 6; ++b) {
            if (b >= NBLK) break;
            gb[(w * NBLK + b) * 64 + gid * 8 + 2 * tig] = acc[b][0];
            gb[(w * NBLK + b) * 64 + gid * 8 + 2 * tig + 1] = acc[b][1];
        }
    }
    __syncthreads();
    const int W = 4 * ((ncols + 3) / 4);
    const int nb4 = W / 4, nblk4 = nb4 * (nb4 + 1) / 2, nw = A / 32;
    for (int e = tid; e < nblk4 * 16; e += T) {
        int b4 = e >> 4, bi = 0;
        while (b4 > bi) {
            b4 -= bi + 1;
            ++bi;
        }
        const int rw4 = 4 * bi + ((e & 15) >> 2), cl = 4 * b4 + (e & 3);
        const int I = rw4 >> 3, J = cl >> 3;
        const int el = (I * (I + 1) / 2 + J) * 64 + (rw4 & 7) * 8 + (cl & 7);
        double s = 0.0;
        for (int v = 0; v < nw; ++v) s += gb[v * NBLK * 64 + el];
        pt[e] = s;
    }
    bad = __syncthreads_or(bad);
    skipped = __syncthreads_or(skipped);
    loss = ft_block_sum<T>(loss, red);
    if (tid == 0) {
        pt[FT_PART_LOSS] = loss;
        pt[FT_PART_BAD] = bad ? 1.0 : 0.0;
        pt[FT_PART_SKIP] = skipped ? 1.0 : 0.0;
    }
}

/* Objective of one tile in f32 or f64 (eval.cu:1808-1855): the forward
   sweep only; a row that is not finite costs 1e30. */
template <typename V, int NR, int T>
__device__ void ft_tile_loss(const FitArgs &a, const FIns *ins, const V *cv,
                             typename FiV<V, NR>::V4 *stk, double *red, int r0, int r1, double *pt,
                             const V *ccols)
{
    constexpr bool F64 = sizeof(V) == 8;
    const V *cols = F64 ? reinterpret_cast<const V *>(a.cols64) : reinterpret_cast<const V *>(a.cols);
    const int tid = threadIdx.x;
    double local = 0.0;
    for (int row = r0 + NR * tid; row < r1; row += NR * T) {
        V pr[NR];
        fi_forward<V, NR, false>(ins, cv, cols, a.npad, row, stk, nullptr, T, tid, pr, ccols);
#pragma unroll
        for (int i = 0; i < NR; ++i) {
            const int rr = row + i;
            if (rr >= r1) continue;
            const double wr = a.w ? a.w[rr] : 1.0;
            if (wr <= 0.0) continue;
            if (F64) {
                const double pred = (double)pr[i];
                const double r = pred - a.y64[rr];
                if (!isfinite(pred) || !isfinite(r)) local += 1e30;
                else if (a.metric == FM_LOGISTIC) {
                    const double tt = a.tsign64 ? a.tsign64[rr] : 0.0;
                    local += isfinite(tt) ? wr * ft_softplus_neg(tt * pred) : 1e30;
                } else if (a.metric == FM_SQUARED) local += wr * r * r;
                else if (a.metric == FM_ABSOLUTE) local += wr * fabs(r);
                else local += wr * log1p(r * r);
            } else {
                const float pred = (float)pr[i];
                const float r = pred - a.y[rr];
                if (!isfinite(pred) || fabsf(pred) > 1e30f || !isfinite(r)) local += 1e30;
                else if (a.metric == FM_LOGISTIC) {
                    const double tt = a.tsign ? (double)a.tsign[rr] : 0.0;
                    local += isfinite(tt) ? wr * ft_softplus_neg(tt * (double)pred) : 1e30;
                } else if (a.metric == FM_SQUARED) local += wr * (double)r * (double)r;
                else local += wr * (double)ft_row_loss_f(r, a.metric);
            }
        }
    }
    const double total = ft_block_sum<T>(local, red);
    if (tid == 0) {
        pt[FT_PART_LOSS] = total;
        pt[FT_PART_BAD] = 0.0;
    }
}

/* The weighted moments of one tile for the correlation trial score
   (eval.cu:2170-2214): W, sum w f, sum w f^2, sum w f y, sum w y,
   sum w y^2 in f64 from the f32 forward sweep, in pt[0..5]. A row whose
   prediction or target is not finite marks the tile bad, which rejects the
   trial. */
template <int NR, int T>
__device__ void ft_tile_corr_score(const FitArgs &a, const FIns *ins, const float *cv,
                                   typename FiV<float, NR>::V4 *stk, double *red, int r0, int r1,
                                   double *pt, const float *ccols)
{
    const int tid = threadIdx.x;
    double m[6] = {0.0, 0.0, 0.0, 0.0, 0.0, 0.0};
    int bad = 0;
    for (int row = r0 + NR * tid; row < r1; row += NR * T) {
        float pr[NR];
        fi_forward<float, NR, false>(ins, cv, a.cols, a.npad, row, stk, nullptr, T, tid, pr, ccols);
#pragma unroll
        for (int i = 0; i < NR; ++i) {
            const int rr = row + i;
            if (rr >= r1) continue;
            const double wr = a.w ? a.w[rr] : 1.0;
            if (wr <= 0.0) continue;
            const double f = (double)pr[i], t = (double)a.y[rr];
            if (!isfinite(f) || fabs(f) > 1e30 || !isfinite(t)) {
                bad = 1;
                continue;
            }
            m[0] += wr;
            m[1] += wr * f;
            m[2] += wr * f * f;
            m[3] += wr * f * t;
            m[4] += wr * t;
            m[5] += wr * t * t;
        }
    }
    bad = __syncthreads_or(bad);
#pragma unroll
    for (int k = 0; k < 6; ++k) {
        const double s = ft_block_sum<T>(m[k], red);
        if (tid == 0) pt[k] = s;
    }
    if (tid == 0) pt[FT_PART_BAD] = bad ? 1.0 : 0.0;
}

/* The assembly / objective sweeps (f32 and f64) over the four-row
   interpreter: a persistent grid over the queued (candidate, tile) items. */
template <int OPK, int T>
__global__ void __launch_bounds__(T) ft_sweep4(FitArgs a, int q)
{
    constexpr int BK = ft_base_kind(OPK);
    using V = typename std::conditional<BK == FOP_ASM64 || BK == FOP_LOSS64, double, float>::type;
    constexpr int NR = (BK == FOP_ASM32 || BK == FOP_CASM) ? FT_ASM32_NR
                       : BK == FOP_ASM64                     ? FT_ASM64_NR
                       : (BK == FOP_LOSS32 || BK == FOP_CSCORE) ? FT_LOSS32_NR
                                                                : FT_LOSS64_NR;
    using V4 = typename FiV<V, NR>::V4;
    extern __shared__ __align__(16) unsigned char sm[];
    FIns *ins = reinterpret_cast<FIns *>(sm);
    V *cv = reinterpret_cast<V *>(sm + 8 * (size_t)((a.fmaxins + 1) & ~1));
    unsigned char *region = reinterpret_cast<unsigned char *>(sm + 8 * (size_t)((a.fmaxins + 1) & ~1) +
                                                              8 * FT_MAX_CONST);
    /* a class queue's region is sized for its class; the 128-thread launch
       of a base assembly kind for every candidate it may hold */
    const size_t asm_reg = OPK != BK ? a.asm_reg[ft_kind_cls(OPK)]
                           : (BK == FOP_CASM ? a.asm_region : a.asm_reg[0]);
    double *red = reinterpret_cast<double *>(
        region + (ft_op_assembles(OPK) ? asm_reg
                                       : 16 * (size_t)(a.fslots > 0 ? a.fslots : 1) * T));
    __shared__ int s_item;
    const int tid = threadIdx.x;
    const int *list = a.lists + ((size_t)q * FOP_COUNT + OPK) * a.nprog;
    const int total = a.counts[q * FOP_COUNT + OPK] * a.ntiles;
    int *work = a.work + q * FOP_COUNT + OPK;
    for (;;) {
        if (tid == 0) s_item = atomicAdd(work, 1);
        __syncthreads();
        const int item = s_item;
        __syncthreads();
        if (item >= total) break;
        const int cand = list[item / a.ntiles];
        const int tile = item % a.ntiles;
        const FitState *st = a.state + cand;
        const int ib = a.fins_off[cand];
        const int4 info = a.finfo[cand];
        const int nr = info.y;
        /* f32 sweeps run the cached forward list (constant-free subtrees read
           from the cache), the f64 polish the full one */
        const bool CACHED = sizeof(V) == 4 || a.cache64 != nullptr;
        const int2 fc = CACHED ? a.fcinfo[cand] : make_int2(info.x, 0);
        const int nf = fc.x;
        const FIns *fsrc = a.fins + ib + (CACHED ? info.x + nr : 0);
        const V *ccols =
            !CACHED ? nullptr
                    : (sizeof(V) == 4 ? reinterpret_cast<const V *>(a.cache)
                                      : reinterpret_cast<const V *>(a.cache64)) +
                          (size_t)fc.y * a.npad;
        const int p = a.pcount[cand];
        const int sel = st->sel;
        for (int i = tid; i < nf; i += T) ins[i] = fsrc[i];
        if (ft_op_assembles(OPK))
            for (int i = tid; i < nr; i += T) ins[nf + i] = a.fins[ib + info.x + i];
        if (tid < p) cv[tid] = (V)(sel ? st->trial[tid] : st->c[tid]);
        __syncthreads();
        const int r0 = tile * FT_TILE_ROWS;
        const int r1 = min(a.n, r0 + FT_TILE_ROWS);
        double *pt = a.part + ((size_t)cand * a.ntiles + tile) * FT_PART_STRIDE;
        if (ft_op_assembles(OPK))
            ft_tile_asm<V, NR, T, BK == FOP_CASM>(a, ins, ins + nf, nr, p, info.z & 0xffff,
                                                  info.w & 0xffff,
                                                  info.w >> 16, cv, region, red, r0, r1, pt, ccols);
        else if (BK == FOP_CSCORE)
            ft_tile_corr_score<NR, T>(a, ins, reinterpret_cast<const float *>(cv),
                                      reinterpret_cast<typename FiV<float, NR>::V4 *>(region), red,
                                      r0, r1, pt, reinterpret_cast<const float *>(ccols));
        else
            ft_tile_loss<V, NR, T>(a, ins, cv, reinterpret_cast<V4 *>(region), red, r0, r1, pt,
                                   ccols);
        __syncthreads();
    }
}

/* Values of the cached constant-free subtrees over all rows, once per fit:
   one block per (subtree, 2048-row tile), four rows per thread, the same
   f32 forward sweep the other kinds run (so a cached value is bit-identical
   to the value a full forward sweep computes). */
#define FT_FILL_T 128
__global__ void __launch_bounds__(FT_FILL_T) ft_cache_fill(FitArgs a)
{
    using V4 = FiV<float, 4>::V4;
    extern __shared__ __align__(16) unsigned char sm[];
    FIns *ins = reinterpret_cast<FIns *>(sm);
    V4 *stk = reinterpret_cast<V4 *>(sm + 8 * (size_t)((a.sub_maxins + 1) & ~1));
    const int s = blockIdx.x / a.ntiles, tile = blockIdx.x % a.ntiles;
    const int tid = threadIdx.x;
    const int b = a.sub_off[s], ni = a.sub_off[s + 1] - b;
    for (int i = tid; i < ni; i += FT_FILL_T) ins[i] = a.sub_fins[b + i];
    __syncthreads();
    const int r0 = tile * FT_TILE_ROWS, r1 = min(a.n, r0 + FT_TILE_ROWS);
    float *out = a.cache + (size_t)a.sub_col[s] * a.npad;
    for (int row = r0 + 4 * tid; row < r1; row += 4 * FT_FILL_T) {
        float pr[4];
        fi_forward<float, 4, false>(ins, nullptr, a.cols, a.npad, row, stk, nullptr, FT_FILL_T, tid,
                                    pr);
#pragma unroll
        for (int i = 0; i < 4; ++i)
            if (row + i < r1) out[row + i] = pr[i];
    }
}

/* The f64 twin of ft_cache_fill for the polish sweeps (two rows per
   thread). The subtrees are the same programs, so each column holds exactly
   the values the f64 sweeps would compute inline. */
__global__ void __launch_bounds__(FT_FILL_T) ft_cache_fill64(FitArgs a)
{
    using V4 = FiV<double, 2>::V4;
    extern __shared__ __align__(16) unsigned char sm[];
    FIns *ins = reinterpret_cast<FIns *>(sm);
    V4 *stk = reinterpret_cast<V4 *>(sm + 8 * (size_t)((a.sub_maxins + 1) & ~1));
    const int s = blockIdx.x / a.ntiles, tile = blockIdx.x % a.ntiles;
    const int tid = threadIdx.x;
    const int b = a.sub_off[s], ni = a.sub_off[s + 1] - b;
    for (int i = tid; i < ni; i += FT_FILL_T) ins[i] = a.sub_fins[b + i];
    __syncthreads();
    const int r0 = tile * FT_TILE_ROWS, r1 = min(a.n, r0 + FT_TILE_ROWS);
    double *out = a.cache64 + (size_t)a.sub_col[s] * a.npad;
    for (int row = r0 + 2 * tid; row < r1; row += 2 * FT_FILL_T) {
        double pr[2];
        fi_forward<double, 2, false>(ins, nullptr, a.cols64, a.npad, row, stk, nullptr, FT_FILL_T,
                                     tid, pr);
#pragma unroll
        for (int i = 0; i < 2; ++i)
            if (row + i < r1) out[row + i] = pr[i];
    }
}

/* ---- the per-candidate controller --------------------------------------- */

/* ---- correlation objective (eval.cu:1959-2262) ----------------------- */

/* From the assembled augmented Gram (columns: the p Jacobian columns,
   sqrt(w), sqrt(w) f, sqrt(w) y; lower triangle, row stride W): rho, the
   variances, the gradient of rho in st.jtr and its Gauss-Newton curvature in
   st.jtj (eval.cu:2118-2160). Returns the objective 1 - |rho| (1 - rho when
   signed); bad marks a non-finite result. */
__device__ double ft_corr_moments(const double *gram, int W, int p, int metric, FitState &st,
                                  int &bad)
{
    auto G = [&](int i, int j) { return gram[i * W + j]; };
    const double Wt = G(p, p);
    const double sum_f = G(p + 1, p), sum_f2 = G(p + 1, p + 1), sum_ft = G(p + 2, p + 1);
    const double sum_t = G(p + 2, p), sum_t2 = G(p + 2, p + 2);
    double sff = 0.0, syy = 0.0, rho = 0.0;
    bool ident = true;
    if (Wt > 0.0) {
        const double mf = sum_f / Wt, mt = sum_t / Wt;
        sff = sum_f2 - Wt * mf * mf;
        syy = sum_t2 - Wt * mt * mt;
        const double sft = sum_ft - Wt * mf * mt;
        if (sff > 0.0 && syy > 0.0) {
            rho = sft / sqrt(sff * syy);
            const double root = sqrt(sff * syy);
            double av[FT_MAX_CONST], gbar[FT_MAX_CONST];
            for (int j = 0; j < p; ++j) {
                gbar[j] = G(p, j) / Wt;
                av[j] = G(p + 1, j) - Wt * gbar[j] * mf;
                const double bj = G(p + 2, j) - Wt * gbar[j] * mt;
                st.jtr[j] = bj / root - rho * av[j] / sff;
            }
            int k = 0;
            for (int i = 0; i < p; ++i)
                for (int j = 0; j <= i; ++j, ++k) {
                    const double centred = G(i, j) - Wt * gbar[i] * gbar[j];
                    st.jtj[k] = (centred - av[i] * av[j] / sff) / sff;
                }
            ident = false;
        }
    }
    if (ident) {
        int k = 0;
        for (int i = 0; i < p; ++i) {
            st.jtr[i] = 0.0;
            for (int j = 0; j <= i; ++j, ++k) st.jtj[k] = i == j ? 1.0 : 0.0;
        }
    }
    st.svar = sff;
    st.syy = syy;
    st.rho = rho;
    const double score = metric == FM_CORRELATION_SIGNED ? 1.0 - rho : 1.0 - fabs(rho);
    bad = (!isfinite(score) || !isfinite(sff) || !isfinite(syy)) ? 1 : 0;
    return score;
}

/* The value-only objective from the six weighted sums (eval.cu:2226-2234). */
__device__ double ft_corr_trial(const double *m, int metric)
{
    const double Wt = m[0];
    if (!(Wt > 0.0)) return 1e30;
    const double mf = m[1] / Wt, mt = m[4] / Wt;
    const double sff = m[2] - Wt * mf * mf;
    const double syy = m[5] - Wt * mt * mt;
    const double sft = m[3] - Wt * mf * mt;
    if (!(sff > 0.0) || !(syy > 0.0)) return 1.0;
    const double rho = sft / sqrt(sff * syy);
    return metric == FM_CORRELATION_SIGNED ? 1.0 - rho : 1.0 - fabs(rho);
}

/* Turn the rho gradient into the objective's (L = 1 - sigma rho, so the
   damped solve with jtr = dL steps along -H^-1 dL) and freeze the gauge
   slots: zero right-hand side, identity row and column (eval.cu:2239-2258).
   Applied in place to the assembled system before every solve, as the
   reference does. */
__device__ void ft_corr_mask(FitState &st, int p, int metric, const int *g)
{
    const double sigma = metric == FM_CORRELATION_SIGNED ? 1.0 : (st.rho >= 0.0 ? 1.0 : -1.0);
    for (int j = 0; j < p; ++j) st.jtr[j] = -sigma * st.jtr[j];
    for (int i = 0; i < p; ++i) {
        const bool gi = g[0] == i || g[1] == i;
        for (int j = 0; j <= i; ++j) {
            const bool gj = g[0] == j || g[1] == j;
            if (gi || gj) st.jtj[i * (i + 1) / 2 + j] = i == j ? 1.0 : 0.0;
        }
        if (gi) st.jtr[i] = 0.0;
    }
}

/* Status labels of a finished fit (eval.cu:2583-2600), then the outputs. */
__device__ void ft_finish(const FitArgs &a, FitState &st, int cand, int p)
{
    int status = st.status;
    if (st.pc == PC_END) {
        if (status == 1 || status == 2) {
            if (!st.start) status = 7;
            else if (st.improved) status = 5;
            else status = 6;
        } else if (status == 0) {
            if (st.skip) status = 8;
            else if (st.rank) status = 4;
            else if (!st.improved && a.iters > 0) status = 6;
        }
    }
    if (st.pc == PC_C_END) {
        /* a finite correlation answer is returned as is (eval.cu:2430-2440) */
        if (status == 1 || status == 2) status = !st.start ? 7 : (st.improved ? 5 : 6);
        else if (status == 0 && st.rank) status = 4;
    }
    for (int j = 0; j < p; ++j) a.outc[(size_t)cand * a.kmax + j] = st.c[j];
    a.outsse[cand] = st.best;
    a.outstatus[cand] = status;
    st.pc = PC_DONE;
    st.op = FOP_NONE;
}

/* Advance one candidate's LM until it needs a sweep (st.op set) or is done.
   `rl`, `rb`, `rs` are the reduced objective / bad / skipped flags of the
   sweep that just ran; jtj/jtr of an assembly are already in `st`. The
   control flow is eval.cu:2437-2580 (and implicit.rs:277-409 for metric 6),
   unrolled into explicit states. Thread 0 only. */
__device__ void ft_advance(const FitArgs &a, FitState &st, int cand, int p, double rl, int rb,
                           int rs, double *L, double *delta)
{
    const int irls = a.metric == FM_ABSOLUTE;
    const int iters = a.iters;
    const int rounds = irls ? (iters < 1 ? 1 : (iters < 4 ? iters : 4)) : 1;
    const int inner = irls ? (iters / rounds < 1 ? 1 : iters / rounds) : iters;
    for (int guard = 0; guard < 256; ++guard) {
        switch (st.pc) {
            case PC_INIT:
                st.lambda = 1e-3;
                st.req = FT_REQ_NONE;
                st.f64 = 0;
                st.nsw[0] = st.nsw[1] = st.nsw[2] = st.nsw[3] = 0;
                st.status = 0;
                st.best = 0.0;
                st.rank = st.skip = st.improved = st.start = 0;
                st.assembled = 0;
                if (!a.valid[cand]) {
                    st.status = 1;
                    st.best = INFINITY;
                    st.pc = PC_DONE;
                    ft_finish(a, st, cand, p);
                    return;
                }
                if (a.metric == FM_IMPLICIT) {
                    st.pc = PC_I_INIT;
                    break;
                }
                if (a.metric == FM_CORRELATION || a.metric == FM_CORRELATION_SIGNED) {
                    st.pc = PC_C_INIT;
                    break;
                }
                if (iters <= 0) {
                    st.pc = PC_END;
                    break;
                }
                st.op = FOP_ASM32;
                st.sel = 0;
                st.pc = PC_AFTER_FIRST_ASM;
                return;
            case PC_AFTER_FIRST_ASM:
                if (ft_rescue(a.flags, st, rb)) return;
                /* in f64 a row skipped for a non-finite Jacobian entry fails
                   the assembly, as it fails the CPU's normal equations */
                if (st.f64) {
                    rb = rb || rs;
                    st.f64 = 2;
                }
                st.best = rl;
                st.start = rb ? 0 : 1;
                st.assembled = 1;
                if (rb) {
                    st.status = 2;
                    st.pc = PC_REBASE;
                    break;
                }
                st.round = 0;
                st.pc = PC_ROUND;
                break;
            case PC_ROUND:
                if (!(st.round < rounds && st.status == 0 && st.best != 0.0)) {
                    st.pc = PC_REBASE;
                    break;
                }
                if (irls && st.round > 0) st.assembled = 0;
                st.it = 0;
                st.pc = PC_ITER;
                break;
            case PC_ITER:
                if (!(st.it < inner && st.status == 0)) {
                    st.round++;
                    st.pc = PC_ROUND;
                    break;
                }
                if (!st.assembled) {
                    st.op = st.f64 ? FOP_ASM64 : FOP_ASM32;
                    st.sel = 0;
                    st.pc = PC_AFTER_ASM;
                    return;
                }
                st.pc = PC_SOLVE;
                break;
            case PC_AFTER_ASM:
                if (ft_rescue(a.flags, st, rb)) return;
                if (st.f64) rb = rb || rs;
                st.assembled = 1;
                if (rb) {
                    st.status = 2;
                    st.round++;
                    st.pc = PC_ROUND;
                    break;
                }
                if (st.f64 == 1) {
                    /* just switched: the loss to beat is the f64 one */
                    st.best = rl;
                    st.f64 = 2;
                }
                st.pc = PC_SOLVE;
                break;
            case PC_SOLVE: {
                if (st.req != FT_REQ_DONE) {
                    ft_request_solve(st, st.lambda);
                    return;
                }
                const int sv = ft_take_solve(st);
                if (sv == 1) {
                    st.status = 1;
                    st.round++;
                    st.pc = PC_ROUND;
                    break;
                }
                if (sv == 4) st.rank = 1;
                for (int j = 0; j < p; ++j) st.trial[j] = fmin(1e6, fmax(-1e6, st.c[j] + delta[j]));
                st.half = 0;
                st.op = st.f64 ? FOP_LOSS64 : FOP_LOSS32;
                st.sel = 1;
                st.pc = PC_AFTER_TRIAL;
                return;
            }
            case PC_AFTER_TRIAL: {
                const double tsse = rl;
                /* true-metric Armijo for L1: two halvings (eval.cu:2486-2497) */
                if (irls && st.half < 2 && !(tsse < st.best)) {
                    for (int j = 0; j < p; ++j) st.trial[j] = st.c[j] + 0.5 * (st.trial[j] - st.c[j]);
                    st.half++;
                    st.op = st.f64 ? FOP_LOSS64 : FOP_LOSS32;
                    st.sel = 1;
                    return;
                }
                if (tsse < st.best) {
                    for (int j = 0; j < p; ++j) st.c[j] = st.trial[j];
                    st.best = tsse;
                    st.lambda = fmax(st.lambda / 8.0, 1e-12);
                    st.improved = 1;
                    st.assembled = 0;
                    if (st.best == 0.0) {
                        st.round++;
                        st.pc = PC_ROUND;
                        break;
                    }
                } else {
                    st.lambda *= 6.0;
                    if (st.lambda > 1e9) {
                        st.round++;
                        st.pc = PC_ROUND;
                        break;
                    }
                }
                st.it++;
                st.pc = PC_ITER;
                break;
            }
            case PC_REBASE:
                if (st.status == 0 && !(a.flags & FT_FLAG_NO_POLISH)) {
                    st.op = FOP_LOSS64;
                    st.sel = 0;
                    st.pc = PC_AFTER_REBASE;
                    return;
                }
                st.pc = PC_END;
                break;
            case PC_AFTER_REBASE:
                if (isfinite(rl)) st.best = rl;
                st.pit = 0;
                st.pc = PC_POLISH;
                break;
            case PC_POLISH:
                if (!(st.pit < 4 && st.status == 0 && st.best != 0.0)) {
                    st.pc = PC_END;
                    break;
                }
                st.op = FOP_ASM64;
                st.sel = 0;
                st.pc = PC_AFTER_PASM;
                return;
            case PC_AFTER_PASM: {
                if (st.req != FT_REQ_DONE) {
                    if (rs) st.skip = 1;
                    if (rb) {
                        st.status = 2;
                        st.pc = PC_END;
                        break;
                    }
                    ft_request_solve(st, 0.0);
                    return;
                }
                const int sv = ft_take_solve(st);
                if (sv == 1) {
                    st.pc = PC_END;
                    break;
                }
                if (sv == 4) st.rank = 1;
                for (int j = 0; j < p; ++j) st.trial[j] = fmin(1e6, fmax(-1e6, st.c[j] + delta[j]));
                st.half = 0;
                st.op = FOP_LOSS64;
                st.sel = 1;
                st.pc = PC_AFTER_PTRIAL;
                return;
            }
            case PC_AFTER_PTRIAL: {
                const double tsse = rl;
                if (irls && st.half == 0 && !(tsse < st.best)) {
                    for (int j = 0; j < p; ++j) st.trial[j] = st.c[j] + 0.5 * (st.trial[j] - st.c[j]);
                    st.half = 1;
                    st.op = FOP_LOSS64;
                    st.sel = 1;
                    return;
                }
                if (tsse < st.best) {
                    for (int j = 0; j < p; ++j) st.c[j] = st.trial[j];
                    st.best = tsse;
                    st.improved = 1;
                    st.pit++;
                    st.pc = PC_POLISH;
                    break;
                }
                st.pc = PC_END;
                break;
            }
            case PC_END:
                ft_finish(a, st, cand, p);
                return;
            /* ---- correlation metric (eval.cu:2316-2440) ---- */
            case PC_C_INIT: {
                const int *g = a.gauge + 2 * cand;
                const int gs = g[0], go = g[1];
                if (gs >= 0 && gs < p && isfinite(st.c[gs]) && st.c[gs] != 0.0)
                    st.c[gs] = st.c[gs] > 0.0 ? 1.0 : -1.0;
                if (go >= 0 && go < p) st.c[go] = 0.0;
                st.best = 1.0;
                st.op = iters > 0 ? FOP_CASM : FOP_CSCORE;
                st.sel = 0;
                st.pc = iters > 0 ? PC_C_AFTER_FIRST : PC_C_SCORE_ONLY;
                return;
            }
            case PC_C_SCORE_ONLY:
                st.best = rl;
                st.pc = PC_C_END;
                break;
            case PC_C_AFTER_FIRST:
                st.start = rb ? 0 : 1;
                st.assembled = 1;
                if (rb) {
                    st.status = 2;
                    st.pc = PC_C_END;
                } else if (!(st.svar > 0.0) || !(st.syy > 0.0)) {
                    st.best = 1.0;
                    st.pc = PC_C_END;
                } else if (st.svar < 1e-24 * st.syy) {
                    st.status = 1;
                    st.pc = PC_C_END;
                } else {
                    st.best = rl;
                    st.lambda = 1e-3;
                    st.it = 0;
                    st.pc = PC_C_ITER;
                }
                break;
            case PC_C_ITER:
                if (!(st.it < iters && st.status == 0)) {
                    st.pit = 0;
                    st.pc = PC_C_POLISH;
                    break;
                }
                if (!st.assembled) {
                    st.op = FOP_CASM;
                    st.sel = 0;
                    st.pc = PC_C_AFTER_ASM;
                    return;
                }
                st.pc = PC_C_SOLVE;
                break;
            case PC_C_AFTER_ASM:
                st.assembled = 1;
                if (rb) {
                    st.status = 2;
                    st.pc = PC_C_END;
                    break;
                }
                if (st.svar < 1e-24 * st.syy) {
                    st.status = 1;
                    st.pc = PC_C_END;
                    break;
                }
                st.pc = PC_C_SOLVE;
                break;
            case PC_C_SOLVE: {
                if (st.req != FT_REQ_DONE) {
                    ft_corr_mask(st, p, a.metric, a.gauge + 2 * cand);
                    ft_request_solve(st, st.lambda);
                    return;
                }
                const int sv = ft_take_solve(st);
                if (sv == 1) {
                    st.status = 1;
                    st.pc = PC_C_END;
                    break;
                }
                if (sv == 4) st.rank = 1;
                for (int j = 0; j < p; ++j) st.trial[j] = fmin(1e6, fmax(-1e6, st.c[j] + delta[j]));
                st.op = FOP_CSCORE;
                st.sel = 1;
                st.pc = PC_C_AFTER_TRIAL;
                return;
            }
            case PC_C_AFTER_TRIAL:
                if (rl < st.best) {
                    for (int j = 0; j < p; ++j) st.c[j] = st.trial[j];
                    st.best = rl;
                    st.lambda = fmax(st.lambda / 8.0, 1e-12);
                    st.assembled = 0;
                    st.improved = 1;
                    if (st.best <= 0.0) {
                        st.pit = 0;
                        st.pc = PC_C_POLISH;
                        break;
                    }
                } else {
                    st.lambda *= 6.0;
                    if (st.lambda > 1e9) {
                        st.pit = 0;
                        st.pc = PC_C_POLISH;
                        break;
                    }
                }
                st.it++;
                st.pc = PC_C_ITER;
                break;
            case PC_C_POLISH:
                if (!(st.pit < 4 && st.status == 0 && st.best > 0.0)) {
                    st.pc = PC_C_END;
                    break;
                }
                st.op = FOP_CASM;
                st.sel = 0;
                st.pc = PC_C_AFTER_PASM;
                return;
            case PC_C_AFTER_PASM: {
                if (st.req != FT_REQ_DONE) {
                    if (rb) {
                        st.status = 2;
                        st.pc = PC_C_END;
                        break;
                    }
                    ft_corr_mask(st, p, a.metric, a.gauge + 2 * cand);
                    ft_request_solve(st, 0.0);
                    return;
                }
                const int sv = ft_take_solve(st);
                if (sv == 1) {
                    st.pc = PC_C_END;
                    break;
                }
                if (sv == 4) st.rank = 1;
                for (int j = 0; j < p; ++j) st.trial[j] = fmin(1e6, fmax(-1e6, st.c[j] + delta[j]));
                st.op = FOP_CSCORE;
                st.sel = 1;
                st.pc = PC_C_AFTER_PTRIAL;
                return;
            }
            case PC_C_AFTER_PTRIAL:
                if (rl < st.best) {
                    for (int j = 0; j < p; ++j) st.c[j] = st.trial[j];
                    st.best = rl;
                    st.improved = 1;
                    st.pit++;
                    st.pc = PC_C_POLISH;
                } else {
                    st.pc = PC_C_END;
                }
                break;
            case PC_C_END:
                ft_finish(a, st, cand, p);
                return;
            /* ---- implicit metric ---- */
            case PC_I_INIT:
                for (int j = 0; j < p; ++j) st.start_c[j] = st.c[j];
                st.op = FOP_ICOST;
                st.sel = 0;
                st.pc = PC_I_AFTER_BASE;
                return;
            case PC_I_AFTER_BASE:
                if (rb) {
                    st.best = INFINITY;
                    st.status = 7;
                    st.pc = PC_I_END;
                    break;
                }
                st.best = rl;
                st.start_best = rl;
                st.it = 0;
                st.pc = (p == 0 || iters <= 0) ? PC_I_END : PC_I_ITER;
                break;
            case PC_I_ITER:
                if (st.it >= (iters < 1 ? 1 : iters)) {
                    st.pc = PC_I_END;
                    break;
                }
                /* the reference recomputes the residuals and Jacobian at an
                   unchanged point after a rejected or singular step; the
                   system kept from the last assembly is the same one */
                if (!st.assembled) {
                    st.op = (a.ijac_small > 0 &&
                             a.node_off[cand + 1] - a.node_off[cand] <= a.ijac_small)
                                ? FOP_IJACS
                                : FOP_IJAC;
                    st.sel = 0;
                    st.pc = PC_I_AFTER_JAC;
                    return;
                }
                st.pc = PC_I_SOLVE;
                break;
            case PC_I_AFTER_JAC:
                if (rb) {
                    st.pc = PC_I_END;
                    break;
                }
                st.assembled = 1;
                st.pc = PC_I_SOLVE;
                break;
            case PC_I_SOLVE: {
                const int sv = ft_gauss_solve(st.jtj, st.jtr, st.lambda, p, delta, L);
                if (sv != 0) {
                    st.lambda *= 6.0;
                    st.it++;
                    st.pc = st.lambda > 1e9 ? PC_I_END : PC_I_ITER;
                    break;
                }
                for (int j = 0; j < p; ++j) st.trial[j] = fmin(1e6, fmax(-1e6, st.c[j] + delta[j]));
                st.op = FOP_ICOST;
                st.sel = 1;
                st.pc = PC_I_AFTER_TRIAL;
                return;
            }
            case PC_I_AFTER_TRIAL:
                st.it++;
                if (!rb && rl < st.best) {
                    st.best = rl;
                    for (int j = 0; j < p; ++j) st.c[j] = st.trial[j];
                    st.lambda = fmax(st.lambda / 8.0, 1e-12);
                    st.improved = 1;
                    st.assembled = 0;
                    st.pc = st.best == 0.0 ? PC_I_END : PC_I_ITER;
                } else {
                    st.lambda *= 6.0;
                    st.pc = st.lambda > 1e9 ? PC_I_END : PC_I_ITER;
                }
                break;
            case PC_I_END:
                /* the reference writes constants back only when they beat the
                   start (implicit.rs:402-405) */
                if (!(st.best < st.start_best))
                    for (int j = 0; j < p; ++j) st.c[j] = st.start_c[j];
                if (st.status != 7) st.status = st.improved ? 0 : 6;
                ft_finish(a, st, cand, p);
                return;
            default:
                st.op = FOP_NONE;
                return;
        }
    }
    /* Unreachable for well-formed state; close the candidate rather than spin. */
    st.pc = PC_END;
    ft_finish(a, st, cand, p);
}

#define FT_CTRL_T 128

/* Reduce the tile partials of each candidate that had a sweep at parity q,
   advance its LM and queue its next sweep at parity q^1. With `init`, start
   every candidate instead. */
__global__ void __launch_bounds__(FT_CTRL_T) ft_control(FitArgs a, int q, int init)
{
    __shared__ FitState sst;
    __shared__ double L[FT_MAX_CONST * (FT_MAX_CONST + 1)];
    __shared__ double delta[FT_MAX_CONST];
    __shared__ double gram[24 * 24];
    __shared__ int s_task, s_cand, s_op;
    __shared__ double s_loss;
    __shared__ double red[FT_CTRL_T];
    __shared__ int s_bad, s_skip;
    const int tid = threadIdx.x;
    const int nq = q ^ 1;
    int total = 0;
    if (init) total = a.nprog;
    else
        for (int k = 1; k < FOP_COUNT; ++k) total += a.counts[q * FOP_COUNT + k];
    int *work = a.work + q * FOP_COUNT + FOP_NONE;
    for (;;) {
        if (tid == 0) {
            const int t = atomicAdd(work, 1);
            s_task = t;
            if (t < total) {
                int cand = t, op = FOP_NONE;
                if (!init) {
                    int k = 1, base = 0;
                    while (t >= base + a.counts[q * FOP_COUNT + k]) {
                        base += a.counts[q * FOP_COUNT + k];
                        ++k;
                    }
                    op = ft_base_kind(k);
                    cand = a.lists[((size_t)q * FOP_COUNT + k) * a.nprog + (t - base)];
                }
                s_cand = cand;
                s_op = op;
            }
        }
        __syncthreads();
        if (s_task >= total) break;
        const int cand = s_cand, op = s_op;
        const int p = a.pcount[cand];
        {
            const double *src = reinterpret_cast<const double *>(a.state + cand);
            double *dst = reinterpret_cast<double *>(&sst);
            for (int i = tid; i < (int)(sizeof(FitState) / 8); i += FT_CTRL_T) dst[i] = src[i];
        }
        if (init && tid < p) {
            /* fresh state: the caller's starting constants */
            sst.c[tid] = a.c0[(size_t)cand * a.kmax + tid];
        }
        __syncthreads();
        if (init && tid == 0) sst.pc = PC_INIT;
        const double *pt = a.part + (size_t)cand * a.ntiles * FT_PART_STRIDE;
        const int W = 4 * ((ft_gram_cols(op, p) + 3) / 4);
        if (!init && ft_op_assembles(op)) {
            const int nb = W / 4;
            const int nblk = nb * (nb + 1) / 2;
            for (int e = tid; e < nblk * 16; e += FT_CTRL_T) {
                double s = 0.0;
                for (int t = 0; t < a.ntiles; ++t) s += pt[(size_t)t * FT_PART_STRIDE + e];
                int b = e >> 4, bi = 0;
                while (b > bi) {
                    b -= bi + 1;
                    ++bi;
                }
                gram[(4 * bi + ((e & 15) >> 2)) * W + 4 * b + (e & 3)] = s;
            }
            __syncthreads();
            for (int e = tid; op != FOP_CASM && e < p * (p + 1) / 2 + p; e += FT_CTRL_T) {
                if (e < p * (p + 1) / 2) {
                    int i = 0, k = e;
                    while (k > i) {
                        k -= i + 1;
                        ++i;
                    }
                    sst.jtj[e] = gram[i * W + k];
                } else {
                    const int j = e - p * (p + 1) / 2;
                    sst.jtr[j] = gram[p * W + j];
                }
            }
        }
        /* loss, flags and (correlation score) moments over the tiles: each
           thread takes every FT_CTRL_T-th tile, then a fixed-order tree */
        {
            double loss = 0.0;
            double m[6] = {0.0, 0.0, 0.0, 0.0, 0.0, 0.0};
            int bad = 0, skip = 0;
            if (!init) {
                const bool asm_ = ft_op_assembles(op), csc = op == FOP_CSCORE;
                for (int t = tid; t < a.ntiles; t += FT_CTRL_T) {
                    const double *pp = pt + (size_t)t * FT_PART_STRIDE;
                    loss += pp[FT_PART_LOSS];
                    bad |= pp[FT_PART_BAD] != 0.0;
                    if (asm_) skip |= pp[FT_PART_SKIP] != 0.0;
                    if (csc)
                        for (int k = 0; k < 6; ++k) m[k] += pp[k];
                }
            }
            bad = __syncthreads_or(bad);
            skip = __syncthreads_or(skip);
            const int nsum = op == FOP_CSCORE ? 7 : 1;
            for (int k = 0; k < nsum; ++k) {
                red[tid] = k == 0 ? loss : m[k - 1];
                __syncthreads();
                for (int h = FT_CTRL_T / 2; h > 0; h >>= 1) {
                    if (tid < h) red[tid] += red[tid + h];
                    __syncthreads();
                }
                if (tid == 0) {
                    if (k == 0) loss = red[0];
                    else m[k - 1] = red[0];
                }
                __syncthreads();
            }
            if (tid == 0) {
                if (!init) {
                    if (op == FOP_CASM) {
                        int cb = 0;
                        loss = ft_corr_moments(gram, W, p, a.metric, sst, cb);
                        bad |= cb;
                    } else if (op == FOP_CSCORE) {
                        loss = bad ? INFINITY : ft_corr_trial(m, a.metric);
                    }
                }
                s_loss = init ? 0.0 : loss;
                s_bad = init ? 0 : bad;
                s_skip = init ? 0 : skip;
            }
        }
        __syncthreads();
        /* the state machine on thread 0; a solve it requests runs on warp 0
           and the state machine resumes (at most one solve per step) */
        for (int round = 0; round < 4; ++round) {
            if (tid == 0) ft_advance(a, sst, cand, p, s_loss, s_bad, s_skip, L, delta);
            __syncthreads();
            if (sst.req != FT_REQ_SOLVE) break;
            if (tid < 32) {
                const int sv = ft_solve_warp(sst.jtj, sst.jtr, sst.req_lambda, p, delta);
                if (tid == 0) {
                    sst.sv = sv;
                    sst.req = FT_REQ_DONE;
                }
            }
            __syncthreads();
        }
        if (tid == 0 && sst.op != FOP_NONE) {
            const int op = sst.op;
            const int k = (op == FOP_ASM32 || op == FOP_CASM)      ? 0
                          : (op == FOP_LOSS32 || op == FOP_CSCORE) ? 1
                          : (op == FOP_ASM64 || ft_op_ijac(op))     ? 2
                                                                    : 3;
            sst.nsw[k]++;
        }
        __syncthreads();
        {
            const double *src = reinterpret_cast<const double *>(&sst);
            double *dst = reinterpret_cast<double *>(a.state + cand);
            for (int i = tid; i < (int)(sizeof(FitState) / 8); i += FT_CTRL_T) dst[i] = src[i];
        }
        if (tid == 0 && sst.op != FOP_NONE) {
            const int kq = ft_queue_kind(sst.op, a.finfo[cand].z >> 16);
            const int k = atomicAdd(&a.counts[nq * FOP_COUNT + kq], 1);
            a.lists[((size_t)nq * FOP_COUNT + kq) * a.nprog + k] = cand;
        }
        __syncthreads();
    }
}

/* Clear the queue that step s fills and the work counters it consumes. */
__global__ void ft_step_reset(FitArgs a, int q)
{
    const int t = threadIdx.x;
    if (t < FOP_COUNT) {
        a.counts[(q ^ 1) * FOP_COUNT + t] = 0;
        a.work[q * FOP_COUNT + t] = 0;
    }
}

/* Close every candidate that has not finished (a bound, never reached). */
__global__ void ft_flush(FitArgs a)
{
    const int cand = blockIdx.x * blockDim.x + threadIdx.x;
    if (cand >= a.nprog) return;
    FitState &st = a.state[cand];
    if (st.pc == PC_DONE) return;
    if (a.metric == FM_IMPLICIT) {
        if (!(st.best < st.start_best))
            for (int j = 0; j < a.pcount[cand]; ++j) st.c[j] = st.start_c[j];
        if (st.status != 7) st.status = st.improved ? 0 : 6;
    } else {
        st.pc = PC_END;
    }
    ft_finish(a, st, cand, a.pcount[cand]);
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

/* Constant gradients of rows [row0, row0 + nrows) through the same forward
   and reverse sweeps as the f32 assembly (FT_ASM32_NR rows per thread), with
   adjoint seed 1: one warp per (candidate, 32 * FT_ASM32_NR-row tile), tiles
   aligned down to a multiple of FT_ASM32_NR rows. */
__global__ void __launch_bounds__(32) ft_grad4_kernel(FitArgs a, int row0, int nrows, int ntiles,
                                                      float *value, float *out)
{
    constexpr int NR = FT_ASM32_NR;
    using V4 = FiV<float, NR>::V4;
    extern __shared__ __align__(16) unsigned char smem[];
    const int cand = blockIdx.x / ntiles;
    const int tile = blockIdx.x % ntiles;
    const int tid = threadIdx.x;
    if (!a.valid[cand]) return;
    const int4 info = a.finfo[cand];
    const int nf = info.x, nr = info.y, slots = info.w & 0xffff, ntape = info.w >> 16;
    const int p = a.pcount[cand];
    FIns *ins = reinterpret_cast<FIns *>(smem);
    float *cf = reinterpret_cast<float *>(smem + 8 * (size_t)((a.fmaxins + 1) & ~1));
    V4 *stk = reinterpret_cast<V4 *>(cf + FT_MAX_CONST);
    V4 *tape = stk + (size_t)slots * 32;
    float *g = reinterpret_cast<float *>(tape + (size_t)ntape * 32);
    const int R = NR * 32 + 4;
    const int ib = a.fins_off[cand];
    for (int i = tid; i < nf + nr; i += 32) ins[i] = a.fins[ib + i];
    if (tid < p) cf[tid] = (float)a.c0[(size_t)cand * a.kmax + tid];
    for (int i = tid; i < p * R; i += 32) g[i] = 0.0f;
    __syncwarp();
    const int row = (row0 & ~(NR - 1)) + tile * 32 * NR + NR * tid;
    if (row >= row0 + nrows || row >= a.n) return;
    float pr[NR], seed[NR];
    for (int i = 0; i < NR; ++i) seed[i] = 1.0f;
    fi_forward<float, NR, true>(ins, cf, a.cols, a.npad, row, stk, tape, 32, tid, pr);
    fi_reverse<float, NR>(ins + nf, nr, stk, tape, 32, tid, g + tid, R, 32, seed);
    for (int i = 0; i < NR; ++i) {
        const int rr = row + i;
        if (rr < row0 || rr >= row0 + nrows) continue;
        const size_t o = (size_t)cand * nrows + (rr - row0);
        value[o] = pr[i];
        for (int j = 0; j < a.kmax; ++j)
            out[o * a.kmax + j] = j < p ? g[(size_t)j * R + i * 32 + tid] : 0.0f;
    }
}

/* Implicit score per (candidate, tile of rows) on the four-row stack
   machine: each thread carries NR rows through the forward sweep (partials
   on input paths kept) and the input-adjoint reverse sweep (fi_reverse_x),
   then d = |f| / ||grad_x f|| per row (implicit.rs:68-104, the zero-gradient
   guard included); partial sums of w * d and w. A row with a non-finite
   weight, value, gradient or distance marks the candidate bad. */
template <int T, int NR>
__global__ void __launch_bounds__(T) ft_implicit_score_x(
    const FIns *__restrict__ fins, const int *__restrict__ fins_off, const int4 *__restrict__ info,
    const int *__restrict__ valid, const double *__restrict__ c, int kmax,
    const float *__restrict__ cols, int npad, int n, int v, const double *__restrict__ w,
    int ntiles, int rows_per_tile, int maxins, int slots, int ntape, double *partial, int *bad)
{
    using F = FiV<float, NR>;
    using V4 = typename F::V4;
    extern __shared__ __align__(16) unsigned char smem[];
    const int cand = blockIdx.x / ntiles;
    const int tile = blockIdx.x % ntiles;
    const int tid = threadIdx.x;
    FIns *ins = reinterpret_cast<FIns *>(smem);
    float *cf = reinterpret_cast<float *>(smem + 8 * (size_t)((maxins + 1) & ~1));
    V4 *stk = reinterpret_cast<V4 *>(cf + FT_MAX_CONST);
    V4 *tape = stk + (size_t)(slots > 0 ? slots : 1) * T;
    V4 *ig = tape + (size_t)(ntape > 0 ? ntape : 1) * T;
    double *red = reinterpret_cast<double *>(ig + (size_t)v * T);
    int isbad = !valid[cand];
    double sum = 0.0, wsum = 0.0;
    const int r0 = tile * rows_per_tile;
    const int r1 = min(n, r0 + rows_per_tile);
    if (!isbad) {
        const int4 in4 = info[cand];
        const int nf = in4.x, nr = in4.y;
        const int ib = fins_off[cand];
        for (int i = tid; i < nf + nr; i += T) ins[i] = fins[ib + i];
        if (tid < kmax) cf[tid] = (float)c[(size_t)cand * kmax + tid];
        __syncthreads();
        for (int row = r0 + NR * tid; row < r1; row += NR * T) {
            float pr[NR];
            fi_forward<float, NR, true>(ins, cf, cols, npad, row, stk, tape, T, tid, pr);
            for (int k = 0; k < v; ++k) {
                float z[NR];
#pragma unroll
                for (int i = 0; i < NR; ++i) z[i] = 0.0f;
                ig[k * T + tid] = F::pack(z);
            }
            float a[NR];
#pragma unroll
            for (int i = 0; i < NR; ++i) a[i] = 1.0f;
            fi_reverse_x<float, NR>(ins + nf, nr, stk, tape, T, tid, ig, a);
            double nsq[NR];
            bool gfin[NR];
#pragma unroll
            for (int i = 0; i < NR; ++i) {
                nsq[i] = 0.0;
                gfin[i] = true;
            }
            for (int k = 0; k < v; ++k) {
                float g[NR];
                F::unpack(ig[k * T + tid], g);
#pragma unroll
                for (int i = 0; i < NR; ++i) {
                    gfin[i] = gfin[i] && isfinite(g[i]);
                    nsq[i] += (double)g[i] * (double)g[i];
                }
            }
#pragma unroll
            for (int i = 0; i < NR; ++i) {
                const int rr = row + i;
                if (rr >= r1) continue;
                const double wr = w ? w[rr] : 1.0;
                if (!isfinite(wr) || wr < 0.0) {
                    isbad = 1;
                    continue;
                }
                if (wr == 0.0) continue;
                const double norm = sqrt(nsq[i]);
                const bool ok = isfinite(pr[i]) && gfin[i] && isfinite(norm) && norm > 0.0;
                const double d = ok ? fabs((double)pr[i]) / norm : 0.0;
                if (!ok || !isfinite(d)) {
                    isbad = 1;
                    continue;
                }
                sum += wr * d;
                wsum += wr;
            }
            /* an infeasible candidate's sums are not read: stop its rows */
            if (__any_sync(0xffffffffu, isbad) || *((volatile int *)(bad + cand))) {
                isbad = 1;
                break;
            }
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


}  // namespace

/* Decode and check a batch of fit-record programs for the device sweeps. */
void prep_batch(const unsigned int *off, const unsigned int *prog, const int *pcount, int nprog,
                int v, FitPrep &b, int extra_cols, size_t cache_bytes_per_col, size_t cache_cap,
                const int *bucket_budget_kb)
{
    b.node_off.resize(nprog + 1);
    b.valid.resize(nprog);
    b.ninternal.assign(nprog, 0);
    for (int i = 0; i <= nprog; ++i) b.node_off[i] = (int)(off[i] / 4);
    for (int i = 0; i < nprog; ++i) {
        const int m = b.node_off[i + 1] - b.node_off[i];
        const int p = pcount[i];
        const bool ok = (off[i] % 4 == 0) && p >= 0 && p <= FT_MAX_CONST &&
                        validate_records(prog + off[i], m, p, v);
        b.valid[i] = ok ? 1 : 0;
        if (ok) {
            b.mmax = std::max(b.mmax, m);
            b.pmax = std::max(b.pmax, p);
            int ni = 0;
            for (int r = 0; r < m; ++r) {
                const uint32_t op = prog[off[i] + 4 * r];
                ni += op != OP_CONST && op != OP_VAR;
            }
            b.ninternal[i] = ni;
        }
    }
    /* the four-row stack machine's translation (a tree not in stack order is
       rejected as well) */
    b.fins.clear();
    b.fins_off.assign(nprog + 1, 0);
    b.finfo.assign(nprog, make_int4(0, 0, 32, 0));
    b.asm_region = 256;
    for (int k = 0; k < FT_NCLS; ++k) {
        b.asm_reg[k] = 256;
        b.nclass[k] = 0;
    }
    const bool caching = cache_bytes_per_col > 0;
    b.fcinfo.assign(nprog, make_int2(0, 0));
    b.sub_fins.clear();
    b.sub_off.assign(1, 0);
    b.sub_col.clear();
    b.sub_cand_off.assign(nprog + 1, 0);
    b.ncache = 0;
    std::vector<FIns> fwd, rev, fwdc, sf, sr;
    std::vector<std::vector<uint32_t>> subs;
    for (int i = 0; i < nprog; ++i) {
        b.fins_off[i] = (int)b.fins.size();
        b.sub_cand_off[i] = (int)b.sub_col.size();
        if (!b.valid[i]) continue;
        int ns = 0, nt = 0;
        const int m = b.node_off[i + 1] - b.node_off[i];
        if (!fi_decode(prog + off[i], m, fwd, rev, &ns, &nt, caching ? &fwdc : nullptr,
                       caching ? &subs : nullptr) ||
            ns > 0xffff || nt > 0x7fff) {
            b.valid[i] = 0;
            continue;
        }
        b.fins.insert(b.fins.end(), fwd.begin(), fwd.end());
        b.fins.insert(b.fins.end(), rev.begin(), rev.end());
        if (caching) {
            /* the cached list (or the full one again past the cap) */
            const bool fits = (size_t)(b.ncache + (int)subs.size()) * cache_bytes_per_col <= cache_cap;
            bool ok = fits && !subs.empty();
            std::vector<FIns> cand_sub;
            std::vector<int> cand_off;
            int smax = 0, imax = 0;
            for (size_t s = 0; ok && s < subs.size(); ++s) {
                int a2 = 0, b2 = 0;
                if (!fi_decode(subs[s].data(), (int)(subs[s].size() / 4), sf, sr, &a2, &b2)) {
                    ok = false;
                    break;
                }
                cand_off.push_back((int)cand_sub.size());
                cand_sub.insert(cand_sub.end(), sf.begin(), sf.end());
                smax = std::max(smax, a2);
                imax = std::max(imax, (int)sf.size());
            }
            const std::vector<FIns> &use = ok ? fwdc : fwd;
            b.fins.insert(b.fins.end(), use.begin(), use.end());
            b.fcinfo[i] = make_int2((int)use.size(), ok ? b.ncache : 0);
            if (ok) {
                const int base = (int)b.sub_fins.size();
                for (size_t s = 0; s < subs.size(); ++s) {
                    b.sub_col.push_back(b.ncache + (int)s);
                    b.sub_off.push_back(base + (s + 1 < subs.size() ? cand_off[s + 1]
                                                                    : (int)cand_sub.size()));
                }
                b.sub_fins.insert(b.sub_fins.end(), cand_sub.begin(), cand_sub.end());
                b.ncache += (int)subs.size();
                b.sub_slots = std::max(b.sub_slots, smax);
                b.sub_maxins = std::max(b.sub_maxins, imax);
            }
        } else {
            /* no cache: the f32 list is the full one again */
            b.fins.insert(b.fins.end(), fwd.begin(), fwd.end());
            b.fcinfo[i] = make_int2((int)fwd.size(), 0);
        }
        const int ncols = pcount[i] + 1 + extra_cols;
        const int bkt = ft_length_bucket(m);
        const size_t budget = (bucket_budget_kb && bucket_budget_kb[bkt] > 0)
                                  ? (size_t)bucket_budget_kb[bkt] * 1024
                                  : (size_t)FT_ASM_BUDGET;
        const int A = ft_asm_threads(ns, nt, ncols, budget);
        const size_t reg = ft_asm_region(A, ns, nt, 8 * ((ncols + 7) / 8));
        const int cls = ft_cls_of(A, reg);
        /* z: active threads, launch class above bit 16 */
        b.finfo[i] = make_int4((int)fwd.size(), (int)rev.size(), A | (cls << 16),
                               ns | (nt << 16));
        b.asm_region = std::max(b.asm_region, reg);
        b.asm_reg[cls] = std::max(b.asm_reg[cls], reg);
        b.nclass[cls]++;
        b.fslots = std::max(b.fslots, ns);
        b.ftape = std::max(b.ftape, nt);
        b.fmaxins = std::max(b.fmaxins, (int)(fwd.size() + rev.size()));
    }
    b.fins_off[nprog] = (int)b.fins.size();
    b.sub_cand_off[nprog] = (int)b.sub_col.size();
    if (b.fins.empty()) b.fins.resize(1);
    if (b.sub_fins.empty()) b.sub_fins.resize(1);
    if (b.sub_col.empty()) b.sub_col.resize(1);
}

namespace {

int occupancy(const void *fn, int threads, size_t smem)
{
    int blocks = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&blocks, fn, threads, smem) != cudaSuccess) {
        cudaGetLastError();
        return 1;
    }
    return blocks < 1 ? 1 : blocks;
}

/* Upper bound on the sweeps one candidate can request: the first assembly,
   per LM iteration an assembly and up to three objective sweeps (L1 Armijo
   halvings) or one, the f64 re-baseline and four polish steps of an
   assembly and two objective sweeps; for the implicit arm one base sweep and
   two per iteration. */
int max_steps(int iters, int metric)
{
    const int it = iters < 1 ? 1 : iters;
    if (metric == FM_IMPLICIT) return 1 + 2 * it + 1;
    /* correlation: the first assembly, per iteration an assembly and a trial,
       four polish assemblies and trials */
    if (metric == FM_CORRELATION || metric == FM_CORRELATION_SIGNED) return 2 + 2 * it + 8 + 2;
    const int per = metric == FM_ABSOLUTE ? 4 : 2;
    /* + 1: the f64 re-assembly of an f32-only failure (once per fit) */
    return 2 + per * it + 1 + 12 + 1 + 1;
}

struct SweepLaunch {
    const void *fn;
    size_t smem;
    int grid;
    int threads;
    int opk; /* the queue kind it serves */
};

/* Input-mode translation (fi_decode with `inputs`) of every valid candidate:
   [forward | reverse] per candidate, counts and slot sizes in info. A
   candidate it cannot translate becomes invalid. */
struct XPrep {
    std::vector<FIns> fins;
    std::vector<int> off;
    std::vector<int4> info;
    int slots = 1, tape = 1, maxins = 2;
};

void prep_inputs(const unsigned int *off, const unsigned int *prog, int nprog,
                 const std::vector<int> &node_off, std::vector<int> &valid, XPrep &x)
{
    std::vector<FIns> fwd, rev;
    x.fins.clear();
    x.off.assign(nprog + 1, 0);
    x.info.assign(nprog, make_int4(0, 0, 0, 0));
    for (int i = 0; i < nprog; ++i) {
        x.off[i] = (int)x.fins.size();
        if (!valid[i]) continue;
        int ns = 0, nt = 0;
        const int m = node_off[i + 1] - node_off[i];
        if (!fi_decode(prog + off[i], m, fwd, rev, &ns, &nt, nullptr, nullptr, true) ||
            ns > 0xffff || nt > 0x7fff) {
            valid[i] = 0;
            continue;
        }
        x.fins.insert(x.fins.end(), fwd.begin(), fwd.end());
        x.fins.insert(x.fins.end(), rev.begin(), rev.end());
        x.info[i] = make_int4((int)fwd.size(), (int)rev.size(), ns, nt);
        x.slots = std::max(x.slots, ns);
        x.tape = std::max(x.tape, nt);
        x.maxins = std::max(x.maxins, (int)(fwd.size() + rev.size()));
    }
    x.off[nprog] = (int)x.fins.size();
    if (x.fins.empty()) x.fins.resize(1);
}

/* The implicit cost sweep on the stack machine. */
SweepLaunch icost_launch(RcCtx *c, const XPrep &x)
{
    SweepLaunch s;
    s.fn = (const void *)ft_sweep<FOP_ICOST, FT_ITHREADS>;
    s.opk = FOP_ICOST;
    s.smem = 8 * (size_t)((x.maxins + 1) & ~1) + 8 * FT_MAX_CONST +
             8 * (size_t)FT_ITHREADS * (x.slots + x.tape + c->v) + 8 * (size_t)FT_ITHREADS;
    rc_raise_smem(s.fn, s.smem);
    s.grid = c->sm_count * occupancy(s.fn, FT_ITHREADS, s.smem);
    s.threads = FT_ITHREADS;
    return s;
}

template <int OPK>
SweepLaunch sweep_launch(RcCtx *c, int mrec, int tcap, int Wmax)
{
    SweepLaunch s;
    s.fn = (const void *)ft_jac_sweep<OPK, FT_ITHREADS>;
    s.opk = OPK;
    s.smem = ft_ijac_smem(mrec, tcap, Wmax, FT_ITHREADS);
    rc_raise_smem(s.fn, s.smem);
    s.grid = c->sm_count * occupancy(s.fn, FT_ITHREADS, s.smem);
    s.threads = FT_ITHREADS;
    return s;
}

/* The tape bound of the Jacobian launch (the most internal nodes of the
   batch) and the record and tape bounds of the short launch. The sweep
   keeps two f64 tapes per row in shared memory, one slot per internal
   node, sized for the largest program of the launch, so one launch sized
   for the batch runs the short programs at the largest one's occupancy.
   Each split (programs of at most t records to the short launch) is
   estimated as the internal nodes swept over the resident blocks each
   launch allows; the best is kept if it saves at least 5 %, else `small`
   is 0 and one launch serves all. The split depends on the batch, but a
   candidate's arithmetic does not depend on which launch runs it. */
struct IjacSplit {
    int tape = 1, small = 0, tape_small = 1;
};

IjacSplit ijac_split(RcCtx *c, const FitPrep &b, int Wmax)
{
    IjacSplit out;
    std::vector<std::pair<int, int>> ms; /* (records, internal nodes) */
    for (size_t i = 0; i + 1 < b.node_off.size(); ++i)
        if (b.valid[i]) {
            ms.emplace_back(b.node_off[i + 1] - b.node_off[i], b.ninternal[i]);
            out.tape = std::max(out.tape, b.ninternal[i]);
        }
    if (ms.size() < 2) return out;
    const void *fn = (const void *)ft_jac_sweep<FOP_IJACS, FT_ITHREADS>;
    /* occupancy queries up to the largest layout the split can choose */
    const size_t smax = ft_ijac_smem(b.mmax, out.tape, Wmax, FT_ITHREADS);
    if (rc_raise_smem(fn, smax) != 0) return out;
    std::sort(ms.begin(), ms.end());
    auto occ = [&](int mrec, int tcap) {
        return (double)occupancy(fn, FT_ITHREADS, ft_ijac_smem(mrec, tcap, Wmax, FT_ITHREADS));
    };
    double total = 0.0;
    for (const auto &e : ms) total += e.second + 1;
    const double big = occ(b.mmax, out.tape);
    const double one = total / big;
    double best = one, below = 0.0;
    int tmax = 1;
    for (size_t i = 0; i < ms.size(); ++i) {
        below += ms[i].second + 1;
        tmax = std::max(tmax, ms[i].second);
        if (ms[i].first >= b.mmax) break;
        if (i + 1 < ms.size() && ms[i + 1].first == ms[i].first) continue;
        const double cost = below / occ(ms[i].first, tmax) + (total - below) / big;
        if (cost < best) {
            best = cost;
            out.small = ms[i].first;
            out.tape_small = tmax;
        }
    }
    if (!(best <= 0.95 * one)) {
        out.small = 0;
        out.tape_small = 1;
    }
    return out;
}

template <int OPK, int T>
SweepLaunch sweep4_launch(RcCtx *c, const FitPrep &b, int Wmax)
{
    SweepLaunch s;
    s.fn = (const void *)ft_sweep4<OPK, T>;
    s.opk = OPK;
    (void)Wmax;
    const int bk = ft_base_kind(OPK);
    const size_t reg = OPK != bk ? b.asm_reg[ft_kind_cls(OPK)]
                       : (bk == FOP_CASM ? b.asm_region : b.asm_reg[0]);
    s.smem = ft_sweep4_smem(OPK, b.fmaxins, b.fslots, reg, T);
    rc_raise_smem(s.fn, s.smem);
    s.grid = c->sm_count * occupancy(s.fn, T, s.smem);
    s.threads = T;
    return s;
}

/* Enqueue the whole fit on the context stream: init, the bounded steps, the
   flush. */
unsigned long long enqueue_fit(cudaStream_t s_, int sm_count, const FitArgs &a, int steps,
                               const SweepLaunch *sw, int nkinds)
{
    /* persistent grids take their items from work counters, so a grid no
       larger than the items that can exist (a small batch) answers the
       same and launches no idle blocks */
    const int ctrl_grid = std::min(sm_count * 8, std::max(a.nprog, 1));
    const int max_items = (int)std::min<long long>((long long)a.nprog * a.ntiles, 1LL << 30);
    unsigned long long k = 0;
    if (a.nsub > 0) {
        const size_t smem = 8 * (size_t)((a.sub_maxins + 1) & ~1) +
                            16 * (size_t)(a.sub_slots > 0 ? a.sub_slots : 1) * FT_FILL_T;
        ft_cache_fill<<<(unsigned)a.nsub * (unsigned)a.ntiles, FT_FILL_T, smem, s_>>>(a);
        k = 1;
        if (a.cache64) {
            ft_cache_fill64<<<(unsigned)a.nsub * (unsigned)a.ntiles, FT_FILL_T, smem, s_>>>(a);
            k = 2;
        }
    }
    ft_step_reset<<<1, 32, 0, s_>>>(a, 1);
    cudaMemsetAsync(a.work + 1 * FOP_COUNT, 0, sizeof(int) * FOP_COUNT, s_);
    ft_control<<<ctrl_grid, FT_CTRL_T, 0, s_>>>(a, 1, 1);
    for (int s = 0; s < steps; ++s) {
        const int q = s & 1;
        ft_step_reset<<<1, 32, 0, s_>>>(a, q);
        for (int k = 0; k < nkinds; ++k) {
            const SweepLaunch &L = sw[k];
            void *args[] = {(void *)&a, (void *)&q};
            const int grid = std::max(1, std::min(L.grid, max_items));
            cudaLaunchKernel(L.fn, dim3(grid), dim3(L.threads), args, L.smem, s_);
        }
        ft_control<<<ctrl_grid, FT_CTRL_T, 0, s_>>>(a, q, 0);
    }
    ft_flush<<<(a.nprog + 127) / 128, 128, 0, s_>>>(a);
    return k + 3ULL + (unsigned long long)steps * (2ULL + (unsigned long long)nkinds);
}

float fit_run(RcCtx *c, const unsigned int *prog, const unsigned int *off, const int *pcount,
              int nprog, int kmax, const double *c0, const int *gauge, int iters, int metric,
              int flags, double *outc, double *outsse, int *outstatus, int mode)
{
    if (!c || !prog || !off || !pcount || !c0 || !outc || !outsse || !outstatus) return -1.0f;
    if (nprog <= 0 || kmax <= 0 || kmax > FT_MAX_CONST || c->n <= 0) return -1.0f;
    if (metric == FM_LOGISTIC && !c->has_tsign) return -1.0f;
    const bool corr = metric == FM_CORRELATION || metric == FM_CORRELATION_SIGNED;
    if (metric != FM_SQUARED && metric != FM_LOG_SQUASHED && metric != FM_ABSOLUTE &&
        metric != FM_LOGISTIC && metric != FM_IMPLICIT && !corr)
        return -1.0f;
    if (corr && !gauge) return -1.0f;
    if (metric == FM_IMPLICIT && c->v > FT_IMPLICIT_MAXV) return -1.0f;
    for (int i = 0; i < nprog; ++i)
        if (pcount[i] < 0 || pcount[i] > kmax) return -1.0f;
    RcStats *st = &c->stats;
    double t = rc_now_ms();
    if (rc_ensure_f64(c) != 0) return -1.0f;
    FitPrep b;
    size_t free_b = 0, total_b = 0;
    if (cudaMemGetInfo(&free_b, &total_b) != cudaSuccess) {
        cudaGetLastError();
        free_b = 0;
    }
    const size_t cache_cap = std::min<size_t>((size_t)48 << 30, free_b / 3);
    const bool use_cache = metric != FM_IMPLICIT;
    prep_batch(off, prog, pcount, nprog, c->v, b, corr ? 2 : 0,
               use_cache ? sizeof(float) * (size_t)c->npad : 0, cache_cap, c->fit_budget_kb);
    XPrep xp;
    if (metric == FM_IMPLICIT) prep_inputs(off, prog, nprog, b.node_off, b.valid, xp);
    else xp.fins.resize(1);
    const int ntiles = (c->n + FT_TILE_ROWS - 1) / FT_TILE_ROWS;
    const int Wmax = 4 * ((b.pmax + 1 + 3) / 4);
    const size_t words = off[nprog];
    size_t cur = 0;
    const size_t o_rec = rc_take(&cur, sizeof(uint32_t) * words);
    const size_t o_noff = rc_take(&cur, sizeof(int) * (nprog + 1));
    const size_t o_p = rc_take(&cur, sizeof(int) * nprog);
    const size_t o_c0 = rc_take(&cur, sizeof(double) * (size_t)nprog * kmax);
    const size_t o_valid = rc_take(&cur, sizeof(int) * nprog);
    const size_t o_gauge = rc_take(&cur, sizeof(int) * 2 * (size_t)nprog);
    const size_t o_fins = rc_take(&cur, sizeof(FIns) * b.fins.size());
    const size_t o_finsoff = rc_take(&cur, sizeof(int) * (nprog + 1));
    const size_t o_finfo = rc_take(&cur, sizeof(int4) * nprog);
    const size_t o_fcinfo = rc_take(&cur, sizeof(int2) * nprog);
    const size_t o_subf = rc_take(&cur, sizeof(FIns) * b.sub_fins.size());
    const size_t o_suboff = rc_take(&cur, sizeof(int) * b.sub_off.size());
    const size_t o_subcol = rc_take(&cur, sizeof(int) * b.sub_col.size());
    const size_t o_xfins = rc_take(&cur, sizeof(FIns) * xp.fins.size());
    const size_t o_xoff = rc_take(&cur, sizeof(int) * xp.off.size());
    const size_t o_xinfo = rc_take(&cur, sizeof(int4) * xp.info.size());
    const size_t in_end = rc_take(&cur, 0);
    const size_t o_c = rc_take(&cur, sizeof(double) * (size_t)nprog * kmax);
    const size_t o_sse = rc_take(&cur, sizeof(double) * nprog);
    const size_t o_status = rc_take(&cur, sizeof(int) * nprog);
    const size_t io_end = rc_take(&cur, 0);
    const size_t o_state = rc_take(&cur, sizeof(FitState) * nprog);
    const size_t o_part = rc_take(&cur, sizeof(double) * (size_t)nprog * ntiles * FT_PART_STRIDE);
    const size_t o_lists = rc_take(&cur, sizeof(int) * 2 * FOP_COUNT * (size_t)nprog);
    const size_t o_counts = rc_take(&cur, sizeof(int) * 2 * FOP_COUNT);
    const size_t o_work = rc_take(&cur, sizeof(int) * 2 * FOP_COUNT);
    const size_t o_cache = rc_take(&cur, sizeof(float) * (size_t)c->npad * (size_t)b.ncache);
    /* the f64 twin of the cache for the polish, when it fits the same cap */
    const bool use64 = use_cache && b.ncache > 0 && !(flags & 1) &&
                       sizeof(double) * (size_t)c->npad * (size_t)b.ncache <= cache_cap;
    const size_t o_cache64 =
        rc_take(&cur, use64 ? sizeof(double) * (size_t)c->npad * (size_t)b.ncache : 0);
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
    if (gauge) memcpy(host + o_gauge, gauge, sizeof(int) * 2 * (size_t)nprog);
    else memset(host + o_gauge, 0xff, sizeof(int) * 2 * (size_t)nprog);
    memcpy(host + o_fins, b.fins.data(), sizeof(FIns) * b.fins.size());
    memcpy(host + o_finsoff, b.fins_off.data(), sizeof(int) * (nprog + 1));
    memcpy(host + o_finfo, b.finfo.data(), sizeof(int4) * nprog);
    memcpy(host + o_fcinfo, b.fcinfo.data(), sizeof(int2) * nprog);
    memcpy(host + o_subf, b.sub_fins.data(), sizeof(FIns) * b.sub_fins.size());
    memcpy(host + o_suboff, b.sub_off.data(), sizeof(int) * b.sub_off.size());
    memcpy(host + o_subcol, b.sub_col.data(), sizeof(int) * b.sub_col.size());
    memcpy(host + o_xfins, xp.fins.data(), sizeof(FIns) * xp.fins.size());
    if (!xp.off.empty()) memcpy(host + o_xoff, xp.off.data(), sizeof(int) * xp.off.size());
    if (!xp.info.empty()) memcpy(host + o_xinfo, xp.info.data(), sizeof(int4) * xp.info.size());
    memcpy(host + o_c, c0, sizeof(double) * (size_t)nprog * kmax);
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
    a.gauge = reinterpret_cast<const int *>(dev + o_gauge);
    a.fins = reinterpret_cast<const FIns *>(dev + o_fins);
    a.fins_off = reinterpret_cast<const int *>(dev + o_finsoff);
    a.finfo = reinterpret_cast<const int4 *>(dev + o_finfo);
    a.fcinfo = reinterpret_cast<const int2 *>(dev + o_fcinfo);
    a.cache = reinterpret_cast<float *>(dev + o_cache);
    a.cache64 = use64 ? reinterpret_cast<double *>(dev + o_cache64) : nullptr;
    a.sub_fins = reinterpret_cast<const FIns *>(dev + o_subf);
    a.sub_off = reinterpret_cast<const int *>(dev + o_suboff);
    a.sub_col = reinterpret_cast<const int *>(dev + o_subcol);
    a.nsub = (int)b.sub_off.size() - 1;
    a.sub_slots = b.sub_slots;
    a.sub_maxins = b.sub_maxins;
    a.xfins = reinterpret_cast<const FIns *>(dev + o_xfins);
    a.xfins_off = reinterpret_cast<const int *>(dev + o_xoff);
    a.xinfo = reinterpret_cast<const int4 *>(dev + o_xinfo);
    a.xmaxins = xp.maxins;
    a.xslots = xp.slots;
    a.xtape = xp.tape;
    a.asm_region = b.asm_region;
    for (int k = 0; k < FT_NCLS; ++k) a.asm_reg[k] = b.asm_reg[k];
    a.fslots = b.fslots;
    a.ftape = b.ftape;
    a.fmaxins = b.fmaxins;
    a.iters = iters;
    a.metric = metric;
    a.flags = flags;
    a.ntiles = ntiles;
    a.mmax = b.mmax;
    a.Wmax = Wmax;
    a.nprog = nprog;
    a.state = reinterpret_cast<FitState *>(dev + o_state);
    a.part = reinterpret_cast<double *>(dev + o_part);
    a.lists = reinterpret_cast<int *>(dev + o_lists);
    a.counts = reinterpret_cast<int *>(dev + o_counts);
    a.work = reinterpret_cast<int *>(dev + o_work);
    a.outc = reinterpret_cast<double *>(dev + o_c);
    a.outsse = reinterpret_cast<double *>(dev + o_sse);
    a.outstatus = reinterpret_cast<int *>(dev + o_status);

    SweepLaunch sw[16];
    int nk = 0;
    if (metric == FM_IMPLICIT) {
        const IjacSplit js = ijac_split(c, b, Wmax);
        a.ijac_small = js.small;
        a.ijac_tape = js.tape;
        a.ijac_tape_small = js.tape_small;
        if (a.ijac_small > 0) {
            sw[nk] = sweep_launch<FOP_IJACS>(c, a.ijac_small, a.ijac_tape_small, Wmax); ++nk;
        }
        sw[nk] = sweep_launch<FOP_IJAC>(c, b.mmax, a.ijac_tape, Wmax); ++nk;
        sw[nk] = icost_launch(c, xp); ++nk;
    } else if (corr) {
        sw[nk] = sweep4_launch<FOP_CASM, FT_ASM_T>(c, b, Wmax); ++nk;
        sw[nk] = sweep4_launch<FOP_CSCORE, 128>(c, b, Wmax); ++nk;
    } else {
        /* one assembly launch per active-thread class present in the batch,
           each in blocks of that many threads */
        if (b.nclass[0]) { sw[nk] = sweep4_launch<FOP_ASM32, FT_ASM_T>(c, b, Wmax); ++nk; }
        if (b.nclass[1]) { sw[nk] = sweep4_launch<FOP_ASM32_64A, 64>(c, b, Wmax); ++nk; }
        if (b.nclass[2]) { sw[nk] = sweep4_launch<FOP_ASM32_64B, 64>(c, b, Wmax); ++nk; }
        if (b.nclass[3]) { sw[nk] = sweep4_launch<FOP_ASM32_64, 64>(c, b, Wmax); ++nk; }
        if (b.nclass[4]) { sw[nk] = sweep4_launch<FOP_ASM32_32, 32>(c, b, Wmax); ++nk; }
        if (b.nclass[5]) { sw[nk] = sweep4_launch<FOP_ASM32_128L, 128>(c, b, Wmax); ++nk; }
        sw[nk] = sweep4_launch<FOP_LOSS32, 128>(c, b, Wmax); ++nk;
        /* the f64 sweeps serve the polish and the f64 rescue */
        if ((flags & (FT_FLAG_NO_POLISH | FT_FLAG_NO_RESCUE)) !=
            (FT_FLAG_NO_POLISH | FT_FLAG_NO_RESCUE)) {
            if (b.nclass[0]) { sw[nk] = sweep4_launch<FOP_ASM64, FT_ASM_T>(c, b, Wmax); ++nk; }
            if (b.nclass[1]) { sw[nk] = sweep4_launch<FOP_ASM64_64A, 64>(c, b, Wmax); ++nk; }
            if (b.nclass[2]) { sw[nk] = sweep4_launch<FOP_ASM64_64B, 64>(c, b, Wmax); ++nk; }
            if (b.nclass[3]) { sw[nk] = sweep4_launch<FOP_ASM64_64, 64>(c, b, Wmax); ++nk; }
            if (b.nclass[4]) { sw[nk] = sweep4_launch<FOP_ASM64_32, 32>(c, b, Wmax); ++nk; }
            if (b.nclass[5]) { sw[nk] = sweep4_launch<FOP_ASM64_128L, 128>(c, b, Wmax); ++nk; }
            sw[nk] = sweep4_launch<FOP_LOSS64, 128>(c, b, Wmax); ++nk;
        }
    }
    const int steps = max_steps(iters, metric);

    t = rc_now_ms();
    cudaEventRecord(c->t0, c->s);
    cudaMemcpyAsync(dev, host, io_end, cudaMemcpyHostToDevice, c->s);
    bool ok = true;
    if (mode == 1) {
        /* plain arm: the same step kernels, one candidate per launch sequence */
        for (int i = 0; i < nprog && ok; ++i) {
            FitArgs one = a;
            one.rec = a.rec;
            one.nprog = 1;
            one.node_off = a.node_off + i;
            one.pcount = a.pcount + i;
            one.c0 = a.c0 + (size_t)i * kmax;
            one.valid = a.valid + i;
            one.gauge = a.gauge + 2 * (size_t)i;
            one.fins_off = a.fins_off + i;
            one.xfins_off = a.xfins_off + i;
            one.xinfo = a.xinfo + i;
            one.finfo = a.finfo + i;
            one.fcinfo = a.fcinfo + i;
            one.sub_off = a.sub_off + b.sub_cand_off[i];
            one.sub_col = a.sub_col + b.sub_cand_off[i];
            one.nsub = b.sub_cand_off[i + 1] - b.sub_cand_off[i];
            one.state = a.state + i;
            one.part = a.part + (size_t)i * ntiles * FT_PART_STRIDE;
            one.outc = a.outc + (size_t)i * kmax;
            one.outsse = a.outsse + i;
            one.outstatus = a.outstatus + i;
            /* only the assembly launches of this candidate's class */
            SweepLaunch swc[16];
            int nkc = 0;
            const int cls = b.finfo[i].z >> 16;
            for (int k = 0; k < nk; ++k) {
                const int o = sw[k].opk;
                const int bk = ft_base_kind(o);
                if ((bk == FOP_ASM32 || bk == FOP_ASM64) && ft_kind_cls(o) != cls) continue;
                swc[nkc++] = sw[k];
            }
            c->launches += enqueue_fit(c->s, c->sm_count, one, steps, swc, nkc);
            ok = cudaGetLastError() == cudaSuccess;
        }
    } else {
        char key[1024];
        snprintf(key, sizeof(key), "%p|%d|%d|%d|%d|%d|%d|%d|%d|%d|%zu|%d|%d|%d|%zu", (void *)dev,
                 nprog, kmax, ntiles, b.mmax, Wmax, iters, metric, flags, steps, io_end, b.fslots,
                 b.ftape, b.fmaxins, b.asm_region);
        const size_t kl = strlen(key);
        snprintf(key + kl, sizeof(key) - kl,
                 "|%d|%d|%d|%d|%d|%d|%d|%d|%d|%d|%d|%zu|%zu|%zu|%d|%d|%d", b.ncache, a.nsub,
                 b.sub_slots, b.sub_maxins, xp.maxins, xp.slots, xp.tape, use64 ? 1 : 0,
                 a.ijac_small, a.ijac_tape, a.ijac_tape_small, b.asm_reg[0], b.asm_reg[1],
                 b.asm_reg[2], b.nclass[0], b.nclass[1], b.nclass[2]);
        const size_t kl2 = strlen(key);
        snprintf(key + kl2, sizeof(key) - kl2, "|%zu|%zu|%zu|%d|%d|%d", b.asm_reg[3],
                 b.asm_reg[4], b.asm_reg[5], b.nclass[3], b.nclass[4], b.nclass[5]);
        const bool replay = c->fit_graph && c->fit_graph_key == key;
        if (!replay && c->fit_seen_key != key) {
            /* a batch shape seen for the first time runs its steps directly:
               a generation loop rarely repeats one, and capturing and
               instantiating the graph costs more than launching it once.
               The second call of a shape captures it, later ones replay. */
            c->fit_seen_key = key;
            c->launches += enqueue_fit(c->s, c->sm_count, a, steps, sw, nk);
            ok = cudaGetLastError() == cudaSuccess;
        } else {
            if (!replay) {
                if (c->fit_graph) {
                    cudaGraphExecDestroy(c->fit_graph);
                    c->fit_graph = nullptr;
                }
                cudaGraph_t g = nullptr;
                cudaStream_t cap = nullptr;
                cudaStreamCreateWithFlags(&cap, cudaStreamNonBlocking);
                ok = cudaStreamBeginCapture(cap, cudaStreamCaptureModeThreadLocal) == cudaSuccess;
                if (ok) {
                    c->fit_graph_kernels = enqueue_fit(cap, c->sm_count, a, steps, sw, nk);
                    ok = cudaStreamEndCapture(cap, &g) == cudaSuccess && g;
                }
                if (ok) ok = cudaGraphInstantiate(&c->fit_graph, g, 0) == cudaSuccess;
                if (g) cudaGraphDestroy(g);
                cudaStreamDestroy(cap);
                if (!ok) {
                    cudaGetLastError();
                    c->fit_graph = nullptr;
                } else {
                    c->fit_graph_key = key;
                }
            }
            if (ok) ok = cudaGraphLaunch(c->fit_graph, c->s) == cudaSuccess;
            if (ok) c->launches += c->fit_graph_kernels;
        }
    }
    cudaEventRecord(c->t1, c->s);
    st->launch_ms += rc_now_ms() - t;
    if (!ok || cudaGetLastError() != cudaSuccess) {
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
    c->fit_state = dev + o_state;
    c->fit_state_n = nprog;
    c->fit_state_stride = sizeof(FitState);
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

/* The fit autotuner. Per length bucket of the caller's batch (fit programs
   of <= 16, <= 32, <= 64 and more records), the assembly region budget that
   sets each candidate's active threads (and so how many of its rows are in
   flight beside its spill slots, tape and Jacobian rows) is chosen by timing
   the fused fit of a tuning batch of the bucket's candidates at each budget
   in {24, 32, 40, 56, 80} KB: one warm-up fit, then the fastest of two. The
   tuning batch must fill the GPU the way the real batch does, or it would
   favour the latency of a few candidates over throughput: it holds about
   16,384 (candidate, tile) work items (`sample` candidates when given > 0),
   the bucket's first candidates repeated when the bucket has fewer. A budget
   replaces the built-in default only when it is at least 3 % faster, and
   the new table as a whole only when the caller's whole batch is at least
   3 % faster with it than with the defaults. The
   choice is kept in the context for its (N, feature count) and, with a path,
   read from / written to that file as lines "fit n v bucket budget_kb" (a
   bucket found there is not re-timed). The budget changes a candidate's
   active threads and with it the order of its sums: results depend on the
   table, never on the batch. Returns the number of buckets with a budget,
   or -1. */
int rc_fit_autotune(void *ctx, const unsigned int *prog, const unsigned int *off,
                    const int *pcount, int nprog, int kmax, const double *c0, const int *gauge,
                    int iters, int metric, int sample, const char *path)
{
    RcCtx *c = (RcCtx *)ctx;
    if (!c || !prog || !off || !pcount || !c0 || nprog <= 0 || kmax <= 0 || kmax > FT_MAX_CONST)
        return -1;
    if (sample <= 0) {
        const int ntiles = (c->n + FT_TILE_ROWS - 1) / FT_TILE_ROWS;
        sample = std::max(16, std::min(512, (16384 + ntiles - 1) / std::max(ntiles, 1)));
    }
    int have[4] = {0, 0, 0, 0};
    std::vector<std::string> keep;
    if (path) {
        std::ifstream in(path);
        std::string line;
        while (std::getline(in, line)) {
            long long n, v;
            int bkt, kb;
            char tag[8] = {0};
            if (sscanf(line.c_str(), "%7s %lld %lld %d %d", tag, &n, &v, &bkt, &kb) == 5 &&
                strcmp(tag, "fit") == 0 && n == c->n && v == c->v && bkt >= 0 && bkt < 4 &&
                kb >= 8 && kb <= 200) {
                c->fit_budget_kb[bkt] = kb;
                have[bkt] = 1;
            } else if (!line.empty()) {
                keep.push_back(line);
            }
        }
    }
    /* the candidates of each bucket, up to `sample`, repeated up to it */
    std::vector<int> pick[4];
    for (int i = 0; i < nprog; ++i) {
        const int m = (int)((off[i + 1] - off[i]) / 4);
        const int b = ft_length_bucket(m);
        if ((int)pick[b].size() < sample) pick[b].push_back(i);
    }
    for (int b = 0; b < 4; ++b) {
        const size_t have_b = pick[b].size();
        for (size_t j = have_b; have_b > 0 && j < (size_t)sample; ++j)
            pick[b].push_back(pick[b][j % have_b]);
    }
    static const int budgets[] = {40, 24, 32, 56, 80}; /* the default first */
    bool tuned[4] = {false, false, false, false};
    for (int b = 0; b < 4; ++b) {
        if (have[b] || pick[b].empty()) continue;
        const int k = (int)pick[b].size();
        std::vector<unsigned int> sp, so(1, 0);
        std::vector<int> spc(k), sg(2 * (size_t)k, -1);
        std::vector<double> sc0((size_t)k * kmax);
        for (int j = 0; j < k; ++j) {
            const int i = pick[b][j];
            sp.insert(sp.end(), prog + off[i], prog + off[i + 1]);
            so.push_back((unsigned int)sp.size());
            spc[j] = pcount[i];
            if (gauge) {
                sg[2 * j] = gauge[2 * i];
                sg[2 * j + 1] = gauge[2 * i + 1];
            }
            memcpy(&sc0[(size_t)j * kmax], c0 + (size_t)i * kmax, sizeof(double) * kmax);
        }
        std::vector<double> oc((size_t)k * kmax), osse(k);
        std::vector<int> ost(k);
        float best = -1.0f, base = -1.0f;
        int best_kb = 0;
        for (int kb : budgets) {
            c->fit_budget_kb[b] = kb;
            float t = fit_run(c, sp.data(), so.data(), spc.data(), k, kmax, sc0.data(),
                              gauge ? sg.data() : nullptr, iters, metric, 0, oc.data(),
                              osse.data(), ost.data(), 0);
            if (t < 0.0f) continue;
            for (int r = 0; r < 2; ++r) {
                const float u = fit_run(c, sp.data(), so.data(), spc.data(), k, kmax, sc0.data(),
                                        gauge ? sg.data() : nullptr, iters, metric, 0, oc.data(),
                                        osse.data(), ost.data(), 0);
                if (u >= 0.0f && u < t) t = u;
            }
            if (kb == FT_ASM_BUDGET / 1024) base = t;
            if (best < 0.0f || t < best) {
                best = t;
                best_kb = kb;
            }
        }
        /* keep the default unless another budget is clearly faster */
        if (base >= 0.0f && best > 0.97f * base) best_kb = FT_ASM_BUDGET / 1024;
        c->fit_budget_kb[b] = best_kb;
        tuned[b] = best_kb != FT_ASM_BUDGET / 1024;
    }
    /* A bucket's budget also changes the launches the other buckets share,
       which the per-bucket timing cannot see: the caller's whole batch is
       timed with the new table and with the default one, and the new
       choices are kept only when the whole batch is at least 3 % faster. */
    if (tuned[0] || tuned[1] || tuned[2] || tuned[3]) {
        std::vector<double> oc((size_t)nprog * kmax), osse(nprog);
        std::vector<int> ost(nprog);
        auto whole = [&]() {
            float t = -1.0f;
            for (int r = 0; r < 3; ++r) {
                const float u = fit_run(c, prog, off, pcount, nprog, kmax, c0, gauge, iters,
                                        metric, 0, oc.data(), osse.data(), ost.data(), 0);
                if (r > 0 && u >= 0.0f && (t < 0.0f || u < t)) t = u;
            }
            return t;
        };
        int table[4];
        for (int b = 0; b < 4; ++b) table[b] = c->fit_budget_kb[b];
        const float t_new = whole();
        for (int b = 0; b < 4; ++b)
            if (tuned[b]) c->fit_budget_kb[b] = FT_ASM_BUDGET / 1024;
        const float t_def = whole();
        if (t_new >= 0.0f && t_def >= 0.0f && t_new <= 0.97f * t_def)
            for (int b = 0; b < 4; ++b) c->fit_budget_kb[b] = table[b];
    }
    for (int b = 0; b < 4; ++b) have[b] = have[b] || c->fit_budget_kb[b] > 0;
    if (path) {
        std::ofstream out(path, std::ios::trunc);
        for (const auto &l : keep) out << l << "\n";
        for (int b = 0; b < 4; ++b)
            if (c->fit_budget_kb[b] > 0)
                out << "fit " << c->n << " " << c->v << " " << b << " " << c->fit_budget_kb[b]
                    << "\n";
    }
    int count = 0;
    for (int b = 0; b < 4; ++b) count += c->fit_budget_kb[b] > 0;
    return count;
}

/* The context's fit assembly budgets (KB) per length bucket, 0 = default. */
int rc_fit_budgets(void *ctx, int *out_kb)
{
    RcCtx *c = (RcCtx *)ctx;
    if (!c || !out_kb) return -1;
    for (int b = 0; b < 4; ++b) out_kb[b] = c->fit_budget_kb[b];
    return 0;
}

/* Sweeps each candidate of the context's last fit ran, out[4 * cand + k]:
   k = 0 f32 assemblies, 1 f32 objective sweeps, 2 f64 assemblies (implicit
   Jacobians), 3 f64 objective sweeps (implicit costs). Returns 0, or -1 when
   no fit of nprog candidates is the last call's. */
int rc_last_fit_sweeps(void *ctx, int nprog, int *out)
{
    RcCtx *c = (RcCtx *)ctx;
    if (!c || !out || !c->fit_state || nprog != c->fit_state_n) return -1;
    const size_t off = offsetof(FitState, nsw);
    if (cudaMemcpy2DAsync(out, 4 * sizeof(int), c->fit_state + off, c->fit_state_stride,
                          4 * sizeof(int), (size_t)nprog, cudaMemcpyDeviceToHost,
                          c->s) != cudaSuccess) {
        cudaGetLastError();
        return -1;
    }
    return rc_finish(c);
}

int rc_fit_kernel_info(int kmax, int *threads, int *smem_bytes, int *max_constants)
{
    if (!threads || !smem_bytes || !max_constants) return -1;
    if (kmax > FT_MAX_CONST || kmax < 0) return -1;
    /* the f32 assembly sweep: its fixed region budget plus the instruction
       lists of the largest accepted tree */
    *threads = FT_ASM_T;
    *smem_bytes = (int)ft_sweep4_smem(FOP_ASM32, 2 * FT_MAX_NODES_ABI + 1, 1, FT_ASM_BUDGET, FT_ASM_T);
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
    FitPrep b;
    prep_batch(off, prog, pcount, nprog, rc->v, b);
    const int mmax = b.mmax;
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
    const size_t o_fins = rc_take(&cur, sizeof(FIns) * b.fins.size());
    const size_t o_finsoff = rc_take(&cur, sizeof(int) * (nprog + 1));
    const size_t o_finfo = rc_take(&cur, sizeof(int4) * nprog);
    const size_t dev_end = rc_take(&cur, 0);
    if (rc_reserve(rc, dev_end, io_end) != 0) return -1;
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
    if (want == 1) {
        /* the four-row sweeps of the f32 assembly */
        std::vector<unsigned char> stage(dev_end - io_end);
        memcpy(stage.data() + (o_fins - io_end), b.fins.data(), sizeof(FIns) * b.fins.size());
        memcpy(stage.data() + (o_finsoff - io_end), b.fins_off.data(), sizeof(int) * (nprog + 1));
        memcpy(stage.data() + (o_finfo - io_end), b.finfo.data(), sizeof(int4) * nprog);
        a.fins = reinterpret_cast<const FIns *>(dev + o_fins);
        a.fins_off = reinterpret_cast<const int *>(dev + o_finsoff);
        a.finfo = reinterpret_cast<const int4 *>(dev + o_finfo);
        a.fmaxins = b.fmaxins;
        cudaMemcpyAsync(dev + io_end, stage.data(), stage.size(), cudaMemcpyHostToDevice, rc->s);
        constexpr int NR = FT_ASM32_NR;
        const int ntiles = ((row0 + nrows) - (row0 & ~(NR - 1)) + 32 * NR - 1) / (32 * NR);
        const size_t smem = 8 * (size_t)((b.fmaxins + 1) & ~1) + 4 * FT_MAX_CONST +
                            4 * NR * 32 * (size_t)(b.fslots + b.ftape) +
                            4 * (size_t)(b.pmax > 0 ? b.pmax : 1) * (NR * 32 + 4);
        if (rc_raise_smem((const void *)ft_grad4_kernel, smem) != 0) return -1;
        rc->launches += 1;
        ft_grad4_kernel<<<nprog * ntiles, 32, smem, rc->s>>>(
            a, row0, nrows, ntiles, reinterpret_cast<float *>(dev + o_val),
            reinterpret_cast<float *>(dev + o_out));
    } else {
    const int T = 128;
    const int ntiles = (nrows + T - 1) / T;
    const size_t smem = sizeof(uint4) * mmax + sizeof(float) * FT_MAX_CONST +
                        sizeof(float) * (size_t)mmax * T + sizeof(double) * FT_MAX_CONST * T +
                        sizeof(float) * (size_t)rc->v * T + 64;
    if (rc_raise_smem((const void *)ft_grad_kernel<128>, smem) != 0) return -1;
    rc->launches += 1;
    ft_grad_kernel<128><<<nprog * ntiles, T, smem, rc->s>>>(
        a, want, row0, nrows, ntiles, reinterpret_cast<float *>(dev + o_val),
        reinterpret_cast<float *>(dev + o_out));
    }
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
    if (rc->v > FT_IMPLICIT_MAXV) return -1.0f;
    RcStats *st = &rc->stats;
    FitPrep b;
    prep_batch(off, prog, pcount, nprog, rc->v, b);
    /* the input-mode translation: partials and pruning along input paths */
    XPrep xp;
    prep_inputs(off, prog, nprog, b.node_off, b.valid, xp);
    std::vector<FIns> &xfins = xp.fins;
    std::vector<int> &xoff = xp.off;
    std::vector<int4> &xinfo = xp.info;
    const int slots = xp.slots, ntape = xp.tape, maxins = xp.maxins;
    const int T = 128;
    constexpr int NR = 2;
    const int rows_per_tile = 16384;
    const int ntiles = (rc->n + rows_per_tile - 1) / rows_per_tile;
    size_t cur = 0;
    const size_t o_fins = rc_take(&cur, sizeof(FIns) * xfins.size());
    const size_t o_xoff = rc_take(&cur, sizeof(int) * (nprog + 1));
    const size_t o_info = rc_take(&cur, sizeof(int4) * nprog);
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
    memcpy(host + o_fins, xfins.data(), sizeof(FIns) * xfins.size());
    memcpy(host + o_xoff, xoff.data(), sizeof(int) * (nprog + 1));
    memcpy(host + o_info, xinfo.data(), sizeof(int4) * nprog);
    memcpy(host + o_c, c, sizeof(double) * (size_t)nprog * kmax);
    memcpy(host + o_valid, b.valid.data(), sizeof(int) * nprog);
    cudaMemcpyAsync(dev, host, in_end, cudaMemcpyHostToDevice, rc->s);
    cudaMemsetAsync(dev + o_bad, 0, sizeof(int) * nprog, rc->s);
    st->h2d_ms += rc_now_ms() - t;
    using V4 = FiV<float, NR>::V4;
    const size_t smem = 8 * (size_t)((maxins + 1) & ~1) + sizeof(float) * FT_MAX_CONST +
                        sizeof(V4) * (size_t)(slots + ntape + rc->v) * T + sizeof(double) * T;
    if (rc_raise_smem((const void *)ft_implicit_score_x<128, NR>, smem) != 0) return -1.0f;
    cudaEventRecord(rc->t0, rc->s);
    rc->launches += 2;
    ft_implicit_score_x<128, NR><<<nprog * ntiles, T, smem, rc->s>>>(
        reinterpret_cast<const FIns *>(dev + o_fins), reinterpret_cast<const int *>(dev + o_xoff),
        reinterpret_cast<const int4 *>(dev + o_info), reinterpret_cast<const int *>(dev + o_valid),
        reinterpret_cast<const double *>(dev + o_c), kmax, rc->d_cols, rc->npad, rc->n, rc->v,
        rc->d_w64, ntiles, rows_per_tile, maxins, slots, ntape,
        reinterpret_cast<double *>(dev + o_part), reinterpret_cast<int *>(dev + o_bad));
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
